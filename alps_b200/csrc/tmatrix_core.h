// tmatrix_core.h -- Lanczos T-matrix analysis usable on the host and on the device.
//
// Tmatrix::compute(do_err = true) of src/ietl/tmatrix.h:121-228 (distinct
// values within thold, multiplicities, ghost test against T without its first
// row and column, error estimates |beta_m z_{m,i}|) with LAPACK dstev
// (src/ietl/ietl2lapack.h:84-99) replaced by an implicit QL eigensolver for
// symmetric tridiagonal matrices (Bowdler, Martin, Reinsch & Wilkinson,
// Numer. Math. 11 (1968) 293-306) that forms only the last row of the
// eigenvector matrix, which is all the error estimates use.  Plain pointers and
// caller-provided scratch, so one thread of a CUDA kernel can run it.
#pragma once

#include <cfloat>
#include <cmath>

#ifdef __CUDACC__
#define AED_HD __host__ __device__
#else
#define AED_HD
#endif

namespace aed {
namespace tcore {

AED_HD inline double dmax(double a, double b) { return a > b ? a : b; }

// d[0..n): diagonal -> eigenvalues ascending.  e[0..n): sub-diagonal in
// e[0..n-2] (destroyed).  zl (optional): last row of the eigenvector matrix.
// zf (optional, n*n column-major): all eigenvectors.  Returns 0, or l+1 when
// eigenvalue l did not converge.
AED_HD inline int ql(int n, double* d, double* e, double* zl, double* zf) {
  if (n <= 0) return 0;
  if (zl) {
    for (int k = 0; k < n; ++k) zl[k] = 0.0;
    zl[n - 1] = 1.0;
  }
  if (zf) {
    for (long k = 0; k < (long)n * n; ++k) zf[k] = 0.0;
    for (int k = 0; k < n; ++k) zf[(long)k * n + k] = 1.0;
  }
  e[n - 1] = 0.0;
  for (int l = 0; l < n; ++l) {
    for (int sweep = 0;; ++sweep) {
      int m = l;
      while (m < n - 1 && fabs(e[m]) > DBL_EPSILON * (fabs(d[m]) + fabs(d[m + 1]))) ++m;
      if (m == l) break;
      if (sweep >= 90) return l + 1;
      // plane rotations with sqrt(f^2 + g^2) rather than hypot: twice as fast,
      // and T's entries (bounded by |H|) cannot overflow the squares
      const double theta = (d[l + 1] - d[l]) / (2.0 * e[l]);
      const double rho = sqrt(theta * theta + 1.0);
      double g = d[m] - d[l] + e[l] / (theta + copysign(rho, theta));
      double s = 1.0, c = 1.0, p = 0.0;
      bool split = false;
      for (int i = m - 1; i >= l; --i) {
        const double f = s * e[i], b = c * e[i];
#ifdef __CUDA_ARCH__
        // one reciprocal square root instead of a square root and two
        // divisions, whose long dependent chains set the pace of the batched
        // check (a GPU thread per matrix); rsqrt is within 1 ulp, so the
        // rotation stays orthogonal to a few ulps and QL backward stable
        const double h2 = f * f + g * g;
        if (h2 == 0.0) {
          e[i + 1] = 0.0;
          d[i + 1] -= p;
          e[m] = 0.0;
          split = true;
          break;
        }
        const double ri = rsqrt(h2);
        e[i + 1] = h2 * ri;
        s = f * ri;
        c = g * ri;
#else
        const double r = sqrt(f * f + g * g);
        e[i + 1] = r;
        if (r == 0.0) {
          d[i + 1] -= p;
          e[m] = 0.0;
          split = true;
          break;
        }
        s = f / r;
        c = g / r;
#endif
        const double gg = d[i + 1] - p;
        const double t = (d[i] - gg) * s + 2.0 * c * b;
        p = s * t;
        d[i + 1] = gg + p;
        g = c * t - b;
        if (zl) {
          const double z1 = zl[i + 1];
          zl[i + 1] = s * zl[i] + c * z1;
          zl[i] = c * zl[i] - s * z1;
        }
        if (zf) {
          double* ci = zf + (long)i * n;
          double* cj = zf + (long)(i + 1) * n;
          for (int k = 0; k < n; ++k) {
            const double z1 = cj[k];
            cj[k] = s * ci[k] + c * z1;
            ci[k] = c * ci[k] - s * z1;
          }
        }
      }
      if (split) continue;
      d[l] -= p;
      e[l] = g;
      e[m] = 0.0;
    }
  }
  // ascending order (insertion sort, stable), carrying zl / zf columns
  for (int i = 1; i < n; ++i) {
    const double v = d[i];
    const double z = zl ? zl[i] : 0.0;
    int j = i - 1;
    while (j >= 0 && d[j] > v) --j;
    ++j;
    if (j == i) continue;
    for (int k = i; k > j; --k) {
      d[k] = d[k - 1];
      if (zl) zl[k] = zl[k - 1];
    }
    d[j] = v;
    if (zl) zl[j] = z;
    if (zf) {  // rotate columns j..i right by one
      for (int r = 0; r < n; ++r) {
        const double t = zf[(long)i * n + r];
        for (int k = i; k > j; --k) zf[(long)k * n + r] = zf[(long)(k - 1) * n + r];
        zf[(long)j * n + r] = t;
      }
    }
  }
  return 0;
}

struct TResult {
  int count;       // distinct non-ghost values written (at most cap)
  double thold, multol;
};

// Tmatrix::compute(true) on alpha[0..n), beta[0..n) (beta[n-1] = beta_{m+1}).
// Writes up to `cap` distinct non-ghost eigenvalues (ascending) with their
// error estimates, multiplicities and first index in the sorted spectrum.
// scratch: 5*n + 2 doubles.  thold_rel > 0 raises the merge threshold to
// thold_rel * max|eigenvalue| (recurrences run with FP32 vectors, whose copies
// of a converged eigenvalue differ by FP32 rounding, far above the FP64
// threshold).  Returns 0 or the eigensolver's failure code.
// analyze in three parts, so that two threads can run the two eigenvalue
// sweeps side by side: analyze_t (eigenvalues and last eigenvector row of T),
// analyze_t2 (eigenvalues of T without its first row and column), both into
// disjoint parts of scratch, then analyze_walk.
AED_HD inline int analyze_t(int n, const double* alpha, const double* beta, double* scratch) {
  if (n < 1) return 0;
  double* ev = scratch;    // n
  double* e = ev + n;      // n + 1
  double* zl = e + n + 1;  // n
  for (int i = 0; i < n; ++i) ev[i] = alpha[i];
  for (int i = 0; i <= n; ++i) e[i] = 0.0;
  for (int i = 0; i + 1 < n; ++i) e[i] = beta[i];
  return ql(n, ev, e, zl, nullptr);
}

AED_HD inline int analyze_t2(int n, const double* alpha, const double* beta, double* scratch) {
  if (n < 2) return 0;
  double* evg = scratch + 3 * n + 1;  // n
  double* eg = evg + n;               // n + 1
  for (int i = 1; i < n; ++i) evg[i - 1] = alpha[i];
  for (int i = 0; i <= n; ++i) eg[i] = 0.0;
  for (int i = 1; i + 1 < n; ++i) eg[i - 1] = beta[i];
  return ql(n - 1, evg, eg, nullptr, nullptr);
}

AED_HD inline int analyze_walk(int n, const double* beta, double alpha_max, double beta_max, double* scratch,
                               int cap, double* evals, double* errs, int* mults, int* first, TResult* res,
                               double thold_rel = 0.0);

AED_HD inline int analyze(int n, const double* alpha, const double* beta, double alpha_max, double beta_max,
                          double* scratch, int cap, double* evals, double* errs, int* mults, int* first,
                          TResult* res, double thold_rel = 0.0) {
  res->count = 0;
  res->thold = res->multol = 0.0;
  if (n < 1) return 0;
  int info = analyze_t(n, alpha, beta, scratch);
  if (info) return info;
  info = analyze_t2(n, alpha, beta, scratch);
  if (info) return info;
  return analyze_walk(n, beta, alpha_max, beta_max, scratch, cap, evals, errs, mults, first, res, thold_rel);
}

AED_HD inline int analyze_walk(int n, const double* beta, double alpha_max, double beta_max, double* scratch,
                               int cap, double* evals, double* errs, int* mults, int* first, TResult* res,
                               double thold_rel) {
  res->count = 0;
  res->thold = res->multol = 0.0;
  if (n < 1) return 0;
  double* ev = scratch;             // n
  double* zl = ev + 2 * n + 1;      // n
  double* evg = zl + n;             // n
  const double eps = DBL_EPSILON;
  const double error_tol = pow(eps, 2.0 / 3.0);  // tmatrix.h:32
  const double multol = dmax(alpha_max, beta_max) * 2 * eps * (10000 + n);
  double thold = dmax(error_tol * dmax(ev[0], ev[n - 1]), 5 * multol);
  if (thold_rel > 0.0) thold = dmax(thold, thold_rel * dmax(fabs(ev[0]), fabs(ev[n - 1])));
  res->thold = thold;
  res->multol = multol;
  const double bl = beta[n - 1];
  // walk the distinct values in ascending order; the ghost test of a simple
  // value only looks at reduced-T eigenvalues from the running index t2 on,
  // so the walk can stop once `cap` non-ghost values are out
  int t2 = 0, out = 0;
  int i0 = 0;  // first index of the current cluster
  while (i0 < n && out < cap) {
    const double temp = ev[i0];
    int i1 = i0 + 1;
    while (i1 < n && !((ev[i1] - temp) > thold)) ++i1;
    int mult = i1 - i0;
    // error of the cluster: 0 if multiple, else |beta_m z_{m, last index}|
    double err = mult > 1 ? 0.0 : fabs(bl * zl[i1 - 1]);
    if (mult == 1) {
      for (int j = t2; j < n - 2; ++j, ++t2) {
        if ((evg[j] - temp) >= multol) break;
        if (fabs(temp - evg[j]) < multol) {
          mult = 0;
          err = 0.0;
          ++t2;
          break;
        }
      }
    }
    if (mult != 0) {
      evals[out] = temp;
      errs[out] = err;
      if (mults) mults[out] = mult;
      if (first) first[out] = i0;
      ++out;
    }
    i0 = i1;
  }
  res->count = out;
  return 0;
}

// Start of the FP64 refinement of the mixed path: the eigenvectors of T with
// sorted indices [0, K) are combined, where K ends the nev-th distinct value's
// cluster.  A cluster holds ghost copies and any pair closer than the FP32
// phase resolves, so the partner of a near-degenerate pair is kept (a guard
// cluster beyond the nev-th made the refinement 1.5-3x longer on the J1-J2
// chain, L=28, without changing a result).  first / mults: analyze's output
// (count values).
AED_HD inline int ritz_span(int count, int nev, const int* first, const int* mults, int n) {
  const int c = count < nev ? count : nev;
  if (c <= 0) return n < 1 ? 0 : 1;
  const int K = first[c - 1] + (mults[c - 1] > 0 ? mults[c - 1] : 1);
  return K < n ? K : n;
}

// Weight of the k-th eigenvector in that combination: +-[0.5, 1.5) from the
// splitmix64 sequence (Steele, Lea & Flood, OOPSLA 2014) of the solve's seed.
// Unit weights could cancel two copies of one eigenvector; these cannot, and
// the start stays reproducible.
AED_HD inline double ritz_weight(unsigned long long seed, int k) {
  unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(k + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  const double u = (double)(z >> 11) * (1.0 / 9007199254740992.0);
  return ((z >> 10) & 1ull ? -1.0 : 1.0) * (0.5 + u);
}

// Eigenvector z of the tridiagonal (alpha, beta[0..n-2]) for eigenvalue lam by
// inverse iteration with a partially pivoted LU of T - lam I (two sweeps),
// normalised.  scratch: 6*n doubles.
AED_HD inline void inverse_iteration(int n, const double* alpha, const double* beta, double lam, double* z,
                                     double* scratch) {
  double* a = scratch;      // diagonal of U
  double* b = a + n;        // first super-diagonal of U
  double* c = b + n;        // second super-diagonal of U (from pivoting)
  double* l = c + n;        // multipliers
  int* piv = (int*)(l + n);  // row swaps (n ints fit in n doubles)
  double* rhs = l + 2 * n;
  double scale = 0.0;
  for (int i = 0; i < n; ++i) scale = dmax(scale, fabs(alpha[i]) + (i + 1 < n ? fabs(beta[i]) : 0.0));
  const double tiny = (scale > 0 ? scale : 1.0) * 1e-14;
  // LU with partial pivoting of the tridiagonal T - lam I
  for (int i = 0; i < n; ++i) {
    a[i] = alpha[i] - lam;
    b[i] = i + 1 < n ? beta[i] : 0.0;
    c[i] = 0.0;
  }
  for (int i = 0; i + 1 < n; ++i) {
    const double sub = beta[i];  // element (i+1, i)
    if (fabs(a[i]) >= fabs(sub)) {
      piv[i] = 0;
      const double piv_v = a[i] != 0.0 ? a[i] : tiny;
      a[i] = piv_v;
      l[i] = sub / piv_v;
      a[i + 1] -= l[i] * b[i];
      // c[i] stays 0
    } else {
      piv[i] = 1;
      // swap rows i and i+1: row i = (sub, a[i+1], b[i+1]); row i+1 = (a[i], b[i], 0)
      const double r0 = a[i], r1 = b[i];
      a[i] = sub;
      b[i] = a[i + 1];
      c[i] = i + 2 < n ? b[i + 1] : 0.0;
      l[i] = r0 / sub;
      a[i + 1] = r1 - l[i] * b[i];
      if (i + 2 < n) b[i + 1] = -l[i] * c[i];
    }
  }
  if (a[n - 1] == 0.0) a[n - 1] = tiny;
  for (int i = 0; i < n; ++i) z[i] = 1.0;
  for (int sweep = 0; sweep < 3; ++sweep) {
    for (int i = 0; i < n; ++i) rhs[i] = z[i];
    // forward: apply the row swaps and multipliers
    for (int i = 0; i + 1 < n; ++i) {
      if (piv[i]) {
        const double t = rhs[i];
        rhs[i] = rhs[i + 1];
        rhs[i + 1] = t;
      }
      rhs[i + 1] -= l[i] * rhs[i];
    }
    // back substitution with U (diagonal a, super-diagonals b, c)
    for (int i = n - 1; i >= 0; --i) {
      double v = rhs[i];
      if (i + 1 < n) v -= b[i] * z[i + 1];
      if (i + 2 < n) v -= c[i] * z[i + 2];
      z[i] = v / a[i];
    }
    double nrm = 0.0;
    for (int i = 0; i < n; ++i) nrm += z[i] * z[i];
    nrm = sqrt(nrm);
    if (!(nrm > 0.0)) break;
    for (int i = 0; i < n; ++i) z[i] /= nrm;
  }
}

// Number of eigenvalues below x of the symmetric tridiagonal matrix with
// diagonal a[0..n) and off-diagonal b[0..n-1): sign changes of the leading
// principal minors det(T_k - x) (Sturm), by the three-term recurrence kept
// in range by power-of-two rescaling.  A zero minor counts as a change (the
// pivot taken as a tiny negative, as dstebz does).
AED_HD inline int sturm_count(const double* __restrict__ a, const double* __restrict__ b, int n,
                                           double x) {
  constexpr double kBig = 0x1p400, kSmall = 0x1p-400, kTiny = 0x1p-800;
  double p0 = 1.0, p1 = a[0] - x;
  if (p1 == 0.0) p1 = -kTiny;
  int cnt = p1 < 0.0 ? 1 : 0;
  for (int k = 1; k < n; ++k) {
    const double bb = b[k - 1];
    double p2 = fma(a[k] - x, p1, -(bb * bb) * p0);
    if (p2 == 0.0) p2 = p1 > 0.0 ? -kTiny : kTiny;
    cnt += (p2 < 0.0) != (p1 < 0.0) ? 1 : 0;
    const double ap = fabs(p2);
    if (ap > kBig) {
      p2 *= kSmall;
      p1 *= kSmall;
    } else if (ap < kSmall && fabs(p1) < kSmall) {
      p2 *= kBig;
      p1 *= kBig;
    }
    p0 = p1;
    p1 = p2;
  }
  return cnt;
}

// Gershgorin interval of (a, b, n), widened by a few ulps of its scale.
AED_HD inline void gershgorin(const double* __restrict__ a, const double* __restrict__ b, int n, double* lo,
                           double* hi) {
  double l = a[0], h = a[0];
  for (int i = 0; i < n; ++i) {
    const double r = (i > 0 ? fabs(b[i - 1]) : 0.0) + (i + 1 < n ? fabs(b[i]) : 0.0);
    l = fmin(l, a[i] - r);
    h = fmax(h, a[i] + r);
  }
  const double pad = 8.0 * DBL_EPSILON * dmax(fabs(l), fabs(h)) + DBL_MIN;
  *lo = l - pad;
  *hi = h + pad;
}

// The k-th smallest eigenvalue (0-based) of (a, b, n) by bisection of
// [lo, hi] (count(lo) <= k < count(hi)): the rule of the batched check's
// lanes (one value per lane), for a host to reproduce.
AED_HD inline double bisect_eigenvalue(const double* a, const double* b, int n, int k, double lo, double hi) {
  for (int it = 0; it < 80; ++it) {
    const double w = hi - lo, x = lo + 0.5 * w;
    if (!(w > 2.0 * DBL_EPSILON * dmax(fabs(lo), fabs(hi))) || x == lo || x == hi) break;
    if (sturm_count(a, b, n, x) > k)
      hi = x;
    else
      lo = x;
  }
  return 0.5 * (lo + hi);
}

// One value of the walk: its first index in the sorted spectrum, its
// multiplicity and the index whose eigenvector's last component gives its
// error (-1: a multiple value, error 0).
struct WalkItem {
  double value;
  int first, mult, zidx;
};

// tcore::analyze_walk over the prefixes ev[0..nt) of T's sorted spectrum and
// evg[0..ng) of the reduced T's, top = T's largest eigenvalue.  Returns the
// number of values written to items (at most cap), or -1 when the walk needs
// an eigenvalue past a prefix.
AED_HD inline int walk_prefix(int n, double alpha_max, double beta_max, const double* ev, int nt, double top,
                           const double* evg, int ng, int cap, double thold_rel, WalkItem* items, double* thold_out,
                           double* multol_out) {
  const double eps = DBL_EPSILON;
  const double error_tol = pow(eps, 2.0 / 3.0);
  const double multol = dmax(alpha_max, beta_max) * 2 * eps * (10000 + n);
  double thold = dmax(error_tol * dmax(ev[0], top), 5 * multol);
  if (thold_rel > 0.0) thold = dmax(thold, thold_rel * dmax(fabs(ev[0]), fabs(top)));
  *thold_out = thold;
  *multol_out = multol;
  int t2 = 0, out = 0, i0 = 0;
  while (i0 < n && out < cap) {
    if (i0 >= nt) return -1;
    const double temp = ev[i0];
    int i1 = i0 + 1;
    while (i1 < n) {
      if (i1 >= nt) return -1;
      if ((ev[i1] - temp) > thold) break;
      ++i1;
    }
    int mult = i1 - i0;
    if (mult == 1) {
      for (int j = t2; j < n - 2; ++j, ++t2) {
        if (j >= ng) return -1;
        if ((evg[j] - temp) >= multol) break;
        if (fabs(temp - evg[j]) < multol) {
          mult = 0;
          ++t2;
          break;
        }
      }
    }
    if (mult != 0) items[out++] = {temp, i0, mult, mult == 1 ? i1 - 1 : -1};
    i0 = i1;
  }
  return out;
}

}  // namespace tcore
}  // namespace aed
