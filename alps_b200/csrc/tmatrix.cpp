// tmatrix.cpp -- host-side Lanczos T-matrix analysis.
//
// Tmatrix::compute(do_err = true) of src/ietl/tmatrix.h:121-228 with the LAPACK
// dstev call (src/ietl/ietl2lapack.h:84-99) replaced by an implicit QL
// eigensolver for symmetric tridiagonal matrices (Bowdler, Martin, Reinsch &
// Wilkinson, Numer. Math. 11 (1968) 293-306).  Only the last row of the
// eigenvector matrix is formed: it is the only part the error estimates
// |beta_m z_{m,i}| use, so each analysis costs O(m^2) instead of O(m^3).

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

#include "aed_internal.h"
#include "tmatrix_core.h"

namespace aed {

// d[0..n): diagonal -> eigenvalues ascending.  e[0..n): sub-diagonal in
// e[0..n-2] (destroyed).  zlast (optional, n entries): last row of Z.
// zfull (optional, n*n, column-major): all eigenvectors (column k <-> d[k]).
int tridiag_eigen(int n, double* d, double* e, double* zlast, double* zfull) {
  if (n <= 0) return 0;
  if (zlast) {
    std::fill(zlast, zlast + n, 0.0);
    zlast[n - 1] = 1.0;
  }
  if (zfull) {
    std::fill(zfull, zfull + (size_t)n * n, 0.0);
    for (int k = 0; k < n; ++k) zfull[(size_t)k * n + k] = 1.0;
  }
  e[n - 1] = 0.0;
  for (int l = 0; l < n; ++l) {
    for (int sweep = 0;; ++sweep) {
      // smallest m >= l where the matrix splits
      int m = l;
      while (m < n - 1 && std::fabs(e[m]) > DBL_EPSILON * (std::fabs(d[m]) + std::fabs(d[m + 1]))) ++m;
      if (m == l) break;
      if (sweep >= 90) return l + 1;
      // shift: eigenvalue of the leading 2x2 block closer to d[l]
      const double theta = (d[l + 1] - d[l]) / (2.0 * e[l]);
      const double rho = std::hypot(theta, 1.0);
      double g = d[m] - d[l] + e[l] / (theta + std::copysign(rho, theta));
      double s = 1.0, c = 1.0, p = 0.0;
      int i = m - 1;
      bool split = false;
      for (; i >= l; --i) {
        const double f = s * e[i], b = c * e[i];
        const double r = std::hypot(f, g);
        e[i + 1] = r;
        if (r == 0.0) {  // underflow: the matrix splits at i+1
          d[i + 1] -= p;
          e[m] = 0.0;
          split = true;
          break;
        }
        s = f / r;
        c = g / r;
        const double gg = d[i + 1] - p;
        const double t = (d[i] - gg) * s + 2.0 * c * b;
        p = s * t;
        d[i + 1] = gg + p;
        g = c * t - b;
        if (zlast) {
          const double z1 = zlast[i + 1];
          zlast[i + 1] = s * zlast[i] + c * z1;
          zlast[i] = c * zlast[i] - s * z1;
        }
        if (zfull) {
          double* ci = zfull + (size_t)i * n;
          double* cj = zfull + (size_t)(i + 1) * n;
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
  // ascending order (stable), carrying zlast / zfull columns
  std::vector<int> ord(n);
  for (int i = 0; i < n; ++i) ord[i] = i;
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return d[a] < d[b]; });
  std::vector<double> tmp(d, d + n);
  for (int i = 0; i < n; ++i) d[i] = tmp[ord[i]];
  if (zlast) {
    tmp.assign(zlast, zlast + n);
    for (int i = 0; i < n; ++i) zlast[i] = tmp[ord[i]];
  }
  if (zfull) {
    std::vector<double> zt(zfull, zfull + (size_t)n * n);
    for (int i = 0; i < n; ++i)
      std::copy(zt.begin() + (size_t)ord[i] * n, zt.begin() + (size_t)(ord[i] + 1) * n, zfull + (size_t)i * n);
  }
  return 0;
}

int tmatrix_analyze(int n, const double* alpha, const double* beta, double alpha_max, double beta_max,
                    TmatInfo& out, double thold_rel) {
  out = TmatInfo();
  if (n < 1) return AED_OK;
  std::vector<double> scratch(5 * (size_t)n + 2), ev(n), er(n);
  std::vector<int> mu(n), fi(n);
  tcore::TResult res;
  if (tcore::analyze(n, alpha, beta, alpha_max, beta_max, scratch.data(), n, ev.data(), er.data(), mu.data(),
                     fi.data(), &res, thold_rel))
    return fail(AED_ERR_TRIDIAG, "tridiagonal eigensolver failed");
  out.thold = res.thold;
  out.multol = res.multol;
  out.evals.assign(ev.begin(), ev.begin() + res.count);
  out.errs.assign(er.begin(), er.begin() + res.count);
  out.mults.assign(mu.begin(), mu.begin() + res.count);
  out.first.assign(fi.begin(), fi.begin() + res.count);
  return AED_OK;
}

// lanczos_iteration_nlowest::converged (src/ietl/iteration.h:115-130)
bool nlowest_converged(const TmatInfo& t, int nev, double rtol, double atol) {
  if ((int)t.evals.size() < nev) return false;
  for (int i = 0; i < nev; ++i)
    if (t.errs[i] > std::max(atol, rtol * std::fabs(t.evals[i]))) return false;
  return true;
}

}  // namespace aed
