// ed_oracle.cpp -- CPU restatement of the ALPS `sparsediag` Lanczos path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the oracle: the tests, the smoke check
// and the CPU-baseline leg of bench.py load it to check (or time beside) the CUDA
// engine.  Nothing in the product (alps_b200/, include/) links, loads or calls it.
//
// Parity status: the basis order, the bond matrix elements and the lattice bond
// order are pinned against the reference's own golden outputs
// (test/model/example10, example12, example3, example4; test/lattice/example5,
// example6) through tests/golden/.  The tridiagonal solver is pinned against
// LAPACK dstev (scipy) in the tests.  Lanczos eigenvalues are pinned against
// dense eigensolves and closed-form energies (the reference's own tests hold
// no sparsediag eigenvalues).
//
// What it restates (reference paths are relative to the ALPS source tree):
//   * basis_states<short>::build       src/alps/model/basisstates.h:175-278
//     (odometer over per-site indices, site 0 most significant, Sz pruning)
//   * basis_states::index              src/alps/model/basisstates.h:68-74
//     (std::lower_bound; returns D when absent)
//   * hamiltonian_matrix::build        src/alps/model/hamiltonian_matrix.hpp:422-450
//     initialized_matrix               hamiltonian_matrix.hpp:44-58  (M(i,i) += 1; -= 1)
//     apply_operator(GlobalOperator)   hamiltonian_matrix.hpp:387-397 (sites, then bonds)
//     apply_operator(site)             hamiltonian_matrix.hpp:268-291
//     apply_operator(bond)             hamiltonian_matrix.hpp:307-345
//     matrix_as_vector element_proxy   src/alps/numeric/matrix_as_vector.hpp:72-73
//   * y = prod(M, x)                   src/ietl/interface/ublas.h:57-63 (row sums in
//     ascending column order, t = 0; t += M(i,j) * x[j])
//   * ietl::lanczos                    src/ietl/lanczos.h:341-406
//   * Tmatrix::compute                 src/ietl/tmatrix.h:121-228
//   * lanczos_iteration_nlowest        src/ietl/iteration.h:66-130
//   * ietl2lapack::stev                src/ietl/ietl2lapack.h:67-99 (LAPACK dstev;
//     restated here as implicit QL, Bowdler, Martin, Reinsch & Wilkinson,
//     Numer. Math. 11 (1968) 293-306)
//
// State encoding: site s <-> bit (N-1-s); spin up (site-basis index 1) = bit set.
// With that encoding the reference's lexicographic order over index vectors is
// ascending unsigned-integer order.

#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------------------
// Basis: odometer enumeration (basisstates.h:175-278).
//
// idx[s] in {0 (Sz=-1/2), 1 (Sz=+1/2)} (sitebasisstates.h:84-85,98-99).  The
// constraint is sum_s Sz = Sz_total, i.e. #up = n_up.  We count in units of
// "number of ups" instead of half-integers: identical pruning.
// ---------------------------------------------------------------------------
static int64_t odometer_basis(int N, int n_up, uint32_t* out, int64_t cap) {
  if (N <= 0) return 0;
  std::vector<int> idx(N, 0);
  const int last = N - 1;
  // max/min number of ups achievable on sites ik+1..N-1
  std::vector<int> max_partial(N, 0), min_partial(N, 0);
  for (int ik = 0; ik < last; ++ik) {
    max_partial[ik] = last - ik;  // every later site up
    min_partial[ik] = 0;
  }
  int64_t count = 0;
  while (true) {
    int k = last;
    while (idx[k] >= 2 && k) {
      idx[k] = 0;
      --k;
      ++idx[k];
      if (idx[k] < 2) {
        int val = 0;
        for (int is = 0; is <= k; ++is) val += idx[is];
        if (val + max_partial[k] < n_up || val + min_partial[k] > n_up) ++idx[k];
      }
    }
    if (k == 0 && idx[k] >= 2) break;
    int ups = 0;
    for (int s = 0; s < N; ++s) ups += idx[s];
    if (ups == n_up) {
      if (out && count < cap) {
        uint32_t st = 0;
        for (int s = 0; s < N; ++s)
          if (idx[s]) st |= 1u << (N - 1 - s);
        out[count] = st;
      }
      ++count;
    }
    ++idx[last];
  }
  return count;
}

// lower_bound lookup (basisstates.h:68-74): D when absent.
static inline int64_t lb_index(const uint32_t* st, int64_t D, uint32_t s) {
  const uint32_t* it = std::lower_bound(st, st + D, s);
  if (it == st + D) return D;
  return (*it == s) ? (it - st) : D;
}

// splitmix64 (Steele, Lea & Flood, OOPSLA 2014): the engine's start-vector
// generator.  The reference draws its start vector from Boost's
// lagged_fibonacci607 (sparsediag.h:98), which is not reproducible without
// Boost; both sides of every parity test use this generator instead.
static inline double start_value(uint64_t seed, uint64_t i) {
  uint64_t z = seed + 0x9E3779B97F4A7C15ull * (i + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (double)(z >> 11) * 0x1.0p-53;
}

// ---------------------------------------------------------------------------
// Explicit matrix, built in the reference's element order.
// ---------------------------------------------------------------------------
struct Matrix {
  int N = 0, n_up = 0;
  int64_t D = 0;
  std::vector<uint32_t> states;
  std::vector<int64_t> rowptr;
  std::vector<int32_t> col;
  std::vector<double> val;
};

struct Entry {
  int64_t j;
  double v;
};

// M(i,j) += v through a row map (matrix_as_vector.hpp:72-73; ublas mapped
// storage starts an absent element at 0).
static inline void row_add(std::vector<Entry>& row, int64_t j, double v) {
  for (auto& e : row)
    if (e.j == j) {
      e.v += v;
      return;
    }
  row.push_back({j, 0.0});
  row.back().v += v;
}

// Symbolic spin-1/2 matrix elements of the "spin" HAMILTONIAN
// (lib/xml/models.xml.in:342-373) as printed by the reference
// (test/model/example3.output, HSpinSite / HSpinBond):
//   site  [0][0] = 0.25*D + 0.5*h        (Sz = -1/2)
//         [1][1] = 0.25*D - 0.5*h        (Sz = +1/2)
//   bond  [a][a][a][a]         =  0.25*Jz + 0.0625*K     (parallel, diagonal)
//         [a][b][a][b], a!=b   = -0.25*Jz + 0.3125*K     (antiparallel, diagonal)
//         [a][b][b][a], a!=b   =  0.5*Jxy - 0.25*K       (spin flip)
struct BondTensor {
  double m[2][2][2][2];
};

static BondTensor spin_bond(double jz, double jxy, double kq) {
  BondTensor t;
  std::memset(&t, 0, sizeof t);
  const double par = 0.25 * jz + 0.0625 * kq;
  const double anti = -0.25 * jz + 0.3125 * kq;
  const double flip = 0.5 * jxy - 0.25 * kq;
  t.m[0][0][0][0] = par;
  t.m[1][1][1][1] = par;
  t.m[0][1][0][1] = anti;
  t.m[1][0][1][0] = anti;
  t.m[0][1][1][0] = flip;
  t.m[1][0][0][1] = flip;
  return t;
}

static Matrix* build_matrix(int N, int n_up, const double* site_h, const double* site_d, int nb,
                            const int* s1, const int* s2, const double* jz, const double* jxy,
                            const double* kq) {
  Matrix* M = new Matrix;
  M->N = N;
  M->n_up = n_up;
  M->D = odometer_basis(N, n_up, nullptr, 0);
  M->states.resize(M->D);
  odometer_basis(N, n_up, M->states.data(), M->D);
  const int64_t D = M->D;
  std::vector<BondTensor> bt(nb);
  for (int b = 0; b < nb; ++b) bt[b] = spin_bond(jz[b], jxy[b], kq ? kq[b] : 0.0);
  M->rowptr.assign(D + 1, 0);
  std::vector<std::vector<Entry>> rows(D);
  for (int64_t i = 0; i < D; ++i) {
    std::vector<Entry>& row = rows[i];
    // initialized_matrix (hamiltonian_matrix.hpp:53-56)
    row_add(row, i, 1.0);
    row_add(row, i, -1.0);
  }
  const uint32_t* st = M->states.data();
  // site terms first (hamiltonian_matrix.hpp:391-392, 268-291)
  if (site_h || site_d) {
    for (int s = 0; s < N; ++s) {
      const double h = site_h ? site_h[s] : 0.0;
      const double dd = site_d ? site_d[s] : 0.0;
      const double mat[2] = {0.25 * dd + 0.5 * h, 0.25 * dd - 0.5 * h};
      const int bit = N - 1 - s;
      for (int64_t i = 0; i < D; ++i) {
        const int is = (st[i] >> bit) & 1;
        const double v = mat[is];
        if (v != 0.0) {
          // diagonal: newstate == state, j == i
          row_add(rows[i], i, v);
        }
      }
    }
  }
  // bonds in graph order (hamiltonian_matrix.hpp:395-396, 307-345)
  for (int b = 0; b < nb; ++b) {
    const int b1 = N - 1 - s1[b], b2 = N - 1 - s2[b];
    for (int64_t i = 0; i < D; ++i) {
      const uint32_t state = st[i];
      const int is1 = (state >> b1) & 1, is2 = (state >> b2) & 1;
      for (int js1 = 0; js1 < 2; ++js1)
        for (int js2 = 0; js2 < 2; ++js2) {
          const double v = bt[b].m[is1][is2][js1][js2];
          if (v == 0.0) continue;
          uint32_t ns = state;
          ns = (ns & ~(1u << b1)) | ((uint32_t)js1 << b1);
          ns = (ns & ~(1u << b2)) | ((uint32_t)js2 << b2);
          const int64_t j = lb_index(st, D, ns);
          if (j < D) row_add(rows[i], j, v);
        }
    }
  }
  int64_t nnz = 0;
  for (int64_t i = 0; i < D; ++i) {
    std::sort(rows[i].begin(), rows[i].end(), [](const Entry& a, const Entry& b) { return a.j < b.j; });
    nnz += (int64_t)rows[i].size();
    M->rowptr[i + 1] = nnz;
  }
  M->col.resize(nnz);
  M->val.resize(nnz);
  for (int64_t i = 0; i < D; ++i) {
    int64_t p = M->rowptr[i];
    for (auto& e : rows[i]) {
      M->col[p] = (int32_t)e.j;
      M->val[p] = e.v;
      ++p;
    }
    std::vector<Entry>().swap(rows[i]);
  }
  return M;
}

// y = prod(M, x): per row, t = 0; t += M(i,j) * x[j] in ascending j.
// volatile-free but compiled with -ffp-contract=off so products and sums round
// separately, as on the reference's x86-64 build.
static void csr_mult(const Matrix* M, const double* x, double* y) {
  const int64_t D = M->D;
  for (int64_t i = 0; i < D; ++i) {
    double t = 0.0;
    for (int64_t p = M->rowptr[i]; p < M->rowptr[i + 1]; ++p) t += M->val[p] * x[M->col[p]];
    y[i] = t;
  }
}

// ---------------------------------------------------------------------------
// Tridiagonal eigenproblem: implicit QL with shifts (Bowdler, Martin, Reinsch &
// Wilkinson 1968).  d: diagonal (overwritten by eigenvalues, ascending on
// return), e: sub-diagonal e[0..n-2] (destroyed; needs n entries).  zlast, if
// given, receives the last row of the orthonormal eigenvector matrix (the only
// part Tmatrix::compute uses); zfull, if given, the full matrix (column-major,
// column k = eigenvector k).  Returns 0, or l+1 if eigenvalue l did not
// converge (LAPACK's info > 0).
// ---------------------------------------------------------------------------
static int tridiag_ql(int n, double* d, double* e, double* zlast, double* zfull) {
  if (n <= 0) return 0;
  if (zlast) {
    for (int k = 0; k < n; ++k) zlast[k] = 0.0;
    zlast[n - 1] = 1.0;
  }
  if (zfull) {
    for (int k = 0; k < n * n; ++k) zfull[k] = 0.0;
    for (int k = 0; k < n; ++k) zfull[k * n + k] = 1.0;
  }
  e[n - 1] = 0.0;
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    while (true) {
      int m = l;
      for (; m < n - 1; ++m) {
        const double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
        if (std::fabs(e[m]) <= DBL_EPSILON * dd) break;
      }
      if (m == l) break;
      if (++iter > 90) return l + 1;
      // Wilkinson-type shift from the leading 2x2 block at l
      double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
      double r = std::hypot(g, 1.0);
      g = d[m] - d[l] + e[l] / (g + std::copysign(r, g));
      double s = 1.0, c = 1.0, p = 0.0;
      bool deflated = false;
      for (int i = m - 1; i >= l; --i) {
        const double f = s * e[i];
        const double b = c * e[i];
        r = std::hypot(f, g);
        e[i + 1] = r;
        if (r == 0.0) {
          d[i + 1] -= p;
          e[m] = 0.0;
          deflated = true;
          break;
        }
        s = f / r;
        c = g / r;
        g = d[i + 1] - p;
        r = (d[i] - g) * s + 2.0 * c * b;
        p = s * r;
        d[i + 1] = g + p;
        g = c * r - b;
        if (zlast) {
          const double t = zlast[i + 1];
          zlast[i + 1] = s * zlast[i] + c * t;
          zlast[i] = c * zlast[i] - s * t;
        }
        if (zfull) {
          double* ci = zfull + (size_t)i * n;
          double* cj = zfull + (size_t)(i + 1) * n;
          for (int k = 0; k < n; ++k) {
            const double t = cj[k];
            cj[k] = s * ci[k] + c * t;
            ci[k] = c * ci[k] - s * t;
          }
        }
      }
      if (deflated) continue;
      d[l] -= p;
      e[l] = g;
      e[m] = 0.0;
    }
  }
  // ascending order, carrying the eigenvector data along (selection sort)
  for (int i = 0; i < n - 1; ++i) {
    int k = i;
    for (int j = i + 1; j < n; ++j)
      if (d[j] < d[k]) k = j;
    if (k != i) {
      std::swap(d[i], d[k]);
      if (zlast) std::swap(zlast[i], zlast[k]);
      if (zfull)
        for (int r2 = 0; r2 < n; ++r2) std::swap(zfull[(size_t)i * n + r2], zfull[(size_t)k * n + r2]);
    }
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Tmatrix::compute(do_err=true) restated (tmatrix.h:121-228).
// ---------------------------------------------------------------------------
struct TmatResult {
  std::vector<double> eval_distinct, err, eval_noghost, err_noghost;
  std::vector<int> mult, mult_noghost;
  double thold = 0, multol = 0;
  int info = 0;
};

static void tmatrix_compute(int n, const double* alpha, const double* beta, double alpha_max,
                            double beta_max, TmatResult& R) {
  R = TmatResult();
  std::vector<double> eval(alpha, alpha + n), e(n + 1, 0.0), zl(n);
  for (int i = 0; i + 1 < n; ++i) e[i] = beta[i];
  R.info = tridiag_ql(n, eval.data(), e.data(), zl.data(), nullptr);
  if (R.info) return;
  const double eps = DBL_EPSILON;
  const double error_tol = std::pow(eps, 2. / 3.);
  R.multol = std::max(alpha_max, beta_max) * 2 * eps * (10000 + n);
  R.thold = std::max(eval[0], eval[n - 1]);
  R.thold = std::max(error_tol * R.thold, 5 * R.multol);
  const double beta_last = beta[n - 1];
  double temp = eval[0];
  R.eval_distinct.push_back(eval[0]);
  int multiple = 1;
  for (int i = 1; i < n; ++i) {
    if ((eval[i] - temp) > R.thold) {
      R.eval_distinct.push_back(eval[i]);
      temp = eval[i];
      R.mult.push_back(multiple);
      R.err.push_back(multiple > 1 ? 0. : std::fabs(beta_last * zl[i - 1]));
      multiple = 1;
    } else {
      multiple++;
    }
  }
  R.mult.push_back(multiple);
  R.err.push_back(multiple > 1 ? 0. : std::fabs(beta_last * zl[n - 1]));
  // ghosts: T with first row and column removed (tmatrix.h:189-217)
  std::vector<double> eval_g(n > 1 ? n - 1 : 0), eg(n + 1, 0.0);
  for (int i = 1; i < n; ++i) eval_g[i - 1] = alpha[i];
  for (int i = 1; i + 1 < n; ++i) eg[i - 1] = beta[i];
  if (n > 1) {
    R.info = tridiag_ql(n - 1, eval_g.data(), eg.data(), nullptr, nullptr);
    if (R.info) return;
  }
  int t2 = 0;
  for (size_t i = 0; i < R.eval_distinct.size(); ++i) {
    const double k = R.eval_distinct[i];
    if (R.mult[i] == 1) {
      for (int j = t2; j < n - 2; j++, t2++) {
        if ((eval_g[j] - k) >= R.multol) break;
        if (std::fabs(k - eval_g[j]) < R.multol) {
          R.mult[i] = 0;
          R.err[i] = 0;
          t2++;
          break;
        }
      }
    }
  }
  for (size_t i = 0; i < R.eval_distinct.size(); ++i)
    if (R.mult[i] != 0) {
      R.eval_noghost.push_back(R.eval_distinct[i]);
      R.mult_noghost.push_back(R.mult[i]);
      R.err_noghost.push_back(R.err[i]);
    }
}

// lanczos_iteration_nlowest::converged (iteration.h:115-130) on a computed T.
static bool nlowest_converged(const TmatResult& R, int nev, double rtol, double atol) {
  if ((int)R.eval_noghost.size() < nev) return false;
  for (int i = 0; i < nev; ++i)
    if (R.err_noghost[i] > std::max(atol, rtol * std::fabs(R.eval_noghost[i]))) return false;
  return true;
}

static double dotv(const std::vector<double>& a, const std::vector<double>& b) {
  double t = 0.0;
  for (size_t i = 0; i < a.size(); ++i) t += a[i] * b[i];
  return t;
}

static double norm2v(const std::vector<double>& a) {
  double t = 0.0;
  for (double v : a) t += v * v;
  return std::sqrt(t);
}

}  // namespace

extern "C" {

int64_t orc_basis_build(int N, int n_up, uint32_t* out, int64_t cap) {
  if (N < 1 || N > 32 || n_up < 0 || n_up > N) return -1;
  return odometer_basis(N, n_up, out, cap);
}

int64_t orc_index(const uint32_t* states, int64_t D, uint32_t s) { return lb_index(states, D, s); }

void orc_start_vector(uint64_t seed, int64_t D, double* out) {
  for (int64_t i = 0; i < D; ++i) out[i] = start_value(seed, (uint64_t)i);
}

void* orc_matrix_build(int N, int n_up, const double* site_h, const double* site_d, int nb,
                       const int* s1, const int* s2, const double* jz, const double* jxy,
                       const double* kq) {
  if (N < 1 || N > 32 || n_up < 0 || n_up > N) return nullptr;
  for (int b = 0; b < nb; ++b)
    if (s1[b] < 0 || s1[b] >= N || s2[b] < 0 || s2[b] >= N || s1[b] == s2[b]) return nullptr;
  return build_matrix(N, n_up, site_h, site_d, nb, s1, s2, jz, jxy, kq);
}

int64_t orc_matrix_dim(void* h) { return static_cast<Matrix*>(h)->D; }
int64_t orc_matrix_nnz(void* h) { return (int64_t) static_cast<Matrix*>(h)->val.size(); }

void orc_matrix_states(void* h, uint32_t* out) {
  Matrix* M = static_cast<Matrix*>(h);
  std::memcpy(out, M->states.data(), sizeof(uint32_t) * M->D);
}

void orc_matrix_csr(void* h, int64_t* rowptr, int32_t* col, double* val) {
  Matrix* M = static_cast<Matrix*>(h);
  std::memcpy(rowptr, M->rowptr.data(), sizeof(int64_t) * (M->D + 1));
  std::memcpy(col, M->col.data(), sizeof(int32_t) * M->col.size());
  std::memcpy(val, M->val.data(), sizeof(double) * M->val.size());
}

void orc_matrix_mult(void* h, const double* x, double* y) { csr_mult(static_cast<Matrix*>(h), x, y); }

// Rows [r0, r1) of y = prod(M, x): the bounded CPU-baseline sample.
void orc_matrix_mult_rows(void* h, const double* x, double* y, int64_t r0, int64_t r1) {
  Matrix* M = static_cast<Matrix*>(h);
  for (int64_t i = r0; i < r1 && i < M->D; ++i) {
    double t = 0.0;
    for (int64_t p = M->rowptr[i]; p < M->rowptr[i + 1]; ++p) t += M->val[p] * x[M->col[p]];
    y[i] = t;
  }
}

void orc_matrix_free(void* h) { delete static_cast<Matrix*>(h); }

// Eigenvalues (ascending) of the tridiagonal (d, e), e[0..n-2]; optional last
// row of the eigenvector matrix and optional full matrix (column-major).
int orc_stev(int n, const double* d, const double* e, double* w, double* zlast, double* zfull) {
  std::vector<double> ee(n + 1, 0.0);
  for (int i = 0; i + 1 < n; ++i) ee[i] = e[i];
  for (int i = 0; i < n; ++i) w[i] = d[i];
  return tridiag_ql(n, w, ee.data(), zlast, zfull);
}

// Tmatrix::compute(true) on (alpha, beta) of length n.  Outputs the distinct
// non-ghost eigenvalues, their errors and multiplicities (capacity cap);
// returns their count, or -info on a tridiagonal failure.  thold/multol out.
int orc_tmatrix(int n, const double* alpha, const double* beta, double* evals, double* errs,
                int* mults, int cap, double* thold_out, double* multol_out) {
  if (n < 1) return 0;
  double amax = alpha[0], bmax = beta[0];
  for (int i = 1; i < n; ++i) {
    amax = std::max(amax, alpha[i]);
    bmax = std::max(bmax, beta[i]);
  }
  TmatResult R;
  tmatrix_compute(n, alpha, beta, amax, bmax, R);
  if (R.info) return -R.info;
  const int cnt = (int)R.eval_noghost.size();
  for (int i = 0; i < cnt && i < cap; ++i) {
    evals[i] = R.eval_noghost[i];
    errs[i] = R.err_noghost[i];
    mults[i] = R.mult_noghost[i];
  }
  if (thold_out) *thold_out = R.thold;
  if (multol_out) *multol_out = R.multol;
  return cnt;
}

// ietl::lanczos::calculate_eigenvalues with lanczos_iteration_nlowest
// (lanczos.h:341-406, iteration.h:66-130), then sparsediag's n = min(k, #distinct)
// (sparsediag.h:115-118).  start: optional start vector (else the splitmix64
// stream for `seed`).  Returns the number of eigenvalues written, or a negative
// code (-1 bad args, -2 tridiagonal failure).  *iters = T-matrix size,
// *fail = 1 when max_iter was reached.
int orc_lanczos(void* h, int nev, int max_iter, uint64_t seed, const double* start, double rtol,
                double atol, double* evals, double* errs, int* iters, int* fail, double* alpha_out,
                double* beta_out, int ab_cap) {
  Matrix* M = static_cast<Matrix*>(h);
  const int64_t D = M->D;
  if (D < 2 || nev < 1 || max_iter < 1) return -1;
  std::vector<double> startvector(D), vec2(D), vec3(D);
  std::vector<double> alpha, beta;
  double amax = 0, bmax = 0;
  auto push = [&](double a, double b) {
    alpha.push_back(a);
    beta.push_back(b);
    if (alpha.size() == 1) {
      amax = a;
      bmax = b;
    } else {
      if (a > amax) amax = a;
      if (b > bmax) bmax = b;
    }
  };
  // make_first_step (lanczos.h:377-390)
  for (int64_t i = 0; i < D; ++i) startvector[i] = start ? start[i] : start_value(seed, (uint64_t)i);
  {
    const double nrm = norm2v(startvector);
    for (auto& v : startvector) v /= nrm;
  }
  csr_mult(M, startvector.data(), vec2.data());
  double a = dotv(startvector, vec2);
  for (int64_t i = 0; i < D; ++i) vec2[i] -= a * startvector[i];
  double b = norm2v(vec2);
  for (auto& v : vec2) v /= b;
  push(a, b);
  unsigned it = 1;  // generate_tmatrix: ++iter once for n = 1
  TmatResult R;
  int failed = 0;
  while (true) {
    // finished() (iteration.h:73-83)
    bool conv = false;
    if (it > 1) {
      tmatrix_compute((int)alpha.size(), alpha.data(), beta.data(), amax, bmax, R);
      if (R.info) return -2;
      conv = nlowest_converged(R, nev, rtol, atol);
    }
    if (conv) break;
    if (it >= (unsigned)max_iter) {
      failed = 1;
      break;
    }
    // make_step (lanczos.h:392-406)
    const double bprev = beta.back();
    csr_mult(M, vec2.data(), vec3.data());
    a = dotv(vec2, vec3);
    for (int64_t i = 0; i < D; ++i) vec3[i] -= a * vec2[i];
    for (int64_t i = 0; i < D; ++i) vec3[i] -= bprev * startvector[i];
    b = norm2v(vec3);
    for (auto& v : vec3) v /= b;
    std::swap(vec2, startvector);
    std::swap(vec3, vec2);
    push(a, b);
    ++it;
  }
  // eigenvalues() of the final T (computed above unless it == 1)
  if (it <= 1 || R.eval_noghost.empty()) {
    tmatrix_compute((int)alpha.size(), alpha.data(), beta.data(), amax, bmax, R);
    if (R.info) return -2;
  }
  const int n = std::min(nev, (int)R.eval_noghost.size());
  for (int i = 0; i < n; ++i) {
    evals[i] = R.eval_noghost[i];
    errs[i] = R.err_noghost[i];
  }
  *iters = (int)alpha.size();
  *fail = failed;
  for (int i = 0; i < (int)alpha.size() && i < ab_cap; ++i) {
    if (alpha_out) alpha_out[i] = alpha[i];
    if (beta_out) beta_out[i] = beta[i];
  }
  return n;
}

// Matrix-free H*x over the same basis with all host threads (the "best CPU"
// baseline; not the reference's algorithm).  Row sums follow the reference's
// ascending-column order so results equal csr_mult bit for bit.
void orc_hv_matfree(int N, const uint32_t* states, int64_t D, int nb, const int* s1, const int* s2,
                    const double* jz, const double* jxy, const double* x, double* y, int64_t r0,
                    int64_t r1) {
  (void)N;
  std::vector<std::pair<int, int>> bits(nb);
  for (int b = 0; b < nb; ++b) bits[b] = {N - 1 - s1[b], N - 1 - s2[b]};
  if (r1 > D) r1 = D;
#pragma omp parallel for schedule(static)
  for (int64_t i = r0; i < r1; ++i) {
    Entry row[130];
    int cnt = 0;
    const uint32_t s = states[i];
    double diag = 0.0;
    for (int b = 0; b < nb; ++b) {
      const int u = (s >> bits[b].first) & 1, v = (s >> bits[b].second) & 1;
      if (u == v) {
        const double d = 0.25 * jz[b];
        if (d != 0.0) diag += d;
      } else {
        const double d = -0.25 * jz[b];
        if (d != 0.0) diag += d;
        const double f = 0.5 * jxy[b];
        if (f != 0.0) {
          const uint32_t ns = s ^ ((1u << bits[b].first) | (1u << bits[b].second));
          const int64_t j = lb_index(states, D, ns);
          int q = 0;
          for (; q < cnt; ++q)
            if (row[q].j == j) break;
          if (q == cnt) row[cnt++] = {j, 0.0};
          row[q].v += f;
        }
      }
    }
    row[cnt++] = {i, diag};
    std::sort(row, row + cnt, [](const Entry& a2, const Entry& b2) { return a2.j < b2.j; });
    double t = 0.0;
    for (int q = 0; q < cnt; ++q) t += row[q].v * x[row[q].j];
    y[i] = t;
  }
}

// The Sz sector in ascending order by stepping to the next integer with the
// same popcount (Gosper's hack, HAKMEM 175): same output as the odometer,
// fast enough for the 10^8-state sectors the CPU-baseline samples need.
int64_t orc_basis_fast(int N, int n_up, uint32_t* out, int64_t cap) {
  if (N < 1 || N > 32 || n_up < 0 || n_up > N) return -1;
  int64_t cnt = 0;
  if (n_up == 0) {
    if (out && cap > 0) out[0] = 0;
    return 1;
  }
  uint64_t v = (1ull << n_up) - 1, lim = 1ull << N;
  while (v < lim) {
    if (out && cnt < cap) out[cnt] = (uint32_t)v;
    ++cnt;
    const uint64_t t = v | (v - 1);
    v = (t + 1) | (((~t & -~t) - 1) >> (__builtin_ctzll(v) + 1));
  }
  return cnt;
}

// Timed sample of the reference algorithm on rows [r0, r1) of a sector whose
// full state list is `states`: (1) build those rows of the explicit matrix in
// the reference's element order (hamiltonian_matrix.hpp:307-345 with
// lower_bound lookups), (2) y = prod(M, x) over them, (3) the per-step vector
// passes of make_step (dot, two axpy, norm, divide) over as many elements.
// One thread, as the reference.  Seconds are written to t_build, t_prod, t_vec.
void orc_sample_times(int N, const uint32_t* states, int64_t D, int nb, const int* s1, const int* s2,
                      const double* jz, const double* jxy, int64_t r0, int64_t r1, double* t_build,
                      double* t_prod, double* t_vec) {
  using clk = std::chrono::steady_clock;
  if (r1 > D) r1 = D;
  const int64_t R = r1 - r0;
  std::vector<BondTensor> bt(nb);
  for (int b = 0; b < nb; ++b) bt[b] = spin_bond(jz[b], jxy[b], 0.0);
  std::vector<int64_t> rp(R + 1, 0);
  std::vector<int32_t> col;
  std::vector<double> val;
  col.reserve(R * 32);
  val.reserve(R * 32);
  auto t0 = clk::now();
  std::vector<Entry> row;
  for (int64_t i = r0; i < r1; ++i) {
    row.clear();
    row_add(row, i, 1.0);
    row_add(row, i, -1.0);
    const uint32_t state = states[i];
    for (int b = 0; b < nb; ++b) {
      const int b1 = N - 1 - s1[b], b2 = N - 1 - s2[b];
      const int is1 = (state >> b1) & 1, is2 = (state >> b2) & 1;
      for (int js1 = 0; js1 < 2; ++js1)
        for (int js2 = 0; js2 < 2; ++js2) {
          const double v = bt[b].m[is1][is2][js1][js2];
          if (v == 0.0) continue;
          uint32_t ns = state;
          ns = (ns & ~(1u << b1)) | ((uint32_t)js1 << b1);
          ns = (ns & ~(1u << b2)) | ((uint32_t)js2 << b2);
          const int64_t j = lb_index(states, D, ns);
          if (j < D) row_add(row, j, v);
        }
    }
    std::sort(row.begin(), row.end(), [](const Entry& a, const Entry& b) { return a.j < b.j; });
    for (auto& e : row) {
      col.push_back((int32_t)e.j);
      val.push_back(e.v);
    }
    rp[i - r0 + 1] = (int64_t)col.size();
  }
  auto t1 = clk::now();
  std::vector<double> x(D);
  for (int64_t i = 0; i < D; ++i) x[i] = start_value(1, (uint64_t)i);
  std::vector<double> y(R);
  auto t2 = clk::now();
  for (int64_t i = 0; i < R; ++i) {
    double t = 0.0;
    for (int64_t p = rp[i]; p < rp[i + 1]; ++p) t += val[p] * x[col[p]];
    y[i] = t;
  }
  auto t3 = clk::now();
  // make_step's vector passes over R elements
  std::vector<double> v2(x.begin() + r0, x.begin() + r1), v0(R, 0.5);
  double a = 0.0;
  for (int64_t i = 0; i < R; ++i) a += v2[i] * y[i];
  for (int64_t i = 0; i < R; ++i) y[i] -= a * v2[i];
  for (int64_t i = 0; i < R; ++i) y[i] -= 0.3 * v0[i];
  double nn = 0.0;
  for (int64_t i = 0; i < R; ++i) nn += y[i] * y[i];
  nn = std::sqrt(nn);
  for (int64_t i = 0; i < R; ++i) y[i] /= nn;
  auto t4 = clk::now();
  volatile double sink = y[R / 2];
  (void)sink;
  *t_build = std::chrono::duration<double>(t1 - t0).count();
  *t_prod = std::chrono::duration<double>(t3 - t2).count();
  *t_vec = std::chrono::duration<double>(t4 - t3).count();
}

// Rows [r0, r1) of the explicit matrix of a sector whose full state list is
// `states`, built row by row in the reference's element order, then
// y[i - r0] = prod(M, x)_i.  Per element M(i,j) the additions come in the order
// of build_matrix (initialized_matrix's +1 -1, the site terms by site, the
// bonds by bond and (js1, js2)), so the rows equal build_matrix's bit for bit;
// this serves sectors too large for the whole matrix (10^8 states): x is the
// full vector, only the window's rows are formed.  yabs (optional) receives
// sum_j |M_ij x_j| per row (the scale of a row's rounding error).  OpenMP
// over rows.
void orc_rows_mult(int N, const uint32_t* states, int64_t D, const double* site_h, const double* site_d, int nb,
                   const int* s1, const int* s2, const double* jz, const double* jxy, const double* kq,
                   const double* x, int64_t r0, int64_t r1, double* y, double* yabs) {
  if (r1 > D) r1 = D;
  std::vector<BondTensor> bt(nb);
  for (int b = 0; b < nb; ++b) bt[b] = spin_bond(jz[b], jxy[b], kq ? kq[b] : 0.0);
#pragma omp parallel
  {
    std::vector<Entry> row;
#pragma omp for schedule(dynamic, 256)
    for (int64_t i = r0; i < r1; ++i) {
      row.clear();
      row_add(row, i, 1.0);
      row_add(row, i, -1.0);
      const uint32_t state = states[i];
      if (site_h || site_d) {
        for (int s = 0; s < N; ++s) {
          const double h = site_h ? site_h[s] : 0.0;
          const double dd = site_d ? site_d[s] : 0.0;
          const double mat[2] = {0.25 * dd + 0.5 * h, 0.25 * dd - 0.5 * h};
          const double v = mat[(state >> (N - 1 - s)) & 1];
          if (v != 0.0) row_add(row, i, v);
        }
      }
      for (int b = 0; b < nb; ++b) {
        const int b1 = N - 1 - s1[b], b2 = N - 1 - s2[b];
        const int is1 = (state >> b1) & 1, is2 = (state >> b2) & 1;
        for (int js1 = 0; js1 < 2; ++js1)
          for (int js2 = 0; js2 < 2; ++js2) {
            const double v = bt[b].m[is1][is2][js1][js2];
            if (v == 0.0) continue;
            uint32_t ns = state;
            ns = (ns & ~(1u << b1)) | ((uint32_t)js1 << b1);
            ns = (ns & ~(1u << b2)) | ((uint32_t)js2 << b2);
            const int64_t j = lb_index(states, D, ns);
            if (j < D) row_add(row, j, v);
          }
      }
      std::sort(row.begin(), row.end(), [](const Entry& a, const Entry& b) { return a.j < b.j; });
      double t = 0.0, ta = 0.0;
      for (auto& e : row) {
        t += e.v * x[e.j];
        ta += std::fabs(e.v * x[e.j]);
      }
      y[i - r0] = t;
      if (yabs) yabs[i - r0] = ta;
    }
  }
}

// orc_sample_times with all host threads: the rows [r0, r1) are dealt to the
// OpenMP threads in contiguous blocks; each thread builds its block's rows of
// the explicit matrix (reference element order, lower_bound lookups), then
// forms its rows of y = prod(M, x), then the make_step vector passes over as
// many elements.  Wall times of the three phases (each ends at a barrier).
void orc_sample_times_mt(int N, const uint32_t* states, int64_t D, int nb, const int* s1, const int* s2,
                         const double* jz, const double* jxy, int64_t r0, int64_t r1, double* t_build,
                         double* t_prod, double* t_vec) {
  using clk = std::chrono::steady_clock;
  if (r1 > D) r1 = D;
  const int64_t R = r1 - r0;
  std::vector<BondTensor> bt(nb);
  for (int b = 0; b < nb; ++b) bt[b] = spin_bond(jz[b], jxy[b], 0.0);
  std::vector<double> x(D), y(R);
  for (int64_t i = 0; i < D; ++i) x[i] = start_value(1, (uint64_t)i);
  double tb = 0, tp = 0, tv = 0, dot_total = 0.0;
#pragma omp parallel
  {
    int nt = 1, id = 0;
#ifdef _OPENMP
    nt = omp_get_num_threads();
    id = omp_get_thread_num();
#endif
    const int64_t a = r0 + R * id / nt, b = r0 + R * (id + 1) / nt;
    std::vector<int64_t> rp(b - a + 1, 0);
    std::vector<int32_t> col;
    std::vector<double> val;
    std::vector<Entry> row;
#pragma omp barrier
    clk::time_point t0 = clk::now();
    for (int64_t i = a; i < b; ++i) {
      row.clear();
      row_add(row, i, 1.0);
      row_add(row, i, -1.0);
      const uint32_t state = states[i];
      for (int q = 0; q < nb; ++q) {
        const int b1 = N - 1 - s1[q], b2 = N - 1 - s2[q];
        const int is1 = (state >> b1) & 1, is2 = (state >> b2) & 1;
        for (int js1 = 0; js1 < 2; ++js1)
          for (int js2 = 0; js2 < 2; ++js2) {
            const double v = bt[q].m[is1][is2][js1][js2];
            if (v == 0.0) continue;
            uint32_t ns = state;
            ns = (ns & ~(1u << b1)) | ((uint32_t)js1 << b1);
            ns = (ns & ~(1u << b2)) | ((uint32_t)js2 << b2);
            const int64_t j = lb_index(states, D, ns);
            if (j < D) row_add(row, j, v);
          }
      }
      std::sort(row.begin(), row.end(), [](const Entry& e1, const Entry& e2) { return e1.j < e2.j; });
      for (auto& e : row) {
        col.push_back((int32_t)e.j);
        val.push_back(e.v);
      }
      rp[i - a + 1] = (int64_t)col.size();
    }
#pragma omp barrier
    clk::time_point t1 = clk::now();
    for (int64_t i = a; i < b; ++i) {
      double t = 0.0;
      for (int64_t p = rp[i - a]; p < rp[i - a + 1]; ++p) t += val[p] * x[col[p]];
      y[i - r0] = t;
    }
#pragma omp barrier
    clk::time_point t2 = clk::now();
    // make_step's vector passes over this thread's elements (dot, two axpy, norm, divide)
    double dd = 0.0;
    for (int64_t i = a; i < b; ++i) dd += x[i] * y[i - r0];
#pragma omp atomic
    dot_total += dd;
#pragma omp barrier
    const double al = dot_total;
    double nn = 0.0;
    for (int64_t i = a; i < b; ++i) {
      y[i - r0] -= al * x[i];
      y[i - r0] -= 0.3 * x[i];
      nn += y[i - r0] * y[i - r0];
    }
    for (int64_t i = a; i < b; ++i) y[i - r0] /= (nn + 1.0);
#pragma omp barrier
    clk::time_point t3 = clk::now();
#pragma omp single
    {
      tb = std::chrono::duration<double>(t1 - t0).count();
      tp = std::chrono::duration<double>(t2 - t1).count();
      tv = std::chrono::duration<double>(t3 - t2).count();
    }
  }
  *t_build = tb;
  *t_prod = tp;
  *t_vec = tv;
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
