// lanczos.cpp -- the Lanczos drivers behind aed_solve.
//
// FP64 path (the drop-in): ietl::lanczos::calculate_eigenvalues with
// lanczos_iteration_nlowest (src/ietl/lanczos.h:341-406,
// src/ietl/iteration.h:66-130) and Tmatrix::compute's distinct / ghost rules
// (src/ietl/tmatrix.h:121-228), as SparseDiagMatrix::do_subspace drives it
// (applications/diag/sparsediag/sparsediag.h:104-118).  Each step is three
// kernels on the handle's stream (apply + alpha partials, update + |w|^2
// partials, normalise); alpha_j and beta_j stay on the device, so the GPU
// never waits for the host.  The host analyses T of size m while the GPU
// already runs step m+1; when T(m) has converged that extra step is
// discarded, so the result is the one the reference's loop stops at.
//
// Mixed path (AED_FP32 handles): the same recurrence with FP32 vectors
// (half the bytes per apply) kept in HBM as a Lanczos basis, run until the
// Ritz residual estimates reach the FP32 level; the Ritz vectors are then
// assembled in FP64 from the stored basis and a short FP64 Lanczos run
// started from them refines the eigenvalues until the residual bound
// r^2 / gap on each eigenvalue is below 1e-11 |lambda|.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

#include "handle.h"
#include "tmatrix_core.h"

namespace aed {
namespace {

struct DevMem {
  void* p = nullptr;
  ~DevMem() {
    if (p) cudaFree(p);
  }
  int alloc(size_t bytes) {
    const cudaError_t e = cudaMalloc(&p, bytes ? bytes : 8);
    if (e != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      return fail(AED_ERR_NOMEM, std::string("device allocation of ") + std::to_string(bytes) +
                                     " bytes failed: " + cudaGetErrorString(e));
    }
    return AED_OK;
  }
};

struct HostPinned {
  double* p = nullptr;
  ~HostPinned() {
    if (p) cudaFreeHost(p);
  }
  int alloc(size_t n) {
    if (cudaMallocHost((void**)&p, n * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      return fail(AED_ERR_NOMEM, "pinned host allocation failed");
    }
    return AED_OK;
  }
};

struct EventRing {
  static constexpr int kN = 4;
  cudaEvent_t ev[kN] = {};
  ~EventRing() {
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
  }
  int init() {
    for (auto& e : ev)
      if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return fail(AED_ERR_CUDA, "event");
    return AED_OK;
  }
};

// Diagonal element of a single-state sector: sparsediag takes matrix()(0,0)
// directly when the dimension is 1 (sparsediag.h:120-124).
double diag_of_state(const HvParams& P, uint32_t s) {
  double d = 0.0;
  for (int q = 0; q < P.n_diag; ++q) {
    const bool eq = ((s & P.diag[q].m1) != 0u) == ((s & P.diag[q].m2) != 0u);
    d += eq ? P.diag[q].veq : P.diag[q].vne;
  }
  return d;
}

// After the apply x -> y (per-tile partials in h->d_partA): alpha, update,
// beta, normalise (lanczos.h:398-402).
int lanczos_step_tail(aed_handle* h, bool f32, const void* vprev, const void* x, void* y, const double* beta_prev,
                      double* alpha, double* beta) {
  const int64_t D = h->tab.D;
  int rc = launch_finish_sum(h->d_partA, h->dt.n_tiles, alpha, false, h->stream);
  if (rc) return rc;
  if (f32)
    rc = launch_lanczos_update(alpha, (const float*)x, (const float*)vprev, beta_prev, (float*)y, D, h->d_partB,
                               h->stream);
  else
    rc = launch_lanczos_update(alpha, (const double*)x, (const double*)vprev, beta_prev, (double*)y, D, h->d_partB,
                               h->stream);
  if (!rc) rc = launch_finish_sum(h->d_partB, red_chunks(D), beta, true, h->stream);
  if (rc) return rc;
  if (f32) return launch_lanczos_normalize(beta, (float*)y, D, h->stream);
  return launch_lanczos_normalize(beta, (double*)y, D, h->stream);
}

// One Lanczos recurrence on device vectors of type T.  Vectors rotate through
// `slot(j)`, the buffer that receives v_j.  Returns T-matrix and convergence.
struct Recurrence {
  aed_handle* h;
  bool f32;
  int64_t D;
  int max_iter;
  double* d_ab;      // device alpha/beta pairs: d_ab[2j] = alpha_j, d_ab[2j+1] = beta_j
  double* h_ab;      // pinned host copy
  EventRing* ring;
  std::vector<double> alpha, beta;
  double amax = 0, bmax = 0;
  bool profile = false;
  std::vector<cudaEvent_t> tev;  // (start, stop) per apply when profiling

  ~Recurrence() {
    for (auto e : tev) cudaEventDestroy(e);
  }

  // mean device time of the applies, ms (profiling only)
  double apply_ms() {
    if (tev.empty()) return 0.0;
    double tot = 0.0;
    for (size_t k = 0; k + 1 < tev.size(); k += 2) {
      float t = 0.f;
      cudaEventElapsedTime(&t, tev[k], tev[k + 1]);
      tot += t;
    }
    return tot / (double)(tev.size() / 2);
  }

  // launch step j: x = v_j -> y = v_{j+1}; vprev = v_{j-1} (NULL for j = 0)
  int launch_step(int j, const void* vprev, const void* x, void* y) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (profile) {
      // the first apply may autotune; keep those launches out of the timing
      const int rt = handle_tune(h, f32, x, y);
      if (rt) return rt;
      AED_CUDA_TRY(cudaEventCreate(&e0));
      AED_CUDA_TRY(cudaEventCreate(&e1));
      tev.push_back(e0);
      tev.push_back(e1);
      AED_CUDA_TRY(cudaEventRecord(e0, h->stream));
    }
    int rc = handle_hv(h, f32, x, y, h->d_partA);
    if (rc) return rc;
    if (profile) AED_CUDA_TRY(cudaEventRecord(e1, h->stream));
    const double* bprev = j > 0 ? d_ab + 2 * (j - 1) + 1 : nullptr;
    rc = lanczos_step_tail(h, f32, vprev, x, y, bprev, d_ab + 2 * j, d_ab + 2 * j + 1);
    if (rc) return rc;
    AED_CUDA_TRY(cudaMemcpyAsync(h_ab + 2 * j, d_ab + 2 * j, 16, cudaMemcpyDeviceToHost, h->stream));
    AED_CUDA_TRY(cudaEventRecord(ring->ev[j % EventRing::kN], h->stream));
    return AED_OK;
  }

  int wait_step(int j) {
    AED_CUDA_TRY(cudaEventSynchronize(ring->ev[j % EventRing::kN]));
    const double a = h_ab[2 * j], b = h_ab[2 * j + 1];
    alpha.push_back(a);
    beta.push_back(b);
    if (alpha.size() == 1) {
      amax = a;
      bmax = b;
    } else {
      amax = std::max(amax, a);
      bmax = std::max(bmax, b);
    }
    return AED_OK;
  }
};

// normalise v in place (lanczos.h:383): v /= |v|
template <typename T>
int normalize(aed_handle* h, T* v, int64_t D) {
  int rc = launch_dot_partials(v, v, D, h->d_partB, true, h->stream);
  if (!rc) rc = launch_finish_sum(h->d_partB, red_chunks(D), h->d_scal + 7, true, h->stream);
  if (!rc) rc = launch_lanczos_normalize(h->d_scal + 7, v, D, h->stream);
  return rc;
}

// Stopping rule of one recurrence.
struct StopRule {
  int nev;
  double rtol, atol;    // ietl rule: err_i <= max(atol, rtol |lambda_i|)
  bool energy_bound;    // mixed refinement: err_i^2 / gap_i <= etol |lambda_i|
  double etol;
  int min_steps;
  bool done(const TmatInfo& t, int m) const {
    if (m < min_steps) return false;
    if (nlowest_converged(t, nev, rtol, atol)) return true;
    if (!energy_bound || (int)t.evals.size() < nev + 1) return false;
    for (int i = 0; i < nev; ++i) {
      const double gap = t.evals[i + 1] - t.evals[i];
      if (!(gap > 0)) return false;
      const double r = t.errs[i];
      if (!(r * r / gap <= etol * std::max(std::fabs(t.evals[i]), 1e-300))) return false;
    }
    return true;
  }
};

// Run a recurrence over rotating vector slots.  `slots(j)` gives the buffer
// of v_j (v_0 already holds the normalised start vector).
template <typename SlotFn>
int run_recurrence(Recurrence& R, const StopRule& stop, SlotFn slot, int* iters, int* failed, TmatInfo& T) {
  int launched = 0;
  int m = 1;
  *failed = 0;
  void* s0 = slot(0);
  void* s1 = slot(1);
  if (!s0 || !s1) return AED_ERR_NOMEM;
  int rc = R.launch_step(0, nullptr, s0, s1);
  if (rc) return rc;
  launched = 1;
  while (true) {
    // keep the device one step ahead of the host analysis
    while (launched < m + 1 && launched < R.max_iter) {
      void* a = slot(launched - 1);
      void* b = slot(launched);
      void* c = slot(launched + 1);
      if (!a || !b || !c) return AED_ERR_NOMEM;
      rc = R.launch_step(launched, a, b, c);
      if (rc) return rc;
      ++launched;
    }
    rc = R.wait_step(m - 1);
    if (rc) return rc;
    if (m > 1) {
      rc = tmatrix_analyze(m, R.alpha.data(), R.beta.data(), R.amax, R.bmax, T, R.f32 ? kFp32MergeRel : 0.0);
      if (rc) return rc;
      if (stop.done(T, m)) break;
    }
    if (m >= R.max_iter) {
      *failed = 1;
      break;
    }
    ++m;
  }
  if (m == 1) {
    rc = tmatrix_analyze(1, R.alpha.data(), R.beta.data(), R.amax, R.bmax, T, R.f32 ? kFp32MergeRel : 0.0);
    if (rc) return rc;
  }
  AED_CUDA_TRY(cudaStreamSynchronize(R.h->stream));
  *iters = m;
  return AED_OK;
}

int solve_fp64(aed_handle* h, const double* start_host, const double* start_dev, uint64_t seed, int nev,
               int max_iter, double rtol, double atol, bool energy_bound, double etol, int min_steps, bool profile,
               aed_solve_result* r, TmatInfo& T) {
  const int64_t D = h->tab.D;
  EventRing ring;
  int rc;
  // workspace: three rotating vectors + the alpha/beta pairs
  const size_t vb = ((size_t)D * 8 + 255) & ~(size_t)255;
  void* ws = nullptr;
  double* hab = nullptr;
  if ((rc = handle_workspace(h, 0, 3 * vb + (size_t)2 * (max_iter + 2) * 8, &ws)) ||
      (rc = handle_pinned(h, (size_t)2 * (max_iter + 2), &hab)) || (rc = ring.init()))
    return rc;
  void* buf[3] = {ws, (char*)ws + vb, (char*)ws + 2 * vb};
  double* d_ab = (double*)((char*)ws + 3 * vb);
  double* v0 = (double*)buf[0];
  if (start_dev) {
    AED_CUDA_TRY(cudaMemcpyAsync(v0, start_dev, D * 8, cudaMemcpyDeviceToDevice, h->stream));
  } else if (start_host) {
    AED_CUDA_TRY(cudaMemcpyAsync(v0, start_host, D * 8, cudaMemcpyHostToDevice, h->stream));
  } else if ((rc = launch_fill_random(v0, D, seed, h->stream))) {
    return rc;
  }
  if ((rc = normalize(h, v0, D))) return rc;
  Recurrence R{h, false, D, max_iter, d_ab, hab, &ring, {}, {}, 0, 0, profile, {}};
  StopRule stop{nev, rtol, atol, energy_bound, etol, min_steps};
  int iters = 0, failed = 0;
  rc = run_recurrence(R, stop, [&](int j) { return buf[j % 3]; }, &iters, &failed, T);
  if (rc) return rc;
  const int n = std::min(nev, (int)T.evals.size());
  r->n_evals = n;
  for (int i = 0; i < n; ++i) {
    r->evals[i] = T.evals[i];
    r->errors[i] = T.errs[i];
  }
  r->iterations = iters;
  r->converged = failed ? 0 : 1;
  if (profile) r->apply_ms = R.apply_ms();
  h->last_alpha = R.alpha;
  h->last_beta = R.beta;
  return AED_OK;
}

// Refinement stop: residual bound r^2 / gap <= kRefineEnergyTol * |lambda| on
// every requested eigenvalue (Kato-Temple), 100x inside the 1e-9 relative
// energy agreement the mixed path promises.
constexpr double kRefineEnergyTol = 1e-11;

// FP32 phase with the Lanczos basis stored in HBM, then FP64 refinement.
int solve_mixed(aed_handle* h, const double* start_host, uint64_t seed, int nev, int max_iter, double rtol,
                double atol, bool profile, aed_solve_result* r) {
  const int64_t D = h->tab.D;
  // Lanczos basis store: chunks of kStoreChunk FP32 vectors, grown as the
  // recurrence advances and kept by the handle for later solves
  const size_t vbytes = (((size_t)D * 4 + 255) & ~(size_t)255);
  const int64_t ldv = (int64_t)(vbytes / 4);  // stride of the stored vectors (256-byte aligned)
  const size_t chunk_bytes = vbytes * kStoreChunk;
  const int cap = std::min(max_iter + 1, kMaxRitzTerms);
  HostPinned hab;
  EventRing ring;
  DevMem small;  // start64 | alpha/beta pairs | Ritz coefficients
  int rc;
  const size_t s64 = (((size_t)D * 8 + 255) & ~(size_t)255);
  const size_t ab_bytes = (((size_t)2 * (cap + 2) * 8 + 255) & ~(size_t)255);
  if ((rc = small.alloc(s64 + ab_bytes + (size_t)kStoreChunk * 8)) || (rc = hab.alloc((size_t)2 * (cap + 2))) ||
      (rc = ring.init()))
    return rc;
  double* start64 = (double*)small.p;
  double* d_ab = (double*)((char*)small.p + s64);
  double* coef = (double*)((char*)small.p + s64 + ab_bytes);
  bool oom = false;
  auto slot = [&](int j) -> void* {
    char* c = (char*)handle_store_chunk(h, j / kStoreChunk, chunk_bytes);
    if (!c) {
      oom = true;
      return nullptr;
    }
    return c + (size_t)(j % kStoreChunk) * vbytes;
  };
  float* V0 = (float*)slot(0);
  if (!V0) return AED_ERR_NOMEM;
  if (start_host) {
    std::vector<float> tmp(D);
    for (int64_t i = 0; i < D; ++i) tmp[i] = (float)start_host[i];
    AED_CUDA_TRY(cudaMemcpyAsync(V0, tmp.data(), (size_t)D * 4, cudaMemcpyHostToDevice, h->stream));
    AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
  } else if ((rc = launch_fill_random(V0, D, seed, h->stream))) {
    return rc;
  }
  if ((rc = normalize(h, V0, D))) return rc;
  // phase 1: FP32 vectors, stop at FP32-level residual estimates
  Recurrence R{h, true, D, cap - 1, d_ab, hab.p, &ring, {}, {}, 0, 0, profile, {}};
  const double tol32 = 2e-6;
  StopRule stop1{nev, tol32, tol32 * 1e-3, false, 0.0, 2};
  TmatInfo T1;
  int it1 = 0, failed1 = 0;
  rc = run_recurrence(R, stop1, slot, &it1, &failed1, T1);
  if (oom) return AED_ERR_NOMEM;
  if (rc) return rc;
  const int m1 = it1;
  const int n1 = std::min(nev, (int)T1.evals.size());
  for (int i = 0; i < n1; ++i) r->evals_low[i] = T1.evals[i];
  r->iterations_low = m1;
  const double apply32_ms = profile ? R.apply_ms() : 0.0;
  // Ritz start: the eigenvectors of T(m1) up to the end of the (nev+1)-th
  // distinct cluster with seeded weights (tcore::ritz_span / ritz_weight),
  // accumulated in FP64 chunk by chunk from the stored basis
  std::vector<double> ev(R.alpha.begin(), R.alpha.begin() + m1), e(m1 + 1, 0.0), Z((size_t)m1 * m1);
  for (int i = 0; i + 1 < m1; ++i) e[i] = R.beta[i];
  if (tridiag_eigen(m1, ev.data(), e.data(), nullptr, Z.data())) return fail(AED_ERR_TRIDIAG, "tridiagonal eigensolver failed");
  const int K = tcore::ritz_span((int)T1.evals.size(), nev, T1.first.data(), T1.mults.data(), m1);
  std::vector<double> c(m1, 0.0);
  for (int k = 0; k < K; ++k) {
    const double w = tcore::ritz_weight(seed, k);
    for (int j = 0; j < m1; ++j) c[j] += w * Z[(size_t)k * m1 + j];
  }
  for (int j0 = 0; j0 < m1; j0 += kStoreChunk) {
    const int cnt = std::min(kStoreChunk, m1 - j0);
    AED_CUDA_TRY(cudaMemcpyAsync(coef, c.data() + j0, cnt * 8, cudaMemcpyHostToDevice, h->stream));
    if ((rc = launch_ritz_combine((const float*)slot(j0), ldv, cnt, coef, start64, D, j0 > 0, h->stream))) return rc;
    // the coefficient buffer is reused by the next chunk: order the host copy after this kernel
    AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
  }
  // phase 2: FP64 refinement from the Ritz combination
  TmatInfo T2;
  const int max2 = std::max(max_iter, nev + 4);
  rc = solve_fp64(h, nullptr, start64, seed, nev, max2, rtol, atol, true, kRefineEnergyTol, nev + 2, false, r, T2);
  // apply_ms of a mixed solve: the FP32 applies (the bulk of the work)
  if (profile) r->apply_ms = apply32_ms;
  return rc;
}

}  // namespace

int lanczos_step_kernels(aed_handle* h, bool f32, const void* v_prev, const void* v_cur, void* v_next,
                         const double* beta_prev, double* alpha, double* beta) {
  int rc = handle_hv(h, f32, v_cur, v_next, h->d_partA);
  if (rc) return rc;
  return lanczos_step_tail(h, f32, v_prev, v_cur, v_next, v_prev ? beta_prev : nullptr, alpha, beta);
}

int solve(aed_handle* h, const aed_solve_opts* o, aed_solve_result* r) {
  std::memset(r, 0, sizeof *r);
  const auto t0 = std::chrono::steady_clock::now();
  const int64_t D = h->tab.D;
  const int nev = o->nev;
  if (nev < 1 || nev > AED_MAX_NEV) return fail(AED_ERR_INVALID, "nev must be in 1..16");
  if (o->max_iter < 0) return fail(AED_ERR_INVALID, "max_iter must be >= 0");
  int rc = AED_OK;
  if (D == 0) {
    r->converged = 1;
  } else if (D == 1) {
    uint32_t s = 0;
    std::vector<uint32_t> st(1);
    DevMem d;
    if ((rc = d.alloc(4))) return rc;
    if ((rc = launch_basis_copy(h->dt, (uint32_t*)d.p, 0, 1, h->stream))) return rc;
    AED_CUDA_TRY(cudaMemcpyAsync(&s, d.p, 4, cudaMemcpyDeviceToHost, h->stream));
    AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
    r->n_evals = 1;
    r->evals[0] = diag_of_state(h->P, s);
    r->converged = 1;
  } else {
    const int max_iter = o->max_iter > 0 ? o->max_iter : (int)std::min<int64_t>(10 * D, 1000);
    const double eps = 2.220446049250313e-16;
    const double rtol = o->rtol > 0 ? o->rtol : 100 * eps;
    const double atol = o->atol > 0 ? o->atol : 100 * eps;
    if (h->precision == AED_FP32 && o->refine != -1) {
      rc = solve_mixed(h, o->start, o->seed, nev, max_iter, rtol, atol, o->profile != 0, r);
    } else {
      TmatInfo T;
      rc = solve_fp64(h, o->start, nullptr, o->seed, nev, max_iter, rtol, atol, false, 0.0, 0, o->profile != 0, r, T);
    }
  }
  r->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return rc;
}

}  // namespace aed
