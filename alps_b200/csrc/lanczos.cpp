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
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <functional>
#include <future>
#include <mutex>
#include <thread>
#include <vector>

#include "handle.h"
#include "rr_core.h"
#include "tmatrix_core.h"

namespace aed {

size_t rr_workspace_bytes(int64_t D, int K) {
  const size_t vb = ((size_t)D * 8 + 255) & ~(size_t)255;
  const int np = K * (K + 1) / 2 + K * K;
  const size_t part_bytes = (((size_t)np * red_chunks(D) * 8) + 255) & ~(size_t)255;
  constexpr int kMaxSums = kMaxRR * (kMaxRR + 1) / 2 + kMaxRR * kMaxRR;
  return 2 * (size_t)K * vb + part_bytes + (size_t)kMaxSums * 8;
}

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

// Host threads for the T-matrix analyses of the recurrences (shared by all
// handles and server lanes of the process; started on first use).  A small
// sector's step takes the GPU microseconds while the analysis of T(m) takes
// O(m^2) host time, so the analyses of several sizes run side by side.
class AnalysisPool {
 public:
  static AnalysisPool& get() {
    static AnalysisPool pool;
    return pool;
  }
  int threads() const { return (int)th_.size(); }
  template <typename F>
  auto submit(F f) -> std::future<decltype(f())> {
    auto task = std::make_shared<std::packaged_task<decltype(f())()>>(std::move(f));
    auto fut = task->get_future();
    {
      std::lock_guard<std::mutex> lk(mu_);
      q_.emplace_back([task] { (*task)(); });
    }
    cv_.notify_one();
    return fut;
  }

 private:
  AnalysisPool() {
    const unsigned hc = std::thread::hardware_concurrency();
    const int n = (int)std::max(2u, std::min(hc ? hc : 2u, 16u));
    for (int i = 0; i < n; ++i) th_.emplace_back([this] { work(); });
  }
  ~AnalysisPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }
  void work() {
    while (true) {
      std::function<void()> job;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [this] { return stop_ || !q_.empty(); });
        if (q_.empty()) return;
        job = std::move(q_.front());
        q_.pop_front();
      }
      job();
    }
  }
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<std::function<void()>> q_;
  std::vector<std::thread> th_;
  bool stop_ = false;
};

struct EventRing {
  static constexpr int kN = 16;  // > the largest lookahead + 1
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
  const int64_t D = h->vlen;
  const int64_t na = h->alpha_tiles(), nb = red_chunks(D);
  // AED_FOLD_FINISH=0 keeps the separate finishing kernels (a test compares
  // the two paths bit for bit)
  static const bool fold = [] {
    const char* e = std::getenv("AED_FOLD_FINISH");
    return !(e && e[0] == '0');
  }();
  if (fold && na <= kFoldFinishMax && nb <= kFoldFinishMax) {
    // short partial lists: the finishing sums inside the update and the
    // normalisation (same alpha and beta to the bit, two launches fewer)
    int rc;
    if (f32)
      rc = launch_lanczos_update_fin(h->d_partA, na, alpha, (const float*)x, (const float*)vprev, beta_prev,
                                     (float*)y, D, h->d_partB, h->stream);
    else
      rc = launch_lanczos_update_fin(h->d_partA, na, alpha, (const double*)x, (const double*)vprev, beta_prev,
                                     (double*)y, D, h->d_partB, h->stream);
    if (rc) return rc;
    if (f32) return launch_lanczos_normalize_fin(h->d_partB, nb, beta, (float*)y, D, h->stream);
    return launch_lanczos_normalize_fin(h->d_partB, nb, beta, (double*)y, D, h->stream);
  }
  int rc = launch_finish_sum(h->d_partA, h->alpha_tiles(), alpha, false, h->stream);
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

// Steps the device runs ahead of the host's T-matrix analysis.  A step of a
// large sector keeps the GPU busy longer than the analysis takes, so one step
// ahead suffices; for mid-size sectors (fewer than 2^24 vector scalars: the
// momentum sectors, chains up to L = 26) three hide the analysis and the
// launch latency; below 2^20 scalars a step takes the GPU a few microseconds
// and the O(m^2) analyses set the pace, so ten run side by side.  The steps
// launched past the stop are discarded.  The recurrence vectors rotate
// through lookahead + 2 slots, so that v_{m-1} and v_m survive the extra
// steps (resume, checkpoint).
constexpr int kMaxRing = 12;
inline int lanczos_lookahead(const aed_handle* h) {
  if (h->vlen >= ((int64_t)1 << 24)) return 1;
  if (h->vlen >= ((int64_t)1 << 20)) return 3;
  return std::min(10, AnalysisPool::get().threads());
}
inline int ring_slots(const aed_handle* h) { return lanczos_lookahead(h) + 2; }

// Full reorthogonalisation of an FP32 recurrence whose vectors v_0 .. v_j are
// kept in the FP32 store (chunks of kStoreChunk vectors, stride ldv): after
// the update, w -= V (V^T w) twice (classical Gram-Schmidt with one repeat,
// Daniel, Gragg, Kaufman & Stewart, Math. Comp. 30 (1976) 772-795), the dots
// and the combination accumulated in FP64, w rounded to FP32 once per pass;
// the T-matrix keeps the recurrence's alpha and beta.  All on the device.
struct Reorth {
  bool on = false;
  std::function<void*(int)> vec;  // v_j in the store
  int64_t ldv = 0;
  double* part = nullptr;  // (cap) x red_chunks(D) chunk partials
  double* coef = nullptr;  // cap coefficients
  double* tmp = nullptr;   // D doubles: V c
  int cap = 0;
};

int reorthogonalise(aed_handle* h, const Reorth& ro, int j, float* w) {
  const int64_t D = h->vlen, nch = red_chunks(D);
  const int m = j + 1;  // against v_0 .. v_j
  if (m > ro.cap) return fail(AED_ERR_INVALID, "reorthogonalisation: more vectors than the store holds");
  int rc = AED_OK;
  for (int pass = 0; pass < 2 && !rc; ++pass) {
    for (int k0 = 0; k0 < m && !rc; k0 += kStoreChunk)
      rc = launch_block_dot((const float*)ro.vec(k0), ro.ldv, std::min(kStoreChunk, m - k0), w, D, ro.part, k0,
                            h->stream);
    if (!rc) rc = launch_finish_many(ro.part, nch, m, ro.coef, h->stream);
    for (int k0 = 0; k0 < m && !rc; k0 += kStoreChunk)
      rc = launch_ritz_combine((const float*)ro.vec(k0), ro.ldv, std::min(kStoreChunk, m - k0), ro.coef + k0, ro.tmp,
                               D, k0 > 0, h->stream);
    if (!rc) rc = launch_sub_round(ro.tmp, w, D, h->stream);
  }
  return rc;
}

// One Lanczos recurrence on device vectors of type T.  Vectors rotate through
// `slot(j)`, the buffer that receives v_j.  Returns T-matrix and convergence.
struct Recurrence {
  aed_handle* h;
  bool f32;
  int64_t D;
  int max_iter;
  int ahead;         // steps launched ahead of the host analysis
  double* d_ab;      // device alpha/beta pairs: d_ab[2j] = alpha_j, d_ab[2j+1] = beta_j
  double* h_ab;      // pinned host copy
  EventRing* ring;
  std::vector<double> alpha, beta;
  double amax = 0, bmax = 0;
  bool profile = false;
  std::vector<cudaEvent_t> tev;  // (start, stop) per apply when profiling
  const Reorth* reorth = nullptr;  // FP32 recurrences over the store: full reorthogonalisation

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
    if (reorth && reorth->on && f32) {
      // update, then w -= V V^T w, then beta = |w| and the normalisation (lanczos.h:398-402)
      double* alpha = d_ab + 2 * j;
      double* beta = d_ab + 2 * j + 1;
      rc = launch_finish_sum(h->d_partA, h->alpha_tiles(), alpha, false, h->stream);
      if (!rc) rc = launch_lanczos_update(alpha, (const float*)x, (const float*)vprev, bprev, (float*)y, D,
                                          h->d_partB, h->stream);
      if (!rc) rc = reorthogonalise(h, *reorth, j, (float*)y);
      if (!rc) rc = launch_dot_partials((const float*)y, (const float*)y, D, h->d_partB, true, h->stream);
      if (!rc) rc = launch_finish_sum(h->d_partB, red_chunks(D), beta, true, h->stream);
      if (!rc) rc = launch_lanczos_normalize(beta, (float*)y, D, h->stream);
    } else {
      rc = lanczos_step_tail(h, f32, vprev, x, y, bprev, d_ab + 2 * j, d_ab + 2 * j + 1);
    }
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

// Rayleigh-Ritz acceptance: every reported value's error bound below
// kRRTol * |theta|, 2x inside the 1e-9 relative agreement (the bound is
// rigorous: the FP64 values lie within it).
constexpr double kRRTol = 5e-10;

// Stopping rule of one recurrence.
struct StopRule {
  int nev;
  double rtol, atol;    // ietl rule: err_i <= max(atol, rtol |lambda_i|)
  bool energy_bound;    // mixed refinement: err_i^2 / gap_i <= etol |lambda_i|
  double etol;
  int min_steps;
  // mixed refinement, block Kato-Temple stop: sum_i err_i^2 / (next_lo -
  // lambda_{nev-1}) <= block_tol |lambda_i|, next_lo a lower bound on the
  // eigenvalue above the nev lowest from the FP32 phase (block_tol 0: off)
  double next_lo = -1e300, block_tol = 0.0;
  bool done(const TmatInfo& t, int m) const {
    if (m < min_steps) return false;
    if (nlowest_converged(t, nev, rtol, atol)) return true;
    if (block_tol > 0.0 && (int)t.evals.size() >= nev && next_lo > t.evals[nev - 1]) {
      double r2 = 0.0;
      for (int i = 0; i < nev; ++i) r2 += t.errs[i] * t.errs[i];
      bool ok = true;
      for (int i = 0; ok && i < nev; ++i)
        ok = r2 / (next_lo - t.evals[nev - 1]) <= block_tol * std::fabs(t.evals[i]);
      if (ok) return true;
    }
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
// of v_j.  m0 = 0: v_0 holds the normalised start vector.  m0 > 0 (resumed
// run): R.alpha / R.beta and the device pairs hold steps 0 .. m0-1 and the
// slots of v_{m0-1} and v_{m0} hold those vectors; T(m0) is tested first.
template <typename SlotFn>
int run_recurrence(Recurrence& R, const StopRule& stop, SlotFn slot, int m0, int* iters, int* failed,
                   TmatInfo& T) {
  // T(m) is analysed for every m in turn, as the reference's iteration does
  // (lanczos.h:366-372); with R.ahead > 1 the analyses of the next R.ahead
  // sizes run on host threads side by side (each is independent of the
  // others' outcome) and their verdicts are read in order.
  const double thold = R.f32 ? kFp32MergeRel : 0.0;
  // alpha / beta keep their storage while later steps append (capacity
  // max_iter + 1); the maxima are taken over the first m pairs at submission
  R.alpha.reserve((size_t)R.max_iter + 1);
  R.beta.reserve((size_t)R.max_iter + 1);
  const double* pa = R.alpha.data();
  const double* pb = R.beta.data();
  auto analysis = [pa, pb, thold](int m, double amax, double bmax) {
    std::pair<int, TmatInfo> out;
    out.first = tmatrix_analyze(m, pa, pb, amax, bmax, out.second, thold);
    return out;
  };
  int launched = 0;
  *failed = 0;
  int rc = AED_OK;
  if (m0 == 0) {
    void* s0 = slot(0);
    void* s1 = slot(1);
    if (!s0 || !s1) return AED_ERR_NOMEM;
    rc = R.launch_step(0, nullptr, s0, s1);
    if (rc) return rc;
    launched = 1;
  } else {
    launched = m0;
  }
  const int par = R.ahead;
  std::deque<std::future<std::pair<int, TmatInfo>>> pending;  // analyses of T(check), T(check + 1), ...
  // the pool's tasks read alpha / beta: every return waits for them first
  struct Drain {
    std::deque<std::future<std::pair<int, TmatInfo>>>& d;
    ~Drain() {
      for (auto& f : d)
        if (f.valid()) f.wait();
    }
  } drain{pending};
  int check = m0 == 0 ? 1 : m0;  // the T size whose verdict comes next
  int submit = check;            // the next T size to analyse
  int m = check;
  // beta_{j} = 0 exactly: the Krylov space is invariant, T(j + 1) holds exact
  // eigenvalues and the next vector would be 0/0; the recurrence stops there
  // (ietl divides by it regardless; an H with no off-diagonal coupling to the
  // start vector's complement is the usual case)
  int invariant_m = 0;
  while (true) {
    // keep the device R.ahead steps ahead of the verdicts
    while (launched < check + R.ahead && launched < R.max_iter) {
      void* a = slot(launched - 1);
      void* b = slot(launched);
      void* c = slot(launched + 1);
      if (!a || !b || !c) return AED_ERR_NOMEM;
      rc = R.launch_step(launched, a, b, c);
      if (rc) return rc;
      ++launched;
    }
    // analyses of the sizes whose recurrence coefficients are in
    while (submit < check + par && submit <= R.max_iter && submit <= launched) {
      if (submit > m0) {
        rc = R.wait_step(submit - 1);
        if (rc) return rc;
        if (!invariant_m && R.beta.back() == 0.0) invariant_m = submit;
      }
      if (submit > 1) {
        if (par > 1) {
          const double am = R.amax, bm = R.bmax;
          const int ms = submit;
          pending.push_back(AnalysisPool::get().submit([analysis, ms, am, bm] { return analysis(ms, am, bm); }));
        } else {
          pending.push_back(std::async(std::launch::deferred, analysis, submit, R.amax, R.bmax));
        }
      } else {
        std::promise<std::pair<int, TmatInfo>> none;
        none.set_value({AED_OK, TmatInfo()});
        pending.push_back(none.get_future());
      }
      ++submit;
    }
    m = check;
    std::pair<int, TmatInfo> v = pending.front().get();
    pending.pop_front();
    if (v.first) return v.first;
    if (m > 1) {
      T = std::move(v.second);
      if (stop.done(T, m)) break;
    }
    if (m == invariant_m) break;  // exact: every value of T(m) is an eigenvalue
    if (m >= R.max_iter) {
      *failed = 1;
      break;
    }
    ++check;
  }
  for (auto& f : pending) f.wait();  // analyses of sizes past the stop: discarded
  if (m == 1) {
    rc = tmatrix_analyze(1, R.alpha.data(), R.beta.data(), R.amax, R.bmax, T, thold);
    if (rc) return rc;
  }
  AED_CUDA_TRY(cudaStreamSynchronize(R.h->stream));
  *iters = m;
  return AED_OK;
}

// The three rotating FP64 vectors of the recurrence in workspace slot 0.
int recurrence_buffers(aed_handle* h, void* buf[kMaxRing]) {
  const size_t vb = ((size_t)h->vlen * 8 + 255) & ~(size_t)255;
  const int nr = ring_slots(h);
  void* ws = nullptr;
  const int rc = handle_workspace(h, 0, (size_t)nr * vb, &ws);
  if (rc) return rc;
  for (int q = 0; q < nr; ++q) buf[q] = (char*)ws + q * vb;
  return AED_OK;
}

// v_0 of a recurrence: copied from the device or the host, else seeded; normalised.
int start_vector(aed_handle* h, const double* start_host, const double* start_dev, uint64_t seed, double* v0) {
  const int64_t D = h->vlen;
  int rc;
  if (start_dev) {
    AED_CUDA_TRY(cudaMemcpyAsync(v0, start_dev, D * 8, cudaMemcpyDeviceToDevice, h->stream));
  } else if (start_host) {
    AED_CUDA_TRY(cudaMemcpyAsync(v0, start_host, D * 8, cudaMemcpyHostToDevice, h->stream));
  } else if ((rc = launch_fill_random(v0, D, seed, h->stream))) {
    return rc;
  }
  return normalize(h, v0, D);
}

// FP64 Lanczos (lanczos.h:341-406 with lanczos_iteration_nlowest).  resume:
// continue the handle's live recurrence (last_alpha / last_beta, v_{m-1}, v_m)
// instead of starting from a vector, like ietl's more_eigenvalues
// (lanczos.h:77-78) after a load (lanczos.h:86-98).
int solve_fp64(aed_handle* h, const double* start_host, const double* start_dev, uint64_t seed, int nev,
               int max_iter, double rtol, double atol, bool energy_bound, double etol, int min_steps, bool profile,
               aed_solve_result* r, TmatInfo& T, bool resume = false, double next_lo = -1e300) {
  const int64_t D = h->vlen;
  EventRing ring;
  int rc;
  const int m0 = resume ? h->rec_m : 0;
  if (resume && (!h->rec_live || m0 < 1 || (int)h->last_alpha.size() != m0))
    return fail(AED_ERR_INVALID, "no live Lanczos recurrence to resume (solve or aed_lanczos_load first)");
  if (m0 >= max_iter) max_iter = m0 + 1;
  void* buf[kMaxRing];
  void* ab = nullptr;  // device alpha/beta pairs
  double* hab = nullptr;
  if ((rc = recurrence_buffers(h, buf)) || (rc = handle_workspace(h, 1, (size_t)2 * (max_iter + 2) * 8, &ab)) ||
      (rc = handle_pinned(h, (size_t)2 * (max_iter + 2), &hab)) || (rc = ring.init()))
    return rc;
  double* d_ab = (double*)ab;
  h->rec_live = false;  // from here on the slots change
  const int nr = ring_slots(h);
  Recurrence R{h, false, D, max_iter, lanczos_lookahead(h), d_ab, hab, &ring, {}, {}, 0, 0, profile, {}};
  if (resume) {
    R.alpha = h->last_alpha;
    R.beta = h->last_beta;
    R.amax = *std::max_element(R.alpha.begin(), R.alpha.end());
    R.bmax = *std::max_element(R.beta.begin(), R.beta.end());
    std::vector<double> pairs((size_t)2 * m0);
    for (int j = 0; j < m0; ++j) {
      pairs[2 * j] = R.alpha[j];
      pairs[2 * j + 1] = R.beta[j];
    }
    AED_CUDA_TRY(cudaMemcpyAsync(d_ab, pairs.data(), pairs.size() * 8, cudaMemcpyHostToDevice, h->stream));
    AED_CUDA_TRY(cudaStreamSynchronize(h->stream));  // host pairs go out of scope
  } else if ((rc = start_vector(h, start_host, start_dev, seed, (double*)buf[0]))) {
    return rc;
  }
  StopRule stop{nev, rtol, atol, energy_bound, etol, min_steps};
  if (energy_bound && next_lo > -1e299) {
    stop.next_lo = next_lo;
    stop.block_tol = kRRTol;
  }
  int iters = 0, failed = 0;
  rc = run_recurrence(R, stop, [&](int j) { return buf[j % nr]; }, m0, &iters, &failed, T);
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
  // the T of the stop (the extra step launched ahead of the analysis is discarded)
  R.alpha.resize(iters);
  R.beta.resize(iters);
  h->last_alpha = R.alpha;
  h->last_beta = R.beta;
  h->rec_m = iters;
  h->rec_live = true;
  return AED_OK;
}

// Refinement stop: residual bound r^2 / gap <= kRefineEnergyTol * |lambda| on
// every requested eigenvalue (Kato-Temple), 100x inside the 1e-9 relative
// energy agreement the mixed path promises.
constexpr double kRefineEnergyTol = 1e-11;


// FP32 phase stop: Ritz residual estimates below kTol32 |lambda|.  The FP64
// Rayleigh-Ritz error bound goes with the square of the residuals, so this
// tolerance sets how often the refinement needs no FP64 Lanczos steps.
constexpr double kTol32 = 1e-6;


// The mixed path's FP64 Rayleigh-Ritz refinement.  The K Ritz vectors of
// T(m1) that span the nev lowest clusters (tcore::ritz_span: ghost copies and
// pairs closer than FP32 resolves included) are formed in FP64 from the
// stored FP32 basis, H is applied to each in FP64, and the projected pencil
// (Psi^T H Psi, Psi^T Psi) is solved on the host: directions whose Gram
// eigenvalue is below 1e-10 of the largest (ghost copies of one vector) are
// dropped, the rest orthonormalised.  The K' Ritz pairs (theta_i, Psi c_i)
// get their FP64 residuals r_i = |H Psi c_i - theta_i Psi c_i|, and the
// block residual bound (Kato-Temple for a Ritz subspace)
//   0 <= theta_i - lambda_i <= sum_r r_r^2 / (lambda_next - theta_{K'-1})
// holds whenever lambda_next, the lowest eigenvalue outside the subspace, is
// above theta_{K'-1}; lambda_next is bounded below by the FP32 phase's next
// distinct value minus its error estimate (and its FP32 resolution).  The
// values are accepted when the bound is below kRRTol |theta_i| for every
// reported value; otherwise *accepted stays false and the caller refines by
// FP64 Lanczos.
template <typename SlotFn>
int rayleigh_ritz(aed_handle* h, const TmatInfo& T1, int m1, const std::vector<double>& Z, int nev, SlotFn slot,
                  int64_t ldv, double* coef_dev, aed_solve_result* r, bool* accepted) {
  *accepted = false;
  const int64_t D = h->vlen;
  const int c = std::min(nev, (int)T1.evals.size());
  if (c < 1 || (int)T1.evals.size() <= c) return AED_OK;  // no value above the clusters to bound the gap
  const int K = tcore::ritz_span((int)T1.evals.size(), c, T1.first.data(), T1.mults.data(), m1);
  const bool verbose = std::getenv("AED_VERBOSE") != nullptr;
  if (K < 1 || K > kMaxRR) {
    if (verbose) std::fprintf(stderr, "[aed] rayleigh-ritz: %d Ritz vectors span the clusters (at most %d)\n", K, kMaxRR);
    return AED_OK;
  }
  // coefficients [k * m1 + j] (Z's layout) and the store's chunks
  static_assert(kStoreChunk == kMaxComb, "the combine walks the store chunk by chunk");
  std::vector<double> cf(Z.begin(), Z.begin() + (size_t)K * m1);
  std::vector<const float*> chunks;
  for (int j0 = 0; j0 < m1; j0 += kStoreChunk) chunks.push_back((const float*)slot(j0));
  const size_t vb = ((size_t)D * 8 + 255) & ~(size_t)255;
  const int64_t nch = red_chunks(D);
  const int np = K * (K + 1) / 2 + K * K;
  const size_t part_bytes = (((size_t)np * nch * 8) + 255) & ~(size_t)255;
  void* ws = nullptr;
  // the finished sums: np Gram entries, then (reused) the residuals
  constexpr int kMaxSums = kMaxRR * (kMaxRR + 1) / 2 + kMaxRR * kMaxRR;
  static_assert(kMaxSums >= kMaxRR, "residual sums fit the Gram buffer");
  int rc = handle_workspace(h, 2, rr_workspace_bytes(D, K), &ws);
  if (rc) return rc;
  VecSet psi{}, img{};
  for (int k = 0; k < K; ++k) {
    psi.p[k] = (double*)((char*)ws + (size_t)k * vb);
    img.p[k] = (double*)((char*)ws + (size_t)(K + k) * vb);
  }
  double* part = (double*)((char*)ws + 2 * (size_t)K * vb);
  double* outd = (double*)((char*)part + part_bytes);
  double* hout = nullptr;
  if ((rc = handle_pinned(h, kMaxSums, &hout))) return rc;
  AED_CUDA_TRY(cudaMemcpyAsync(coef_dev, cf.data(), cf.size() * 8, cudaMemcpyHostToDevice, h->stream));
  if ((rc = launch_ritz_combine_chunks(chunks.data(), ldv, m1, coef_dev, K, psi, D, h->stream))) return rc;
  for (int k = 0; k < K; ++k)
    if ((rc = handle_hv(h, false, psi.p[k], img.p[k], nullptr))) return rc;
  if ((rc = launch_gram(psi, img, K, D, part, outd, h->stream))) return rc;
  AED_CUDA_TRY(cudaMemcpyAsync(hout, outd, (size_t)np * 8, cudaMemcpyDeviceToHost, h->stream));
  AED_CUDA_TRY(cudaStreamSynchronize(h->stream));  // the host copy of cf is read by the copy above too
  double G[kMaxRR * kMaxRR], A[kMaxRR * kMaxRR];
  int p = 0;
  for (int a = 0; a < K; ++a)
    for (int b = a; b < K; ++b, ++p) G[a * K + b] = G[b * K + a] = hout[p];
  for (int a = 0; a < K; ++a)
    for (int b = 0; b < K; ++b, ++p) A[a * K + b] = hout[p];
  // Ritz pairs of the pencil, values as Rayleigh quotients (rr_core.h)
  double th[kMaxRR], cr[kMaxRR][kMaxRR];
  int ord[kMaxRR];
  const int Kp = rrcore::ritz_pairs(K, G, A, th, cr, ord);
  if (Kp < 1) return AED_OK;
  for (int a = 0; a < K; ++a)
    for (int b = a + 1; b < K; ++b) A[a * K + b] = A[b * K + a] = 0.5 * (A[a * K + b] + A[b * K + a]);
  std::vector<std::pair<double, int>> byval;
  for (int i = 0; i < Kp; ++i) byval.push_back({th[ord[i]], ord[i]});
  // lowest eigenvalue outside the Ritz pairs that are bounded, from below: the
  // FP32 phase's next distinct value less its error estimate and its FP32
  // resolution.  Only the pairs below it are bounded (block Kato-Temple over
  // their span: 0 <= sum (theta_i - lambda_i) <= sum |r_i|^2 / (lambda_next -
  // theta_max)); a pair above it (the difference of a vector and its ghost
  // copy, mostly FP32 noise) is left out
  const double next = T1.evals[c];
  const double next_lo = next - std::max(T1.errs[c], kFp32MergeRel * std::fabs(next)) -
                         kFp32MergeRel * std::max(std::fabs(T1.evals.front()), std::fabs(T1.evals.back()));
  int nb = 0;
  while (nb < Kp && byval[nb].first < next_lo) ++nb;
  if (nb < 1) return AED_OK;
  ResidCoef rcoef{};
  for (int i = 0; i < nb; ++i) {
    const int q = byval[i].second;
    for (int k = 0; k < K; ++k) {
      rcoef.cw[i][k] = cr[q][k];
      rcoef.cx[i][k] = -th[q] * cr[q][k];
    }
  }
  if ((rc = launch_resid(psi, img, rcoef, K, nb, D, part, outd, h->stream))) return rc;
  AED_CUDA_TRY(cudaMemcpyAsync(hout, outd, (size_t)nb * 8, cudaMemcpyDeviceToHost, h->stream));
  AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
  double r2 = 0.0, rn2 = 0.0;
  for (int i = 0; i < nb; ++i) {
    const int q = byval[i].second;
    double den = 0.0;  // |Psi c_q|^2
    for (int a = 0; a < K; ++a)
      for (int b = 0; b < K; ++b) den += cr[q][a] * G[a * K + b] * cr[q][b];
    r2 += hout[i];
    rn2 += den > 0 ? hout[i] / den : hout[i];
  }
  const double gap = next_lo - byval[nb - 1].first;
  const double bound = rn2 / gap;
  if (verbose)
    std::fprintf(stderr,
                 "[aed] rayleigh-ritz: K=%d kept=%d bounded=%d m=%d sum r^2=%.3e gap=%.3e bound=%.3e (accept <= %.3e)\n",
                 K, Kp, nb, m1, r2, gap, bound, kRRTol * std::fabs(byval[0].first));
  if (!(gap > 0)) return AED_OK;
  // distinct values: merged below the FP64 T-matrix threshold eps^(2/3) max|lambda| (tmatrix.h:148-150)
  const double scale = std::max(std::fabs(T1.evals.front()), std::fabs(T1.evals.back()));
  const double thold = std::pow(2.220446049250313e-16, 2.0 / 3.0) * scale;
  std::vector<int> pick;
  for (int i = 0; i < nb && (int)pick.size() < nev; ++i)
    if (pick.empty() || th[byval[i].second] - th[pick.back()] > thold) pick.push_back(byval[i].second);
  if ((int)pick.size() < c) return AED_OK;  // fewer distinct values than the FP32 phase resolved
  for (int q : pick)
    if (!(bound <= kRRTol * std::max(std::fabs(th[q]), 1e-300))) return AED_OK;
  // accepted: the values and, for aed_eigenvectors, their coefficients over the stored basis
  const int n = (int)pick.size();
  r->n_evals = n;
  h->rr_m = m1;
  h->rr_coef.assign((size_t)n * m1, 0.0);
  h->rr_evals.assign(n, 0.0);
  for (int i = 0; i < n; ++i) {
    r->evals[i] = th[pick[i]];
    h->rr_evals[i] = th[pick[i]];
    r->errors[i] = bound;
    for (int k = 0; k < K; ++k)
      for (int j = 0; j < m1; ++j) h->rr_coef[(size_t)i * m1 + j] += cr[pick[i]][k] * Z[(size_t)k * m1 + j];
  }
  r->iterations = K;
  r->converged = 1;
  r->refined_by = AED_REFINE_RAYLEIGH_RITZ;
  *accepted = true;
  return AED_OK;
}

// FP32 phase with the Lanczos basis stored in HBM, then FP64 refinement.
int solve_mixed(aed_handle* h, const double* start_host, uint64_t seed, int nev, int max_iter, double rtol,
                double atol, bool profile, bool rayleigh_ritz_first, bool reorth, aed_solve_result* r) {
  const int64_t D = h->vlen;
  // Lanczos basis store: chunks of kStoreChunk FP32 vectors, grown as the
  // recurrence advances and kept by the handle for later solves
  const size_t chunk_bytes = store_chunk_bytes_of(D);
  const size_t vbytes = chunk_bytes / kStoreChunk;
  const int64_t ldv = (int64_t)(vbytes / 4);  // stride of the stored vectors (256-byte aligned)
  const int cap = std::min(max_iter + 1, kMaxRitzTerms);
  EventRing ring;
  void* small = nullptr;  // alpha/beta pairs | Ritz coefficients (workspace slot 1, reused by the FP64 phase after)
  double* hab = nullptr;
  int rc;
  const size_t ab_bytes = (((size_t)2 * (cap + 2) * 8 + 255) & ~(size_t)255);
  if ((rc = handle_workspace(h, 1, ab_bytes + (size_t)kMaxRR * (cap + kStoreChunk) * 8, &small)) ||
      (rc = handle_pinned(h, (size_t)2 * (cap + 2), &hab)) || (rc = ring.init()))
    return rc;
  // the FP64 phase's start stays with the handle (eigenvector replay)
  if (!h->d_start64 && (rc = mem_dev_alloc_n(&h->d_start64, (size_t)D))) return rc;
  double* start64 = h->d_start64;
  double* d_ab = (double*)small;
  double* coef = (double*)((char*)small + ab_bytes);
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
  Recurrence R{h, true, D, cap - 1, lanczos_lookahead(h), d_ab, hab, &ring, {}, {}, 0, 0, profile, {}};
  Reorth ro;
  if (reorth) {
    const size_t part_bytes = (((size_t)cap * red_chunks(D) * 8) + 255) & ~(size_t)255;
    const size_t coef_bytes = (((size_t)cap * 8) + 255) & ~(size_t)255;
    void* w = nullptr;
    if ((rc = handle_workspace(h, 2, part_bytes + coef_bytes + (size_t)D * 8, &w))) return rc;
    ro.on = true;
    ro.vec = slot;
    ro.ldv = ldv;
    ro.part = (double*)w;
    ro.coef = (double*)((char*)w + part_bytes);
    ro.tmp = (double*)((char*)w + part_bytes + coef_bytes);
    ro.cap = cap;
    R.reorth = &ro;
  }
  StopRule stop1{nev, kTol32, kTol32 * 1e-3, false, 0.0, 2};
  TmatInfo T1;
  int it1 = 0, failed1 = 0;
  rc = run_recurrence(R, stop1, slot, 0, &it1, &failed1, T1);
  if (oom) return AED_ERR_NOMEM;
  if (rc) return rc;
  const int m1 = it1;
  h->store_m = m1 + 1;  // v_0 .. v_m1 of this FP32 phase stay in the store
  h->low_alpha.assign(R.alpha.begin(), R.alpha.begin() + m1);
  h->low_beta.assign(R.beta.begin(), R.beta.begin() + m1);
  const int n1 = std::min(nev, (int)T1.evals.size());
  for (int i = 0; i < n1; ++i) r->evals_low[i] = T1.evals[i];
  r->iterations_low = m1;
  const double apply32_ms = profile ? R.apply_ms() : 0.0;
  // eigenvectors of T(m1): the Rayleigh-Ritz refinement's Ritz vectors, or
  // the FP64 Lanczos refinement's start
  std::vector<double> ev(R.alpha.begin(), R.alpha.begin() + m1), e(m1 + 1, 0.0), Z((size_t)m1 * m1);
  for (int i = 0; i + 1 < m1; ++i) e[i] = R.beta[i];
  if (tridiag_eigen(m1, ev.data(), e.data(), nullptr, Z.data())) return fail(AED_ERR_TRIDIAG, "tridiagonal eigensolver failed");
  h->last_rr = false;
  if (rayleigh_ritz_first) {
    bool accepted = false;
    if ((rc = rayleigh_ritz(h, T1, m1, Z, nev, slot, ldv, coef, r, &accepted))) return rc;
    if (oom) return AED_ERR_NOMEM;
    if (accepted) {
      h->last_mixed = true;
      h->last_rr = true;
      h->rec_live = false;  // no FP64 recurrence to save or resume
      h->last_alpha.assign(R.alpha.begin(), R.alpha.begin() + m1);
      h->last_beta.assign(R.beta.begin(), R.beta.begin() + m1);
      if (profile) r->apply_ms = apply32_ms;
      return AED_OK;
    }
  }
  // Ritz start of the FP64 Lanczos refinement: the eigenvectors of T(m1) up
  // to the end of the nev-th distinct cluster with seeded weights
  // (tcore::ritz_span / ritz_weight), accumulated in FP64 chunk by chunk from
  // the stored basis
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
  // the FP32 phase's lower bound on the eigenvalue above the nev lowest (as
  // in rayleigh_ritz) for the block Kato-Temple stop of the refinement
  double next_lo = -1e300;
  {
    const int c = std::min(nev, (int)T1.evals.size());
    if (c >= 1 && (int)T1.evals.size() > c) {
      const double nx = T1.evals[c];
      next_lo = nx - std::max(T1.errs[c], kFp32MergeRel * std::fabs(nx)) -
                kFp32MergeRel * std::max(std::fabs(T1.evals.front()), std::fabs(T1.evals.back()));
    }
  }
  rc = solve_fp64(h, nullptr, start64, seed, nev, max2, rtol, atol, true, kRefineEnergyTol, nev + 2, false, r, T2,
                  false, next_lo);
  h->last_mixed = true;
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
  const int64_t D = h->dim;
  const int nev = o->nev;
  if (nev < 1 || nev > AED_MAX_NEV) return fail(AED_ERR_INVALID, "nev must be in 1..16");
  if (o->max_iter < 0) return fail(AED_ERR_INVALID, "max_iter must be >= 0");
  int rc = AED_OK;
  if (D == 0) {
    r->converged = 1;
  } else if (D == 1 && (h->mom || h->gen)) {  // M(0,0) = Re (M e_0)_0 (a momentum sector: flips back into the orbit)
    void* w = nullptr;
    if ((rc = handle_workspace(h, 0, 64, &w))) return rc;
    double* x = (double*)w;
    double* y = x + 2;
    const double one[2] = {1.0, 0.0};
    double out[2] = {0.0, 0.0};
    AED_CUDA_TRY(cudaMemcpyAsync(x, one, h->mom ? 16 : 8, cudaMemcpyHostToDevice, h->stream));
    if ((rc = handle_hv(h, false, x, y, nullptr))) return rc;
    AED_CUDA_TRY(cudaMemcpyAsync(out, y, 16, cudaMemcpyDeviceToHost, h->stream));
    AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
    r->n_evals = 1;
    r->evals[0] = out[0];
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
    if (o->refine < -1 || o->refine > 1) return fail(AED_ERR_INVALID, "refine must be -1, 0 or 1");
    if (o->reorth && (h->precision != AED_FP32 || o->refine == -1 || o->resume))
      return fail(AED_ERR_INVALID, "reorth needs the mixed path of an AED_FP32 handle (its Lanczos basis is stored)");
    if (o->resume) {  // continue the live FP64 recurrence (any handle precision)
      TmatInfo T;
      h->last_rr = false;
      rc = solve_fp64(h, nullptr, nullptr, 0, nev, max_iter, rtol, atol, false, 0.0, 0, o->profile != 0, r, T, true);
    } else if (h->precision == AED_FP32 && o->refine != -1) {
      rc = solve_mixed(h, o->start, o->seed, nev, max_iter, rtol, atol, o->profile != 0, o->refine == 0,
                       o->reorth != 0, r);
      if (!rc && r->refined_by == AED_REFINE_NONE) r->refined_by = AED_REFINE_LANCZOS;
    } else {
      h->last_rr = false;
      TmatInfo T;
      rc = solve_fp64(h, o->start, nullptr, o->seed, nev, max_iter, rtol, atol, false, 0.0, 0, o->profile != 0, r, T);
      h->last_mixed = false;
    }
  }
  r->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return rc;
}

namespace {

// |v| on the host (deterministic reduction, FP64 vector).
int host_norm(aed_handle* h, const double* v, double* out) {
  const int64_t D = h->vlen;
  int rc = launch_dot_partials(v, v, D, h->d_partB, true, h->stream);
  if (!rc) rc = launch_finish_sum(h->d_partB, red_chunks(D), h->d_scal + 6, true, h->stream);
  if (rc) return rc;
  AED_CUDA_TRY(cudaMemcpyAsync(h->h_scal + 6, h->d_scal + 6, 8, cudaMemcpyDeviceToHost, h->stream));
  AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
  *out = h->h_scal[6];
  return AED_OK;
}

// FNV-1a of the model (sector and couplings): a saved recurrence only loads
// into a handle of the same Hamiltonian.
uint64_t model_hash(const Model& m, const MomParams* mp, int two_s) {
  uint64_t x = 1469598103934665603ull;
  auto mix = [&](const void* p, size_t n) {
    const unsigned char* b = (const unsigned char*)p;
    for (size_t i = 0; i < n; ++i) x = (x ^ b[i]) * 1099511628211ull;
  };
  mix(&m.N, sizeof m.N);
  mix(&m.n_up, sizeof m.n_up);
  for (size_t b = 0; b < m.s1.size(); ++b) {
    mix(&m.s1[b], sizeof(int));
    mix(&m.s2[b], sizeof(int));
    mix(&m.jz[b], 8);
    mix(&m.jxy[b], 8);
    mix(&m.kq[b], 8);
  }
  for (double v : m.site_h) mix(&v, 8);
  for (double v : m.site_d) mix(&v, 8);
  if (two_s != 1) mix(&two_s, sizeof two_s);
  if (mp) {  // a momentum sector: its translations and phases
    mix(&mp->n_trans, sizeof mp->n_trans);
    for (int t = 0; t < mp->n_trans; ++t) {
      mix(&mp->phase_re[t], 8);
      mix(&mp->phase_im[t], 8);
      mix(mp->dst[t], 32);
    }
  }
  return x;
}

struct StateHeader {
  char magic[8];
  int64_t D;
  int32_t N, n_up;
  int32_t m, reserved;
  uint64_t model;
};
constexpr char kStateMagic[8] = {'A', 'E', 'D', 'L', 'N', 'C', 'Z', '1'};

}  // namespace

// Ritz vectors of a mixed solve refined by Rayleigh-Ritz: psi_i =
// sum_j rr_coef[i][j] v_j over the FP32 Lanczos basis the handle kept,
// accumulated in FP64 (ritz_combine_chunks, kMaxRR vectors per pass),
// normalised; residual |H psi_i - theta_i psi_i| with the FP64 apply.
int rr_eigenvectors(aed_handle* h, int k, void* const* vecs, double* evals, double* resid) {
  const int n = (int)h->rr_evals.size(), m1 = h->rr_m;
  if (k > n) return fail(AED_ERR_INVALID, "eigenvectors: k exceeds the distinct eigenvalues found");
  for (int i = 0; i < k; ++i)
    if (!vecs[i]) return fail(AED_ERR_INVALID, "eigenvectors: NULL output vector");
  const int64_t D = h->vlen;
  const size_t cb = h->store_chunk_bytes;
  if (cb == 0 || (int)h->store_chunks.size() * kStoreChunk < m1)
    return fail(AED_ERR_INVALID, "eigenvectors: the mixed solve's Lanczos basis is gone");
  const int64_t ldv = (int64_t)(cb / kStoreChunk / 4);
  const size_t vb = ((size_t)D * 8 + 255) & ~(size_t)255;
  DevMem rb, cd;
  int rc;
  if ((rc = rb.alloc((size_t)(k + 1) * vb)) || (rc = cd.alloc((size_t)kMaxRR * m1 * 8))) return rc;
  std::vector<double*> acc(k);
  for (int i = 0; i < k; ++i) acc[i] = (double*)((char*)rb.p + (size_t)i * vb);
  double* w = (double*)((char*)rb.p + (size_t)k * vb);
  for (int i0 = 0; i0 < k; i0 += kMaxRR) {
    const int K = std::min(kMaxRR, k - i0);
    std::vector<double> cf(h->rr_coef.begin() + (size_t)i0 * m1, h->rr_coef.begin() + (size_t)(i0 + K) * m1);
    AED_CUDA_TRY(cudaMemcpyAsync(cd.p, cf.data(), cf.size() * 8, cudaMemcpyHostToDevice, h->stream));
    VecSet out{};
    for (int q = 0; q < K; ++q) out.p[q] = acc[i0 + q];
    std::vector<const float*> chunks;
    for (int j0 = 0; j0 < m1; j0 += kStoreChunk) chunks.push_back((const float*)h->store_chunks[j0 / kStoreChunk]);
    if ((rc = launch_ritz_combine_chunks(chunks.data(), ldv, m1, (const double*)cd.p, K, out, D, h->stream)))
      return rc;
    AED_CUDA_TRY(cudaStreamSynchronize(h->stream));  // cf and the coefficient buffer are reused
  }
  const bool f32 = h->precision == AED_FP32;
  for (int i = 0; i < k; ++i) {
    double nrm = 0.0;
    if ((rc = host_norm(h, acc[i], &nrm))) return rc;
    if (!(nrm > 0.0)) return fail(AED_ERR_INVALID, "eigenvectors: zero Ritz vector");
    if ((rc = launch_scal<double>(nrm, acc[i], D, true, h->stream))) return rc;
    if ((rc = handle_hv(h, false, acc[i], w, nullptr))) return rc;
    if ((rc = launch_axpy<double>(-h->rr_evals[i], acc[i], w, D, h->stream))) return rc;
    double rn = 0.0;
    if ((rc = host_norm(h, w, &rn))) return rc;
    if (resid) resid[i] = rn;
    if (evals) evals[i] = h->rr_evals[i];
    if (f32)
      rc = launch_round_to_f32(acc[i], (float*)vecs[i], D, h->stream);
    else
      rc = launch_copy<double>(acc[i], (double*)vecs[i], D, h->stream);
    if (rc) return rc;
  }
  AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return AED_OK;
}

// lanczos::eigenvectors (src/ietl/lanczos.h:134-336): the Lanczos vectors are
// not stored, so the recurrence of the last solve is run again from its start
// (the seeded or given vector of `o`; for a mixed solve the kept start of its
// FP64 phase) and psi_i = sum_j z_i[j] v_j accumulates step by step, z_i the
// eigenvector of T(m) of the i-th lowest distinct eigenvalue.  The replayed
// alpha/beta must equal the stored ones bit for bit (lanczos.h:248-250,
// 266-268), else AED_ERR_MISMATCH.  Then psi_i /= |psi_i| and the residual
// |H psi_i - lambda_i psi_i| (lanczos.h:284-295).
int eigenvectors(aed_handle* h, const aed_solve_opts* o, int k, void* const* vecs, double* evals, double* resid) {
  if (!o || !vecs || k < 1) return fail(AED_ERR_INVALID, "eigenvectors: NULL argument or k < 1");
  if (h->last_rr) return rr_eigenvectors(h, k, vecs, evals, resid);
  const int m = (int)h->last_alpha.size();
  if (m < 1) return fail(AED_ERR_INVALID, "eigenvectors: no solve to take eigenvectors from");
  for (int i = 0; i < k; ++i)
    if (!vecs[i]) return fail(AED_ERR_INVALID, "eigenvectors: NULL output vector");
  const int64_t D = h->vlen;
  const bool f32 = h->precision == AED_FP32;
  const std::vector<double>& al = h->last_alpha;
  const std::vector<double>& be = h->last_beta;
  TmatInfo T;
  int rc = tmatrix_analyze(m, al.data(), be.data(), *std::max_element(al.begin(), al.end()),
                           *std::max_element(be.begin(), be.end()), T, 0.0);
  if (rc) return rc;
  if (k > (int)T.evals.size()) return fail(AED_ERR_INVALID, "eigenvectors: k exceeds the distinct eigenvalues found");
  std::vector<double> ev(al), e(m + 1, 0.0), Z((size_t)m * m);
  for (int i = 0; i + 1 < m; ++i) e[i] = be[i];
  if (tridiag_eigen(m, ev.data(), e.data(), nullptr, Z.data())) return fail(AED_ERR_TRIDIAG, "tridiagonal eigensolver failed");
  const size_t vb = ((size_t)D * 8 + 255) & ~(size_t)255;
  DevMem rb, dab;
  if ((rc = rb.alloc((3 + (f32 ? k : 0)) * vb)) || (rc = dab.alloc((size_t)2 * m * 8))) return rc;
  double* buf[3] = {(double*)rb.p, (double*)((char*)rb.p + vb), (double*)((char*)rb.p + 2 * vb)};
  std::vector<double*> acc(k);
  for (int i = 0; i < k; ++i) {
    acc[i] = f32 ? (double*)((char*)rb.p + (3 + i) * vb) : (double*)vecs[i];
    AED_CUDA_TRY(cudaMemsetAsync(acc[i], 0, (size_t)D * 8, h->stream));
  }
  if (h->last_mixed) {
    if (!h->d_start64) return fail(AED_ERR_INVALID, "eigenvectors: the mixed solve's start is gone");
    rc = start_vector(h, nullptr, h->d_start64, 0, buf[0]);
  } else {
    rc = start_vector(h, o->start, nullptr, o->seed, buf[0]);
  }
  if (rc) return rc;
  double* d_ab = (double*)dab.p;
  for (int j = 0; j < m; ++j) {
    double* vj = buf[j % 3];
    for (int i = 0; i < k; ++i)
      if ((rc = launch_axpy<double>(Z[(size_t)T.first[i] * m + j], vj, acc[i], D, h->stream))) return rc;
    if (j + 1 < m) {
      double* w = buf[(j + 1) % 3];
      const double* vp = j > 0 ? buf[(j + 2) % 3] : nullptr;
      if ((rc = handle_hv(h, false, vj, w, h->d_partA))) return rc;
      if ((rc = lanczos_step_tail(h, false, vp, vj, w, j > 0 ? d_ab + 2 * (j - 1) + 1 : nullptr, d_ab + 2 * j,
                                  d_ab + 2 * j + 1)))
        return rc;
    }
  }
  if (m > 1) {
    std::vector<double> rep((size_t)2 * (m - 1));
    AED_CUDA_TRY(cudaMemcpyAsync(rep.data(), d_ab, rep.size() * 8, cudaMemcpyDeviceToHost, h->stream));
    AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (int j = 0; j + 1 < m; ++j)
      if (std::memcmp(&rep[2 * j], &al[j], 8) != 0 || std::memcmp(&rep[2 * j + 1], &be[j], 8) != 0)
        return fail(AED_ERR_MISMATCH, "eigenvectors: the replayed recurrence differs from the solve's at step " +
                                          std::to_string(j) + " (different start vector?)");
  }
  for (int i = 0; i < k; ++i) {
    double nrm = 0.0;
    if ((rc = host_norm(h, acc[i], &nrm))) return rc;
    if (!(nrm > 0.0)) return fail(AED_ERR_INVALID, "eigenvectors: zero Ritz vector");
    if ((rc = launch_scal<double>(nrm, acc[i], D, true, h->stream))) return rc;
    double* w = buf[0];
    if ((rc = handle_hv(h, false, acc[i], w, nullptr))) return rc;
    if ((rc = launch_axpy<double>(-T.evals[i], acc[i], w, D, h->stream))) return rc;
    double rn = 0.0;
    if ((rc = host_norm(h, w, &rn))) return rc;
    if (resid) resid[i] = rn;
    if (evals) evals[i] = T.evals[i];
    if (f32 && (rc = launch_round_to_f32(acc[i], (float*)vecs[i], D, h->stream))) return rc;
  }
  AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return AED_OK;
}

int64_t lanczos_state_bytes(const aed_handle* h) {
  if (!h->rec_live) return 0;
  return (int64_t)sizeof(StateHeader) + (int64_t)16 * h->rec_m + (int64_t)16 * h->vlen;
}

// Tmatrix::save + lanczos::save (src/ietl/tmatrix.h:66-77, lanczos.h:86-98):
// the recurrence (alpha, beta) and the two live vectors v_{m-1}, v_m.
int lanczos_save(aed_handle* h, void* buf, int64_t bytes) {
  if (!buf) return fail(AED_ERR_INVALID, "lanczos_save: NULL buffer");
  if (!h->rec_live) return fail(AED_ERR_INVALID, "lanczos_save: no live Lanczos recurrence (solve first)");
  if (bytes < lanczos_state_bytes(h)) return fail(AED_ERR_INVALID, "lanczos_save: buffer too small");
  const int m = h->rec_m;
  const int64_t D = h->vlen;
  StateHeader hd{};
  std::memcpy(hd.magic, kStateMagic, 8);
  hd.D = D;
  hd.N = h->model.N;
  hd.n_up = h->model.n_up;
  hd.m = m;
  hd.model = model_hash(h->model, h->mp, h->two_s);
  char* p = (char*)buf;
  std::memcpy(p, &hd, sizeof hd);
  p += sizeof hd;
  std::memcpy(p, h->last_alpha.data(), (size_t)m * 8);
  p += (size_t)m * 8;
  std::memcpy(p, h->last_beta.data(), (size_t)m * 8);
  p += (size_t)m * 8;
  void* slots[kMaxRing];
  int rc = recurrence_buffers(h, slots);
  if (rc) return rc;
  AED_CUDA_TRY(cudaMemcpyAsync(p, slots[(m - 1) % ring_slots(h)], (size_t)D * 8, cudaMemcpyDeviceToHost, h->stream));
  AED_CUDA_TRY(cudaMemcpyAsync(p + (size_t)D * 8, slots[m % ring_slots(h)], (size_t)D * 8, cudaMemcpyDeviceToHost, h->stream));
  AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return AED_OK;
}

int lanczos_load(aed_handle* h, const void* buf, int64_t bytes) {
  if (!buf || bytes < (int64_t)sizeof(StateHeader)) return fail(AED_ERR_INVALID, "lanczos_load: no state");
  StateHeader hd;
  std::memcpy(&hd, buf, sizeof hd);
  if (std::memcmp(hd.magic, kStateMagic, 8) != 0) return fail(AED_ERR_INVALID, "lanczos_load: not a saved recurrence");
  if (hd.D != h->vlen || hd.N != h->model.N || hd.n_up != h->model.n_up || hd.model != model_hash(h->model, h->mp, h->two_s))
    return fail(AED_ERR_INVALID, "lanczos_load: the state belongs to a different Hamiltonian");
  const int m = hd.m;
  const int64_t D = hd.D;
  if (m < 1 || bytes < (int64_t)sizeof hd + (int64_t)16 * m + (int64_t)16 * D)
    return fail(AED_ERR_INVALID, "lanczos_load: truncated state");
  const char* p = (const char*)buf + sizeof hd;
  std::vector<double> al(m), be(m);
  std::memcpy(al.data(), p, (size_t)m * 8);
  std::memcpy(be.data(), p + (size_t)m * 8, (size_t)m * 8);
  p += (size_t)16 * m;
  void* slots[kMaxRing];
  int rc = recurrence_buffers(h, slots);
  if (rc) return rc;
  AED_CUDA_TRY(cudaMemcpyAsync(slots[(m - 1) % ring_slots(h)], p, (size_t)D * 8, cudaMemcpyHostToDevice, h->stream));
  AED_CUDA_TRY(cudaMemcpyAsync(slots[m % ring_slots(h)], p + (size_t)D * 8, (size_t)D * 8, cudaMemcpyHostToDevice, h->stream));
  AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->last_alpha = al;
  h->last_beta = be;
  h->rec_m = m;
  h->rec_live = true;
  h->last_mixed = false;
  return AED_OK;
}

}  // namespace aed
