// batch.cu -- kernels of the batched / served Lanczos engine.
//
// One engine step advances every resident instance by one Lanczos step
// (lanczos::make_step, src/ietl/lanczos.h:392-406):
//   b_hv32/64  y = H x over the (instance, bundle) queue, per-tile <x,y> partials
//   b_alpha    alpha_j = sum of the instance's tile partials (one CTA each)
//   b_update   y = (y - alpha x) - beta_{j-1} v_{j-1} over (instance, chunk), chunk partials of |y|^2
//   b_beta     beta_j = sqrt(sum of the chunk partials)
//   b_norm     y /= beta_j
//   b_advance  j += 1
// After S steps the graph runs b_check (one thread per instance: the
// T-matrix analysis of tmatrix_core.h and the phase rules), then the FP32 ->
// FP64 hand-over (b_ritz, b_ritz_norm, b_ritz_scale, b_ritz_commit).
// Every sum is formed per instance in a fixed order, so an instance's result
// does not depend on which other instances share the batch.

#include <cuda_runtime.h>

#include "apply.cuh"
#include "apply_blocks.cuh"
#include "batch.cuh"
#include "reduce.cuh"
#include "tmatrix_core.h"

namespace aed {
namespace {

using apply::AccExact64;
using apply::AccWide32;
using apply::ApplyCtx;
using apply::ApplySmem;


__device__ __forceinline__ bool stepping(const BInst& I) {
  if (I.phase == kPhLow) return I.j + 1 < I.n_store && I.j < I.cap;
  if (I.phase == kPhHigh) return I.j < I.cap;
  return false;
}

__device__ __forceinline__ float* low_vec(const BInst& I, int j) {
  return I.chunk[j / kStoreChunkB] + (int64_t)(j % kStoreChunkB) * I.ldv;
}
__device__ __forceinline__ double* high_vec(const BInst& I, int j) { return I.v64[j % 3]; }

// The apply of every stepping instance over its (instance, bundle) items: the
// bundle apply (apply_blocks.cuh) with the instance's tables; the staged
// pairs and the shared-memory layout change with the instance.  FP32 vectors:
// one kernel per sector-size bucket (the rows of the largest hi block,
// maxrows in (mr_lo, mr_hi]), each a template instance picked for its bucket
// by the autotuner (batch_tune_bucket): R rows per thread, MINB CTAs per SM,
// B = 1 (the item's hi blocks one at a time) or kBatchBundle (both at once).
// FP64 vectors (b_hv64): 4 rows per thread, 3 CTAs per SM.
template <int R, int MINB, int B>
__global__ void __launch_bounds__(kHvThreads, MINB) b_hv32(BatchArgs a, int mr_lo, int mr_hi) {
  static_assert(B == 1 || B == kBatchBundle, "an item is one bundle or its blocks one by one");
  extern __shared__ __align__(16) unsigned char b_dyn[];
  __shared__ bapply::BundleSmem<B> sm;
  const int n = *a.n_tiles;
  int cur = -1, rc = 0;
  float* xs = nullptr;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const BItem w = a.tiles[it];
    const BInst& I = a.inst[w.inst];
    if (I.phase != kPhLow || !stepping(I) || I.t.maxrows <= mr_lo || I.t.maxrows > mr_hi)
      continue;  // same for every thread of the CTA
    const int j = I.j;
    if (w.inst != cur) {
      __syncthreads();  // the previous block is done with the staged pairs
      xs = bapply::carve<float, B>(*I.P, I.t, b_dyn, sm);
      bapply::stage_pairs<B>(*I.P, sm);
      cur = w.inst;
    }
    const ApplyCtx c = apply::ctx_of(*I.P);
    if (B == kBatchBundle) {  // both blocks of the item at once
      bapply::apply_bundle<float, AccWide32, R, B>(c, I.t, w.idx, low_vec(I, j), low_vec(I, j + 1), I.partA, sm, xs,
                                                   rc);
    } else {
      for (int q = 0; q < kBatchBundle; ++q)  // the item's blocks one at a time (block-list entries)
        bapply::apply_bundle<float, AccWide32, R, B>(c, I.t, (int64_t)w.idx * kBatchBundle + q, low_vec(I, j),
                                                     low_vec(I, j + 1), I.partA, sm, xs, rc);
    }
  }
}

__global__ void __launch_bounds__(kHvThreads, 3) b_hv64(BatchArgs a) {
  extern __shared__ __align__(16) unsigned char b_dyn[];
  __shared__ bapply::BundleSmem<1> sm;
  const int n = *a.n_tiles;
  int cur = -1, rc = 0;
  double* xs = nullptr;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const BItem w = a.tiles[it];
    const BInst& I = a.inst[w.inst];
    if (I.phase != kPhHigh || !stepping(I)) continue;
    const int j = I.j;
    if (w.inst != cur) {
      __syncthreads();
      xs = bapply::carve<double, 1>(*I.P, I.t, b_dyn, sm);
      bapply::stage_pairs<1>(*I.P, sm);
      cur = w.inst;
    }
    const ApplyCtx c = apply::ctx_of(*I.P);
    for (int q = 0; q < kBatchBundle; ++q)  // the item's blocks one at a time (block-list entries)
      bapply::apply_bundle<double, AccExact64, 4, 1>(c, I.t, (int64_t)w.idx * kBatchBundle + q, high_vec(I, j),
                                                     high_vec(I, j + 1), I.partA, sm, xs, rc);
  }
}

__global__ void __launch_bounds__(256) b_alpha(BatchArgs a) {
  __shared__ double red[33];
  if ((int)blockIdx.x >= *a.n_inst) return;
  BInst& I = a.inst[blockIdx.x];
  if (!stepping(I)) return;
  double v = 0.0;
  for (int i = threadIdx.x; i < I.n_tiles; i += 256) v += I.partA[i];
  const double tot = block_sum_all<256>(v, red);
  if (threadIdx.x == 0) I.ab[2 * I.j] = tot;
}

template <typename T>
__device__ __forceinline__ double update_chunk(const T* x, const T* vp, T* y, int64_t e0, int64_t e1, double alpha,
                                               double b) {
  double acc = 0.0;
  for (int64_t i = e0 + threadIdx.x; i < e1; i += kRedThreads) {
    double w = __dsub_rn((double)y[i], __dmul_rn(alpha, (double)x[i]));
    if (vp) w = __dsub_rn(w, __dmul_rn(b, (double)vp[i]));
    const T wt = (T)w;
    y[i] = wt;
    acc = fma((double)wt, (double)wt, acc);
  }
  return acc;
}

__global__ void __launch_bounds__(kRedThreads) b_update(BatchArgs a) {
  __shared__ double red[33];
  const int n = *a.n_chunks;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const BItem w = a.chunks[it];
    BInst& I = a.inst[w.inst];
    if (!stepping(I)) continue;
    const int j = I.j;
    const double alpha = I.ab[2 * j];
    const double b = j > 0 ? I.ab[2 * (j - 1) + 1] : 0.0;
    const int64_t e0 = (int64_t)w.idx * kRedChunk, e1 = e0 + kRedChunk < I.D ? e0 + kRedChunk : I.D;
    double acc;
    if (I.phase == kPhLow)
      acc = update_chunk<float>(low_vec(I, j), j > 0 ? low_vec(I, j - 1) : nullptr, low_vec(I, j + 1), e0, e1, alpha, b);
    else
      acc = update_chunk<double>(high_vec(I, j), j > 0 ? high_vec(I, j - 1) : nullptr, high_vec(I, j + 1), e0, e1,
                                 alpha, b);
    const double tot = block_sum_all<kRedThreads>(acc, red);
    if (threadIdx.x == 0) I.partB[w.idx] = tot;
  }
}

__global__ void __launch_bounds__(256) b_beta(BatchArgs a) {
  __shared__ double red[33];
  if ((int)blockIdx.x >= *a.n_inst) return;
  BInst& I = a.inst[blockIdx.x];
  if (!stepping(I)) return;
  double v = 0.0;
  for (int64_t i = threadIdx.x; i < I.n_chunks; i += 256) v += I.partB[i];
  const double tot = block_sum_all<256>(v, red);
  if (threadIdx.x == 0) I.ab[2 * I.j + 1] = sqrt(tot);
}

__global__ void __launch_bounds__(kRedThreads) b_norm(BatchArgs a) {
  const int n = *a.n_chunks;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const BItem w = a.chunks[it];
    const BInst& I = a.inst[w.inst];
    if (!stepping(I)) continue;
    const int j = I.j;
    const double beta = I.ab[2 * j + 1];
    const int64_t e0 = (int64_t)w.idx * kRedChunk, e1 = e0 + kRedChunk < I.D ? e0 + kRedChunk : I.D;
    if (I.phase == kPhLow) {
      float* y = low_vec(I, j + 1);
      for (int64_t i = e0 + threadIdx.x; i < e1; i += kRedThreads) y[i] = (float)__ddiv_rn((double)y[i], beta);
    } else {
      double* y = high_vec(I, j + 1);
      for (int64_t i = e0 + threadIdx.x; i < e1; i += kRedThreads) y[i] = __ddiv_rn(y[i], beta);
    }
  }
}

__global__ void b_advance(BatchArgs a) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= *a.n_inst) return;
  BInst& I = a.inst[s];
  if (stepping(I)) I.j += 1;
}

// End of a graph launch: T-matrix analysis of every stepping instance and the
// phase rules.  Two threads per instance: the eigenvalue sweeps of T and of T
// without its first row and column run side by side (tcore::analyze_t /
// analyze_t2, the bulk of the work), then the first thread finishes.
__global__ void __launch_bounds__(32) b_check(BatchArgs a) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = g >> 1, lane = g & 1;
  const unsigned pair = 3u << (threadIdx.x & 30);  // the two threads of this instance
  if (s >= *a.n_inst) return;  // both threads of a pair leave together
  BInst& I = a.inst[s];
  if (I.phase != kPhLow && I.phase != kPhHigh) return;
  const int m = I.j;  // alpha_0 .. alpha_{j-1} are final
  if (m < 2) return;
  const int cap = I.cap;
  double* al = I.scratch;
  double* be = al + cap;
  double* work = be + cap;      // 5 cap + 2
  double* z = work + 5 * cap + 2;  // cap
  double* inv = z + cap;         // 6 cap
  if (lane == 0)
    for (int q = 0; q < m; ++q) {
      al[q] = I.ab[2 * q];
      be[q] = I.ab[2 * q + 1];
    }
  __syncwarp(pair);
  const int info = lane == 0 ? tcore::analyze_t(m, al, be, work) : tcore::analyze_t2(m, al, be, work);
  const int info2 = __shfl_xor_sync(pair, info, 1);
  if (lane != 0) return;
  double amax = I.ab[0], bmax = I.ab[1];
  for (int q = 0; q < m; ++q) {
    amax = tcore::dmax(amax, al[q]);
    bmax = tcore::dmax(bmax, be[q]);
  }
  const int nev = I.nev;
  double ev[AED_MAX_NEV + 1], er[AED_MAX_NEV + 1];
  int first[AED_MAX_NEV + 1], mults[AED_MAX_NEV + 1];
  tcore::TResult res;
  res.count = 0;
  const int want = nev + 1;
  const bool bad = info != 0 || info2 != 0 ||
                   tcore::analyze_walk(m, be, amax, bmax, work, want, ev, er, mults, first, &res,
                                       I.phase == kPhLow ? kFp32MergeRel : 0.0) != 0;
  const int cnt = res.count;
  bool conv = !bad && cnt >= nev;
  if (I.phase == kPhLow) {
    for (int i = 0; conv && i < nev; ++i)
      if (!(er[i] <= tcore::dmax(I.tol32 * 1e-3, I.tol32 * fabs(ev[i])))) conv = false;
    const bool full = !stepping(I);
    if (!(conv || full || bad)) return;
    // Ritz coefficients: the unit eigenvectors of T(m) with sorted indices
    // [0, K) (the nev lowest distinct values, whole clusters:
    // tcore::ritz_span) with seeded weights; work[0..m) holds the sorted
    // eigenvalues of T after analyze
    const int n1 = cnt < nev ? cnt : nev;
    for (int q = 0; q < m; ++q) I.coef[q] = 0.0;
    const int K = bad ? 0 : tcore::ritz_span(cnt, nev, first, mults, m);
    for (int k = 0; k < K; ++k) {
      tcore::inverse_iteration(m, al, be, work[k], z, inv);
      const double w = tcore::ritz_weight(I.seed, k);
      for (int q = 0; q < m; ++q) I.coef[q] += w * z[q];
    }
    if (K == 0) I.coef[0] = 1.0;
    for (int i = 0; i < n1; ++i) I.evals_low[i] = ev[i];
    I.m_low = m;
    I.phase = kPhRitz;
  } else {
    if (m < nev + 2) conv = false;
    bool ietl = conv;
    for (int i = 0; ietl && i < nev; ++i)
      if (er[i] > tcore::dmax(I.atol, I.rtol * fabs(ev[i]))) ietl = false;
    bool energy = conv && I.etol > 0.0 && cnt >= nev + 1;
    for (int i = 0; energy && i < nev; ++i) {
      const double gap = ev[i + 1] - ev[i];
      if (!(gap > 0.0) || !(er[i] * er[i] / gap <= I.etol * fabs(ev[i]))) energy = false;
    }
    const bool full = !stepping(I);
    if (!(ietl || energy || full || bad)) return;
    const int n = cnt < nev ? cnt : nev;
    for (int i = 0; i < n; ++i) {
      I.evals[i] = ev[i];
      I.errs[i] = er[i];
    }
    I.n_evals = n;
    I.iters = m;
    I.converged = (ietl || energy) ? 1 : 0;
    I.phase = kPhDone;
  }
}

// FP64 start of the refinement: v = sum_q coef[q] v_q (stored FP32 basis),
// chunk partials of |v|^2.
__global__ void __launch_bounds__(kRedThreads) b_ritz(BatchArgs a) {
  __shared__ double red[33];
  __shared__ double cs[kStoreChunkB];
  const int n = *a.n_chunks;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const BItem w = a.chunks[it];
    BInst& I = a.inst[w.inst];
    if (I.phase != kPhRitz) continue;
    const int64_t e0 = (int64_t)w.idx * kRedChunk, e1 = e0 + kRedChunk < I.D ? e0 + kRedChunk : I.D;
    double* out = I.v64[0];
    double acc[kRedChunk / kRedThreads];
#pragma unroll
    for (int u = 0; u < kRedChunk / kRedThreads; ++u) acc[u] = 0.0;
    for (int q0 = 0; q0 < I.m_low; q0 += kStoreChunkB) {
      const int cnt = I.m_low - q0 < kStoreChunkB ? I.m_low - q0 : kStoreChunkB;
      __syncthreads();
      if (threadIdx.x < cnt) cs[threadIdx.x] = I.coef[q0 + threadIdx.x];
      __syncthreads();
      for (int q = 0; q < cnt; ++q) {
        const float* v = low_vec(I, q0 + q);
#pragma unroll
        for (int u = 0; u < kRedChunk / kRedThreads; ++u) {
          const int64_t i = e0 + threadIdx.x + u * kRedThreads;
          if (i < e1) acc[u] = fma(cs[q], (double)v[i], acc[u]);
        }
      }
    }
    double sq = 0.0;
#pragma unroll
    for (int u = 0; u < kRedChunk / kRedThreads; ++u) {
      const int64_t i = e0 + threadIdx.x + u * kRedThreads;
      if (i < e1) {
        out[i] = acc[u];
        sq = fma(acc[u], acc[u], sq);
      }
    }
    const double tot = block_sum_all<kRedThreads>(sq, red);
    if (threadIdx.x == 0) I.partB[w.idx] = tot;
  }
}

__global__ void __launch_bounds__(256) b_ritz_norm(BatchArgs a) {
  __shared__ double red[33];
  if ((int)blockIdx.x >= *a.n_inst) return;
  BInst& I = a.inst[blockIdx.x];
  if (I.phase != kPhRitz) return;
  double v = 0.0;
  for (int64_t i = threadIdx.x; i < I.n_chunks; i += 256) v += I.partB[i];
  const double tot = block_sum_all<256>(v, red);
  if (threadIdx.x == 0) I.ritz_norm = sqrt(tot);
}

__global__ void __launch_bounds__(kRedThreads) b_ritz_scale(BatchArgs a) {
  const int n = *a.n_chunks;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const BItem w = a.chunks[it];
    const BInst& I = a.inst[w.inst];
    if (I.phase != kPhRitz) continue;
    const int64_t e0 = (int64_t)w.idx * kRedChunk, e1 = e0 + kRedChunk < I.D ? e0 + kRedChunk : I.D;
    double* v = I.v64[0];
    for (int64_t i = e0 + threadIdx.x; i < e1; i += kRedThreads) v[i] = __ddiv_rn(v[i], I.ritz_norm);
  }
}

__global__ void b_ritz_commit(BatchArgs a) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= *a.n_inst) return;
  BInst& I = a.inst[s];
  if (I.phase != kPhRitz) return;
  I.phase = kPhHigh;
  I.j = 0;
}

int g_sms = 0;
int sms() {
  if (!g_sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_sms <= 0) g_sms = 148;
  }
  return g_sms;
}

// The FP32 apply candidates of the autotuner.  Every candidate adds each
// row's terms in the same order (apply_blocks.cuh), so the choice changes the
// speed, not the results.
struct Cand32 {
  void (*kern)(BatchArgs, int, int);
  const char* name;
};
const Cand32 kCand32[kBatchCand32] = {
    {b_hv32<1, 6, 1>, "r1b6"},          {b_hv32<2, 4, kBatchBundle>, "blk2r2b4"}, {b_hv32<2, 4, 1>, "r2b4"},
    {b_hv32<1, 4, kBatchBundle>, "blk2r1b4"}, {b_hv32<4, 3, 1>, "r4b3"},
};
int g_c32[kBatchCand32] = {}, g_c32_smem[kBatchCand32] = {-1, -1, -1, -1, -1};
int g_hv64 = 0, g_hv64_smem = -1;

// Grid of an apply kernel for `smem` bytes of dynamic shared memory (cached per size).
template <typename K>
int hv_grid(K kern, int smem, int* g, int* g_smem) {
  if (smem != *g_smem) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    int per = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, kHvThreads, smem);
    *g = sms() * (per < 1 ? 1 : per);
    *g_smem = smem;
  }
  return *g;
}

int check(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(AED_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return AED_OK;
}

}  // namespace

size_t batch_hv_smem_bytes(int maxrows, const HvParams& P) {
  const size_t f64 = bapply::bundle_smem_bytes<double>(1, maxrows, P.n_pairs, P.n_lolo);
  const size_t f32 = bapply::bundle_smem_bytes<float>(kBatchBundle, maxrows, P.n_pairs, P.n_lolo);
  return f64 > f32 ? f64 : f32;
}

size_t batch_hv_smem_limit() {
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes f64{};
  cudaFuncGetAttributes(&f64, b_hv64);
  size_t st = f64.sharedSizeBytes;
  for (const Cand32& c : kCand32) {
    cudaFuncAttributes f{};
    cudaFuncGetAttributes(&f, c.kern);
    if (f.sharedSizeBytes > st) st = f.sharedSizeBytes;
  }
  return optin > (int)st ? (size_t)optin - st : 0;
}

int batch_prepare(const BatchArgs& a) {
  for (int c = 0; c < kBatchCand32; ++c) hv_grid(kCand32[c].kern, a.hv_smem, &g_c32[c], &g_c32_smem[c]);
  hv_grid(b_hv64, a.hv_smem, &g_hv64, &g_hv64_smem);
  return check("batched apply attributes");
}

int batch_bucket_of(int maxrows) {
  int b = 0;
  while (b + 1 < kBatchBuckets && maxrows > kBatchBucketHi[b]) ++b;
  return b;
}

const char* batch_cand32_name(int c) { return (c >= 0 && c < kBatchCand32) ? kCand32[c].name : "?"; }

int batch_launch_hv32(const BatchArgs& a, int cand, int bucket, cudaStream_t st) {
  if (cand < 0 || cand >= kBatchCand32 || bucket < 0 || bucket >= kBatchBuckets)
    return fail(AED_ERR_INVALID, "batched apply: bad candidate or bucket");
  const int lo = bucket == 0 ? -1 : kBatchBucketHi[bucket - 1];
  const int hi = bucket + 1 == kBatchBuckets ? 0x7fffffff : kBatchBucketHi[bucket];
  kCand32[cand].kern<<<hv_grid(kCand32[cand].kern, a.hv_smem, &g_c32[cand], &g_c32_smem[cand]), kHvThreads,
                       a.hv_smem, st>>>(a, lo, hi);
  return check("batched FP32 apply");
}

// Time every FP32 candidate on the resident work of `bucket` (one warm-up and
// three timed launches each; the applies only rewrite y = H x of the current
// step, which the next step computes again) and return the fastest.
int batch_tune_bucket(const BatchArgs& a, int bucket, cudaStream_t st, int* best, float* best_ms) {
  cudaEvent_t e0, e1;
  AED_CUDA_TRY(cudaEventCreate(&e0));
  AED_CUDA_TRY(cudaEventCreate(&e1));
  int rc = AED_OK;
  *best = -1;
  *best_ms = 0.f;
  for (int c = 0; c < kBatchCand32 && !rc; ++c) {
    rc = batch_launch_hv32(a, c, bucket, st);
    if (!rc) AED_CUDA_TRY(cudaEventRecord(e0, st));
    for (int r = 0; r < 3 && !rc; ++r) rc = batch_launch_hv32(a, c, bucket, st);
    if (rc) break;
    AED_CUDA_TRY(cudaEventRecord(e1, st));
    AED_CUDA_TRY(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (*best < 0 || ms < *best_ms) {
      *best = c;
      *best_ms = ms;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

int batch_record_step(const BatchArgs& a, const int* choice32, cudaStream_t st) {
  const int ni = a.max_inst;
  const int gchunk = sms() * 8;
  for (int b = 0; b < kBatchBuckets; ++b) {
    const int rc = batch_launch_hv32(a, choice32[b], b, st);
    if (rc) return rc;
  }
  b_hv64<<<hv_grid(b_hv64, a.hv_smem, &g_hv64, &g_hv64_smem), kHvThreads, a.hv_smem, st>>>(a);
  b_alpha<<<ni, 256, 0, st>>>(a);
  b_update<<<gchunk, kRedThreads, 0, st>>>(a);
  b_beta<<<ni, 256, 0, st>>>(a);
  b_norm<<<gchunk, kRedThreads, 0, st>>>(a);
  b_advance<<<(ni + 127) / 128, 128, 0, st>>>(a);
  return check("batched Lanczos step");
}

int batch_record_check(const BatchArgs& a, cudaStream_t st) {
  const int ni = a.max_inst;
  const int gchunk = sms() * 8;
  b_check<<<(2 * ni + 31) / 32, 32, 0, st>>>(a);
  b_ritz<<<gchunk, kRedThreads, 0, st>>>(a);
  b_ritz_norm<<<ni, 256, 0, st>>>(a);
  b_ritz_scale<<<gchunk, kRedThreads, 0, st>>>(a);
  b_ritz_commit<<<(ni + 127) / 128, 128, 0, st>>>(a);
  return check("batched Lanczos check");
}

}  // namespace aed
