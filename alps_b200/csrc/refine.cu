// refine.cu -- kernels of the mixed path's Rayleigh-Ritz refinement.
//
// After the FP32 Lanczos phase the mixed solve forms K Ritz vectors in FP64
// from the stored FP32 basis (psi_k = sum_j z_k[j] v_j), applies H to each in
// FP64 (W_k = H psi_k), and solves the K x K projected problem
// (Psi^T H Psi) c = theta (Psi^T Psi) c on the host.  These kernels form the
// K Ritz vectors in one pass over the stored basis, the Gram matrices
// Psi^T Psi and Psi^T W in one pass over the 2K vectors, and the residual
// norms |sum_k c_k (W_k - theta psi_k)| of the Ritz pairs in one pass.  All
// sums use fixed chunks and a fixed tree (reduce.cuh), so the results are
// bit-reproducible.

#include <cuda_runtime.h>

#include <string>

#include "kernels.cuh"
#include "reduce.cuh"

namespace aed {
namespace {

constexpr int kCombThreads = 256;

struct ChunkSet {
  const float* p[kCombChunks];
};

// out_k[i] = (accumulate ? out_k[i] : 0) + sum_{j < mg} coef[k * m + j0 + j] v_j[i] for k < K, v_j the
// stored vector j of this launch's chunks: FP64 sums in ascending j, the coefficients of the launch in
// shared memory, a chunk's kMaxComb loads issued before their sums.
template <int K>
__global__ void __launch_bounds__(kCombThreads) ritz_combine_chunks_kernel(const __grid_constant__ ChunkSet V,
                                                                          int64_t ld, int mg, int m, int j0,
                                                                          const double* __restrict__ coef,
                                                                          VecSet out, int64_t n, bool accumulate) {
  extern __shared__ double cs[];  // [K][mg]
  for (int q = threadIdx.x; q < K * mg; q += kCombThreads) cs[q] = coef[(int64_t)(q / mg) * m + j0 + q % mg];
  __syncthreads();
  const int64_t stride = (int64_t)gridDim.x * kCombThreads;
  for (int64_t i = (int64_t)blockIdx.x * kCombThreads + threadIdx.x; i < n; i += stride) {
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = accumulate ? out.p[k][i] : 0.0;
    for (int j = 0; j < mg; j += kMaxComb) {
      const float* base = V.p[j / kMaxComb] + i;
      if (j + kMaxComb <= mg) {
        float v[kMaxComb];
#pragma unroll
        for (int u = 0; u < kMaxComb; ++u) v[u] = __ldg(base + (int64_t)u * ld);
#pragma unroll
        for (int u = 0; u < kMaxComb; ++u)
#pragma unroll
          for (int k = 0; k < K; ++k) acc[k] = fma(cs[k * mg + j + u], (double)v[u], acc[k]);
      } else {
        for (int u = 0; u < mg - j; ++u) {
          const double v = (double)__ldg(base + (int64_t)u * ld);
#pragma unroll
          for (int k = 0; k < K; ++k) acc[k] = fma(cs[k * mg + j + u], v, acc[k]);
        }
      }
    }
#pragma unroll
    for (int k = 0; k < K; ++k) out.p[k][i] = acc[k];
  }
}

// Chunk partials of <X_a, X_b> (a <= b) and <X_a, Y_b> (all a, b) for K
// vectors each: part[p * nch + c] for pair p in the order G(0,0), G(0,1), ...,
// G(K-1,K-1), A(0,0), A(0,1), ..., A(K-1,K-1).
template <int K>
__global__ void __launch_bounds__(kRedThreads) gram_partials_kernel(VecSet X, VecSet Y, int64_t n,
                                                                   double* __restrict__ part, int64_t nch) {
  constexpr int NG = K * (K + 1) / 2, NP = NG + K * K;
  __shared__ double sm[33];
  for (int64_t c = blockIdx.x; c < nch; c += gridDim.x) {
    const int64_t e0 = c * kRedChunk, e1 = e0 + kRedChunk < n ? e0 + kRedChunk : n;
    double acc[NP];
#pragma unroll
    for (int p = 0; p < NP; ++p) acc[p] = 0.0;
    for (int64_t i = e0 + threadIdx.x; i < e1; i += kRedThreads) {
      double x[K], y[K];
#pragma unroll
      for (int k = 0; k < K; ++k) {
        x[k] = __ldg(X.p[k] + i);
        y[k] = __ldg(Y.p[k] + i);
      }
      int p = 0;
#pragma unroll
      for (int a = 0; a < K; ++a)
#pragma unroll
        for (int b = a; b < K; ++b) {
          acc[p] = fma(x[a], x[b], acc[p]);
          ++p;
        }
#pragma unroll
      for (int a = 0; a < K; ++a)
#pragma unroll
        for (int b = 0; b < K; ++b) {
          acc[p] = fma(x[a], y[b], acc[p]);
          ++p;
        }
    }
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      const double tot = block_sum_all<kRedThreads>(acc[p], sm);
      if (threadIdx.x == 0) part[p * nch + c] = tot;
    }
  }
}

// Chunk partials of |r_i|^2, r_i = sum_k (cw[i][k] Y_k + cx[i][k] X_k), for
// the Ritz pairs i < R (coefficients in the kernel's parameters).
template <int K>
__global__ void __launch_bounds__(kRedThreads) resid_partials_kernel(VecSet X, VecSet Y, ResidCoef rc, int R,
                                                                    int64_t n, double* __restrict__ part,
                                                                    int64_t nch) {
  __shared__ double sm[33];
  for (int64_t c = blockIdx.x; c < nch; c += gridDim.x) {
    const int64_t e0 = c * kRedChunk, e1 = e0 + kRedChunk < n ? e0 + kRedChunk : n;
    double acc[K];
#pragma unroll
    for (int r = 0; r < K; ++r) acc[r] = 0.0;
    for (int64_t i = e0 + threadIdx.x; i < e1; i += kRedThreads) {
      double x[K], y[K];
#pragma unroll
      for (int k = 0; k < K; ++k) {
        x[k] = __ldg(X.p[k] + i);
        y[k] = __ldg(Y.p[k] + i);
      }
#pragma unroll
      for (int r = 0; r < K; ++r) {
        if (r < R) {
          double t = 0.0;
#pragma unroll
          for (int k = 0; k < K; ++k) t = fma(rc.cw[r][k], y[k], fma(rc.cx[r][k], x[k], t));
          acc[r] = fma(t, t, acc[r]);
        }
      }
    }
#pragma unroll
    for (int r = 0; r < K; ++r) {
      if (r < R) {
        const double tot = block_sum_all<kRedThreads>(acc[r], sm);
        if (threadIdx.x == 0) part[r * nch + c] = tot;
      }
    }
  }
}

// Chunk partials of <V_k, w> for the m <= kMaxComb stored FP32 vectors of one
// store chunk (stride ld) and an FP32 vector w: part[(k0 + k) * pstride + c],
// FP64 sums in chunk c's thread order and block tree.
__global__ void __launch_bounds__(kRedThreads) block_dot_partials_kernel(const float* __restrict__ V, int64_t ld,
                                                                        int m, const float* __restrict__ w,
                                                                        int64_t n, double* __restrict__ part,
                                                                        int k0, int64_t pstride) {
  __shared__ double sm[33];
  const int64_t nch = (n + kRedChunk - 1) / kRedChunk;
  for (int64_t c = blockIdx.x; c < nch; c += gridDim.x) {
    const int64_t e0 = c * kRedChunk, e1 = e0 + kRedChunk < n ? e0 + kRedChunk : n;
    double acc[kMaxComb];
#pragma unroll
    for (int k = 0; k < kMaxComb; ++k) acc[k] = 0.0;
    for (int64_t i = e0 + threadIdx.x; i < e1; i += kRedThreads) {
      const double wv = (double)__ldg(w + i);
#pragma unroll
      for (int k = 0; k < kMaxComb; ++k)
        if (k < m) acc[k] = fma((double)__ldg(V + (int64_t)k * ld + i), wv, acc[k]);
    }
#pragma unroll
    for (int k = 0; k < kMaxComb; ++k) {
      if (k < m) {
        const double tot = block_sum_all<kRedThreads>(acc[k], sm);
        if (threadIdx.x == 0) part[(int64_t)(k0 + k) * pstride + c] = tot;
      }
    }
  }
}

// w = (float)((double)w - t)
__global__ void sub_round_kernel(const double* __restrict__ t, float* __restrict__ w, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    w[i] = __double2float_rn((double)w[i] - t[i]);
}

// out[p] = sum of part[p * nch .. p * nch + nch) for p < np (one CTA each, finish_sum's order).
__global__ void __launch_bounds__(kFinishThreads) finish_many_kernel(const double* __restrict__ part, int64_t nch,
                                                                     double* __restrict__ out) {
  finish_sum(part + (int64_t)blockIdx.x * nch, nch, out + blockIdx.x, false);
}

int grid_for(int64_t nch) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t cap = (int64_t)sms * 4;
  return (int)(nch < 1 ? 1 : (nch < cap ? nch : cap));
}

}  // namespace

int launch_ritz_combine_chunks(const float* const* chunks, int64_t ld, int m, const double* coef, int K,
                               const VecSet& out, int64_t n, cudaStream_t st) {
  if (m < 1 || K < 1 || K > kMaxRR) return fail(AED_ERR_INVALID, "ritz_combine_chunks: bad sizes");
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t want = (n + kCombThreads - 1) / kCombThreads, cap = (int64_t)sms * 8;
  const int grid = (int)(want < 1 ? 1 : (want < cap ? want : cap));
  constexpr int kGroup = kCombChunks * kMaxComb;  // vectors per launch
  for (int j0 = 0; j0 < m; j0 += kGroup) {
    const int mg = m - j0 < kGroup ? m - j0 : kGroup;
    ChunkSet cs{};
    for (int c = 0; c < (mg + kMaxComb - 1) / kMaxComb; ++c) cs.p[c] = chunks[j0 / kMaxComb + c];
    const size_t smem = (size_t)K * mg * sizeof(double);  // at most 32 KB
    switch (K) {
#define AED_CASE(k)                                                                                   \
  case k:                                                                                             \
    ritz_combine_chunks_kernel<k><<<grid, kCombThreads, smem, st>>>(cs, ld, mg, m, j0, coef, out, n, j0 > 0); \
    break;
      AED_CASE(1) AED_CASE(2) AED_CASE(3) AED_CASE(4) AED_CASE(5) AED_CASE(6) AED_CASE(7) AED_CASE(8)
#undef AED_CASE
      default: return fail(AED_ERR_INVALID, "ritz_combine_chunks: K");
    }
    if (int rc = check_launch_counted("ritz_combine_chunks_kernel")) return rc;
  }
  return AED_OK;
}

int launch_gram(const VecSet& X, const VecSet& Y, int K, int64_t n, double* part, double* out, cudaStream_t st) {
  const int64_t nch = red_chunks(n);
  const int grid = grid_for(nch);
  switch (K) {
#define AED_CASE(k) case k: gram_partials_kernel<k><<<grid, kRedThreads, 0, st>>>(X, Y, n, part, nch); break;
    AED_CASE(1) AED_CASE(2) AED_CASE(3) AED_CASE(4) AED_CASE(5) AED_CASE(6) AED_CASE(7) AED_CASE(8)
#undef AED_CASE
    default: return fail(AED_ERR_INVALID, "gram: K");
  }
  int rc = check_launch_counted("gram_partials_kernel");
  if (rc) return rc;
  const int np = K * (K + 1) / 2 + K * K;
  finish_many_kernel<<<np, kFinishThreads, 0, st>>>(part, nch, out);
  return check_launch_counted("finish_many_kernel");
}

int launch_resid(const VecSet& X, const VecSet& Y, const ResidCoef& rcoef, int K, int R, int64_t n, double* part,
                 double* out, cudaStream_t st) {
  if (R < 1 || R > K) return fail(AED_ERR_INVALID, "resid: R");
  const int64_t nch = red_chunks(n);
  const int grid = grid_for(nch);
  switch (K) {
#define AED_CASE(k) \
  case k: resid_partials_kernel<k><<<grid, kRedThreads, 0, st>>>(X, Y, rcoef, R, n, part, nch); break;
    AED_CASE(1) AED_CASE(2) AED_CASE(3) AED_CASE(4) AED_CASE(5) AED_CASE(6) AED_CASE(7) AED_CASE(8)
#undef AED_CASE
    default: return fail(AED_ERR_INVALID, "resid: K");
  }
  int rc = check_launch_counted("resid_partials_kernel");
  if (rc) return rc;
  finish_many_kernel<<<R, kFinishThreads, 0, st>>>(part, nch, out);
  return check_launch_counted("finish_many_kernel");
}

int launch_block_dot(const float* V, int64_t ld, int m, const float* w, int64_t n, double* part, int k0,
                     cudaStream_t st) {
  if (m < 1 || m > kMaxComb) return fail(AED_ERR_INVALID, "block_dot: bad sizes");
  const int64_t nch = red_chunks(n);
  block_dot_partials_kernel<<<grid_for(nch), kRedThreads, 0, st>>>(V, ld, m, w, n, part, k0, nch);
  return check_launch_counted("block_dot_partials_kernel");
}

int launch_finish_many(const double* part, int64_t nch, int np, double* out, cudaStream_t st) {
  if (np < 1) return AED_OK;
  finish_many_kernel<<<np, kFinishThreads, 0, st>>>(part, nch, out);
  return check_launch_counted("finish_many_kernel");
}

int launch_sub_round(const double* t, float* w, int64_t n, cudaStream_t st) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t want = (n + 255) / 256, cap = (int64_t)sms * 8;
  sub_round_kernel<<<(int)(want < 1 ? 1 : (want < cap ? want : cap)), 256, 0, st>>>(t, w, n);
  return check_launch_counted("sub_round_kernel");
}

}  // namespace aed
