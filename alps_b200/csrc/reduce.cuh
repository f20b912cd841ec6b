// reduce.cuh -- deterministic reductions shared by the engine's kernels.
//
// Sums are formed over fixed chunks of kRedChunk elements: chunk c is always
// reduced by one CTA of kRedThreads threads in the same thread order and the
// same shuffle tree, whatever the grid, and the chunk partials are then summed
// by one CTA of kFinishThreads threads in a fixed order.  Every total is
// therefore reproducible bit for bit, on any GPU and any launch shape.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.cuh"

namespace aed {

constexpr int kFinishThreads = 1024;

// Block reduction: warp shuffles, then warp 0 over the warp sums; the total is
// returned to every thread.  sm needs 33 doubles.
template <int NT>
__device__ __forceinline__ double block_sum_all(double v, double* sm) {
  static_assert(NT % 32 == 0 && NT <= 1024, "block size");
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sm[w] = v;
  __syncthreads();
  if (w == 0) {
    double r = (l < NT / 32) ? sm[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    if (l == 0) sm[32] = r;
  }
  __syncthreads();
  const double r = sm[32];
  __syncthreads();
  return r;
}

// part[c] = sum over chunk c of x_i * y_i (x_i^2 when sq), for every chunk
// this CTA takes (c = blockIdx.x, blockIdx.x + gridDim.x, ...).
template <typename T>
__device__ __forceinline__ void chunk_dot_partials(const T* __restrict__ x, const T* __restrict__ y, int64_t n,
                                                   double* __restrict__ part, bool sq) {
  __shared__ double sm[33];
  const int64_t nch = (n + kRedChunk - 1) / kRedChunk;
  for (int64_t c = blockIdx.x; c < nch; c += gridDim.x) {
    const int64_t e0 = c * kRedChunk, e1 = e0 + kRedChunk < n ? e0 + kRedChunk : n;
    double acc = 0.0;
    for (int64_t i = e0 + threadIdx.x; i < e1; i += kRedThreads) {
      const double a = (double)x[i];
      acc = fma(a, sq ? a : (double)y[i], acc);
    }
    const double tot = block_sum_all<kRedThreads>(acc, sm);
    if (threadIdx.x == 0) part[c] = tot;
  }
}

// *out = sum of part[0..n) (sqrt of it when take_sqrt); one CTA of kFinishThreads.
__device__ __forceinline__ void finish_sum(const double* __restrict__ part, int64_t n, double* __restrict__ out,
                                           bool take_sqrt) {
  __shared__ double sm[33];
  double v = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += kFinishThreads) v += part[i];
  const double tot = block_sum_all<kFinishThreads>(v, sm);
  if (threadIdx.x == 0) *out = take_sqrt ? sqrt(tot) : tot;
}

// The total finish_sum forms, computed by any CTA of NT threads (NT a
// multiple of 32 dividing kFinishThreads) and returned to every thread: real
// warp r plays the kFinishThreads / NT virtual warps r, r + NT/32, ...; each
// virtual thread sums its strided share and each virtual warp its shuffle
// tree exactly as in finish_sum, so the result is bit-identical.  For short
// partial lists, where every CTA of a kernel can afford to read them all.
template <int NT>
__device__ __forceinline__ double finish_sum_in_cta(const double* __restrict__ part, int64_t n, double* sm) {
  static_assert(NT % 32 == 0 && kFinishThreads % NT == 0, "block size");
  constexpr int kVirt = kFinishThreads / NT;  // virtual warps per real warp
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  for (int q = 0; q < kVirt; ++q) {
    const int vw = w + q * (NT / 32);  // virtual warp
    const int vt = vw * 32 + l;        // virtual thread of finish_sum
    double v = 0.0;
    for (int64_t i = vt; i < n; i += kFinishThreads) v += part[i];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (l == 0) sm[vw] = v;
  }
  __syncthreads();
  if (w == 0) {
    double r = sm[l];  // kFinishThreads / 32 = 32 virtual warp sums
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    if (l == 0) sm[32] = r;
  }
  __syncthreads();
  const double r = sm[32];
  __syncthreads();
  return r;
}

}  // namespace aed
