// kernels.cu -- sm_100a kernels of the exact-diagonalisation engine.
//
// The apply y = H x is matrix-free: each thread owns one row (one basis
// state s), walks the coupling tables held in the kernel's parameter space and
// gathers x at the rank of every reachable state s' = s ^ (bit pair).  Ranks
// come from the two-table (Lin) scheme rank(s) = thi[s >> Nlo] + tlo[s & lomask].
// No tensor cores: the apply is a bandwidth-bound gather.
//
// Reference paths are relative to the ALPS source tree.

#include <cuda_runtime.h>

#include <atomic>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <type_traits>

#include "apply.cuh"
#include "apply_blocks.cuh"
#include "apply_stream.cuh"
#include "kernels.cuh"
#include "reduce.cuh"

namespace aed {
namespace {
using apply::AccExact64;
using apply::AccTwoSum32;
using apply::AccWide32;
using apply::kTileRows;

// y = H x.  Tiles are taken in a static round robin; alpha_part (optional)
// receives one partial sum of x_i * y_i per tile, so the reduction does not
// depend on the grid.  R rows per thread per pass, MINB CTAs per SM.
template <typename T, typename Acc, int R, int MINB>
__global__ void __launch_bounds__(kHvThreads, MINB) hv_kernel(const __grid_constant__ HvParams P, const DevTables t,
                                                              const T* __restrict__ x, T* __restrict__ y,
                                                              double* __restrict__ alpha_part) {
  __shared__ apply::ApplySmem sm;
  apply::stage_pairs(P, sm);
  const apply::ApplyCtx c = apply::ctx_of(P);
  for (int64_t it = blockIdx.x; it < t.n_tiles; it += gridDim.x) apply::apply_tile<T, Acc, R>(c, t, it, x, y, alpha_part, sm);
}

// y = H x over bundles of B hi blocks with x staged in shared memory (dynamic:
// B * maxrows values).  Bundles are taken in a static round robin; the block
// list puts the largest blocks first.
template <typename T, typename Acc, int R, int B, int MINB>
__global__ void __launch_bounds__(kHvThreads, MINB) hvb_kernel(const __grid_constant__ HvParams P, const DevTables t,
                                                               const T* __restrict__ x, T* __restrict__ y,
                                                               double* __restrict__ alpha_part) {
  extern __shared__ __align__(16) unsigned char hvb_dyn[];
  __shared__ bapply::BundleSmem<B> sm;
  T* xs = bapply::carve<T, B>(P, t, hvb_dyn, sm);
  bapply::stage_pairs<B>(P, sm);
  const apply::ApplyCtx c = apply::ctx_of(P);
  const int64_t nb = t.n_blk / B;
  int rc = 0;
  for (int64_t ub = blockIdx.x; ub < nb; ub += gridDim.x)
    bapply::apply_bundle<T, Acc, R, B>(c, t, ub, x, y, alpha_part, sm, xs, rc);
}

// y = H x with the flips' x segments staged by bulk copies (apply_stream.cuh).
using sapply::hvs_kernel;

// Diagonal M(i,i) of every row, accumulated in the reference's term order
// (site terms, then bonds; hamiltonian_matrix.hpp:387-397 starting from the
// 0 of initialized_matrix, :53-56).  Run once per handle.
__global__ void __launch_bounds__(256) diag_table_kernel(const __grid_constant__ HvParams P, const DevTables t,
                                                         double* __restrict__ dg) {
  for (int64_t it = blockIdx.x; it < t.n_tiles; it += gridDim.x) {
    const uint32_t h = t.tile_h[it];
    const int k = P.n_up - __popc(h);
    const uint32_t lbase = t.looff[k];
    const uint32_t rows = t.looff[k + 1] - lbase;
    const uint32_t r0 = t.tile_r[it];
    for (uint32_t r = r0 + threadIdx.x; r < rows && r < r0 + kTileRows; r += 256) {
      const uint32_t s = (h << P.Nlo) | t.lolist[lbase + r];
      double d = 0.0;
      for (int q = 0; q < P.n_diag; ++q) {
        const bool eq = ((s & P.diag[q].m1) != 0u) == ((s & P.diag[q].m2) != 0u);
        d = __dadd_rn(d, eq ? P.diag[q].veq : P.diag[q].vne);
      }
      dg[t.thi[h] + r] = d;
    }
  }
}

// basis_states order (basisstates.h:175-278) from the tables: row idx lies in
// the hi block h with the largest thi[h] <= idx.
__global__ void basis_copy_kernel(const DevTables t, uint32_t* __restrict__ out, int64_t offset, int64_t count) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= count) return;
  const uint32_t idx = (uint32_t)(offset + n);
  uint32_t lo = 0, hi = (1u << t.Nhi) - 1u;
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo + 1) / 2;
    if (t.thi[mid] <= idx)
      lo = mid;
    else
      hi = mid - 1;
  }
  const uint32_t h = lo;
  const uint32_t r = idx - t.thi[h];
  const int k = t.n_up - __popc(h);
  out[n] = (h << t.Nlo) | t.lolist[t.looff[k] + r];
}

// basis_states::index (basisstates.h:68-74): D when the state is not in the sector.
__global__ void rank_kernel(const DevTables t, int N, const uint32_t* __restrict__ st, int64_t count,
                            int64_t* __restrict__ out) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= count) return;
  const uint32_t s = st[n];
  const bool outside = (N < 32 && (s >> N) != 0u) || __popc(s) != t.n_up;
  out[n] = outside ? t.D : (int64_t)(t.thi[s >> t.Nlo] + t.tlo[s & ((1u << t.Nlo) - 1u)]);
}

// splitmix64 (Steele, Lea & Flood, OOPSLA 2014)
__device__ __forceinline__ uint64_t splitmix64(uint64_t seed, uint64_t i) {
  uint64_t z = seed + 0x9E3779B97F4A7C15ull * (i + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

template <typename T>
__global__ void fill_random_kernel(T* __restrict__ x, int64_t n, uint64_t seed) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t z = splitmix64(seed, (uint64_t)i);
    if constexpr (sizeof(T) == 8)
      x[i] = (double)(z >> 11) * 0x1.0p-53;
    else
      x[i] = (float)((double)(z >> 40) * 0x1.0p-24);
  }
}

// y = (float) x, round to nearest
__global__ void round_to_f32_kernel(const double* __restrict__ x, float* __restrict__ y, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = __double2float_rn(x[i]);
}

template <typename T>
__global__ void copy_kernel(const T* __restrict__ x, T* __restrict__ y, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = x[i];
}

// y += a*x, as ublas evaluates v += s*w: the product rounds, then the sum.
template <typename T>
__global__ void axpy_kernel(double a, const T* __restrict__ x, T* __restrict__ y, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = (T)__dadd_rn((double)y[i], __dmul_rn(a, (double)x[i]));
}

template <typename T>
__global__ void scal_kernel(double a, T* __restrict__ x, int64_t n, bool divide) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = (T)(divide ? __ddiv_rn((double)x[i], a) : __dmul_rn((double)x[i], a));
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads) dot_partials_kernel(const T* __restrict__ x, const T* __restrict__ y,
                                                                  int64_t n, double* __restrict__ part, bool sq) {
  chunk_dot_partials<T>(x, y, n, part, sq);
}

__global__ void __launch_bounds__(kFinishThreads) finish_sum_kernel(const double* __restrict__ part, int64_t n,
                                                                    double* __restrict__ out, bool take_sqrt) {
  finish_sum(part, n, out, take_sqrt);
}

// This thread's elements e0 + threadIdx.x + u kRedThreads of the chunk [e0, e1) of the update
// w = (y - a x) - b v_prev (stored into y), and the sum of their w^2 in element order.  FP32 vectors
// in a full chunk issue all their loads before the arithmetic (4-byte loads leave too few bytes in
// flight otherwise); the arithmetic and the order of the sum are the same, so are the bits.
template <typename T>
__device__ __forceinline__ double update_chunk(double alpha, double b, const T* __restrict__ x,
                                               const T* __restrict__ vprev, T* __restrict__ y, int64_t e0,
                                               int64_t e1) {
  double acc = 0.0;
  if constexpr (sizeof(T) == 4) {
    constexpr int U = (int)(kRedChunk / kRedThreads);
    if (e1 - e0 == kRedChunk) {
      const int64_t i0 = e0 + threadIdx.x;
      T yv[U], xv[U], pv[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        yv[u] = y[i0 + u * kRedThreads];
        xv[u] = x[i0 + u * kRedThreads];
        pv[u] = vprev ? vprev[i0 + u * kRedThreads] : T(0);
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        double w = __dsub_rn((double)yv[u], __dmul_rn(alpha, (double)xv[u]));
        if (vprev) w = __dsub_rn(w, __dmul_rn(b, (double)pv[u]));
        const T wt = (T)w;
        y[i0 + u * kRedThreads] = wt;
        acc = fma((double)wt, (double)wt, acc);
      }
      return acc;
    }
  }
  for (int64_t i = e0 + threadIdx.x; i < e1; i += kRedThreads) {
    double w = __dsub_rn((double)y[i], __dmul_rn(alpha, (double)x[i]));
    if (vprev) w = __dsub_rn(w, __dmul_rn(b, (double)vprev[i]));
    const T wt = (T)w;
    y[i] = wt;
    acc = fma((double)wt, (double)wt, acc);
  }
  return acc;
}

// y /= beta over the grid-stride elements of this thread; each element is
// divided on its own, so the grouping below does not change the bits.  FP32:
// four elements loaded before dividing (float4 vectors measured slower);
// FP64: 16-byte double2 vectors, two in flight, when y is 16-byte aligned,
// then the tail element by element.
template <typename T>
__device__ __forceinline__ void normalize_elems(double beta, T* __restrict__ y, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * kRedThreads;
  int64_t i = blockIdx.x * (int64_t)kRedThreads + threadIdx.x;
  if constexpr (sizeof(T) == 4) {
    constexpr int U = 4;
    for (; i + (U - 1) * stride < n; i += U * stride) {
      T v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) v[u] = y[i + u * stride];
#pragma unroll
      for (int u = 0; u < U; ++u) y[i + u * stride] = (T)__ddiv_rn((double)v[u], beta);
    }
  } else if ((reinterpret_cast<uintptr_t>(y) & 15u) == 0) {
    const int64_t nv = n / 2, t0 = i;
    double2* yv = reinterpret_cast<double2*>(y);
    int64_t k = t0;
    for (; k + stride < nv; k += 2 * stride) {
      double2 a = yv[k], b = yv[k + stride];
      a.x = __ddiv_rn(a.x, beta);
      a.y = __ddiv_rn(a.y, beta);
      b.x = __ddiv_rn(b.x, beta);
      b.y = __ddiv_rn(b.y, beta);
      yv[k] = a;
      yv[k + stride] = b;
    }
    for (; k < nv; k += stride) {
      double2 a = yv[k];
      a.x = __ddiv_rn(a.x, beta);
      a.y = __ddiv_rn(a.y, beta);
      yv[k] = a;
    }
    i = nv * 2 + t0;
  }
  for (; i < n; i += stride) y[i] = (T)__ddiv_rn((double)y[i], beta);
}

// make_step middle part (lanczos.h:398-401): w -= a v; w -= b v_prev; chunk partials of |w|^2
template <typename T>
__global__ void __launch_bounds__(kRedThreads) lanczos_update_kernel(const double* __restrict__ alpha_p,
                                                                    const T* __restrict__ x,
                                                                    const T* __restrict__ vprev,
                                                                    const double* __restrict__ beta_prev,
                                                                    T* __restrict__ y, int64_t n,
                                                                    double* __restrict__ partB) {
  __shared__ double sm[33];
  const double alpha = *alpha_p;
  const double b = vprev ? *beta_prev : 0.0;
  const int64_t nch = (n + kRedChunk - 1) / kRedChunk;
  for (int64_t c = blockIdx.x; c < nch; c += gridDim.x) {
    const int64_t e0 = c * kRedChunk, e1 = min(n, e0 + kRedChunk);
    const double acc = update_chunk(alpha, b, x, vprev, y, e0, e1);
    const double tot = block_sum_all<kRedThreads>(acc, sm);
    if (threadIdx.x == 0) partB[c] = tot;
  }
}

// The update with alpha's finishing sum folded in: every CTA sums the
// apply's tile partials itself (the order of finish_sum, so the same alpha to
// the bit) and CTA 0 stores it.  For sectors with few tiles, where this saves
// a launch per step.
template <typename T>
__global__ void __launch_bounds__(kRedThreads) lanczos_update_fin_kernel(
    const double* __restrict__ alpha_part, int64_t n_apart, double* __restrict__ alpha_out, const T* __restrict__ x,
    const T* __restrict__ vprev, const double* __restrict__ beta_prev, T* __restrict__ y, int64_t n,
    double* __restrict__ partB) {
  __shared__ double sm[33];
  const double alpha = finish_sum_in_cta<kRedThreads>(alpha_part, n_apart, sm);
  if (blockIdx.x == 0 && threadIdx.x == 0) *alpha_out = alpha;
  const double b = vprev ? *beta_prev : 0.0;
  const int64_t nch = (n + kRedChunk - 1) / kRedChunk;
  for (int64_t c = blockIdx.x; c < nch; c += gridDim.x) {
    const int64_t e0 = c * kRedChunk, e1 = min(n, e0 + kRedChunk);
    const double acc = update_chunk(alpha, b, x, vprev, y, e0, e1);
    const double tot = block_sum_all<kRedThreads>(acc, sm);
    if (threadIdx.x == 0) partB[c] = tot;
  }
}

// The normalisation with beta's finishing sum folded in (as above).
template <typename T>
__global__ void __launch_bounds__(kRedThreads) lanczos_normalize_fin_kernel(const double* __restrict__ beta_part,
                                                                           int64_t n_bpart,
                                                                           double* __restrict__ beta_out,
                                                                           T* __restrict__ y, int64_t n) {
  __shared__ double sm[33];
  const double beta = sqrt(finish_sum_in_cta<kRedThreads>(beta_part, n_bpart, sm));
  if (blockIdx.x == 0 && threadIdx.x == 0) *beta_out = beta;
  normalize_elems(beta, y, n);
}

// make_step tail (lanczos.h:402): w /= b
template <typename T>
__global__ void __launch_bounds__(kRedThreads) lanczos_normalize_kernel(const double* __restrict__ beta_p,
                                                                       T* __restrict__ y, int64_t n) {
  const double beta = *beta_p;
  normalize_elems(beta, y, n);
}

// Ritz vector from the stored FP32 Lanczos basis, accumulated in FP64.
// Each thread owns elements i (coalesced across the warp) and walks the m
// stored vectors; coefficients are staged in shared memory in chunks.
__global__ void __launch_bounds__(256) ritz_combine_kernel(const float* __restrict__ V, int64_t ld, int m,
                                                          const double* __restrict__ coef, double* __restrict__ out,
                                                          int64_t n, bool accumulate) {
  __shared__ double cs[512];
  const int64_t stride = (int64_t)gridDim.x * 256;
  for (int64_t base = (int64_t)blockIdx.x * 256; base < n; base += stride) {
    const int64_t i = base + threadIdx.x;
    double acc = 0.0;
    for (int j0 = 0; j0 < m; j0 += 512) {
      const int cnt = min(512, m - j0);
      __syncthreads();
      for (int q = threadIdx.x; q < cnt; q += 256) cs[q] = coef[j0 + q];
      __syncthreads();
      if (i < n)
        for (int q = 0; q < cnt; ++q) acc = fma(cs[q], (double)__ldg(V + (int64_t)(j0 + q) * ld + i), acc);
    }
    if (i < n) out[i] = accumulate ? out[i] + acc : acc;
  }
}

std::atomic<int64_t> g_launches{0};

int num_sms() {
  static const int n = [] {  // thread-safe one-time initialisation
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return v > 0 ? v : 148;
  }();
  return n;
}

inline int elem_grid(int64_t n) {
  const int64_t want = (n + 255) / 256;
  const int64_t cap = (int64_t)num_sms() * 8;
  return (int)(want < 1 ? 1 : (want > cap ? cap : want));
}

inline int check_launch(const char* what) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(AED_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return AED_OK;
}

}  // namespace

int64_t launch_count() { return g_launches.load(); }

int check_launch_counted(const char* what) { return check_launch(what); }

int launch_ritz_combine(const float* V, int64_t ld, int m, const double* coef, double* out, int64_t n,
                        bool accumulate, cudaStream_t st) {
  if (m < 1 || m > kMaxRitzTerms) return fail(AED_ERR_INVALID, "ritz_combine: bad number of terms");
  ritz_combine_kernel<<<elem_grid(n), 256, 0, st>>>(V, ld, m, coef, out, n, accumulate);
  return check_launch("ritz_combine_kernel");
}

// ---- apply variants -------------------------------------------------------------
// Tile apply (apply.cuh): R rows per thread, MINB CTAs per SM.  Bundle apply
// (apply_blocks.cuh): B hi blocks per CTA with x in shared memory.
struct HvVariant {
  int B, R, minb;  // B = 0: tile apply; B = -1: stream apply (R = rows per thread, minb = own-x buffers)
  const char* name;
};
constexpr HvVariant kVariants[] = {
    {0, 4, 6, "r4b6"},      {0, 4, 5, "r4b5"},      {0, 4, 4, "r4b4"},      {0, 2, 8, "r2b8"},
    {0, 2, 6, "r2b6"},      {0, 8, 3, "r8b3"},      {1, 4, 3, "blk1r4b3"},  {2, 2, 4, "blk2r2b4"},
    {2, 4, 2, "blk2r4b2"},  {2, 2, 3, "blk2r2b3"},  {1, 4, 4, "blk1r4b4"},  {1, 2, 4, "blk1r2b4"},
    {-1, 14, 2, "str14o2"}, {-1, 14, 1, "str14o1"}, {-1, 26, 2, "str26o2"}, {-1, 26, 1, "str26o1"},
    {-1, 14, 1, "str14w"},  {-1, 26, 1, "str26w"},  // FP32: own x widened once
};
constexpr int kNumVariants = (int)(sizeof(kVariants) / sizeof(kVariants[0]));

// Launch shapes are computed once per kernel (and per shared-memory size or
// sector shape) and kept in maps guarded by g_grid_mu: handles on several host
// threads launch the same kernels.  The dynamic shared-memory limit of a
// kernel is raised once, to the most the device allows, so that a launch on
// one thread never sees another thread's smaller limit.
std::mutex g_grid_mu;

template <typename K>
int raise_smem_limit(K kern, size_t* static_bytes) {
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa{};
  if (cudaFuncGetAttributes(&fa, kern) != cudaSuccess) {
    const cudaError_t e = cudaGetLastError();
    return fail(AED_ERR_CUDA, std::string("kernel attributes: ") + cudaGetErrorString(e));
  }
  const int most = optin - (int)fa.sharedSizeBytes;
  if (most > 0 && cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, most) != cudaSuccess) {
    const cudaError_t e = cudaGetLastError();
    return fail(AED_ERR_CUDA, std::string("kernel shared memory limit: ") + cudaGetErrorString(e));
  }
  *static_bytes = fa.sharedSizeBytes;
  return most > 0 ? AED_OK : kVariantNotApplicable;
}

template <typename T, typename Acc, int R, int B>
int launch_one(const HvParams& P, const DevTables& t, const T* x, T* y, double* alpha_part, cudaStream_t st) {
  static int grid_all = 0;
  int grid;
  {
    std::lock_guard<std::mutex> lk(g_grid_mu);
    if (grid_all <= 0) {
      int per_sm = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hv_kernel<T, Acc, R, B>, kHvThreads, 0);
      grid_all = num_sms() * (per_sm < 1 ? 1 : per_sm);
    }
    grid = grid_all;
  }
  if (grid > t.n_tiles) grid = (int)t.n_tiles;
  hv_kernel<T, Acc, R, B><<<grid, kHvThreads, 0, st>>>(P, t, x, y, alpha_part);
  return check_launch("hv_kernel");
}

// Bundle apply: grid from the occupancy at this sector's dynamic shared
// memory (sectors of one process share a few sizes).
template <typename T, typename Acc, int R, int B, int MINB>
int launch_bundle(const HvParams& P, const DevTables& t, const T* x, T* y, double* alpha_part, cudaStream_t st) {
  if (!t.blk_h || t.maxrows <= 0) return kVariantNotApplicable;
  const size_t dyn = bapply::bundle_smem_bytes<T>(B, t.maxrows, P.n_pairs, P.n_lolo);
  auto kern = hvb_kernel<T, Acc, R, B, MINB>;
  static int limit_rc = -1;
  static size_t static_bytes = 0;
  static std::map<size_t, int> grids;  // dyn -> grid (0: does not fit)
  int grid = 0;
  {
    std::lock_guard<std::mutex> lk(g_grid_mu);
    if (limit_rc < 0) limit_rc = raise_smem_limit(kern, &static_bytes);
    if (limit_rc == AED_ERR_CUDA) return limit_rc;
    auto it = grids.find(dyn);
    if (it == grids.end()) {
      int per_sm = 0;
      int dev = 0, optin = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
      if (limit_rc == AED_OK && static_bytes + dyn <= (size_t)optin)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kHvThreads, dyn);
      it = grids.emplace(dyn, per_sm < 1 ? 0 : num_sms() * per_sm).first;
    }
    grid = it->second;
  }
  if (grid <= 0) return kVariantNotApplicable;
  int64_t g = grid;
  const int64_t nb = t.n_blk / B;
  if (g > nb) g = nb;
  if (g < 1) return AED_OK;
  kern<<<(unsigned)g, kHvThreads, dyn, st>>>(P, t, x, y, alpha_part);
  return check_launch("hvb_kernel");
}

// Stream apply: one CTA per SM with OB own-x buffers and as many ring stages
// as the shared memory holds (at most sapply::kMaxStages).  Not applicable to
// sectors whose blocks need more than U rows per thread, to lo parts under
// 8 bits (the crossing-table rows must be 16-byte multiples), or to vectors
// that are not 16-byte aligned (bulk copies).
struct StreamShape {
  sapply::StreamCfg cfg{};
  size_t dyn = 0;
  bool fits = false;
};

template <typename T, typename Acc, int U, bool kOwnD>
int launch_stream(int OB, const HvParams& P, const DevTables& t, const T* x, T* y, double* alpha_part,
                  cudaStream_t st) {
  if constexpr (kOwnD && sizeof(T) != 4) {
    return kVariantNotApplicable;  // FP64 rows read their own x as it is
  } else {
  if (!t.blk_h || !t.flag || t.maxrows <= 0 || t.Nlo < 8 || t.Nlo > 16) return kVariantNotApplicable;
  if ((t.maxrows + kHvThreads - 1) / kHvThreads > U) return kVariantNotApplicable;
  if ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y) | reinterpret_cast<uintptr_t>(t.xtab)) & 15u)
    return kVariantNotApplicable;
  auto kern = hvs_kernel<T, Acc, U, kOwnD>;
  static int limit_rc = -1;
  static size_t static_bytes = 0;
  static std::map<std::pair<int, int>, StreamShape> shapes;  // (maxrows, OB) -> shape
  StreamShape sh;
  {
    std::lock_guard<std::mutex> lk(g_grid_mu);
    if (limit_rc < 0) limit_rc = raise_smem_limit(kern, &static_bytes);
    if (limit_rc == AED_ERR_CUDA) return limit_rc;
    const auto key = std::make_pair(t.maxrows, OB);
    auto it = shapes.find(key);
    if (it == shapes.end()) {
      StreamShape n;
      int dev = 0, optin = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
      n.cfg.own_bytes = (uint32_t)bapply::bundle_align16((size_t)t.maxrows * sizeof(T) + 32);
      n.cfg.xoff = n.cfg.own_bytes;
      n.cfg.stage_bytes = n.cfg.xoff + (uint32_t)bapply::bundle_align16((size_t)t.maxrows * 2 + 32);
      const uint32_t ownd_bytes = kOwnD ? (uint32_t)bapply::bundle_align16((size_t)t.maxrows * 8 + 32) : 0u;
      n.cfg.ownd_off = (uint32_t)OB * n.cfg.own_bytes;
      n.cfg.ring_off = n.cfg.ownd_off + ownd_bytes;
      const int64_t avail = (int64_t)optin - (int64_t)static_bytes - 1024;
      const int64_t S = (avail - (int64_t)n.cfg.ring_off) / (int64_t)n.cfg.stage_bytes;
      if (limit_rc == AED_OK && S >= 2) {
        n.cfg.S = (int)(S < sapply::kMaxStages ? S : sapply::kMaxStages);
        n.cfg.OB = OB;
        n.dyn = (size_t)n.cfg.ring_off + (size_t)n.cfg.S * n.cfg.stage_bytes;
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, sapply::kThreads, n.dyn);
        n.fits = per_sm >= 1;
      }
      it = shapes.emplace(key, n).first;
    }
    sh = it->second;
  }
  if (!sh.fits) return kVariantNotApplicable;
  sapply::StreamCfg cfg = sh.cfg;
  cfg.flag = t.flag;
  int64_t grid = num_sms();
  if (grid > t.n_blk) grid = t.n_blk;
  if (grid < 1) return AED_OK;
  kern<<<(unsigned)grid, sapply::kThreads, sh.dyn, st>>>(P, t, x, y, alpha_part, cfg);
  return check_launch("hvs_kernel");
  }
}

template <typename T, typename Acc>
int launch_hv_t(int v, const HvParams& P, const DevTables& t, const T* x, T* y, double* alpha_part,
                cudaStream_t st) {
  if (t.n_tiles == 0) return AED_OK;
  switch (v) {
    case 0: return launch_one<T, Acc, 4, 6>(P, t, x, y, alpha_part, st);
    case 1: return launch_one<T, Acc, 4, 5>(P, t, x, y, alpha_part, st);
    case 2: return launch_one<T, Acc, 4, 4>(P, t, x, y, alpha_part, st);
    case 3: return launch_one<T, Acc, 2, 8>(P, t, x, y, alpha_part, st);
    case 4: return launch_one<T, Acc, 2, 6>(P, t, x, y, alpha_part, st);
    case 5: return launch_one<T, Acc, 8, 3>(P, t, x, y, alpha_part, st);
    case 6: return launch_bundle<T, Acc, 4, 1, 3>(P, t, x, y, alpha_part, st);
    case 7: return launch_bundle<T, Acc, 2, 2, 4>(P, t, x, y, alpha_part, st);
    case 8: return launch_bundle<T, Acc, 4, 2, 2>(P, t, x, y, alpha_part, st);
    case 9: return launch_bundle<T, Acc, 2, 2, 3>(P, t, x, y, alpha_part, st);
    case 10: return launch_bundle<T, Acc, 4, 1, 4>(P, t, x, y, alpha_part, st);
    case 11: return launch_bundle<T, Acc, 2, 1, 4>(P, t, x, y, alpha_part, st);
    case 12: return launch_stream<T, Acc, 14, false>(2, P, t, x, y, alpha_part, st);
    case 13: return launch_stream<T, Acc, 14, false>(1, P, t, x, y, alpha_part, st);
    case 14: return launch_stream<T, Acc, 26, false>(2, P, t, x, y, alpha_part, st);
    case 15: return launch_stream<T, Acc, 26, false>(1, P, t, x, y, alpha_part, st);
    case 16: return launch_stream<T, Acc, 14, true>(1, P, t, x, y, alpha_part, st);
    case 17: return launch_stream<T, Acc, 26, true>(1, P, t, x, y, alpha_part, st);
    default: return fail(AED_ERR_INVALID, "unknown apply variant");
  }
}

int hv_num_variants() { return kNumVariants; }
// The stream applies trail the bundle applies on every sector measured (1.9 to
// 2.3 times slower: one CTA per SM leaves too few warps to issue), so the
// autotuner does not time them; AED_HV_VARIANT still selects them.
bool hv_variant_tuned(int v) { return v >= 0 && v < kNumVariants && kVariants[v].B >= 0; }
const char* hv_variant_name(int v) { return (v >= 0 && v < kNumVariants) ? kVariants[v].name : "?"; }

int launch_hv_f64(int variant, const HvParams& P, const DevTables& t, const double* x, double* y,
                  double* alpha_part, cudaStream_t st) {
  return launch_hv_t<double, AccExact64>(variant, P, t, x, y, alpha_part, st);
}

int launch_hv_f32(int variant, const HvParams& P, const DevTables& t, const float* x, float* y,
                  double* alpha_part, cudaStream_t st) {
  static const bool twosum = [] {
    const char* e = std::getenv("AED_FP32_ACCUM");
    return e && std::string(e) == "twosum";
  }();
  if (twosum) return launch_hv_t<float, AccTwoSum32>(variant, P, t, x, y, alpha_part, st);
  return launch_hv_t<float, AccWide32>(variant, P, t, x, y, alpha_part, st);
}

int launch_diag_table(const HvParams& P, const DevTables& t, double* dg, cudaStream_t st) {
  if (t.n_tiles == 0) return AED_OK;
  diag_table_kernel<<<num_sms() * 8, 256, 0, st>>>(P, t, dg);
  return check_launch("diag_table_kernel");
}

int launch_basis_copy(const DevTables& t, uint32_t* out, int64_t offset, int64_t count, cudaStream_t st) {
  if (count <= 0) return AED_OK;
  basis_copy_kernel<<<(unsigned)((count + 255) / 256), 256, 0, st>>>(t, out, offset, count);
  return check_launch("basis_copy_kernel");
}

int launch_rank(const DevTables& t, int N, const uint32_t* states, int64_t count, int64_t* out, cudaStream_t st) {
  if (count <= 0) return AED_OK;
  rank_kernel<<<(unsigned)((count + 255) / 256), 256, 0, st>>>(t, N, states, count, out);
  return check_launch("rank_kernel");
}

template <typename T>
int launch_fill_random(T* x, int64_t n, uint64_t seed, cudaStream_t st) {
  fill_random_kernel<T><<<elem_grid(n), 256, 0, st>>>(x, n, seed);
  return check_launch("fill_random_kernel");
}

int launch_round_to_f32(const double* x, float* y, int64_t n, cudaStream_t st) {
  round_to_f32_kernel<<<elem_grid(n), 256, 0, st>>>(x, y, n);
  return check_launch("round_to_f32_kernel");
}

template <typename T>
int launch_copy(const T* x, T* y, int64_t n, cudaStream_t st) {
  copy_kernel<T><<<elem_grid(n), 256, 0, st>>>(x, y, n);
  return check_launch("copy_kernel");
}

template <typename T>
int launch_axpy(double a, const T* x, T* y, int64_t n, cudaStream_t st) {
  axpy_kernel<T><<<elem_grid(n), 256, 0, st>>>(a, x, y, n);
  return check_launch("axpy_kernel");
}

template <typename T>
int launch_scal(double a, T* x, int64_t n, bool divide, cudaStream_t st) {
  scal_kernel<T><<<elem_grid(n), 256, 0, st>>>(a, x, n, divide);
  return check_launch("scal_kernel");
}

int64_t red_chunks(int64_t n) { return (n + kRedChunk - 1) / kRedChunk; }

template <typename T>
int launch_dot_partials(const T* x, const T* y, int64_t n, double* part, bool sq, cudaStream_t st) {
  const int64_t nch = red_chunks(n);
  const int grid = (int)(nch < (int64_t)num_sms() * 8 ? nch : (int64_t)num_sms() * 8);
  dot_partials_kernel<T><<<grid < 1 ? 1 : grid, kRedThreads, 0, st>>>(x, y, n, part, sq);
  return check_launch("dot_partials_kernel");
}

int launch_finish_sum(const double* part, int64_t n, double* out, bool take_sqrt, cudaStream_t st) {
  finish_sum_kernel<<<1, kFinishThreads, 0, st>>>(part, n, out, take_sqrt);
  return check_launch("finish_sum_kernel");
}

template <typename T>
int launch_lanczos_update(const double* alpha, const T* x, const T* vprev, const double* beta_prev, T* y,
                          int64_t n, double* partB, cudaStream_t st) {
  const int64_t nch = red_chunks(n);
  const int grid = (int)(nch < (int64_t)num_sms() * 8 ? nch : (int64_t)num_sms() * 8);
  lanczos_update_kernel<T><<<grid < 1 ? 1 : grid, kRedThreads, 0, st>>>(alpha, x, vprev, beta_prev, y, n, partB);
  return check_launch("lanczos_update_kernel");
}

template <typename T>
int launch_lanczos_update_fin(const double* alpha_part, int64_t n_apart, double* alpha, const T* x, const T* vprev,
                              const double* beta_prev, T* y, int64_t n, double* partB, cudaStream_t st) {
  const int64_t nch = red_chunks(n);
  const int grid = (int)(nch < (int64_t)num_sms() * 8 ? nch : (int64_t)num_sms() * 8);
  lanczos_update_fin_kernel<T><<<grid < 1 ? 1 : grid, kRedThreads, 0, st>>>(alpha_part, n_apart, alpha, x, vprev,
                                                                           beta_prev, y, n, partB);
  return check_launch("lanczos_update_fin_kernel");
}

template <typename T>
int launch_lanczos_normalize_fin(const double* beta_part, int64_t n_bpart, double* beta, T* y, int64_t n,
                                 cudaStream_t st) {
  lanczos_normalize_fin_kernel<T><<<elem_grid(n), kRedThreads, 0, st>>>(beta_part, n_bpart, beta, y, n);
  return check_launch("lanczos_normalize_fin_kernel");
}

template <typename T>
int launch_lanczos_normalize(const double* beta, T* y, int64_t n, cudaStream_t st) {
  lanczos_normalize_kernel<T><<<elem_grid(n), kRedThreads, 0, st>>>(beta, y, n);
  return check_launch("lanczos_normalize_kernel");
}

#define AED_INST(T)                                                                                          \
  template int launch_fill_random<T>(T*, int64_t, uint64_t, cudaStream_t);                                   \
  template int launch_copy<T>(const T*, T*, int64_t, cudaStream_t);                                          \
  template int launch_axpy<T>(double, const T*, T*, int64_t, cudaStream_t);                                  \
  template int launch_scal<T>(double, T*, int64_t, bool, cudaStream_t);                                      \
  template int launch_dot_partials<T>(const T*, const T*, int64_t, double*, bool, cudaStream_t);             \
  template int launch_lanczos_update<T>(const double*, const T*, const T*, const double*, T*, int64_t,      \
                                        double*, cudaStream_t);                                              \
  template int launch_lanczos_normalize<T>(const double*, T*, int64_t, cudaStream_t);                          \
  template int launch_lanczos_update_fin<T>(const double*, int64_t, double*, const T*, const T*, const double*, T*, \
                                            int64_t, double*, cudaStream_t);                                      \
  template int launch_lanczos_normalize_fin<T>(const double*, int64_t, double*, T*, int64_t, cudaStream_t);
AED_INST(double)
AED_INST(float)
#undef AED_INST

}  // namespace aed
