// apply_blocks.cuh -- y = H x over bundles of whole hi blocks, x staged in
// shared memory.
//
// A bundle is up to B hi blocks with the same lo popcount k, so the same lo
// states, the same rows per block and the same lo-neighbour table.  A CTA
// copies x of its B blocks into shared memory, then walks the rows: the flips
// inside the lo part (the lo-neighbour table, about half of all flips) read x
// from shared memory, and one table entry serves all B blocks.  Flips that
// touch the hi part read x from global memory as in the tile apply
// (apply.cuh), from a per-block program compiled by one warp per block.
//
// Each row adds its terms in the same order as the tile apply, so FP64 rows
// stay bit-identical to y = prod(M, x) of the reference's explicit matrix
// (src/ietl/interface/ublas.h:57-63 over hamiltonian_matrix.hpp:307-345).
// The <x, y> partials are formed per 2048-row tile with the same per-thread
// order and the same shuffle tree as the tile apply, so they are identical
// between the two kernels and across variants.
//
// Reference paths are relative to the ALPS source tree.
#pragma once

#include "apply.cuh"

namespace aed {
namespace bapply {

using apply::ApplyCtx;
using apply::kTileRows;
using apply::SPair;
using apply::TileOp;

constexpr uint32_t kNoBlock = 0xffffffffu;
constexpr int kWarps = kHvThreads / 32;

// Start moving the line holding p from HBM into L2 (no register, no wait).
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// Shared memory of a CTA.  The arrays sized by the sector live in dynamic
// shared memory (bundle_smem_bytes), so that small flip lists leave room for
// more CTAs per SM: x of the B blocks (B * maxrows values), the B compiled
// programs (one direction per flip pair: at most n_pairs entries each), the
// flip pairs of both directions and the lo-part couplings.
template <int B>
struct BundleSmem {
  TileOp* prog[B];
  SPair* low;
  SPair* rise;
  double* lolo_c;
  int nlow[B], nops[B];
  double red[2][B][kWarps];
};

__host__ __device__ inline size_t bundle_align16(size_t n) { return (n + 15) & ~(size_t)15; }

// Dynamic shared memory of one CTA: x, programs, pairs, couplings.
template <typename T>
__host__ __device__ inline size_t bundle_smem_bytes(int B, int maxrows, int n_pairs, int n_lolo) {
  return bundle_align16((size_t)B * (size_t)maxrows * sizeof(T)) +
         (size_t)B * (size_t)n_pairs * sizeof(TileOp) + 2 * (size_t)n_pairs * sizeof(SPair) +
         (size_t)n_lolo * sizeof(double);
}

template <typename T, int B>
__device__ __forceinline__ T* carve(const HvParams& P, const DevTables& t, unsigned char* dyn, BundleSmem<B>& sm) {
  T* xs = reinterpret_cast<T*>(dyn);
  unsigned char* p = dyn + bundle_align16((size_t)B * (size_t)t.maxrows * sizeof(T));
#pragma unroll
  for (int j = 0; j < B; ++j) {
    sm.prog[j] = reinterpret_cast<TileOp*>(p);
    p += (size_t)P.n_pairs * sizeof(TileOp);
  }
  sm.low = reinterpret_cast<SPair*>(p);
  p += (size_t)P.n_pairs * sizeof(SPair);
  sm.rise = reinterpret_cast<SPair*>(p);
  p += (size_t)P.n_pairs * sizeof(SPair);
  sm.lolo_c = reinterpret_cast<double*>(p);
  return xs;
}

template <int B>
__device__ __forceinline__ void stage_pairs(const HvParams& P, BundleSmem<B>& sm) {
  for (int q = threadIdx.x; q < P.n_pairs; q += kHvThreads) {
    const PairTerm a = P.low[q], b = P.rise[q];
    sm.low[q] = {a.mhi | a.mlo, a.mhi, a.c};
    sm.rise[q] = {b.mhi | b.mlo, b.mlo, b.c};
  }
  for (int q = threadIdx.x; q < P.n_lolo; q += kHvThreads) sm.lolo_c[q] = P.lolo_c[q];
}

// Partials of <x, y> over one tile of each block: the tree of block_sum_all
// (warp shuffles, then warp 0 over the warp sums), B sums at once.  red is
// used in alternation so that one barrier per tile suffices.
template <int B>
__device__ __forceinline__ void tile_partials(double (&dot)[B], int nv, const uint32_t (&tile)[B],
                                              double (*red)[kWarps], double* __restrict__ alpha_part) {
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
  for (int j = 0; j < B; ++j) {
    double v = dot[j];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (l == 0) red[j][w] = v;
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int j = 0; j < B; ++j) {
      double r = l < kWarps ? red[j][l] : 0.0;
      for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
      if (l == 0 && j < nv) alpha_part[tile[j]] = r;
    }
  }
}

template <typename T, int B>
struct BundlePass;

// FP32 rows, crossing flips of all B blocks: every block has one entry per
// crossing pair, in pair order, so entry o of each block's crossing segment
// names the same lo bit and one crossing-flip table load per row serves all
// blocks (their targets and required bit values differ).
template <typename T, typename Acc, int R, int B>
__device__ __forceinline__ void run_cross_shared(const BundleSmem<B>& sm, const BundlePass<T, B>& q, int nv,
                                                 const uint16_t* __restrict__ xt, uint32_t nlo, uint32_t nrow,
                                                 const T* __restrict__ x, Acc (*acc)[R]) {
  constexpr int U = 2;
  const int nc = q.nops[0] - q.nlow[0];  // crossing entries per block (equal for all blocks)
  int o = 0;
  for (; o < nc; o += U) {
    uint32_t ent[U][R];
#pragma unroll
    for (int v = 0; v < U; ++v) {
      const bool live = o + v < nc;
      const uint32_t mc0 = live ? sm.prog[0][q.nlow[0] + o + v].mc : 0u;
      const uint16_t* xb = xt + (size_t)(mc0 >> 16) * nlo;
#pragma unroll
      for (int u = 0; u < R; ++u) ent[v][u] = (live && (uint32_t)u < nrow) ? (uint32_t)__ldg(xb + u * kHvThreads) : 0u;
    }
    T xv[U][B][R];
    bool p[U][B][R];
    double cc[U][B];
#pragma unroll
    for (int v = 0; v < U; ++v)
#pragma unroll
      for (int j = 0; j < B; ++j) {
        const bool live = o + v < nc && j < nv;
        const TileOp e = live ? sm.prog[j][q.nlow[j] + o + v] : TileOp{0u, 0u, 0.0};
        cc[v][j] = e.c;
#pragma unroll
        for (int u = 0; u < R; ++u) {
          p[v][j][u] = live && (uint32_t)u < nrow && ((ent[v][u] ^ e.mc) & 0x8000u) == 0u;
          xv[v][j][u] = p[v][j][u] ? __ldg(x + (e.nb + ent[v][u])) : T(0);
        }
      }
#pragma unroll
    for (int v = 0; v < U; ++v)
#pragma unroll
      for (int j = 0; j < B; ++j)
#pragma unroll
        for (int u = 0; u < R; ++u)
          if (p[v][j][u]) acc[j][u].add(cc[v][j], xv[v][j][u]);
  }
}

template <typename T, int B>
struct BundlePass {
  int nv;                   // blocks in the bundle
  const uint32_t* bj;       // [B] base row of each block
  const int* nlow;          // [B] program split (FP64: smaller / larger states; FP32: hi part / crossing)
  const int* nops;          // [B] program lengths
  uint32_t lbase, nk;       // lo class offset and rows per block
  const uint32_t* E;        // lo-neighbour table of the class
  const T* xs;              // staged x of the blocks
  uint32_t maxrows;         // stride of xs per block
  uint32_t rt;              // this thread's row for u = 0
};

// One pass of R rows per thread over the bundle's blocks.  kFull: all R rows
// exist (the bounds tests fold away).
template <typename T, typename Acc, int R, int B, bool kFull>
__device__ __forceinline__ void bundle_pass(const ApplyCtx& c, const DevTables& t, const BundleSmem<B>& sm,
                                            const BundlePass<T, B>& q, const T* __restrict__ x,
                                            T* __restrict__ y, double (&dot)[B]) {
  constexpr bool kOrdered = sizeof(T) == 8;
  const int nv = q.nv;
  const uint32_t rt = q.rt, nk = q.nk;
  uint32_t nrow = kFull ? (uint32_t)R : 0u;
  if (!kFull) {
#pragma unroll
    for (int u = 0; u < R; ++u) nrow += rt + u * kHvThreads < nk ? 1u : 0u;
  }
  Acc acc[B][R];
  if (kOrdered) {
    // M(i,i) is added in the middle of the row: start its fetch from HBM now,
    // so that the load at its column finds it in L2
#pragma unroll
    for (int j = 0; j < B; ++j)
#pragma unroll
      for (int u = 0; u < R; ++u)
        if (j < nv && (uint32_t)u < nrow) prefetch_l2(t.dg + q.bj[j] + rt + u * kHvThreads);
    // flips to smaller states outside the lo part; the lo part with the
    // diagonal at its column; the larger states outside the lo part
#pragma unroll
    for (int j = 0; j < B; ++j)
      if (j < nv)
        apply::run_ordered<T, Acc, R>(sm.prog[j], 0, q.nlow[j], t.xtab + q.lbase + rt, 1u << c.Nlo, nrow, rt, x, acc[j]);
    bool dd[R];
#pragma unroll
    for (int u = 0; u < R; ++u) dd[u] = false;
    // two table entries per round trip (loaded together, added in order)
    constexpr int UE = 2;
    for (int e = 0; e < t.ell_w; e += UE) {
      uint32_t ent[UE][R];
      bool any = false;
#pragma unroll
      for (int v = 0; v < UE; ++v)
#pragma unroll
        for (int u = 0; u < R; ++u) {
          ent[v][u] = ((uint32_t)u < nrow && e + v < t.ell_w) ? __ldg(q.E + (size_t)(e + v) * nk + rt + u * kHvThreads)
                                                               : kEllPad;
          any |= ent[v][u] != kEllPad;
        }
      if (!__any_sync(0xffffffffu, any)) break;
#pragma unroll
      for (int v = 0; v < UE; ++v)
#pragma unroll
        for (int u = 0; u < R; ++u) {
          if (ent[v][u] != kEllPad) {
            const uint32_t r = rt + u * kHvThreads;
            const uint32_t rp = ent[v][u] & 0xffffu;
            if (!dd[u] && rp > r) {
#pragma unroll
              for (int j = 0; j < B; ++j)
                if (j < nv) acc[j][u].add(__ldg(t.dg + q.bj[j] + r), q.xs[(size_t)j * q.maxrows + r]);
              dd[u] = true;
            }
            const double cq = sm.lolo_c[ent[v][u] >> 16];
#pragma unroll
            for (int j = 0; j < B; ++j)
              if (j < nv) acc[j][u].add(cq, q.xs[(size_t)j * q.maxrows + rp]);
          }
        }
    }
#pragma unroll
    for (int u = 0; u < R; ++u) {
      if ((uint32_t)u < nrow && !dd[u]) {
        const uint32_t r = rt + u * kHvThreads;
#pragma unroll
        for (int j = 0; j < B; ++j)
          if (j < nv) acc[j][u].add(__ldg(t.dg + q.bj[j] + r), q.xs[(size_t)j * q.maxrows + r]);
      }
    }
#pragma unroll
    for (int j = 0; j < B; ++j)
      if (j < nv)
        apply::run_ordered<T, Acc, R>(sm.prog[j], q.nlow[j], q.nops[j], t.xtab + q.lbase + rt, 1u << c.Nlo, nrow, rt,
                                      x, acc[j]);
  } else {
#pragma unroll
    for (int u = 0; u < R; ++u) {
      if ((uint32_t)u < nrow) {
        const uint32_t r = rt + u * kHvThreads;
#pragma unroll
        for (int j = 0; j < B; ++j)
          if (j < nv) acc[j][u].add(apply::diag_fp32(t, q.bj[j] + r), q.xs[(size_t)j * q.maxrows + r]);
      }
    }
#pragma unroll
    for (int j = 0; j < B; ++j)
      if (j < nv) apply::run_hihi<T, Acc, R>(sm.prog[j], 0, q.nlow[j], nrow, rt, x, acc[j]);
    if (B == 1) {
      apply::run_cross<T, Acc, R>(sm.prog[0], q.nlow[0], q.nops[0], t.xtab + q.lbase + rt, 1u << c.Nlo, nrow, x,
                                  acc[0]);
    } else {
      run_cross_shared<T, Acc, R, B>(sm, q, nv, t.xtab + q.lbase + rt, 1u << c.Nlo, nrow, x, acc);
    }
    // lo-part flips: four table entries at a time, x from shared memory
    constexpr int U = 4;
    for (int e = 0; e < t.ell_w; e += U) {
      uint32_t ent[U][R];
      bool any = false;
#pragma unroll
      for (int v = 0; v < U; ++v)
#pragma unroll
        for (int u = 0; u < R; ++u) {
          ent[v][u] = ((uint32_t)u < nrow && e + v < t.ell_w) ? __ldg(q.E + (size_t)(e + v) * nk + rt + u * kHvThreads)
                                                               : kEllPad;
          any |= ent[v][u] != kEllPad;
        }
      if (!__any_sync(0xffffffffu, any)) break;
#pragma unroll
      for (int v = 0; v < U; ++v)
#pragma unroll
        for (int u = 0; u < R; ++u)
          if (ent[v][u] != kEllPad) {
            const double cq = sm.lolo_c[ent[v][u] >> 16];
            const uint32_t rp = ent[v][u] & 0xffffu;
#pragma unroll
            for (int j = 0; j < B; ++j)
              if (j < nv) acc[j][u].add(cq, q.xs[(size_t)j * q.maxrows + rp]);
          }
    }
  }
#pragma unroll
  for (int u = 0; u < R; ++u) {
    if ((uint32_t)u < nrow) {
      const uint32_t r = rt + u * kHvThreads;
#pragma unroll
      for (int j = 0; j < B; ++j)
        if (j < nv) {
          const T v = acc[j][u].value();
          y[q.bj[j] + r] = v;
          dot[j] = fma((double)q.xs[(size_t)j * q.maxrows + r], (double)v, dot[j]);
        }
    }
  }
}

// Bundle `ub` (entries ub*B .. ub*B+B-1 of the block list).  xs: B * maxrows
// staged x values.  rc counts this CTA's tile reductions (alternation of red).
template <typename T, typename Acc, int R, int B>
__device__ __forceinline__ void apply_bundle(const ApplyCtx& c, const DevTables& t, int64_t ub,
                                             const T* __restrict__ x, T* __restrict__ y,
                                             double* __restrict__ alpha_part, BundleSmem<B>& sm, T* xs,
                                             int& rc) {
  static_assert(kTileRows % (kHvThreads * R) == 0, "rows per thread must divide the tile");
  constexpr bool kOrdered = sizeof(T) == 8;
  constexpr int kPassRows = kHvThreads * R;
  constexpr int kPasses = kTileRows / kPassRows;
  uint32_t hb[B], bj[B];
  int nv = 0;
#pragma unroll
  for (int j = 0; j < B; ++j) {
    hb[j] = __ldg(t.blk_h + ub * B + j);
    nv += hb[j] != kNoBlock ? 1 : 0;  // real blocks come first in a bundle
  }
  if (nv == 0) return;  // padding of the block list
#pragma unroll
  for (int j = 0; j < B; ++j) bj[j] = j < nv ? __ldg(t.thi + hb[j]) : 0u;
  const int k = c.n_up - __popc(hb[0]);
  const uint32_t lbase = __ldg(t.looff + k);
  const uint32_t nk = __ldg(t.looff + k + 1) - lbase;
  const int warp = threadIdx.x >> 5;
  __syncthreads();  // the previous bundle is done with prog and xs
  if (warp < nv) {
    const uint32_t h = __ldg(t.blk_h + ub * B + warp);
    int nl, cnt;
    if (kOrdered) {
      nl = apply::compile_ordered(sm.low, c.np, h, c.Nlo, c.lm, t.thi, sm.prog[warp], 0);
      cnt = apply::compile_ordered(sm.rise, c.np, h, c.Nlo, c.lm, t.thi, sm.prog[warp], nl);
    } else {
      nl = apply::compile_any(sm.low, c.np, h, c.Nlo, c.lm, t.thi, sm.prog[warp], 0, false);
      cnt = apply::compile_any(sm.low, c.np, h, c.Nlo, c.lm, t.thi, sm.prog[warp], nl, true);
    }
    if ((threadIdx.x & 31) == 0) {
      sm.nlow[warp] = nl;
      sm.nops[warp] = cnt;
    }
  }
  // x of the blocks into shared memory, four loads in flight per thread
  constexpr int kStage = 4;
#pragma unroll
  for (int j = 0; j < B; ++j) {
    if (j < nv) {
      const T* src = x + bj[j];
      T* dst = xs + (size_t)j * t.maxrows;
      for (uint32_t i0 = threadIdx.x; i0 < nk; i0 += kStage * kHvThreads) {
        T v[kStage];
#pragma unroll
        for (int a = 0; a < kStage; ++a) v[a] = i0 + a * kHvThreads < nk ? __ldg(src + i0 + a * kHvThreads) : T(0);
#pragma unroll
        for (int a = 0; a < kStage; ++a)
          if (i0 + a * kHvThreads < nk) dst[i0 + a * kHvThreads] = v[a];
      }
    }
  }
  __syncthreads();
  int nlow[B], nops[B];
#pragma unroll
  for (int j = 0; j < B; ++j) {
    nlow[j] = j < nv ? sm.nlow[j] : 0;
    nops[j] = j < nv ? sm.nops[j] : 0;
  }
  const uint32_t* E = t.ell + (size_t)t.ell_w * lbase;
  uint32_t tf[B];
#pragma unroll
  for (int j = 0; j < B; ++j) tf[j] = j < nv ? __ldg(t.tfirst + hb[j]) : 0u;
#pragma unroll 1
  for (uint32_t r0 = 0; r0 < nk; r0 += kTileRows) {
    double dot[B];
#pragma unroll
    for (int j = 0; j < B; ++j) dot[j] = 0.0;
#pragma unroll 1
    for (int pass = 0; pass < kPasses; ++pass) {
      const uint32_t p0 = r0 + pass * kPassRows;
      if (p0 >= nk) break;
      const uint32_t rt = p0 + threadIdx.x;  // row of u = 0
      BundlePass<T, B> bp{nv, bj, nlow, nops, lbase, nk, E, xs, (uint32_t)t.maxrows, rt};
      if (p0 + kPassRows <= nk)  // every row of the pass exists: no per-row bounds
        bundle_pass<T, Acc, R, B, true>(c, t, sm, bp, x, y, dot);
      else
        bundle_pass<T, Acc, R, B, false>(c, t, sm, bp, x, y, dot);
    }
    if (alpha_part) {
      uint32_t tile[B];
#pragma unroll
      for (int j = 0; j < B; ++j) tile[j] = tf[j] + r0 / kTileRows;
      tile_partials<B>(dot, nv, tile, sm.red[rc & 1], alpha_part);
      ++rc;
    }
  }
}

}  // namespace bapply
}  // namespace aed
