// apply.cuh -- the tile apply y = H x shared by the single-instance and the
// batched kernels.
//
// Reference paths are relative to the ALPS source tree.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.cuh"
#include "reduce.cuh"

namespace aed {
namespace apply {

// ---------------------------------------------------------------------------
// The apply.  A tile is up to kTileRows consecutive rows of one hi block h: all
// its states share the high Nhi bits.  For such a tile every flip pair falls
// into one of three cases, decided once per tile:
//   * both bits in the hi part: the flip applies to all rows of the tile or to
//     none (it depends on h only); its target is row thi[h'] + r of the hi
//     block h' = h ^ flip (same lo state, so the same offset r): a coalesced
//     stream of x;
//   * one bit in each part: applies iff the lo state has one given bit value;
//     target thi[h'] + tlo[l ^ bit];
//   * both bits in the lo part: applies iff the two lo bits differ (in a given
//     order for the FP64 row order); target thi[h] + tlo[l ^ flip].
// Warp 0 compiles the tile's "program": the flips that can apply, with their
// target block base already looked up, plus the diagonal.  All threads then
// run it on R rows each.  The coupling tables are staged in shared memory
// once per CTA (indexing them from parameter space with a loop counter
// serialises on the constant-load path).
//
// FP64 rows are bit-identical to y = prod(M, x) over the reference's explicit
// matrix (src/ietl/interface/ublas.h:57-63 over hamiltonian_matrix.hpp:307-345):
// a row of M holds the flips to smaller states (ascending column = hi bit
// descending, then lo bit ascending), the diagonal M(i,i), then the flips to
// larger states (hi ascending, lo descending), summed left to right from 0.
// Products and sums round separately (__dmul_rn/__dadd_rn: no FMA
// contraction), as on the reference's x86-64 build.  M(i,i) comes from a
// per-row table filled once per handle in the reference's term order; the
// program for FP64 holds the "smaller" flips, the diagonal, then the "larger"
// flips, in that column order.
//
// FP32 rows (mixed path) take each flip once in any order and accumulate the
// terms c * x_j in FP64 (c is FP64, x_j FP32: every product carries a 53-bit
// significand), rounding to FP32 once at the end; the alternative TwoSum
// (Knuth) + FMA-product-error accumulation in FP32 (Ogita, Rump & Oishi,
// "Dot2") is kept as AccTwoSum.
// ---------------------------------------------------------------------------
constexpr int kTileRows = kHvTileRows;
constexpr uint32_t kCrossOp = 1u << 14;  // program entry of a crossing flip (ordered programs)
constexpr int kMaxOps = 2 * kMaxBonds + 1;

struct SPair {
  uint32_t flip, cond;
  double c;
};

// One program entry.  Hi-part flip: mc = 0, nb = base row of the target hi
// block (target row nb + r).  Crossing flip: mc = lo bit b << 16 | required
// lo-bit value v << 15 (| kCrossOp in ordered programs), nb = target base -
// (v << 15), so that the target row is nb + (crossing-flip table entry).
// c = coupling.
struct TileOp {
  uint32_t mc, nb;
  double c;
};

// ---- row accumulators ----
struct AccExact64 {  // FP64 vectors, the reference's rounding
  double a = 0.0;
  __device__ __forceinline__ void add(double c, double xv) { a = __dadd_rn(a, __dmul_rn(c, xv)); }
  __device__ __forceinline__ double value() const { return a; }
};

struct AccWide32 {  // FP32 vectors, FP64 accumulator
  double a = 0.0;
  __device__ __forceinline__ void add(double c, float xv) { a = fma(c, (double)xv, a); }
  // an FP32 value already widened (exactly) to FP64: the same arithmetic
  __device__ __forceinline__ void add(double c, double xv) { a = fma(c, xv, a); }
  __device__ __forceinline__ float value() const { return (float)a; }
};

struct AccTwoSum32 {  // FP32 vectors, TwoSum + exact product error in FP32
  float s = 0.f, e = 0.f;
  __device__ __forceinline__ void add(double c, float xv) {
    const float ch = (float)c, cl = (float)(c - (double)ch);
    const float p = __fmul_rn(ch, xv);
    const float pe = __fmaf_rn(ch, xv, -p);  // exact: ch*xv - p
    const float t = __fadd_rn(s, p);
    const float bb = __fsub_rn(t, s);
    const float se = __fadd_rn(__fsub_rn(s, __fsub_rn(t, bb)), __fsub_rn(p, bb));
    s = t;
    e = __fadd_rn(e, __fadd_rn(se, __fmaf_rn(cl, xv, pe)));
  }
  __device__ __forceinline__ void add(double c, double xv) { add(c, (float)xv); }  // xv holds an FP32 value
  __device__ __forceinline__ float value() const { return __fadd_rn(s, e); }
};

// Warp 0: append to prog the entries of `list` that can apply in hi block h
// (FP64 order: cond fixes which of the two bits must be set).  Hi-part flips
// get mc = 0; crossing flips get kCrossOp with the encoding of compile_any.
__device__ __forceinline__ int compile_ordered(const SPair* list, int np, uint32_t h, int Nlo, uint32_t lm,
                                               const uint32_t* __restrict__ thi, TileOp* prog, int cnt) {
  const int lane = threadIdx.x & 31;
  for (int q0 = 0; q0 < np; q0 += 32) {
    const int q = q0 + lane;
    bool emit = false;
    TileOp op;
    if (q < np) {
      const SPair e = list[q];
      const uint32_t fhi = e.flip >> Nlo, chi = e.cond >> Nlo;
      if (fhi != 0u && (h & fhi) == chi) {  // lo-part flips come from the lo-neighbour table
        emit = true;
        const uint32_t flo = e.flip & lm, nb = __ldg(thi + (h ^ fhi));
        if (flo == 0u) {  // hi part only: every row of the tile, target row nb + r
          op = {0u, nb, e.c};
        } else {  // crossing: the row's lo bit must equal the condition's (crossing-flip table)
          const uint32_t v = (e.cond & lm) != 0u ? 1u : 0u;
          op = {kCrossOp | ((uint32_t)(__ffs(flo) - 1) << 16) | (v << 15), nb - (v << 15), e.c};
        }
      }
    }
    const unsigned m = __ballot_sync(0xffffffffu, emit);
    if (emit) prog[cnt + __popc(m & ((1u << lane) - 1u))] = op;
    cnt += __popc(m);
  }
  return cnt;
}

// Warp 0: every flip once, either direction (FP32 rows: order is free).
// want_cross = false: the hi-part flips that apply to the tile (all rows);
// true: the crossing flips.  A crossing entry names its lo bit b (mc >> 16)
// and the lo-bit value v that the row must have (bit 15 of mc), for the
// crossing-flip table: entry e = rank | (bit b << 15) applies iff bit 15 of
// e equals v, and then its target row is nb + e with nb = base - (v << 15).
__device__ __forceinline__ int compile_any(const SPair* list, int np, uint32_t h, int Nlo, uint32_t lm,
                                          const uint32_t* __restrict__ thi, TileOp* prog, int cnt,
                                          bool want_cross) {
  const int lane = threadIdx.x & 31;
  for (int q0 = 0; q0 < np; q0 += 32) {
    const int q = q0 + lane;
    bool emit = false;
    TileOp op;
    if (q < np) {
      const SPair e = list[q];
      const uint32_t fhi = e.flip >> Nlo, flo = e.flip & lm;
      const uint32_t hb = h & fhi;
      if (flo == 0u) {  // hi part only: applies to the whole tile iff the two bits differ
        emit = !want_cross && __popc(hb) == 1;
        if (emit) op = {0u, __ldg(thi + (h ^ fhi)), e.c};
      } else if (fhi == 0u) {  // lo part only: from the lo-neighbour table
        emit = false;
      } else {  // crossing: the lo bit must differ from the hi bit
        emit = want_cross;
        const uint32_t v = hb ? 0u : 1u;
        if (emit) op = {((uint32_t)(__ffs(flo) - 1) << 16) | (v << 15), __ldg(thi + (h ^ fhi)) - (v << 15), e.c};
      }
    }
    const unsigned m = __ballot_sync(0xffffffffu, emit);
    if (emit) prog[cnt + __popc(m & ((1u << lane) - 1u))] = op;
    cnt += __popc(m);
  }
  return cnt;
}

// FP64 rows: the program's flips in program (column) order.  The x values of
// four flips are loaded before their terms are added, in order.  xt: as for
// run_cross.
template <typename T, typename Acc, int R>
__device__ __forceinline__ void run_ordered(const TileOp* prog, int o0, int o1, const uint16_t* __restrict__ xt,
                                            uint32_t nlo, uint32_t nrow, uint32_t rt, const T* __restrict__ x,
                                            Acc* acc) {
  constexpr int U = R >= 8 ? 1 : 8 / R;  // about eight loads in flight per thread
  int o = o0;
  for (; o + U <= o1; o += U) {
    TileOp e[U];
    bool p[U][R];
    T xv[U][R];
#pragma unroll
    for (int v = 0; v < U; ++v) {
      e[v] = prog[o + v];
      if (e[v].mc & kCrossOp) {
        const uint16_t* xb = xt + (size_t)((e[v].mc >> 16) & 0xffffu) * nlo;
#pragma unroll
        for (int u = 0; u < R; ++u) {
          const uint32_t ent = (uint32_t)u < nrow ? (uint32_t)__ldg(xb + u * kHvThreads) : (~e[v].mc & 0x8000u);
          p[v][u] = ((ent ^ e[v].mc) & 0x8000u) == 0u;
          xv[v][u] = p[v][u] ? __ldg(x + (e[v].nb + ent)) : T(0);
        }
      } else {
#pragma unroll
        for (int u = 0; u < R; ++u) {
          p[v][u] = (uint32_t)u < nrow;
          xv[v][u] = p[v][u] ? __ldg(x + e[v].nb + rt + u * kHvThreads) : T(0);
        }
      }
    }
#pragma unroll
    for (int v = 0; v < U; ++v)
#pragma unroll
      for (int u = 0; u < R; ++u)
        if (p[v][u]) acc[u].add(e[v].c, xv[v][u]);
  }
  for (; o < o1; ++o) {
    const TileOp e = prog[o];
    if (e.mc & kCrossOp) {
      const uint16_t* xb = xt + (size_t)((e.mc >> 16) & 0xffffu) * nlo;
#pragma unroll
      for (int u = 0; u < R; ++u)
        if ((uint32_t)u < nrow) {
          const uint32_t ent = __ldg(xb + u * kHvThreads);
          if (((ent ^ e.mc) & 0x8000u) == 0u) acc[u].add(e.c, __ldg(x + (e.nb + ent)));
        }
    } else {
#pragma unroll
      for (int u = 0; u < R; ++u)
        if ((uint32_t)u < nrow) acc[u].add(e.c, __ldg(x + e.nb + rt + u * kHvThreads));
    }
  }
}

struct ApplyCtx {
  int np, Nlo, n_up;
  uint32_t lm;
};

// M(i,i) for an FP32 row: the FP32 copy of the diagonal when the handle keeps
// one (single-instance FP32 handles: half the bytes of the FP64 table; the
// FP32 phase tolerates the rounding, its FP64 refinement uses dg), else dg.
// Every FP32 variant reads it the same way, so their rows stay identical.
__device__ __forceinline__ double diag_fp32(const DevTables& t, uint32_t i) {
  return t.dgf ? (double)__ldg(t.dgf + i) : __ldg(t.dg + i);
}

// Shared memory of one CTA running tiles.
struct ApplySmem {
  SPair low[kMaxBonds];
  SPair rise[kMaxBonds];
  TileOp prog[kMaxOps];
  double lolo_c[kMaxBonds];
  int nlow, nops;
  double red[33];
};

__device__ __forceinline__ ApplyCtx ctx_of(const HvParams& P) { return {P.n_pairs, P.Nlo, P.n_up, P.lomask}; }

// Stage the flip pairs of P in shared memory (all threads; the next
// apply_tile starts with a barrier).  Flips to smaller states need the higher
// bit set, flips to larger states the lower one.
__device__ __forceinline__ void stage_pairs(const HvParams& P, ApplySmem& sm) {
  for (int q = threadIdx.x; q < P.n_pairs; q += kHvThreads) {
    const PairTerm a = P.low[q], b = P.rise[q];
    sm.low[q] = {a.mhi | a.mlo, a.mhi, a.c};
    sm.rise[q] = {b.mhi | b.mlo, b.mlo, b.c};
  }
  for (int q = threadIdx.x; q < P.n_lolo; q += kHvThreads) sm.lolo_c[q] = P.lolo_c[q];
}

// FP32 rows, hi-part flips: every row of the tile takes them; four flips at a
// time so that 4*R independent loads of x are in flight per thread.
template <typename T, typename Acc, int R>
__device__ __forceinline__ void run_hihi(const TileOp* prog, int o0, int o1, uint32_t nrow, uint32_t rt,
                                         const T* __restrict__ x, Acc* acc) {
  int o = o0;
  for (; o + 4 <= o1; o += 4) {
    TileOp e[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) e[v] = prog[o + v];
    T xv[4][R];
#pragma unroll
    for (int u = 0; u < R; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) xv[v][u] = (uint32_t)u < nrow ? __ldg(x + e[v].nb + rt + u * kHvThreads) : T(0);
#pragma unroll
    for (int u = 0; u < R; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v)
        if ((uint32_t)u < nrow) acc[u].add(e[v].c, xv[v][u]);
  }
  for (; o < o1; ++o) {
    const TileOp e = prog[o];
#pragma unroll
    for (int u = 0; u < R; ++u)
      if ((uint32_t)u < nrow) acc[u].add(e.c, __ldg(x + e.nb + rt + u * kHvThreads));
  }
}

// FP32 rows, crossing flips from the crossing-flip table (coalesced 16-bit
// loads, no dependent rank lookup), four flips at a time.  xt: table entries
// of this thread's u = 0 row for lo bit 0 (xtab + lbase + rt); nlo = 2^Nlo,
// the table's stride per lo bit.
template <typename T, typename Acc, int R>
__device__ __forceinline__ void run_cross(const TileOp* prog, int o0, int o1, const uint16_t* __restrict__ xt,
                                          uint32_t nlo, uint32_t nrow, const T* __restrict__ x, Acc* acc) {
  constexpr int U = 4;
  int o = o0;
  for (; o + U <= o1; o += U) {
    TileOp e[U];
    uint32_t ent[U][R];
#pragma unroll
    for (int v = 0; v < U; ++v) {
      e[v] = prog[o + v];
      const uint16_t* xb = xt + (size_t)(e[v].mc >> 16) * nlo;
#pragma unroll
      for (int u = 0; u < R; ++u)
        ent[v][u] = (uint32_t)u < nrow ? (uint32_t)__ldg(xb + u * kHvThreads) : (~e[v].mc & 0x8000u);
    }
    T xv[U][R];
#pragma unroll
    for (int v = 0; v < U; ++v)
#pragma unroll
      for (int u = 0; u < R; ++u)
        xv[v][u] = ((ent[v][u] ^ e[v].mc) & 0x8000u) == 0u ? __ldg(x + (e[v].nb + ent[v][u])) : T(0);
#pragma unroll
    for (int v = 0; v < U; ++v)
#pragma unroll
      for (int u = 0; u < R; ++u)
        if (((ent[v][u] ^ e[v].mc) & 0x8000u) == 0u) acc[u].add(e[v].c, xv[v][u]);
  }
  for (; o < o1; ++o) {
    const TileOp e = prog[o];
    const uint16_t* xb = xt + (size_t)(e.mc >> 16) * nlo;
#pragma unroll
    for (int u = 0; u < R; ++u) {
      if ((uint32_t)u < nrow) {
        const uint32_t ent = __ldg(xb + u * kHvThreads);
        if (((ent ^ e.mc) & 0x8000u) == 0u) acc[u].add(e.c, __ldg(x + (e.nb + ent)));
      }
    }
  }
}

// FP32 rows, lo-part flips from the lo-neighbour table, two entries at a time.
template <typename T, typename Acc, int R>
__device__ __forceinline__ void run_lo_table_any(const DevTables& t, uint32_t lbase, uint32_t nk, uint32_t base,
                                                 uint32_t rt, uint32_t nrow, const double* lolo_c,
                                                 const T* __restrict__ x, Acc* acc) {
  const uint32_t* E = t.ell + (size_t)t.ell_w * lbase;
  for (int e = 0; e < t.ell_w; e += 2) {
    uint32_t ent[2][R];
    bool any = false;
#pragma unroll
    for (int v = 0; v < 2; ++v)
#pragma unroll
      for (int u = 0; u < R; ++u) {
        ent[v][u] = ((uint32_t)u < nrow && e + v < t.ell_w) ? __ldg(E + (size_t)(e + v) * nk + rt + u * kHvThreads)
                                                             : kEllPad;
        any |= ent[v][u] != kEllPad;
      }
    if (!__any_sync(0xffffffffu, any)) break;
    T xv[2][R];
#pragma unroll
    for (int v = 0; v < 2; ++v)
#pragma unroll
      for (int u = 0; u < R; ++u) xv[v][u] = ent[v][u] != kEllPad ? __ldg(x + base + (ent[v][u] & 0xffffu)) : T(0);
#pragma unroll
    for (int v = 0; v < 2; ++v)
#pragma unroll
      for (int u = 0; u < R; ++u)
        if (ent[v][u] != kEllPad) acc[u].add(lolo_c[ent[v][u] >> 16], xv[v][u]);
  }
}

// Flips inside the lo part, from the lo-neighbour table: entry e of the R rows
// of this thread.  All targets lie in the thread's own hi block (base).  With
// kOrdered the entries come in ascending target rank, so the diagonal is
// added just before the first target above the row (the explicit matrix's
// column order); `dd` records that it was added.
template <typename T, typename Acc, int R, bool kOrdered>
__device__ __forceinline__ void run_lo_table(const DevTables& t, uint32_t lbase, uint32_t nk, uint32_t base,
                                             uint32_t rt, uint32_t nrow, const double* lolo_c,
                                             const T* __restrict__ x, Acc* acc, bool* dd) {
  const uint32_t* E = t.ell + (size_t)t.ell_w * lbase;
  for (int e = 0; e < t.ell_w; ++e) {
    uint32_t ent[R];
    bool any = false;
#pragma unroll
    for (int u = 0; u < R; ++u) {
      ent[u] = (uint32_t)u < nrow ? __ldg(E + (size_t)e * nk + rt + u * kHvThreads) : kEllPad;
      any |= ent[u] != kEllPad;
    }
    if (!__any_sync(0xffffffffu, any)) break;  // rows are padded at the end: nothing left in this warp
#pragma unroll
    for (int u = 0; u < R; ++u) {
      if (ent[u] != kEllPad) {
        const uint32_t rp = ent[u] & 0xffffu;
        if (kOrdered && !dd[u] && rp > rt + u * kHvThreads) {
          const uint32_t i = base + rt + u * kHvThreads;
          acc[u].add(__ldg(t.dg + i), __ldg(x + i));
          dd[u] = true;
        }
        acc[u].add(lolo_c[ent[u] >> 16], __ldg(x + base + rp));
      }
    }
  }
}

// Tile `it` of y = H x.  alpha_part (optional) receives the tile's partial sum
// of x_i * y_i at index it.  All threads of the CTA call it together.
template <typename T, typename Acc, int R>
__device__ __forceinline__ void apply_tile(const ApplyCtx& c, const DevTables& t, int64_t it,
                                           const T* __restrict__ x, T* __restrict__ y,
                                           double* __restrict__ alpha_part, ApplySmem& sm) {
  static_assert(kTileRows % (kHvThreads * R) == 0, "rows per thread must divide the tile");
  constexpr bool kOrdered = sizeof(T) == 8;
  constexpr int kPasses = kTileRows / (kHvThreads * R);
  const uint32_t h = __ldg(t.tile_h + it);
  const uint32_t r0 = __ldg(t.tile_r + it);
  const int k = c.n_up - __popc(h);
  const uint32_t lbase = __ldg(t.looff + k);
  const uint32_t rows = __ldg(t.looff + k + 1) - lbase;
  const uint32_t base = __ldg(t.thi + h);
  __syncthreads();  // tables staged; previous tile done with prog
  if (threadIdx.x < 32) {
    int nl, cnt;
    if (kOrdered) {
      nl = compile_ordered(sm.low, c.np, h, c.Nlo, c.lm, t.thi, sm.prog, 0);
      cnt = compile_ordered(sm.rise, c.np, h, c.Nlo, c.lm, t.thi, sm.prog, nl);
    } else {
      nl = compile_any(sm.low, c.np, h, c.Nlo, c.lm, t.thi, sm.prog, 0, false);  // hi-part flips
      cnt = compile_any(sm.low, c.np, h, c.Nlo, c.lm, t.thi, sm.prog, nl, true);  // crossing flips
    }
    if (threadIdx.x == 0) {
      sm.nlow = nl;
      sm.nops = cnt;
    }
  }
  __syncthreads();
  const int nlow = sm.nlow, nops = sm.nops;
  double dotacc = 0.0;
#pragma unroll 1
  for (int pass = 0; pass < kPasses; ++pass) {
    const uint32_t rt = r0 + pass * (kHvThreads * R) + threadIdx.x;  // row offset of u = 0
    uint32_t nrow = 0;  // rows of this thread that exist (a prefix of u)
#pragma unroll
    for (int u = 0; u < R; ++u) {
      const uint32_t r = rt + u * kHvThreads;
      nrow += (r < rows && r < r0 + kTileRows) ? 1u : 0u;
    }
    Acc acc[R];
    bool dd[R];
#pragma unroll
    for (int u = 0; u < R; ++u) dd[u] = false;
    if (kOrdered) {
      // flips to smaller states outside the lo part, then the lo-part flips
      // with the diagonal at its column, then the larger states outside
      run_ordered<T, Acc, R>(sm.prog, 0, nlow, t.xtab + lbase + rt, 1u << c.Nlo, nrow, rt, x, acc);
      run_lo_table<T, Acc, R, true>(t, lbase, rows, base, rt, nrow, sm.lolo_c, x, acc, dd);
#pragma unroll
      for (int u = 0; u < R; ++u)
        if ((uint32_t)u < nrow && !dd[u]) {
          const uint32_t i = base + rt + u * kHvThreads;
          acc[u].add(__ldg(t.dg + i), __ldg(x + i));
        }
      run_ordered<T, Acc, R>(sm.prog, nlow, nops, t.xtab + lbase + rt, 1u << c.Nlo, nrow, rt, x, acc);
    } else {
#pragma unroll
      for (int u = 0; u < R; ++u)
        if ((uint32_t)u < nrow) {
          const uint32_t i = base + rt + u * kHvThreads;
          acc[u].add(diag_fp32(t, i), __ldg(x + i));
        }
      run_hihi<T, Acc, R>(sm.prog, 0, nlow, nrow, rt, x, acc);
      run_cross<T, Acc, R>(sm.prog, nlow, nops, t.xtab + lbase + rt, 1u << c.Nlo, nrow, x, acc);
      run_lo_table_any<T, Acc, R>(t, lbase, rows, base, rt, nrow, sm.lolo_c, x, acc);
    }
#pragma unroll
    for (int u = 0; u < R; ++u) {
      if ((uint32_t)u < nrow) {
        const uint32_t i = base + rt + u * kHvThreads;
        const T v = acc[u].value();
        y[i] = v;
        if (alpha_part) dotacc = fma((double)__ldg(x + i), (double)v, dotacc);
      }
    }
  }
  if (alpha_part) {
    const double tot = block_sum_all<kHvThreads>(dotacc, sm.red);
    if (threadIdx.x == 0) alpha_part[it] = tot;
  }
}

}  // namespace apply
}  // namespace aed
