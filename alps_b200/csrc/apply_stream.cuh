// apply_stream.cuh -- y = H x with every flip's x segment staged in shared
// memory by the bulk-copy (TMA) engine.
//
// A CTA (one per SM) walks hi blocks.  For a block h every flip that leaves
// the lo part reads a whole other block of x: a hi-part flip reads block
// h ^ fhi row for row (same lo states), a crossing flip reads rows of block
// h ^ (its hi bit) picked by the crossing-flip table.  Blocks are contiguous
// in x, so each such flip becomes one contiguous segment.  A producer warp
// compiles the block's program (the flips that apply, with their target
// blocks), and one of its lanes streams the segments into a ring of shared
// memory stages with cp.async.bulk (global -> shared, completion counted on
// an mbarrier), together with the block's own x (read by the flips inside the
// lo part and by the diagonal).  Eight consumer warps own the block's rows
// (row r = thread + 256 j) and add one staged segment at a time.  The copies
// run ahead of the arithmetic by the depth of the ring, so the gathers no
// longer stall on dependent global loads.
//
// Each row adds its terms in the same order as the tile and bundle applies
// (apply.cuh, apply_blocks.cuh), so FP64 rows are bit-identical to
// y = prod(M, x) of the reference's explicit matrix
// (src/ietl/interface/ublas.h:57-63 over hamiltonian_matrix.hpp:307-345),
// FP32 rows are identical to the other variants', and the <x, y> partials
// are formed per 2048-row tile with the same per-thread order and tree.
//
// Bulk copies need 16-byte aligned addresses and sizes: a segment is copied
// from the 16-byte boundary at or below its start up to the one at or above
// its end, except at the end of the vector, whose last partial 16 bytes the
// producer lane copies with ordinary loads (nothing is read past element D-1).
// Only this GPU's own memory is read; no copy is multicast.
//
// Every wait on an mbarrier is bounded: after about two seconds a waiting
// thread raises the handle's flag (the host reports AED_ERR_TIMEOUT) and the
// CTA winds down; the producer lane waits (again bounded) for the copies it
// issued before it returns.
//
// Reference paths are relative to the ALPS source tree.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "apply.cuh"

namespace aed {
namespace sapply {

using apply::ApplyCtx;
using apply::kCrossOp;
using apply::kTileRows;
using apply::SPair;

constexpr int kConsumerWarps = kHvThreads / 32;  // 8: the partial-sum tree of the other variants
constexpr int kThreads = kHvThreads + 32;        // + the producer warp
constexpr int kMaxStages = 16;
constexpr uint32_t kNoBlock = 0xffffffffu;
constexpr uint32_t kFlagTimeout = 1u;

// One staged flip.  Hi-part flip: mc = 0, row r reads stage[sb + r].
// Crossing flip: mc = kCrossOp | lo bit b << 16 | required bit v << 15, row r
// reads stage[sb + e] with e = the crossing-flip table entry (rank | bit << 15)
// when bit 15 of e equals v (sb carries - v << 15).  e0, n: the target
// block's first element and rows (the copy).
struct SegOp {
  uint32_t mc;
  int32_t sb;
  double c;
  uint32_t e0, n;
};

// Program of one block, written by the producer warp.
struct Prog {
  uint32_t h, base, lbase, nk, tf;
  int nlow, nops;  // ordered (FP64): ops [0, nlow) before the lo part; FP32: hi-part ops first
  int own_sb;      // own x: row r at own[own_sb + r]
  SegOp ops[kMaxBonds];
};

struct StreamCfg {
  int S;                 // ring stages
  int OB;                // own-x buffers (1 or 2)
  uint32_t own_bytes;    // bytes per own-x buffer (16-byte multiple)
  uint32_t ownd_off;     // FP32 rows widened once: the block's own x in FP64 at this offset
  uint32_t ring_off;     // offset of the ring
  uint32_t xoff;         // offset of the crossing-table rows in a stage
  uint32_t stage_bytes;  // bytes per stage (16-byte multiple)
  uint32_t* flag;        // raised on a wait timeout
};

// ---- PTX wrappers (mbarrier, bulk copy) ----
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* b) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(b))
               : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

constexpr uint64_t kWaitNs = 2000000000ull;  // 2 s: far beyond any copy

// Start moving the line holding p from HBM into L2 (no register, no wait).
__device__ __forceinline__ void bapply_prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// Bounded wait by one thread for the phase of parity `parity` of b.  Returns
// false (raising the CTA's abort word and the handle's flag on a timeout)
// when it gives up or another thread of the CTA already did.
__device__ __forceinline__ bool wait_phase_lane(uint64_t* b, uint32_t parity, volatile int* abort, uint32_t* flag) {
  if (mbar_try(b, parity)) return true;
  const uint64_t t0 = gtimer();
  for (uint32_t it = 1;; ++it) {
    if (mbar_try(b, parity)) return true;
    if ((it & 255u) == 0u) {
      if (*abort) return false;
      if (gtimer() - t0 > kWaitNs) {
        *abort = 1;
        atomicOr(flag, kFlagTimeout);
        return false;
      }
    }
  }
}

// The same by a whole warp (every lane waits, as each reads what the phase
// publishes); the verdict is made uniform across the warp.
__device__ __forceinline__ bool wait_phase(uint64_t* b, uint32_t parity, volatile int* abort, uint32_t* flag) {
  const bool ok = wait_phase_lane(b, parity, abort, flag);
  return __all_sync(0xffffffffu, ok);
}

// Smem of one CTA (static part); the stages and own buffers are dynamic.
struct StreamSmem {
  Prog prog[2];
  SPair low[kMaxBonds];
  SPair rise[kMaxBonds];
  double lolo_c[kMaxBonds];
  double red[2][kConsumerWarps];
  uint64_t full[kMaxStages], empty[kMaxStages];
  uint64_t own_full[2], own_empty[2];
  uint64_t prog_full[2], prog_empty[2];
  uint64_t red_full[2], red_empty[2];  // the per-tile reduction across the consumer warps
  uint64_t cvt_done, ownd_free;        // the widened own x: written by all warps / free again
  int abort;
};

// Rows of hi block h2 (0 when its lo class is outside 0..Nlo: such a target
// is never reached from a state of the sector).
__device__ __forceinline__ uint32_t class_rows(const DevTables& t, const ApplyCtx& c, uint32_t h2) {
  const int k2 = c.n_up - __popc(h2);
  if (k2 < 0 || k2 > c.Nlo) return 0u;
  return __ldg(t.looff + k2 + 1) - __ldg(t.looff + k2);
}

// ---- producer side ----
// Warp-cooperative program compile, FP64 order: the entries of `list` that
// apply in block h (cond fixes which of the two bits is set), target block
// base and rows looked up.  es = element size; a0 = elements per 16 bytes - 1.
__device__ __forceinline__ int compile_seg_ordered(const SPair* list, int np, uint32_t h, const ApplyCtx& c,
                                                   const DevTables& t, uint32_t a0, SegOp* ops, int cnt) {
  const int lane = threadIdx.x & 31;
  for (int q0 = 0; q0 < np; q0 += 32) {
    const int q = q0 + lane;
    bool emit = false;
    SegOp op;
    if (q < np) {
      const SPair e = list[q];
      const uint32_t fhi = e.flip >> c.Nlo, chi = e.cond >> c.Nlo;
      if (fhi != 0u && (h & fhi) == chi) {
        emit = true;
        const uint32_t h2 = h ^ fhi, e0 = __ldg(t.thi + h2);
        const uint32_t n = class_rows(t, c, h2);
        const int32_t sb = (int32_t)(e0 & a0);
        const uint32_t flo = e.flip & c.lm;
        if (flo == 0u) {
          op = {0u, sb, e.c, e0, n};
        } else {
          const uint32_t v = (e.cond & c.lm) != 0u ? 1u : 0u;
          op = {kCrossOp | ((uint32_t)(__ffs(flo) - 1) << 16) | (v << 15), sb - (int32_t)(v << 15), e.c, e0, n};
        }
      }
    }
    const unsigned m = __ballot_sync(0xffffffffu, emit);
    if (emit) ops[cnt + __popc(m & ((1u << lane) - 1u))] = op;
    cnt += __popc(m);
  }
  return cnt;
}

// FP32 order: want_cross = false -> the hi-part flips that apply to the block;
// true -> the crossing flips (every crossing pair, either direction).
__device__ __forceinline__ int compile_seg_any(const SPair* list, int np, uint32_t h, const ApplyCtx& c,
                                               const DevTables& t, uint32_t a0, SegOp* ops, int cnt,
                                               bool want_cross) {
  const int lane = threadIdx.x & 31;
  for (int q0 = 0; q0 < np; q0 += 32) {
    const int q = q0 + lane;
    bool emit = false;
    SegOp op;
    if (q < np) {
      const SPair e = list[q];
      const uint32_t fhi = e.flip >> c.Nlo, flo = e.flip & c.lm;
      const uint32_t hb = h & fhi;
      if (flo == 0u) {
        emit = !want_cross && __popc(hb) == 1;
      } else if (fhi != 0u) {
        emit = want_cross;
      }
      if (emit) {
        const uint32_t h2 = h ^ fhi, e0 = __ldg(t.thi + h2);
        const uint32_t n = class_rows(t, c, h2);
        const int32_t sb = (int32_t)(e0 & a0);
        if (flo == 0u) {
          op = {0u, sb, e.c, e0, n};
        } else {
          const uint32_t v = hb ? 0u : 1u;
          op = {kCrossOp | ((uint32_t)(__ffs(flo) - 1) << 16) | (v << 15), sb - (int32_t)(v << 15), e.c, e0, n};
        }
      }
    }
    const unsigned m = __ballot_sync(0xffffffffu, emit);
    if (emit) ops[cnt + __popc(m & ((1u << lane) - 1u))] = op;
    cnt += __popc(m);
  }
  return cnt;
}

// Producer lane: plan the copy of elements [e0, e0 + n) of x into `dst`
// (16-byte aligned) so that element e0 + r lands at dst[(e0 & a0) + r].  The
// bulk copy covers the segment's 16-byte granules below floor16(D * es);
// elements past that bound (the last partial granule of x, at most
// 16 / es - 1 of them) are loaded and stored here.  Returns the bulk bytes;
// *src receives the copy's first byte.
template <typename T>
__device__ __forceinline__ uint32_t plan_segment(const T* __restrict__ x, uint32_t e0, uint32_t n, int64_t D, T* dst,
                                                 const char** src) {
  constexpr uint64_t es = sizeof(T);
  const uint64_t B0 = (uint64_t)e0 * es, B1 = ((uint64_t)e0 + n) * es;
  const uint64_t lim = ((uint64_t)D * es) & ~(uint64_t)15;
  const uint64_t A0 = B0 & ~(uint64_t)15;
  uint64_t A1 = (B1 + 15) & ~(uint64_t)15;
  if (A1 > lim) A1 = lim;
  if (A1 < A0) A1 = A0;
  if (B1 > A1) {
    const uint64_t i0 = A1 / es > e0 ? A1 / es : e0;
    for (uint64_t i = i0; i < (uint64_t)e0 + n; ++i) dst[(i * es - A0) / es] = __ldg(x + i);
    fence_proxy_async();  // these generic stores before later bulk copies into the same stage
  }
  *src = reinterpret_cast<const char*>(x) + A0;
  return (uint32_t)(A1 - A0);
}

// Rows of the crossing-flip table that a crossing op reads: entries
// b * 2^Nlo + lbase .. + nk (lo bit b of the op), whose end lies inside the
// table (its rows are 2^Nlo >= 256 entries long, a 16-byte multiple).
__device__ __forceinline__ uint32_t xtab_first(uint32_t mc, uint32_t nlo, uint32_t lbase) {
  return ((mc >> 16) & 0xffu) * nlo + lbase;
}

struct Producer {
  uint32_t q = 0;    // ring copies issued
  uint32_t owns = 0; // own-x copies issued (= blocks begun)
};

template <typename T>
__device__ __forceinline__ bool issue_own(Producer& pr, const T* __restrict__ x, const DevTables& t, const Prog& pg,
                                          const StreamCfg& cfg, StreamSmem& sm, unsigned char* own) {
  const uint32_t os = pr.owns % (uint32_t)cfg.OB;
  if (!wait_phase_lane(&sm.own_empty[os], ((pr.owns / (uint32_t)cfg.OB) & 1u) ^ 1u, &sm.abort, cfg.flag))
    return false;
  T* dst = reinterpret_cast<T*>(own + (size_t)os * cfg.own_bytes);
  const char* src;
  const uint32_t bytes = plan_segment(x, pg.base, pg.nk, t.D, dst, &src);
  mbar_arrive_tx(&sm.own_full[os], bytes);
  if (bytes) bulk_g2s(dst, src, bytes, &sm.own_full[os]);
  ++pr.owns;
  return true;
}

template <typename T>
__device__ __forceinline__ bool issue_ring(Producer& pr, const T* __restrict__ x, const DevTables& t, const Prog& pg,
                                           const SegOp& op, uint32_t nlo, const StreamCfg& cfg, StreamSmem& sm,
                                           unsigned char* ring) {
  const uint32_t s = pr.q % (uint32_t)cfg.S;
  if (!wait_phase_lane(&sm.empty[s], ((pr.q / (uint32_t)cfg.S) & 1u) ^ 1u, &sm.abort, cfg.flag)) return false;
  unsigned char* stg = ring + (size_t)s * cfg.stage_bytes;
  const char* src;
  const uint32_t bytes = plan_segment(x, op.e0, op.n, t.D, reinterpret_cast<T*>(stg), &src);
  uint32_t xbytes = 0;
  const char* xsrc = nullptr;
  if (op.mc & kCrossOp) {
    const uint64_t B0 = (uint64_t)xtab_first(op.mc, nlo, pg.lbase) * 2u, B1 = B0 + (uint64_t)pg.nk * 2u;
    const uint64_t A0 = B0 & ~(uint64_t)15, A1 = (B1 + 15) & ~(uint64_t)15;
    xsrc = reinterpret_cast<const char*>(t.xtab) + A0;
    xbytes = (uint32_t)(A1 - A0);
  }
  mbar_arrive_tx(&sm.full[s], bytes + xbytes);
  if (bytes) bulk_g2s(stg, src, bytes, &sm.full[s]);
  if (xbytes) bulk_g2s(stg + cfg.xoff, xsrc, xbytes, &sm.full[s]);
  ++pr.q;
  return true;
}

// Wait, without the abort word but bounded, for the copies still in flight
// (the last S ring copies and the last OB own copies) before the CTA exits.
__device__ __forceinline__ void drain(const Producer& pr, const StreamCfg& cfg, StreamSmem& sm) {
  const uint64_t t0 = gtimer();
  const uint32_t S = (uint32_t)cfg.S, OB = (uint32_t)cfg.OB;
  for (uint32_t q = pr.q > S ? pr.q - S : 0u; q < pr.q; ++q)
    while (!mbar_try(&sm.full[q % S], (q / S) & 1u))
      if (gtimer() - t0 > kWaitNs) return;
  for (uint32_t o = pr.owns > OB ? pr.owns - OB : 0u; o < pr.owns; ++o)
    while (!mbar_try(&sm.own_full[o % OB], (o / OB) & 1u))
      if (gtimer() - t0 > kWaitNs) return;
}

// The producer warp: compile each block's program (whole warp), then lane 0
// issues the block's copies in the order the consumers use them: FP64 the
// ops before the lo part, own x, the ops after; FP32 own x, then the ops.
template <typename T>
__device__ __forceinline__ void produce(const ApplyCtx& c, const DevTables& t, const T* __restrict__ x,
                                        const StreamCfg& cfg, StreamSmem& sm, unsigned char* own,
                                        unsigned char* ring) {
  constexpr bool kOrdered = sizeof(T) == 8;
  constexpr uint32_t a0 = 16u / sizeof(T) - 1u;
  const int lane = threadIdx.x & 31;
  const uint32_t nlo = 1u << c.Nlo;
  Producer pr;
  uint32_t b = 0;
  for (int64_t ib = blockIdx.x; ib < t.n_blk; ib += gridDim.x) {
    const uint32_t h = __ldg(t.blk_h + ib);
    if (h == kNoBlock) continue;
    const uint32_t pb = b & 1u;
    if (!wait_phase(&sm.prog_empty[pb], ((b >> 1) & 1u) ^ 1u, &sm.abort, cfg.flag)) break;
    Prog& pg = sm.prog[pb];
    int nl, cnt;
    if (kOrdered) {
      nl = compile_seg_ordered(sm.low, c.np, h, c, t, a0, pg.ops, 0);
      cnt = compile_seg_ordered(sm.rise, c.np, h, c, t, a0, pg.ops, nl);
    } else {
      nl = compile_seg_any(sm.low, c.np, h, c, t, a0, pg.ops, 0, false);
      cnt = compile_seg_any(sm.low, c.np, h, c, t, a0, pg.ops, nl, true);
    }
    bool ok = true;
    if (lane == 0) {
      const int k = c.n_up - __popc(h);
      pg.h = h;
      pg.base = __ldg(t.thi + h);
      pg.lbase = __ldg(t.looff + k);
      pg.nk = __ldg(t.looff + k + 1) - pg.lbase;
      pg.tf = __ldg(t.tfirst + h);
      pg.nlow = nl;
      pg.nops = cnt;
      pg.own_sb = (int)(pg.base & a0);
    }
    __syncwarp();
    if (lane == 0) {
      mbar_arrive(&sm.prog_full[pb]);
      if (kOrdered) {
        for (int o = 0; ok && o < nl; ++o) ok = issue_ring(pr, x, t, pg, pg.ops[o], nlo, cfg, sm, ring);
        if (ok) ok = issue_own(pr, x, t, pg, cfg, sm, own);
        for (int o = nl; ok && o < cnt; ++o) ok = issue_ring(pr, x, t, pg, pg.ops[o], nlo, cfg, sm, ring);
      } else {
        ok = issue_own(pr, x, t, pg, cfg, sm, own);
        for (int o = 0; ok && o < cnt; ++o) ok = issue_ring(pr, x, t, pg, pg.ops[o], nlo, cfg, sm, ring);
      }
    }
    ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
    if (!ok) break;
    ++b;
  }
  if (lane == 0 && sm.abort) drain(pr, cfg, sm);
}

// Consumers: the staged ops [o0, o1) over this thread's rows.
template <typename T, typename Acc, int U>
__device__ __forceinline__ bool consume_ops(const Prog& pg, int o0, int o1, uint32_t& q, uint32_t nlo,
                                            const StreamCfg& cfg, StreamSmem& sm, const unsigned char* ring,
                                            Acc (&acc)[U]) {
  const uint32_t tid = threadIdx.x;
  const uint32_t nk = pg.nk;
  for (int o = o0; o < o1; ++o) {
    const SegOp op = pg.ops[o];
    const uint32_t s = q % (uint32_t)cfg.S;
    if (!wait_phase(&sm.full[s], (q / (uint32_t)cfg.S) & 1u, &sm.abort, cfg.flag)) return false;
    const unsigned char* stg = ring + (size_t)s * cfg.stage_bytes;
    const T* st = reinterpret_cast<const T*>(stg) + op.sb;
    if (op.mc & kCrossOp) {
      const uint16_t* xs = reinterpret_cast<const uint16_t*>(stg + cfg.xoff) + (xtab_first(op.mc, nlo, pg.lbase) & 7u);
#pragma unroll
      for (int j = 0; j < U; ++j) {
        const uint32_t r = tid + j * kHvThreads;
        if (r < nk) {
          const uint32_t e = xs[r];
          if (((e ^ op.mc) & 0x8000u) == 0u) acc[j].add(op.c, st[(int32_t)e]);
        }
      }
    } else {
#pragma unroll
      for (int j = 0; j < U; ++j) {
        const uint32_t r = tid + j * kHvThreads;
        if (r < nk) acc[j].add(op.c, st[r]);
      }
    }
    __syncwarp();
    if ((tid & 31u) == 0u) mbar_arrive(&sm.empty[s]);
    ++q;
  }
  return true;
}

// kOwnD (FP32 rows): the block's own x is widened to FP64 once into a shared
// buffer, so that the diagonal, the lo-part flips and the <x, y> partials
// read it without a conversion each (the FP32 -> FP64 conversions run on a
// quarter-rate pipe); the FP32 own buffer is released right after.
template <typename T, typename Acc, int U, bool kOwnD>
__device__ __forceinline__ void consume(const ApplyCtx& c, const DevTables& t, T* __restrict__ y,
                                        double* __restrict__ alpha_part, const StreamCfg& cfg, StreamSmem& sm,
                                        const unsigned char* own, const unsigned char* ring, double* ownd) {
  constexpr bool kOrdered = sizeof(T) == 8;
  const uint32_t tid = threadIdx.x;
  const int lane = (int)(tid & 31u), warp = (int)(tid >> 5);
  const uint32_t nlo = 1u << c.Nlo;
  uint32_t q = 0, b = 0, rc = 0;
  for (int64_t ib = blockIdx.x; ib < t.n_blk; ib += gridDim.x) {
    const uint32_t h = __ldg(t.blk_h + ib);
    if (h == kNoBlock) continue;
    const uint32_t pb = b & 1u;
    if (!wait_phase(&sm.prog_full[pb], (b >> 1) & 1u, &sm.abort, cfg.flag)) return;
    const Prog& pg = sm.prog[pb];
    const uint32_t base = pg.base, nk = pg.nk;
    const uint32_t os = b % (uint32_t)cfg.OB;
    const T* ox = reinterpret_cast<const T*>(own + (size_t)os * cfg.own_bytes) + pg.own_sb;
    const uint32_t* E = t.ell + (size_t)t.ell_w * pg.lbase;
    Acc acc[U];
    if (kOrdered) {
      // M(i,i) is added mid-row: start its fetch now
#pragma unroll
      for (int j = 0; j < U; ++j)
        if (tid + j * kHvThreads < nk) bapply_prefetch_l2(t.dg + base + tid + j * kHvThreads);
      if (!consume_ops<T, Acc, U>(pg, 0, pg.nlow, q, nlo, cfg, sm, ring, acc)) return;
      if (!wait_phase(&sm.own_full[os], (b / (uint32_t)cfg.OB) & 1u, &sm.abort, cfg.flag)) return;
      bool dd[U];
#pragma unroll
      for (int j = 0; j < U; ++j) dd[j] = false;
      for (int e = 0; e < t.ell_w; e += 2) {
        uint32_t ent[2][U];
        bool any = false;
#pragma unroll
        for (int v = 0; v < 2; ++v)
#pragma unroll
          for (int j = 0; j < U; ++j) {
            const uint32_t r = tid + j * kHvThreads;
            ent[v][j] = (r < nk && e + v < t.ell_w) ? __ldg(E + (size_t)(e + v) * nk + r) : kEllPad;
            any |= ent[v][j] != kEllPad;
          }
        if (!__any_sync(0xffffffffu, any)) break;
#pragma unroll
        for (int v = 0; v < 2; ++v)
#pragma unroll
          for (int j = 0; j < U; ++j)
            if (ent[v][j] != kEllPad) {
              const uint32_t r = tid + j * kHvThreads;
              const uint32_t rp = ent[v][j] & 0xffffu;
              if (!dd[j] && rp > r) {
                acc[j].add(__ldg(t.dg + base + r), ox[r]);
                dd[j] = true;
              }
              acc[j].add(sm.lolo_c[ent[v][j] >> 16], ox[rp]);
            }
      }
#pragma unroll
      for (int j = 0; j < U; ++j) {
        const uint32_t r = tid + j * kHvThreads;
        if (r < nk && !dd[j]) acc[j].add(__ldg(t.dg + base + r), ox[r]);
      }
      if (!consume_ops<T, Acc, U>(pg, pg.nlow, pg.nops, q, nlo, cfg, sm, ring, acc)) return;
    } else {
      if (!wait_phase(&sm.own_full[os], (b / (uint32_t)cfg.OB) & 1u, &sm.abort, cfg.flag)) return;
      if (kOwnD) {
        // the widened buffer is free once every warp finished the previous block
        if (b > 0 && !wait_phase(&sm.ownd_free, (b - 1u) & 1u, &sm.abort, cfg.flag)) return;
#pragma unroll
        for (int j = 0; j < U; ++j) {
          const uint32_t r = tid + j * kHvThreads;
          if (r < nk) ownd[r] = (double)ox[r];
        }
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(&sm.own_empty[os]);  // the FP32 copy is no longer read
          mbar_arrive(&sm.cvt_done);
        }
        if (!wait_phase(&sm.cvt_done, b & 1u, &sm.abort, cfg.flag)) return;
      }
#pragma unroll
      for (int j = 0; j < U; ++j) {
        const uint32_t r = tid + j * kHvThreads;
        if (r < nk) {
          if (kOwnD)
            acc[j].add(apply::diag_fp32(t, base + r), ownd[r]);
          else
            acc[j].add(apply::diag_fp32(t, base + r), ox[r]);
        }
      }
      if (!consume_ops<T, Acc, U>(pg, 0, pg.nops, q, nlo, cfg, sm, ring, acc)) return;
      for (int e = 0; e < t.ell_w; e += 2) {
        uint32_t ent[2][U];
        bool any = false;
#pragma unroll
        for (int v = 0; v < 2; ++v)
#pragma unroll
          for (int j = 0; j < U; ++j) {
            const uint32_t r = tid + j * kHvThreads;
            ent[v][j] = (r < nk && e + v < t.ell_w) ? __ldg(E + (size_t)(e + v) * nk + r) : kEllPad;
            any |= ent[v][j] != kEllPad;
          }
        if (!__any_sync(0xffffffffu, any)) break;
#pragma unroll
        for (int v = 0; v < 2; ++v)
#pragma unroll
          for (int j = 0; j < U; ++j)
            if (ent[v][j] != kEllPad) {
              if (kOwnD)
                acc[j].add(sm.lolo_c[ent[v][j] >> 16], ownd[ent[v][j] & 0xffffu]);
              else
                acc[j].add(sm.lolo_c[ent[v][j] >> 16], ox[ent[v][j] & 0xffffu]);
            }
      }
    }
    // the rows, then the <x, y> partials per 2048-row tile (tree of block_sum_all)
    T yv[U];
#pragma unroll
    for (int j = 0; j < U; ++j) {
      const uint32_t r = tid + j * kHvThreads;
      yv[j] = acc[j].value();
      if (r < nk) y[base + r] = yv[j];
    }
    if (alpha_part) {
      constexpr int kJ = kTileRows / kHvThreads;  // rows per thread per tile
#pragma unroll
      for (int tq = 0; tq < (U + kJ - 1) / kJ; ++tq) {
        if ((uint32_t)tq * kTileRows < nk) {
          double dot = 0.0;
#pragma unroll
          for (int jj = 0; jj < kJ; ++jj) {
            const int j = tq * kJ + jj;
            if (j < U) {
              const uint32_t r = tid + j * kHvThreads;
              if (r < nk) dot = fma(kOwnD ? ownd[r] : (double)ox[r], (double)yv[j], dot);
            }
          }
          for (int o = 16; o > 0; o >>= 1) dot += __shfl_down_sync(0xffffffffu, dot, o);
          // warp sums through red[rc & 1]: its writers wait until warp 0 has read
          // the previous tile there, warp 0 waits for all eight
          const uint32_t rb = rc & 1u, rp = (rc >> 1) & 1u;
          if (!wait_phase(&sm.red_empty[rb], rp ^ 1u, &sm.abort, cfg.flag)) return;
          if (lane == 0) {
            sm.red[rb][warp] = dot;
            mbar_arrive(&sm.red_full[rb]);
          }
          if (warp == 0) {
            if (!wait_phase(&sm.red_full[rb], rp, &sm.abort, cfg.flag)) return;
            double r = lane < kConsumerWarps ? sm.red[rb][lane] : 0.0;
            for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
            if (lane == 0) {
              alpha_part[pg.tf + tq] = r;
              mbar_arrive(&sm.red_empty[rb]);
            }
          }
          ++rc;
        }
      }
    }
    __syncwarp();
    if (lane == 0) {
      if (kOwnD)
        mbar_arrive(&sm.ownd_free);
      else
        mbar_arrive(&sm.own_empty[os]);
      mbar_arrive(&sm.prog_empty[pb]);
    }
    ++b;
  }
}

// y = H x, one CTA per SM: warps 0-7 consume, warp 8 produces.
template <typename T, typename Acc, int U, bool kOwnD>
__global__ void __launch_bounds__(kThreads, 1) hvs_kernel(const __grid_constant__ HvParams P, const DevTables t,
                                                         const T* __restrict__ x, T* __restrict__ y,
                                                         double* __restrict__ alpha_part, const StreamCfg cfg) {
  static_assert(!kOwnD || sizeof(T) == 4, "the widened own x is for FP32 rows");
  extern __shared__ __align__(128) unsigned char hvs_dyn[];
  __shared__ StreamSmem sm;
  for (int q = threadIdx.x; q < P.n_pairs; q += kThreads) {
    const PairTerm a = P.low[q], b = P.rise[q];
    sm.low[q] = {a.mhi | a.mlo, a.mhi, a.c};
    sm.rise[q] = {b.mhi | b.mlo, b.mlo, b.c};
  }
  for (int q = threadIdx.x; q < P.n_lolo; q += kThreads) sm.lolo_c[q] = P.lolo_c[q];
  if (threadIdx.x == 0) {
    for (int s = 0; s < cfg.S; ++s) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.empty[s], kConsumerWarps);
    }
    for (int s = 0; s < 2; ++s) {
      mbar_init(&sm.own_full[s], 1);
      mbar_init(&sm.own_empty[s], kConsumerWarps);
      mbar_init(&sm.prog_full[s], 1);
      mbar_init(&sm.prog_empty[s], kConsumerWarps);
      mbar_init(&sm.red_full[s], kConsumerWarps);
      mbar_init(&sm.red_empty[s], 1);
    }
    mbar_init(&sm.cvt_done, kConsumerWarps);
    mbar_init(&sm.ownd_free, kConsumerWarps);
    sm.abort = 0;
    mbar_fence_init();
  }
  __syncthreads();
  const ApplyCtx c = apply::ctx_of(P);
  unsigned char* own = hvs_dyn;
  unsigned char* ring = hvs_dyn + cfg.ring_off;
  double* ownd = reinterpret_cast<double*>(hvs_dyn + cfg.ownd_off);
  if (threadIdx.x >= kHvThreads)
    produce<T>(c, t, x, cfg, sm, own, ring);
  else
    consume<T, Acc, U, kOwnD>(c, t, y, alpha_part, cfg, sm, own, ring, ownd);
}

}  // namespace sapply
}  // namespace aed
