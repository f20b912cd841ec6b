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

#include <cfloat>

#include "apply.cuh"
#include "apply_blocks.cuh"
#include "batch.cuh"
#include "reduce.cuh"
#include "rr_core.h"
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
__global__ void __launch_bounds__(kHvThreads, MINB) b_hv32(BatchArgs a, int bucket, int mr_lo, int mr_hi) {
  static_assert(B == 1 || B == kBatchBundle, "an item is one bundle or its blocks one by one");
  extern __shared__ __align__(16) unsigned char b_dyn[];
  __shared__ bapply::BundleSmem<B> sm;
  const int i0 = a.tile_start[bucket], i1 = a.tile_start[bucket + 1];  // this bucket's items
  int cur = -1, rc = 0;
  float* xs = nullptr;
  for (int it = i0 + (int)blockIdx.x; it < i1; it += gridDim.x) {
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

// This thread's elements e0 + threadIdx.x + u kRedThreads of the chunk [e0, e1): w = (y - alpha x) -
// b v_prev into y, and the sum of w^2 in element order.  FP32 in a full chunk: all loads issued before
// the arithmetic (the same operations in the same order, so the same bits).
template <typename T>
__device__ __forceinline__ double update_chunk(const T* x, const T* vp, T* y, int64_t e0, int64_t e1, double alpha,
                                               double b) {
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
        pv[u] = vp ? vp[i0 + u * kRedThreads] : T(0);
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        double w = __dsub_rn((double)yv[u], __dmul_rn(alpha, (double)xv[u]));
        if (vp) w = __dsub_rn(w, __dmul_rn(b, (double)pv[u]));
        const T wt = (T)w;
        y[i0 + u * kRedThreads] = wt;
        acc = fma((double)wt, (double)wt, acc);
      }
      return acc;
    }
  }
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
      constexpr int U = (int)(kRedChunk / kRedThreads);
      if (e1 - e0 == kRedChunk) {  // a full chunk: every load before the divisions
        float v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) v[u] = y[e0 + threadIdx.x + u * kRedThreads];
#pragma unroll
        for (int u = 0; u < U; ++u) y[e0 + threadIdx.x + u * kRedThreads] = (float)__ddiv_rn((double)v[u], beta);
      } else {
        for (int64_t i = e0 + threadIdx.x; i < e1; i += kRedThreads) y[i] = (float)__ddiv_rn((double)y[i], beta);
      }
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

// ---- lowest part of a T-matrix spectrum, one warp per T ----------------------
// The check needs the lowest few distinct non-ghost eigenvalues of T(m)
// (Tmatrix::compute's walk, tmatrix.h:121-228, stops after `want` of them),
// the matching low eigenvalues of T without its first row and column (the
// ghost test), the largest eigenvalue of T (the merge threshold) and, for
// each reported simple value, the last component of its eigenvector (the
// error estimate).  A QL sweep over the whole spectrum costs O(m^2) serial
// plane rotations on one thread (9.6 ms for the longest T of a served batch);
// here each lane bisects one of the low eigenvalues by Sturm counts, O(m)
// per count, the largest is bracketed by all 32 lanes at once (multisection,
// 33x narrower per round), and the eigenvector components come from inverse
// iteration, one lane each.

// The k-th smallest eigenvalue (0-based) of (a, b, n) by multisection of
// [lo, hi] (count(lo) <= k < count(hi)); all 32 lanes take part and get it.
// At most 40 rounds (each narrows the bracket 33x; it stops once the bracket
// is within 2 eps of its ends or stops moving).
__device__ double warp_eigenvalue(const double* __restrict__ a, const double* __restrict__ b, int n, int k,
                                  double lo, double hi) {
  const int lane = threadIdx.x & 31;
  for (int it = 0; it < 40; ++it) {
    const double w = hi - lo;
    if (!(w > 2.0 * DBL_EPSILON * tcore::dmax(fabs(lo), fabs(hi)))) break;
    const double x = fma(w, (double)(lane + 1) * (1.0 / 33.0), lo);
    const unsigned above = __ballot_sync(0xffffffffu, tcore::sturm_count(a, b, n, x) > k);
    const int j = above ? __ffs(above) - 1 : 32;  // first point with more than k eigenvalues below
    const double xh = __shfl_sync(0xffffffffu, x, j < 32 ? j : 31);
    const double xl = __shfl_sync(0xffffffffu, x, j > 0 ? j - 1 : 0);
    const double nlo = j > 0 ? xl : lo, nhi = j < 32 ? xh : hi;
    if (nlo == lo && nhi == hi) break;
    lo = nlo;
    hi = nhi;
  }
  return 0.5 * (lo + hi);
}

// Eigenvalues k0 .. kn-1 of (a, b, n), ascending, into out: lane i bisects
// eigenvalue k0 + 32 g + i of group g on its own (count(x) > k: the upper
// half), so a group of 32 values costs the rounds of one (about 55 Sturm
// counts at full precision; at most 80).  Ghost-rich FP32 T-matrices need
// tens of values before the walk has nev + 1 distinct ones.
__device__ void warp_lowest(const double* __restrict__ a, const double* __restrict__ b, int n, int k0, int kn,
                            double glo, double ghi, double* out) {
  const int lane = threadIdx.x & 31;
  for (int g0 = k0; g0 < kn; g0 += 32) {
    const int k = g0 + lane;
    bool done = k >= kn;
    double lo = glo, hi = ghi;
    for (int it = 0; it < 80; ++it) {
      if (__all_sync(0xffffffffu, done)) break;
      if (!done) {
        const double w = hi - lo;
        const double x = lo + 0.5 * w;
        if (!(w > 2.0 * DBL_EPSILON * tcore::dmax(fabs(lo), fabs(hi))) || x == lo || x == hi) {
          done = true;
        } else if (tcore::sturm_count(a, b, n, x) > k) {
          hi = x;
        } else {
          lo = x;
        }
      }
    }
    if (k < kn) out[k] = 0.5 * (lo + hi);
  }
}

// End of a graph launch: T-matrix analysis of every stepping instance and the
// phase rules, one warp per instance.  The lowest want + 4 eigenvalues of T
// and want + 5 of the reduced T (a lane per value) and T's largest; the
// walk over them on lane 0; the error estimates' eigenvector components by
// inverse iteration, eight lanes at a time.  A walk that needs more of the
// spectrum (many ghost copies) falls back to the QL sweeps of tmatrix_core.h
// (lanes 0 and 1: T and the reduced T side by side).
__global__ void __launch_bounds__(32) b_check(BatchArgs a) {
  const int s = blockIdx.x;
  const int lane = threadIdx.x & 31;
  if (s >= *a.n_inst) return;  // the whole warp leaves together
  BInst& I = a.inst[s];
  if (I.phase != kPhLow && I.phase != kPhHigh) return;
  const int m = I.j;  // alpha_0 .. alpha_{j-1} are final
  if (m < 2) return;
  const int cap = I.cap;
  double* al = I.scratch;
  double* be = al + cap;
  double* work = be + cap;         // 5 cap + 2: sorted spectrum of T (prefix and top), reduced T's
  double* z = work + 5 * cap + 2;  // cap
  double* inv = z + cap;           // 6 cap
  double* zz = I.scratch + 16 * cap;  // kCheckLanes x 7 cap: the lanes' inverse iterations
  for (int q = lane; q < m; q += 32) {
    al[q] = I.ab[2 * q];
    be[q] = I.ab[2 * q + 1];
  }
  __syncwarp();
  double amax = I.ab[0], bmax = I.ab[1];
  for (int q = 0; q < m; ++q) {
    amax = tcore::dmax(amax, al[q]);
    bmax = tcore::dmax(bmax, be[q]);
  }
  const int nev = I.nev;
  const int want = nev + 1;
  const double thold_rel = I.phase == kPhLow ? kFp32MergeRel : 0.0;
  double* evt = work;              // T's sorted spectrum (prefix), its largest at work[m - 1]
  double* evg = work + 3 * cap + 1;  // the reduced T's (prefix)
  double glo, ghi, glo2, ghi2;
  tcore::gershgorin(al, be, m, &glo, &ghi);
  tcore::gershgorin(al + 1, be + 1, m - 1, &glo2, &ghi2);
  const double top = warp_eigenvalue(al, be, m, m - 1, glo, ghi);
  __shared__ tcore::WalkItem items[AED_MAX_NEV + 1];
  __shared__ double zlast[kCheckLanes];
  __shared__ int n_items;
  __shared__ double walk_thold, walk_multol;
  // prefixes of want + 4 and want + 5 values, grown (up to three times) while
  // the walk needs more; the largest of T stays apart at work[m - 1]
  int nt = m < want + 4 ? m : want + 4, ng = m - 1 < want + 5 ? m - 1 : want + 5, pt = 0, pg = 0;
  for (int round = 0; round < 4; ++round) {
    warp_lowest(al, be, m, pt, nt, glo, ghi, evt);
    warp_lowest(al + 1, be + 1, m - 1, pg, ng, glo2, ghi2, evg);
    __syncwarp();
    if (lane == 0)
      n_items = tcore::walk_prefix(m, amax, bmax, evt, nt, top, evg, ng, want, thold_rel, items, &walk_thold, &walk_multol);
    __syncwarp();
    if (n_items >= 0) break;
    pt = nt;
    pg = ng;
    nt = 2 * nt + 4 < m ? 2 * nt + 4 : m;
    ng = 2 * ng + 4 < m - 1 ? 2 * ng + 4 : m - 1;
  }
  if (lane == 0) evt[m - 1] = top;
  __syncwarp();
  double ev[AED_MAX_NEV + 1], er[AED_MAX_NEV + 1];
  int first[AED_MAX_NEV + 1], mults[AED_MAX_NEV + 1];
  tcore::TResult res;
  res.count = 0;
  bool bad = false;
  if (n_items >= 0) {
    // error estimates |beta_m z_{m,i}| of the simple values, eight lanes at a time
    const double bl = be[m - 1];
    for (int r0 = 0; r0 < n_items; r0 += kCheckLanes) {
      const int r = r0 + lane;
      if (lane < kCheckLanes && r < n_items && items[r].zidx >= 0) {
        double* zr = zz + (size_t)lane * 7 * cap;
        tcore::inverse_iteration(m, al, be, evt[items[r].zidx], zr, zr + cap);
        zlast[lane] = zr[m - 1];
      }
      __syncwarp();
      if (lane == 0)
        for (int q = r0; q < n_items && q < r0 + kCheckLanes; ++q)
          er[q] = items[q].zidx >= 0 ? fabs(bl * zlast[q - r0]) : 0.0;
      __syncwarp();
    }
    if (lane != 0) return;
    for (int q = 0; q < n_items; ++q) {
      ev[q] = items[q].value;
      mults[q] = items[q].mult;
      first[q] = items[q].first;
    }
    res.count = n_items;
    res.thold = walk_thold;
    res.multol = walk_multol;
  } else {
    // fallback: the full QL sweeps (T on lane 0, the reduced T on lane 1)
    int info = 0;
    if (lane == 0) info = tcore::analyze_t(m, al, be, work);
    if (lane == 1) info = tcore::analyze_t2(m, al, be, work);
    const int info2 = __shfl_sync(0xffffffffu, info, 1);
    if (lane != 0) return;
    bad = info != 0 || info2 != 0 ||
          tcore::analyze_walk(m, be, amax, bmax, work, want, ev, er, mults, first, &res, thold_rel) != 0;
  }
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
    // the Rayleigh-Ritz step needs a value above the clusters (the gap) and
    // room for its K vectors
    const bool rr = !bad && K > 0 && K <= I.rr_kmax && cnt > nev;
    for (int k = 0; k < K; ++k) {
      tcore::inverse_iteration(m, al, be, work[k], z, inv);
      const double w = tcore::ritz_weight(I.seed, k);
      for (int q = 0; q < m; ++q) I.coef[q] += w * z[q];
      if (rr)
        for (int q = 0; q < m; ++q) I.rr_coef[(size_t)k * cap + q] = z[q];
    }
    if (K == 0) I.coef[0] = 1.0;
    for (int i = 0; i < n1; ++i) I.evals_low[i] = ev[i];
    // lower bound on the eigenvalue above the nev lowest: the next distinct
    // value less its error estimate and the FP32 resolution (work[0..m): the
    // sorted eigenvalues of T)
    I.next_lo = -1e300;
    if (!bad && cnt > nev) {
      const double scale = tcore::dmax(fabs(work[0]), fabs(work[m - 1]));
      I.next_lo = ev[nev] - tcore::dmax(er[nev], kFp32MergeRel * fabs(ev[nev])) - kFp32MergeRel * scale;
    }
    I.m_low = m;
    I.rr_k = rr ? K : 0;
    I.rr_need = cnt < nev ? cnt : nev;
    I.rr_scale = tcore::dmax(fabs(work[0]), fabs(work[m - 1]));
    I.rr_done = 0;
    I.phase = rr && I.next_lo > -1e299 ? kPhRR : kPhRitz;
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
    // block Kato-Temple against the FP32 phase's bound on the next eigenvalue
    bool block = conv && I.etol > 0.0 && I.next_lo > -1e299;
    if (block) {
      double r2 = 0.0;
      for (int i = 0; i < nev; ++i) r2 += er[i] * er[i];
      const double gap = I.next_lo - ev[nev - 1];
      block = gap > 0.0;
      for (int i = 0; block && i < nev; ++i)
        if (!(r2 / gap <= kBatchBlockTol * fabs(ev[i]))) block = false;
    }
    energy = energy || block;
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

// ---- Rayleigh-Ritz hand-over of the mixed path (phase kPhRR) -----------------
// The single-instance refinement of lanczos.cpp (rayleigh_ritz) for every
// request whose FP32 phase ended at this graph launch: the K Ritz vectors of
// T that span its nev lowest clusters are formed in FP64 from the stored
// basis, H is applied to each (the FP64 bundle apply), the Gram matrices
// Psi^T Psi and Psi^T H Psi are summed per chunk and finished per request,
// one thread per request solves the K x K pencil (rr_core.h), the residuals
// of the pairs below the FP32 phase's gap bound are summed, and the block
// Kato-Temple bound sum |r|^2 / (next_lo - theta_max) decides: at most
// kBatchBlockTol |theta| for every reported value and the result is taken
// (K FP64 applies instead of 16-24 FP64 Lanczos steps); otherwise the request
// goes on to the FP64 Lanczos refinement (phase kPhRitz, below).  Every sum
// has a fixed order, so a request's result does not depend on the batch.

__device__ __forceinline__ double* rr_psi(const BInst& I, int k) { return I.rr_v + (size_t)k * I.D; }
__device__ __forceinline__ double* rr_img(const BInst& I, int k) { return I.rr_v + (size_t)(I.rr_kmax + k) * I.D; }

// Psi_k = sum_j coef_k[j] v_j over the stored FP32 basis (FP64, ascending j).
__global__ void __launch_bounds__(kRedThreads) b_rr_combine(BatchArgs a) {
  __shared__ double cs[kStoreChunkB * kMaxRR];
  const int n = *a.n_chunks;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const BItem w = a.chunks[it];
    const BInst& I = a.inst[w.inst];
    if (I.phase != kPhRR) continue;
    const int K = I.rr_k, m = I.m_low;
    const int64_t e0 = (int64_t)w.idx * kRedChunk, e1 = e0 + kRedChunk < I.D ? e0 + kRedChunk : I.D;
    for (int64_t i0 = e0; i0 < e1; i0 += kRedThreads) {
      const int64_t i = i0 + threadIdx.x;
      double acc[kMaxRR];
#pragma unroll
      for (int k = 0; k < kMaxRR; ++k) acc[k] = 0.0;
      for (int j0 = 0; j0 < m; j0 += kStoreChunkB) {
        const int cnt = m - j0 < kStoreChunkB ? m - j0 : kStoreChunkB;
        __syncthreads();
        for (int q = threadIdx.x; q < cnt * K; q += kRedThreads)
          cs[q] = I.rr_coef[(size_t)(q % K) * I.cap + j0 + q / K];  // cs[jj * K + k]
        __syncthreads();
        if (i < e1)
          for (int jj = 0; jj < cnt; ++jj) {
            const double v = (double)low_vec(I, j0 + jj)[i];
#pragma unroll
            for (int k = 0; k < kMaxRR; ++k)
              if (k < K) acc[k] = fma(cs[jj * K + k], v, acc[k]);
          }
      }
      if (i < e1)
        for (int k = 0; k < K; ++k) rr_psi(I, k)[i] = acc[k];
    }
  }
}

// H Psi_k for k < K over the request's (bundle) items: the FP64 bundle apply.
__global__ void __launch_bounds__(kHvThreads, 3) b_rr_apply(BatchArgs a) {
  extern __shared__ __align__(16) unsigned char b_dyn[];
  __shared__ bapply::BundleSmem<1> sm;
  const int n = *a.n_tiles;
  int cur = -1, rc = 0;
  double* xs = nullptr;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const BItem w = a.tiles[it];
    const BInst& I = a.inst[w.inst];
    if (I.phase != kPhRR) continue;
    if (w.inst != cur) {
      __syncthreads();
      xs = bapply::carve<double, 1>(*I.P, I.t, b_dyn, sm);
      bapply::stage_pairs<1>(*I.P, sm);
      cur = w.inst;
    }
    const ApplyCtx c = apply::ctx_of(*I.P);
    for (int k = 0; k < I.rr_k; ++k)
      for (int q = 0; q < kBatchBundle; ++q)
        bapply::apply_bundle<double, AccExact64, 4, 1>(c, I.t, (int64_t)w.idx * kBatchBundle + q, rr_psi(I, k),
                                                       rr_img(I, k), nullptr, sm, xs, rc);
  }
}

// Chunk partials of the Gram matrices: G(a, b), a <= b, then A(a, b) =
// <Psi_a, H Psi_b>, at part[p * n_chunks + chunk].
template <int K>
__device__ __forceinline__ void rr_gram_chunk(const BInst& I, int64_t c, double* red) {
  constexpr int NP = K * (K + 1) / 2 + K * K;
  const int64_t e0 = c * kRedChunk, e1 = e0 + kRedChunk < I.D ? e0 + kRedChunk : I.D;
  double acc[NP];
#pragma unroll
  for (int p = 0; p < NP; ++p) acc[p] = 0.0;
  for (int64_t i = e0 + threadIdx.x; i < e1; i += kRedThreads) {
    double x[K], y[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      x[k] = rr_psi(I, k)[i];
      y[k] = rr_img(I, k)[i];
    }
    int p = 0;
#pragma unroll
    for (int u = 0; u < K; ++u)
#pragma unroll
      for (int v = u; v < K; ++v) {
        acc[p] = fma(x[u], x[v], acc[p]);
        ++p;
      }
#pragma unroll
    for (int u = 0; u < K; ++u)
#pragma unroll
      for (int v = 0; v < K; ++v) {
        acc[p] = fma(x[u], y[v], acc[p]);
        ++p;
      }
  }
#pragma unroll
  for (int p = 0; p < NP; ++p) {
    const double tot = block_sum_all<kRedThreads>(acc[p], red);
    if (threadIdx.x == 0) I.rr_part[(size_t)p * I.n_chunks + c] = tot;
  }
}

__global__ void __launch_bounds__(kRedThreads) b_rr_gram(BatchArgs a) {
  __shared__ double red[33];
  const int n = *a.n_chunks;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const BItem w = a.chunks[it];
    const BInst& I = a.inst[w.inst];
    if (I.phase != kPhRR) continue;
    switch (I.rr_k) {
      case 1: rr_gram_chunk<1>(I, w.idx, red); break;
      case 2: rr_gram_chunk<2>(I, w.idx, red); break;
      case 3: rr_gram_chunk<3>(I, w.idx, red); break;
      case 4: rr_gram_chunk<4>(I, w.idx, red); break;
      case 5: rr_gram_chunk<5>(I, w.idx, red); break;
      case 6: rr_gram_chunk<6>(I, w.idx, red); break;
      case 7: rr_gram_chunk<7>(I, w.idx, red); break;
      case 8: rr_gram_chunk<8>(I, w.idx, red); break;
      default: break;
    }
  }
}

// rr_small[p] = the request's sum of partial p over its chunks (finish_sum's
// order), for p < np (np: the Gram entries, or the bounded pairs' residuals).
__global__ void __launch_bounds__(256) b_rr_finish(BatchArgs a, int residuals) {
  __shared__ double red[33];
  if ((int)blockIdx.x >= *a.n_inst) return;
  const BInst& I = a.inst[blockIdx.x];
  if (I.phase != kPhRR) return;
  const int K = I.rr_k;
  const int np = residuals ? I.rr_nb : K * (K + 1) / 2 + K * K;
  for (int p = 0; p < np; ++p) {
    const double tot = finish_sum_in_cta<256>(I.rr_part + (size_t)p * I.n_chunks, I.n_chunks, red);
    if (threadIdx.x == 0) I.rr_small[p] = tot;
  }
}

// One thread per request: the Ritz pairs of the pencil, the pairs below the
// gap bound and their residual coefficients.
__global__ void b_rr_solve(BatchArgs a) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= *a.n_inst) return;
  BInst& I = a.inst[s];
  if (I.phase != kPhRR) return;
  const int K = I.rr_k;
  double G[kMaxRR * kMaxRR], A[kMaxRR * kMaxRR];
  const double* sum = I.rr_small;
  int p = 0;
  for (int u = 0; u < K; ++u)
    for (int v = u; v < K; ++v, ++p) G[u * K + v] = G[v * K + u] = sum[p];
  for (int u = 0; u < K; ++u)
    for (int v = 0; v < K; ++v, ++p) A[u * K + v] = sum[p];
  double th[kMaxRR], cr[kMaxRR][kMaxRR];
  int ord[kMaxRR];
  const int Kp = rrcore::ritz_pairs(K, G, A, th, cr, ord);
  int nb = 0;
  while (nb < Kp && th[ord[nb]] < I.next_lo) ++nb;
  if (nb < 1) {
    I.phase = kPhRitz;
    return;
  }
  double* sm = I.rr_small;
  for (int i = 0; i < nb; ++i) {
    const int q = ord[i];
    sm[100 + i] = th[q];
    for (int k = 0; k < kMaxRR; ++k) {
      sm[116 + i * kMaxRR + k] = k < K ? cr[q][k] : 0.0;
      sm[180 + i * kMaxRR + k] = k < K ? -th[q] * cr[q][k] : 0.0;
    }
    sm[244 + i] = rrcore::form(K, G, cr[q], cr[q]);
  }
  I.rr_nb = nb;
}

// Chunk partials of |sum_k cw[r][k] H Psi_k + cx[r][k] Psi_k|^2 for r < nb.
template <int K>
__device__ __forceinline__ void rr_resid_chunk(const BInst& I, int64_t c, double* red, const double* cw,
                                               const double* cx) {
  const int nb = I.rr_nb;
  const int64_t e0 = c * kRedChunk, e1 = e0 + kRedChunk < I.D ? e0 + kRedChunk : I.D;
  double acc[K];
#pragma unroll
  for (int r = 0; r < K; ++r) acc[r] = 0.0;
  for (int64_t i = e0 + threadIdx.x; i < e1; i += kRedThreads) {
    double x[K], y[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      x[k] = rr_psi(I, k)[i];
      y[k] = rr_img(I, k)[i];
    }
#pragma unroll
    for (int r = 0; r < K; ++r) {
      if (r < nb) {
        double t = 0.0;
#pragma unroll
        for (int k = 0; k < K; ++k) t = fma(cw[r * kMaxRR + k], y[k], fma(cx[r * kMaxRR + k], x[k], t));
        acc[r] = fma(t, t, acc[r]);
      }
    }
  }
#pragma unroll
  for (int r = 0; r < K; ++r) {
    if (r < nb) {
      const double tot = block_sum_all<kRedThreads>(acc[r], red);
      if (threadIdx.x == 0) I.rr_part[(size_t)r * I.n_chunks + c] = tot;
    }
  }
}

__global__ void __launch_bounds__(kRedThreads) b_rr_resid(BatchArgs a) {
  __shared__ double red[33];
  __shared__ double cw[kMaxRR * kMaxRR], cx[kMaxRR * kMaxRR];
  const int n = *a.n_chunks;
  int cur = -1;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const BItem w = a.chunks[it];
    const BInst& I = a.inst[w.inst];
    if (I.phase != kPhRR) continue;
    if (w.inst != cur) {
      __syncthreads();
      for (int q = threadIdx.x; q < kMaxRR * kMaxRR; q += kRedThreads) {
        cw[q] = I.rr_small[116 + q];
        cx[q] = I.rr_small[180 + q];
      }
      __syncthreads();
      cur = w.inst;
    }
    switch (I.rr_k) {
      case 1: rr_resid_chunk<1>(I, w.idx, red, cw, cx); break;
      case 2: rr_resid_chunk<2>(I, w.idx, red, cw, cx); break;
      case 3: rr_resid_chunk<3>(I, w.idx, red, cw, cx); break;
      case 4: rr_resid_chunk<4>(I, w.idx, red, cw, cx); break;
      case 5: rr_resid_chunk<5>(I, w.idx, red, cw, cx); break;
      case 6: rr_resid_chunk<6>(I, w.idx, red, cw, cx); break;
      case 7: rr_resid_chunk<7>(I, w.idx, red, cw, cx); break;
      case 8: rr_resid_chunk<8>(I, w.idx, red, cw, cx); break;
      default: break;
    }
  }
}

// One thread per request: the block Kato-Temple bound and the verdict.
__global__ void b_rr_accept(BatchArgs a) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= *a.n_inst) return;
  BInst& I = a.inst[s];
  if (I.phase != kPhRR) return;
  const double* sm = I.rr_small;
  const int nb = I.rr_nb;
  double rn2 = 0.0;
  for (int i = 0; i < nb; ++i) rn2 += sm[244 + i] > 0.0 ? sm[i] / sm[244 + i] : sm[i];
  const double gap = I.next_lo - sm[100 + nb - 1];
  const double bound = rn2 / gap;
  // distinct values: merged below the FP64 T-matrix threshold eps^(2/3) max|lambda| (tmatrix.h:148-150)
  const double thold = pow(DBL_EPSILON, 2.0 / 3.0) * I.rr_scale;
  double vals[AED_MAX_NEV];
  int n = 0;
  for (int i = 0; i < nb && n < I.nev; ++i)
    if (n == 0 || sm[100 + i] - vals[n - 1] > thold) vals[n++] = sm[100 + i];
  bool ok = gap > 0.0 && n >= I.rr_need;
  for (int i = 0; ok && i < n; ++i)
    if (!(bound <= kBatchBlockTol * fabs(vals[i]))) ok = false;
  if (!ok) {
    I.phase = kPhRitz;  // on to the FP64 Lanczos refinement
    return;
  }
  for (int i = 0; i < n; ++i) {
    I.evals[i] = vals[i];
    I.errs[i] = bound;
  }
  I.n_evals = n;
  I.iters = I.rr_k;  // the FP64 applies of the refinement
  I.converged = 1;
  I.rr_done = 1;
  I.phase = kPhDone;
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
  void (*kern)(BatchArgs, int, int, int);
  const char* name;
};
const Cand32 kCand32[kBatchCand32] = {
    {b_hv32<1, 6, 1>, "r1b6"},          {b_hv32<2, 4, kBatchBundle>, "blk2r2b4"}, {b_hv32<2, 4, 1>, "r2b4"},
    {b_hv32<1, 4, kBatchBundle>, "blk2r1b4"}, {b_hv32<4, 3, 1>, "r4b3"},
};
int g_c32[kBatchCand32] = {}, g_c32_smem[kBatchCand32] = {-1, -1, -1, -1, -1};
int g_hv64 = 0, g_hv64_smem = -1;
int g_rr = 0, g_rr_smem = -1;

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
  hv_grid(b_rr_apply, a.hv_smem, &g_rr, &g_rr_smem);
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
                       a.hv_smem, st>>>(a, bucket, lo, hi);
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
  // two rounds over the candidates, each candidate's faster round counting: one slow window (a
  // clock change, another stream's work) does not decide the bucket's kernel for the engine's life
  float cand_ms[kBatchCand32];
  for (int round = 0; round < 2 && !rc; ++round)
    for (int c = 0; c < kBatchCand32 && !rc; ++c) {
      rc = batch_launch_hv32(a, c, bucket, st);
      if (!rc) AED_CUDA_TRY(cudaEventRecord(e0, st));
      for (int r = 0; r < 3 && !rc; ++r) rc = batch_launch_hv32(a, c, bucket, st);
      if (rc) break;
      AED_CUDA_TRY(cudaEventRecord(e1, st));
      AED_CUDA_TRY(cudaEventSynchronize(e1));
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      cand_ms[c] = round == 0 || ms < cand_ms[c] ? ms : cand_ms[c];
    }
  for (int c = 0; c < kBatchCand32 && !rc; ++c)
    if (*best < 0 || cand_ms[c] < *best_ms) {
      *best = c;
      *best_ms = cand_ms[c];
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
  b_check<<<ni, 32, 0, st>>>(a);
  b_rr_combine<<<gchunk, kRedThreads, 0, st>>>(a);
  b_rr_apply<<<hv_grid(b_rr_apply, a.hv_smem, &g_rr, &g_rr_smem), kHvThreads, a.hv_smem, st>>>(a);
  b_rr_gram<<<gchunk, kRedThreads, 0, st>>>(a);
  b_rr_finish<<<ni, 256, 0, st>>>(a, 0);
  b_rr_solve<<<(ni + 127) / 128, 128, 0, st>>>(a);
  b_rr_resid<<<gchunk, kRedThreads, 0, st>>>(a);
  b_rr_finish<<<ni, 256, 0, st>>>(a, 1);
  b_rr_accept<<<(ni + 127) / 128, 128, 0, st>>>(a);
  b_ritz<<<gchunk, kRedThreads, 0, st>>>(a);
  b_ritz_norm<<<ni, 256, 0, st>>>(a);
  b_ritz_scale<<<gchunk, kRedThreads, 0, st>>>(a);
  b_ritz_commit<<<(ni + 127) / 128, 128, 0, st>>>(a);
  return check("batched Lanczos check");
}

}  // namespace aed
