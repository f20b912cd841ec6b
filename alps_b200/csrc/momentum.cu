// momentum.cu -- momentum (Bloch) sectors on the GPU: the basis of
// representatives, the state -> (representative, translation) map, and the
// complex H x.  Layout and formulas: momentum.cuh.
//
// Reference paths are relative to the ALPS source tree.

#include <cmath>
#include <type_traits>
#include <vector>

#include "handle.h"
#include "momentum.cuh"
#include "reduce.cuh"

namespace aed {
namespace {

constexpr int kMomThreads = 256;
constexpr int kMomChunk = kMomThreads * 8;  // states per chunk of the basis scan (8 per thread)

// States of the two kinds of site basis.  BitCodec: spin 1/2, one bit per
// site (up = 1), ranks by the two tables of the Sz sector (kernels.cuh).
// DigitCodec: spin S, the digit m + S of each site in `bits` bits, ranks by
// the spin-S tables (spin.cuh).  Site i sits at position N-1-i in both, and a
// translation moves it to position dst[t][i].
struct BitCodec {
  using Word = uint32_t;
  DevTables t;
  __device__ __forceinline__ Word translate(const MomParams& mp, Word s, int tr) const {
    Word out = 0u;
    const int N = mp.N;
    for (int i = 0; i < N; ++i) out |= ((s >> (N - 1 - i)) & 1u) << mp.dst[tr][i];
    return out;
  }
  __device__ __forceinline__ uint32_t rank(Word s) const {
    return t.thi[s >> t.Nlo] + t.tlo[s & ((1u << t.Nlo) - 1u)];
  }
};

struct DigitCodec {
  using Word = uint64_t;
  SpinDev t;
  __device__ __forceinline__ Word translate(const MomParams& mp, Word s, int tr) const {
    Word out = 0u;
    const int N = t.N, b = t.bits;
    const uint64_t dm = (1ull << b) - 1ull;
    for (int i = 0; i < N; ++i) out |= ((s >> (b * (N - 1 - i))) & dm) << (b * mp.dst[tr][i]);
    return out;
  }
  __device__ __forceinline__ uint32_t rank(Word s) const {
    const int sh = t.bits * t.Nl;
    return t.thi[(uint32_t)(s >> sh)] + t.tlo[(uint32_t)(s & ((1ull << sh) - 1ull))];
  }
};

// The orbit of s: its smallest state, the first translation reaching it, and
// the phase sum of the translations that fix s (identity included), in list
// order as bloch_basis_states::build adds them (blochbasisstates.h:199-240).
template <class W>
struct Orbit {
  W min;
  int tmin;
  double fre, fim;
};

template <class C>
__device__ __forceinline__ Orbit<typename C::Word> orbit_of(const MomParams& mp, const C& c, typename C::Word s) {
  using W = typename C::Word;
  Orbit<W> o{s, 0, 1.0, 0.0};
  for (int t = 1; t < mp.n_trans; ++t) {
    const W ts = c.translate(mp, s, t);
    if (ts < o.min) {
      o.min = ts;
      o.tmin = t;
    }
    if (ts == s) {
      o.fre += mp.phase_re[t];
      o.fim += mp.phase_im[t];
    }
  }
  return o;
}

// sqrt|phase sum| of a representative (w of blochbasisstates.h:243)
template <class W>
__device__ __forceinline__ double orbit_weight(const Orbit<W>& o) {
  return sqrt(hypot(o.fre, o.fim));
}

template <class C>
__device__ __forceinline__ bool kept_rep(const MomParams& mp, const C& c, typename C::Word s) {
  const auto o = orbit_of(mp, c, s);
  return o.min == s && orbit_weight(o) >= 0.01;
}

// Exclusive scan of one value per thread over the CTA; *total gets the sum.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* sm, uint32_t* total) {
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  uint32_t inc = v;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t n = __shfl_up_sync(0xffffffffu, inc, o);
    if (l >= o) inc += n;
  }
  if (l == 31) sm[w] = inc;
  __syncthreads();
  if (w == 0) {
    uint32_t s = l < kMomThreads / 32 ? sm[l] : 0u;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t n = __shfl_up_sync(0xffffffffu, s, o);
      if (l >= o) s += n;
    }
    if (l < kMomThreads / 32) sm[l] = s;  // inclusive warp totals
  }
  __syncthreads();
  const uint32_t before = (w > 0 ? sm[w - 1] : 0u) + inc - v;
  *total = sm[kMomThreads / 32 - 1];
  __syncthreads();
  return before;
}

// Pass 1: flags of the kept representatives and their count per chunk.
template <class C>
__global__ void __launch_bounds__(kMomThreads) mom_flag_kernel(const __grid_constant__ MomParams mp, const C cd,
                                                               const typename C::Word* __restrict__ states, int64_t D,
                                                               uint8_t* __restrict__ flag,
                                                               uint32_t* __restrict__ count) {
  __shared__ uint32_t sm[kMomThreads / 32];
  const int64_t nch = (D + kMomChunk - 1) / kMomChunk;
  for (int64_t c = blockIdx.x; c < nch; c += gridDim.x) {
    const int64_t r0 = c * kMomChunk + (int64_t)threadIdx.x * 8;
    uint32_t n = 0;
    for (int u = 0; u < 8; ++u) {
      const int64_t r = r0 + u;
      if (r < D) {
        const bool k = kept_rep(mp, cd, states[r]);
        flag[r] = k ? 1 : 0;
        n += k ? 1u : 0u;
      }
    }
    uint32_t total;
    block_exclusive_scan(n, sm, &total);
    if (threadIdx.x == 0) count[c] = total;
  }
}

__device__ __forceinline__ double diag_of(const HvParams& P, uint32_t s) {
  double d = 0.0;
  for (int q = 0; q < P.n_diag; ++q) {
    const bool eq = ((s & P.diag[q].m1) != 0u) == ((s & P.diag[q].m2) != 0u);
    d = __dadd_rn(d, eq ? P.diag[q].veq : P.diag[q].vne);
  }
  return d;
}

// Pass 2: representatives in order (chunk offsets from the host scan); the
// map entry of every representative is its index, every other entry kMomNone.
// diag (spin 1/2 only; may be null): the diagonal terms of each representative.
template <class C>
__global__ void __launch_bounds__(kMomThreads) mom_rep_kernel(const __grid_constant__ MomParams mp,
                                                              const __grid_constant__ HvParams P, const C cd,
                                                              const typename C::Word* __restrict__ states, int64_t D,
                                                              const uint8_t* __restrict__ flag,
                                                              const uint32_t* __restrict__ offset,
                                                              typename C::Word* __restrict__ reps,
                                                              double* __restrict__ norm, double* __restrict__ diag,
                                                              uint32_t* __restrict__ map) {
  __shared__ uint32_t sm[kMomThreads / 32];
  const int64_t nch = (D + kMomChunk - 1) / kMomChunk;
  for (int64_t c = blockIdx.x; c < nch; c += gridDim.x) {
    const int64_t r0 = c * kMomChunk + (int64_t)threadIdx.x * 8;
    uint32_t n = 0;
    for (int u = 0; u < 8; ++u) n += (r0 + u < D && flag[r0 + u]) ? 1u : 0u;
    uint32_t total;
    uint32_t idx = offset[c] + block_exclusive_scan(n, sm, &total);
    for (int u = 0; u < 8; ++u) {
      const int64_t r = r0 + u;
      if (r >= D) break;
      if (flag[r]) {
        const typename C::Word s = states[r];
        reps[idx] = s;
        norm[idx] = orbit_weight(orbit_of(mp, cd, s)) * mp.inv_sqrt_n;
        if constexpr (std::is_same<C, BitCodec>::value) {
          if (diag) diag[idx] = diag_of(P, s);
        }
        map[r] = idx;
        ++idx;
      } else {
        map[r] = kMomNone;
      }
    }
  }
}

// Pass 3: every state that is not the smallest of its orbit maps to the
// representative of its orbit through the first translation reaching it
// (blochbasisstates.h:221-230); reads only entries of orbit minima, which
// this pass does not write.
template <class C>
__global__ void __launch_bounds__(kMomThreads) mom_member_kernel(const __grid_constant__ MomParams mp, const C cd,
                                                                 const typename C::Word* __restrict__ states,
                                                                 int64_t D, uint32_t* __restrict__ map) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < D; r += (int64_t)gridDim.x * blockDim.x) {
    const typename C::Word s = states[r];
    const auto o = orbit_of(mp, cd, s);
    if (o.min == s) continue;
    const uint32_t e = map[cd.rank(o.min)];
    map[r] = e == kMomNone ? kMomNone : ((uint32_t)o.tmin << kMomRepBits) | e;
  }
}

__global__ void __launch_bounds__(kMomThreads) mom_diag_kernel(const __grid_constant__ HvParams P,
                                                               const uint32_t* __restrict__ reps, int64_t dim,
                                                               double* __restrict__ diag) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < dim; i += (int64_t)gridDim.x * blockDim.x)
    diag[i] = diag_of(P, reps[i]);
}

// y = H x, interleaved complex.  Flip list and phases staged in shared memory.
__global__ void __launch_bounds__(kMomThreads) mom_hv_kernel(const __grid_constant__ MomParams mp, const DevTables t,
                                                             const MomTables m, const double2* __restrict__ x,
                                                             double2* __restrict__ y, double* __restrict__ alpha_part) {
  __shared__ uint32_t fm[kMaxBonds];
  __shared__ double fc[kMaxBonds];
  __shared__ double pre[kMaxTrans], pim[kMaxTrans];
  __shared__ double red[33];
  for (int q = threadIdx.x; q < mp.n_flip; q += kMomThreads) {
    fm[q] = mp.flip_mask[q];
    fc[q] = mp.flip_c[q];
  }
  for (int q = threadIdx.x; q < mp.n_trans; q += kMomThreads) {
    pre[q] = mp.phase_re[q];
    pim[q] = mp.phase_im[q];
  }
  __syncthreads();
  const uint32_t lm = (1u << t.Nlo) - 1u;
  const uint32_t jmask = (1u << kMomRepBits) - 1u;
  const int nf = mp.n_flip;
  const int64_t ntile = mom_tiles(m.dim);
  for (int64_t tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    double dot = 0.0;
    for (int u = 0; u < kMomTileRows / kMomThreads; ++u) {
      const int64_t i = tile * kMomTileRows + u * kMomThreads + threadIdx.x;
      if (i >= m.dim) break;
      const uint32_t r = m.reps[i];
      const double ni = m.norm[i];
      const double2 xi = x[i];
      const double d = m.diag[i];
      double are = d * xi.x, aim = d * xi.y;
      for (int q = 0; q < nf; ++q) {
        const uint32_t b = r & fm[q];
        if (b == 0u || b == fm[q]) continue;  // parallel spins: no flip
        const uint32_t s2 = r ^ fm[q];
        const uint32_t e = __ldg(m.map + __ldg(t.thi + (s2 >> t.Nlo)) + __ldg(t.tlo + (s2 & lm)));
        if (e == kMomNone) continue;
        const uint32_t j = e & jmask, tt = e >> kMomRepBits;
        const double f = fc[q] * (__ldg(m.norm + j) / ni);
        const double cr = f * pre[tt], ci = f * pim[tt];
        const double2 xj = x[j];
        are = fma(cr, xj.x, fma(-ci, xj.y, are));
        aim = fma(cr, xj.y, fma(ci, xj.x, aim));
      }
      y[i] = make_double2(are, aim);
      dot = fma(xi.x, are, fma(xi.y, aim, dot));
    }
    if (alpha_part) {
      const double tot = block_sum_all<kMomThreads>(dot, red);
      if (threadIdx.x == 0) alpha_part[tile] = tot;
    }
  }
}

// One pass per call: each CTA sums its rows' terms into part[blockIdx.x].
template <int KIND>
__global__ void __launch_bounds__(kMomThreads) mom_expect_kernel(const __grid_constant__ MomParams mp,
                                                                 const DevTables t, const MomTables m,
                                                                 const double2* __restrict__ psi,
                                                                 const __grid_constant__ MomPairs pairs,
                                                                 double* __restrict__ part) {
  __shared__ double pre[kMaxTrans], pim[kMaxTrans];
  __shared__ double red[33];
  for (int q = threadIdx.x; q < mp.n_trans; q += kMomThreads) {
    pre[q] = mp.phase_re[q];
    pim[q] = mp.phase_im[q];
  }
  __syncthreads();
  const uint32_t lm = (1u << t.Nlo) - 1u;
  const uint32_t jmask = (1u << kMomRepBits) - 1u;
  double acc = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)kMomThreads + threadIdx.x; i < m.dim; i += (int64_t)gridDim.x * kMomThreads) {
    const uint32_t r = m.reps[i];
    const double2 pi = psi[i];
    const double w = pi.x * pi.x + pi.y * pi.y;
    double d = 0.0;    // diagonal part of the pair sum on r
    double ore = 0.0;  // Re conj(psi_i) (off-diagonal part applied to psi)_i
    for (int p = 0; p < pairs.n; ++p) {
      const uint32_t mi = pairs.mi[p], mj = pairs.mj[p];
      if (KIND == AED_OBS_SZ) {
        d += (r & mi) ? 0.5 : -0.5;
      } else if (KIND == AED_OBS_SZSZ) {
        d += ((r & mi) ? 0.5 : -0.5) * ((r & mj) ? 0.5 : -0.5);
      } else if (mi == mj) {
        d += (r & mi) ? 1.0 : 0.0;
      } else if (!(r & mi) && (r & mj)) {
        const uint32_t s2 = r ^ mi ^ mj;
        const uint32_t e = __ldg(m.map + __ldg(t.thi + (s2 >> t.Nlo)) + __ldg(t.tlo + (s2 & lm)));
        if (e == kMomNone) continue;
        const uint32_t j = e & jmask, tt = e >> kMomRepBits;
        const double f = __ldg(m.norm + j) / m.norm[i];
        const double cr = f * pre[tt], ci = f * pim[tt];
        const double2 xj = psi[j];
        // conj(psi_i) * (c * psi_j), real part
        const double yr = cr * xj.x - ci * xj.y, yi = cr * xj.y + ci * xj.x;
        ore += pi.x * yr + pi.y * yi;
      }
    }
    acc += w * d + ore;
  }
  const double tot = block_sum_all<kMomThreads>(acc, red);
  if (threadIdx.x == 0) part[blockIdx.x] = tot;
}

int grid_for(int64_t units) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t cap = (int64_t)sms * 8;
  return (int)(units < 1 ? 1 : (units < cap ? units : cap));
}

// The sector's states in basis order (the two-table ranks' inverse).
int fill_states(const BitCodec& c, uint32_t* states, int64_t D, cudaStream_t st) {
  return launch_basis_copy(c.t, states, 0, D, st);
}
int fill_states(const DigitCodec& c, uint64_t* states, int64_t D, cudaStream_t st) {
  return launch_spin_basis(c.t, states, 0, D, st);
}

// The three passes over the D states of the Sz sector (flags and counts, host
// scan of the counts, representatives, members).  diag == nullptr: no
// diagonal array.
template <class C>
int mom_build_t(const MomParams& mp, const HvParams& P, const C& cd, int64_t D, cudaStream_t st,
                typename C::Word** reps, double** norm, double** diag, uint32_t** map, int64_t* dim) {
  using W = typename C::Word;
  *reps = nullptr;
  *norm = nullptr;
  if (diag) *diag = nullptr;
  *map = nullptr;
  *dim = 0;
  if (D == 0) return AED_OK;
  const int64_t nch = (D + kMomChunk - 1) / kMomChunk;
  W* states = nullptr;
  uint8_t* flag = nullptr;
  uint32_t *count = nullptr, *offset = nullptr;
  int rc = AED_OK;
  auto cleanup = [&] {
    mem_dev_free(states, st);
    mem_dev_free(flag, st);
    mem_dev_free(count, st);
    mem_dev_free(offset, st);
  };
  if ((rc = mem_dev_alloc_n(&states, (size_t)D)) || (rc = mem_dev_alloc_n(&flag, (size_t)D)) ||
      (rc = mem_dev_alloc_n(&count, (size_t)nch)) || (rc = mem_dev_alloc_n(&offset, (size_t)nch)) ||
      (rc = fill_states(cd, states, D, st))) {
    cleanup();
    return rc;
  }
  mom_flag_kernel<C><<<grid_for(nch), kMomThreads, 0, st>>>(mp, cd, states, D, flag, count);
  if ((rc = check_launch_counted("mom_flag_kernel"))) {
    cleanup();
    return rc;
  }
  std::vector<uint32_t> hc((size_t)nch), ho((size_t)nch);
  cudaMemcpyAsync(hc.data(), count, (size_t)nch * 4, cudaMemcpyDeviceToHost, st);
  const cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    cleanup();
    return fail(AED_ERR_CUDA, std::string("momentum basis scan: ") + cudaGetErrorString(e));
  }
  uint64_t total = 0;
  for (int64_t c = 0; c < nch; ++c) {
    ho[(size_t)c] = (uint32_t)total;
    total += hc[(size_t)c];
  }
  if (total >= ((uint64_t)1 << kMomRepBits)) {
    cleanup();
    return fail(AED_ERR_INVALID, "momentum sector larger than 2^26 representatives");
  }
  if ((rc = mem_dev_alloc_n(reps, (size_t)total)) || (rc = mem_dev_alloc_n(norm, (size_t)total)) ||
      (diag && (rc = mem_dev_alloc_n(diag, (size_t)total))) || (rc = mem_dev_alloc_n(map, (size_t)D))) {
    cleanup();
    return rc;
  }
  cudaMemcpyAsync(offset, ho.data(), (size_t)nch * 4, cudaMemcpyHostToDevice, st);
  mom_rep_kernel<C><<<grid_for(nch), kMomThreads, 0, st>>>(mp, P, cd, states, D, flag, offset, *reps, *norm,
                                                          diag ? *diag : nullptr, *map);
  if (!(rc = check_launch_counted("mom_rep_kernel"))) {
    mom_member_kernel<C><<<grid_for((D + kMomThreads - 1) / kMomThreads), kMomThreads, 0, st>>>(mp, cd, states, D,
                                                                                                 *map);
    rc = check_launch_counted("mom_member_kernel");
  }
  if (!rc) {
    const cudaError_t e2 = cudaStreamSynchronize(st);  // ho goes out of scope
    if (e2 != cudaSuccess) rc = fail(AED_ERR_CUDA, std::string("momentum basis: ") + cudaGetErrorString(e2));
  }
  cleanup();
  *dim = (int64_t)total;
  return rc;
}

}  // namespace

int mom_build(const MomParams& mp, const HvParams& P, const DevTables& t, cudaStream_t st, uint32_t** reps,
              double** norm, double** diag, uint32_t** map, int64_t* dim) {
  return mom_build_t(mp, P, BitCodec{t}, t.D, st, reps, norm, diag, map, dim);
}

int spin_mom_build(const MomParams& mp, const SpinDev& t, cudaStream_t st, uint64_t** reps, double** norm,
                   uint32_t** map, int64_t* dim) {
  static const HvParams no_diag{};  // the spin-S apply forms its diagonal itself
  return mom_build_t(mp, no_diag, DigitCodec{t}, t.D, st, reps, norm, (double**)nullptr, map, dim);
}

int launch_mom_diag(const HvParams& P, const uint32_t* reps, int64_t dim, double* diag, cudaStream_t st) {
  if (dim == 0) return AED_OK;
  mom_diag_kernel<<<grid_for((dim + kMomThreads - 1) / kMomThreads), kMomThreads, 0, st>>>(P, reps, dim, diag);
  return check_launch_counted("mom_diag_kernel");
}

int mom_expect_grid(int64_t dim) { return grid_for((dim + kMomThreads - 1) / kMomThreads); }

int mom_expectation(const MomParams& mp, const DevTables& t, const MomTables& m, const double* psi, int kind,
                    const MomPairs& pairs, double* part, int grid, cudaStream_t st) {
  const double2* p2 = reinterpret_cast<const double2*>(psi);
  if (kind == AED_OBS_SZ)
    mom_expect_kernel<AED_OBS_SZ><<<grid, kMomThreads, 0, st>>>(mp, t, m, p2, pairs, part);
  else if (kind == AED_OBS_SZSZ)
    mom_expect_kernel<AED_OBS_SZSZ><<<grid, kMomThreads, 0, st>>>(mp, t, m, p2, pairs, part);
  else
    mom_expect_kernel<AED_OBS_SPSM><<<grid, kMomThreads, 0, st>>>(mp, t, m, p2, pairs, part);
  return check_launch_counted("mom_expect_kernel");
}

int launch_mom_hv(const MomParams& mp, const DevTables& t, const MomTables& m, const double* x, double* y,
                  double* alpha_part, cudaStream_t st) {
  if (m.dim == 0) return AED_OK;
  mom_hv_kernel<<<grid_for(mom_tiles(m.dim)), kMomThreads, 0, st>>>(mp, t, m, reinterpret_cast<const double2*>(x),
                                                                     reinterpret_cast<double2*>(y), alpha_part);
  return check_launch_counted("mom_hv_kernel");
}

}  // namespace aed
