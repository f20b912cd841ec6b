// spin.cu -- Sz sectors of spin-S models (S = 1/2, 1, 3/2, 2): the sector's
// tables, the rank -> state copy and the apply y = H x.  Layout: spin.cuh.
//
// H = sum_i (-h_i Sz_i + D_i Sz_i^2) + sum_bonds (Jz Sz_i Sz_j + Jxy exchange_xy(i,j)
//     + K biquadratic(i,j)), the spin HAMILTONIAN of lib/xml/models.xml.in:342-373
// with the site operators of :24-36 (S+ |m> = sqrt(S(S+1) - m(m+1)) |m+1>) and
// the bond operators of :290-300 (biquadratic = (exchange_xy + Sz Sz)^2).
// Each row takes its site terms, then its bonds in order; a bond contributes
// the transitions of its two digits (the diagonal one to M(i,i)).  Rows agree
// with the reference's explicit matrix to rounding (the local elements come
// from the operator algebra in another order than the reference's symbolic
// evaluation); the spin-1/2 engine's bit-exact rows are the handles of
// aed_create.
//
// Reference paths are relative to the ALPS source tree.

#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "handle.h"
#include "reduce.cuh"
#include "spin.cuh"

namespace aed {

int build_spin_tables(int N, int twoS, int T, SpinTables& t) {
  t = SpinTables();
  if (twoS < 1 || twoS + 1 > kSpinMaxDim) return fail(AED_ERR_INVALID, "local spin S must be in 1/2 .. 2");
  const int d = twoS + 1;
  int bits = 1;
  while ((1 << bits) < d) ++bits;
  if (N < 1 || N > kSpinMaxSites || N * bits > 48)
    return fail(AED_ERR_INVALID, "spin sector: number of sites x bits per site must be at most 48");
  t.N = N;
  t.twoS = twoS;
  t.d = d;
  t.bits = bits;
  t.Nl = N / 2;
  t.Nh = N - t.Nl;
  t.T = T;
  const int maxlo = (d - 1) * t.Nl, maxhi = (d - 1) * t.Nh;
  if (T < 0 || T > maxlo + maxhi) return fail(AED_ERR_INVALID, "Sz_total outside the range of the sites");
  auto digits_ok_sum = [&](uint32_t code, int n, int* sum) {
    int s = 0;
    for (int i = 0; i < n; ++i) {
      const int v = (int)((code >> (bits * i)) & ((1u << bits) - 1u));
      if (v >= d) return false;
      s += v;
    }
    *sum = s;
    return true;
  };
  const uint32_t nlo = 1u << (bits * t.Nl), nhi = 1u << (bits * t.Nh);
  std::vector<uint32_t> count(maxlo + 1, 0);
  t.tlo.assign(nlo, kSpinNone);
  std::vector<int> losum(nlo, -1);
  for (uint32_t c = 0; c < nlo; ++c) {
    int s;
    if (digits_ok_sum(c, t.Nl, &s)) {
      losum[c] = s;
      t.tlo[c] = count[s]++;
    }
  }
  t.looff.assign(maxlo + 2, 0);
  for (int k = 0; k <= maxlo; ++k) t.looff[k + 1] = t.looff[k] + count[k];
  t.lolist.assign(t.looff[maxlo + 1], 0);
  {
    std::vector<uint32_t> fill(t.looff.begin(), t.looff.end() - 1);
    for (uint32_t c = 0; c < nlo; ++c)
      if (losum[c] >= 0) t.lolist[fill[losum[c]]++] = c;
  }
  t.thi.assign(nhi, kSpinNone);
  uint64_t run = 0;
  for (uint32_t h = 0; h < nhi; ++h) {
    int s;
    if (!digits_ok_sum(h, t.Nh, &s)) continue;
    const int k = T - s;
    if (k < 0 || k > maxlo || count[k] == 0) continue;
    t.thi[h] = (uint32_t)run;
    t.blk_hi.push_back(h);
    t.blk_off.push_back((uint32_t)run);
    for (uint32_t r0 = 0; r0 < count[k]; r0 += kSpinTileRows) {
      t.tile_blk.push_back((uint32_t)(t.blk_hi.size() - 1));
      t.tile_r.push_back(r0);
    }
    run += count[k];
    if (run >= 0xffffffffull) return fail(AED_ERR_INVALID, "spin sector larger than 2^32 states");
  }
  t.D = (int64_t)run;
  return AED_OK;
}

void spin_set_couplings(const std::vector<int>& s1, const std::vector<int>& s2, const std::vector<double>& jz,
                        const std::vector<double>& jxy, const std::vector<double>& kq,
                        const std::vector<double>& site_h, const std::vector<double>& site_d, int N, SpinParams& p) {
  p.N = N;
  p.n_bonds = (int)s1.size();
  const int d = p.twoS + 1;
  const double S = p.twoS / 2.0;
  for (int i = 0; i < N; ++i) {
    p.site_h[i] = site_h.empty() ? 0.0 : site_h[i];
    p.site_d[i] = site_d.empty() ? 0.0 : site_d[i];
    for (int v = 0; v < d; ++v) {
      const double m = v - S;
      p.sdiag[i][v] = -p.site_h[i] * m + p.site_d[i] * m * m;
    }
  }
  p.n_cls = 0;
  bool tab = true;
  for (int b = 0; b < p.n_bonds; ++b) {
    p.s1[b] = s1[b];
    p.s2[b] = s2[b];
    p.jz[b] = jz[b];
    p.jxy[b] = jxy[b];
    p.kq[b] = kq[b];
    int c = 0;
    while (c < p.n_cls && !(p.jz[p.cls[c]] == jz[b] && p.jxy[p.cls[c]] == jxy[b] && p.kq[p.cls[c]] == kq[b])) ++c;
    if (c == p.n_cls) {  // a new class: cls[c] temporarily names its first bond
      if (p.n_cls == kSpinMaxCls) {
        tab = false;
        break;
      }
      p.cls[p.n_cls++] = b;
    }
  }
  if (!tab) {
    for (int b = 0; b < p.n_bonds; ++b) {
      p.s1[b] = s1[b];
      p.s2[b] = s2[b];
      p.jz[b] = jz[b];
      p.jxy[b] = jxy[b];
      p.kq[b] = kq[b];
    }
    p.n_cls = 0;
    return;
  }
  int first[kSpinMaxCls];
  for (int c = 0; c < p.n_cls; ++c) first[c] = p.cls[c];
  p.pmo = 0;
  for (int c = 0; c < p.n_cls; ++c)
    for (int pr = 0; pr < d * d; ++pr) {
      const int a = pr / d, cc = pr % d;
      int n = 0;
      p.pdg[c][pr] = 0.0;
      p.pk[c][pr] = 0;
      for (int s = 0; s < kSpinMaxOff; ++s) p.pov[c][pr][s] = 0.0;
      for (int e = p.tstart[pr]; e < p.tstart[pr + 1]; ++e) {
        const double v = p.jz[first[c]] * p.trans[e].A + p.jxy[first[c]] * p.trans[e].B + p.kq[first[c]] * p.trans[e].C;
        const int k = p.trans[e].a2 - a;
        if (k == 0 && p.trans[e].c2 == cc) {
          p.pdg[c][pr] = v;
        } else if (v != 0.0) {
          if (k == 0 || p.trans[e].c2 - cc != -k || n == kSpinMaxOff) {  // not of the form (a + k, c - k)
            p.n_cls = 0;
            return;
          }
          p.pov[c][pr][n] = v;
          p.pk[c][pr] |= (uint32_t)(k & 255) << (8 * n);
          ++n;
        }
      }
      p.pmo = std::max(p.pmo, n);
    }
  for (int b = 0; b < p.n_bonds; ++b) {
    int c = 0;
    while (!(p.jz[first[c]] == jz[b] && p.jxy[first[c]] == jxy[b] && p.kq[first[c]] == kq[b])) ++c;
    p.cls[b] = c;
  }
}

void spin_transitions(int twoS, SpinParams& p) {
  p.twoS = twoS;
  const int d = twoS + 1;
  const double S = twoS / 2.0;
  auto m = [&](int v) { return v - S; };
  const int n2 = d * d;
  // two-site matrices on (a, c) -> index a d + c: A = Sz Sz, B = exchange_xy, C = (A + B)^2
  std::vector<double> A(n2 * n2, 0.0), B(n2 * n2, 0.0), X(n2 * n2, 0.0), C(n2 * n2, 0.0);
  auto at = [&](std::vector<double>& M, int row, int col) -> double& { return M[(size_t)row * n2 + col]; };
  for (int a = 0; a < d; ++a)
    for (int c = 0; c < d; ++c) {
      const int src = a * d + c;
      at(A, src, src) = m(a) * m(c);
      if (a + 1 < d && c - 1 >= 0)  // S+_i S-_j: <m+1|S+|m> <m-1|S-|m>
        at(B, (a + 1) * d + (c - 1), src) += 0.5 * std::sqrt(S * (S + 1) - m(a) * (m(a) + 1)) *
                                              std::sqrt(S * (S + 1) - m(c) * (m(c) - 1));
      if (a - 1 >= 0 && c + 1 < d)  // S-_i S+_j
        at(B, (a - 1) * d + (c + 1), src) += 0.5 * std::sqrt(S * (S + 1) - m(a) * (m(a) - 1)) *
                                              std::sqrt(S * (S + 1) - m(c) * (m(c) + 1));
    }
  for (int k = 0; k < n2 * n2; ++k) X[k] = A[k] + B[k];
  for (int r = 0; r < n2; ++r)
    for (int c = 0; c < n2; ++c) {
      double s = 0.0;
      for (int q = 0; q < n2; ++q) s += X[(size_t)r * n2 + q] * X[(size_t)q * n2 + c];
      C[(size_t)r * n2 + c] = s;
    }
  int n = 0;
  for (int src = 0; src < n2; ++src) {
    p.tstart[src] = n;
    for (int dst = 0; dst < n2; ++dst) {  // targets in (a2, c2) order, as the reference loops js1, js2
      const double a = at(A, dst, src), b = at(B, dst, src), c = at(C, dst, src);
      if (a == 0.0 && b == 0.0 && c == 0.0) continue;
      p.trans[n++] = {(uint8_t)(dst / d), (uint8_t)(dst % d), a, b, c};
    }
  }
  p.tstart[n2] = n;
}

namespace {

constexpr int kSpinThreads = 256;

__global__ void spin_basis_kernel(const SpinDev t, uint64_t* __restrict__ out, int64_t offset, int64_t count) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= count) return;
  const uint32_t idx = (uint32_t)(offset + n);
  int64_t lo = 0, hi = t.n_blk - 1;
  while (lo < hi) {  // the block holding row idx: the last with blk_off <= idx
    const int64_t mid = lo + (hi - lo + 1) / 2;
    if (t.blk_off[mid] <= idx)
      lo = mid;
    else
      hi = mid - 1;
  }
  const uint32_t h = t.blk_hi[lo];
  int sum = 0;
  for (int i = 0; i < t.N - t.Nl; ++i) sum += (int)((h >> (t.bits * i)) & ((1u << t.bits) - 1u));
  const uint32_t r = idx - t.blk_off[lo];
  out[n] = ((uint64_t)h << (t.bits * t.Nl)) | t.lolist[t.looff[t.T - sum] + r];
}

// The couplings of SpinParams staged in shared memory for the row walk, when
// more than kSpinMaxCls coupling classes leave the elements untabulated.  A
// state is a hi word (the first Nh = N - Nl sites) and a lo word (the last Nl
// sites), each with `bits` bits per site; bw1 / bw2 are the shifts of a bond's
// two digits within their words and bk its kind: 0 both sites in lo, 1 both
// in hi, 2 site i in hi and j in lo, 3 site i in lo and j in hi.
struct SpinShared {
  double cv[3 * kSpinMaxTrans];  // A, B, C of each transition
  short2 dl[kSpinMaxTrans];      // digit changes (a2 - a, c2 - c) of each transition
  int ts[kSpinMaxPairs + 1];
  int bw1[kMaxBonds], bw2[kMaxBonds], bk[kMaxBonds];
  double bj[3][kMaxBonds];
  double sdg[kSpinMaxSites * kSpinMaxDim];
};

// The tabulated form (every bond in one of at most kSpinMaxCls coupling
// classes; D = 2S + 1 digits, MO >= SpinParams::pmo off-diagonal slots):
// per class and digit pair the diagonal element, the nonzero off-diagonal
// ones and their k; per bond one record
//   x  class x D^2 (its pair tables),
//   y  wi | wj << 8 | (site i in hi) << 16 | (site j in hi) << 17,
//   z  bh, w  bl: the change of the hi and of the lo word per unit of k.
// A transition (a, c) -> (a + k, c - k) moves hi to hi + k bh and lo to
// lo + k bl; a word it leaves alone keeps its part of the rank (the block's
// first row for hi, the rank r within the block for lo), so a bond inside one
// word looks up one table and only a bond across the split looks up both.
template <int D, int MO>
struct SpinTabShared {
  double dg[kSpinMaxCls * D * D];
  double ov[kSpinMaxCls * D * D * MO];
  uint32_t pk[kSpinMaxCls * D * D];
  int4 bond[kMaxBonds];
  double sdg[kSpinMaxSites * D];
};

// In the Sz-sector apply all rows of a work tile share their hi word, so a
// bond with both sites in hi has the same digits, elements and target hi
// words in every row: the CTA forms them once per tile.  tb = thi of the
// target hi word (the target row is tb + r), kSpinNone for an empty slot.
template <int MO>
struct SpinTileHi {
  double dg[kMaxBonds];
  double v[kMaxBonds][MO];
  uint32_t tb[kMaxBonds][MO];
};
template <class Sh>
struct TileHiOf {
  using type = char;
};
template <int D, int MO>
struct TileHiOf<SpinTabShared<D, MO>> {
  using type = SpinTileHi<MO>;
};

// Bond record flags: bit 0 site i in hi, bit 1 site j in hi.
__device__ __forceinline__ int bond_side(const int4& b) { return (b.y >> 16) & 3; }

__device__ __forceinline__ int stage_site_terms(const SpinParams& p, int N, int d, double* sdg) {
  int nz = 0;
  for (int q = threadIdx.x; q < N * d; q += blockDim.x) {
    sdg[q] = p.sdiag[q / d][q % d];
    nz |= sdg[q] != 0.0;
  }
  return nz;
}

// Fill sh (all threads of the CTA); returns whether this thread staged a
// nonzero site term (the caller reduces it with __syncthreads_or, which is
// also the barrier after the staging).
__device__ __forceinline__ int stage_spin(const SpinParams& p, const SpinDev& t, SpinShared& sh) {
  const int d = t.d, N = t.N, bits = t.bits, Nl = t.Nl, Nh = N - Nl;
  const int ntr = p.tstart[d * d];
  for (int q = threadIdx.x; q <= d * d; q += blockDim.x) sh.ts[q] = p.tstart[q];
  for (int pr = threadIdx.x; pr < d * d; pr += blockDim.x)
    for (int e = p.tstart[pr]; e < p.tstart[pr + 1]; ++e)
      sh.dl[e] = make_short2((short)(p.trans[e].a2 - pr / d), (short)(p.trans[e].c2 - pr % d));
  for (int q = threadIdx.x; q < ntr; q += blockDim.x) {
    sh.cv[3 * q] = p.trans[q].A;
    sh.cv[3 * q + 1] = p.trans[q].B;
    sh.cv[3 * q + 2] = p.trans[q].C;
  }
  for (int q = threadIdx.x; q < p.n_bonds; q += blockDim.x) {
    const int i = p.s1[q], j = p.s2[q];
    const bool li = i >= Nh, lj = j >= Nh;
    sh.bw1[q] = li ? bits * (N - 1 - i) : bits * (Nh - 1 - i);
    sh.bw2[q] = lj ? bits * (N - 1 - j) : bits * (Nh - 1 - j);
    sh.bk[q] = (li && lj) ? 0 : (!li && !lj) ? 1 : !li ? 2 : 3;
    sh.bj[0][q] = p.jz[q];
    sh.bj[1][q] = p.jxy[q];
    sh.bj[2][q] = p.kq[q];
  }
  return stage_site_terms(p, N, d, sh.sdg);
}

template <int D, int MO>
__device__ __forceinline__ int stage_spin(const SpinParams& p, const SpinDev& t, SpinTabShared<D, MO>& sh) {
  constexpr int P = D * D;
  const int N = t.N, bits = t.bits, Nh = N - t.Nl;
  for (int q = threadIdx.x; q < p.n_cls * P; q += blockDim.x) {
    const int c = q / P, pr = q % P;
    sh.dg[q] = p.pdg[c][pr];
    sh.pk[q] = p.pk[c][pr];
#pragma unroll
    for (int s = 0; s < MO; ++s) sh.ov[q * MO + s] = s < kSpinMaxOff ? p.pov[c][pr][s] : 0.0;
  }
  for (int q = threadIdx.x; q < p.n_bonds; q += blockDim.x) {
    const int i = p.s1[q], j = p.s2[q];
    const bool li = i >= Nh, lj = j >= Nh;
    const int wi = li ? bits * (N - 1 - i) : bits * (Nh - 1 - i);
    const int wj = lj ? bits * (N - 1 - j) : bits * (Nh - 1 - j);
    int bh, bl;
    if (li && lj) {
      bh = 0;
      bl = (1 << wi) - (1 << wj);
    } else if (!li && !lj) {
      bh = (1 << wi) - (1 << wj);
      bl = 0;
    } else if (!li) {
      bh = 1 << wi;
      bl = -(1 << wj);
    } else {
      bh = -(1 << wj);
      bl = 1 << wi;
    }
    sh.bond[q] = make_int4(p.cls[q] * P, wi | (wj << 8) | ((int)!li << 16) | ((int)!lj << 17), bh, bl);
  }
  return stage_site_terms(p, N, D, sh.sdg);
}

// One row of H: state (h, lo), its block's first row `base` and its rank r
// within the block (row = base + r).  Returns the diagonal element (site
// terms in site order unless all are zero, then the diagonal transitions of
// the bonds in order) and calls off(v, rank) for every off-diagonal
// transition, bonds in order.  A bond inside lo keeps the hi word (rank =
// base + tlo[lo']), a bond inside hi keeps lo (rank = thi[h'] + r); only
// bonds across the split rank through both tables.
template <class Off>
__device__ __forceinline__ double spin_row(const SpinShared& sh, int n_bonds, bool has_site, const SpinDev& t,
                                           uint32_t h, uint32_t lo, uint32_t base, uint32_t r, Off&& off) {
  const int d = t.d, N = t.N, bits = t.bits, Nh = N - t.Nl;
  const uint32_t dm = (1u << bits) - 1u;
  double dg = 0.0;
  if (has_site) {  // -h Sz + D Sz^2
    for (int i = 0; i < Nh; ++i) dg += sh.sdg[i * d + (int)((h >> (bits * (Nh - 1 - i))) & dm)];
    for (int i = Nh; i < N; ++i) dg += sh.sdg[i * d + (int)((lo >> (bits * (N - 1 - i))) & dm)];
  }
  for (int q = 0; q < n_bonds; ++q) {
    const int k = sh.bk[q], wi = sh.bw1[q], wj = sh.bw2[q];
    const uint32_t wa = (k == 0 || k == 3) ? lo : h;  // the word holding site i
    const uint32_t wc = (k == 0 || k == 2) ? lo : h;  // the word holding site j
    const int a = (int)((wa >> wi) & dm), c = (int)((wc >> wj) & dm);
    const int pr = a * d + c;
    for (int e = sh.ts[pr]; e < sh.ts[pr + 1]; ++e) {
      const double v = sh.bj[0][q] * sh.cv[3 * e] + sh.bj[1][q] * sh.cv[3 * e + 1] + sh.bj[2][q] * sh.cv[3 * e + 2];
      const short2 dl = sh.dl[e];
      if (dl.x == 0 && dl.y == 0) {
        dg += v;
        continue;
      }
      const uint32_t di = (uint32_t)((int)dl.x * (1 << wi)), dj = (uint32_t)((int)dl.y * (1 << wj));
      uint32_t rk;
      if (k == 0)
        rk = base + __ldg(t.tlo + (lo + di + dj));
      else if (k == 1)
        rk = __ldg(t.thi + (h + di + dj)) + r;
      else if (k == 2)
        rk = __ldg(t.thi + (h + di)) + __ldg(t.tlo + (lo + dj));
      else
        rk = __ldg(t.thi + (h + dj)) + __ldg(t.tlo + (lo + di));
      off(v, rk);
    }
  }
  return dg;
}

// The same row from the tabulated form: the same diagonal sum and the same
// off-diagonal calls in the same order, less the zero elements.
template <int D, int MO, class Off>
__device__ __forceinline__ double spin_row(const SpinTabShared<D, MO>& sh, int n_bonds, bool has_site,
                                           const SpinDev& t, uint32_t h, uint32_t lo, uint32_t base, uint32_t r,
                                           Off&& off) {
  constexpr int BITS = D <= 2 ? 1 : D <= 4 ? 2 : 3;
  constexpr uint32_t dm = (1u << BITS) - 1u;
  const int N = t.N, Nh = N - t.Nl;
  double dg = 0.0;
  if (has_site) {
    for (int i = 0; i < Nh; ++i) dg += sh.sdg[i * D + (int)((h >> (BITS * (Nh - 1 - i))) & dm)];
    for (int i = Nh; i < N; ++i) dg += sh.sdg[i * D + (int)((lo >> (BITS * (N - 1 - i))) & dm)];
  }
  for (int q = 0; q < n_bonds; ++q) {
    const int4 b = sh.bond[q];
    const uint32_t wa = (b.y & 0x10000) ? h : lo, wc = (b.y & 0x20000) ? h : lo;
    const int a = (int)((wa >> (b.y & 255)) & dm), c = (int)((wc >> ((b.y >> 8) & 255)) & dm);
    const int pr = b.x + a * D + c;
    dg += sh.dg[pr];
    const uint32_t kp = sh.pk[pr];
#pragma unroll
    for (int s = 0; s < MO; ++s) {
      const int k = (int)(int8_t)(uint8_t)(kp >> (8 * s));
      if (k != 0) {
        const uint32_t th = b.z ? __ldg(t.thi + (h + (uint32_t)(k * b.z))) : base;
        const uint32_t tl = b.w ? __ldg(t.tlo + (lo + (uint32_t)(k * b.w))) : r;
        off(sh.ov[pr * MO + s], th + tl);
      }
    }
  }
  return dg;
}

// The hi-hi bonds' shared entries of the tile whose hi word is h (all threads
// of the CTA; barriers before, against the readers of the last tile, and after).
template <int D, int MO>
__device__ __forceinline__ void tile_hi_entries(const SpinTabShared<D, MO>& sh, SpinTileHi<MO>& hh, int n_bonds,
                                                const SpinDev& t, uint32_t h) {
  constexpr int BITS = D <= 2 ? 1 : D <= 4 ? 2 : 3;
  constexpr uint32_t dm = (1u << BITS) - 1u;
  __syncthreads();
  for (int q = threadIdx.x; q < n_bonds; q += blockDim.x) {
    const int4 b = sh.bond[q];
    if (bond_side(b) != 3) continue;
    const int a = (int)((h >> (b.y & 255)) & dm), c = (int)((h >> ((b.y >> 8) & 255)) & dm);
    const int pr = b.x + a * D + c;
    hh.dg[q] = sh.dg[pr];
    const uint32_t kp = sh.pk[pr];
#pragma unroll
    for (int s = 0; s < MO; ++s) {
      const int k = (int)(int8_t)(uint8_t)(kp >> (8 * s));
      hh.v[q][s] = sh.ov[pr * MO + s];
      hh.tb[q][s] = k != 0 ? __ldg(t.thi + (h + (uint32_t)(k * b.z))) : kSpinNone;
    }
  }
  __syncthreads();
}

// The tabulated row of the Sz-sector apply: hi-hi bonds from the tile's
// entries, lo-lo bonds from the lo table (u = the row's lo code's index in
// lolist), bonds across the split as spin_row.  The same diagonal sum and the
// same off-diagonal calls in the same order as spin_row.
template <int D, int MO, class Off>
__device__ __forceinline__ double spin_row_tile(const SpinTabShared<D, MO>& sh, const SpinTileHi<MO>& hh, int n_bonds,
                                                bool has_site, const SpinDev& t, uint32_t h, uint32_t lo,
                                                uint32_t base, uint32_t r, uint32_t u, Off&& off) {
  constexpr int BITS = D <= 2 ? 1 : D <= 4 ? 2 : 3;
  constexpr uint32_t dm = (1u << BITS) - 1u;
  const int N = t.N, Nh = N - t.Nl;
  const bool lot = MO <= 2 && t.lol != nullptr;
  double dg = 0.0;
  if (has_site) {
    for (int i = 0; i < Nh; ++i) dg += sh.sdg[i * D + (int)((h >> (BITS * (Nh - 1 - i))) & dm)];
    for (int i = Nh; i < N; ++i) dg += sh.sdg[i * D + (int)((lo >> (BITS * (N - 1 - i))) & dm)];
  }
  const uint2* lol = t.lol + u;
  for (int q = 0; q < n_bonds; ++q) {
    const int4 b = sh.bond[q];
    const int side = bond_side(b);
    if (side == 3) {
      dg += hh.dg[q];
#pragma unroll
      for (int s = 0; s < MO; ++s) {
        const uint32_t tb = hh.tb[q][s];
        if (tb != kSpinNone) off(hh.v[q][s], tb + r);
      }
      continue;
    }
    if (side == 0 && lot) {
      const uint2 e = __ldg(lol);
      lol += t.n_lo;
      const int pr = b.x + (int)(e.x >> 26);
      dg += sh.dg[pr];
      const uint32_t r0 = e.x & kSpinLoNone;
      if (r0 != kSpinLoNone) off(sh.ov[pr * MO], base + r0);
      if (MO > 1 && e.y != kSpinLoNone) off(sh.ov[pr * MO + (MO > 1 ? 1 : 0)], base + e.y);
      continue;
    }
    const uint32_t wa = (b.y & 0x10000) ? h : lo, wc = (b.y & 0x20000) ? h : lo;
    const int a = (int)((wa >> (b.y & 255)) & dm), c = (int)((wc >> ((b.y >> 8) & 255)) & dm);
    const int pr = b.x + a * D + c;
    dg += sh.dg[pr];
    const uint32_t kp = sh.pk[pr];
#pragma unroll
    for (int s = 0; s < MO; ++s) {
      const int k = (int)(int8_t)(uint8_t)(kp >> (8 * s));
      if (k != 0) {
        const uint32_t th = b.z ? __ldg(t.thi + (h + (uint32_t)(k * b.z))) : base;
        const uint32_t tl = b.w ? __ldg(t.tlo + (lo + (uint32_t)(k * b.w))) : r;
        off(sh.ov[pr * MO + s], th + tl);
      }
    }
  }
  return dg;
}

// The lo table (SpinDev::lol): one thread per (lo-lo bond j, lo code u).
template <int D, int MO>
__global__ void spin_lo_table_kernel(const __grid_constant__ SpinParams p, const SpinDev t, uint2* __restrict__ out) {
  constexpr int BITS = D <= 2 ? 1 : D <= 4 ? 2 : 3;
  constexpr uint32_t dm = (1u << BITS) - 1u;
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= t.n_lo * t.n_ll) return;
  const int j = (int)(n / t.n_lo);
  const int64_t u = n - (int64_t)j * t.n_lo;
  const int N = t.N, Nh = N - t.Nl;
  int q = 0;
  for (int c = -1; q < p.n_bonds; ++q)
    if (p.s1[q] >= Nh && p.s2[q] >= Nh && ++c == j) break;
  const int wi = BITS * (N - 1 - p.s1[q]), wj = BITS * (N - 1 - p.s2[q]);
  const uint32_t lo = t.lolist[u];
  const int pr = (int)((lo >> wi) & dm) * D + (int)((lo >> wj) & dm);
  const uint32_t kp = p.pk[p.cls[q]][pr];
  const int bl = (1 << wi) - (1 << wj);
  uint32_t rk[2] = {kSpinLoNone, kSpinLoNone};
#pragma unroll
  for (int s = 0; s < MO && s < 2; ++s) {
    const int k = (int)(int8_t)(uint8_t)(kp >> (8 * s));
    if (k != 0) rk[s] = t.tlo[lo + (uint32_t)(k * bl)];
  }
  out[n] = make_uint2(rk[0] | ((uint32_t)pr << 26), rk[1]);
}

template <class Sh>
__global__ void __launch_bounds__(kSpinThreads) spin_hv_kernel(const __grid_constant__ SpinParams p, const SpinDev t,
                                                               const double* __restrict__ x, double* __restrict__ y,
                                                               double* __restrict__ alpha_part) {
  constexpr bool kTab = !std::is_same<Sh, SpinShared>::value;
  __shared__ Sh sh;
  __shared__ typename TileHiOf<Sh>::type hh;
  __shared__ double red[33];
  const int N = t.N, bits = t.bits;
  const bool has_site = __syncthreads_or(stage_spin(p, t, sh)) != 0;
  const uint32_t dm = (1u << bits) - 1u;
  for (int64_t it = blockIdx.x; it < t.n_tiles; it += gridDim.x) {
    const uint32_t b = t.tile_blk[it], r0 = t.tile_r[it];
    const uint32_t h = t.blk_hi[b], base = t.blk_off[b];
    int sum = 0;
    for (int i = 0; i < N - t.Nl; ++i) sum += (int)((h >> (bits * i)) & dm);
    const uint32_t lbase = t.looff[t.T - sum], rows = t.looff[t.T - sum + 1] - lbase;
    const uint32_t r1 = rows < r0 + kSpinTileRows ? rows : r0 + kSpinTileRows;
    double dot = 0.0;
    if constexpr (kTab) {
      tile_hi_entries(sh, hh, p.n_bonds, t, h);
      for (uint32_t r = r0 + threadIdx.x; r < r1; r += kSpinThreads) {
        const uint32_t lo = t.lolist[lbase + r];
        double off = 0.0;
        const double dg = spin_row_tile(sh, hh, p.n_bonds, has_site, t, h, lo, base, r, lbase + r,
                                        [&](double v, uint32_t rk) { off = fma(v, __ldg(x + rk), off); });
        const double xi = x[base + r];
        const double yi = fma(dg, xi, off);
        y[base + r] = yi;
        dot = fma(xi, yi, dot);
      }
    } else {
      for (uint32_t r = r0 + threadIdx.x; r < r1; r += kSpinThreads) {
        const uint32_t lo = t.lolist[lbase + r];
        const uint32_t row = base + r;
        double off = 0.0;
        const double dg = spin_row(sh, p.n_bonds, has_site, t, h, lo, base, r,
                                   [&](double v, uint32_t rk) { off = fma(v, __ldg(x + rk), off); });
        const double xi = x[row];
        const double yi = fma(dg, xi, off);
        y[row] = yi;
        dot = fma(xi, yi, dot);
      }
    }
    if (alpha_part) {
      const double tot = block_sum_all<kSpinThreads>(dot, red);
      if (threadIdx.x == 0) alpha_part[it] = tot;
    }
  }
}

// y = H x on a momentum sector of a spin-S model, interleaved complex: row i
// is representative r_i (ascending); its site terms and diagonal transitions
// multiply x_i, and an off-diagonal transition to s' adds
// v * phase_t * n_j / n_i * x_j with (j, t) the map entry of s'
// (hamiltonian_matrix.hpp:307-345 with the Bloch basis of
// blochbasisstates.h:92-271).  alpha_part: one partial of Re<x, y> per
// kMomTileRows rows.
// Five CTAs per SM (48 registers, no spill in the tabulated forms): the walk is
// bound by its dependent loads, and a fifth CTA hides more of them than the
// registers it takes away (0.366 against 0.452 ms on the spin-1 chain L=18).
template <class Sh>
__global__ void __launch_bounds__(kSpinThreads, 5) spin_mom_hv_kernel(const __grid_constant__ SpinParams p,
                                                                   const __grid_constant__ MomParams mp,
                                                                   const SpinDev t, const SpinMomTables m,
                                                                   const double2* __restrict__ x,
                                                                   double2* __restrict__ y,
                                                                   double* __restrict__ alpha_part) {
  __shared__ Sh sh;
  __shared__ double pre[kMaxTrans], pim[kMaxTrans];
  __shared__ double red[33];
  const int nz = stage_spin(p, t, sh);
  for (int q = threadIdx.x; q < mp.n_trans; q += kSpinThreads) {
    pre[q] = mp.phase_re[q];
    pim[q] = mp.phase_im[q];
  }
  const bool has_site = __syncthreads_or(nz) != 0;
  const int shift = t.bits * t.Nl;
  const uint64_t lm = (1ull << shift) - 1ull;
  const uint32_t jmask = (1u << kMomRepBits) - 1u;
  const int64_t ntile = mom_tiles(m.dim);
  for (int64_t tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    double dot = 0.0;
    for (int u = 0; u < kMomTileRows / kSpinThreads; ++u) {
      const int64_t i = tile * kMomTileRows + u * kSpinThreads + threadIdx.x;
      if (i >= m.dim) break;
      const uint64_t r = m.reps[i];
      const uint32_t rh = (uint32_t)(r >> shift), rl = (uint32_t)(r & lm);
      const double ni = m.norm[i];
      double are = 0.0, aim = 0.0;
      const double dg = spin_row(sh, p.n_bonds, has_site, t, rh, rl, __ldg(t.thi + rh), __ldg(t.tlo + rl),
                                 [&](double v, uint32_t rk) {
        const uint32_t e = __ldg(m.map + rk);
        if (e == kMomNone) return;
        const uint32_t j = e & jmask, tt = e >> kMomRepBits;
        const double f = v * (__ldg(m.norm + j) / ni);
        const double cr = f * pre[tt], ci = f * pim[tt];
        const double2 xj = x[j];
        are = fma(cr, xj.x, fma(-ci, xj.y, are));
        aim = fma(cr, xj.y, fma(ci, xj.x, aim));
      });
      const double2 xi = x[i];
      are = fma(dg, xi.x, are);
      aim = fma(dg, xi.y, aim);
      y[i] = make_double2(are, aim);
      dot = fma(xi.x, are, fma(xi.y, aim, dot));
    }
    if (alpha_part) {
      const double tot = block_sum_all<kSpinThreads>(dot, red);
      if (threadIdx.x == 0) alpha_part[tile] = tot;
    }
  }
}

// Expectation values in one vector of the sector (the spin-S counterpart of
// measure.cu's meas_kernel): per site pair p,
//   kind SZ     sum_s psi_s^2 m_i(s)
//   kind SZSZ   sum_s psi_s^2 m_i(s) m_j(s)
//   kind SPSM   sum_s psi_{s'} psi_s <a+1|S+|a> <c-1|S-|c>, s' = s with digit a of
//               site i raised and digit c of site j lowered (i = j: the diagonal
//               S+ S- = S(S+1) - m^2 + m)
// with S+- the site operators of models.xml.in:24-36.  Rows are walked by the
// apply's work tiles; each CTA writes one partial sum per pair, which the host
// adds in order.
struct SpinMeasArgs {
  int np;
  int wi[kMeasPairs], wj[kMeasPairs];  // bit offsets of the digits of sites i and j
  double m[kSpinMaxDim];               // Sz of each digit
  double cp[kSpinMaxDim];              // <v+1|S+|v>
  double cm[kSpinMaxDim];              // <v-1|S-|v>
};

constexpr int kSpinMeasThreads = 256;

template <int KIND>
__global__ void __launch_bounds__(kSpinMeasThreads, 1)
    spin_meas_kernel(const SpinDev t, const double* __restrict__ psi, const __grid_constant__ SpinMeasArgs a,
                     double* __restrict__ part) {
  __shared__ double red[33];
  double acc[kMeasPairs];
#pragma unroll
  for (int p = 0; p < kMeasPairs; ++p) acc[p] = 0.0;
  const int N = t.N, bits = t.bits, d = t.d;
  const int shift = bits * t.Nl;
  const uint64_t lm = (1ull << shift) - 1ull;
  const uint32_t dm = (1u << bits) - 1u;
  for (int64_t it = blockIdx.x; it < t.n_tiles; it += gridDim.x) {
    const uint32_t b = t.tile_blk[it], r0 = t.tile_r[it];
    const uint32_t h = t.blk_hi[b], base = t.blk_off[b];
    int sum = 0;
    for (int i = 0; i < N - t.Nl; ++i) sum += (int)((h >> (bits * i)) & dm);
    const uint32_t lbase = t.looff[t.T - sum], rows = t.looff[t.T - sum + 1] - lbase;
    const uint32_t r1 = rows < r0 + kSpinTileRows ? rows : r0 + kSpinTileRows;
    for (uint32_t r = r0 + threadIdx.x; r < r1; r += kSpinMeasThreads) {
      const uint64_t s = ((uint64_t)h << shift) | t.lolist[lbase + r];
      const double v = psi[base + r];
#pragma unroll
      for (int p = 0; p < kMeasPairs; ++p) {
        if (p >= a.np) continue;  // (no break: the accumulators stay in registers)
        const int wi = a.wi[p];
        const int da = (int)((s >> wi) & dm);
        if (KIND == kMeasSz) {
          acc[p] = fma(v * v, a.m[da], acc[p]);
        } else if (KIND == kMeasSzSz) {
          const int dc = (int)((s >> a.wj[p]) & dm);
          acc[p] = fma(v * v, a.m[da] * a.m[dc], acc[p]);
        } else {
          const int wj = a.wj[p];
          if (wi == wj) {
            acc[p] = fma(v * v, a.cm[da] * a.cm[da], acc[p]);
          } else {
            const int dc = (int)((s >> wj) & dm);
            if (da + 1 < d && dc > 0) {  // s' is a state of the same digit sum: its rank exists
              const uint64_t s2 = s + (1ull << wi) - (1ull << wj);
              const uint32_t rk = __ldg(t.thi + (uint32_t)(s2 >> shift)) + __ldg(t.tlo + (uint32_t)(s2 & lm));
              acc[p] = fma(__ldg(psi + rk) * v, a.cp[da] * a.cm[dc], acc[p]);
            }
          }
        }
      }
    }
  }
#pragma unroll
  for (int p = 0; p < kMeasPairs; ++p) {
    if (p >= a.np) continue;
    const double tot = block_sum_all<kSpinMeasThreads>(acc[p], red);
    if (threadIdx.x == 0) part[(size_t)blockIdx.x * kMeasPairs + p] = tot;
  }
}

// <psi| sum_p O(i_p, j_p) |psi> in a spin-S momentum sector for site pairs
// whose sum is translation invariant (mom_expect_kernel's rule with digits):
// diagonal parts on the representative, S+_i S-_j through the map with the
// phase and n_j / n_i of a Hamiltonian transition.
struct SpinMomPairs {
  int n;
  int wi[kMomPairs], wj[kMomPairs];  // bit offsets of the digits of sites i and j
  double m[kSpinMaxDim], cp[kSpinMaxDim], cm[kSpinMaxDim];
};

template <int KIND>
__global__ void __launch_bounds__(kSpinThreads) spin_mom_expect_kernel(const __grid_constant__ MomParams mp,
                                                                       const SpinDev t, const SpinMomTables m,
                                                                       const double2* __restrict__ psi,
                                                                       const __grid_constant__ SpinMomPairs a,
                                                                       double* __restrict__ part) {
  __shared__ double pre[kMaxTrans], pim[kMaxTrans];
  __shared__ double red[33];
  for (int q = threadIdx.x; q < mp.n_trans; q += kSpinThreads) {
    pre[q] = mp.phase_re[q];
    pim[q] = mp.phase_im[q];
  }
  __syncthreads();
  const int shift = t.bits * t.Nl, d = t.d;
  const uint64_t lm = (1ull << shift) - 1ull;
  const uint32_t dm = (1u << t.bits) - 1u;
  const uint32_t jmask = (1u << kMomRepBits) - 1u;
  double acc = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)kSpinThreads + threadIdx.x; i < m.dim;
       i += (int64_t)gridDim.x * kSpinThreads) {
    const uint64_t r = m.reps[i];
    const double2 pi = psi[i];
    const double w = pi.x * pi.x + pi.y * pi.y;
    double dsum = 0.0;  // diagonal part of the pair sum on r
    double ore = 0.0;   // Re conj(psi_i) (off-diagonal part applied to psi)_i
    for (int p = 0; p < a.n; ++p) {
      const int wi = a.wi[p];
      const int da = (int)((r >> wi) & dm);
      if (KIND == kMeasSz) {
        dsum += a.m[da];
      } else if (KIND == kMeasSzSz) {
        dsum += a.m[da] * a.m[(int)((r >> a.wj[p]) & dm)];
      } else if (wi == a.wj[p]) {
        dsum += a.cm[da] * a.cm[da];
      } else {
        const int wj = a.wj[p];
        const int dc = (int)((r >> wj) & dm);
        if (da + 1 >= d || dc == 0) continue;
        const uint64_t s2 = r + (1ull << wi) - (1ull << wj);
        const uint32_t e =
            __ldg(m.map + __ldg(t.thi + (uint32_t)(s2 >> shift)) + __ldg(t.tlo + (uint32_t)(s2 & lm)));
        if (e == kMomNone) continue;
        const uint32_t j = e & jmask, tt = e >> kMomRepBits;
        const double f = a.cp[da] * a.cm[dc] * (__ldg(m.norm + j) / m.norm[i]);
        const double cr = f * pre[tt], ci = f * pim[tt];
        const double2 xj = psi[j];
        const double yr = cr * xj.x - ci * xj.y, yi = cr * xj.y + ci * xj.x;
        ore += pi.x * yr + pi.y * yi;
      }
    }
    acc += w * dsum + ore;
  }
  const double tot = block_sum_all<kSpinThreads>(acc, red);
  if (threadIdx.x == 0) part[blockIdx.x] = tot;
}

// Sz, <v+1|S+|v> and <v-1|S-|v> of every digit v of spin S = (d - 1) / 2.
void spin_factors(int d, double* m, double* cp, double* cm) {
  const double S = d / 2.0 - 0.5;
  for (int v = 0; v < d; ++v) {
    const double mv = v - S;
    m[v] = mv;
    cp[v] = v + 1 < d ? std::sqrt(S * (S + 1) - mv * (mv + 1)) : 0.0;
    cm[v] = v > 0 ? std::sqrt(S * (S + 1) - mv * (mv - 1)) : 0.0;
  }
}

int sm_count() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

}  // namespace

int spin_measure_pairs(aed_handle* h, const double* psi, int kind, int n, const int32_t* si, const int32_t* sj,
                       double* out) {
  const SpinDev& t = h->sdev;
  if (t.n_tiles == 0) {
    for (int p = 0; p < n; ++p) out[p] = 0.0;
    return AED_OK;
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = (int)std::min<int64_t>(t.n_tiles, (int64_t)sms * 4);
  void* w = nullptr;
  int rc = handle_workspace(h, 1, (size_t)grid * kMeasPairs * 8, &w);
  if (rc) return rc;
  double* part = static_cast<double*>(w);
  std::vector<double> hp((size_t)grid * kMeasPairs);
  SpinMeasArgs a{};
  spin_factors(t.d, a.m, a.cp, a.cm);
  for (int p0 = 0; p0 < n; p0 += kMeasPairs) {
    a.np = std::min(kMeasPairs, n - p0);
    for (int p = 0; p < a.np; ++p) {
      a.wi[p] = t.bits * (t.N - 1 - si[p0 + p]);
      a.wj[p] = kind == kMeasSz ? 0 : t.bits * (t.N - 1 - sj[p0 + p]);
    }
    switch (kind) {
      case kMeasSz: spin_meas_kernel<kMeasSz><<<grid, kSpinMeasThreads, 0, h->stream>>>(t, psi, a, part); break;
      case kMeasSzSz: spin_meas_kernel<kMeasSzSz><<<grid, kSpinMeasThreads, 0, h->stream>>>(t, psi, a, part); break;
      default: spin_meas_kernel<kMeasSpSm><<<grid, kSpinMeasThreads, 0, h->stream>>>(t, psi, a, part); break;
    }
    if ((rc = check_launch_counted("spin_meas_kernel"))) return rc;
    AED_CUDA_TRY(cudaMemcpyAsync(hp.data(), part, hp.size() * 8, cudaMemcpyDeviceToHost, h->stream));
    AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (int p = 0; p < a.np; ++p) {
      double sum = 0.0;
      for (int b = 0; b < grid; ++b) sum += hp[(size_t)b * kMeasPairs + p];
      out[p0 + p] = sum;
    }
  }
  return AED_OK;
}

int spin_mom_expectation(aed_handle* h, const double* psi, int kind, int n, const int32_t* si, const int32_t* sj,
                         double* out) {
  *out = 0.0;
  if (n <= 0 || h->dim == 0) return AED_OK;
  const SpinDev& t = h->sdev;
  const SpinMomTables m = h->spin_mom_tables();
  const int grid = mom_expect_grid(h->dim);
  void* w = nullptr;
  int rc = handle_workspace(h, 1, (size_t)grid * 8, &w);
  if (rc) return rc;
  double* part = static_cast<double*>(w);
  std::vector<double> hp((size_t)grid);
  SpinMomPairs a{};
  spin_factors(t.d, a.m, a.cp, a.cm);
  const double2* p2 = reinterpret_cast<const double2*>(psi);
  double total = 0.0;
  for (int p0 = 0; p0 < n; p0 += kMomPairs) {
    a.n = std::min(kMomPairs, n - p0);
    for (int p = 0; p < a.n; ++p) {
      a.wi[p] = t.bits * (t.N - 1 - si[p0 + p]);
      a.wj[p] = kind == kMeasSz ? 0 : t.bits * (t.N - 1 - sj[p0 + p]);
    }
    switch (kind) {
      case kMeasSz:
        spin_mom_expect_kernel<kMeasSz><<<grid, kSpinThreads, 0, h->stream>>>(*h->mp, t, m, p2, a, part);
        break;
      case kMeasSzSz:
        spin_mom_expect_kernel<kMeasSzSz><<<grid, kSpinThreads, 0, h->stream>>>(*h->mp, t, m, p2, a, part);
        break;
      default:
        spin_mom_expect_kernel<kMeasSpSm><<<grid, kSpinThreads, 0, h->stream>>>(*h->mp, t, m, p2, a, part);
        break;
    }
    if ((rc = check_launch_counted("spin_mom_expect_kernel"))) return rc;
    AED_CUDA_TRY(cudaMemcpyAsync(hp.data(), part, hp.size() * 8, cudaMemcpyDeviceToHost, h->stream));
    AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (double v : hp) total += v;
  }
  *out = total;
  return AED_OK;
}

template <class T>
struct Form {
  using type = T;
};

// Calls f(Form<shared layout>) with the layout of the apply for p: the
// tabulated form with D = d digits and enough off-diagonal slots, or the
// per-bond form when the couplings have more than kSpinMaxCls classes.
template <class F>
void with_spin_form(const SpinParams& p, const SpinDev& t, F&& f) {
  if (p.n_cls == 0) return f(Form<SpinShared>{});
  switch (t.d) {
    case 2:
      return f(Form<SpinTabShared<2, 1>>{});
    case 3:
      return f(Form<SpinTabShared<3, 2>>{});
    case 4:
      return p.pmo <= 2 ? f(Form<SpinTabShared<4, 2>>{}) : f(Form<SpinTabShared<4, 3>>{});
    default:
      return p.pmo <= 2 ? f(Form<SpinTabShared<5, 2>>{}) : f(Form<SpinTabShared<5, 4>>{});
  }
}

int launch_spin_mom_hv(const SpinParams& p, const MomParams& mp, const SpinDev& t, const SpinMomTables& m,
                       const double* x, double* y, double* alpha_part, cudaStream_t st) {
  if (m.dim == 0) return AED_OK;
  const int64_t tiles = mom_tiles(m.dim), cap = (int64_t)sm_count() * 8;
  const int grid = (int)(tiles < cap ? tiles : cap);
  const double2* xc = reinterpret_cast<const double2*>(x);
  double2* yc = reinterpret_cast<double2*>(y);
  with_spin_form(p, t, [&](auto form) {
    spin_mom_hv_kernel<typename decltype(form)::type><<<grid, kSpinThreads, 0, st>>>(p, mp, t, m, xc, yc, alpha_part);
  });
  return check_launch_counted("spin_mom_hv_kernel");
}

size_t spin_lo_table_bytes(const SpinParams& p, SpinDev& t) {
  const int Nh = t.N - t.Nl;
  t.n_ll = 0;
  for (int q = 0; q < p.n_bonds; ++q) t.n_ll += p.s1[q] >= Nh && p.s2[q] >= Nh;
  // the forms with at most two off-diagonal slots (tile row walk, MO <= 2)
  const bool two = p.n_cls > 0 && (t.d <= 3 || p.pmo <= 2);
  return two && t.n_ll > 0 && t.n_lo > 0 ? (size_t)t.n_lo * t.n_ll * sizeof(uint2) : 0;
}

int launch_spin_lo_table(const SpinParams& p, const SpinDev& t, uint2* dst, cudaStream_t st) {
  const int64_t n = t.n_lo * t.n_ll;
  if (n == 0) return AED_OK;
  const unsigned grid = (unsigned)((n + 255) / 256);
  switch (t.d) {
    case 2:
      spin_lo_table_kernel<2, 1><<<grid, 256, 0, st>>>(p, t, dst);
      break;
    case 3:
      spin_lo_table_kernel<3, 2><<<grid, 256, 0, st>>>(p, t, dst);
      break;
    case 4:
      spin_lo_table_kernel<4, 2><<<grid, 256, 0, st>>>(p, t, dst);
      break;
    default:
      spin_lo_table_kernel<5, 2><<<grid, 256, 0, st>>>(p, t, dst);
      break;
  }
  return check_launch_counted("spin_lo_table_kernel");
}

int launch_spin_basis(const SpinDev& t, uint64_t* out, int64_t offset, int64_t count, cudaStream_t st) {
  if (count <= 0) return AED_OK;
  spin_basis_kernel<<<(unsigned)((count + 255) / 256), 256, 0, st>>>(t, out, offset, count);
  return check_launch_counted("spin_basis_kernel");
}

int launch_spin_hv(const SpinParams& p, const SpinDev& t, const double* x, double* y, double* alpha_part,
                   cudaStream_t st) {
  if (t.n_tiles == 0) return AED_OK;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t cap = (int64_t)sms * 8;
  const int grid = (int)(t.n_tiles < cap ? t.n_tiles : cap);
  with_spin_form(p, t, [&](auto form) {
    spin_hv_kernel<typename decltype(form)::type><<<grid, kSpinThreads, 0, st>>>(p, t, x, y, alpha_part);
  });
  return check_launch_counted("spin_hv_kernel");
}

}  // namespace aed
