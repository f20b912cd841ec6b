// spin.cuh -- Sz sectors of spin-S models with S >= 1/2: tables and launch wrappers.
//
// Site i holds digit v_i = m_i + S in [0, 2S] (the index of its state in the
// spin site basis, Sz ascending; lib/xml/models.xml.in:24-36), stored in
// `bits` bits with site 0 most significant, so that integer order of the
// packed states is the basis order of basis_states::build (odometer, last
// site fastest; src/alps/model/basisstates.h:175-278).  The sector is the set
// of states with digit sum T = Sz_total + N S.  Ranks use two tables: the
// packed state splits into a hi part (the first Nh sites) and a lo part (the
// last Nl); rank = thi[hi] + tlo[lo], tlo[lo] the rank of lo among lo codes
// of the same digit sum, thi[hi] the number of sector states with a smaller
// hi code.  The sector's states come in blocks of one hi code each.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "kernels.cuh"

namespace aed {

constexpr int kSpinMaxSites = 32;
constexpr int kSpinMaxDim = 5;                     // 2S + 1 <= 5 (S <= 2)
constexpr int kSpinMaxPairs = kSpinMaxDim * kSpinMaxDim;
constexpr int kSpinMaxTrans = kSpinMaxPairs * kSpinMaxDim;
constexpr int kSpinTileRows = 1024;                // rows per <x, y> partial of the apply

// Host tables of one sector.
struct SpinTables {
  int N = 0, twoS = 0, d = 0, bits = 0, Nh = 0, Nl = 0, T = 0;
  int64_t D = 0;
  std::vector<uint32_t> thi;      // 2^(bits Nh): states before hi code h (kSpinNone: not a digit string)
  std::vector<uint32_t> tlo;      // 2^(bits Nl): rank of lo among lo codes of its digit sum
  std::vector<uint32_t> lolist;   // valid lo codes grouped by digit sum, ascending
  std::vector<uint32_t> looff;    // offsets into lolist per digit sum (max sum + 2 entries)
  std::vector<uint32_t> blk_hi;   // hi code of every block (ascending = basis order)
  std::vector<uint32_t> blk_off;  // first row of every block
  std::vector<uint32_t> tile_blk, tile_r;  // work tiles: (block, first row within it)
};
constexpr uint32_t kSpinNone = 0xffffffffu;
int build_spin_tables(int N, int twoS, int T, SpinTables& t);

struct SpinDev {
  const uint32_t *thi, *tlo, *lolist, *looff, *blk_hi, *blk_off, *tile_blk, *tile_r;
  int64_t D, n_blk, n_tiles;
  int N, bits, Nl, d, T;
  // the lo table of the tabulated form (nullptr: none): per bond with both
  // sites in lo (the j-th such bond, in bond order) and per lo code u (its
  // index in lolist), entry [j n_lo + u] = (r0 | pr << 26, r1): the digit
  // pair pr = a d + c and the ranks within the block (tlo of the target lo
  // code) of the pair's off-diagonal slots 0 and 1, kSpinLoNone where empty
  const uint2* lol;
  int64_t n_lo;
  int n_ll;
};
constexpr uint32_t kSpinLoNone = (1u << 26) - 1u;

// One transition of a bond's pair of digits (a, c) -> (a2, c2) with the
// element Jz * A + Jxy * B + K * C (A: Sz Sz, B: exchange_xy, C: biquadratic).
struct SpinTrans {
  uint8_t a2, c2;
  double A, B, C;
};

constexpr int kSpinMaxCls = 8;  // coupling classes whose elements are tabulated
constexpr int kSpinMaxOff = kSpinMaxDim - 1;  // off-diagonal transitions of one digit pair (they keep a + c)

struct SpinParams {
  int N, n_bonds, twoS;
  double site_h[kSpinMaxSites], site_d[kSpinMaxSites];
  int s1[kMaxBonds], s2[kMaxBonds];
  double jz[kMaxBonds], jxy[kMaxBonds], kq[kMaxBonds];
  int tstart[kSpinMaxPairs + 1];  // transitions of pair (a, c) = a d + c: [tstart[p], tstart[p+1])
  SpinTrans trans[kSpinMaxTrans];
  // bonds with the same (Jz, Jxy, K) share a class; with at most kSpinMaxCls
  // classes the elements Jz A + Jxy B + K C are tabulated per class and digit
  // pair (a, c) = a d + c (n_cls = 0: formed per bond in the kernel): pdg the
  // diagonal element, pov the off-diagonal elements that are nonzero (zero
  // elements are skipped, hamiltonian_matrix.hpp:316) in target order (a2, c2),
  // each with k = a2 - a = c - c2 in one signed byte of pk (byte s for pov[s],
  // 0 past the last); pmo the most off-diagonal elements of any class and pair
  int n_cls;
  int cls[kMaxBonds];
  int pmo;
  double pdg[kSpinMaxCls][kSpinMaxPairs];
  double pov[kSpinMaxCls][kSpinMaxPairs][kSpinMaxOff];
  uint32_t pk[kSpinMaxCls][kSpinMaxPairs];
  double sdiag[kSpinMaxSites][kSpinMaxDim];  // -h m + D m^2 of every site and digit
};
// The local operators of the spin model (models.xml.in:24-36, 282-300): the
// transitions of Sz Sz, exchange_xy and biquadratic for spin S = twoS / 2.
void spin_transitions(int twoS, SpinParams& p);
// Bonds, site terms, coupling classes and their tabulated elements (after
// spin_transitions).
void spin_set_couplings(const std::vector<int>& s1, const std::vector<int>& s2, const std::vector<double>& jz,
                        const std::vector<double>& jxy, const std::vector<double>& kq,
                        const std::vector<double>& site_h, const std::vector<double>& site_d, int N, SpinParams& p);

int launch_spin_basis(const SpinDev& t, uint64_t* out, int64_t offset, int64_t count, cudaStream_t st);
int launch_spin_hv(const SpinParams& p, const SpinDev& t, const double* x, double* y, double* alpha_part,
                   cudaStream_t st);
// Bytes of the lo table for p and t (0: the apply's form uses none), and its
// fill (the table at dst, t.n_lo set); t.n_ll is set by the first call.
size_t spin_lo_table_bytes(const SpinParams& p, SpinDev& t);
int launch_spin_lo_table(const SpinParams& p, const SpinDev& t, uint2* dst, cudaStream_t st);
__host__ __device__ inline int64_t spin_tiles_of(const SpinDev& t) { return t.n_tiles; }

}  // namespace aed
