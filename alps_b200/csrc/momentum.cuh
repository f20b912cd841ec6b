// momentum.cuh -- momentum (Bloch) sectors: tables and launch wrappers.
//
// A momentum sector of an Sz sector has one row per representative: the
// smallest state of its translation orbit, kept when w = sqrt|sum of the
// phases of the translations that fix it| >= 0.01, with normalisation
// n = w / sqrt(N) (bloch_basis_states::build, src/alps/model/blochbasisstates.h:
// 92-271; the identity is the first translation and its phase 1 starts the
// sum).  Every state of the Sz sector maps to (its representative j, the first
// translation t in list order that takes it there), or to nothing when its
// orbit is not kept.  Row i of H is
//   y_i = M_d(r_i) x_i + sum over the flips s' of r_i:  c * phase_t * n_j / n_i * x_j
// with M_d the diagonal terms of r_i: hamiltonian_matrix.hpp:307-345 builds
// M(i,j) += val * phase * n_j / n_i for every image of representative i.
// Vectors are complex, interleaved (re, im) doubles: the Lanczos vector
// kernels run unchanged on 2 * dim doubles, and alpha = Re<v, H v>
// (ietl::real(ietl::dot), src/ietl/lanczos.h:385-398) is their real dot product.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.cuh"
#include "spin.cuh"

namespace aed {

constexpr int kMaxTrans = 62;              // translations per sector (6 bits in a map entry, 63 = none)
constexpr int kMomRepBits = 26;            // representative index bits of a map entry
constexpr uint32_t kMomNone = 0xffffffffu;  // map entry of a state whose orbit is not kept
constexpr int kMomTileRows = 1024;          // rows per <x, y> partial of the apply

struct MomParams {
  int N, n_trans, n_flip;
  double inv_sqrt_n;  // 1 / sqrt(N)
  double phase_re[kMaxTrans], phase_im[kMaxTrans];
  uint8_t dst[kMaxTrans][32];  // translation t moves the bit of site i to bit dst[t][i]
  uint32_t flip_mask[kMaxBonds];
  double flip_c[kMaxBonds];  // 0.5 Jxy - 0.25 K of each bond with a nonzero flip term, in bond order
};

struct MomTables {
  const uint32_t* reps;  // dim representative states, ascending
  const double* norm;    // dim normalisations
  const double* diag;    // dim diagonal terms of the representatives
  const uint32_t* map;   // D entries: (t << kMomRepBits) | j, or kMomNone
  int64_t dim;
};

// Build the sector's tables on the device: reps / norm / diag (dim entries)
// and map (D entries) are allocated with mem_dev_alloc and owned by the
// caller.  HvParams supplies the diagonal terms (site terms, then bonds).
int mom_build(const MomParams& mp, const HvParams& P, const DevTables& t, cudaStream_t st, uint32_t** reps,
              double** norm, double** diag, uint32_t** map, int64_t* dim);
// Recompute the diagonal terms of the representatives (new couplings).
int launch_mom_diag(const HvParams& P, const uint32_t* reps, int64_t dim, double* diag, cudaStream_t st);
// y = H x on interleaved complex vectors; alpha_part (optional): one partial
// of Re<x, y> per kMomTileRows rows.
int launch_mom_hv(const MomParams& mp, const DevTables& t, const MomTables& m, const double* x, double* y,
                  double* alpha_part, cudaStream_t st);
__host__ __device__ inline int64_t mom_tiles(int64_t dim) { return (dim + kMomTileRows - 1) / kMomTileRows; }

// <psi| sum_p O(i_p, j_p) |psi> in a momentum sector for a list of site pairs
// whose sum is translation invariant (a distance class): kind AED_OBS_SZ
// (sum of Sz_i), AED_OBS_SZSZ, AED_OBS_SPSM (S+_i S-_j; i = j: the projector
// on spin up).  Diagonal terms are read on the representative; S+_i S-_j maps
// a representative with site j up and site i down to its image's orbit with
// the same phase and normalisation factor as a Hamiltonian flip.
constexpr int kMomPairs = 64;
struct MomPairs {
  int n;
  uint32_t mi[kMomPairs], mj[kMomPairs];
};
int mom_expectation(const MomParams& mp, const DevTables& t, const MomTables& m, const double* psi, int kind,
                    const MomPairs& pairs, double* part, int grid, cudaStream_t st);
int mom_expect_grid(int64_t dim);

// Momentum sectors of spin-S models (aed_create_spin_momentum): the same
// Bloch basis over the spin-S sector's states (64-bit packed digits,
// spin.cuh).  The apply forms each representative's diagonal itself, so
// there is no diagonal array.
struct SpinMomTables {
  const uint64_t* reps;  // dim representative states, ascending
  const double* norm;    // dim normalisations
  const uint32_t* map;   // D entries: (t << kMomRepBits) | j, or kMomNone
  int64_t dim;
};
int spin_mom_build(const MomParams& mp, const SpinDev& t, cudaStream_t st, uint64_t** reps, double** norm,
                   uint32_t** map, int64_t* dim);
// y = H x on interleaved complex vectors (spin.cu); alpha_part as launch_mom_hv.
int launch_spin_mom_hv(const SpinParams& p, const MomParams& mp, const SpinDev& t, const SpinMomTables& m,
                       const double* x, double* y, double* alpha_part, cudaStream_t st);

}  // namespace aed
