// kernels.cuh -- launch wrappers of the engine's sm_100a kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "aed_internal.h"

namespace aed {

// Device-resident basis tables of one sector.
struct DevTables {
  const uint32_t* thi;     // 2^Nhi
  const uint16_t* tlo;     // 2^Nlo
  const uint16_t* lolist;  // 2^Nlo
  const uint32_t* looff;   // Nlo+2
  const uint32_t* tile_h;  // n_tiles
  const uint32_t* tile_r;  // n_tiles
  const double* dg;        // D: diagonal M(i,i) of every row
  const uint32_t* ell;     // lo-neighbour table (build_lo_table), ell_w entries per lo state
  const uint16_t* xtab = nullptr;  // crossing-flip table (build_cross_table), Nlo x 2^Nlo
  int ell_w;
  int64_t n_tiles;
  int64_t D;
  int Nlo, Nhi, n_up;
  // block list of the bundle apply (build_block_list): hi blocks grouped by
  // lo popcount, each group padded with kNoBlock to a multiple of kBundleMax
  const uint32_t* blk_h = nullptr;   // n_blk
  const uint32_t* tfirst = nullptr;  // 2^Nhi: index of the first tile of each hi block
  int64_t n_blk = 0;
  int maxrows = 0;  // rows of the largest hi block
  // raised by a kernel whose bounded wait gave up (read and cleared by the host)
  uint32_t* flag = nullptr;
  // FP32 handles: M(i,i) rounded to FP32 (D floats), read by the FP32 applies
  // in place of dg (half its bytes; the FP64 applies keep dg)
  const float* dgf = nullptr;
};

constexpr int kHvThreads = 256;
constexpr int kHvTileRows = 2048;  // rows per work tile (a multiple of kHvThreads x rows per thread)
constexpr int kRedThreads = 256;

// y = H x with apply variant `variant` (0 .. hv_num_variants()-1).  A
// variant that does not fit the sector (shared memory) returns
// kVariantNotApplicable without launching.
// alpha_part (optional): one partial sum of x_i * y_i per tile (n_tiles entries).
int launch_hv_f64(int variant, const HvParams& P, const DevTables& t, const double* x, double* y,
                  double* alpha_part, cudaStream_t st);
int launch_hv_f32(int variant, const HvParams& P, const DevTables& t, const float* x, float* y,
                  double* alpha_part, cudaStream_t st);
constexpr int kVariantNotApplicable = 2;
int hv_num_variants();
const char* hv_variant_name(int v);
// Whether the autotuner times variant v (the stream applies are left out).
bool hv_variant_tuned(int v);

// per-row diagonal table (once per handle)
int launch_diag_table(const HvParams& P, const DevTables& t, double* dg, cudaStream_t st);

// basis / rank
int launch_basis_copy(const DevTables& t, uint32_t* out, int64_t offset, int64_t count, cudaStream_t st);
int launch_rank(const DevTables& t, int N, const uint32_t* states, int64_t count, int64_t* out, cudaStream_t st);

// vector kernels (T = double or float)
template <typename T>
int launch_fill_random(T* x, int64_t n, uint64_t seed, cudaStream_t st);
template <typename T>
int launch_copy(const T* x, T* y, int64_t n, cudaStream_t st);
int launch_round_to_f32(const double* x, float* y, int64_t n, cudaStream_t st);
template <typename T>
int launch_axpy(double a, const T* x, T* y, int64_t n, cudaStream_t st);
template <typename T>
int launch_scal(double a, T* x, int64_t n, bool divide, cudaStream_t st);

// Deterministic reductions: one partial per fixed chunk of kRedChunk elements
// (red_chunks(n) of them), then one fixed-order sum.  sq: sum of squares of x.
constexpr int64_t kRedChunk = 4096;
int64_t red_chunks(int64_t n);
template <typename T>
int launch_dot_partials(const T* x, const T* y, int64_t n, double* part, bool sq, cudaStream_t st);
int launch_finish_sum(const double* part, int64_t n, double* out, bool take_sqrt, cudaStream_t st);

// Fused Lanczos step (make_step, src/ietl/lanczos.h:392-406), after the apply
// x -> y with per-tile partials and launch_finish_sum(partials -> *alpha):
//   update:    y = (y - alpha x) - beta_prev v_prev; chunk partials of |y|^2
//   (launch_finish_sum(partB -> *beta, sqrt))
//   normalize: y /= beta
// alpha, beta, beta_prev are device scalars (vprev == NULL: first step).
template <typename T>
int launch_lanczos_update(const double* alpha, const T* x, const T* vprev, const double* beta_prev, T* y,
                          int64_t n, double* partB, cudaStream_t st);
template <typename T>
int launch_lanczos_normalize(const double* beta, T* y, int64_t n, cudaStream_t st);
// The same two kernels with the finishing sums of alpha (the apply's tile
// partials) and beta (the update's chunk partials) done inside every CTA, in
// finish_sum's order: the same alpha and beta to the bit and two launches
// fewer per step; for short partial lists (kFoldFinishMax).
constexpr int64_t kFoldFinishMax = 2048;
template <typename T>
int launch_lanczos_update_fin(const double* alpha_part, int64_t n_apart, double* alpha, const T* x, const T* vprev,
                              const double* beta_prev, T* y, int64_t n, double* partB, cudaStream_t st);
template <typename T>
int launch_lanczos_normalize_fin(const double* beta_part, int64_t n_bpart, double* beta, T* y, int64_t n,
                                 cudaStream_t st);

// out[i] = sum_j coef[j] * V[j*ld + i] (FP32 Lanczos store -> FP64 vector),
// coef in device memory (m <= kMaxRitzTerms).
constexpr int kMaxRitzTerms = 4096;
int launch_ritz_combine(const float* V, int64_t ld, int m, const double* coef, double* out, int64_t n,
                        bool accumulate, cudaStream_t st);

// ---- Rayleigh-Ritz refinement of the mixed path (refine.cu) ----
constexpr int kMaxRR = 8;     // Ritz vectors in one refinement
constexpr int kMaxComb = 16;  // vectors of one chunk of the FP32 basis store
struct VecSet {
  double* p[kMaxRR];
};
struct ResidCoef {
  double cw[kMaxRR][kMaxRR], cx[kMaxRR][kMaxRR];
};
// The FP32 basis store: chunk c holds v_{kMaxComb c} .. v_{kMaxComb c + kMaxComb - 1}, ld apart.
// out.p[k][i] = sum_{j < m} coef[k * m + j] v_j[i] for k < K: one pass over the m stored vectors
// (kCombChunks chunks per launch, the K sums held in registers throughout), FP64 sums in ascending j.
constexpr int kCombChunks = 32;
int launch_ritz_combine_chunks(const float* const* chunks, int64_t ld, int m, const double* coef, int K,
                               const VecSet& out, int64_t n, cudaStream_t st);
// out = [<X_a, X_b> for a <= b (row-major upper triangle), <X_a, Y_b> for all a, b];
// part: (K(K+1)/2 + K^2) * red_chunks(n) doubles of scratch.
int launch_gram(const VecSet& X, const VecSet& Y, int K, int64_t n, double* part, double* out, cudaStream_t st);
// out[r] = |sum_k cw[r][k] Y_k + cx[r][k] X_k|^2 for r < R; part: R * red_chunks(n) doubles.
int launch_resid(const VecSet& X, const VecSet& Y, const ResidCoef& rc, int K, int R, int64_t n, double* part,
                 double* out, cudaStream_t st);

// Full reorthogonalisation of the mixed path (refine.cu): chunk partials of
// <V_k, w> for the m <= kMaxComb vectors of one store chunk into
// part[(k0 + k) * red_chunks(n) + c]; the sums of np such rows; w -= t with
// one rounding to FP32.
int launch_block_dot(const float* V, int64_t ld, int m, const float* w, int64_t n, double* part, int k0,
                     cudaStream_t st);
int launch_finish_many(const double* part, int64_t nch, int np, double* out, cudaStream_t st);
int launch_sub_round(const double* t, float* w, int64_t n, cudaStream_t st);

int64_t launch_count();
// After a launch in another translation unit: counts it and returns
// AED_ERR_CUDA (with the launch error) if it failed.
int check_launch_counted(const char* what);

}  // namespace aed
