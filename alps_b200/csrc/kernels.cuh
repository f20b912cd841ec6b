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
  int64_t n_tiles;
  int64_t D;
  int Nlo, Nhi, n_up;
};

constexpr int kHvThreads = 256;
constexpr int kHvTileRows = 1024;  // rows per work tile (kHvThreads x rows per thread)
constexpr int kRedThreads = 256;

// y = H x.  alpha_part (optional): per-CTA partial sums of x_i * y_i.
// grid = number of CTAs (fixed per handle so partial sums are deterministic).
int launch_hv_f64(const HvParams& P, const DevTables& t, const double* x, double* y, double* alpha_part,
                  int grid, cudaStream_t st);
int launch_hv_f32(const HvParams& P, const DevTables& t, const float* x, float* y, double* alpha_part,
                  int grid, cudaStream_t st);
int hv_grid_size(bool f32, int rows_per_thread_unused);

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
template <typename T>
int launch_axpy(double a, const T* x, T* y, int64_t n, cudaStream_t st);
template <typename T>
int launch_scal(double a, T* x, int64_t n, bool divide, cudaStream_t st);

// deterministic reductions: partials over a fixed grid, then one fixed-order
// final sum into *out (device).  sq: sum of squares of x (y ignored).
template <typename T>
int launch_dot_partials(const T* x, const T* y, int64_t n, double* part, int grid, bool sq, cudaStream_t st);
int launch_finish_sum(const double* part, int n, double* out, bool take_sqrt, cudaStream_t st);

// fused Lanczos step (make_step, src/ietl/lanczos.h:392-406), after
// launch_hv_*(x -> y, alpha partials):
//   update:    alpha = sum(partA); y = (y - alpha x) - beta_prev v_prev; partB = |y|^2
//   normalize: beta = sqrt(sum(partB)); y /= beta
// beta_prev is read from device memory (NULL: first step, no v_prev term).
template <typename T>
int launch_lanczos_update(const double* partA, int nA, const T* x, const T* vprev, const double* beta_prev, T* y,
                          int64_t n, double* partB, int gridB, double* alpha_out, cudaStream_t st);
template <typename T>
int launch_lanczos_normalize(const double* partB, int nB, T* y, int64_t n, double* beta_out, int grid,
                             cudaStream_t st);

// out[i] = sum_j coef[j] * V[j*ld + i] (FP32 Lanczos store -> FP64 vector),
// coef in device memory (m <= kMaxRitzTerms).
constexpr int kMaxRitzTerms = 4096;
int launch_ritz_combine(const float* V, int64_t ld, int m, const double* coef, double* out, int64_t n,
                        bool accumulate, cudaStream_t st);

int red_grid_size();
int64_t launch_count();

}  // namespace aed
