// handle.h -- the engine handle behind the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "aed_internal.h"
#include "kernels.cuh"
#include "momentum.cuh"
#include "spin.cuh"

struct aed_handle {
  int device = 0;
  int precision = AED_FP64;
  cudaStream_t stream = nullptr;
  aed::Model model;
  aed::HvParams P;
  aed::BasisTables tab;
  aed::DevTables dt;
  // device memory
  uint32_t* d_thi = nullptr;
  uint16_t* d_tlo = nullptr;
  uint16_t* d_lolist = nullptr;
  uint32_t* d_looff = nullptr;
  uint32_t* d_tile_h = nullptr;
  uint32_t* d_tile_r = nullptr;
  uint32_t* d_blk_h = nullptr;   // block list of the bundle apply
  uint32_t* d_tfirst = nullptr;  // first tile of each hi block
  double* d_dg = nullptr;     // per-row diagonal
  uint32_t* d_ell = nullptr;  // lo-neighbour table
  size_t d_ell_n = 0;         // its capacity (entries), kept across aed_set_couplings
  uint16_t* d_xtab = nullptr;  // crossing-flip table
  double* d_partA = nullptr;  // per-tile partial sums (n_tiles)
  double* d_partB = nullptr;  // per-chunk partial sums (red_chunks(D))
  double* d_scal = nullptr;   // 8 device scalars
  uint32_t* d_flag = nullptr;  // raised by a kernel whose bounded wait gave up
  float* d_dgf = nullptr;      // FP32 handles: the diagonal rounded to FP32
  double* h_scal = nullptr;   // 8 pinned host scalars
  int hv_var[2] = {-1, -1};  // apply variant per precision (FP64, FP32), -1 = not tuned yet
  size_t elem_size() const { return precision == AED_FP32 ? 4 : 8; }
  // rows of H (D, or the representatives of a momentum sector) and the
  // length of a vector in scalars (D, or 2 x rows: interleaved complex)
  int64_t dim = 0;
  int64_t vlen = 0;
  // momentum sector (aed_create_momentum): the tables of momentum.cuh
  bool mom = false;
  aed::MomParams* mp = nullptr;  // host copy (large: kept off the handle's inline storage)
  uint32_t* d_reps = nullptr;
  double* d_norm = nullptr;
  double* d_mdiag = nullptr;
  uint32_t* d_map = nullptr;
  aed::MomTables mom_tables() const { return {d_reps, d_norm, d_mdiag, d_map, dim}; }
  uint64_t* d_sreps = nullptr;  // representatives of a spin-S momentum sector (mom && gen)
  aed::SpinMomTables spin_mom_tables() const { return {d_sreps, d_norm, d_map, dim}; }
  // spin-S sector (aed_create_spin): tables of spin.cuh
  bool gen = false;
  aed::SpinParams* sp = nullptr;
  aed::SpinDev sdev{};
  int two_s = 1;
  uint32_t *d_sthi = nullptr, *d_stlo = nullptr, *d_slolist = nullptr, *d_slooff = nullptr;
  uint32_t *d_sblk_hi = nullptr, *d_sblk_off = nullptr, *d_stile_blk = nullptr, *d_stile_r = nullptr;
  uint2* d_slol = nullptr;  // the lo table of the tabulated Sz-sector apply (sdev.lol), slol_bytes allocated
  size_t slol_bytes = 0;
  // <x, y> partials of one apply (tiles of the real apply, the momentum apply or the spin-S apply)
  int64_t alpha_tiles() const { return mom ? aed::mom_tiles(dim) : gen ? sdev.n_tiles : dt.n_tiles; }
  // solve workspaces, kept between solves (grown on demand, so that a solve
  // makes no allocation once the handle is warm): slot 0 = the three FP64
  // recurrence vectors, slot 1 = device alpha/beta pairs and Ritz coefficients,
  // slot 2 = the Ritz vectors, their images and the partial sums of the mixed
  // path's Rayleigh-Ritz refinement
  static constexpr int kWorkspaces = 3;
  void* ws[kWorkspaces] = {nullptr, nullptr, nullptr};
  size_t ws_bytes[kWorkspaces] = {0, 0, 0};
  std::vector<void*> store_chunks;  // FP32 Lanczos basis of the mixed path, kStoreChunk vectors each
  size_t store_chunk_bytes = 0;
  int store_m = 0;  // vectors of the last mixed solve's FP32 phase in the store (v_0 .. v_{m-1})
  std::vector<double> low_alpha, low_beta;  // that FP32 phase's recurrence
  double* h_ab = nullptr;  // pinned alpha/beta staging
  size_t h_ab_n = 0;
  // last solve: the alpha/beta recurrence of its FP64 phase.  v_{m-1} and v_m
  // of that recurrence stay in workspace slot 0 (buffers (m-1) % 3 and m % 3)
  // while rec_live, for aed_lanczos_save and resumed solves.
  std::vector<double> last_alpha, last_beta;
  int rec_m = 0;
  bool rec_live = false;
  bool last_mixed = false;      // the last solve was the mixed path
  // a mixed solve refined by Rayleigh-Ritz: eigenvector i is
  // sum_j rr_coef[i * rr_m + j] v_j over the FP32 Lanczos basis kept in store_chunks
  bool last_rr = false;
  int rr_m = 0;
  std::vector<double> rr_coef, rr_evals;
  double* d_start64 = nullptr;  // mixed path: start vector of its FP64 phase (D doubles)
};

namespace aed {

// RAII device switch for an API call.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// Memory of handles.  Device and pinned host memory come from per-process
// free lists that keep what handles give back, so that a loop of create /
// solve / destroy allocates once instead of paying cudaFree (a device-wide
// synchronisation) and cudaMallocHost / cudaFreeHost for every handle.
// aed_empty_cache returns the blocks not in use; a failed cudaMalloc does so
// for its device and tries again.
// mem_dev_free(p, st): waits for the work queued on st so far, then caches p.
int mem_dev_alloc(void** p, size_t bytes);
void mem_dev_free(void* p, cudaStream_t st);
int mem_host_alloc(void** p, size_t bytes);
void mem_host_free(void* p);
void mem_empty_cache(int device);

template <typename T>
int mem_dev_alloc_n(T** p, size_t count) {
  void* v = nullptr;
  const int rc = mem_dev_alloc(&v, (count ? count : 1) * sizeof(T));
  *p = static_cast<T*>(v);
  return rc;
}

// Expectation values of site operators in one vector (measure.cu): kind
// kMeasSz <Sz_i>, kMeasSzSz <Sz_i Sz_j>, kMeasSpSm <S+_i S-_j>, n pairs.
constexpr int kMeasSz = AED_OBS_SZ, kMeasSzSz = AED_OBS_SZSZ, kMeasSpSm = AED_OBS_SPSM;
constexpr int kMeasPairs = 32;  // pairs per pass over the vector
struct MeasPairs {
  uint32_t mi[kMeasPairs], mj[kMeasPairs];
};
int measure_pairs(aed_handle* h, const void* psi, int kind, int n, const int32_t* si, const int32_t* sj, double* out);
// The same for a spin-S sector (aed_create_spin; FP64 vectors): spin.cu.
int spin_measure_pairs(aed_handle* h, const double* psi, int kind, int n, const int32_t* si, const int32_t* sj,
                       double* out);
// <psi| sum_p O(si[p], sj[p]) |psi> in a spin-S momentum sector (spin.cu).
int spin_mom_expectation(aed_handle* h, const double* psi, int kind, int n, const int32_t* si, const int32_t* sj,
                         double* out);

int handle_hv(aed_handle* h, bool f32, const void* x, void* y, double* alpha_part);
// AED_ERR_TIMEOUT (and the flag cleared) when a kernel of the handle gave up a
// bounded wait since the last check; waits for the handle's stream.
int handle_check_flag(aed_handle* h);
// Choose the apply variant for this precision now (timed launches on x, y)
// unless already chosen; handle_hv does this on its first call otherwise.
int handle_tune(aed_handle* h, bool f32, const void* x, void* y);
// Workspace of at least `bytes` device bytes / `n` pinned doubles, reused across solves.
int handle_workspace(aed_handle* h, int slot, size_t bytes, void** out);
// Workspace slot 2 of the mixed path's Rayleigh-Ritz step with K Ritz vectors
// of D scalars: the K vectors, their images, the Gram partials and sums.
size_t rr_workspace_bytes(int64_t D, int K);
int handle_pinned(aed_handle* h, size_t n, double** out);
void handle_release_workspace(aed_handle* h);
constexpr int kStoreChunk = 16;
// Bytes of one chunk of the FP32 basis store for vectors of D floats, each
// vector 256-byte aligned within the chunk.
inline size_t store_chunk_bytes_of(int64_t D) { return (((size_t)D * 4 + 255) & ~(size_t)255) * kStoreChunk; }
// Pointer to chunk `c` of the FP32 basis store (allocated on first use), or nullptr.
void* handle_store_chunk(aed_handle* h, int c, size_t chunk_bytes);
int solve(aed_handle* h, const aed_solve_opts* o, aed_solve_result* r);
// Ritz vectors of the last solve by replaying its FP64 recurrence (lanczos.cpp).
int eigenvectors(aed_handle* h, const aed_solve_opts* o, int k, void* const* vecs, double* evals, double* resid);
// Serialised FP64 recurrence of the last solve (lanczos.cpp).
int64_t lanczos_state_bytes(const aed_handle* h);
int lanczos_save(aed_handle* h, void* buf, int64_t bytes);
int lanczos_load(aed_handle* h, const void* buf, int64_t bytes);
// One make_step on device vectors: apply, alpha, update, beta, normalise.
// beta_prev / alpha / beta are device scalars; v_prev may be NULL.
int lanczos_step_kernels(aed_handle* h, bool f32, const void* v_prev, const void* v_cur, void* v_next,
                         const double* beta_prev, double* alpha, double* beta);

}  // namespace aed
