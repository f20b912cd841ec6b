// batch.cuh -- device state of the batched / served Lanczos engine.
//
// Many independent Lanczos solves (one per request) advance together: every
// step of the engine runs one Lanczos step for every resident instance, with
// work queues of (instance, tile) and (instance, chunk) items, so instances of
// very different dimension share the GPU without one kernel per instance.
// A CUDA graph holds S such steps plus the convergence check and the hand-over
// from the FP32 phase to the FP64 refinement; the host only admits and retires
// requests between graph launches.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "aed_internal.h"
#include "kernels.cuh"

namespace aed {

constexpr int kBatchMaxChunks = 64;  // FP32 basis store: chunks of kStoreChunkB vectors
constexpr int kStoreChunkB = 16;

// Instance phases
enum : int32_t {
  kPhIdle = 0,   // slot free
  kPhLow = 1,    // FP32 Lanczos recurrence, basis kept in HBM
  kPhRitz = 2,   // FP32 phase done: Ritz vectors being assembled into the FP64 start
  kPhHigh = 3,   // FP64 Lanczos recurrence (refinement, or the whole solve in FP64 mode)
  kPhDone = 4,   // results ready
  kPhRR = 5,     // FP32 phase done: the Rayleigh-Ritz step on its Ritz vectors, in FP64
};

// Rayleigh-Ritz hand-over of the batched mixed path: chunk sums of the Gram
// matrices (K (K + 1) / 2 + K^2 for K <= kMaxRR) and the per-request small
// arrays: sums [0, 100), values [100, 108), value order [108, 116), residual
// coefficients cw [116, 180) and cx [180, 244), squared norms [244, 252).
constexpr int kRRSums = kMaxRR * (kMaxRR + 1) / 2 + kMaxRR * kMaxRR;
constexpr int kRRSmall = 256;

struct BInst {
  // set at admission
  const HvParams* P;  // device copy of the coupling tables
  DevTables t;        // sector tables (shared per sector), tiles, per-instance diagonal
  int64_t D;
  int32_t nev;
  int32_t cap;        // alpha/beta capacity (steps) of each phase
  int32_t n_store;    // FP32 basis capacity (vectors)
  int32_t n_tiles;
  int64_t n_chunks;   // reduction chunks (kRedChunk elements)
  int64_t ldv;        // stride of stored FP32 vectors (elements)
  double tol32;       // FP32 phase: residual estimate <= tol32 * |lambda|
  double etol;        // FP64 phase: r^2 / gap <= etol * |lambda| (0: ietl rule only)
  double next_lo;     // mixed: the FP32 phase's lower bound on the eigenvalue above the nev lowest (-1e300: none)
  double rtol, atol;  // ietl rule
  uint64_t seed;      // the request's seed (start vector, Ritz weights)
  float* chunk[kBatchMaxChunks];
  double* v64[3];     // FP64 vectors (rotating)
  double* partA;      // n_tiles
  double* partB;      // n_chunks
  double* ab;         // 2 * cap: alpha_j, beta_j of the current phase
  double* scratch;    // kCheckScratch * cap doubles for the T-matrix analysis
  double* coef;       // cap: Ritz coefficients
  // dynamic
  int32_t phase;
  int32_t j;          // index of the newest Lanczos vector of the current phase
  int32_t m_low;      // FP32 phase length (T size) when it ended
  int32_t n_evals;
  int32_t iters;      // FP64 phase T size at the end
  int32_t converged;
  double ritz_norm;
  // Rayleigh-Ritz hand-over (mixed servers; rr_kmax = 0: none)
  int32_t rr_kmax;    // Ritz vectors budgeted at admission
  int32_t rr_k;       // Ritz vectors of this hand-over
  int32_t rr_nb;      // Ritz pairs below the gap bound
  int32_t rr_need;    // distinct values it must resolve
  int32_t rr_done;    // 1: the result is the Rayleigh-Ritz step's
  double rr_scale;    // largest |eigenvalue| of the FP32 phase's T (merge threshold)
  double* rr_v;       // 2 rr_kmax D doubles: Psi_k at k D, H Psi_k at (rr_kmax + k) D
  double* rr_coef;    // rr_kmax cap: coefficients of the Ritz vectors over the stored basis
  double* rr_part;    // kRRSums n_chunks chunk partials
  double* rr_small;   // kRRSmall doubles
  double evals[AED_MAX_NEV];
  double errs[AED_MAX_NEV];
  double evals_low[AED_MAX_NEV];
};

// Mixed FP64 phase, block Kato-Temple stop: sum_i r_i^2 / (next_lo - theta_max)
// <= kBatchBlockTol |theta_i| over the nev lowest Ritz pairs of the FP64 T,
// next_lo from the FP32 phase (the single-instance Rayleigh-Ritz acceptance).
constexpr double kBatchBlockTol = 5e-10;

// Per-instance T-matrix scratch of the check, in doubles per step of capacity:
// alpha, beta, the spectra and one inverse iteration (16), and kCheckLanes
// lanes' inverse iterations (7 each).
constexpr int kCheckLanes = 8;
constexpr int kCheckScratch = 16 + 7 * kCheckLanes;

struct BItem {
  int32_t inst;
  int32_t idx;  // tile or chunk index within the instance
};

// Kernels of one engine step and of the end-of-graph phase logic.  All take
// the instance table, the item lists and their counts from device memory, so
// a captured graph stays valid while the host changes them between launches.
struct BatchArgs {
  BInst* inst;
  int32_t* n_inst;     // number of slots in use (device)
  BItem* tiles;        // apply items: (instance, bundle of kBatchBundle hi blocks)
  int32_t* n_tiles;
  BItem* chunks;
  int32_t* n_chunks;
  int max_inst;
  int hv_smem;         // dynamic shared memory of the apply (batch_hv_smem_bytes, max over residents)
  // tiles are ordered by FP32 size bucket: bucket b's items are [tile_start[b], tile_start[b + 1])
  // (kBatchBuckets + 1 offsets, device), so each bucket's apply walks only its own items
  int32_t* tile_start;
};

// Hi blocks per work item of the batched apply (entries ub * kBatchBundle ..
// of a sector's block list, applied one block at a time).
constexpr int kBatchBundle = 2;
// Dynamic shared memory the batched apply needs for one instance (the larger
// of its FP64 layout, one block, and its FP32 layout, two blocks).
size_t batch_hv_smem_bytes(int maxrows, const HvParams& P);
// Largest dynamic shared memory a CTA of the batched apply may take on this device.
size_t batch_hv_smem_limit();
// Set the apply kernels' shared-memory limits for a.hv_smem; call before capturing.
int batch_prepare(const BatchArgs& a);
// The FP32 apply is tuned per sector-size bucket: bucket b holds the sectors
// whose largest hi block has maxrows in (kBatchBucketHi[b-1], kBatchBucketHi[b]]
// (the last bucket: everything above).  kBatchCand32 kernel candidates;
// choice32[b] is bucket b's.  Untuned: kBatchDefault32[b].
constexpr int kBatchBuckets = 4;
constexpr int kBatchBucketHi[kBatchBuckets] = {300, 1000, 4000, 0x7fffffff};
constexpr int kBatchCand32 = 5;
constexpr int kBatchDefault32[kBatchBuckets] = {0, 1, 1, 1};
int batch_bucket_of(int maxrows);
const char* batch_cand32_name(int c);
int batch_launch_hv32(const BatchArgs& a, int cand, int bucket, cudaStream_t st);
int batch_tune_bucket(const BatchArgs& a, int bucket, cudaStream_t st, int* best, float* best_ms);
int batch_record_step(const BatchArgs& a, const int* choice32, cudaStream_t st);
int batch_record_check(const BatchArgs& a, cudaStream_t st);
int batch_max_inst_grid();

}  // namespace aed
