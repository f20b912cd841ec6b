// server.cpp -- the batched / served Lanczos engine (aed_server_* in include/aed.h).
//
// Requests (a model + solve options) are queued on submission and admitted
// into device-resident slots while the server's HBM budget allows: the
// footprint of a request is its diagonal, FP64 vectors, FP32 Lanczos basis
// and T-matrix scratch, plus its sector's tables if no resident request
// already holds them.  Every aed_server_step admits what fits, rebuilds the
// (instance, tile) and (instance, chunk) work queues when the resident set
// changed, launches one CUDA graph of S engine steps plus the convergence
// check, and harvests finished requests (freeing their slots and memory), so
// requests that arrive while others run join at the next step: continuous
// batching.  All device memory is taken with cudaMallocAsync on the server's
// stream and returned with cudaFreeAsync.

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "batch.cuh"
#include "handle.h"

namespace aed {
namespace {

using clk = std::chrono::steady_clock;

struct Sector {
  BasisTables tab;
  uint32_t *thi = nullptr, *looff = nullptr, *tile_h = nullptr, *tile_r = nullptr;
  uint16_t* xtab = nullptr;  // crossing-flip table
  uint32_t *blk_h = nullptr, *tfirst = nullptr;  // block list of the bundle apply, first tile per hi block
  std::vector<uint32_t> blk;                     // host copy of the block list (work items)
  int maxrows = 0;
  uint16_t *tlo = nullptr, *lolist = nullptr;
  int64_t n_tiles = 0;
  size_t bytes = 0;
  int refs = 0;
};

struct Request {
  int64_t ticket = 0;
  int64_t dim = 0;  // sector dimension
  Model model;
  aed_solve_opts opts{};
  clk::time_point t_submit;
  int status = AED_PENDING;  // AED_PENDING, AED_OK or an error code
  aed_solve_result res{};
  size_t footprint = 0;
  bool cancelled = false;
  std::string error;  // message of a failed request (the solving thread's aed_last_error)
};

struct Slot {
  bool used = false;
  bool has_sector = false;
  std::shared_ptr<Request> req;
  std::pair<int, int> sector{0, 0};
  std::vector<void*> allocs;  // freed at retirement
  size_t bytes = 0;
  BInst inst{};
};

// A request solved on its own handle (single-instance engine: the tuned apply
// variants, the Rayleigh-Ritz refinement) by a host thread, beside the batch.
struct Lane {
  std::shared_ptr<Request> req;
  std::thread th;
  std::atomic<bool> done{false};
  size_t bytes = 0;
};

}  // namespace
}  // namespace aed

// The server's device counters: n_inst, n_tiles, n_chunks, one unused, then the
// start of every FP32 size bucket's apply items and the end of the last.
constexpr int kBucketStarts = 4;
constexpr int kCounts = kBucketStarts + aed::kBatchBuckets + 1;

struct aed_server {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaMemPool_t pool = nullptr;
  int max_slots = 0;
  int S = 8;
  int precision = AED_FP32;
  size_t budget = 0, used = 0;
  std::mutex mu;
  int64_t next_ticket = 1;
  std::deque<std::shared_ptr<aed::Request>> queue;
  std::map<int64_t, std::shared_ptr<aed::Request>> requests;
  std::vector<aed::Slot> slots;
  std::map<std::pair<int, int>, aed::Sector> sectors;
  // device tables of the engine
  aed::BInst* d_inst = nullptr;
  int32_t* d_counts = nullptr;  // n_inst, n_tiles, n_chunks, (unused), the buckets' tile starts (kCounts)
  aed::BItem* d_tiles = nullptr;
  aed::BItem* d_chunks = nullptr;
  size_t cap_tiles = 0, cap_chunks = 0;
  std::vector<aed::BInst> h_inst;  // readback of d_inst
  int32_t* h_counts = nullptr;     // pinned
  bool dirty = true;
  cudaGraphExec_t graph = nullptr;
  bool graph_stale = true;
  int hv_smem = 0;  // dynamic shared memory of the apply in the graph
  int64_t launches = 0;
  // the FP32 apply kernel of each sector-size bucket (batch.cuh), tuned on
  // the first resident work of the bucket unless AED_BATCH_VARIANT forces one
  int choice32[aed::kBatchBuckets] = {};
  bool tuned32[aed::kBatchBuckets] = {};
  // single-instance lanes for the large sectors
  int max_lanes = 2;
  int64_t lane_min_dim = (int64_t)1 << 21;
  std::vector<std::unique_ptr<aed::Lane>> lanes;
};

namespace aed {
namespace {

int64_t sector_tiles_est(int64_t D) { return (D + kHvTileRows - 1) / kHvTileRows + 64; }

int dmalloc(aed_server* s, void** p, size_t bytes) {
  *p = nullptr;
  const cudaError_t e = cudaMallocAsync(p, bytes ? bytes : 8, s->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return fail(AED_ERR_NOMEM, std::string("server allocation of ") + std::to_string(bytes) +
                                   " bytes: " + cudaGetErrorString(e));
  }
  return AED_OK;
}

// Ritz vectors a request's Rayleigh-Ritz hand-over may use (the clusters of
// its nev lowest values with a few ghost copies); more falls back to the
// FP64 Lanczos refinement.
int rr_kmax_of(int nev) { return std::min(kMaxRR, nev + 3); }

// Bytes a request holds while resident (the admission footprint).
size_t request_bytes(const aed_server* s, int N, int64_t D, int nev, int cap, int n_store) {
  const size_t ldv = ((size_t)D * 4 + 255) & ~(size_t)255;
  size_t b = (size_t)D * 8;                      // diagonal
  b += 3 * (((size_t)D * 8 + 255) & ~(size_t)255);  // FP64 vectors
  if (s->precision == AED_FP32) b += ldv * (size_t)((n_store + kStoreChunkB - 1) / kStoreChunkB) * kStoreChunkB;
  b += (size_t)sector_tiles_est(D) * 8 + (size_t)red_chunks(D) * 8;  // partials
  b += (size_t)cap * 8 * (2 + kCheckScratch + 1);                               // alpha/beta, scratch, coefficients
  b += sizeof(HvParams) + 4096;
  b += (size_t)40 * ((size_t)1 << ((N + 1) / 2)) * 4;  // lo-neighbour table (width <= 40)
  if (s->precision == AED_FP32) {  // the Rayleigh-Ritz hand-over: K vectors and their images, sums
    const size_t k = (size_t)rr_kmax_of(nev);
    b += 2 * k * (((size_t)D * 8 + 255) & ~(size_t)255) + k * (size_t)cap * 8 +
         (size_t)kRRSums * (size_t)red_chunks(D) * 8 + (size_t)kRRSmall * 8;
  }
  return b;
}

size_t sector_bytes(int N, int n_up) {
  BasisTables t;
  if (build_tables(N, n_up, t)) return 0;
  return t.thi.size() * 4 + t.tlo.size() * 2 + t.lolist.size() * 2 + t.looff.size() * 4 +
         (size_t)t.Nlo * t.tlo.size() * 2 + (size_t)sector_tiles_est(t.D) * 8 + t.thi.size() * 8 + 4096 +
         (size_t)4 * kBundleMax * (t.Nlo + 1);
}

int sector_acquire(aed_server* s, int N, int n_up, Sector** out) {
  auto key = std::make_pair(N, n_up);
  auto it = s->sectors.find(key);
  if (it != s->sectors.end()) {
    it->second.refs++;
    *out = &it->second;
    return AED_OK;
  }
  Sector sec;
  int rc = build_tables(N, n_up, sec.tab);
  if (rc) return rc;
  std::vector<uint32_t> th, tr, tf;
  std::vector<uint16_t> xt;
  build_tiles(sec.tab, kHvTileRows, th, tr, &tf);
  build_cross_table(sec.tab, xt);
  build_block_list(sec.tab, sec.blk, &sec.maxrows);
  sec.n_tiles = (int64_t)th.size();
  const size_t nhi = sec.tab.thi.size(), nlo = sec.tab.tlo.size(), nof = sec.tab.looff.size();
  if ((rc = dmalloc(s, (void**)&sec.thi, nhi * 4)) || (rc = dmalloc(s, (void**)&sec.tlo, nlo * 2)) ||
      (rc = dmalloc(s, (void**)&sec.lolist, nlo * 2)) || (rc = dmalloc(s, (void**)&sec.looff, nof * 4)) ||
      (rc = dmalloc(s, (void**)&sec.tile_h, th.size() * 4 + 4)) ||
      (rc = dmalloc(s, (void**)&sec.tile_r, tr.size() * 4 + 4)) ||
      (rc = dmalloc(s, (void**)&sec.xtab, xt.size() * 2 + 4)) ||
      (rc = dmalloc(s, (void**)&sec.blk_h, sec.blk.size() * 4 + 4)) ||
      (rc = dmalloc(s, (void**)&sec.tfirst, tf.size() * 4 + 4)))
    return rc;
  cudaMemcpyAsync(sec.thi, sec.tab.thi.data(), nhi * 4, cudaMemcpyHostToDevice, s->stream);
  cudaMemcpyAsync(sec.tlo, sec.tab.tlo.data(), nlo * 2, cudaMemcpyHostToDevice, s->stream);
  cudaMemcpyAsync(sec.lolist, sec.tab.lolist.data(), nlo * 2, cudaMemcpyHostToDevice, s->stream);
  cudaMemcpyAsync(sec.looff, sec.tab.looff.data(), nof * 4, cudaMemcpyHostToDevice, s->stream);
  if (!th.empty()) {
    cudaMemcpyAsync(sec.tile_h, th.data(), th.size() * 4, cudaMemcpyHostToDevice, s->stream);
    cudaMemcpyAsync(sec.tile_r, tr.data(), tr.size() * 4, cudaMemcpyHostToDevice, s->stream);
  }
  if (!xt.empty()) cudaMemcpyAsync(sec.xtab, xt.data(), xt.size() * 2, cudaMemcpyHostToDevice, s->stream);
  if (!sec.blk.empty())
    cudaMemcpyAsync(sec.blk_h, sec.blk.data(), sec.blk.size() * 4, cudaMemcpyHostToDevice, s->stream);
  if (!tf.empty()) cudaMemcpyAsync(sec.tfirst, tf.data(), tf.size() * 4, cudaMemcpyHostToDevice, s->stream);
  AED_CUDA_TRY(cudaStreamSynchronize(s->stream));  // host vectors th/tr/xt/tf go out of scope
  sec.bytes = sector_bytes(N, n_up);
  sec.refs = 1;
  s->used += sec.bytes;
  auto ins = s->sectors.emplace(key, std::move(sec));
  *out = &ins.first->second;
  return AED_OK;
}

void sector_release(aed_server* s, std::pair<int, int> key) {
  auto it = s->sectors.find(key);
  if (it == s->sectors.end()) return;
  if (--it->second.refs > 0) return;
  Sector& sec = it->second;
  for (void* p : {(void*)sec.thi, (void*)sec.tlo, (void*)sec.lolist, (void*)sec.looff, (void*)sec.tile_h,
                  (void*)sec.tile_r, (void*)sec.xtab, (void*)sec.blk_h, (void*)sec.tfirst})
    if (p) cudaFreeAsync(p, s->stream);
  s->used -= std::min(s->used, sec.bytes);
  s->sectors.erase(it);
}

constexpr int kServerStore = 144;  // FP32 basis vectors per request (9 chunks)

int cap_of(const Request& r, int64_t D) {
  int cap = r.opts.max_iter > 0 ? r.opts.max_iter : (int)std::min<int64_t>(10 * D, 1000);
  return std::max(cap, r.opts.nev + 4);
}

// Place request r into slot k: allocations, tables, couplings, diagonal, start vector.
int admit(aed_server* s, int k, const std::shared_ptr<Request>& r) {
  Slot& sl = s->slots[k];
  sl = Slot();
  sl.req = r;
  Sector* sec = nullptr;
  int rc = sector_acquire(s, r->model.N, r->model.n_up, &sec);
  if (rc) return rc;
  sl.sector = {r->model.N, r->model.n_up};
  sl.has_sector = true;
  const int64_t D = sec->tab.D;
  BInst& I = sl.inst;
  I = BInst{};
  HvParams P;
  if ((rc = build_hv_params(r->model, sec->tab.Nlo, P))) return rc;
  const size_t smem = batch_hv_smem_bytes(sec->maxrows, P);
  if (smem > batch_hv_smem_limit())
    return fail(AED_ERR_INVALID, "sector too large for the batched apply's shared memory");
  if ((int)smem > s->hv_smem) {  // the graph's apply needs more shared memory: capture again
    s->hv_smem = (int)((smem + 1023) & ~(size_t)1023);
    s->graph_stale = true;
  }
  const int cap = cap_of(*r, D);
  const int n_store = s->precision == AED_FP32 ? std::min(kServerStore, std::min(cap + 1, kBatchMaxChunks * kStoreChunkB)) : 0;
  auto take = [&](void** p, size_t bytes) -> int {
    int e = dmalloc(s, p, bytes);
    if (!e) sl.allocs.push_back(*p);
    return e;
  };
  void* pP = nullptr;
  void* pdg = nullptr;
  if ((rc = take(&pP, sizeof(HvParams))) || (rc = take(&pdg, (size_t)D * 8))) return rc;
  for (int q = 0; q < 3; ++q)
    if ((rc = take((void**)&I.v64[q], (size_t)D * 8))) return rc;
  if ((rc = take((void**)&I.partA, (size_t)sec->n_tiles * 8 + 8)) ||
      (rc = take((void**)&I.partB, (size_t)red_chunks(D) * 8 + 8)) || (rc = take((void**)&I.ab, (size_t)cap * 16)) ||
      (rc = take((void**)&I.scratch, (size_t)cap * kCheckScratch * 8 + 64)) || (rc = take((void**)&I.coef, (size_t)cap * 8)))
    return rc;
  I.rr_kmax = 0;
  I.rr_k = 0;
  I.rr_done = 0;
  if (s->precision == AED_FP32) {
    const int k = rr_kmax_of(r->opts.nev);
    const size_t vd = ((size_t)D * 8 + 255) & ~(size_t)255;
    void* pv = nullptr;
    if ((rc = take(&pv, 2 * (size_t)k * vd)) || (rc = take((void**)&I.rr_coef, (size_t)k * cap * 8)) ||
        (rc = take((void**)&I.rr_part, (size_t)kRRSums * (size_t)red_chunks(D) * 8 + 8)) ||
        (rc = take((void**)&I.rr_small, (size_t)kRRSmall * 8)))
      return rc;
    I.rr_v = (double*)pv;
    I.rr_kmax = k;
  }
  const size_t vb = ((size_t)D * 4 + 255) & ~(size_t)255;
  I.ldv = (int64_t)(vb / 4);
  for (int c = 0; c * kStoreChunkB < n_store; ++c)
    if ((rc = take((void**)&I.chunk[c], vb * kStoreChunkB))) return rc;
  cudaMemcpyAsync(pP, &P, sizeof(HvParams), cudaMemcpyHostToDevice, s->stream);
  I.P = (const HvParams*)pP;
  DevTables& t = I.t;
  t.thi = sec->thi;
  t.tlo = sec->tlo;
  t.lolist = sec->lolist;
  t.looff = sec->looff;
  t.tile_h = sec->tile_h;
  t.tile_r = sec->tile_r;
  t.xtab = sec->xtab;
  t.blk_h = sec->blk_h;
  t.tfirst = sec->tfirst;
  t.n_blk = (int64_t)sec->blk.size();
  t.maxrows = sec->maxrows;
  t.n_tiles = sec->n_tiles;
  t.D = D;
  t.Nlo = sec->tab.Nlo;
  t.Nhi = sec->tab.Nhi;
  t.n_up = sec->tab.n_up;
  t.dg = (const double*)pdg;
  {
    std::vector<uint32_t> ell;
    int W = 0;
    build_lo_table(sec->tab, P, ell, &W);
    void* pe = nullptr;
    if ((rc = take(&pe, ell.size() * 4 + 4))) return rc;
    if (!ell.empty()) {
      cudaMemcpyAsync(pe, ell.data(), ell.size() * 4, cudaMemcpyHostToDevice, s->stream);
      AED_CUDA_TRY(cudaStreamSynchronize(s->stream));  // host vector goes out of scope
    }
    t.ell = (const uint32_t*)pe;
    t.ell_w = W;
  }
  if ((rc = launch_diag_table(P, t, (double*)pdg, s->stream))) return rc;
  I.D = D;
  I.nev = r->opts.nev;
  I.cap = cap;
  I.n_store = n_store;
  I.n_tiles = (int32_t)sec->n_tiles;
  I.n_chunks = red_chunks(D);
  const double eps = 2.220446049250313e-16;
  I.seed = r->opts.seed;
  I.rtol = r->opts.rtol > 0 ? r->opts.rtol : 100 * eps;
  I.atol = r->opts.atol > 0 ? r->opts.atol : 100 * eps;
  I.tol32 = 2e-6;
  I.etol = s->precision == AED_FP32 ? 1e-11 : 0.0;
  I.next_lo = -1e300;
  I.j = 0;
  // start vector, normalised (lanczos.h:381-383)
  double* nrm = I.scratch;
  if (s->precision == AED_FP32) {
    float* v0 = I.chunk[0];
    if ((rc = launch_fill_random(v0, D, r->opts.seed, s->stream)) ||
        (rc = launch_dot_partials(v0, v0, D, I.partB, true, s->stream)) ||
        (rc = launch_finish_sum(I.partB, red_chunks(D), nrm, true, s->stream)) ||
        (rc = launch_lanczos_normalize(nrm, v0, D, s->stream)))
      return rc;
    I.phase = kPhLow;
  } else {
    double* v0 = I.v64[0];
    if ((rc = launch_fill_random(v0, D, r->opts.seed, s->stream)) ||
        (rc = launch_dot_partials(v0, v0, D, I.partB, true, s->stream)) ||
        (rc = launch_finish_sum(I.partB, red_chunks(D), nrm, true, s->stream)) ||
        (rc = launch_lanczos_normalize(nrm, v0, D, s->stream)))
      return rc;
    I.phase = kPhHigh;
  }
  sl.bytes = r->footprint;
  sl.used = true;
  s->used += sl.bytes;
  // publish the slot's descriptor (the running graph only sees it at the next launch)
  AED_CUDA_TRY(cudaMemcpyAsync(s->d_inst + k, &I, sizeof(BInst), cudaMemcpyHostToDevice, s->stream));
  return AED_OK;
}

void release_slot(aed_server* s, int k) {
  Slot& sl = s->slots[k];
  for (void* p : sl.allocs) cudaFreeAsync(p, s->stream);
  sl.allocs.clear();
  if (sl.used) s->used -= std::min(s->used, sl.bytes);
  if (sl.has_sector) sector_release(s, sl.sector);
  BInst idle{};
  idle.phase = kPhIdle;
  s->h_inst[k] = idle;
  cudaMemcpyAsync(s->d_inst + k, &s->h_inst[k], sizeof(BInst), cudaMemcpyHostToDevice, s->stream);
  // the copy above reads h_inst[k] asynchronously; h_inst is only rewritten
  // after the next stream synchronisation
  sl = Slot();
}

int rebuild_items(aed_server* s) {
  std::vector<BItem> tiles, chunks, by_bucket[kBatchBuckets];
  int n_inst = 0;
  for (int k = 0; k < (int)s->slots.size(); ++k) {
    if (!s->slots[k].used) continue;
    n_inst = k + 1;
    const BInst& I = s->slots[k].inst;
    const std::vector<uint32_t>& blk = s->sectors.at(s->slots[k].sector).blk;
    std::vector<BItem>& mine = by_bucket[batch_bucket_of(I.t.maxrows)];
    for (size_t ub = 0; ub * kBatchBundle < blk.size(); ++ub)  // bundles holding at least one block
      if (blk[ub * kBatchBundle] != kNoBlockEntry) mine.push_back({k, (int32_t)ub});
    for (int64_t c = 0; c < I.n_chunks; ++c) chunks.push_back({k, (int32_t)c});
  }
  // the apply items bucket by bucket (an instance's items stay together), with each bucket's start
  for (int b = 0; b < kBatchBuckets; ++b) {
    s->h_counts[kBucketStarts + b] = (int32_t)tiles.size();
    tiles.insert(tiles.end(), by_bucket[b].begin(), by_bucket[b].end());
  }
  s->h_counts[kBucketStarts + kBatchBuckets] = (int32_t)tiles.size();
  if (tiles.size() > s->cap_tiles || chunks.size() > s->cap_chunks) {
    AED_CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (s->d_tiles) cudaFree(s->d_tiles);
    if (s->d_chunks) cudaFree(s->d_chunks);
    s->d_tiles = nullptr;
    s->d_chunks = nullptr;
    s->cap_tiles = std::max<size_t>(tiles.size() * 2, 1 << 14);
    s->cap_chunks = std::max<size_t>(chunks.size() * 2, 1 << 14);
    if (cudaMalloc(&s->d_tiles, s->cap_tiles * sizeof(BItem)) != cudaSuccess ||
        cudaMalloc(&s->d_chunks, s->cap_chunks * sizeof(BItem)) != cudaSuccess) {
      cudaGetLastError();
      return fail(AED_ERR_NOMEM, "server work queues");
    }
    s->graph_stale = true;
  }
  if (!tiles.empty())
    AED_CUDA_TRY(cudaMemcpyAsync(s->d_tiles, tiles.data(), tiles.size() * sizeof(BItem), cudaMemcpyHostToDevice,
                                 s->stream));
  if (!chunks.empty())
    AED_CUDA_TRY(cudaMemcpyAsync(s->d_chunks, chunks.data(), chunks.size() * sizeof(BItem), cudaMemcpyHostToDevice,
                                 s->stream));
  s->h_counts[0] = n_inst;
  s->h_counts[1] = (int32_t)tiles.size();
  s->h_counts[2] = (int32_t)chunks.size();
  AED_CUDA_TRY(cudaMemcpyAsync(s->d_counts, s->h_counts, kCounts * sizeof(int32_t), cudaMemcpyHostToDevice, s->stream));
  // tiles/chunks are host temporaries: finish the copies before they go
  AED_CUDA_TRY(cudaStreamSynchronize(s->stream));
  s->dirty = false;
  return AED_OK;
}

// Autotuner of the batched apply: every bucket that has instances in the
// FP32 phase and no choice yet gets the fastest candidate on that work
// (batch_tune_bucket; the choice is kept for the server's life); the graph is
// captured again with it.
int tune_buckets(aed_server* s) {
  bool want[kBatchBuckets] = {};
  for (const Slot& sl : s->slots)
    if (sl.used && sl.inst.phase == kPhLow) want[batch_bucket_of(sl.inst.t.maxrows)] = true;
  BatchArgs a{s->d_inst, s->d_counts, s->d_tiles, s->d_counts + 1, s->d_chunks, s->d_counts + 2, s->max_slots,
              s->hv_smem, s->d_counts + kBucketStarts};
  for (int b = 0; b < kBatchBuckets; ++b) {
    if (!want[b] || s->tuned32[b]) continue;
    int rc = batch_prepare(a);
    int best = -1;
    float ms = 0.f;
    if (!rc) rc = batch_tune_bucket(a, b, s->stream, &best, &ms);
    if (rc) return rc;
    s->choice32[b] = best;
    s->tuned32[b] = true;
    s->graph_stale = true;
    if (std::getenv("AED_VERBOSE"))
      std::fprintf(stderr, "[aed] batched FP32 apply, bucket %d: %s (%.3f ms for 3 launches)\n", b,
                   batch_cand32_name(best), ms);
  }
  return AED_OK;
}

// Device bytes of a single-instance solve of dimension D with FP32 store
// capacity n_store: the handle's per-row tables and vectors (diagonal in FP64
// and FP32, five recurrence vectors, the refinement's start and Rayleigh-Ritz
// vectors) and the FP32 basis.
size_t lane_bytes(const aed_server* s, int64_t D, int n_store) {
  const size_t per_row = 8 + 4 + 5 * 8 + 8 + 2 * kMaxRR * 8 + (s->precision == AED_FP32 ? 4 * (size_t)n_store : 0);
  return (size_t)D * per_row + ((size_t)64 << 20);
}

void lane_main(aed_server* s, Lane* L) {
  cudaSetDevice(s->device);
  Request& r = *L->req;
  const Model& m = r.model;
  std::vector<int32_t> s1(m.s1.begin(), m.s1.end()), s2(m.s2.begin(), m.s2.end());
  const aed_model_desc md{m.N,          m.n_up,      (int32_t)s1.size(),
                          s1.data(),    s2.data(),   m.jz.data(),
                          m.jxy.data(), m.kq.data(), m.site_h.empty() ? nullptr : m.site_h.data(),
                          m.site_d.empty() ? nullptr : m.site_d.data()};
  aed_handle* h = nullptr;
  aed_solve_result res{};
  int rc = aed_create(&md, s->precision, s->device, &h);
  if (!rc) {
    aed_solve_opts o = r.opts;
    rc = aed_solve(h, &o, &res);
  }
  const std::string err = rc ? std::string(aed_last_error()) : std::string();
  if (h) aed_destroy(h);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (!r.cancelled) {
      r.res = res;
      r.res.seconds = std::chrono::duration<double>(clk::now() - r.t_submit).count();
      r.status = rc ? rc : AED_OK;
      r.error = err;
    }
    s->used -= std::min(s->used, L->bytes);
  }
  L->done = true;
}

// Join the lanes whose solve has finished (they set `done` after their last
// use of the server's lock).
void reap_lanes(aed_server* s) {
  for (size_t i = 0; i < s->lanes.size();) {
    if (s->lanes[i]->done) {
      s->lanes[i]->th.join();
      s->lanes.erase(s->lanes.begin() + (long)i);
    } else {
      ++i;
    }
  }
}

int capture_graph(aed_server* s) {
  if (s->graph) {
    cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
  }
  BatchArgs a{s->d_inst, s->d_counts, s->d_tiles, s->d_counts + 1, s->d_chunks, s->d_counts + 2, s->max_slots,
              s->hv_smem, s->d_counts + kBucketStarts};
  cudaGraph_t g = nullptr;
  const int rp = batch_prepare(a);
  if (rp) return rp;
  AED_CUDA_TRY(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
  int rc = AED_OK;
  for (int k = 0; k < s->S && !rc; ++k) rc = batch_record_step(a, s->choice32, s->stream);
  if (!rc) rc = batch_record_check(a, s->stream);
  const cudaError_t e = cudaStreamEndCapture(s->stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return fail(AED_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  const cudaError_t e2 = cudaGraphInstantiate(&s->graph, g, 0);
  cudaGraphDestroy(g);
  if (e2 != cudaSuccess) return fail(AED_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e2));
  s->graph_stale = false;
  return AED_OK;
}

void finish_request(aed_server* s, int k) {
  Slot& sl = s->slots[k];
  const BInst& I = s->h_inst[k];
  Request& r = *sl.req;
  std::memset(&r.res, 0, sizeof r.res);
  r.res.n_evals = I.n_evals;
  r.res.iterations = I.iters;
  r.res.iterations_low = s->precision == AED_FP32 ? I.m_low : 0;
  r.res.converged = I.converged;
  // the batched mixed path refines by the Rayleigh-Ritz step or FP64 Lanczos steps
  r.res.refined_by = s->precision != AED_FP32 ? AED_REFINE_NONE
                     : I.rr_done           ? AED_REFINE_RAYLEIGH_RITZ
                                           : AED_REFINE_LANCZOS;
  for (int i = 0; i < I.n_evals && i < AED_MAX_NEV; ++i) {
    r.res.evals[i] = I.evals[i];
    r.res.errors[i] = I.errs[i];
    r.res.evals_low[i] = I.evals_low[i];
  }
  r.res.seconds = std::chrono::duration<double>(clk::now() - r.t_submit).count();
  r.status = AED_OK;
  release_slot(s, k);
}

}  // namespace
}  // namespace aed

using namespace aed;

extern "C" {

int aed_server_create(const aed_server_opts* o, aed_server** out) {
  if (!o || !out) return fail(AED_ERR_INVALID, "NULL argument");
  *out = nullptr;
  if (o->precision != AED_FP32 && o->precision != AED_FP64) return fail(AED_ERR_INVALID, "precision");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(AED_ERR_CUDA, "no CUDA device available");
  }
  if (o->device < 0 || o->device >= ndev) return fail(AED_ERR_INVALID, "device index out of range");
  DeviceGuard g(o->device);
  std::unique_ptr<aed_server> s(new aed_server);
  s->device = o->device;
  s->max_slots = o->max_slots > 0 ? o->max_slots : 512;
  s->S = o->steps_per_launch > 0 ? o->steps_per_launch : 8;
  s->precision = o->precision;
  AED_CUDA_TRY(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
  size_t fr = 0, tot = 0;
  AED_CUDA_TRY(cudaMemGetInfo(&fr, &tot));
  const double frac = (o->hbm_fraction > 0 && o->hbm_fraction <= 0.95) ? o->hbm_fraction : 0.8;
  s->budget = o->hbm_budget_bytes > 0 ? (size_t)o->hbm_budget_bytes : (size_t)(frac * (double)fr);
  // keep freed memory in the stream-ordered pool for the next requests
  AED_CUDA_TRY(cudaDeviceGetDefaultMemPool(&s->pool, s->device));
  uint64_t thresh = UINT64_MAX;
  cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &thresh);
  if (o->reserve_bytes != 0) {  // map memory into the pool now (best effort): later requests reuse it
    const size_t want = o->reserve_bytes < 0 ? s->budget : std::min((size_t)o->reserve_bytes, s->budget);
    void* p = nullptr;
    if (want > 0 && cudaMallocAsync(&p, want, s->stream) == cudaSuccess) {
      cudaFreeAsync(p, s->stream);
      cudaStreamSynchronize(s->stream);
    } else {
      cudaGetLastError();
    }
  }
  if (o->max_lanes > 0) s->max_lanes = o->max_lanes;
  if (o->lane_min_dim > 0) s->lane_min_dim = o->lane_min_dim;
  if (o->lane_min_dim < 0) s->max_lanes = 0;
  for (int b = 0; b < kBatchBuckets; ++b) s->choice32[b] = kBatchDefault32[b];
  if (const char* env = std::getenv("AED_BATCH_VARIANT")) {  // one candidate for every bucket, no tuning
    const int v = std::atoi(env);
    if (v >= 0 && v < kBatchCand32)
      for (int b = 0; b < kBatchBuckets; ++b) {
        s->choice32[b] = v;
        s->tuned32[b] = true;
      }
  }
  s->slots.resize(s->max_slots);
  s->h_inst.resize(s->max_slots);
  for (auto& b : s->h_inst) b = BInst{};
  if (cudaMalloc(&s->d_inst, sizeof(BInst) * s->max_slots) != cudaSuccess ||
      cudaMalloc(&s->d_counts, kCounts * sizeof(int32_t)) != cudaSuccess ||
      cudaMallocHost(&s->h_counts, kCounts * sizeof(int32_t)) != cudaSuccess) {
    cudaGetLastError();
    return fail(AED_ERR_NOMEM, "server tables");
  }
  AED_CUDA_TRY(cudaMemset(s->d_inst, 0, sizeof(BInst) * s->max_slots));
  AED_CUDA_TRY(cudaMemset(s->d_counts, 0, kCounts * sizeof(int32_t)));
  s->cap_tiles = s->cap_chunks = 1 << 14;
  if (cudaMalloc(&s->d_tiles, s->cap_tiles * sizeof(BItem)) != cudaSuccess ||
      cudaMalloc(&s->d_chunks, s->cap_chunks * sizeof(BItem)) != cudaSuccess) {
    cudaGetLastError();
    return fail(AED_ERR_NOMEM, "server work queues");
  }
  int rc = rebuild_items(s.get());
  if (!rc) rc = capture_graph(s.get());
  if (rc) return rc;
  *out = s.release();
  return AED_OK;
}

int aed_server_destroy(aed_server* s) {
  if (!s) return AED_OK;
  DeviceGuard g(s->device);
  for (auto& L : s->lanes) L->th.join();  // a lane's solve cannot be interrupted: wait for it
  s->lanes.clear();
  cudaStreamSynchronize(s->stream);
  for (int k = 0; k < (int)s->slots.size(); ++k)
    if (s->slots[k].used) release_slot(s, k);
  cudaStreamSynchronize(s->stream);
  for (auto& kv : s->sectors) {
    Sector& sec = kv.second;
    for (void* p : {(void*)sec.thi, (void*)sec.tlo, (void*)sec.lolist, (void*)sec.looff, (void*)sec.tile_h,
                    (void*)sec.tile_r, (void*)sec.xtab, (void*)sec.blk_h, (void*)sec.tfirst})
      if (p) cudaFreeAsync(p, s->stream);
  }
  cudaStreamSynchronize(s->stream);
  if (s->graph) cudaGraphExecDestroy(s->graph);
  cudaMemPoolTrimTo(s->pool, 0);
  cudaFree(s->d_inst);
  cudaFree(s->d_counts);
  cudaFree(s->d_tiles);
  cudaFree(s->d_chunks);
  if (s->h_counts) cudaFreeHost(s->h_counts);
  cudaStreamDestroy(s->stream);
  delete s;
  return AED_OK;
}

int aed_server_submit(aed_server* s, const aed_model_desc* model, const aed_solve_opts* opts, int64_t* ticket) {
  if (!s || !model || !opts || !ticket) return fail(AED_ERR_INVALID, "NULL argument");
  if (opts->nev < 1 || opts->nev > AED_MAX_NEV) return fail(AED_ERR_INVALID, "nev must be in 1..16");
  auto r = std::make_shared<Request>();
  int rc = model_from_desc(model, r->model);
  if (rc) return rc;
  BasisTables t;
  if ((rc = build_tables(r->model.N, r->model.n_up, t))) return rc;
  if (t.D < 2) return fail(AED_ERR_INVALID, "the server solves sectors of dimension >= 2 (use aed_solve)");
  r->opts = *opts;
  r->opts.start = nullptr;  // the server draws its own start vectors
  r->dim = t.D;
  const int cap = cap_of(*r, t.D);
  const int n_store = s->precision == AED_FP32 ? std::min(kServerStore, cap + 1) : 0;
  r->footprint = request_bytes(s, r->model.N, t.D, opts->nev, cap, n_store);
  if (r->footprint + sector_bytes(r->model.N, r->model.n_up) > s->budget)
    return fail(AED_ERR_ADMISSION, "request footprint (" + std::to_string(r->footprint) +
                                       " bytes) exceeds the server's HBM budget (" + std::to_string(s->budget) + ")");
  r->t_submit = clk::now();
  std::lock_guard<std::mutex> lk(s->mu);
  r->ticket = s->next_ticket++;
  s->requests[r->ticket] = r;
  s->queue.push_back(r);
  *ticket = r->ticket;
  return AED_OK;
}

int aed_server_cancel(aed_server* s, int64_t ticket) {
  if (!s) return fail(AED_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->requests.find(ticket);
  if (it == s->requests.end()) return fail(AED_ERR_INVALID, "unknown ticket");
  if (it->second->status == AED_PENDING) {
    it->second->cancelled = true;
    it->second->status = AED_ERR_CANCELLED;
  }
  return AED_OK;
}

int aed_server_step(aed_server* s, int32_t* n_pending) {
  if (!s) return fail(AED_ERR_INVALID, "NULL argument");
  DeviceGuard g(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  int rc;
  // drop cancelled requests that are still resident
  for (int k = 0; k < (int)s->slots.size(); ++k)
    if (s->slots[k].used && s->slots[k].req->cancelled) {
      release_slot(s, k);
      s->dirty = true;
    }
  reap_lanes(s);
  const bool use_lanes = s->max_lanes > 0 && s->lane_min_dim > 0;
  // large sectors: single-instance lanes, in arrival order while lanes and budget allow
  if (use_lanes) {
    for (auto it = s->queue.begin(); it != s->queue.end() && (int)s->lanes.size() < s->max_lanes;) {
      auto r = *it;
      if (r->cancelled) {
        it = s->queue.erase(it);
        continue;
      }
      if (r->dim < s->lane_min_dim) {
        ++it;
        continue;
      }
      const size_t need = lane_bytes(s, r->dim, std::min(kServerStore, cap_of(*r, r->dim) + 1));
      if (s->used + need > s->budget) break;
      std::unique_ptr<Lane> L(new Lane);
      L->req = r;
      L->bytes = need;
      s->used += need;
      Lane* lp = L.get();
      L->th = std::thread(lane_main, s, lp);
      s->lanes.push_back(std::move(L));
      it = s->queue.erase(it);
    }
  }
  // the rest: admitted to the batch in arrival order while the budget and the
  // slots allow (large requests waiting for a lane are passed over)
  for (auto qit = s->queue.begin(); qit != s->queue.end();) {
    auto r = *qit;
    if (r->cancelled) {
      qit = s->queue.erase(qit);
      continue;
    }
    if (use_lanes && r->dim >= s->lane_min_dim) {
      ++qit;
      continue;
    }
    const auto key = std::make_pair(r->model.N, r->model.n_up);
    const size_t need = r->footprint + (s->sectors.count(key) ? 0 : sector_bytes(key.first, key.second));
    if (s->used + need > s->budget) break;
    int k = -1;
    for (int q = 0; q < (int)s->slots.size(); ++q)
      if (!s->slots[q].used) {
        k = q;
        break;
      }
    if (k < 0) break;
    qit = s->queue.erase(qit);
    rc = admit(s, k, r);
    if (rc) {
      r->status = rc;
      r->error = aed_last_error();
      release_slot(s, k);
      continue;
    }
    s->h_inst[k] = s->slots[k].inst;
    s->dirty = true;
  }
  if (s->dirty && (rc = rebuild_items(s))) return rc;
  if ((rc = tune_buckets(s))) return rc;
  if (s->graph_stale && (rc = capture_graph(s))) return rc;
  int resident = 0;
  for (auto& sl : s->slots) resident += sl.used ? 1 : 0;
  if (resident > 0) {
    AED_CUDA_TRY(cudaGraphLaunch(s->graph, s->stream));
    s->launches++;
    const int n_inst = s->h_counts[0];
    AED_CUDA_TRY(cudaMemcpyAsync(s->h_inst.data(), s->d_inst, sizeof(BInst) * n_inst, cudaMemcpyDeviceToHost,
                                 s->stream));
    AED_CUDA_TRY(cudaStreamSynchronize(s->stream));
    for (int k = 0; k < n_inst; ++k) {
      if (!s->slots[k].used) continue;
      s->slots[k].inst = s->h_inst[k];
      if (s->h_inst[k].phase == kPhDone) {
        finish_request(s, k);
        s->dirty = true;
        --resident;
      }
    }
  }
  if (resident == 0 && !s->lanes.empty()) {  // only lanes at work: do not spin the caller
    lk.unlock();
    std::this_thread::sleep_for(std::chrono::microseconds(200));
    lk.lock();
  }
  if (n_pending) *n_pending = resident + (int32_t)s->queue.size() + (int32_t)s->lanes.size();
  return AED_OK;
}

int aed_server_poll(aed_server* s, int64_t ticket, aed_solve_result* out) {
  if (!s || !out) return fail(AED_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->requests.find(ticket);
  if (it == s->requests.end()) return fail(AED_ERR_INVALID, "unknown ticket");
  const int st = it->second->status;
  if (st == AED_PENDING) return AED_PENDING;
  *out = it->second->res;
  const std::string err = it->second->error;
  s->requests.erase(it);
  if (st != AED_OK) return fail(st, err.empty() ? std::string("request failed or was cancelled") : "request failed: " + err);
  return AED_OK;
}

int aed_server_get_stats(aed_server* s, aed_server_stats* out) {
  if (!s || !out) return fail(AED_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  std::memset(out, 0, sizeof *out);
  for (auto& sl : s->slots) out->resident += sl.used ? 1 : 0;
  out->queued = (int32_t)s->queue.size();
  out->bytes_used = (int64_t)s->used;
  out->bytes_budget = (int64_t)s->budget;
  out->graph_launches = s->launches;
  out->lanes = (int32_t)s->lanes.size();
  return AED_OK;
}

}  // extern "C"
