// api.cpp -- the C ABI of libaed.so (declared in include/aed.h).

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>

#include "handle.h"

namespace aed {
const char* last_error_cstr();

// ---- memory of handles ------------------------------------------------------------
namespace {

std::mutex g_mem_mu;
// device blocks not in use, by (device, size); every cached device block's size
std::multimap<std::pair<int, size_t>, void*> g_dev_free;
std::map<void*, std::pair<int, size_t>> g_dev_block;
std::multimap<size_t, void*> g_host_free;  // pinned blocks not in use, by size
std::map<void*, size_t> g_host_size;       // every pinned block of the cache

constexpr size_t kDevRound = (size_t)2 << 20;  // device blocks: multiples of 2 MiB (the driver's own granule)

size_t dev_block_bytes(size_t bytes) {
  if (bytes < kDevRound) return (bytes + 255) & ~(size_t)255;
  return (bytes + kDevRound - 1) & ~(kDevRound - 1);
}
size_t host_block_bytes(size_t bytes) { return (bytes + 4095) & ~(size_t)4095; }

void trim_device(int dev) {  // callers hold g_mem_mu
  for (auto it = g_dev_free.begin(); it != g_dev_free.end();) {
    if (it->first.first == dev) {
      cudaFree(it->second);
      g_dev_block.erase(it->second);
      it = g_dev_free.erase(it);
    } else {
      ++it;
    }
  }
}

}  // namespace

int mem_dev_alloc(void** p, size_t bytes) {
  *p = nullptr;
  int dev = 0;
  AED_CUDA_TRY(cudaGetDevice(&dev));
  const size_t b = dev_block_bytes(bytes ? bytes : 8);
  std::lock_guard<std::mutex> lk(g_mem_mu);
  // the smallest cached block that fits and wastes at most half of itself
  auto it = g_dev_free.lower_bound({dev, b});
  if (it != g_dev_free.end() && it->first.first == dev && it->first.second <= 2 * b) {
    *p = it->second;
    g_dev_free.erase(it);
    return AED_OK;
  }
  cudaError_t e = cudaMalloc(p, b);
  if (e == cudaErrorMemoryAllocation) {  // give the cached blocks back and try once more
    cudaGetLastError();
    trim_device(dev);
    e = cudaMalloc(p, b);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return fail(AED_ERR_NOMEM, std::string("device allocation of ") + std::to_string(bytes) +
                                   " bytes: " + cudaGetErrorString(e));
  }
  g_dev_block[*p] = {dev, b};
  return AED_OK;
}

void mem_dev_free(void* p, cudaStream_t st) {
  if (!p) return;
  cudaStreamSynchronize(st);  // no work queued so far on st uses the block any more
  std::lock_guard<std::mutex> lk(g_mem_mu);
  auto it = g_dev_block.find(p);
  if (it != g_dev_block.end()) g_dev_free.emplace(it->second, p);
}

int mem_host_alloc(void** p, size_t bytes) {
  const size_t b = host_block_bytes(bytes ? bytes : 8);
  {
    std::lock_guard<std::mutex> lk(g_mem_mu);
    auto it = g_host_free.find(b);
    if (it != g_host_free.end()) {
      *p = it->second;
      g_host_free.erase(it);
      return AED_OK;
    }
  }
  if (cudaMallocHost(p, b) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return fail(AED_ERR_NOMEM, "pinned host allocation of " + std::to_string(bytes) + " bytes failed");
  }
  std::lock_guard<std::mutex> lk(g_mem_mu);
  g_host_size[*p] = b;
  return AED_OK;
}

void mem_host_free(void* p) {
  if (!p) return;
  std::lock_guard<std::mutex> lk(g_mem_mu);
  auto it = g_host_size.find(p);
  if (it != g_host_size.end()) g_host_free.emplace(it->second, p);
}

void mem_empty_cache(int device) {
  DeviceGuard g(device);
  std::lock_guard<std::mutex> lk(g_mem_mu);
  trim_device(device);
  for (auto& f : g_host_free) {
    cudaFreeHost(f.second);
    g_host_size.erase(f.second);
  }
  g_host_free.clear();
}

namespace {

template <typename T>
int dev_alloc(T** p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  const cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return fail(AED_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  return AED_OK;
}

void release(aed_handle* h) {
  if (!h) return;
  handle_release_workspace(h);
  for (void* p : {(void*)h->d_thi, (void*)h->d_tlo, (void*)h->d_lolist, (void*)h->d_looff, (void*)h->d_tile_h,
                  (void*)h->d_tile_r, (void*)h->d_blk_h, (void*)h->d_tfirst, (void*)h->d_dg, (void*)h->d_ell,
                  (void*)h->d_xtab, (void*)h->d_partA, (void*)h->d_partB, (void*)h->d_scal, (void*)h->d_flag, (void*)h->d_dgf,
                  (void*)h->d_start64,
                  (void*)h->d_reps, (void*)h->d_norm, (void*)h->d_mdiag, (void*)h->d_map, (void*)h->d_sthi,
                  (void*)h->d_stlo, (void*)h->d_slolist, (void*)h->d_slooff, (void*)h->d_sblk_hi,
                  (void*)h->d_sblk_off, (void*)h->d_stile_blk, (void*)h->d_stile_r, (void*)h->d_sreps,
                  (void*)h->d_slol})
    mem_dev_free(p, h->stream);
  delete h->mp;
  delete h->sp;
  mem_host_free(h->h_scal);
  if (h->stream) {
    cudaStreamSynchronize(h->stream);  // the frees are done: the memory is back in the pool
    cudaStreamDestroy(h->stream);
  }
  delete h;
}

// (Re)build the lo-neighbour table of the handle's couplings on the device.
int upload_lo_table(aed_handle* h) {
  std::vector<uint32_t> ell;
  int W = 0;
  build_lo_table(h->tab, h->P, ell, &W);
  cudaStreamSynchronize(h->stream);  // no apply reads the old table any more
  if (ell.size() + 1 > h->d_ell_n) {  // grow only: new couplings usually keep the width
    mem_dev_free(h->d_ell, h->stream);
    h->d_ell = nullptr;
    h->d_ell_n = 0;
    const int rc = mem_dev_alloc_n(&h->d_ell, ell.size() + 1);
    if (rc) return rc;
    h->d_ell_n = ell.size() + 1;
  }
  if (!ell.empty()) {
    AED_CUDA_TRY(cudaMemcpyAsync(h->d_ell, ell.data(), ell.size() * 4, cudaMemcpyHostToDevice, h->stream));
    AED_CUDA_TRY(cudaStreamSynchronize(h->stream));  // host vector goes out of scope
  }
  h->dt.ell = h->d_ell;
  h->dt.ell_w = W;
  return AED_OK;
}

int check_vec(const aed_handle* h, const void* p, const char* name) {
  if (!h) return fail(AED_ERR_INVALID, "handle is NULL");
  if (!p) return fail(AED_ERR_INVALID, std::string(name) + " is NULL");
  return AED_OK;
}

}  // namespace

int handle_workspace(aed_handle* h, int slot, size_t bytes, void** out) {
  if (bytes > h->ws_bytes[slot]) {
    mem_dev_free(h->ws[slot], h->stream);
    h->ws[slot] = nullptr;
    h->ws_bytes[slot] = 0;
    const int rc = mem_dev_alloc(&h->ws[slot], bytes);
    if (rc) return rc;
    h->ws_bytes[slot] = bytes;
  }
  *out = h->ws[slot];
  return AED_OK;
}

int handle_pinned(aed_handle* h, size_t n, double** out) {
  if (n > h->h_ab_n) {
    if (h->h_ab) {
      cudaStreamSynchronize(h->stream);  // no copy into the old buffer in flight
      mem_host_free(h->h_ab);
    }
    h->h_ab = nullptr;
    h->h_ab_n = 0;
    void* p = nullptr;
    const int rc = mem_host_alloc(&p, n * sizeof(double));
    if (rc) return rc;
    h->h_ab = static_cast<double*>(p);
    h->h_ab_n = n;
  }
  *out = h->h_ab;
  return AED_OK;
}

void* handle_store_chunk(aed_handle* h, int c, size_t chunk_bytes) {
  if (chunk_bytes != h->store_chunk_bytes) {
    for (void* p : h->store_chunks) mem_dev_free(p, h->stream);
    h->store_chunks.clear();
    h->store_chunk_bytes = chunk_bytes;
  }
  while ((int)h->store_chunks.size() <= c) {
    void* p = nullptr;
    if (mem_dev_alloc(&p, chunk_bytes)) {
      fail(AED_ERR_NOMEM, "device memory exhausted by the FP32 Lanczos basis (" +
                              std::to_string(h->store_chunks.size() * kStoreChunk) + " vectors)");
      return nullptr;
    }
    h->store_chunks.push_back(p);
  }
  return h->store_chunks[c];
}

void handle_release_workspace(aed_handle* h) {
  h->rec_live = false;
  for (void* p : h->store_chunks) mem_dev_free(p, h->stream);
  h->store_chunks.clear();
  h->store_chunk_bytes = 0;
  h->store_m = 0;
  h->last_rr = false;
  for (int k = 0; k < aed_handle::kWorkspaces; ++k) {
    mem_dev_free(h->ws[k], h->stream);
    h->ws[k] = nullptr;
    h->ws_bytes[k] = 0;
  }
  if (h->h_ab) {
    cudaStreamSynchronize(h->stream);  // no copy into it in flight
    mem_host_free(h->h_ab);
  }
  h->h_ab = nullptr;
  h->h_ab_n = 0;
}

namespace {

// Returns kVariantNotApplicable (nothing launched) for a variant that does not fit the sector.
int launch_variant(aed_handle* h, bool f32, int v, const void* x, void* y, double* alpha_part) {
  if (f32) return launch_hv_f32(v, h->P, h->dt, (const float*)x, (float*)y, alpha_part, h->stream);
  return launch_hv_f64(v, h->P, h->dt, (const double*)x, (double*)y, alpha_part, h->stream);
}

int launch_checked(aed_handle* h, bool f32, int v, const void* x, void* y, double* alpha_part) {
  const int rc = launch_variant(h, f32, v, x, y, alpha_part);
  if (rc == kVariantNotApplicable)
    return fail(AED_ERR_INVALID, std::string("apply variant ") + hv_variant_name(v) + " does not fit this sector");
  return rc;
}

// Autotuner: the apply variant (rows per thread, ops per group, CTAs per SM)
// is picked by timing every variant on the first apply of a handle, once per
// (precision, size bucket, number of flip pairs); later handles in the same
// bucket reuse the choice.  Results do not depend on the variant (each row
// adds its terms in the same order).  AED_HV_VARIANT=<index> forces one.
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int>, int> g_tune;

int pick_variant(aed_handle* h, bool f32, const void* x, void* y, int* out) {
  if (const char* env = std::getenv("AED_HV_VARIANT")) {
    const int v = std::atoi(env);
    if (v >= 0 && v < hv_num_variants()) {
      *out = v;
      return AED_OK;
    }
  }
  const int64_t D = h->tab.D;
  int bucket = 0;
  while ((1ll << (bucket + 1)) <= D) ++bucket;
  const auto key = std::make_tuple(f32 ? 1 : 0, bucket, h->P.n_pairs);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) {
      *out = it->second;
      return AED_OK;
    }
  }
  if (D < (1 << 12)) {  // tiny sectors: launch-bound, not worth timing (from L = 16 up the
                        // bundle apply's 16 CTAs beat the tile apply's 7: 241 against 214 solves/s)
    *out = 0;
    return AED_OK;
  }
  cudaEvent_t e0, e1;
  AED_CUDA_TRY(cudaEventCreate(&e0));
  AED_CUDA_TRY(cudaEventCreate(&e1));
  int best = 0;
  float best_ms = 1e30f;
  int rc = AED_OK;
  // as solves run them: with the per-tile <x,y> partials; best of three
  for (int v = 0; v < hv_num_variants() && !rc; ++v) {
    if (!hv_variant_tuned(v)) continue;
    rc = launch_variant(h, f32, v, x, y, h->d_partA);  // warm-up
    if (rc == kVariantNotApplicable) {  // does not fit this sector
      rc = AED_OK;
      continue;
    }
    for (int r = 0; r < 3 && !rc; ++r) {
      cudaEventRecord(e0, h->stream);
      rc = launch_variant(h, f32, v, x, y, h->d_partA);
      cudaEventRecord(e1, h->stream);
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms < best_ms) {
        best_ms = ms;
        best = v;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[key] = best;
  }
  if (std::getenv("AED_VERBOSE"))
    std::fprintf(stderr, "[aed] apply %s D=%lld: variant %s (%.3f ms)\n", f32 ? "fp32" : "fp64", (long long)D,
                 hv_variant_name(best), best_ms);
  *out = best;
  return AED_OK;
}

}  // namespace

int handle_tune(aed_handle* h, bool f32, const void* x, void* y) {
  if (h->mom || h->gen) return AED_OK;  // one kernel
  int& v = h->hv_var[f32 ? 1 : 0];
  return v < 0 ? pick_variant(h, f32, x, y, &v) : AED_OK;
}

int handle_hv(aed_handle* h, bool f32, const void* x, void* y, double* alpha_part) {
  if (h->gen && h->mom)
    return launch_spin_mom_hv(*h->sp, *h->mp, h->sdev, h->spin_mom_tables(), (const double*)x, (double*)y,
                              alpha_part, h->stream);
  if (h->gen) return launch_spin_hv(*h->sp, h->sdev, (const double*)x, (double*)y, alpha_part, h->stream);
  if (h->mom)
    return launch_mom_hv(*h->mp, h->dt, h->mom_tables(), (const double*)x, (double*)y, alpha_part, h->stream);
  int rc = handle_tune(h, f32, x, y);
  if (rc) return rc;
  rc = launch_variant(h, f32, h->hv_var[f32 ? 1 : 0], x, y, alpha_part);
  // the tuned variant may not take these vectors (bulk copies need 16-byte
  // aligned x and y): the tile apply takes any, with the same rows and partials
  if (rc == kVariantNotApplicable) rc = launch_checked(h, f32, 0, x, y, alpha_part);
  return rc;
}

int handle_check_flag(aed_handle* h) {
  if (!h->d_flag) return AED_OK;
  uint32_t* hf = reinterpret_cast<uint32_t*>(h->h_scal + 5);
  AED_CUDA_TRY(cudaMemcpyAsync(hf, h->d_flag, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
  AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (*hf == 0u) return AED_OK;
  AED_CUDA_TRY(cudaMemsetAsync(h->d_flag, 0, sizeof(uint32_t), h->stream));
  return fail(AED_ERR_TIMEOUT, "a bounded device wait of the apply gave up; its result is not valid");
}

// Mean CUDA-event time of `reps` applies through handle_hv.
int time_hv(aed_handle* h, const void* x, void* y, int reps, double* alpha_part, double* ms) {
  int rc = AED_OK;
  cudaEvent_t e0, e1;
  AED_CUDA_TRY(cudaEventCreate(&e0));
  AED_CUDA_TRY(cudaEventCreate(&e1));
  cudaEventRecord(e0, h->stream);
  for (int r = 0; r < reps && !rc; ++r) rc = handle_hv(h, h->precision == AED_FP32, x, y, alpha_part);
  cudaEventRecord(e1, h->stream);
  cudaEventSynchronize(e1);
  float t = 0.f;
  cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc || (rc = handle_check_flag(h))) return rc;
  *ms = (double)t / reps;
  return AED_OK;
}

// Off-diagonal terms of the momentum apply: every bond whose spin-flip
// element 0.5 Jxy - 0.25 K is nonzero, in bond order (the flip entry of the
// spin-1/2 bond matrix, as in build_hv_params).
void mom_flips(const Model& m, MomParams& mp) {
  mp.n_flip = 0;
  for (size_t b = 0; b < m.s1.size(); ++b) {
    const double k = m.kq.empty() ? 0.0 : m.kq[b];
    const double c = 0.5 * m.jxy[b] - 0.25 * k;
    if (c == 0.0) continue;
    mp.flip_mask[mp.n_flip] = (1u << (m.N - 1 - m.s1[b])) | (1u << (m.N - 1 - m.s2[b]));
    mp.flip_c[mp.n_flip] = c;
    ++mp.n_flip;
  }
}

}  // namespace aed

using namespace aed;

extern "C" {

const char* aed_last_error(void) { return last_error_cstr(); }

namespace {

// Copy a parse result to the caller's arrays (any of them may be NULL).
int copy_parsed(const ParsedParams& pp, aed_param_info* info, int32_t* s1, int32_t* s2, double* jz, double* jxy,
                double* kq, double* site_h, double* site_d, int32_t bond_capacity, int32_t site_capacity) {
  *info = pp.info;
  const int nb = pp.info.n_bonds;
  if (s1 || s2 || jz || jxy || kq) {
    if (bond_capacity < nb) return fail(AED_ERR_INVALID, "bond_capacity too small");
    for (int b = 0; b < nb; ++b) {
      if (s1) s1[b] = pp.s1[b];
      if (s2) s2[b] = pp.s2[b];
      if (jz) jz[b] = pp.jz[b];
      if (jxy) jxy[b] = pp.jxy[b];
      if (kq) kq[b] = pp.kq[b];
    }
  }
  if (site_h || site_d) {
    if (site_capacity < pp.info.n_sites) return fail(AED_ERR_INVALID, "site_capacity too small");
    for (int s = 0; s < pp.info.n_sites; ++s) {
      if (site_h) site_h[s] = pp.site_h.empty() ? 0.0 : pp.site_h[s];
      if (site_d) site_d[s] = pp.site_d.empty() ? 0.0 : pp.site_d[s];
    }
  }
  return AED_OK;
}

}  // namespace

int aed_parse_parameters(const char* text, aed_param_info* info, int32_t* s1, int32_t* s2, double* jz, double* jxy,
                         double* kq, double* site_h, double* site_d, int32_t bond_capacity, int32_t site_capacity) {
  if (!info) return fail(AED_ERR_INVALID, "info is NULL");
  if (!text) return fail(AED_ERR_INVALID, "text is NULL");
  ParsedParams pp;
  const int rc = parse_parameters(text, pp);
  if (rc) return rc;
  return copy_parsed(pp, info, s1, s2, jz, jxy, kq, site_h, site_d, bond_capacity, site_capacity);
}

int aed_parse_graph_parameters(const char* text, int32_t n_vertices, const int32_t* vertex_type, int32_t n_edges,
                               const int32_t* edge_source, const int32_t* edge_target, const int32_t* edge_type,
                               aed_param_info* info, int32_t* s1, int32_t* s2, double* jz, double* jxy, double* kq,
                               double* site_h, double* site_d, int32_t bond_capacity, int32_t site_capacity) {
  if (!info || !text) return fail(AED_ERR_INVALID, "NULL argument");
  if (n_vertices < 0 || n_edges < 0 || (n_edges > 0 && (!edge_source || !edge_target)))
    return fail(AED_ERR_INVALID, "graph: bad vertex or edge arrays");
  if (n_edges > kMaxBonds) return fail(AED_ERR_INVALID, "too many bonds");
  GraphSpec g;
  g.n = n_vertices;
  g.vtype.assign(n_vertices, 0);
  if (vertex_type)
    for (int i = 0; i < n_vertices; ++i) g.vtype[i] = vertex_type[i];
  for (int e = 0; e < n_edges; ++e) {
    g.src.push_back(edge_source[e]);
    g.tgt.push_back(edge_target[e]);
    g.etype.push_back(edge_type ? edge_type[e] : 0);
  }
  ParsedParams pp;
  const int rc = parse_parameters(text, pp, &g);
  if (rc) return rc;
  return copy_parsed(pp, info, s1, s2, jz, jxy, kq, site_h, site_d, bond_capacity, site_capacity);
}

int aed_create(const aed_model_desc* model, int precision, int device, aed_handle** out) {
  if (!out) return fail(AED_ERR_INVALID, "out is NULL");
  *out = nullptr;
  if (precision != AED_FP64 && precision != AED_FP32) return fail(AED_ERR_INVALID, "precision must be AED_FP64 or AED_FP32");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(AED_ERR_CUDA, "no CUDA device available");
  }
  if (device < 0 || device >= ndev) return fail(AED_ERR_INVALID, "device index out of range");
  DeviceGuard g(device);
  aed_handle* h = new aed_handle;
  h->device = device;
  h->precision = precision;
  int rc = model_from_desc(model, h->model);
  if (!rc) rc = build_tables(h->model.N, h->model.n_up, h->tab);
  if (!rc) rc = build_hv_params(h->model, h->tab.Nlo, h->P);
  if (rc) {
    release(h);
    return rc;
  }
  std::vector<uint32_t> th, tr, tf, blk;
  std::vector<uint16_t> xt;
  int maxrows = 0;
  build_tiles(h->tab, kHvTileRows, th, tr, &tf);
  build_block_list(h->tab, blk, &maxrows);
  build_cross_table(h->tab, xt);
  const size_t nlo = h->tab.tlo.size(), nhi = h->tab.thi.size();
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    release(h);
    return fail(AED_ERR_CUDA, "stream creation failed");
  }
  void* hs = nullptr;
  if ((rc = mem_dev_alloc_n(&h->d_thi, nhi)) || (rc = mem_dev_alloc_n(&h->d_tlo, nlo)) ||
      (rc = mem_dev_alloc_n(&h->d_lolist, nlo)) || (rc = mem_dev_alloc_n(&h->d_looff, h->tab.looff.size())) ||
      (rc = mem_dev_alloc_n(&h->d_tile_h, th.size())) || (rc = mem_dev_alloc_n(&h->d_tile_r, tr.size())) ||
      (rc = mem_dev_alloc_n(&h->d_scal, 8)) || (rc = mem_dev_alloc_n(&h->d_flag, 1)) ||
      (rc = mem_dev_alloc_n(&h->d_blk_h, blk.size() + 1)) ||
      (rc = mem_dev_alloc_n(&h->d_tfirst, tf.size() + 1)) || (rc = mem_dev_alloc_n(&h->d_xtab, xt.size() + 1)) ||
      (rc = mem_dev_alloc_n(&h->d_dg, (size_t)h->tab.D)) || (rc = mem_dev_alloc_n(&h->d_partA, th.size() + 1)) ||
      (rc = mem_dev_alloc_n(&h->d_partB, (size_t)red_chunks(h->tab.D) + 1)) ||
      (rc = mem_host_alloc(&hs, 8 * sizeof(double)))) {
    release(h);
    return rc;
  }
  h->h_scal = static_cast<double*>(hs);
  cudaMemcpyAsync(h->d_thi, h->tab.thi.data(), nhi * 4, cudaMemcpyHostToDevice, h->stream);
  cudaMemcpyAsync(h->d_tlo, h->tab.tlo.data(), nlo * 2, cudaMemcpyHostToDevice, h->stream);
  cudaMemcpyAsync(h->d_lolist, h->tab.lolist.data(), nlo * 2, cudaMemcpyHostToDevice, h->stream);
  cudaMemcpyAsync(h->d_looff, h->tab.looff.data(), h->tab.looff.size() * 4, cudaMemcpyHostToDevice, h->stream);
  if (!th.empty()) {
    cudaMemcpyAsync(h->d_tile_h, th.data(), th.size() * 4, cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(h->d_tile_r, tr.data(), tr.size() * 4, cudaMemcpyHostToDevice, h->stream);
  }
  if (!blk.empty()) cudaMemcpyAsync(h->d_blk_h, blk.data(), blk.size() * 4, cudaMemcpyHostToDevice, h->stream);
  if (!tf.empty()) cudaMemcpyAsync(h->d_tfirst, tf.data(), tf.size() * 4, cudaMemcpyHostToDevice, h->stream);
  if (!xt.empty()) cudaMemcpyAsync(h->d_xtab, xt.data(), xt.size() * 2, cudaMemcpyHostToDevice, h->stream);
  cudaMemsetAsync(h->d_flag, 0, sizeof(uint32_t), h->stream);
  const cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    release(h);
    return fail(AED_ERR_CUDA, std::string("table upload: ") + cudaGetErrorString(e));
  }
  DevTables& t = h->dt;
  t.thi = h->d_thi;
  t.tlo = h->d_tlo;
  t.lolist = h->d_lolist;
  t.looff = h->d_looff;
  t.tile_h = h->d_tile_h;
  t.tile_r = h->d_tile_r;
  t.n_tiles = (int64_t)th.size();
  t.xtab = h->d_xtab;
  t.blk_h = h->d_blk_h;
  t.tfirst = h->d_tfirst;
  t.n_blk = (int64_t)blk.size();
  t.maxrows = maxrows;
  t.D = h->tab.D;
  t.Nlo = h->tab.Nlo;
  t.Nhi = h->tab.Nhi;
  t.n_up = h->tab.n_up;
  t.dg = h->d_dg;
  t.flag = h->d_flag;
  if ((rc = upload_lo_table(h))) {
    release(h);
    return rc;
  }
  rc = launch_diag_table(h->P, t, h->d_dg, h->stream);
  if (!rc && precision == AED_FP32) {  // the FP32 applies read the diagonal rounded to FP32
    rc = mem_dev_alloc_n(&h->d_dgf, (size_t)h->tab.D);
    if (!rc) rc = launch_round_to_f32(h->d_dg, h->d_dgf, h->tab.D, h->stream);
    t.dgf = h->d_dgf;
  }
  const cudaError_t e2 = rc ? cudaSuccess : cudaStreamSynchronize(h->stream);
  if (rc || e2 != cudaSuccess) {
    release(h);
    return rc ? rc : fail(AED_ERR_CUDA, std::string("diagonal table: ") + cudaGetErrorString(e2));
  }
  h->dim = h->vlen = h->tab.D;
  *out = h;
  return AED_OK;
}

namespace {
int translation_invariant(const Model& m, int n_trans, const int* maps);
}  // namespace

namespace {

// Check the translations of a momentum sector (permutations of the N sites,
// the identity first) and fill the phases and destinations of mp.
int momentum_params(int N, const aed_translations* tr, MomParams& mp) {
  if (tr->n_trans < 1 || tr->n_trans > kMaxTrans) return fail(AED_ERR_INVALID, "n_trans must be in 1..62");
  if (!tr->site_map || !tr->phase) return fail(AED_ERR_INVALID, "translations: NULL site_map or phase");
  if (N < 1 || N > 32) return fail(AED_ERR_INVALID, "number of sites must be in 1..32");
  for (int t = 0; t < tr->n_trans; ++t) {
    uint32_t seen = 0;
    for (int i = 0; i < N; ++i) {
      const int j = tr->site_map[(size_t)t * N + i];
      if (j < 0 || j >= N || (seen >> j & 1u)) return fail(AED_ERR_INVALID, "translation is not a permutation of the sites");
      if (t == 0 && j != i) return fail(AED_ERR_INVALID, "the first translation must be the identity");
      seen |= 1u << j;
    }
  }
  mp.N = N;
  mp.n_trans = tr->n_trans;
  mp.inv_sqrt_n = 1.0 / std::sqrt((double)N);
  for (int t = 0; t < tr->n_trans; ++t) {
    mp.phase_re[t] = tr->phase[2 * t];
    mp.phase_im[t] = tr->phase[2 * t + 1];
    for (int i = 0; i < N; ++i) mp.dst[t][i] = (uint8_t)(N - 1 - tr->site_map[(size_t)t * N + i]);
  }
  return AED_OK;
}

}  // namespace

int aed_create_momentum(const aed_model_desc* model, const aed_translations* tr, int device, aed_handle** out) {
  if (!out || !model || !tr) return fail(AED_ERR_INVALID, "NULL argument");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(AED_ERR_CUDA, "no CUDA device available");
  }
  if (device < 0 || device >= ndev) return fail(AED_ERR_INVALID, "device index out of range");
  const int N = model->n_sites;
  std::unique_ptr<MomParams> mpp(new MomParams());
  {
    const int rc0 = momentum_params(N, tr, *mpp);
    if (rc0) return rc0;
  }
  {
    Model m;
    int rc0 = model_from_desc(model, m);
    if (rc0) return rc0;
    std::vector<int> maps(tr->site_map, tr->site_map + (size_t)tr->n_trans * N);
    if ((rc0 = translation_invariant(m, tr->n_trans, maps.data()))) return rc0;
  }
  DeviceGuard g(device);
  aed_handle* h = new aed_handle;
  h->device = device;
  h->precision = AED_FP64;
  h->mom = true;
  int rc = model_from_desc(model, h->model);
  if (!rc) rc = build_tables(h->model.N, h->model.n_up, h->tab);
  if (!rc) rc = build_hv_params(h->model, h->tab.Nlo, h->P);
  if (rc) {
    release(h);
    return rc;
  }
  MomParams* mp = mpp.release();
  h->mp = mp;
  mom_flips(h->model, *mp);
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    release(h);
    return fail(AED_ERR_CUDA, "stream creation failed");
  }
  const size_t nlo = h->tab.tlo.size(), nhi = h->tab.thi.size();
  void* hs = nullptr;
  if ((rc = mem_dev_alloc_n(&h->d_thi, nhi)) || (rc = mem_dev_alloc_n(&h->d_tlo, nlo)) ||
      (rc = mem_dev_alloc_n(&h->d_lolist, nlo)) || (rc = mem_dev_alloc_n(&h->d_looff, h->tab.looff.size())) ||
      (rc = mem_dev_alloc_n(&h->d_scal, 8)) || (rc = mem_host_alloc(&hs, 8 * sizeof(double)))) {
    release(h);
    return rc;
  }
  h->h_scal = static_cast<double*>(hs);
  cudaMemcpyAsync(h->d_thi, h->tab.thi.data(), nhi * 4, cudaMemcpyHostToDevice, h->stream);
  cudaMemcpyAsync(h->d_tlo, h->tab.tlo.data(), nlo * 2, cudaMemcpyHostToDevice, h->stream);
  cudaMemcpyAsync(h->d_lolist, h->tab.lolist.data(), nlo * 2, cudaMemcpyHostToDevice, h->stream);
  cudaMemcpyAsync(h->d_looff, h->tab.looff.data(), h->tab.looff.size() * 4, cudaMemcpyHostToDevice, h->stream);
  const cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    release(h);
    return fail(AED_ERR_CUDA, std::string("table upload: ") + cudaGetErrorString(e));
  }
  DevTables& t = h->dt;
  t = DevTables{};
  t.thi = h->d_thi;
  t.tlo = h->d_tlo;
  t.lolist = h->d_lolist;
  t.looff = h->d_looff;
  t.D = h->tab.D;
  t.Nlo = h->tab.Nlo;
  t.Nhi = h->tab.Nhi;
  t.n_up = h->tab.n_up;
  int64_t dim = 0;
  if ((rc = mom_build(*mp, h->P, t, h->stream, &h->d_reps, &h->d_norm, &h->d_mdiag, &h->d_map, &dim))) {
    release(h);
    return rc;
  }
  h->dim = dim;
  h->vlen = 2 * dim;
  if ((rc = mem_dev_alloc_n(&h->d_partA, (size_t)mom_tiles(dim) + 1)) ||
      (rc = mem_dev_alloc_n(&h->d_partB, (size_t)red_chunks(h->vlen) + 1))) {
    release(h);
    return rc;
  }
  *out = h;
  return AED_OK;
}

namespace {

// The Bloch basis needs H to commute with every translation (the reference
// offers no translations on inhomogeneous lattices, graph_helper.h:585-607).
// maps: n_trans x N, site i -> maps[t * N + i].
int translation_invariant(const Model& m, int n_trans, const int* maps) {
  const int N = m.N;
  std::map<std::pair<int, int>, std::tuple<double, double, double>> bond;
  for (size_t b = 0; b < m.s1.size(); ++b) {
    auto key = std::minmax(m.s1[b], m.s2[b]);
    auto& v = bond[{key.first, key.second}];
    std::get<0>(v) += m.jz[b];
    std::get<1>(v) += m.jxy[b];
    std::get<2>(v) += m.kq[b];
  }
  for (int t = 1; t < n_trans; ++t) {
    const int* mp = maps + (size_t)t * N;
    for (const auto& e : bond) {
      auto key = std::minmax(mp[e.first.first], mp[e.first.second]);
      auto it = bond.find({key.first, key.second});
      if (it == bond.end() || it->second != e.second)
        return fail(AED_ERR_INVALID, "the couplings are not invariant under the translations");
    }
    for (int i = 0; i < N; ++i)
      if ((!m.site_h.empty() && m.site_h[mp[i]] != m.site_h[i]) ||
          (!m.site_d.empty() && m.site_d[mp[i]] != m.site_d[i]))
        return fail(AED_ERR_INVALID, "the site terms are not invariant under the translations");
  }
  return AED_OK;
}

// Site terms and bonds of a spin-S handle's parameters.
void spin_couplings(const Model& m, SpinParams& p) {
  spin_set_couplings(m.s1, m.s2, m.jz, m.jxy, m.kq, m.site_h, m.site_d, m.N, p);
}

// The lo table of a spin-S Sz-sector handle for its current couplings (none
// for a momentum sector, whose apply walks representatives, or a form
// without one); filled on the handle's stream and waited for.
int spin_lo_table(aed_handle* h) {
  SpinDev& t = h->sdev;
  size_t bytes = h->mom ? 0 : spin_lo_table_bytes(*h->sp, t);
  if (bytes > (size_t(1) << 30)) bytes = 0;  // a bond list this long walks the lo words instead
  t.lol = nullptr;
  if (bytes == 0) return AED_OK;
  if (bytes > h->slol_bytes) {
    mem_dev_free(h->d_slol, h->stream);
    h->d_slol = nullptr;
    h->slol_bytes = 0;
    if (int rc = mem_dev_alloc_n(&h->d_slol, bytes / sizeof(uint2))) return rc;
    h->slol_bytes = bytes;
  }
  if (int rc = launch_spin_lo_table(*h->sp, t, h->d_slol, h->stream)) return rc;
  AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
  t.lol = h->d_slol;
  return AED_OK;
}

}  // namespace

int aed_create_spin(const aed_model_desc* model, int32_t two_s, int device, aed_handle** out) {
  if (!out || !model) return fail(AED_ERR_INVALID, "NULL argument");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(AED_ERR_CUDA, "no CUDA device available");
  }
  if (device < 0 || device >= ndev) return fail(AED_ERR_INVALID, "device index out of range");
  if (two_s < 1 || two_s + 1 > kSpinMaxDim) return fail(AED_ERR_INVALID, "two_s must be in 1..4 (S = 1/2 .. 2)");
  aed_model_desc md = *model;
  md.n_up = 0;  // the digit sum is checked against the sector below
  DeviceGuard g(device);
  aed_handle* h = new aed_handle;
  h->device = device;
  h->precision = AED_FP64;
  h->gen = true;
  h->two_s = two_s;
  int rc = model_from_desc(&md, h->model);
  if (rc) {
    release(h);
    return rc;
  }
  h->model.n_up = model->n_up;
  SpinTables tb;
  if ((rc = build_spin_tables(h->model.N, two_s, model->n_up, tb))) {
    release(h);
    return rc;
  }
  h->sp = new SpinParams();
  spin_transitions(two_s, *h->sp);
  spin_couplings(h->model, *h->sp);
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    release(h);
    return fail(AED_ERR_CUDA, "stream creation failed");
  }
  struct Up {
    uint32_t** d;
    const std::vector<uint32_t>* v;
  } ups[] = {{&h->d_sthi, &tb.thi},         {&h->d_stlo, &tb.tlo},         {&h->d_slolist, &tb.lolist},
             {&h->d_slooff, &tb.looff},     {&h->d_sblk_hi, &tb.blk_hi},   {&h->d_sblk_off, &tb.blk_off},
             {&h->d_stile_blk, &tb.tile_blk}, {&h->d_stile_r, &tb.tile_r}};
  for (auto& u : ups) {
    if ((rc = mem_dev_alloc_n(u.d, u.v->size() + 1))) {
      release(h);
      return rc;
    }
    if (!u.v->empty())
      cudaMemcpyAsync(*u.d, u.v->data(), u.v->size() * 4, cudaMemcpyHostToDevice, h->stream);
  }
  const int64_t D = tb.D;
  void* hs = nullptr;
  if ((rc = mem_dev_alloc_n(&h->d_partA, tb.tile_blk.size() + 1)) ||
      (rc = mem_dev_alloc_n(&h->d_partB, (size_t)red_chunks(D) + 1)) || (rc = mem_dev_alloc_n(&h->d_scal, 8)) ||
      (rc = mem_host_alloc(&hs, 8 * sizeof(double)))) {
    release(h);
    return rc;
  }
  h->h_scal = static_cast<double*>(hs);
  const cudaError_t e = cudaStreamSynchronize(h->stream);  // host tables go out of scope
  if (e != cudaSuccess) {
    release(h);
    return fail(AED_ERR_CUDA, std::string("table upload: ") + cudaGetErrorString(e));
  }
  SpinDev& t = h->sdev;
  t.thi = h->d_sthi;
  t.tlo = h->d_stlo;
  t.lolist = h->d_slolist;
  t.looff = h->d_slooff;
  t.blk_hi = h->d_sblk_hi;
  t.blk_off = h->d_sblk_off;
  t.tile_blk = h->d_stile_blk;
  t.tile_r = h->d_stile_r;
  t.D = D;
  t.n_blk = (int64_t)tb.blk_hi.size();
  t.n_tiles = (int64_t)tb.tile_blk.size();
  t.N = tb.N;
  t.bits = tb.bits;
  t.Nl = tb.Nl;
  t.d = tb.d;
  t.T = tb.T;
  t.n_lo = (int64_t)tb.lolist.size();
  h->dim = h->vlen = D;
  if ((rc = spin_lo_table(h))) {
    release(h);
    return rc;
  }
  *out = h;
  return AED_OK;
}

int aed_create_spin_momentum(const aed_model_desc* model, int32_t two_s, const aed_translations* tr, int device,
                             aed_handle** out) {
  if (!out || !model || !tr) return fail(AED_ERR_INVALID, "NULL argument");
  *out = nullptr;
  std::unique_ptr<MomParams> mpp(new MomParams());
  int rc = momentum_params(model->n_sites, tr, *mpp);
  if (rc) return rc;
  aed_handle* h = nullptr;
  if ((rc = aed_create_spin(model, two_s, device, &h))) return rc;
  {
    std::vector<int> maps(tr->site_map, tr->site_map + (size_t)tr->n_trans * model->n_sites);
    if ((rc = translation_invariant(h->model, tr->n_trans, maps.data()))) {
      aed_destroy(h);
      return rc;
    }
  }
  DeviceGuard g(device);
  h->mom = true;
  h->mp = mpp.release();
  h->sdev.lol = nullptr;  // the momentum apply walks representatives, not tiles
  mem_dev_free(h->d_slol, h->stream);
  h->d_slol = nullptr;
  h->slol_bytes = 0;
  // the Sz sector's partial-sum arrays give way to the momentum sector's
  mem_dev_free(h->d_partA, h->stream);
  mem_dev_free(h->d_partB, h->stream);
  h->d_partA = h->d_partB = nullptr;
  int64_t dim = 0;
  if ((rc = spin_mom_build(*h->mp, h->sdev, h->stream, &h->d_sreps, &h->d_norm, &h->d_map, &dim))) {
    release(h);
    return rc;
  }
  h->dim = dim;
  h->vlen = 2 * dim;
  if ((rc = mem_dev_alloc_n(&h->d_partA, (size_t)mom_tiles(dim) + 1)) ||
      (rc = mem_dev_alloc_n(&h->d_partB, (size_t)red_chunks(h->vlen) + 1))) {
    release(h);
    return rc;
  }
  *out = h;
  return AED_OK;
}

int aed_spin_basis(aed_handle* h, uint64_t* states, int64_t offset, int64_t count) {
  if (!h || (!states && count > 0)) return fail(AED_ERR_INVALID, "NULL argument");
  if (!h->gen) return fail(AED_ERR_INVALID, "aed_spin_basis: not a spin-S sector (aed_create_spin)");
  if (offset < 0 || count < 0 || offset + count > h->dim) return fail(AED_ERR_INVALID, "range outside the basis");
  if (count == 0) return AED_OK;
  DeviceGuard g(h->device);
  if (h->mom) {  // the representatives of a momentum sector
    AED_CUDA_TRY(cudaMemcpyAsync(states, h->d_sreps + offset, (size_t)count * 8, cudaMemcpyDeviceToHost, h->stream));
    AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return AED_OK;
  }
  uint64_t* d = nullptr;
  int rc = mem_dev_alloc_n(&d, (size_t)count);
  if (rc) return rc;
  rc = launch_spin_basis(h->sdev, d, offset, count, h->stream);
  if (!rc) {
    cudaMemcpyAsync(states, d, (size_t)count * 8, cudaMemcpyDeviceToHost, h->stream);
    const cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) rc = fail(AED_ERR_CUDA, std::string("basis copy: ") + cudaGetErrorString(e));
  }
  mem_dev_free(d, h->stream);
  return rc;
}

int aed_momentum_basis(aed_handle* h, uint32_t* states, double* norms, int64_t offset, int64_t count) {
  if (!h) return fail(AED_ERR_INVALID, "handle is NULL");
  if (!h->mom) return fail(AED_ERR_INVALID, "aed_momentum_basis: not a momentum sector");
  if (h->gen && states)
    return fail(AED_ERR_INVALID, "aed_momentum_basis: spin-S representatives are 64-bit (aed_spin_basis)");
  if (offset < 0 || count < 0 || offset + count > h->dim) return fail(AED_ERR_INVALID, "range outside the basis");
  if (count == 0) return AED_OK;
  DeviceGuard g(h->device);
  if (states)
    AED_CUDA_TRY(cudaMemcpyAsync(states, h->d_reps + offset, (size_t)count * 4, cudaMemcpyDeviceToHost, h->stream));
  if (norms)
    AED_CUDA_TRY(cudaMemcpyAsync(norms, h->d_norm + offset, (size_t)count * 8, cudaMemcpyDeviceToHost, h->stream));
  AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return AED_OK;
}

int aed_lattice_momenta(const char* params, int32_t* n_momenta, int32_t* n_dirs, double* k, int32_t capacity) {
  if (!params || !n_momenta || !n_dirs) return fail(AED_ERR_INVALID, "NULL argument");
  std::vector<std::vector<double>> ks;
  int nd = 0;
  const int rc = lattice_momenta(params, &nd, ks);
  if (rc) return rc;
  *n_momenta = (int32_t)ks.size();
  *n_dirs = nd;
  if (k) {
    if (capacity < (int32_t)ks.size()) return fail(AED_ERR_INVALID, "capacity too small");
    for (size_t m = 0; m < ks.size(); ++m)
      for (int d = 0; d < nd; ++d) k[m * nd + d] = ks[m][d];
  }
  return AED_OK;
}

int aed_lattice_translations(const char* params, const double* k, int32_t n_dirs, int32_t* n_trans, int32_t* n_sites,
                             int32_t* site_map, double* phase, int32_t capacity) {
  if (!params || !n_trans || !n_sites || (n_dirs > 0 && !k)) return fail(AED_ERR_INVALID, "NULL argument");
  std::vector<int> maps;
  std::vector<double> re, im;
  int ns = 0;
  const int rc = lattice_translations(params, k, n_dirs, &ns, maps, re, im);
  if (rc) return rc;
  *n_trans = (int32_t)re.size();
  *n_sites = ns;
  if (site_map || phase) {
    if (capacity < (int32_t)re.size()) return fail(AED_ERR_INVALID, "capacity too small");
    for (size_t t = 0; t < re.size(); ++t) {
      if (phase) {
        phase[2 * t] = re[t];
        phase[2 * t + 1] = im[t];
      }
      if (site_map)
        for (int i = 0; i < ns; ++i) site_map[t * ns + i] = maps[t * ns + i];
    }
  }
  return AED_OK;
}

int aed_momentum_expectation(aed_handle* h, const void* psi, int32_t kind, int32_t n, const int32_t* site_i,
                             const int32_t* site_j, double* out) {
  if (!h || !psi || !out || (n > 0 && (!site_i || (kind != AED_OBS_SZ && !site_j))))
    return fail(AED_ERR_INVALID, "NULL argument");
  if (!h->mom) return fail(AED_ERR_INVALID, "aed_momentum_expectation: not a momentum sector");
  if (kind < AED_OBS_SZ || kind > AED_OBS_SPSM) return fail(AED_ERR_INVALID, "unknown observable kind");
  const int N = h->model.N;
  for (int p = 0; p < n; ++p)
    if (site_i[p] < 0 || site_i[p] >= N || (kind != AED_OBS_SZ && (site_j[p] < 0 || site_j[p] >= N)))
      return fail(AED_ERR_INVALID, "site index out of range");
  *out = 0.0;
  if (n <= 0 || h->dim == 0) return AED_OK;
  DeviceGuard g(h->device);
  if (h->gen) return spin_mom_expectation(h, static_cast<const double*>(psi), kind, n, site_i, site_j, out);
  const int grid = mom_expect_grid(h->dim);
  void* w = nullptr;
  int rc = handle_workspace(h, 1, (size_t)grid * 8, &w);
  if (rc) return rc;
  std::vector<double> hp((size_t)grid);
  double total = 0.0;
  for (int p0 = 0; p0 < n; p0 += kMomPairs) {
    MomPairs pairs{};
    pairs.n = std::min(kMomPairs, n - p0);
    for (int p = 0; p < pairs.n; ++p) {
      pairs.mi[p] = 1u << (N - 1 - site_i[p0 + p]);
      pairs.mj[p] = kind == AED_OBS_SZ ? 0u : 1u << (N - 1 - site_j[p0 + p]);
    }
    if ((rc = mom_expectation(*h->mp, h->dt, h->mom_tables(), (const double*)psi, kind, pairs, (double*)w, grid,
                              h->stream)))
      return rc;
    AED_CUDA_TRY(cudaMemcpyAsync(hp.data(), w, hp.size() * 8, cudaMemcpyDeviceToHost, h->stream));
    AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (double v : hp) total += v;
  }
  *out = total;
  return AED_OK;
}

int aed_expectation(aed_handle* h, const void* psi, int32_t kind, int32_t n, const int32_t* site_i,
                    const int32_t* site_j, double* out) {
  if (!h || !psi || (n > 0 && (!site_i || !out || (kind != AED_OBS_SZ && !site_j))))
    return fail(AED_ERR_INVALID, "NULL argument");
  if (h->mom) return fail(AED_ERR_INVALID, "aed_expectation: Sz sectors only (aed_momentum_expectation)");
  if (kind < AED_OBS_SZ || kind > AED_OBS_SPSM) return fail(AED_ERR_INVALID, "unknown observable kind");
  const int N = h->model.N;
  for (int p = 0; p < n; ++p)
    if (site_i[p] < 0 || site_i[p] >= N || (kind != AED_OBS_SZ && (site_j[p] < 0 || site_j[p] >= N)))
      return fail(AED_ERR_INVALID, "site index out of range");
  if (n <= 0) return AED_OK;
  DeviceGuard g(h->device);
  if (h->gen) return spin_measure_pairs(h, static_cast<const double*>(psi), kind, n, site_i, site_j, out);
  return measure_pairs(h, psi, kind, n, site_i, site_j, out);
}

int aed_lattice_geometry(const char* params, int32_t* dim, int32_t* extent, int32_t* periodic) {
  if (!params || !dim || !extent || !periodic) return fail(AED_ERR_INVALID, "NULL argument");
  int d = 0, ext[2] = {1, 1}, per[2] = {0, 0};
  const int rc = lattice_geometry(params, &d, ext, per);
  if (rc) return rc;
  *dim = d;
  for (int i = 0; i < d; ++i) {
    extent[i] = ext[i];
    periodic[i] = per[i];
  }
  return AED_OK;
}

int aed_set_couplings(aed_handle* h, const aed_model_desc* model) {
  if (!h || !model) return fail(AED_ERR_INVALID, "NULL argument");
  if (model->n_sites != h->model.N || model->n_up != h->model.n_up)
    return fail(AED_ERR_INVALID, "aed_set_couplings: the sector (n_sites, n_up) must stay the same");
  Model m;
  aed_model_desc md = *model;
  if (h->gen) md.n_up = 0;  // a spin-S digit sum may exceed n_sites
  int rc = model_from_desc(&md, m);
  if (rc) return rc;
  m.n_up = model->n_up;
  HvParams P;
  if (!h->gen && (rc = build_hv_params(m, h->tab.Nlo, P))) return rc;
  if (h->mom) {  // the new couplings must keep the translations a symmetry
    std::vector<int> maps((size_t)h->mp->n_trans * m.N);
    for (int t = 0; t < h->mp->n_trans; ++t)
      for (int i = 0; i < m.N; ++i) maps[(size_t)t * m.N + i] = m.N - 1 - h->mp->dst[t][i];
    if ((rc = translation_invariant(m, h->mp->n_trans, maps.data()))) return rc;
  }
  DeviceGuard g(h->device);
  AED_CUDA_TRY(cudaStreamSynchronize(h->stream));  // no apply of the old couplings in flight
  h->model = m;
  h->P = P;
  // the recurrence of the last solve belongs to the old Hamiltonian
  h->last_alpha.clear();
  h->last_beta.clear();
  h->rec_m = 0;
  h->rec_live = false;
  if (h->gen) {  // same sector: new site terms and bonds
    spin_couplings(h->model, *h->sp);
    return spin_lo_table(h);
  }
  if (h->mom) {  // same basis and translations: new flip list and diagonal
    mom_flips(h->model, *h->mp);
    if ((rc = launch_mom_diag(h->P, h->d_reps, h->dim, h->d_mdiag, h->stream))) return rc;
    AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return AED_OK;
  }
  if ((rc = upload_lo_table(h))) return rc;
  rc = launch_diag_table(h->P, h->dt, h->d_dg, h->stream);
  if (!rc && h->d_dgf) rc = launch_round_to_f32(h->d_dg, h->d_dgf, h->tab.D, h->stream);
  if (rc) return rc;
  AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return AED_OK;
}

int aed_destroy(aed_handle* h) {
  if (!h) return AED_OK;
  DeviceGuard g(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  release(h);
  return AED_OK;
}

int aed_reserve_basis(aed_handle* h, int32_t vectors) {
  if (!h) return fail(AED_ERR_INVALID, "NULL handle");
  if (h->precision != AED_FP32 || h->mom || h->gen)
    return fail(AED_ERR_INVALID, "aed_reserve_basis: only mixed-precision spin-1/2 Sz-sector handles keep a basis");
  if (vectors < 0 || vectors > kMaxRitzTerms) return fail(AED_ERR_INVALID, "aed_reserve_basis: vectors out of range");
  DeviceGuard g(h->device);
  const size_t cb = store_chunk_bytes_of(h->vlen);
  for (int c = 0; c * kStoreChunk < vectors; ++c)
    if (!handle_store_chunk(h, c, cb)) return AED_ERR_NOMEM;
  // and the Rayleigh-Ritz step's workspace for the most Ritz vectors it takes
  void* ws = nullptr;
  return vectors > 0 ? handle_workspace(h, 2, rr_workspace_bytes(h->vlen, kMaxRR), &ws) : AED_OK;
}

int aed_empty_cache(int device) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return fail(AED_ERR_INVALID, "device index out of range");
  }
  mem_empty_cache(device);
  return AED_OK;
}

int aed_dimension(const aed_handle* h, int64_t* dim) {
  if (!h || !dim) return fail(AED_ERR_INVALID, "NULL argument");
  *dim = h->dim;
  return AED_OK;
}

int aed_basis_copy(aed_handle* h, uint32_t* host_out, int64_t offset, int64_t count) {
  if (!h || (!host_out && count > 0)) return fail(AED_ERR_INVALID, "NULL argument");
  if (offset < 0 || count < 0 || offset + count > h->dim) return fail(AED_ERR_INVALID, "range outside the basis");
  if (count == 0) return AED_OK;
  DeviceGuard g(h->device);
  if (h->mom) return aed_momentum_basis(h, host_out, nullptr, offset, count);
  if (h->gen) return fail(AED_ERR_INVALID, "aed_basis_copy: spin-S states are 64-bit (aed_spin_basis)");
  uint32_t* d = nullptr;
  int rc = dev_alloc(&d, (size_t)count);
  if (rc) return rc;
  rc = launch_basis_copy(h->dt, d, offset, count, h->stream);
  if (!rc) {
    cudaMemcpyAsync(host_out, d, count * 4, cudaMemcpyDeviceToHost, h->stream);
    const cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) rc = fail(AED_ERR_CUDA, std::string("basis copy: ") + cudaGetErrorString(e));
  }
  cudaFree(d);
  return rc;
}

int aed_basis_state(aed_handle* h, int64_t idx, uint64_t* state) {
  if (!h || !state) return fail(AED_ERR_INVALID, "NULL argument");
  if (idx < 0 || idx >= h->dim) return fail(AED_ERR_INVALID, "index outside the basis");
  if (h->gen) return aed_spin_basis(h, state, idx, 1);
  uint32_t s = 0;
  const int rc = aed_basis_copy(h, &s, idx, 1);
  if (!rc) *state = s;
  return rc;
}

int aed_index(aed_handle* h, const uint32_t* host_states, int64_t count, int64_t* host_idx) {
  if (!h || ((!host_states || !host_idx) && count > 0)) return fail(AED_ERR_INVALID, "NULL argument");
  if (h->mom || h->gen) return fail(AED_ERR_INVALID, "aed_index: spin-1/2 Sz sectors only");
  if (count <= 0) return AED_OK;
  DeviceGuard g(h->device);
  uint32_t* ds = nullptr;
  int64_t* di = nullptr;
  int rc = dev_alloc(&ds, (size_t)count);
  if (!rc) rc = dev_alloc(&di, (size_t)count);
  if (!rc) {
    cudaMemcpyAsync(ds, host_states, count * 4, cudaMemcpyHostToDevice, h->stream);
    rc = launch_rank(h->dt, h->model.N, ds, count, di, h->stream);
    if (!rc) {
      cudaMemcpyAsync(host_idx, di, count * 8, cudaMemcpyDeviceToHost, h->stream);
      const cudaError_t e = cudaStreamSynchronize(h->stream);
      if (e != cudaSuccess) rc = fail(AED_ERR_CUDA, std::string("index: ") + cudaGetErrorString(e));
    }
  }
  cudaFree(ds);
  cudaFree(di);
  return rc;
}

int aed_vec_alloc(aed_handle* h, void** v) {
  if (!h || !v) return fail(AED_ERR_INVALID, "NULL argument");
  DeviceGuard g(h->device);
  const size_t bytes = (size_t)h->vlen * h->elem_size();
  const cudaError_t e = cudaMalloc(v, bytes ? bytes : 8);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *v = nullptr;
    return fail(AED_ERR_NOMEM, std::string("vector allocation: ") + cudaGetErrorString(e));
  }
  AED_CUDA_TRY(cudaMemsetAsync(*v, 0, bytes, h->stream));
  AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return AED_OK;
}

int aed_vec_free(aed_handle* h, void* v) {
  if (!h) return fail(AED_ERR_INVALID, "handle is NULL");
  DeviceGuard g(h->device);
  cudaStreamSynchronize(h->stream);
  AED_CUDA_TRY(cudaFree(v));
  return AED_OK;
}

int aed_vec_upload(aed_handle* h, void* v, const double* host) {
  int rc = check_vec(h, v, "vector");
  if (rc) return rc;
  if (!host) return fail(AED_ERR_INVALID, "host is NULL");
  DeviceGuard g(h->device);
  const int64_t D = h->vlen;
  if (h->precision == AED_FP64) {
    AED_CUDA_TRY(cudaMemcpyAsync(v, host, D * 8, cudaMemcpyHostToDevice, h->stream));
  } else {
    std::vector<float> tmp(D);
    for (int64_t i = 0; i < D; ++i) tmp[i] = (float)host[i];
    AED_CUDA_TRY(cudaMemcpyAsync(v, tmp.data(), D * 4, cudaMemcpyHostToDevice, h->stream));
    AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
  }
  AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return AED_OK;
}

int aed_vec_download(aed_handle* h, const void* v, double* host) {
  int rc = check_vec(h, v, "vector");
  if (rc) return rc;
  if (!host) return fail(AED_ERR_INVALID, "host is NULL");
  DeviceGuard g(h->device);
  const int64_t D = h->vlen;
  if (h->precision == AED_FP64) {
    AED_CUDA_TRY(cudaMemcpyAsync(host, v, D * 8, cudaMemcpyDeviceToHost, h->stream));
    AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
  } else {
    std::vector<float> tmp(D);
    AED_CUDA_TRY(cudaMemcpyAsync(tmp.data(), v, D * 4, cudaMemcpyDeviceToHost, h->stream));
    AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (int64_t i = 0; i < D; ++i) host[i] = tmp[i];
  }
  return AED_OK;
}

int aed_vec_copy(aed_handle* h, const void* x, void* y) {
  int rc = check_vec(h, x, "x");
  if (!rc) rc = check_vec(h, y, "y");
  if (rc) return rc;
  DeviceGuard g(h->device);
  AED_CUDA_TRY(cudaMemcpyAsync(y, x, h->vlen * h->elem_size(), cudaMemcpyDeviceToDevice, h->stream));
  return AED_OK;
}

int aed_vec_clear(aed_handle* h, void* x) {
  int rc = check_vec(h, x, "x");
  if (rc) return rc;
  DeviceGuard g(h->device);
  AED_CUDA_TRY(cudaMemsetAsync(x, 0, h->vlen * h->elem_size(), h->stream));
  return AED_OK;
}

int aed_vec_fill_random(aed_handle* h, void* x, uint64_t seed) {
  int rc = check_vec(h, x, "x");
  if (rc) return rc;
  DeviceGuard g(h->device);
  if (h->precision == AED_FP64) return launch_fill_random((double*)x, h->vlen, seed, h->stream);
  return launch_fill_random((float*)x, h->vlen, seed, h->stream);
}

int aed_mult(aed_handle* h, const void* x, void* y) {
  int rc = check_vec(h, x, "x");
  if (!rc) rc = check_vec(h, y, "y");
  if (rc) return rc;
  if (x == y) return fail(AED_ERR_INVALID, "x and y must not alias");
  DeviceGuard g(h->device);
  return handle_hv(h, h->precision == AED_FP32, x, y, nullptr);
}

static int reduce_to_host(aed_handle* h, const void* x, const void* y, bool sq, bool take_sqrt, double* out) {
  int rc;
  if (h->precision == AED_FP64)
    rc = launch_dot_partials((const double*)x, (const double*)y, h->vlen, h->d_partB, sq, h->stream);
  else
    rc = launch_dot_partials((const float*)x, (const float*)y, h->vlen, h->d_partB, sq, h->stream);
  if (!rc) rc = launch_finish_sum(h->d_partB, red_chunks(h->vlen), h->d_scal, take_sqrt, h->stream);
  if (rc) return rc;
  AED_CUDA_TRY(cudaMemcpyAsync(h->h_scal, h->d_scal, 8, cudaMemcpyDeviceToHost, h->stream));
  AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
  *out = h->h_scal[0];
  return AED_OK;
}

int aed_dot(aed_handle* h, const void* x, const void* y, double* out) {
  int rc = check_vec(h, x, "x");
  if (!rc) rc = check_vec(h, y, "y");
  if (rc) return rc;
  if (!out) return fail(AED_ERR_INVALID, "out is NULL");
  DeviceGuard g(h->device);
  return reduce_to_host(h, x, y, false, false, out);
}

int aed_nrm2(aed_handle* h, const void* x, double* out) {
  int rc = check_vec(h, x, "x");
  if (rc) return rc;
  if (!out) return fail(AED_ERR_INVALID, "out is NULL");
  DeviceGuard g(h->device);
  return reduce_to_host(h, x, x, true, true, out);
}

int aed_axpy(aed_handle* h, double a, const void* x, void* y) {
  int rc = check_vec(h, x, "x");
  if (!rc) rc = check_vec(h, y, "y");
  if (rc) return rc;
  DeviceGuard g(h->device);
  if (h->precision == AED_FP64) return launch_axpy(a, (const double*)x, (double*)y, h->vlen, h->stream);
  return launch_axpy(a, (const float*)x, (float*)y, h->vlen, h->stream);
}

int aed_scal(aed_handle* h, double a, void* x) {
  int rc = check_vec(h, x, "x");
  if (rc) return rc;
  DeviceGuard g(h->device);
  if (h->precision == AED_FP64) return launch_scal(a, (double*)x, h->vlen, false, h->stream);
  return launch_scal(a, (float*)x, h->vlen, false, h->stream);
}

int aed_div(aed_handle* h, double a, void* x) {
  int rc = check_vec(h, x, "x");
  if (rc) return rc;
  DeviceGuard g(h->device);
  if (h->precision == AED_FP64) return launch_scal(a, (double*)x, h->vlen, true, h->stream);
  return launch_scal(a, (float*)x, h->vlen, true, h->stream);
}

int aed_lanczos_step(aed_handle* h, const void* v_prev, const void* v_cur, void* v_next, double beta_prev,
                     double* alpha, double* beta) {
  int rc = check_vec(h, v_cur, "v_cur");
  if (!rc) rc = check_vec(h, v_next, "v_next");
  if (rc) return rc;
  if (v_cur == v_next || (v_prev && (v_prev == v_cur || v_prev == v_next)))
    return fail(AED_ERR_INVALID, "Lanczos vectors must not alias");
  DeviceGuard g(h->device);
  const bool f32 = h->precision == AED_FP32;
  h->h_scal[4] = beta_prev;
  AED_CUDA_TRY(cudaMemcpyAsync(h->d_scal + 4, h->h_scal + 4, 8, cudaMemcpyHostToDevice, h->stream));
  rc = lanczos_step_kernels(h, f32, v_prev, v_cur, v_next, h->d_scal + 4, h->d_scal + 0, h->d_scal + 1);
  if (rc) return rc;
  AED_CUDA_TRY(cudaMemcpyAsync(h->h_scal, h->d_scal, 16, cudaMemcpyDeviceToHost, h->stream));
  AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (alpha) *alpha = h->h_scal[0];
  if (beta) *beta = h->h_scal[1];
  return AED_OK;
}

int aed_solve(aed_handle* h, const aed_solve_opts* opts, aed_solve_result* res) {
  if (!h || !opts || !res) return fail(AED_ERR_INVALID, "NULL argument");
  DeviceGuard g(h->device);
  const int rc = solve(h, opts, res);
  return rc ? rc : handle_check_flag(h);
}

int aed_eigenvectors(aed_handle* h, const aed_solve_opts* opts, int32_t k, void* const* vecs, double* evals,
                     double* residuals) {
  if (!h) return fail(AED_ERR_INVALID, "handle is NULL");
  DeviceGuard g(h->device);
  const int rc = eigenvectors(h, opts, k, vecs, evals, residuals);
  return rc ? rc : handle_check_flag(h);
}

int aed_lanczos_state_bytes(aed_handle* h, int64_t* bytes) {
  if (!h || !bytes) return fail(AED_ERR_INVALID, "NULL argument");
  *bytes = lanczos_state_bytes(h);
  return AED_OK;
}

int aed_lanczos_save(aed_handle* h, void* buf, int64_t bytes) {
  if (!h) return fail(AED_ERR_INVALID, "handle is NULL");
  DeviceGuard g(h->device);
  return lanczos_save(h, buf, bytes);
}

int aed_lanczos_load(aed_handle* h, const void* buf, int64_t bytes) {
  if (!h) return fail(AED_ERR_INVALID, "handle is NULL");
  DeviceGuard g(h->device);
  return lanczos_load(h, buf, bytes);
}

int aed_last_tmatrix(aed_handle* h, double* alpha, double* beta, int32_t cap, int32_t* n) {
  if (!h || !n) return fail(AED_ERR_INVALID, "NULL argument");
  *n = (int32_t)h->last_alpha.size();
  for (int32_t i = 0; i < *n && i < cap; ++i) {
    if (alpha) alpha[i] = h->last_alpha[i];
    if (beta) beta[i] = h->last_beta[i];
  }
  return AED_OK;
}

int aed_last_tmatrix_fp32(aed_handle* h, double* alpha, double* beta, int32_t cap, int32_t* n) {
  if (!h || !n) return fail(AED_ERR_INVALID, "NULL argument");
  *n = (int32_t)h->low_alpha.size();
  for (int32_t i = 0; i < *n && i < cap; ++i) {
    if (alpha) alpha[i] = h->low_alpha[i];
    if (beta) beta[i] = h->low_beta[i];
  }
  return AED_OK;
}

int aed_time_apply(aed_handle* h, const void* x, void* y, int32_t reps, int32_t variant, int32_t with_alpha,
                   double* ms, int32_t* variant_used) {
  int rc = check_vec(h, x, "x");
  if (!rc) rc = check_vec(h, y, "y");
  if (rc) return rc;
  if (reps < 1 || !ms) return fail(AED_ERR_INVALID, "reps must be >= 1 and ms non-NULL");
  if (variant >= hv_num_variants()) return fail(AED_ERR_INVALID, "unknown variant");
  DeviceGuard g(h->device);
  if (h->mom || h->gen) {  // one kernel: aed_time_mult with the partials when asked
    if (variant_used) *variant_used = -1;
    return time_hv(h, x, y, reps, with_alpha ? h->d_partA : nullptr, ms);
  }
  const bool f32 = h->precision == AED_FP32;
  int v = variant;
  if (v < 0) {
    int& hv = h->hv_var[f32 ? 1 : 0];
    if (hv < 0 && (rc = pick_variant(h, f32, x, y, &hv))) return rc;
    v = hv;
  }
  double* part = with_alpha ? h->d_partA : nullptr;
  if ((rc = launch_checked(h, f32, v, x, y, part))) return rc;  // warm-up
  cudaEvent_t e0, e1;
  AED_CUDA_TRY(cudaEventCreate(&e0));
  AED_CUDA_TRY(cudaEventCreate(&e1));
  cudaEventRecord(e0, h->stream);
  for (int r = 0; r < reps && !rc; ++r) rc = launch_checked(h, f32, v, x, y, part);
  cudaEventRecord(e1, h->stream);
  cudaEventSynchronize(e1);
  float t = 0.f;
  cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc || (rc = handle_check_flag(h))) return rc;
  *ms = (double)t / reps;
  if (variant_used) *variant_used = v;
  return AED_OK;
}

int32_t aed_apply_variant_count(void) { return hv_num_variants(); }

const char* aed_apply_variant_name(int32_t variant) {
  return (variant >= 0 && variant < hv_num_variants()) ? hv_variant_name(variant) : nullptr;
}

int aed_time_mult(aed_handle* h, const void* x, void* y, int32_t reps, double* ms) {
  int rc = check_vec(h, x, "x");
  if (!rc) rc = check_vec(h, y, "y");
  if (rc) return rc;
  if (reps < 1 || !ms) return fail(AED_ERR_INVALID, "reps must be >= 1 and ms non-NULL");
  DeviceGuard g(h->device);
  return time_hv(h, x, y, reps, nullptr, ms);
}

int aed_tmatrix(int32_t n, const double* alpha, const double* beta, int32_t cap, double* evals, double* errors,
                int32_t* mults, int32_t* count) {
  if (n < 0 || (n > 0 && (!alpha || !beta)) || !count) return fail(AED_ERR_INVALID, "NULL argument");
  *count = 0;
  if (n == 0) return AED_OK;
  double amax = alpha[0], bmax = beta[0];
  for (int i = 1; i < n; ++i) {
    amax = std::max(amax, alpha[i]);
    bmax = std::max(bmax, beta[i]);
  }
  TmatInfo t;
  const int rc = tmatrix_analyze(n, alpha, beta, amax, bmax, t);
  if (rc) return rc;
  const int c = (int)t.evals.size();
  for (int i = 0; i < c && i < cap; ++i) {
    if (evals) evals[i] = t.evals[i];
    if (errors) errors[i] = t.errs[i];
    if (mults) mults[i] = t.mults[i];
  }
  *count = c;
  return AED_OK;
}

int aed_lanczos_vector(aed_handle* h, int32_t j, void* out) {
  if (!h || !out) return fail(AED_ERR_INVALID, "NULL argument");
  if (h->precision != AED_FP32 || j < 0 || j >= h->store_m || h->store_chunk_bytes == 0 ||
      (size_t)(j / kStoreChunk) >= h->store_chunks.size())
    return fail(AED_ERR_INVALID, "lanczos_vector: no such vector of a mixed solve's FP32 phase");
  DeviceGuard g(h->device);
  const size_t vbytes = h->store_chunk_bytes / kStoreChunk;
  const char* src = (const char*)h->store_chunks[j / kStoreChunk] + (size_t)(j % kStoreChunk) * vbytes;
  AED_CUDA_TRY(cudaMemcpyAsync(out, src, (size_t)h->vlen * 4, cudaMemcpyDeviceToDevice, h->stream));
  AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return AED_OK;
}

int aed_get_stream(aed_handle* h, void** stream) {
  if (!h || !stream) return fail(AED_ERR_INVALID, "NULL argument");
  *stream = (void*)h->stream;
  return AED_OK;
}

int aed_launch_count(int64_t* count) {
  if (!count) return fail(AED_ERR_INVALID, "NULL argument");
  *count = launch_count();
  return AED_OK;
}

}  // extern "C"
