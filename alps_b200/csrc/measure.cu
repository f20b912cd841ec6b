// measure.cu -- expectation values of site operators and their products in
// one vector of an Sz sector: the quantities DiagMatrix::perform_measurements
// forms (applications/diag/diag.h:191-314, through calculate() at :316-339),
// for the spin-1/2 operators Sz, S+, S-.
//
// For a list of up to kMeasPairs site pairs (i, j) one pass over the sector
// accumulates, per pair:
//   kind SZ     <Sz_i>          = sum_s |psi_s|^2 sz_i(s)
//   kind SZSZ   <Sz_i Sz_j>     = sum_s |psi_s|^2 sz_i(s) sz_j(s)       (i = j: 1/4 |psi|^2)
//   kind SPSM   <S+_i S-_j>     = sum_s psi_{s'} psi_s over states with site j up and site i down,
//                                 s' = s with both flipped (i = j: the weight of site i up)
// (spin-1/2: Sz = diag(-1/2, 1/2), S+ and S- have the matrix element 1,
// models.xml.in's spin site operators).  Rows are walked by the work tiles of
// the apply (hi block h, row range), so the state of a row is
// (h << Nlo) | lolist[looff[k] + r] and a flipped state's row is its
// two-table rank.  Each CTA writes its partial sums; the host adds them in
// order, so results do not depend on timing.
//
// Reference paths are relative to the ALPS source tree.

#include <vector>

#include "handle.h"
#include "reduce.cuh"

namespace aed {
namespace {

constexpr int kMeasThreads = 256;

template <typename T, int KIND>
__global__ void __launch_bounds__(kMeasThreads, 1) meas_kernel(const DevTables t, const T* __restrict__ psi, int np,
                                                            const __grid_constant__ MeasPairs pairs,
                                                            double* __restrict__ part) {
  __shared__ double red[33];
  double acc[kMeasPairs];
#pragma unroll
  for (int p = 0; p < kMeasPairs; ++p) acc[p] = 0.0;
  const uint32_t lm = (1u << t.Nlo) - 1u;
  for (int64_t it = blockIdx.x; it < t.n_tiles; it += gridDim.x) {
    const uint32_t h = t.tile_h[it];
    const uint32_t r0 = t.tile_r[it];
    const int k = t.n_up - __popc(h);
    const uint32_t lbase = t.looff[k];
    const uint32_t rows = t.looff[k + 1] - lbase;
    const uint32_t base = t.thi[h];
    const uint32_t r1 = rows < r0 + kHvTileRows ? rows : r0 + kHvTileRows;
    for (uint32_t r = r0 + threadIdx.x; r < r1; r += kMeasThreads) {
      const uint32_t s = (h << t.Nlo) | t.lolist[lbase + r];
      const double v = (double)psi[base + r];
#pragma unroll
      for (int p = 0; p < kMeasPairs; ++p) {
        if (p >= np) continue;  // (no break: the accumulators stay in registers)
        const uint32_t mi = pairs.mi[p], mj = pairs.mj[p];
        if (KIND == kMeasSz) {
          acc[p] = fma(v * v, (s & mi) ? 0.5 : -0.5, acc[p]);
        } else if (KIND == kMeasSzSz) {
          const double si = (s & mi) ? 0.5 : -0.5, sj = (s & mj) ? 0.5 : -0.5;
          acc[p] = fma(v * v, si * sj, acc[p]);
        } else {
          if (mi == mj) {
            if (s & mi) acc[p] = fma(v, v, acc[p]);
          } else if (!(s & mi) && (s & mj)) {
            const uint32_t s2 = s ^ mi ^ mj;
            const uint32_t rk = t.thi[s2 >> t.Nlo] + t.tlo[s2 & lm];
            acc[p] = fma((double)psi[rk], v, acc[p]);
          }
        }
      }
    }
  }
#pragma unroll
  for (int p = 0; p < kMeasPairs; ++p) {
    if (p >= np) continue;
    const double tot = block_sum_all<kMeasThreads>(acc[p], red);
    if (threadIdx.x == 0) part[(size_t)blockIdx.x * kMeasPairs + p] = tot;
  }
}

template <typename T>
int launch_meas(const DevTables& t, const T* psi, int kind, int np, const MeasPairs& pairs, double* part, int grid,
                cudaStream_t st) {
  switch (kind) {
    case kMeasSz: meas_kernel<T, kMeasSz><<<grid, kMeasThreads, 0, st>>>(t, psi, np, pairs, part); break;
    case kMeasSzSz: meas_kernel<T, kMeasSzSz><<<grid, kMeasThreads, 0, st>>>(t, psi, np, pairs, part); break;
    default: meas_kernel<T, kMeasSpSm><<<grid, kMeasThreads, 0, st>>>(t, psi, np, pairs, part); break;
  }
  return check_launch_counted("meas_kernel");
}

}  // namespace

int measure_pairs(aed_handle* h, const void* psi, int kind, int n, const int32_t* si, const int32_t* sj, double* out) {
  const int N = h->model.N;
  const int64_t tiles = h->dt.n_tiles;
  if (tiles == 0) {
    for (int p = 0; p < n; ++p) out[p] = 0.0;
    return AED_OK;
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = (int)std::min<int64_t>(tiles, (int64_t)sms * 4);
  void* w = nullptr;
  int rc = handle_workspace(h, 1, (size_t)grid * kMeasPairs * 8, &w);
  if (rc) return rc;
  double* part = static_cast<double*>(w);
  std::vector<double> hp((size_t)grid * kMeasPairs);
  for (int p0 = 0; p0 < n; p0 += kMeasPairs) {
    const int np = std::min(kMeasPairs, n - p0);
    MeasPairs pairs{};
    for (int p = 0; p < np; ++p) {
      pairs.mi[p] = 1u << (N - 1 - si[p0 + p]);
      pairs.mj[p] = kind == kMeasSz ? 0u : 1u << (N - 1 - sj[p0 + p]);
    }
    if (h->precision == AED_FP32)
      rc = launch_meas(h->dt, (const float*)psi, kind, np, pairs, part, grid, h->stream);
    else
      rc = launch_meas(h->dt, (const double*)psi, kind, np, pairs, part, grid, h->stream);
    if (rc) return rc;
    AED_CUDA_TRY(cudaMemcpyAsync(hp.data(), part, hp.size() * 8, cudaMemcpyDeviceToHost, h->stream));
    AED_CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (int p = 0; p < np; ++p) {
      double sum = 0.0;
      for (int b = 0; b < grid; ++b) sum += hp[(size_t)b * kMeasPairs + p];
      out[p0 + p] = sum;
    }
  }
  return AED_OK;
}

}  // namespace aed
