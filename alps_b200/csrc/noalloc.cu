// noalloc.cu -- a dot product that allocates nothing (aed_dot_noalloc).
//
// Some callers cannot let a library call cudaMalloc: applications whose device
// memory is owned by another allocator (a framework's caching allocator, or a
// fixed arena handed to a simulation code at start-up) must not see memory
// taken behind their back, and latency-critical loops cannot afford
// cudaMalloc/cudaFree, whose cost is unpredictable and where cudaFree
// synchronises the whole device.  For them this file provides the engine's
// deterministic dot product with its scratch -- the per-chunk partial sums --
// in a fixed file-scope __device__ array instead of memory allocated per call
// or per handle.  Every GPU that loads libaed.so holds that array (512 KiB)
// until the process exits.
//
// The sums are the same as those of aed_dot: same chunks, same trees, same
// order, so the two entry points return the same bits for the same inputs.

#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/aed.h"
#include "aed_internal.h"
#include "kernels.cuh"
#include "reduce.cuh"

namespace aed {
namespace {

// Largest number of chunk partials the static scratch holds, and so the
// largest n: kNoAllocMaxChunks * kRedChunk = 268,435,456 elements.
constexpr int64_t kNoAllocMaxChunks = 65536;
constexpr int64_t kNoAllocMaxElements = kNoAllocMaxChunks * kRedChunk;

// The scratch.  In host code this name is only a host-side stand-in, not a
// device address: host code passes the address obtained from
// cudaGetSymbolAddress below.
static __device__ __align__(256) double g_noalloc_partials[kNoAllocMaxChunks];

template <typename T>
__global__ void __launch_bounds__(kRedThreads) noalloc_dot_partials_kernel(const T* __restrict__ x,
                                                                          const T* __restrict__ y, int64_t n,
                                                                          double* __restrict__ part) {
  chunk_dot_partials<T>(x, y, n, part, false);
}

__global__ void __launch_bounds__(kFinishThreads) noalloc_finish_kernel(const double* __restrict__ part, int64_t n,
                                                                        double* __restrict__ out) {
  finish_sum(part, n, out, false);
}

// Device address of the scratch on each device, looked up once per device
// with that device current.
constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
double* g_scratch[kMaxDevices] = {};
int g_num_sms[kMaxDevices] = {};

int scratch_for_current_device(double** out, int* sms) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(AED_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(AED_ERR_INVALID, "device index beyond 64");
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return fail(AED_ERR_CUDA, std::string("cudaGetSymbolAddress of the static scratch: ") + cudaGetErrorString(e));
    }
    int n = 0;
    e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return fail(AED_ERR_CUDA, std::string("device attribute: ") + cudaGetErrorString(e));
    g_num_sms[dev] = n > 0 ? n : 1;
    g_scratch[dev] = (double*)p;
  }
  *out = g_scratch[dev];
  *sms = g_num_sms[dev];
  return AED_OK;
}

template <typename T>
int noalloc_dot(const T* x, const T* y, int64_t n, double* out, cudaStream_t st) {
  double* part = nullptr;
  int sms = 0;
  int rc = scratch_for_current_device(&part, &sms);
  if (rc) return rc;
  const int64_t nch = (n + kRedChunk - 1) / kRedChunk;
  if (nch > 0) {
    const int64_t cap = (int64_t)sms * 8;
    const int grid = (int)(nch < cap ? nch : cap);
    noalloc_dot_partials_kernel<T><<<grid, kRedThreads, 0, st>>>(x, y, n, part);
  }
  noalloc_finish_kernel<<<1, kFinishThreads, 0, st>>>(part, nch, out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(AED_ERR_CUDA, std::string("aed_dot_noalloc launch: ") + cudaGetErrorString(e));
  return AED_OK;
}

}  // namespace
}  // namespace aed

extern "C" int aed_dot_noalloc(const void* x, const void* y, int64_t n, int precision, double* out, void* stream) {
  using namespace aed;
  if (!out || (n > 0 && (!x || !y))) return fail(AED_ERR_INVALID, "aed_dot_noalloc: NULL pointer");
  if (n < 0) return fail(AED_ERR_INVALID, "aed_dot_noalloc: negative length");
  if (n > kNoAllocMaxElements)
    return fail(AED_ERR_INVALID, "aed_dot_noalloc: n = " + std::to_string(n) + " exceeds the static scratch (at most " +
                                     std::to_string(kNoAllocMaxElements) + " elements)");
  const cudaStream_t st = (cudaStream_t)stream;
  if (precision == AED_FP64) return noalloc_dot((const double*)x, (const double*)y, n, out, st);
  if (precision == AED_FP32) return noalloc_dot((const float*)x, (const float*)y, n, out, st);
  return fail(AED_ERR_INVALID, "aed_dot_noalloc: precision must be AED_FP64 or AED_FP32");
}
