// An objective reduction that allocates nothing.
//
// swfwi_cal_objective() allocates its reduction scratch with cudaMalloc on
// every call.  Some callers cannot allocate device memory: code running
// inside a host-side callback or a memory-pool-managed framework that forbids
// outside allocations, or an embedding that has handed all device memory to
// its own allocator.  swfwi_cal_objective_static() does the same sums (the
// same kernels' arithmetic, 256 FP64 partials a slot, so the results are the
// same bits) with its partials in a file-scope device array that every GPU
// loading this library holds until exit.
//
// The array's host-side name is not a device address, so the first call in
// each CUDA context (with its device current) looks the address up with
// cudaGetSymbolAddress and caches it under that context; that first call
// should come before any stream capture.  A context created later on the
// same device (after cudaDeviceReset, or a non-primary context) gets its
// own lookup.  Every call shares the array and leaves its partials
// there: each call overwrites all the partials it reads, so nothing has to
// start at zero, but calls whose kernels overlap on the GPU (different
// streams, or different host threads) race on it.
#include <cuda.h>
#include <cuda_runtime.h>
#include <map>
#include <mutex>
#include <utility>
#include "common.hpp"
#include "kernels.cuh"

namespace swfwi {
namespace {

constexpr int kStaticSlots = 32;      // at most 32 sums a call
constexpr int kStaticPartials = 256;  // partial sums a slot (as swfwi_cal_objective)
constexpr int kThreads = 256;

static __device__ __align__(256) double g_objective_partials[kStaticSlots * kStaticPartials];

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double ws[32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) ws[w] = v;
  __syncthreads();
  int nw = (blockDim.x + 31) >> 5;
  v = (threadIdx.x < nw) ? ws[threadIdx.x] : 0.0;
  if (w == 0)
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  return v;
}

__global__ void k_static_partials(double *partials, const float *x, long long n) {
  int slot = blockIdx.y;
  const float *v = x + (long long)slot * n;
  double acc = 0.0;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    double a = (double)v[q];
    acc = fma(a, a, acc);
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partials[(long long)slot * kStaticPartials + blockIdx.x] = acc;
}

__global__ void k_static_final(double *out, const double *partials) {
  int slot = blockIdx.x;
  double acc = 0.0;
  for (int i = threadIdx.x; i < kStaticPartials; i += blockDim.x)
    acc += partials[(long long)slot * kStaticPartials + i];
  acc = block_sum(acc);
  if (threadIdx.x == 0) out[slot] = acc;
}

// The current CUDA context (the driver's cuCtxGetCurrent, reached through
// the runtime so the library needs no link against the driver library).
CUcontext current_context() {
  using Fn = CUresult (*)(CUcontext *);
  static Fn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<Fn>(p);
  });
  SWFWI_REQUIRE(fn != nullptr, "cuCtxGetCurrent is not available from the CUDA driver");
  CUcontext c = nullptr;
  SWFWI_REQUIRE(fn(&c) == CUDA_SUCCESS && c != nullptr, "no current CUDA context");
  return c;
}

// Device address of the partials array, looked up once per context.
double *partials_on_current_device() {
  static std::mutex mu;
  static std::map<std::pair<int, CUcontext>, double *> addr;
  int dev = 0;
  SWFWI_CUDA(cudaGetDevice(&dev));
  SWFWI_CUDA(cudaFree(nullptr));   // makes the device's primary context current if none is
  const std::pair<int, CUcontext> key(dev, current_context());
  std::lock_guard<std::mutex> g(mu);
  auto it = addr.find(key);
  if (it != addr.end()) return it->second;
  void *p = nullptr;
  SWFWI_CUDA(cudaGetSymbolAddress(&p, g_objective_partials));
  return addr[key] = static_cast<double *>(p);
}

}  // namespace
}  // namespace swfwi

using namespace swfwi;

extern "C" int swfwi_cal_objective_static(const float *r, long long n_per_slot, int nslots,
                                          double *obj, void *stream) {
  return guarded([&] {
    SWFWI_REQUIRE(r && obj && n_per_slot > 0, "null array or empty slot");
    SWFWI_REQUIRE(nslots >= 1 && nslots <= kStaticSlots,
                  "nslots must be 1..32: the static scratch holds 32 slots of partial sums");
    double *partials = partials_on_current_device();
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    k_static_partials<<<dim3(kStaticPartials, nslots), kThreads, 0, st>>>(partials, r, n_per_slot);
    note_launch();
    k_static_final<<<nslots, kThreads, 0, st>>>(obj, partials);
    note_launch();
    SWFWI_CUDA(cudaGetLastError());
  });
}
