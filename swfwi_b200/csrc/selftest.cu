// Failure-detection self-test: the stencil kernels' bounded mbarrier wait
// (stream.cuh, mbar_wait) must give up by itself when nothing arrives, raise
// the error flag, and leave the context usable.  One thread waits on a
// barrier no one arrives at; no fault, trap or unbounded loop is involved.
#include "common.hpp"
#include "kernels.cuh"
#include "stream.cuh"

namespace swfwi {
namespace {

__global__ void k_selftest_mbar_timeout(int *err) {
  using namespace stream_detail;
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0 && !mbar_wait(&bar, 0)) atomicExch(err, 1);
}

}  // namespace
}  // namespace swfwi

using namespace swfwi;

extern "C" int swfwi_selftest_bounded_wait(void *stream) {
  return guarded([&] {
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    DevBuf<int> err(1);
    SWFWI_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), st));
    k_selftest_mbar_timeout<<<1, 32, 0, st>>>(err.get());
    note_launch();
    SWFWI_CUDA(cudaGetLastError());
    int h = 0;
    SWFWI_CUDA(cudaMemcpyAsync(&h, err.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    SWFWI_CUDA(cudaStreamSynchronize(st));
    if (h) throw Error(SWFWI_ERR_TIMEOUT, "bounded wait gave up as designed (self-test)");
  });
}
