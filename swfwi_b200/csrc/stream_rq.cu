// Launcher of the register-queue streaming step (stream_rq.cuh); its own
// translation unit so it compiles beside kernels.cu.
#include <algorithm>
#include "common.hpp"
#include "kernels.cuh"
#include "stream_rq.cuh"
#include "stream_rq2.cuh"

namespace swfwi {

namespace {

// The longest task (at least 8 rows) with which every (shot, depth slice)
// column's tasks fit in one wave of `resident` warps: a partial last wave
// costs a whole task duration, and shorter tasks spend more of their steps
// filling the register queue.
int one_wave_rows(int nx, long long columns, long long resident) {
  const long long per_column = std::max<long long>(1, resident / columns);
  return std::max(8, (int)((nx - 12 + per_column - 1) / per_column));
}

template <int ARITH, bool DAMPED, int NW, int D>
void rq_t(const StreamArgs &a, int nslots, cudaStream_t st) {
  constexpr size_t smem = rq_smem_bytes<NW, D>();
  // raise the dynamic shared memory limit once (thread-safe static init)
  static const cudaError_t attr = cudaFuncSetAttribute(fd_step_rq<ARITH, DAMPED, NW, D>,
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  SWFWI_CUDA(attr);
  StreamArgs b = a;
  const long long pairs = (long long)nslots * rq_detail::slices(a.nz);   // (shot, depth slice) columns
  if (b.xchunk <= 0) {
    // automatic task length: the longest chunk of rows with which every
    // column's tasks fit in one wave of resident warps (a partial last wave
    // costs a whole task duration; shorter tasks spend more of their steps
    // filling the register queue)
    // resident warps of the device (once, thread-safe static init)
    static const long long resident = [] {
      int dev = 0, sms = 0, per_sm = 0;
      SWFWI_CUDA(cudaGetDevice(&dev));
      SWFWI_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      SWFWI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fd_step_rq<ARITH, DAMPED, NW, D>, NW * 32,
                                                               smem));
      return (long long)std::max(per_sm, 1) * NW * sms;
    }();
    b.xchunk = one_wave_rows(a.nx, pairs, resident);
  }
  const long long nchunks = (b.nx - 12 + b.xchunk - 1) / b.xchunk;
  const long long tasks = pairs * nchunks;
  const long long blocks = (tasks + NW - 1) / NW;
  if (blocks > 0x7fffffffLL) throw Error(SWFWI_ERR_BAD_ARG, "too many stencil tasks for one launch");
  fd_step_rq<ARITH, DAMPED, NW, D><<<(unsigned)blocks, NW * 32, smem, st>>>(b, nslots);
}

// One warp per CTA: the warps' tasks are independent, and a one-warp CTA
// frees its slot as soon as its task ends (measured faster than 2-4 warps
// per CTA, which also need more registers than the 20-warp occupancy
// leaves).
template <int ARITH, bool DAMPED>
void rq_d(int depth, const StreamArgs &a, int nslots, cudaStream_t st) {
  if (depth >= 7) rq_t<ARITH, DAMPED, 1, 7>(a, nslots, st);
  else rq_t<ARITH, DAMPED, 1, 3>(a, nslots, st);
}

template <bool DAMPED>
void rq2_t(const StreamArgs &a, int nslots, cudaStream_t st) {
  constexpr size_t smem = rq2_smem_bytes();
  // raise the dynamic shared memory limit once (thread-safe static init)
  static const cudaError_t attr = cudaFuncSetAttribute(fd_step_rq2<DAMPED>,
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  SWFWI_CUDA(attr);
  StreamArgs b = a;
  const long long columns = (long long)nslots * rq2_detail::slices(a.nz);
  if (b.xchunk <= 0) {
    static const long long resident = [] {
      int dev = 0, sms = 0, per_sm = 0;
      SWFWI_CUDA(cudaGetDevice(&dev));
      SWFWI_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      SWFWI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fd_step_rq2<DAMPED>, 32, smem));
      return (long long)std::max(per_sm, 1) * sms;
    }();
    b.xchunk = one_wave_rows(a.nx, columns, resident);
  }
  const long long tasks = columns * ((b.nx - 12 + b.xchunk - 1) / b.xchunk);
  if (tasks > 0x7fffffffLL) throw Error(SWFWI_ERR_BAD_ARG, "too many stencil tasks for one launch");
  fd_step_rq2<DAMPED><<<(unsigned)tasks, 32, smem, st>>>(b, nslots);
}

}  // namespace

void launch_rq2_step(bool damped, const StreamArgs &a, int nslots, cudaStream_t st) {
  if (nslots <= 0 || a.nx <= 12 || a.nz <= 12) return;
  if (damped) rq2_t<true>(a, nslots, st);
  else rq2_t<false>(a, nslots, st);
  note_launch();
}

void launch_rq_step(int arith, bool damped, int depth, const StreamArgs &a, int nslots, cudaStream_t st) {
  if (nslots <= 0 || a.nx <= 12 || a.nz <= 12) return;
  if (arith == ARITH_REF) {
    if (damped) rq_d<ARITH_REF, true>(depth, a, nslots, st);
    else rq_d<ARITH_REF, false>(depth, a, nslots, st);
  } else {
    if (damped) rq_d<ARITH_FAST, true>(depth, a, nslots, st);
    else rq_d<ARITH_FAST, false>(depth, a, nslots, st);
  }
  note_launch();
}

}  // namespace swfwi
