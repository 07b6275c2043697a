// Launcher of the two-rows-per-step warp-specialised step (stream_ws2.cuh);
// its own translation unit so it compiles beside kernels.cu.
#include <atomic>
#include "kernels.cuh"
#include "stream_ws2.cuh"

namespace swfwi {

namespace {

template <int ARITH, bool DAMPED, int NW, int D>
void ws2_t(const StreamArgs &a, int nslots, cudaStream_t st) {
  constexpr int BZ = 128 * NW - 8;
  constexpr size_t smem = ws2_smem_bytes<NW, D>();
  static bool attr_set = false;   // raise the dynamic shared memory limit once
  if (!attr_set) {
    cudaFuncSetAttribute(fd_step_ws2<ARITH, DAMPED, NW, D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    attr_set = true;
  }
  int nbands = (a.nz - 10 + BZ - 1) / BZ;
  int nchunks = (a.nx - 12 + a.xchunk - 1) / a.xchunk;
  dim3 g = a.shot_major ? dim3(nbands, nchunks, nslots) : dim3(nslots, nbands, nchunks);
  fd_step_ws2<ARITH, DAMPED, NW, D><<<g, (NW + 1) * 32, smem, st>>>(a);
}

template <int ARITH, bool DAMPED, int D>
void ws2_nw(int bz, const StreamArgs &a, int nslots, cudaStream_t st) {
  if (bz >= 376) ws2_t<ARITH, DAMPED, 3, D>(a, nslots, st);
  else if (bz >= 248) ws2_t<ARITH, DAMPED, 2, D>(a, nslots, st);
  else ws2_t<ARITH, DAMPED, 1, D>(a, nslots, st);
}

template <int ARITH, bool DAMPED>
void ws2_d(int depth, int bz, const StreamArgs &a, int nslots, cudaStream_t st) {
  if (depth >= 7) ws2_nw<ARITH, DAMPED, 7>(bz, a, nslots, st);
  else ws2_nw<ARITH, DAMPED, 3>(bz, a, nslots, st);
}

}  // namespace

void launch_ws2_step(int arith, bool damped, int bz, int depth, const StreamArgs &a, int nslots,
                     cudaStream_t st) {
  if (nslots <= 0 || a.nx <= 12 || a.nz <= 12) return;
  if (arith == ARITH_REF) {
    if (damped) ws2_d<ARITH_REF, true>(depth, bz, a, nslots, st);
    else ws2_d<ARITH_REF, false>(depth, bz, a, nslots, st);
  } else {
    if (damped) ws2_d<ARITH_FAST, true>(depth, bz, a, nslots, st);
    else ws2_d<ARITH_FAST, false>(depth, bz, a, nslots, st);
  }
  note_launch();
}

}  // namespace swfwi
