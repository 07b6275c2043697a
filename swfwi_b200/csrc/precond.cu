// Learned preconditioner: BF16 convolutions on the fifth-generation tensor
// cores (forward, data gradient and weight gradient: tcgen05.mma with FP32
// accumulators in tensor memory), the encoder-decoder around them, its
// training step and the features/scatter between the padded model grid and
// the network's image.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <random>
#include "kernels.cuh"
#include "precond.hpp"
#include "stream.cuh"

namespace swfwi {
namespace {

using bf16 = __nv_bfloat16;
constexpr int kEw = 256;   // threads of the elementwise kernels

inline void noted() { g_kernel_launches.fetch_add(1, std::memory_order_relaxed); }
inline unsigned blocks_for(long long n, int threads = kEw) {
  long long b = (n + threads - 1) / threads;
  return (unsigned)std::max(1LL, std::min(b, 148LL * 64));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t *>(&v);
}

// ---------------------------------------------------------------- 3x3 conv, tcgen05
// Implicit GEMM on the fifth-generation tensor cores.  A CTA of 128 threads
// owns 128 consecutive pixels of the flattened (n, h, w) index (M = 128) and
// every output channel (N = cout, a multiple of 16 up to 256); K = 9 taps x
// cin, 16 channels per MMA.  The taps go in rounds of T (9, 3 or 1, the most
// whose tiles fit the shared-memory budget): per round the threads copy, for
// each of its taps, the 128 shifted pixel rows (zero-filled outside the
// image) and the tap's weights into shared memory with cp.async, as K-major
// core matrices without swizzle (8 rows x 16 bytes; the 8-row groups 256 B
// apart, the two 8-channel halves of a 16-channel chunk 128 B apart).  With
// more than one round, two stages: while the tensor cores run one round, the
// copies of the next land in the other stage.  One thread issues a round's
// T x cin/16 tcgen05.mma into the FP32 accumulator in tensor memory and
// commits them to the stage's mbarrier; a stage is refilled only after its
// barrier shows those MMAs done (bounded waits).  Narrow layers take all 9
// taps in one round: one copy, MMA and commit latency per CTA instead of 9.
// The epilogue reads the accumulator 16 columns at a time (warp w holds the
// tensor-memory lanes, i.e. pixels, 32w .. 32w+31) and writes BF16 with
// bias and ReLU, or FP32 (optionally added to the output).  A wait that
// gives up sets g_conv_timeout; the CTA still frees its tensor memory.
// (The row-tile kernel below replaces this one wherever its stages fit.)
__device__ int g_conv_timeout;

namespace tc {
__device__ __forceinline__ uint32_t saddr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
// shared-memory matrix descriptor: start address, leading (K) byte offset
// 128, stride (8-row group) byte offset 256, descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)(256u >> 4) << 32) |
         (1ull << 46);
}
__host__ __device__ inline int tmem_cols(int n) { return n <= 32 ? 32 : (n <= 64 ? 64 : (n <= 128 ? 128 : 256)); }
// 16 bytes global -> shared, zero-filled when !valid (src is then not read)
__device__ __forceinline__ void cp16(uint32_t dst, const void *src, bool valid) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
// bytes of one stage of T taps (A and B tiles)
__host__ __device__ inline int stage_bytes(int cin, int cout, int T) { return T * (cin / 16) * (4096 + 32 * cout); }
constexpr int kStageBudget = 96 * 1024;   // shared memory the stages may take
// taps per round: the most of 9, 3, 1 whose stages fit the budget
__host__ __device__ inline int taps_per_round(int cin, int cout) {
  if (stage_bytes(cin, cout, 9) <= kStageBudget) return 9;
  return 2 * stage_bytes(cin, cout, 3) <= kStageBudget ? 3 : 1;
}
}  // namespace tc

template <bool F32>
__global__ void __launch_bounds__(128) k_conv3x3_tc(const bf16 *__restrict__ in, int cin,
                                                    const bf16 *__restrict__ w, const float *__restrict__ bias,
                                                    void *out, int accum, int cout, int N, int H, int W) {
  using namespace stream_detail;
  extern __shared__ __align__(1024) unsigned char sm[];
  const int KC = cin / 16, T = tc::taps_per_round(cin, cout), R = 9 / T;
  const int SB = tc::stage_bytes(cin, cout, T), NS = R > 1 ? 2 : 1;
  // stage s at sm + s*SB: the round's A tiles (T x KC x 4 KB, tap-major),
  // then its B tiles (T x KC x cout x 32 B)
  uint64_t *bar = reinterpret_cast<uint64_t *>(sm + NS * SB);   // one per stage
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long HW = (long long)H * W, P = (long long)N * HW;
  const long long p0 = (long long)blockIdx.x * 128;
  const uint32_t ncols = (uint32_t)tc::tmem_cols(cout);
  // thread tid copies A row tid (its pixel, decoded once; valid = inside the
  // batch) and the B rows co = tid, tid + 128, ... of every tap
  const long long pm = p0 + tid;
  const bool pin = pm < P;
  const int pn = pin ? (int)(pm / HW) : 0, pr = pin ? (int)(pm - (long long)pn * HW) : 0;
  const int ph = pr / W, pw = pr - ph * W;
  // the row's place in a 16-channel chunk's A tile (core matrix, row within it)
  const uint32_t arow = (uint32_t)((tid >> 3) * 256 + (tid & 7) * 16);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::saddr(tslot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t taddr = *tslot;
  // kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B, both
  // K-major, N = cout, M = 128
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(cout >> 3) << 17) | ((128u >> 4) << 24);
  const uint32_t sbase = tc::saddr(sm);

  auto load_round = [&](int rd) {
    const uint32_t sa = sbase + (uint32_t)((rd % NS) * SB), sb = sa + (uint32_t)(T * KC * 4096);
    for (int t = 0; t < T; t++) {
      const int tap = rd * T + t, ky = tap / 3, kx = tap - 3 * ky;
      const uint32_t at = sa + (uint32_t)(t * KC * 4096) + arow, bt = sb + (uint32_t)(t * KC * cout * 32);
      const int hh = ph + ky - 1, xx = pw + kx - 1;
      const bool ok = pin && hh >= 0 && hh < H && xx >= 0 && xx < W;
      const bf16 *src = ok ? in + (((long long)pn * H + hh) * W + xx) * cin : in;
      // 16 bytes per step along the pixel's channels: chunk q >> 1, half q & 1
      for (int q = 0; q < 2 * KC; q++)
        tc::cp16(at + (uint32_t)((q >> 1) * 4096 + (q & 1) * 128), ok ? src + q * 8 : in, ok);
      for (int co = tid; co < cout; co += 128) {
        const bf16 *wr = w + ((long long)co * 9 + tap) * cin;
        const uint32_t brow = bt + (uint32_t)((co >> 3) * 256 + (co & 7) * 16);
        for (int q = 0; q < 2 * KC; q++)
          tc::cp16(brow + (uint32_t)((q >> 1) * cout * 32 + (q & 1) * 128), wr + q * 8, true);
      }
    }
    tc::cp_commit();
  };

  bool ok = true;
  load_round(0);
  for (int rd = 0; rd < R && ok; rd++) {
    if (rd + 1 < R) {
      // the next round's stage was read by the MMAs of round rd-1: wait for them
      if (rd >= 1 && !__syncthreads_and(mbar_wait(&bar[(rd + 1) & 1], (uint32_t)(((rd - 1) >> 1) & 1)))) {
        ok = false;
        break;
      }
      load_round(rd + 1);
      tc::cp_wait<1>();   // this round's copies are complete, the next round's may be in flight
    } else {
      tc::cp_wait<0>();
    }
    // the tiles were written through the generic proxy; the MMA reads them
    // through the async proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t sa = sbase + (uint32_t)((rd % NS) * SB), sb = sa + (uint32_t)(T * KC * 4096);
      for (int kc = 0; kc < T * KC; kc++) {   // (tap within the round, 16-channel chunk)
        const uint64_t ad = tc::kmajor_desc(sa + kc * 4096);
        const uint64_t bd = tc::kmajor_desc(sb + kc * cout * 32);
        const uint32_t acc = (rd > 0 || kc > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(taddr),
            "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       tc::saddr(&bar[rd & 1]))
                   : "memory");
    }
  }
  // the last commit (round R-1, its barrier's ((R-1)/2 + 1)-th phase) covers every MMA
  if (ok && !__syncthreads_and(mbar_wait(&bar[(R - 1) & 1], (uint32_t)(((R - 1) >> 1) & 1)))) ok = false;
  tc::cp_wait<0>();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok) {
    const long long p = p0 + warp * 32 + lane;
    for (int c0 = 0; c0 < cout; c0 += 16) {
      uint32_t r[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (p < P) {
        if constexpr (F32) {
          float4 *o = reinterpret_cast<float4 *>(reinterpret_cast<float *>(out) + p * cout + c0);
#pragma unroll
          for (int i = 0; i < 4; i++) {
            float4 v = make_float4(__uint_as_float(r[4 * i]), __uint_as_float(r[4 * i + 1]),
                                   __uint_as_float(r[4 * i + 2]), __uint_as_float(r[4 * i + 3]));
            if (accum) {
              const float4 q = o[i];
              v.x += q.x; v.y += q.y; v.z += q.z; v.w += q.w;
            }
            o[i] = v;
          }
        } else {
          uint4 *o = reinterpret_cast<uint4 *>(reinterpret_cast<bf16 *>(out) + p * cout + c0);
          uint32_t pk[8];
#pragma unroll
          for (int i = 0; i < 8; i++)
            pk[i] = pack_bf16(fmaxf(__uint_as_float(r[2 * i]) + bias[c0 + 2 * i], 0.0f),
                              fmaxf(__uint_as_float(r[2 * i + 1]) + bias[c0 + 2 * i + 1], 0.0f));
          o[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
          o[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
        }
      }
    }
  } else if (tid == 0) {
    atomicExch(&g_conv_timeout, 1);
    // bounded: whatever MMAs are still in flight, before their tensor memory goes
    mbar_wait(&bar[0], 0u);
    mbar_wait(&bar[1], 1u);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// ---------------------------------------------------------------- 3x3 conv, tcgen05, row tiles
// The same implicit GEMM with row-aligned tiles: the CTA's 128 pixels are
// 16 groups of 8 consecutive pixels of one image row each.  For every group
// the three input rows it needs (h-1, h, h+1) are staged once, 10 pixels
// wide (the group and a one-pixel halo), as 16-byte rows per 8-channel half:
// A(tap ky, kx) is then the staged rows of ky seen from a start address
// shifted by kx rows, with the 8-row groups 160 B apart -- the three column
// taps share one copy, and the input is copied 30/8 times instead of 9.
// The rows of ky go in rounds (all three at once when they fit, else one
// ky a round, double-buffered).
namespace tg {
constexpr int kGroupBytes = 160;                  // 10 pixels x 16 bytes
constexpr int kPlaneRow = 16 * kGroupBytes;       // one ky row of the 16 groups
__host__ __device__ inline int rows_per_round(int cin, int cout) {
  const int kc = cin / 16;
  if (kc * (2 * 3 * kPlaneRow + 9 * 32 * cout) <= 96 * 1024) return 3;
  return 1;
}
__host__ __device__ inline int stage_bytes(int cin, int cout, int nky) {
  const int kc = cin / 16;
  return kc * (2 * nky * kPlaneRow + 3 * nky * 32 * cout);
}
}  // namespace tg

// KC = cin / 16 is a template parameter: the staging's divisions by the
// channel count are by constants.
template <bool F32, int KC>
__global__ void __launch_bounds__(128) k_conv3x3_tg(const bf16 *__restrict__ in, const bf16 *__restrict__ w,
                                                    const float *__restrict__ bias, void *out, int accum, int cout,
                                                    int N, int H, int W) {
  using namespace stream_detail;
  extern __shared__ __align__(1024) unsigned char sm[];
  constexpr int cin = 16 * KC;
  const int NKY = tg::rows_per_round(cin, cout), R = 3 / NKY, NS = R > 1 ? 2 : 1;
  const int SB = tg::stage_bytes(cin, cout, NKY), ABYTES = KC * 2 * NKY * tg::kPlaneRow;
  uint64_t *bar = reinterpret_cast<uint64_t *>(sm + NS * SB);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 2);
  int *gn = reinterpret_cast<int *>(bar + 3), *gh = gn + 16, *gw = gh + 16;   // the 16 groups (n = -1: none)
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int GW = (W + 7) / 8;
  const long long groups = (long long)N * H * GW;
  const uint32_t ncols = (uint32_t)tc::tmem_cols(cout);
  if (tid < 16) {
    const long long gi = (long long)blockIdx.x * 16 + tid;
    const long long row = gi / GW;
    gn[tid] = gi < groups ? (int)(row / H) : -1;
    gh[tid] = gi < groups ? (int)(row % H) : 0;
    gw[tid] = gi < groups ? (int)(gi % GW) * 8 : 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::saddr(tslot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t taddr = *tslot;
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(cout >> 3) << 17) | ((128u >> 4) << 24);
  const uint32_t sbase = tc::saddr(sm);

  // round rd: input rows ky = rd*NKY .. +NKY-1 and the taps 3*ky + kx
  auto load_round = [&](int rd) {
    const uint32_t sa = sbase + (uint32_t)((rd % NS) * SB), sb = sa + (uint32_t)ABYTES;
    // A: [kc][half][kyl][group][10 px][16 B], 16 bytes per step along a pixel's channels
    for (int u = tid; u < NKY * 16 * 10 * 2 * KC; u += 128) {
      const int q = u % (2 * KC), v = u / (2 * KC), px = v % 10, gk = v / 10, g = gk & 15, kyl = gk >> 4;
      const int n = gn[g], hh = gh[g] + rd * NKY + kyl - 1, xx = gw[g] + px - 1;
      const bool ok = n >= 0 && hh >= 0 && hh < H && xx >= 0 && xx < W;
      tc::cp16(sa + (uint32_t)((((q >> 1) * 2 + (q & 1)) * NKY + kyl) * tg::kPlaneRow + g * tg::kGroupBytes + px * 16),
               ok ? in + (((long long)n * H + hh) * W + xx) * cin + q * 8 : in, ok);
    }
    // B: the round's 3*NKY taps x [kc] x cout rows in K-major core matrices
    for (int u = tid; u < 3 * NKY * cout * 2 * KC; u += 128) {
      const int q = u % (2 * KC), v = u / (2 * KC), co = v % cout, t = v / cout;
      const int tap = rd * 3 * NKY + t;
      tc::cp16(sb + (uint32_t)((t * KC + (q >> 1)) * cout * 32 + ((co >> 3) * 2 + (q & 1)) * 128 + (co & 7) * 16),
               w + ((long long)co * 9 + tap) * cin + q * 8, true);
    }
    tc::cp_commit();
  };

  bool ok = true;
  load_round(0);
  for (int rd = 0; rd < R && ok; rd++) {
    if (rd + 1 < R) {
      if (rd >= 1 && !__syncthreads_and(mbar_wait(&bar[(rd + 1) & 1], (uint32_t)(((rd - 1) >> 1) & 1)))) {
        ok = false;
        break;
      }
      load_round(rd + 1);
      tc::cp_wait<1>();
    } else {
      tc::cp_wait<0>();
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t sa = sbase + (uint32_t)((rd % NS) * SB), sb = sa + (uint32_t)ABYTES;
      for (int t = 0; t < 3 * NKY; t++) {
        const int kyl = t / 3, kx = t - 3 * kyl;
        for (int kc = 0; kc < KC; kc++) {
          // A rows: group g at g*160, row i of the group at (i + kx)*16; the
          // channel halves NKY planes apart
          const uint32_t a_addr = sa + (uint32_t)((kc * 2 * NKY + kyl) * tg::kPlaneRow + kx * 16);
          const uint64_t ad = (uint64_t)((a_addr >> 4) & 0x3FFFu) |
                              ((uint64_t)((uint32_t)(NKY * tg::kPlaneRow) >> 4) << 16) |
                              ((uint64_t)((uint32_t)tg::kGroupBytes >> 4) << 32) | (1ull << 46);
          const uint64_t bd = tc::kmajor_desc(sb + (uint32_t)((t * KC + kc) * cout * 32));
          const uint32_t acc = (rd > 0 || t > 0 || kc > 0) ? 1u : 0u;
          asm volatile(
              "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(taddr),
              "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
              : "memory");
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       tc::saddr(&bar[rd & 1]))
                   : "memory");
    }
  }
  if (ok && !__syncthreads_and(mbar_wait(&bar[(R - 1) & 1], (uint32_t)(((R - 1) >> 1) & 1)))) ok = false;
  tc::cp_wait<0>();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok) {
    const int r = warp * 32 + lane, g = r >> 3, i = r & 7;
    const bool valid = gn[g] >= 0 && gw[g] + i < W;
    const long long p = valid ? ((long long)gn[g] * H + gh[g]) * W + gw[g] + i : 0;
    for (int c0 = 0; c0 < cout; c0 += 16) {
      uint32_t v[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (valid) {
        if constexpr (F32) {
          float4 *o = reinterpret_cast<float4 *>(reinterpret_cast<float *>(out) + p * cout + c0);
#pragma unroll
          for (int k = 0; k < 4; k++) {
            float4 x4 = make_float4(__uint_as_float(v[4 * k]), __uint_as_float(v[4 * k + 1]),
                                    __uint_as_float(v[4 * k + 2]), __uint_as_float(v[4 * k + 3]));
            if (accum) {
              const float4 q = o[k];
              x4.x += q.x; x4.y += q.y; x4.z += q.z; x4.w += q.w;
            }
            o[k] = x4;
          }
        } else {
          uint4 *o = reinterpret_cast<uint4 *>(reinterpret_cast<bf16 *>(out) + p * cout + c0);
          uint32_t pk[8];
#pragma unroll
          for (int k = 0; k < 8; k++)
            pk[k] = pack_bf16(fmaxf(__uint_as_float(v[2 * k]) + bias[c0 + 2 * k], 0.0f),
                              fmaxf(__uint_as_float(v[2 * k + 1]) + bias[c0 + 2 * k + 1], 0.0f));
          o[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
          o[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
        }
      }
    }
  } else if (tid == 0) {
    atomicExch(&g_conv_timeout, 1);
    mbar_wait(&bar[0], 0u);   // bounded: whatever MMAs are still in flight
    mbar_wait(&bar[1], 1u);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// ---------------------------------------------------------------- weight gradient, tcgen05
// part[chunk][co][tap * cin + ci] = sum_{p in chunk} dz[p][co] x[p + tap][ci]
// as D (M x N) = A (M x K) B (K x N) on the fifth-generation tensor cores:
// M = output channels (padded to 128 with zero rows), N = a tile of the
// 9 * cin (tap, input channel) columns, K = the chunk's pixels, 16 per MMA.
// Both operands are MN-major (NHWC keeps a pixel's channels contiguous), as
// core matrices without swizzle: 8 pixels x 16 bytes (8 channels), the
// 8-channel groups 128 B apart, the two 8-pixel halves of a 16-pixel step
// (16 groups x 128 B) apart.  Rounds of kWgRound steps are copied with
// cp.async into two stages while the tensor cores run the previous round;
// each round's MMAs are committed to its stage's mbarrier (bounded waits).
// The chunks are summed afterwards in a fixed order (k_reduce_rows):
// training stays bit-reproducible.
constexpr int kWgRound = 4;   // 16-pixel steps per round (64 pixels)

__host__ __device__ inline int wg_tiles(int cin) { return (9 * cin + 255) / 256; }
__host__ __device__ inline int wg_cols(int cin) { return ((9 * cin + wg_tiles(cin) - 1) / wg_tiles(cin) + 15) / 16 * 16; }
__host__ __device__ inline int wg_stage_bytes(int cin) { return kWgRound * (4096 + 32 * wg_cols(cin)); }

// CIN is a template parameter: the staging divides by constants.
template <int CIN>
__global__ void __launch_bounds__(128) k_wgrad_tc(const bf16 *__restrict__ dz, int cout, const bf16 *__restrict__ x,
                                                  float *__restrict__ part, int N, int H, int W, int ppc) {
  using namespace stream_detail;
  extern __shared__ __align__(1024) unsigned char sm[];
  constexpr int cin = CIN;
  const int NT = 9 * cin, NNmax = wg_cols(cin);
  const int n0 = blockIdx.y * NNmax, NN = min(NNmax, NT - n0);   // this CTA's columns
  const int SB = wg_stage_bytes(cin);
  uint64_t *bar = reinterpret_cast<uint64_t *>(sm + 2 * SB);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 2);
  int *dec = reinterpret_cast<int *>(bar + 3);   // [stage][3][64]: n (-1: none), h, w of the round's pixels
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long HW = (long long)H * W, P = (long long)N * HW;
  const long long pb = (long long)blockIdx.x * ppc, pe = min(P, pb + ppc);
  const int R = (int)((pe - pb + 16 * kWgRound - 1) / (16 * kWgRound));   // rounds
  const uint32_t ncols = (uint32_t)tc::tmem_cols(NN);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::saddr(tslot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t taddr = *tslot;
  // kind::f16: FP32 accumulator, BF16 A and B, both MN-major, N = NN, M = 128
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) |
                         ((uint32_t)(NN >> 3) << 17) | ((128u >> 4) << 24);
  const uint32_t sbase = tc::saddr(sm);
  const int zgroups = cout / 8, bgroups = NN / 8;

  auto load_round = [&](int rd) {
    const int st = rd & 1;
    int *dn = dec + st * 192, *dh = dn + 64, *dw = dh + 64;
    if (tid < 64) {   // decode the round's 64 pixels once
      const long long p = pb + (long long)rd * 64 + tid;
      const int n = p < pe ? (int)(p / HW) : -1;
      const int r = p < pe ? (int)(p - (long long)n * HW) : 0;
      dn[tid] = n;
      dh[tid] = r / W;
      dw[tid] = r - (r / W) * W;
    }
    __syncthreads();
    const uint32_t sa = sbase + (uint32_t)(st * SB), sb = sa + (uint32_t)(kWgRound * 4096);
    // A: 64 pixels x 16 channel groups (groups past cout are zero rows)
    for (int u = tid; u < 64 * 16; u += 128) {
      const int g = u & 15, pi = u >> 4, ks = pi >> 4, r = pi & 15;
      const bool ok = g < zgroups && dn[pi] >= 0;
      const long long p = pb + (long long)rd * 64 + pi;
      tc::cp16(sa + (uint32_t)(ks * 4096 + (r >> 3) * 2048 + g * 128 + (r & 7) * 16), ok ? dz + p * cout + g * 8 : dz,
               ok);
    }
    // B: 64 pixels x this tile's (tap, 8-channel) groups, zero outside the image
    for (int u = tid; u < 64 * bgroups; u += 128) {
      const int g = u % bgroups, pi = u / bgroups, ks = pi >> 4, r = pi & 15;
      const int col = n0 + g * 8, tap = col / cin, c8 = col - tap * cin;
      const int ky = tap / 3, kx = tap - 3 * ky;
      const int n = dn[pi], hh = dh[pi] + ky - 1, xx = dw[pi] + kx - 1;
      const bool ok = n >= 0 && hh >= 0 && hh < H && xx >= 0 && xx < W;
      tc::cp16(sb + (uint32_t)(ks * NN * 32 + (r >> 3) * (NN * 16) + g * 128 + (r & 7) * 16),
               ok ? x + (((long long)n * H + hh) * W + xx) * cin + c8 : x, ok);
    }
    tc::cp_commit();
  };

  bool ok = true;
  if (R > 0) load_round(0);
  for (int rd = 0; rd < R && ok; rd++) {
    if (rd + 1 < R) {
      if (rd >= 1 && !__syncthreads_and(mbar_wait(&bar[(rd + 1) & 1], (uint32_t)(((rd - 1) >> 1) & 1)))) {
        ok = false;
        break;
      }
      load_round(rd + 1);
      tc::cp_wait<1>();
    } else {
      tc::cp_wait<0>();
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t sa = sbase + (uint32_t)((rd & 1) * SB), sb = sa + (uint32_t)(kWgRound * 4096);
      for (int ks = 0; ks < kWgRound; ks++) {
        // MN-major descriptors: leading (K-half) offset, stride (8-channel group) offset 128
        const uint64_t ad = (uint64_t)(((sa + ks * 4096) >> 4) & 0x3FFFu) | ((uint64_t)(2048u >> 4) << 16) |
                            ((uint64_t)(128u >> 4) << 32) | (1ull << 46);
        const uint64_t bd = (uint64_t)(((sb + ks * NN * 32) >> 4) & 0x3FFFu) |
                            ((uint64_t)((uint32_t)(NN * 16) >> 4) << 16) | ((uint64_t)(128u >> 4) << 32) | (1ull << 46);
        const uint32_t acc = (rd > 0 || ks > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(taddr),
            "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       tc::saddr(&bar[rd & 1]))
                   : "memory");
    }
  }
  if (ok && R > 0 && !__syncthreads_and(mbar_wait(&bar[(R - 1) & 1], (uint32_t)(((R - 1) >> 1) & 1)))) ok = false;
  tc::cp_wait<0>();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok && warp * 32 < cout) {   // lanes = output channels
    const int co = warp * 32 + lane;
    float *dst = part + ((long long)blockIdx.x * cout + co) * NT + n0;
    for (int c0 = 0; c0 < NN; c0 += 16) {
      uint32_t r[16];
      if (R > 0) {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      } else {
#pragma unroll
        for (int i = 0; i < 16; i++) r[i] = 0u;   // an empty chunk contributes zeros
      }
      if (co < cout) {
        float4 *o = reinterpret_cast<float4 *>(dst + c0);
#pragma unroll
        for (int i = 0; i < 4; i++)
          o[i] = make_float4(__uint_as_float(r[4 * i]), __uint_as_float(r[4 * i + 1]), __uint_as_float(r[4 * i + 2]),
                             __uint_as_float(r[4 * i + 3]));
      }
    }
  } else if (!ok && tid == 0) {
    atomicExch(&g_conv_timeout, 1);
    mbar_wait(&bar[0], 0u);   // bounded: whatever MMAs are still in flight
    mbar_wait(&bar[1], 1u);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// out[i] = sum over r = 0..rows-1, in order, of part[r * len + i]
__global__ void k_reduce_rows(const float *__restrict__ part, int rows, long long len,
                              float *__restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len;
       i += (long long)gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int r = 0; r < rows; r++) s += part[(long long)r * len + i];
    out[i] = s;
  }
}

// --------------------------------------------------------- elementwise parts
__global__ void k_pack3(const float *__restrict__ x3, bf16 *__restrict__ x16, long long P) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P;
       p += (long long)gridDim.x * blockDim.x) {
    uint4 lo, hi;
    lo.x = pack_bf16(x3[3 * p], x3[3 * p + 1]);
    lo.y = pack_bf16(x3[3 * p + 2], 0.0f);
    lo.z = lo.w = 0u;
    hi.x = hi.y = hi.z = hi.w = 0u;
    uint4 *o = reinterpret_cast<uint4 *>(x16 + p * 16);
    o[0] = lo;
    o[1] = hi;
  }
}

__global__ void k_pool(const bf16 *__restrict__ in, bf16 *__restrict__ out, int N, int H, int W,
                       int C) {
  const int Ho = H / 2, Wo = W / 2, cp = C / 2;
  const long long total = (long long)N * Ho * Wo * cp;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = 2 * (int)(e % cp);
    long long q = e / cp;
    const int wo = (int)(q % Wo);
    q /= Wo;
    const int ho = (int)(q % Ho);
    const int n = (int)(q / Ho);
    const long long r0 = ((long long)(n * H + 2 * ho) * W + 2 * wo) * C + c;
    const long long r1 = r0 + (long long)W * C;
    const __nv_bfloat162 a = *reinterpret_cast<const __nv_bfloat162 *>(in + r0);
    const __nv_bfloat162 b = *reinterpret_cast<const __nv_bfloat162 *>(in + r0 + C);
    const __nv_bfloat162 d = *reinterpret_cast<const __nv_bfloat162 *>(in + r1);
    const __nv_bfloat162 f = *reinterpret_cast<const __nv_bfloat162 *>(in + r1 + C);
    const float lo = (((__low2float(a) + __low2float(b)) + __low2float(d)) + __low2float(f)) * 0.25f;
    const float hi = (((__high2float(a) + __high2float(b)) + __high2float(d)) + __high2float(f)) * 0.25f;
    reinterpret_cast<uint32_t *>(out)[(((long long)(n * Ho + ho) * Wo + wo) * C + c) / 2] = pack_bf16(lo, hi);
  }
}

// din (fine grid) += 0.25 dout (coarse grid)
__global__ void k_pool_bwd(const float *__restrict__ dout, float *__restrict__ din, int N, int H,
                           int W, int C) {
  const long long total = (long long)N * H * W * C;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e % C);
    long long q = e / C;
    const int w = (int)(q % W);
    q /= W;
    const int h = (int)(q % H);
    const int n = (int)(q / H);
    din[e] += 0.25f * dout[((long long)(n * (H / 2) + h / 2) * (W / 2) + w / 2) * C + c];
  }
}

// cat[n][h][w] = (low[n][h/2][w/2][0..C1), skip[n][h][w][0..C2))
__global__ void k_upcat(const bf16 *__restrict__ low, int C1, const bf16 *__restrict__ skip, int C2,
                        bf16 *__restrict__ cat, int N, int H, int W) {
  const int Ct = C1 + C2, cp = Ct / 2;
  const long long total = (long long)N * H * W * cp;
  const uint32_t *lo = reinterpret_cast<const uint32_t *>(low);
  const uint32_t *sk = reinterpret_cast<const uint32_t *>(skip);
  uint32_t *o = reinterpret_cast<uint32_t *>(cat);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = 2 * (int)(e % cp);
    const long long pix = e / cp;
    const int w = (int)(pix % W);
    const long long nh = pix / W;
    const int h = (int)(nh % H);
    const int n = (int)(nh / H);
    uint32_t v;
    if (c < C1) v = lo[(((long long)(n * (H / 2) + h / 2) * (W / 2) + w / 2) * C1 + c) / 2];
    else v = sk[(pix * C2 + (c - C1)) / 2];
    o[e] = v;
  }
}

// dlow[n][h][w][c] = sum of the four fine gradients of its copies
__global__ void k_upcat_bwd_low(const float *__restrict__ dcat, int Ct, int C1, float *__restrict__ dlow,
                                int N, int Hl, int Wl) {
  const long long total = (long long)N * Hl * Wl * C1;
  const int H = 2 * Hl, W = 2 * Wl;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e % C1);
    long long q = e / C1;
    const int w = (int)(q % Wl);
    q /= Wl;
    const int h = (int)(q % Hl);
    const int n = (int)(q / Hl);
    const long long r0 = ((long long)(n * H + 2 * h) * W + 2 * w) * Ct + c;
    const long long r1 = r0 + (long long)W * Ct;
    dlow[e] = ((dcat[r0] + dcat[r0 + Ct]) + dcat[r1]) + dcat[r1 + Ct];
  }
}

__global__ void k_upcat_bwd_skip(const float *__restrict__ dcat, int Ct, int C1, float *__restrict__ dskip,
                                 long long P, int C2) {
  const long long total = P * C2;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long p = e / C2;
    const int c = (int)(e - p * C2);
    dskip[e] = dcat[p * Ct + C1 + c];
  }
}

// y[p] = b + sum_c w[c] u[p][c]   (FP32)
__global__ void k_out_fwd(const bf16 *__restrict__ u, const float *__restrict__ w,
                          const float *__restrict__ b, float *__restrict__ y, long long P, int C) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P;
       p += (long long)gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int c = 0; c < C; c++) s = fmaf(w[c], __bfloat162float(u[p * C + c]), s);
    y[p] = s + b[0];
  }
}

__global__ void k_out_bwd_dx(const float *__restrict__ dy, const float *__restrict__ w,
                             float *__restrict__ du, long long P, int C) {
  const long long total = P * C;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long p = e / C;
    du[e] = dy[p] * w[e - p * C];
  }
}

// part[block][c] = sum over the block's pixels of a[p][c] * (wgt ? wgt[p] :
// 1); C divides the block size.  Summed over blocks by k_reduce_rows.
__global__ void k_chan_dot(const bf16 *__restrict__ a, const float *__restrict__ wgt, long long P,
                           int C, float *__restrict__ part) {
  __shared__ float red[kEw];
  const int c = threadIdx.x % C, lp = threadIdx.x / C, ps = kEw / C;
  float s = 0.0f;
  for (long long p = (long long)blockIdx.x * ps + lp; p < P; p += (long long)gridDim.x * ps) {
    const float v = __bfloat162float(a[p * C + c]);
    s += wgt ? v * wgt[p] : v;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x < C) {
    float tsum = 0.0f;
    for (int k = 0; k < ps; k++) tsum += red[k * C + threadIdx.x];
    part[(long long)blockIdx.x * C + threadIdx.x] = tsum;
  }
}

// part[block] = the block's sum of a (fixed order)
__global__ void k_sum(const float *__restrict__ a, long long n, float *__restrict__ part) {
  __shared__ float red[kEw / 32];
  float s = 0.0f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    s += a[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.0f;
    for (int w = 0; w < kEw / 32; w++) t += red[w];
    part[blockIdx.x] = t;
  }
}

// dy = scale (y - t); loss += (y - t)^2 (FP64)
__global__ void k_mse(const float *__restrict__ y, const float *__restrict__ t, float *__restrict__ dy,
                      long long P, float scale, double *__restrict__ loss) {
  double s = 0.0;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P;
       p += (long long)gridDim.x * blockDim.x) {
    const float r = y[p] - t[p];
    dy[p] = scale * r;
    s += (double)r * r;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, s);
}

// ReLU gradient, rounded to BF16 for the tensor-core products
__global__ void k_relu_mask(const float *__restrict__ dy, const bf16 *__restrict__ y, bf16 *__restrict__ dz,
                            long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    dz[i] = __float2bfloat16_rn(__bfloat162float(y[i]) > 0.0f ? dy[i] : 0.0f);
}

// wt[ci][tap][co] = w[co][8 - tap][ci]: the data gradient as a forward conv
__global__ void k_flip(const bf16 *__restrict__ w, bf16 *__restrict__ wt, int cout, int cin) {
  const long long total = (long long)cout * 9 * cin;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int co = (int)(e % cout);
    const long long q = e / cout;
    const int tap = (int)(q % 9);
    const int ci = (int)(q / 9);
    wt[e] = w[((long long)co * 9 + (8 - tap)) * cin + ci];
  }
}

__global__ void k_adam(float *__restrict__ p, float *__restrict__ m, float *__restrict__ v,
                       const float *__restrict__ g, long long n, float lr_t, float b1, float b2,
                       float eps) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr_t * mi / (sqrtf(vi) + eps);
  }
}

__global__ void k_to_bf16(const float *__restrict__ a, bf16 *__restrict__ b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    b[i] = __float2bfloat16_rn(a[i]);
}

// Interior statistics, per block: part[block][0..3] = sum a^2, sum b,
// sum b^2, max c (c >= 0); k_stats_final adds the blocks in order.
__global__ void k_stats(const float *__restrict__ a, const float *__restrict__ b,
                        const float *__restrict__ c, int nzpad, int x0, int z0, int nx, int nz,
                        double *__restrict__ part) {
  double sa = 0, sb = 0, sb2 = 0, mc = 0;
  const long long total = (long long)nx * nz;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(e / nz), iz = (int)(e - (long long)ix * nz);
    const long long q = (long long)(x0 + ix) * nzpad + z0 + iz;
    if (a) sa += (double)a[q] * a[q];
    if (b) { sb += b[q]; sb2 += (double)b[q] * b[q]; }
    if (c) mc = fmax(mc, (double)fmaxf(c[q], 0.0f));
  }
  for (int o = 16; o > 0; o >>= 1) {
    sa += __shfl_down_sync(0xffffffffu, sa, o);
    sb += __shfl_down_sync(0xffffffffu, sb, o);
    sb2 += __shfl_down_sync(0xffffffffu, sb2, o);
    mc = fmax(mc, __shfl_down_sync(0xffffffffu, mc, o));
  }
  __shared__ double red[kEw / 32][4];
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5][0] = sa;
    red[threadIdx.x >> 5][1] = sb;
    red[threadIdx.x >> 5][2] = sb2;
    red[threadIdx.x >> 5][3] = mc;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t0 = 0, t1 = 0, t2 = 0, t3 = 0;
    for (int w = 0; w < kEw / 32; w++) {
      t0 += red[w][0];
      t1 += red[w][1];
      t2 += red[w][2];
      t3 = fmax(t3, red[w][3]);
    }
    part[4 * blockIdx.x] = t0;
    part[4 * blockIdx.x + 1] = t1;
    part[4 * blockIdx.x + 2] = t2;
    part[4 * blockIdx.x + 3] = t3;
  }
}

__global__ void k_stats_final(const double *__restrict__ part, int blocks, double *__restrict__ s) {
  double t0 = 0, t1 = 0, t2 = 0, t3 = 0;
  for (int i = 0; i < blocks; i++) {
    t0 += part[4 * i];
    t1 += part[4 * i + 1];
    t2 += part[4 * i + 2];
    t3 = fmax(t3, part[4 * i + 3]);
  }
  s[0] = t0;
  s[1] = t1;
  s[2] = t2;
  s[3] = t3;
}

__global__ void k_features(const float *__restrict__ gr, const float *__restrict__ vel,
                           const float *__restrict__ il, int nzpad, int x0, int z0, int nx, int nz,
                           int Hp, int Wp, const double *__restrict__ s, float *__restrict__ x3) {
  const double cnt = (double)nx * nz;
  const double rms = sqrt(s[0] / cnt);
  const double mean = s[1] / cnt;
  const double var = fmax(s[2] / cnt - mean * mean, 0.0);
  const double sd = sqrt(var);
  const double imax = s[3];
  const long long total = (long long)Hp * Wp;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int h = (int)(e / Wp), w = (int)(e - (long long)h * Wp);
    float f0 = 0, f1 = 0, f2 = 0;
    if (h < nx && w < nz) {
      const long long q = (long long)(x0 + h) * nzpad + z0 + w;
      if (rms > 0) f0 = (float)(gr[q] / rms);
      if (sd > 0) f1 = (float)((vel[q] - mean) / sd);
      if (il && imax > 0) f2 = (log10f((float)(fmaxf(il[q], 0.0f) / imax) + 1e-6f) + 3.0f) / 3.0f;
    }
    x3[3 * e] = f0;
    x3[3 * e + 1] = f1;
    x3[3 * e + 2] = f2;
  }
}

__global__ void k_target(const float *__restrict__ dv, int nzpad, int x0, int z0, int nx, int nz,
                         int Hp, int Wp, const double *__restrict__ s, float *__restrict__ t) {
  const double rms = sqrt(s[0] / ((double)nx * nz));
  const long long total = (long long)Hp * Wp;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int h = (int)(e / Wp), w = (int)(e - (long long)h * Wp);
    float v = 0;
    if (h < nx && w < nz && rms > 0) v = (float)(dv[(long long)(x0 + h) * nzpad + z0 + w] / rms);
    t[e] = v;
  }
}

__global__ void k_scatter(const float *__restrict__ y, int nzpad, int x0, int z0, int nx, int nz,
                          int Wp, float *__restrict__ dir) {
  const long long total = (long long)nx * nz;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(e / nz), iz = (int)(e - (long long)ix * nz);
    dir[(long long)(x0 + ix) * nzpad + z0 + iz] = y[(long long)ix * Wp + iz];
  }
}

__global__ void k_illum(float *__restrict__ illum, const float *__restrict__ p, long long fstride,
                        int n, int nxpad, int nzpad, int pitch) {
  const long long total = (long long)nxpad * nzpad;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(e / nzpad), z = (int)(e - (long long)x * nzpad);
    float s = 0.0f;
    for (int j = 0; j < n; j++) {
      const float v = p[j * fstride + (long long)x * pitch + z];
      s = fmaf(v, v, s);
    }
    illum[e] += s;
  }
}

// Dynamic shared memory of a launch: two stages, the barriers, the tensor
// memory address and the decoded pixels -- raised where needed so that no
// more CTAs are resident on an SM than its 512 tensor-memory columns hold
// (a CTA that cannot allocate would wait inside tcgen05.alloc).
size_t conv_tc_smem(int cin, int cout) {
  const int T = tc::taps_per_round(cin, cout);
  const size_t need = (T == 9 ? 1 : 2) * (size_t)tc::stage_bytes(cin, cout, T) + 32;
  const int fit = 512 / tc::tmem_cols(cout);   // CTAs whose accumulators fit
  if (fit >= 16) return need;                 // 16 CTAs of 128 threads fill an SM
  const size_t sm_bytes = 228 * 1024, reserve = 1024;   // per SM, per CTA
  const size_t cap = sm_bytes / (fit + 1) - reserve + 16;   // fit + 1 CTAs no longer fit
  return std::max(need, cap);
}

template <bool F32>
void conv_tc_go(const bf16 *in, int cin, const bf16 *w, const float *bias, void *out, bool accum, int cout,
                int N, int H, int W, cudaStream_t st) {
  static const bool attr = [] {
    SWFWI_CUDA(cudaFuncSetAttribute(k_conv3x3_tc<F32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)conv_tc_smem(128, 256)));   // the largest accepted widths
    return true;
  }();
  (void)attr;
  const long long P = (long long)N * H * W;
  k_conv3x3_tc<F32><<<(unsigned)((P + 127) / 128), 128, conv_tc_smem(cin, cout), st>>>(
      in, cin, w, bias, out, accum ? 1 : 0, cout, N, H, W);
  noted();
}

constexpr int kRedBlocks = 256;           // blocks of the channel sums

// Pixels per chunk of a weight gradient: a multiple of one round (64), about
// 444 CTAs (3 per SM) over the column tiles.
long long wgrad_pix_per_chunk(long long P, int cin) {
  const long long chunks = std::max(1, 444 / wg_tiles(cin));
  return 64 * std::max(1LL, (P + 64 * chunks - 1) / (64 * chunks));
}

size_t wgrad_tc_smem(int cin) {
  const size_t need = 2 * (size_t)wg_stage_bytes(cin) + 32 + 2 * 3 * 64 * 4;
  const int fit = 512 / tc::tmem_cols(wg_cols(cin));   // CTAs whose accumulators fit
  if (fit >= 16) return need;
  const size_t cap = 228 * 1024 / (fit + 1) - 1024 + 16;   // fit + 1 CTAs no longer fit
  return std::max(need, cap);
}

template <int CIN>
void wgrad_tc_cin(const bf16 *dz, int cout, const bf16 *x, float *part, int N, int H, int W, long long ppc,
                  unsigned chunks, cudaStream_t st) {
  static const bool attr = [] {
    SWFWI_CUDA(cudaFuncSetAttribute(k_wgrad_tc<CIN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)wgrad_tc_smem(CIN)));
    return true;
  }();
  (void)attr;
  dim3 grid(chunks, wg_tiles(CIN));
  k_wgrad_tc<CIN><<<grid, 128, wgrad_tc_smem(CIN), st>>>(dz, cout, x, part, N, H, W, (int)ppc);
}

void wgrad_tc_go(const bf16 *dz, int cout, const bf16 *x, int cin, float *dw, float *part, int N, int H, int W,
                 cudaStream_t st) {
  const long long P = (long long)N * H * W;
  const long long ppc = wgrad_pix_per_chunk(P, cin);
  const unsigned chunks = (unsigned)((P + ppc - 1) / ppc);
  switch (cin) {
    case 16: wgrad_tc_cin<16>(dz, cout, x, part, N, H, W, ppc, chunks, st); break;
    case 32: wgrad_tc_cin<32>(dz, cout, x, part, N, H, W, ppc, chunks, st); break;
    case 48: wgrad_tc_cin<48>(dz, cout, x, part, N, H, W, ppc, chunks, st); break;
    case 64: wgrad_tc_cin<64>(dz, cout, x, part, N, H, W, ppc, chunks, st); break;
    case 96: wgrad_tc_cin<96>(dz, cout, x, part, N, H, W, ppc, chunks, st); break;
    case 128: wgrad_tc_cin<128>(dz, cout, x, part, N, H, W, ppc, chunks, st); break;
    default: throw Error(SWFWI_ERR_BAD_ARG, "weight gradient: input width must be 16/32/48/64/96/128");
  }
  noted();
  const long long len = (long long)cout * 9 * cin;
  k_reduce_rows<<<blocks_for(len), kEw, 0, st>>>(part, (int)chunks, len, dw);
  noted();
}

// Channel sums into out[C] (overwritten), in a fixed order.
void chan_sum(const bf16 *a, const float *wgt, long long P, int C, float *out, float *part, cudaStream_t st) {
  k_chan_dot<<<kRedBlocks, kEw, 0, st>>>(a, wgt, P, C, part);
  noted();
  k_reduce_rows<<<1, kEw, 0, st>>>(part, kRedBlocks, C, out);
  noted();
}

int roundup8(int v) { return (v + 7) / 8 * 8; }

}  // namespace

size_t conv_tg_smem(int cin, int cout) {
  const int nky = tg::rows_per_round(cin, cout);
  const size_t need = (nky == 3 ? 1 : 2) * (size_t)tg::stage_bytes(cin, cout, nky) + 24 + 3 * 16 * 4 + 8;
  const int fit = 512 / tc::tmem_cols(cout);
  if (fit >= 16) return need;
  const size_t cap = 228 * 1024 / (fit + 1) - 1024 + 16;
  return std::max(need, cap);
}

template <bool F32, int KC>
void conv_tg_kc(const bf16 *in, const bf16 *w, const float *bias, void *out, bool accum, int cout, int N, int H,
                int W, cudaStream_t st) {
  static const bool attr = [] {
    SWFWI_CUDA(cudaFuncSetAttribute(k_conv3x3_tg<F32, KC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    227 * 1024));
    return true;
  }();
  (void)attr;
  const long long groups = (long long)N * H * ((W + 7) / 8);
  k_conv3x3_tg<F32, KC><<<(unsigned)((groups + 15) / 16), 128, conv_tg_smem(16 * KC, cout), st>>>(
      in, w, bias, out, accum ? 1 : 0, cout, N, H, W);
  noted();
}

// true when a row-tile kernel exists for cin
template <bool F32>
bool conv_tg_go(const bf16 *in, int cin, const bf16 *w, const float *bias, void *out, bool accum, int cout,
                int N, int H, int W, cudaStream_t st) {
  switch (cin / 16) {
    case 1: conv_tg_kc<F32, 1>(in, w, bias, out, accum, cout, N, H, W, st); return true;
    case 2: conv_tg_kc<F32, 2>(in, w, bias, out, accum, cout, N, H, W, st); return true;
    case 3: conv_tg_kc<F32, 3>(in, w, bias, out, accum, cout, N, H, W, st); return true;
    case 4: conv_tg_kc<F32, 4>(in, w, bias, out, accum, cout, N, H, W, st); return true;
    case 6: conv_tg_kc<F32, 6>(in, w, bias, out, accum, cout, N, H, W, st); return true;
    case 8: conv_tg_kc<F32, 8>(in, w, bias, out, accum, cout, N, H, W, st); return true;
    default: return false;
  }
}

void launch_conv3x3(const bf16 *in, int cin, const bf16 *w, const float *bias, void *out,
                    bool out_f32, bool accum, int cout, int N, int H, int W, cudaStream_t st) {
  SWFWI_REQUIRE(cin > 0 && cin % 16 == 0 && cin <= 128 && cout > 0 && cout % 16 == 0 && cout <= 256,
                "conv widths must be multiples of 16, at most 128 in and 256 out");
  SWFWI_REQUIRE(N > 0 && H > 0 && W > 0, "conv image size out of range");
  SWFWI_REQUIRE(out_f32 || bias, "BF16 conv output needs a bias");
  // row tiles (each input row staged once) where their stages fit twice on
  // an SM, else the pixel-run tiles
  const bool rows = conv_tg_smem(cin, cout) <= 100 * 1024;
  if (out_f32) {
    if (!(rows && conv_tg_go<true>(in, cin, w, bias, out, accum, cout, N, H, W, st)))
      conv_tc_go<true>(in, cin, w, bias, out, accum, cout, N, H, W, st);
  } else {
    if (!(rows && conv_tg_go<false>(in, cin, w, bias, out, false, cout, N, H, W, st)))
      conv_tc_go<false>(in, cin, w, bias, out, false, cout, N, H, W, st);
  }
}

size_t conv3x3_wgrad_scratch(int cout, int cin, int N, int H, int W) {
  const long long P = (long long)N * H * W;
  const long long ppc = wgrad_pix_per_chunk(P, cin);
  return (size_t)((P + ppc - 1) / ppc) * cout * 9 * cin;
}

void launch_conv3x3_wgrad(const bf16 *dz, int cout, const bf16 *x, int cin, float *dw, float *scratch,
                          size_t scratch_floats, int N, int H, int W, cudaStream_t st) {
  SWFWI_REQUIRE(cout > 0 && cout % 16 == 0 && cout <= 128, "weight gradient: output width must be a multiple of 16, at most 128");
  SWFWI_REQUIRE(cin == 16 || cin == 32 || cin == 48 || cin == 64 || cin == 96 || cin == 128,
                "weight gradient: input width must be 16/32/48/64/96/128");
  SWFWI_REQUIRE(scratch && scratch_floats >= conv3x3_wgrad_scratch(cout, cin, N, H, W),
                "weight gradient scratch too small");
  wgrad_tc_go(dz, cout, x, cin, dw, scratch, N, H, W, st);
}

void launch_illum_accum(float *illum, const float *p, long long fstride, int n, int nxpad, int nzpad,
                        int pitch, cudaStream_t st) {
  const long long total = (long long)nxpad * nzpad;
  k_illum<<<blocks_for(total), kEw, 0, st>>>(illum, p, fstride, n, nxpad, nzpad, pitch);
  noted();
}

// ------------------------------------------------------------------ network
Preconditioner::Preconditioner(const int widths[4]) {
  for (int i = 0; i < 4; i++) {
    SWFWI_REQUIRE(widths[i] > 0 && widths[i] % 16 == 0 && widths[i] <= 64,
                  "preconditioner widths must be multiples of 16 up to 64");
    w_[i] = widths[i];
  }
  const int c0 = w_[0], c1 = w_[1], c2 = w_[2], c3 = w_[3];
  const int io[kConvs][2] = {{kInCh, c0}, {c0, c0}, {c0, c1}, {c1, c1}, {c1, c2},
                             {c2, c2},    {c2, c3}, {c3, c3}, {c3 + c2, c2}, {c2, c2},
                             {c2 + c1, c1}, {c1, c1}, {c1 + c0, c0}, {c0, c0}};
  long long off = 0;
  size_t maxw = 0;
  for (int l = 0; l < kConvs; l++) {
    ConvSpec s{io[l][0], io[l][1], 0, 0};
    s.w_off = off;
    off += (long long)s.cout * 9 * s.cin;
    s.b_off = off;
    off += s.cout;
    maxw = std::max(maxw, (size_t)s.cout * 9 * s.cin);
    conv_.push_back(s);
  }
  out_w_ = off;
  off += c0;
  out_b_ = off;
  off += 1;
  nparam_ = off;
  params_.resize(nparam_);
  grads_.resize(nparam_);
  m_.resize(nparam_);
  v_.resize(nparam_);
  wbf_.resize(nparam_);
  wflip_.resize(maxw);
  red_.resize(8 + 4 * 256);   // loss, statistics and their per-block partials
  // He-uniform conv weights, zero biases, small output layer (seeded)
  std::vector<float> h(nparam_, 0.0f);
  std::mt19937 gen(12345u);
  for (const ConvSpec &s : conv_) {
    const float lim = std::sqrt(6.0f / (9.0f * s.cin));
    std::uniform_real_distribution<float> U(-lim, lim);
    for (long long i = 0; i < (long long)s.cout * 9 * s.cin; i++) h[s.w_off + i] = U(gen);
  }
  {
    const float lim = 1.0f / std::sqrt((float)c0);
    std::uniform_real_distribution<float> U(-lim, lim);
    for (int i = 0; i < c0; i++) h[out_w_ + i] = U(gen);
  }
  set_params(h.data());
}

void Preconditioner::refresh_bf16() {
  k_to_bf16<<<blocks_for(nparam_), kEw, 0, st_>>>(params_.get(), wbf_.get(), nparam_);
  noted();
}

void Preconditioner::set_params(const float *host) {
  SWFWI_REQUIRE(host, "null parameters");
  params_.upload(host, nparam_, st_);
  refresh_bf16();
  reset_optimizer();
}

void Preconditioner::reset_optimizer() {
  m_.zero(st_);
  v_.zero(st_);
  grads_.zero(st_);
  step_ = 0;
  SWFWI_CUDA(cudaStreamSynchronize(st_));
}

void Preconditioner::get_params(float *host) {
  SWFWI_CUDA(cudaMemcpyAsync(host, params_.get(), sizeof(float) * nparam_, cudaMemcpyDeviceToHost, st_));
  SWFWI_CUDA(cudaStreamSynchronize(st_));
}

void Preconditioner::get_grads(float *host) {
  SWFWI_CUDA(cudaMemcpyAsync(host, grads_.get(), sizeof(float) * nparam_, cudaMemcpyDeviceToHost, st_));
  SWFWI_CUDA(cudaStreamSynchronize(st_));
}

void Preconditioner::conv_fwd(int l, const bf16 *in, bf16 *out, long long, int H, int W) {
  const ConvSpec &s = conv_[l];
  launch_conv3x3(in, s.cin, wbf_.get() + s.w_off, params_.get() + s.b_off, out, false, false, s.cout,
                 N_, H, W, st_);
}

void Preconditioner::forward(const float *x, float *y, int N, int H, int W) {
  SWFWI_REQUIRE(x && N > 0 && H > 0 && W > 0 && H % 8 == 0 && W % 8 == 0,
                "network input must be N x H x W with H and W multiples of 8");
  SWFWI_REQUIRE((long long)N * H <= 65535, "network batch too large");
  N_ = N;
  H_ = H;
  W_ = W;
  const int c0 = w_[0], c1 = w_[1], c2 = w_[2], c3 = w_[3];
  const long long P0 = (long long)N * H * W, P1 = P0 / 4, P2 = P0 / 16, P3 = P0 / 64;
  x16_.resize(P0 * kInCh);
  a0_.resize(P0 * c0); s0_.resize(P0 * c0); p0_.resize(P1 * c0);
  a1_.resize(P1 * c1); s1_.resize(P1 * c1); p1_.resize(P2 * c1);
  a2_.resize(P2 * c2); s2_.resize(P2 * c2); p2_.resize(P3 * c2);
  a3_.resize(P3 * c3); b3_.resize(P3 * c3);
  cat2_.resize(P2 * (c3 + c2)); a4_.resize(P2 * c2); u2_.resize(P2 * c2);
  cat1_.resize(P1 * (c2 + c1)); a5_.resize(P1 * c1); u1_.resize(P1 * c1);
  cat0_.resize(P0 * (c1 + c0)); a6_.resize(P0 * c0); u0_.resize(P0 * c0);
  y_.resize(P0);
  k_pack3<<<blocks_for(P0), kEw, 0, st_>>>(x, x16_.get(), P0);
  noted();
  const int H1 = H / 2, W1 = W / 2, H2 = H / 4, W2 = W / 4, H3 = H / 8, W3 = W / 8;
  conv_fwd(0, x16_.get(), a0_.get(), P0, H, W);
  conv_fwd(1, a0_.get(), s0_.get(), P0, H, W);
  k_pool<<<blocks_for(P1 * c0 / 2), kEw, 0, st_>>>(s0_.get(), p0_.get(), N, H, W, c0);
  noted();
  conv_fwd(2, p0_.get(), a1_.get(), P1, H1, W1);
  conv_fwd(3, a1_.get(), s1_.get(), P1, H1, W1);
  k_pool<<<blocks_for(P2 * c1 / 2), kEw, 0, st_>>>(s1_.get(), p1_.get(), N, H1, W1, c1);
  noted();
  conv_fwd(4, p1_.get(), a2_.get(), P2, H2, W2);
  conv_fwd(5, a2_.get(), s2_.get(), P2, H2, W2);
  k_pool<<<blocks_for(P3 * c2 / 2), kEw, 0, st_>>>(s2_.get(), p2_.get(), N, H2, W2, c2);
  noted();
  conv_fwd(6, p2_.get(), a3_.get(), P3, H3, W3);
  conv_fwd(7, a3_.get(), b3_.get(), P3, H3, W3);
  k_upcat<<<blocks_for(P2 * (c3 + c2) / 2), kEw, 0, st_>>>(b3_.get(), c3, s2_.get(), c2, cat2_.get(), N, H2, W2);
  noted();
  conv_fwd(8, cat2_.get(), a4_.get(), P2, H2, W2);
  conv_fwd(9, a4_.get(), u2_.get(), P2, H2, W2);
  k_upcat<<<blocks_for(P1 * (c2 + c1) / 2), kEw, 0, st_>>>(u2_.get(), c2, s1_.get(), c1, cat1_.get(), N, H1, W1);
  noted();
  conv_fwd(10, cat1_.get(), a5_.get(), P1, H1, W1);
  conv_fwd(11, a5_.get(), u1_.get(), P1, H1, W1);
  k_upcat<<<blocks_for(P0 * (c1 + c0) / 2), kEw, 0, st_>>>(u1_.get(), c1, s0_.get(), c0, cat0_.get(), N, H, W);
  noted();
  conv_fwd(12, cat0_.get(), a6_.get(), P0, H, W);
  conv_fwd(13, a6_.get(), u0_.get(), P0, H, W);
  k_out_fwd<<<blocks_for(P0), kEw, 0, st_>>>(u0_.get(), params_.get() + out_w_, params_.get() + out_b_,
                                              y_.get(), P0, c0);
  noted();
  if (y) SWFWI_CUDA(cudaMemcpyAsync(y, y_.get(), sizeof(float) * P0, cudaMemcpyDeviceToDevice, st_));
}

void Preconditioner::conv_bwd(int l, const bf16 *in, const bf16 *out, const float *dY, float *dX,
                              int H, int W) {
  const ConvSpec &s = conv_[l];
  const long long P = (long long)N_ * H * W;
  k_relu_mask<<<blocks_for(P * s.cout), kEw, 0, st_>>>(dY, out, dz_.get(), P * s.cout);
  noted();
  chan_sum(dz_.get(), nullptr, P, s.cout, grads_.get() + s.b_off, part_.get(), st_);
  launch_conv3x3_wgrad(dz_.get(), s.cout, in, s.cin, grads_.get() + s.w_off, part_.get(), part_.size(), N_, H, W,
                       st_);
  if (dX) {
    k_flip<<<blocks_for((long long)s.cout * 9 * s.cin), kEw, 0, st_>>>(wbf_.get() + s.w_off, wflip_.get(),
                                                                        s.cout, s.cin);
    noted();
    launch_conv3x3(dz_.get(), s.cout, wflip_.get(), nullptr, dX, true, false, s.cin, N_, H, W, st_);
  }
}

double Preconditioner::backward(const float *t) {
  SWFWI_REQUIRE(t && N_ > 0, "backward needs a forward and a target");
  const int N = N_, H = H_, W = W_;
  const int c0 = w_[0], c1 = w_[1], c2 = w_[2], c3 = w_[3];
  const long long P0 = (long long)N * H * W, P1 = P0 / 4, P2 = P0 / 16, P3 = P0 / 64;
  const int H1 = H / 2, W1 = W / 2, H2 = H / 4, W2 = W / 4, H3 = H / 8, W3 = W / 8;
  const long long big = std::max({P0 * (c1 + c0), P1 * (c2 + c1), P2 * (c3 + c2), P0 * c0});
  dy_.resize(P0);
  dA_.resize(big);
  dB_.resize(big);
  dCat_.resize(big);
  dLow_.resize(big);
  dS0_.resize(P0 * c0);
  dS1_.resize(P1 * c1);
  dS2_.resize(P2 * c2);
  dz_.resize(big);
  size_t need = (size_t)kRedBlocks * 64;
  {
    const int hw[4][2] = {{H, W}, {H1, W1}, {H2, W2}, {H3, W3}};
    const int level[kConvs] = {0, 0, 1, 1, 2, 2, 3, 3, 2, 2, 1, 1, 0, 0};
    for (int l = 0; l < kConvs; l++)
      need = std::max(need, conv3x3_wgrad_scratch(conv_[l].cout, conv_[l].cin, N, hw[level[l]][0],
                                                  hw[level[l]][1]));
  }
  part_.resize(need);
  grads_.zero(st_);
  red_.zero(st_);
  k_mse<<<blocks_for(P0), kEw, 0, st_>>>(y_.get(), t, dy_.get(), P0, 2.0f / (float)P0, red_.get());
  noted();
  // output layer
  chan_sum(u0_.get(), dy_.get(), P0, c0, grads_.get() + out_w_, part_.get(), st_);
  k_sum<<<kRedBlocks, kEw, 0, st_>>>(dy_.get(), P0, part_.get());
  noted();
  k_reduce_rows<<<1, kEw, 0, st_>>>(part_.get(), kRedBlocks, 1, grads_.get() + out_b_);
  noted();
  k_out_bwd_dx<<<blocks_for(P0 * c0), kEw, 0, st_>>>(dy_.get(), params_.get() + out_w_, dA_.get(), P0, c0);
  noted();
  // decoder level 0
  conv_bwd(13, a6_.get(), u0_.get(), dA_.get(), dB_.get(), H, W);
  conv_bwd(12, cat0_.get(), a6_.get(), dB_.get(), dCat_.get(), H, W);
  k_upcat_bwd_low<<<blocks_for(P1 * c1), kEw, 0, st_>>>(dCat_.get(), c1 + c0, c1, dLow_.get(), N, H1, W1);
  noted();
  k_upcat_bwd_skip<<<blocks_for(P0 * c0), kEw, 0, st_>>>(dCat_.get(), c1 + c0, c1, dS0_.get(), P0, c0);
  noted();
  // decoder level 1
  conv_bwd(11, a5_.get(), u1_.get(), dLow_.get(), dA_.get(), H1, W1);
  conv_bwd(10, cat1_.get(), a5_.get(), dA_.get(), dCat_.get(), H1, W1);
  k_upcat_bwd_low<<<blocks_for(P2 * c2), kEw, 0, st_>>>(dCat_.get(), c2 + c1, c2, dLow_.get(), N, H2, W2);
  noted();
  k_upcat_bwd_skip<<<blocks_for(P1 * c1), kEw, 0, st_>>>(dCat_.get(), c2 + c1, c2, dS1_.get(), P1, c1);
  noted();
  // decoder level 2
  conv_bwd(9, a4_.get(), u2_.get(), dLow_.get(), dA_.get(), H2, W2);
  conv_bwd(8, cat2_.get(), a4_.get(), dA_.get(), dCat_.get(), H2, W2);
  k_upcat_bwd_low<<<blocks_for(P3 * c3), kEw, 0, st_>>>(dCat_.get(), c3 + c2, c3, dLow_.get(), N, H3, W3);
  noted();
  k_upcat_bwd_skip<<<blocks_for(P2 * c2), kEw, 0, st_>>>(dCat_.get(), c3 + c2, c3, dS2_.get(), P2, c2);
  noted();
  // bottleneck
  conv_bwd(7, a3_.get(), b3_.get(), dLow_.get(), dA_.get(), H3, W3);
  conv_bwd(6, p2_.get(), a3_.get(), dA_.get(), dB_.get(), H3, W3);
  k_pool_bwd<<<blocks_for(P2 * c2), kEw, 0, st_>>>(dB_.get(), dS2_.get(), N, H2, W2, c2);
  noted();
  // encoder level 2
  conv_bwd(5, a2_.get(), s2_.get(), dS2_.get(), dA_.get(), H2, W2);
  conv_bwd(4, p1_.get(), a2_.get(), dA_.get(), dB_.get(), H2, W2);
  k_pool_bwd<<<blocks_for(P1 * c1), kEw, 0, st_>>>(dB_.get(), dS1_.get(), N, H1, W1, c1);
  noted();
  // encoder level 1
  conv_bwd(3, a1_.get(), s1_.get(), dS1_.get(), dA_.get(), H1, W1);
  conv_bwd(2, p0_.get(), a1_.get(), dA_.get(), dB_.get(), H1, W1);
  k_pool_bwd<<<blocks_for(P0 * c0), kEw, 0, st_>>>(dB_.get(), dS0_.get(), N, H, W, c0);
  noted();
  // encoder level 0
  conv_bwd(1, a0_.get(), s0_.get(), dS0_.get(), dA_.get(), H, W);
  conv_bwd(0, x16_.get(), a0_.get(), dA_.get(), nullptr, H, W);
  double loss = 0;
  SWFWI_CUDA(cudaMemcpyAsync(&loss, red_.get(), sizeof(double), cudaMemcpyDeviceToHost, st_));
  SWFWI_CUDA(cudaStreamSynchronize(st_));
  int timeout = 0;
  SWFWI_CUDA(cudaMemcpyFromSymbol(&timeout, g_conv_timeout, sizeof(int)));
  if (timeout) {
    const int zero = 0;
    SWFWI_CUDA(cudaMemcpyToSymbol(g_conv_timeout, &zero, sizeof(int)));
    throw Error(SWFWI_ERR_TIMEOUT, "a convolution's bounded wait on its tensor-core MMAs gave up");
  }
  if (!std::isfinite(loss)) throw Error(SWFWI_ERR_NONFINITE, "preconditioner loss is not finite");
  return loss / (double)P0;
}

void Preconditioner::adam_step(float lr, float beta1, float beta2, float eps) {
  step_++;
  const double bc1 = 1.0 - std::pow((double)beta1, (double)step_);
  const double bc2 = 1.0 - std::pow((double)beta2, (double)step_);
  const float lr_t = (float)(lr * std::sqrt(bc2) / bc1);
  k_adam<<<blocks_for(nparam_), kEw, 0, st_>>>(params_.get(), m_.get(), v_.get(), grads_.get(), nparam_,
                                               lr_t, beta1, beta2, eps);
  noted();
  refresh_bf16();
}

double Preconditioner::train_step(const float *x, const float *t, int N, int H, int W, float lr) {
  forward(x, nullptr, N, H, W);
  const double loss = backward(t);
  adam_step(lr);
  return loss;
}

void Preconditioner::stats(const float *a, const float *b, const float *c, int nzpad, int x0, int z0, int nx,
                           int nz) {
  constexpr int blocks = 256;
  red_.resize(8 + 4 * blocks);
  k_stats<<<blocks, kEw, 0, st_>>>(a, b, c, nzpad, x0, z0, nx, nz, red_.get() + 8);
  noted();
  k_stats_final<<<1, 1, 0, st_>>>(red_.get() + 8, blocks, red_.get());
  noted();
}

void Preconditioner::features(const float *grad, const float *vel, const float *illum, int nxpad,
                              int nzpad, int bx0, int bxn, int bz0, int bzn, float *x3) {
  SWFWI_REQUIRE(grad && vel && x3, "null field");
  const int nx = nxpad - bx0 - bxn, nz = nzpad - bz0 - bzn;
  SWFWI_REQUIRE(nx > 0 && nz > 0, "empty interior");
  const int Hp = roundup8(nx), Wp = roundup8(nz);
  stats(grad, vel, illum, nzpad, bx0, bz0, nx, nz);
  k_features<<<blocks_for((long long)Hp * Wp), kEw, 0, st_>>>(grad, vel, illum, nzpad, bx0, bz0, nx, nz, Hp,
                                                                Wp, red_.get(), x3);
  noted();
}

void Preconditioner::target(const float *dv, int nxpad, int nzpad, int bx0, int bxn, int bz0, int bzn,
                            float *t) {
  SWFWI_REQUIRE(dv && t, "null field");
  const int nx = nxpad - bx0 - bxn, nz = nzpad - bz0 - bzn;
  SWFWI_REQUIRE(nx > 0 && nz > 0, "empty interior");
  const int Hp = roundup8(nx), Wp = roundup8(nz);
  stats(dv, nullptr, nullptr, nzpad, bx0, bz0, nx, nz);
  k_target<<<blocks_for((long long)Hp * Wp), kEw, 0, st_>>>(dv, nzpad, bx0, bz0, nx, nz, Hp, Wp, red_.get(), t);
  noted();
}

void Preconditioner::scatter(const float *y, int nxpad, int nzpad, int bx0, int bxn, int bz0, int bzn,
                             float *dir) {
  SWFWI_REQUIRE(y && dir, "null field");
  const int nx = nxpad - bx0 - bxn, nz = nzpad - bz0 - bzn;
  SWFWI_REQUIRE(nx > 0 && nz > 0, "empty interior");
  SWFWI_CUDA(cudaMemsetAsync(dir, 0, sizeof(float) * (size_t)nxpad * nzpad, st_));
  k_scatter<<<blocks_for((long long)nx * nz), kEw, 0, st_>>>(y, nzpad, bx0, bz0, nx, nz, roundup8(nz), dir);
  noted();
}

void Preconditioner::propose(const float *grad, const float *vel, const float *illum, int nxpad,
                             int nzpad, int bx0, int bxn, int bz0, int bzn, float *dir) {
  const int nx = nxpad - bx0 - bxn, nz = nzpad - bz0 - bzn;
  const int Hp = roundup8(nx), Wp = roundup8(nz);
  feat_.resize((size_t)Hp * Wp * 3);
  outimg_.resize((size_t)Hp * Wp);
  features(grad, vel, illum, nxpad, nzpad, bx0, bxn, bz0, bzn, feat_.get());
  forward(feat_.get(), outimg_.get(), 1, Hp, Wp);
  scatter(outimg_.get(), nxpad, nzpad, bx0, bxn, bz0, bzn, dir);
}

}  // namespace swfwi
