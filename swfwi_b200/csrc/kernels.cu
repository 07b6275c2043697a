// Kernels around the stencil; see kernels.cuh for the reference citations.
#include <climits>
#include <atomic>
#include <cmath>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include "common.hpp"
#include "kernels.cuh"
#include "swfwi_gpu.h"

namespace swfwi {

std::atomic<long long> g_kernel_launches{0};
namespace {
thread_local long long t_launches = 0;   // this thread's launches (captures count their own)
}
void note_launch() {
  g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  ++t_launches;
}
long long thread_launches() { return t_launches; }

namespace {
constexpr int kThreads = 256;
inline unsigned grid_for(long long n, int threads = kThreads) {
  long long g = (n + threads - 1) / threads;
  return (unsigned)(g < 1 ? 1 : (g > 2147483647LL ? 2147483647LL : g));
}

// Exact float add/sub regardless of the caller's arithmetic mode: the
// reference's manipSource is one float operation per point.
template <typename T>
__device__ __forceinline__ T exact_add(T a, T b) { return a + b; }
template <>
__device__ __forceinline__ float exact_add<float>(float a, float b) { return __fadd_rn(a, b); }
template <typename T>
__device__ __forceinline__ T exact_sub(T a, T b) { return a - b; }
template <>
__device__ __forceinline__ float exact_sub<float>(float a, float b) { return __fsub_rn(a, b); }

// Deterministic FP64 block reduction with warp shuffles.
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
}  // namespace

// ---------------------------------------------------------------- inject
template <typename T>
__global__ void k_inject(T *field, long long shot_stride, int nslots, PointSet ps, const T *vals,
                         long long val_slot_stride, int val_stride, int sign) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int slot = blockIdx.y;
  if (i >= ps.per_shot || slot >= nslots) return;
  int shot = ps.slot_shot ? ps.slot_shot[slot] : slot;
  int p = ps.pos[(long long)shot * ps.per_shot + i];
  if (p < 0) return;
  T v = vals[(long long)slot * val_slot_stride + (long long)i * val_stride];
  T *f = field + (long long)slot * shot_stride + p;
  *f = sign > 0 ? exact_add<T>(*f, v) : exact_sub<T>(*f, v);
}

template <typename T>
void launch_inject(T *field, long long shot_stride, int nslots, PointSet ps, const T *vals,
                   long long val_slot_stride, int val_stride, int sign, cudaStream_t st) {
  if (nslots <= 0 || ps.per_shot <= 0) return;
  dim3 g(grid_for(ps.per_shot, 128), nslots);
  k_inject<T><<<g, 128, 0, st>>>(field, shot_stride, nslots, ps, vals, val_slot_stride, val_stride,
                                 sign);
  note_launch();
}

// ---------------------------------------------------------------- record
template <typename T>
__global__ void k_record(T *seis, long long seis_slot_stride, const T *field, long long shot_stride,
                         int nslots, PointSet ps) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int slot = blockIdx.y;
  if (i >= ps.per_shot || slot >= nslots) return;
  int shot = ps.slot_shot ? ps.slot_shot[slot] : slot;
  int p = ps.pos[(long long)shot * ps.per_shot + i];
  seis[(long long)slot * seis_slot_stride + i] = p < 0 ? T(0) : field[(long long)slot * shot_stride + p];
}

template <typename T>
void launch_record(T *seis, long long seis_slot_stride, const T *field, long long shot_stride,
                   int nslots, PointSet ps, cudaStream_t st) {
  if (nslots <= 0 || ps.per_shot <= 0) return;
  dim3 g(grid_for(ps.per_shot, 128), nslots);
  k_record<T><<<g, 128, 0, st>>>(seis, seis_slot_stride, field, shot_stride, nslots, ps);
  note_launch();
}

// ---------------------------------------------------------------- strips
int strip_size(int nx, int nz, int bx0) {
  return 6 * ((nx - 2 * (bx0 - 6)) + 2 * (nz - 6 - bx0));
}

// Strip element i -> padded field index.  Bottom: 6 rows below the
// interior, x from bx0-6 to nx-bx0+6, stored [ix][iz]; then the left and
// right 6-column bands over the interior depth, stored [ix][iz].
__device__ __forceinline__ long long strip_index(int i, int nx, int nz, int bx0, int pitch) {
  const int w = 6, nxs = nx - 2 * (bx0 - w), nzs = nz - 6 - bx0;
  if (i < w * nxs) {
    int ix = i / w, iz = i - ix * w;
    return (long long)(ix + bx0 - w) * pitch + (nz - bx0 + iz);
  }
  int j = i - w * nxs;
  int ix = j / nzs, iz = j - ix * nzs;
  int gx = ix < w ? (bx0 - w + ix) : (nx - bx0 + ix - w);
  return (long long)gx * pitch + (6 + iz);
}

template <typename T, bool WRITE>
__global__ void k_strip(T *bndr, long long bndr_slot_stride, T *field, long long shot_stride, int bs,
                        int nx, int nz, int bx0, int pitch) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int slot = blockIdx.y;
  if (i >= bs) return;
  long long p = strip_index(i, nx, nz, bx0, pitch);
  T *f = field + (long long)slot * shot_stride + p;
  T *b = bndr + (long long)slot * bndr_slot_stride + i;
  if (WRITE) *b = *f; else *f = *b;
}

template <typename T>
void launch_strip_write(T *bndr, long long bndr_slot_stride, const T *field, long long shot_stride,
                        int nslots, int nx, int nz, int bx0, int pitch, cudaStream_t st) {
  int bs = strip_size(nx, nz, bx0);
  dim3 g(grid_for(bs), nslots);
  k_strip<T, true><<<g, kThreads, 0, st>>>(bndr, bndr_slot_stride, const_cast<T *>(field), shot_stride,
                                            bs, nx, nz, bx0, pitch);
  note_launch();
}

template <typename T>
void launch_strip_read(const T *bndr, long long bndr_slot_stride, T *field, long long shot_stride,
                       int nslots, int nx, int nz, int bx0, int pitch, cudaStream_t st) {
  int bs = strip_size(nx, nz, bx0);
  dim3 g(grid_for(bs), nslots);
  k_strip<T, false><<<g, kThreads, 0, st>>>(const_cast<T *>(bndr), bndr_slot_stride, field,
                                             shot_stride, bs, nx, nz, bx0, pitch);
  note_launch();
}

// ---------------------------------------------------------------- fused small steps
// The point work around one stencil step, in one launch instead of up to
// three.  After a forward step: record the current field, save its FP32
// strips, and add the next step's source into the other field
// (FwiForwardModeling and calgradient's forward, damp4t10d.cpp:283-288,
// fwiframework.cpp:137-144).  The first two read `cur`, the third writes
// `next`, so the three commute; each element is the same single operation
// as in k_record, k_strip and k_inject.  Grid (blocks over the longest of
// the three lists, slots).
// Each thread takes kSmallE elements a grid-stride apart and issues every
// load of its elements before any store: the position gathers and the
// field reads of the four overlap instead of running as four dependent
// chains (these launches are latency-bound).  The loads and stores touch
// disjoint arrays (cur vs seis, bndr and next), so the order changes no bits.
constexpr int kSmallE = 4;

template <typename T>
__global__ void k_after_forward(T *seis, long long seis_slot_stride, const T *cur, PointSet rec, T *bndr,
                                long long bndr_slot_stride, int bs, int nx, int nz, int bx0, int pitch, T *next,
                                PointSet src, const T *vals, long long val_slot_stride, int val_stride,
                                long long shot_stride, int most) {
  const int slot = blockIdx.y;
  const long long off = (long long)slot * shot_stride;
  const int stride = gridDim.x * blockDim.x;
  const int rshot = rec.slot_shot ? rec.slot_shot[slot] : slot;
  const int sshot = src.slot_shot ? src.slot_shot[slot] : slot;
  for (int i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < most; i0 += kSmallE * stride) {
    int rp[kSmallE], sp[kSmallE];
#pragma unroll
    for (int e = 0; e < kSmallE; e++) {
      const int i = i0 + e * stride;
      rp[e] = (seis && i < rec.per_shot) ? rec.pos[(long long)rshot * rec.per_shot + i] : INT_MIN;
      sp[e] = (next && i < src.per_shot) ? src.pos[(long long)sshot * src.per_shot + i] : -1;
    }
    T rv[kSmallE], bv[kSmallE], nv[kSmallE], vv[kSmallE];
#pragma unroll
    for (int e = 0; e < kSmallE; e++) {
      const int i = i0 + e * stride;
      rv[e] = rp[e] >= 0 ? cur[off + rp[e]] : T(0);
      bv[e] = (bndr && i < bs) ? cur[off + strip_index(i, nx, nz, bx0, pitch)] : T(0);
      if (sp[e] >= 0) {
        nv[e] = next[off + sp[e]];
        vv[e] = vals[(long long)slot * val_slot_stride + (long long)i * val_stride];
      }
    }
#pragma unroll
    for (int e = 0; e < kSmallE; e++) {
      const int i = i0 + e * stride;
      if (rp[e] != INT_MIN) seis[(long long)slot * seis_slot_stride + i] = rv[e];   // position < 0: 0
      if (bndr && i < bs) bndr[(long long)slot * bndr_slot_stride + i] = bv[e];
      if (sp[e] >= 0) next[off + sp[e]] = exact_add<T>(nv[e], vv[e]);
    }
  }
}

template <typename T>
void launch_after_forward(T *seis, long long seis_slot_stride, const T *cur, PointSet rec, T *bndr,
                          long long bndr_slot_stride, int nx, int nz, int bx0, int pitch, T *next, PointSet src,
                          const T *vals, long long val_slot_stride, int val_stride, long long shot_stride,
                          int nslots, cudaStream_t st) {
  if (nslots <= 0) return;
  const int bs = bndr ? strip_size(nx, nz, bx0) : 0;
  const int nr = seis ? rec.per_shot : 0, ni = next ? src.per_shot : 0;
  const int most = nr > bs ? (nr > ni ? nr : ni) : (bs > ni ? bs : ni);
  if (most <= 0) return;
  const dim3 g(grid_for(most, 128 * kSmallE), nslots);
  k_after_forward<T><<<g, 128, 0, st>>>(seis, seis_slot_stride, cur, rec, bndr, bndr_slot_stride, bs, nx, nz, bx0,
                                        pitch, next, src, vals, val_slot_stride, val_stride, shot_stride, most);
  note_launch();
}

// Two injections into two different fields in one launch (calgradient's
// backward step, fwiframework.cpp:152-160: subSource on the back-stepped
// source field, addSource of the residual on the receiver field).  The same
// single float operation per point as k_inject.
template <typename T>
__global__ void k_inject2(T *fa, PointSet pa, const T *va, long long va_slot_stride, int va_stride, int sign_a,
                          T *fb, PointSet pb, const T *vb, long long vb_slot_stride, int vb_stride, int sign_b,
                          long long shot_stride, const T *bndr, long long bndr_slot_stride, int bs, int nx, int nz,
                          int bx0, int pitch, int most) {
  const int slot = blockIdx.y;
  const long long off = (long long)slot * shot_stride;
  const int stride = gridDim.x * blockDim.x;
  const int ashot = pa.slot_shot ? pa.slot_shot[slot] : slot;
  const int bshot = pb.slot_shot ? pb.slot_shot[slot] : slot;
  // as k_after_forward: all loads of a thread's elements before its stores;
  // the strip band and the source and receiver points are disjoint cells
  for (int i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < most; i0 += kSmallE * stride) {
    int ap[kSmallE], bp[kSmallE];
#pragma unroll
    for (int e = 0; e < kSmallE; e++) {
      const int i = i0 + e * stride;
      ap[e] = i < pa.per_shot ? pa.pos[(long long)ashot * pa.per_shot + i] : -1;
      bp[e] = i < pb.per_shot ? pb.pos[(long long)bshot * pb.per_shot + i] : -1;
    }
    T sv[kSmallE], af[kSmallE], av[kSmallE], bf[kSmallE], bv[kSmallE];
#pragma unroll
    for (int e = 0; e < kSmallE; e++) {
      const int i = i0 + e * stride;
      sv[e] = (bndr && i < bs) ? bndr[(long long)slot * bndr_slot_stride + i] : T(0);
      if (ap[e] >= 0) {
        af[e] = fa[off + ap[e]];
        av[e] = va[(long long)slot * va_slot_stride + (long long)i * va_stride];
      }
      if (bp[e] >= 0) {
        bf[e] = fb[off + bp[e]];
        bv[e] = vb[(long long)slot * vb_slot_stride + (long long)i * vb_stride];
      }
    }
#pragma unroll
    for (int e = 0; e < kSmallE; e++) {
      const int i = i0 + e * stride;
      if (bndr && i < bs) fa[off + strip_index(i, nx, nz, bx0, pitch)] = sv[e];
      if (ap[e] >= 0) fa[off + ap[e]] = sign_a > 0 ? exact_add<T>(af[e], av[e]) : exact_sub<T>(af[e], av[e]);
      if (bp[e] >= 0) fb[off + bp[e]] = sign_b > 0 ? exact_add<T>(bf[e], bv[e]) : exact_sub<T>(bf[e], bv[e]);
    }
  }
}

template <typename T>
void launch_inject2(T *fa, PointSet pa, const T *va, long long va_slot_stride, int va_stride, int sign_a, T *fb,
                    PointSet pb, const T *vb, long long vb_slot_stride, int vb_stride, int sign_b,
                    long long shot_stride, int nslots, cudaStream_t st, const T *bndr, long long bndr_slot_stride,
                    int nx, int nz, int bx0, int pitch) {
  if (nslots <= 0) return;
  const int bs = bndr ? strip_size(nx, nz, bx0) : 0;
  int most = pa.per_shot > pb.per_shot ? pa.per_shot : pb.per_shot;
  most = most > bs ? most : bs;
  if (most <= 0) return;
  const dim3 g(grid_for(most, 128 * kSmallE), nslots);
  k_inject2<T><<<g, 128, 0, st>>>(fa, pa, va, va_slot_stride, va_stride, sign_a, fb, pb, vb, vb_slot_stride,
                                  vb_stride, sign_b, shot_stride, bndr, bndr_slot_stride, bs, nx, nz, bx0, pitch,
                                  most);
  note_launch();
}

// ---------------------------------------------------------------- image
template <typename T>
__global__ void k_image(T *image, long long image_stride, const T *s, const T *r,
                        long long shot_stride, int n, float scale) {
  int slot = blockIdx.y;
  T *g = image + (long long)slot * image_stride;
  const T *a = s + (long long)slot * shot_stride;
  const T *b = r + (long long)slot * shot_stride;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if constexpr (sizeof(T) == 4) {
      g[i] = __fsub_rn(g[i], __fmul_rn(__fmul_rn(a[i], b[i]), scale));
    } else {
      g[i] = g[i] - a[i] * b[i] * (double)scale;
    }
  }
}

// All slots' cross-correlations into one image (FAST arithmetic):
// image[p] -= (sum over slots, in slot order, of s*r) * scale, four points
// a thread; one image read-modify-write for all slots.  n % 4 == 0 and
// every array 16-byte aligned.
__global__ void __launch_bounds__(kThreads)
k_image_sum(float *image, const float *s, const float *r, long long shot_stride, int nslots, int x0, int nrows,
            int g0, int ngroups, int pitch4, float scale) {
  const int n = nrows * ngroups;
  const long long st4 = shot_stride / 4;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const int row = q / ngroups;
    const long long e = (long long)(x0 + row) * pitch4 + g0 + (q - row * ngroups);   // float4 index
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 *a = reinterpret_cast<const float4 *>(s) + e;
    const float4 *b = reinterpret_cast<const float4 *>(r) + e;
#pragma unroll 8
    for (int slot = 0; slot < nslots; slot++) {
      const float4 x = __ldcs(a + slot * st4), y = __ldcs(b + slot * st4);
      acc.x = fmaf(x.x, y.x, acc.x);
      acc.y = fmaf(x.y, y.y, acc.y);
      acc.z = fmaf(x.z, y.z, acc.z);
      acc.w = fmaf(x.w, y.w, acc.w);
    }
    float4 *g = reinterpret_cast<float4 *>(image) + e;
    float4 v = *g;
    v.x = __fsub_rn(v.x, __fmul_rn(acc.x, scale));
    v.y = __fsub_rn(v.y, __fmul_rn(acc.y, scale));
    v.z = __fsub_rn(v.z, __fmul_rn(acc.z, scale));
    v.w = __fsub_rn(v.w, __fmul_rn(acc.w, scale));
    *g = v;
  }
}

void launch_image_sum(float *image, const float *s, const float *r, long long shot_stride, int nslots, int x0,
                      int x1, int z0, int z1, int pitch, float scale, cudaStream_t st) {
  if (pitch % 4 != 0 || shot_stride % 4 != 0 || (reinterpret_cast<uintptr_t>(image) |
                                                  reinterpret_cast<uintptr_t>(s) | reinterpret_cast<uintptr_t>(r)) %
                                                     16 != 0)
    throw Error(SWFWI_ERR_BAD_ARG, "summed image: sizes and arrays must be 16-byte aligned");
  if (x1 <= x0 || z1 <= z0) return;
  const int g0 = z0 / 4, ngroups = (z1 + 3) / 4 - g0, nrows = x1 - x0;
  k_image_sum<<<grid_for((long long)nrows * ngroups), kThreads, 0, st>>>(image, s, r, shot_stride, nslots, x0,
                                                                         nrows, g0, ngroups, pitch / 4, scale);
  note_launch();
}

template <typename T>
void launch_image(T *image, long long image_stride, const T *s, const T *r, long long shot_stride,
                  int nslots, int n, float scale, cudaStream_t st) {
  unsigned gx = grid_for(n);
  if (gx > 1184) gx = 1184;
  dim3 g(gx, nslots);
  k_image<T><<<g, kThreads, 0, st>>>(image, image_stride, s, r, shot_stride, n, scale);
  note_launch();
}

// ---------------------------------------------------------------- step
template <int ARITH, bool DAMPED, bool RCP, int TX>
static void step_t(const StepArgs &a, int nslots, cudaStream_t st) {
  dim3 g((a.nz - 12 + kTZ - 1) / kTZ, (a.nx - 12 + TX - 1) / TX, nslots);
  fd_step_tile<ARITH, DAMPED, RCP, TX><<<g, kStepThreads, 0, st>>>(a);
  note_launch();
}

template <int ARITH, bool DAMPED, bool RCP>
static void step_tx(int tx, const StepArgs &a, int nslots, cudaStream_t st) {
  if (tx >= 64) step_t<ARITH, DAMPED, RCP, 64>(a, nslots, st);
  else step_t<ARITH, DAMPED, RCP, 32>(a, nslots, st);
}

template <int ARITH>
static void step_a(bool damped, bool rcp, int tx, const StepArgs &a, int nslots, cudaStream_t st) {
  if (damped) {
    if (rcp) step_tx<ARITH, true, true>(tx, a, nslots, st);
    else step_tx<ARITH, true, false>(tx, a, nslots, st);
  } else {
    if (rcp) step_tx<ARITH, false, true>(tx, a, nslots, st);
    else step_tx<ARITH, false, false>(tx, a, nslots, st);
  }
}

void launch_step(int arith, bool damped, bool vel_is_rcp, int tx, const StepArgs &a, int nslots,
                 cudaStream_t st) {
  if (nslots <= 0 || a.nx <= 12 || a.nz <= 12) return;
  if (arith == ARITH_REF) step_a<ARITH_REF>(damped, vel_is_rcp, tx, a, nslots, st);
  else if (arith == ARITH_FAST) step_a<ARITH_FAST>(damped, vel_is_rcp, tx, a, nslots, st);
  else step_a<ARITH_F64>(damped, vel_is_rcp, tx, a, nslots, st);
}

// ---------------------------------------------------------------- mute
// One block per slot.  The velocity mean is the reference's sequential
// float sum (damp4t10d.cpp:338-343): the block stages values in shared
// memory and thread 0 adds them in the reference's (x, then depth) order.
__global__ void k_mute_windows(int *win, const float *vel, int nxpad, int nzpad,
                               const int *src_x, const int *src_z, const int *rec_x,
                               const int *rec_z, long long rec_row_stride, int ng,
                               const int *slot_shot, int half_len, int nt) {
  constexpr int CH = 2048;
  __shared__ float buf[CH];
  __shared__ float s_avg;
  int slot = blockIdx.x;
  int shot = slot_shot ? slot_shot[slot] : slot;
  int sx = src_x[shot], sz = src_z[shot];
  const int *rx = rec_x + (long long)shot * rec_row_stride;
  const int *rz = rec_z + (long long)shot * rec_row_stride;
  int gz0 = rz[0];
  int gmin = sz < gz0 ? sz : gz0, gmax = sz > gz0 ? sz : gz0;
  int rows = gmax - gmin + 1;
  if (gmin < 0 || gmax >= nzpad) rows = 0;   // positions off the grid: mute nothing
  long long total = (long long)nxpad * rows;
  float acc = 0.0f;
  for (long long base = 0; base < total; base += CH) {
    int cnt = (int)((total - base) < CH ? (total - base) : CH);
    for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
      long long q = base + j;
      int i = (int)(q / rows), k = gmin + (int)(q - (long long)i * rows);
      buf[j] = vel[(long long)i * nzpad + k];
    }
    __syncthreads();
    if (threadIdx.x == 0)
      for (int j = 0; j < cnt; j++) acc = __fadd_rn(acc, buf[j]);
    __syncthreads();
  }
  if (threadIdx.x == 0) s_avg = rows > 0 ? __fdiv_rn(acc, (float)(nxpad * rows)) : -1.0f;
  __syncthreads();
  float avg = s_avg;
  for (int ig = threadIdx.x; ig < ng; ig += blockDim.x) {
    int gx = rx[ig], gz = rz[ig];
    int start = nt, end = nt;   // an unused receiver entry mutes nothing
    if (gx >= 0 && avg >= 0.0f) {
      float dist = (float)((gx - sx) * (gx - sx) + (gz - sz) * (gz - sz));
      int t = (int)__fsqrt_rn(__fmul_rn(dist, avg));
      start = t;
      end = (t + 2 * half_len) > nt ? nt : (t + 2 * half_len);
    }
    win[((long long)slot * ng + ig) * 2] = start;
    win[((long long)slot * ng + ig) * 2 + 1] = end;
  }
}

void launch_mute_windows(int *win, const float *vel, int nxpad, int nzpad, const int *src_x,
                         const int *src_z, const int *rec_x, const int *rec_z,
                         long long rec_row_stride, int ng, const int *slot_shot, int half_len,
                         int nt, int nslots, cudaStream_t st) {
  if (nslots <= 0) return;
  k_mute_windows<<<nslots, kThreads, 0, st>>>(win, vel, nxpad, nzpad, src_x, src_z, rec_x, rec_z,
                                              rec_row_stride, ng, slot_shot, half_len, nt);
  note_launch();
}

__global__ void k_apply_mute(float *d, long long slot_stride, const int *win, int nt, int ng) {
  int slot = blockIdx.y;
  long long n = (long long)nt * ng;
  float *x = d + (long long)slot * slot_stride;
  const int *w = win + (long long)slot * ng * 2;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    int it = (int)(q / ng), ig = (int)(q - (long long)it * ng);
    if (it >= w[2 * ig] && it < w[2 * ig + 1]) x[q] = 0.0f;
  }
}

void launch_apply_mute(float *d, long long slot_stride, const int *win, int nt, int ng, int nslots,
                       cudaStream_t st) {
  if (nslots <= 0) return;
  unsigned gx = grid_for((long long)nt * ng);
  if (gx > 2048) gx = 2048;
  k_apply_mute<<<dim3(gx, nslots), kThreads, 0, st>>>(d, slot_stride, win, nt, ng);
  note_launch();
}

// ---------------------------------------------------------------- residual
__global__ void k_muted_residual(float *r, const float *obs, long long obs_shot_stride,
                                 const int *slot_shot, const float *cal, const int *win_obs,
                                 const int *win_cal, int nt, int ng) {
  int slot = blockIdx.y;
  int shot = slot_shot ? slot_shot[slot] : slot;
  long long n = (long long)nt * ng;
  const float *o = obs + (long long)shot * obs_shot_stride;
  const float *c = cal + (long long)slot * n;
  const int *wo = win_obs + (long long)slot * ng * 2;
  const int *wc = win_cal + (long long)slot * ng * 2;
  float *y = r + (long long)slot * n;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    int it = (int)(q / ng), ig = (int)(q - (long long)it * ng);
    float a = (it >= wo[2 * ig] && it < wo[2 * ig + 1]) ? 0.0f : o[q];
    float b = (it >= wc[2 * ig] && it < wc[2 * ig + 1]) ? 0.0f : c[q];
    y[q] = __fsub_rn(a, b);
  }
}

void launch_muted_residual(float *r, const float *obs, long long obs_shot_stride,
                           const int *slot_shot, const float *cal, const int *win_obs,
                           const int *win_cal, int nt, int ng, int nslots, cudaStream_t st) {
  if (nslots <= 0) return;
  unsigned gx = grid_for((long long)nt * ng);
  if (gx > 2048) gx = 2048;
  k_muted_residual<<<dim3(gx, nslots), kThreads, 0, st>>>(r, obs, obs_shot_stride, slot_shot, cal,
                                                          win_obs, win_cal, nt, ng);
  note_launch();
}

__global__ void k_residual(float *r, const float *obs, long long obs_slot_stride, const float *cal,
                           long long n) {
  int slot = blockIdx.y;
  const float *o = obs + (long long)slot * obs_slot_stride;
  const float *c = cal + (long long)slot * n;
  float *y = r + (long long)slot * n;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x)
    y[q] = __fsub_rn(o[q], c[q]);
}

void launch_residual(float *r, const float *obs, long long obs_slot_stride, const float *cal,
                     long long n_per_slot, int nslots, cudaStream_t st) {
  if (nslots <= 0) return;
  unsigned gx = grid_for(n_per_slot);
  if (gx > 2048) gx = 2048;
  k_residual<<<dim3(gx, nslots), kThreads, 0, st>>>(r, obs, obs_slot_stride, cal, n_per_slot);
  note_launch();
}

__global__ void k_sumsq_partial(double *partials, const float *x, long long n, int pps) {
  int slot = blockIdx.y;
  const float *v = x + (long long)slot * n;
  double acc = 0.0;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    double a = (double)v[q];
    acc = fma(a, a, acc);
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partials[(long long)slot * pps + blockIdx.x] = acc;
}

__global__ void k_sum_partials(double *out, const double *partials, int pps) {
  int slot = blockIdx.x;
  double acc = 0.0;
  for (int i = threadIdx.x; i < pps; i += blockDim.x) acc += partials[(long long)slot * pps + i];
  acc = block_sum(acc);
  if (threadIdx.x == 0) out[slot] = acc;
}

void launch_sumsq_f64(double *out, const float *x, long long n_per_slot, int nslots,
                      double *partials, int partials_per_slot, cudaStream_t st) {
  if (nslots <= 0) return;
  k_sumsq_partial<<<dim3(partials_per_slot, nslots), kThreads, 0, st>>>(partials, x, n_per_slot,
                                                                       partials_per_slot);
  note_launch();
  k_sum_partials<<<nslots, kThreads, 0, st>>>(out, partials, partials_per_slot);
  note_launch();
}

// ---------------------------------------------------------------- transVsrc
// fwiframework.cpp:90-91 in double:
//   -1./12 r[i-2] + 4./3 r[i-1] - 2.5 r[i] + 4./3 r[i+1] - 1./12 r[i+2]
// zero for i <= 1 and i >= nt-2.
__global__ void k_trans_vsrc(float *out, const float *in, int nt, int ng) {
  int slot = blockIdx.y;
  long long n = (long long)nt * ng;
  const float *x = in + (long long)slot * n;
  float *y = out + (long long)slot * n;
  const double c1 = -1. / 12, c2 = 4. / 3;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    int it = (int)(q / ng);
    float v = 0.0f;
    if (it > 1 && it < nt - 2) {
      double acc = __dmul_rn(c1, (double)x[q - 2 * ng]);
      acc = __dadd_rn(acc, __dmul_rn(c2, (double)x[q - ng]));
      acc = __dsub_rn(acc, __dmul_rn(2.5, (double)x[q]));
      acc = __dadd_rn(acc, __dmul_rn(c2, (double)x[q + ng]));
      acc = __dsub_rn(acc, __dmul_rn(-c1, (double)x[q + 2 * ng]));
      v = __double2float_rn(acc);
    }
    y[q] = v;
  }
}

void launch_trans_vsrc(float *out, const float *in, int nt, int ng, int nslots, cudaStream_t st) {
  if (nslots <= 0) return;
  unsigned gx = grid_for((long long)nt * ng);
  if (gx > 2048) gx = 2048;
  k_trans_vsrc<<<dim3(gx, nslots), kThreads, 0, st>>>(out, in, nt, ng);
  note_launch();
}

// ---------------------------------------------------------------- gradient
__global__ void k_finalize_gradient(float *g2, const float *gs, long long g_stride, int nslots,
                                    int nxpad, int nzpad, int bx0, int pitch, int accumulate) {
  const int bz0 = 6, bzn = bx0, bxn = bx0;
  int n = nxpad * nzpad;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    int ix = q / nzpad, iz = q - ix * nzpad;
    long long qp = (long long)ix * pitch + iz;
    bool inside = !(ix < bx0 || iz < bz0 || ix >= nxpad - bxn || iz >= nzpad - bzn);
    float acc = accumulate ? g2[q] : 0.0f;
    if (inside) {
      int izi = iz - bz0;  // scaleGradient multiplies interior rows iz >= 1 by sqrt(iz)
      float sc = izi >= 1 ? __fsqrt_rn((float)izi) : 1.0f;
      for (int s = 0; s < nslots; s++) {
        float v = gs[(long long)s * g_stride + qp];
        if (izi >= 1) v = __fmul_rn(v, sc);
        acc = __fadd_rn(acc, v);
      }
    }
    g2[q] = acc;
  }
}

void launch_finalize_gradient(float *g2, const float *gs, long long g_stride, int nslots, int nxpad,
                              int nzpad, int bx0, int pitch, int accumulate, cudaStream_t st) {
  unsigned gx = grid_for((long long)nxpad * nzpad);
  k_finalize_gradient<<<gx, kThreads, 0, st>>>(g2, gs, g_stride, nslots, nxpad, nzpad, bx0, pitch,
                                               accumulate);
  note_launch();
}

__global__ void k_cg_dots(double *partials, const float *g, const float *g0, int n) {
  double a = 0, b = 0, c = 0;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    double x = g[q], y = g0[q];
    a = fma(x, x, a);
    b = fma(x, y, b);
    c = fma(y, y, c);
  }
  a = block_sum(a);
  b = block_sum(b);
  c = block_sum(c);
  if (threadIdx.x == 0) {
    partials[blockIdx.x * 3 + 0] = a;
    partials[blockIdx.x * 3 + 1] = b;
    partials[blockIdx.x * 3 + 2] = c;
  }
}

__global__ void k_cg_dots_final(double *out, const double *partials, int nb) {
  double a = 0, b = 0, c = 0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) {
    a += partials[3 * i];
    b += partials[3 * i + 1];
    c += partials[3 * i + 2];
  }
  a = block_sum(a);
  b = block_sum(b);
  c = block_sum(c);
  if (threadIdx.x == 0) {
    out[0] = a;
    out[1] = b;
    out[2] = c;
  }
}

void launch_cg_dots(double *out, const float *g, const float *g0, int n, double *partials,
                    cudaStream_t st) {
  const int nb = 256;
  k_cg_dots<<<nb, kThreads, 0, st>>>(partials, g, g0, n);
  note_launch();
  k_cg_dots_final<<<1, kThreads, 0, st>>>(out, partials, nb);
  note_launch();
}

__global__ void k_cg_update(float *d, float *g0, const float *g, float beta, int n, int first) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    float x = g[q];
    d[q] = first ? x : __fadd_rn(x, __fmul_rn(beta, d[q]));
    g0[q] = x;
  }
}

void launch_cg_update(float *d, float *g0, const float *g, float beta, int n, int first,
                      cudaStream_t st) {
  k_cg_update<<<grid_for(n), kThreads, 0, st>>>(d, g0, g, beta, n, first);
  note_launch();
}

// Ordered-int encoding so that atomicMin on int orders floats.
__device__ __forceinline__ int float_to_ordered(float f) {
  int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float ordered_to_float(int i) {
  return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff);
}

__global__ void k_max_alpha(int *out, const float *vel, const float *grad, int n, float dt, float dx,
                            float maxdv) {
  float best = 3.402823466e+38f;  // FLT_MAX, the reference's initial value
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    float v = vel[q];
    float tmpv = __fdiv_rn(dx, __fmul_rn(dt, __fsqrt_rn(v)));
    tmpv = __fsub_rn(tmpv, maxdv);
    float t = __fdiv_rn(dx, __fmul_rn(dt, tmpv));
    tmpv = __fmul_rn(t, t);
    float ag = fabsf(grad[q]);
    if ((double)ag < 1e-10) continue;
    float cand = __fdiv_rn(__fsub_rn(tmpv, v), ag);
    if (best > cand) best = cand;
  }
  for (int o = 16; o > 0; o >>= 1) best = fminf(best, __shfl_down_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0) atomicMin(out, float_to_ordered(best));
}

__global__ void k_init_ordered(int *out) { *out = float_to_ordered(3.402823466e+38f); }
__global__ void k_decode_ordered(float *out, const int *in) { *out = ordered_to_float(*in); }

void launch_max_alpha(float *out_alpha2, const float *vel, const float *grad, int n, float dt,
                      float dx, float maxdv, cudaStream_t st) {
  int *tmp = reinterpret_cast<int *>(out_alpha2);
  k_init_ordered<<<1, 1, 0, st>>>(tmp);
  note_launch();
  k_max_alpha<<<592, kThreads, 0, st>>>(tmp, vel, grad, n, dt, dx, maxdv);
  note_launch();
  k_decode_ordered<<<1, 1, 0, st>>>(out_alpha2, tmp);
  note_launch();
}

__global__ void k_update_vel(float *newv, const float *v, const float *g, int n, float steplen,
                             float vmin, float vmax) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    float x = __fadd_rn(v[q], __fmul_rn(steplen, g[q]));
    if (x > vmax) x = vmax;
    if (x < vmin) x = vmin;
    newv[q] = x;
  }
}

void launch_update_vel(float *newv, const float *v, const float *g, int n, float steplen,
                       float vmin, float vmax, cudaStream_t st) {
  k_update_vel<<<grid_for(n), kThreads, 0, st>>>(newv, v, g, n, steplen, vmin, vmax);
  note_launch();
}

// Two phases as the reference's loops: top/bottom rows per column first,
// then whole left/right columns.
__global__ void k_refill_z(float *v, int nxpad, int nzpad, int bz0, int bzn) {
  int ix = blockIdx.x * blockDim.x + threadIdx.x;
  if (ix >= nxpad) return;
  float *col = v + (long long)ix * nzpad;
  float top = col[bz0], bot = col[nzpad - bzn - 1];
  for (int iz = 0; iz < bz0; iz++) col[iz] = top;
  for (int iz = nzpad - bzn; iz < nzpad; iz++) col[iz] = bot;
}

__global__ void k_refill_x(float *v, int nxpad, int nzpad, int bx0, int bxn) {
  int iz = blockIdx.x * blockDim.x + threadIdx.x;
  int ix = blockIdx.y;
  if (iz >= nzpad) return;
  if (ix < bx0) v[(long long)ix * nzpad + iz] = v[(long long)bx0 * nzpad + iz];
  else if (ix >= nxpad - bxn) v[(long long)ix * nzpad + iz] = v[(long long)(nxpad - bxn - 1) * nzpad + iz];
}

void launch_refill_boundary(float *v, int nxpad, int nzpad, int bz0, int bzn, int bx0, int bxn,
                            cudaStream_t st) {
  k_refill_z<<<grid_for(nxpad), kThreads, 0, st>>>(v, nxpad, nzpad, bz0, bzn);
  note_launch();
  k_refill_x<<<dim3(grid_for(nzpad), nxpad), kThreads, 0, st>>>(v, nxpad, nzpad, bx0, bxn);
  note_launch();
}

__global__ void k_reciprocal(float *out, const float *in, long long n) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x)
    out[q] = __fdiv_rn(1.0f, in[q]);
}

void launch_reciprocal(float *out, const float *in, long long n, cudaStream_t st) {
  unsigned g = grid_for(n);
  if (g > 4096) g = 4096;
  k_reciprocal<<<g, kThreads, 0, st>>>(out, in, n);
  note_launch();
}

// out[x*pitch + z] = 1/in[x*nz + z] (padding columns set to 1).
template <typename T>
__global__ void k_pitched_rcp(T *out, const float *in, int nx, int nz, int pitch) {
  long long n = (long long)nx * pitch;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    int x = (int)(q / pitch), z = (int)(q - (long long)x * pitch);
    if (z < nz) {
      float v = in[(long long)x * nz + z];
      if constexpr (sizeof(T) == 4) out[q] = __fdiv_rn(1.0f, v);
      else out[q] = 1.0 / (double)v;
    } else {
      out[q] = T(1);
    }
  }
}

void launch_pitched_reciprocal(float *out, const float *in, int nx, int nz, int pitch,
                               cudaStream_t st) {
  unsigned g = grid_for((long long)nx * pitch);
  if (g > 4096) g = 4096;
  k_pitched_rcp<float><<<g, kThreads, 0, st>>>(out, in, nx, nz, pitch);
  note_launch();
}

void launch_to_f64_reciprocal(double *out, const float *in, int nx, int nz, int pitch,
                              cudaStream_t st) {
  unsigned g = grid_for((long long)nx * pitch);
  if (g > 4096) g = 4096;
  k_pitched_rcp<double><<<g, kThreads, 0, st>>>(out, in, nx, nz, pitch);
  note_launch();
}

// Sponge ramps of fd4t10s-damp-zjh.c:64-80 split by axis: dist_x[ix] is the
// left/right ramp (0 inside), dist_z[iz] the bottom ramp (-1 above it, where
// the left/right one applies).
__global__ void k_damp_tables(float *dist_x, float *dist_z, float2 *coef_x, int nx, int nz, int nb) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nx) {
    float d = 0.0f;
    if (i < nb) d = __fdiv_rn((float)(nb - i), (float)nb);
    if (i >= nx - nb) d = __fdiv_rn((float)(i - (nx - nb) + 1), (float)nb);
    dist_x[i] = d;
    if (coef_x) coef_x[i] = fast_damp_coef(d);
  }
  if (i < nz) dist_z[i] = i >= nz - nb ? __fdiv_rn((float)(i - (nz - nb) + 1), (float)nb) : -1.0f;
}

void launch_damp_tables(float *dist_x, float *dist_z, float2 *coef_x, int nx, int nz, int nb, cudaStream_t st) {
  int n = nx > nz ? nx : nz;
  k_damp_tables<<<grid_for(n), kThreads, 0, st>>>(dist_x, dist_z, coef_x, nx, nz, nb);
  note_launch();
}

// ---------------------------------------------------------------- warp-specialised step
template <int ARITH, bool DAMPED, int NW, int D, int EPI>
static void ws_launch(const StreamArgs &a, int nslots, cudaStream_t st) {
  constexpr int BZ = 128 * NW - 8;
  constexpr size_t smem = ws_smem_bytes<NW, D, EPI>();
  // raise the dynamic shared memory limit once (thread-safe static init)
  static const cudaError_t attr = cudaFuncSetAttribute(fd_step_ws<ARITH, DAMPED, NW, D, EPI>,
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  SWFWI_CUDA(attr);
  int nbands = (a.nz - 10 + BZ - 1) / BZ;
  int nchunks = (a.nx - 12 + a.xchunk - 1) / a.xchunk;
  dim3 g = a.shot_major ? dim3(nbands, nchunks, nslots) : dim3(nslots, nbands, nchunks);
  fd_step_ws<ARITH, DAMPED, NW, D, EPI><<<g, (NW + 1) * 32, smem, st>>>(a);
}

template <int ARITH, bool DAMPED, int NW, int D>
static void ws_t(const StreamArgs &a, int nslots, cudaStream_t st) {
  const Epilogue &e = a.epi;
  const int mode = (e.sub || e.image) ? 2 : (e.inj ? 3 : 0);
  if (mode == 2 && e.inj) throw Error(SWFWI_ERR_BAD_ARG, "mixed fused epilogue parts");
  if constexpr (NW == 3) {
    if (mode == 2) return ws_launch<ARITH, DAMPED, NW, D, 2>(a, nslots, st);
    if (mode == 3) return ws_launch<ARITH, DAMPED, NW, D, 3>(a, nslots, st);
  } else {
    if (mode) throw Error(SWFWI_ERR_BAD_ARG, "the fused step runs with 376-deep bands only");
  }
  ws_launch<ARITH, DAMPED, NW, D, 0>(a, nslots, st);
}

template <int ARITH, bool DAMPED, int D>
static void ws_nw(int bz, const StreamArgs &a, int nslots, cudaStream_t st) {
  if (bz >= 376) ws_t<ARITH, DAMPED, 3, D>(a, nslots, st);
  else if (bz >= 248) ws_t<ARITH, DAMPED, 2, D>(a, nslots, st);
  else ws_t<ARITH, DAMPED, 1, D>(a, nslots, st);
}

template <int ARITH, bool DAMPED>
static void ws_d(int depth, int bz, const StreamArgs &a, int nslots, cudaStream_t st) {
  if (depth >= 7) ws_nw<ARITH, DAMPED, 7>(bz, a, nslots, st);
  else ws_nw<ARITH, DAMPED, 3>(bz, a, nslots, st);
}

void launch_ws_step(int arith, bool damped, int bz, int depth, const StreamArgs &a, int nslots,
                    cudaStream_t st) {
  if (nslots <= 0 || a.nx <= 12 || a.nz <= 12) return;
  if (arith == ARITH_REF) {
    if (damped) ws_d<ARITH_REF, true>(depth, bz, a, nslots, st);
    else ws_d<ARITH_REF, false>(depth, bz, a, nslots, st);
  } else {
    if (damped) ws_d<ARITH_FAST, true>(depth, bz, a, nslots, st);
    else ws_d<ARITH_FAST, false>(depth, bz, a, nslots, st);
  }
  note_launch();
}

__global__ void k_encode_source(float *encsrc, const float *wlt, const int *codes, int nt, int ns) {
  long long n = (long long)nt * ns;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    int it = (int)(q / ns), is = (int)(q - (long long)it * ns);
    encsrc[q] = __fmul_rn(wlt[it], (float)codes[is]);
  }
}

void launch_encode_source(float *encsrc, const float *wlt, const int *codes, int nt, int ns,
                          cudaStream_t st) {
  k_encode_source<<<grid_for((long long)nt * ns), kThreads, 0, st>>>(encsrc, wlt, codes, nt, ns);
  note_launch();
}

__global__ void k_encode_obs(float *encobs, const float *dobs, const int *codes, long long n, int ns) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    float acc = 0.0f;
    for (int is = 0; is < ns; is++)
      acc = __fadd_rn(acc, __fmul_rn(dobs[(long long)is * n + q], (float)codes[is]));
    encobs[q] = acc;
  }
}

void launch_encode_obs(float *encobs, const float *dobs, const int *codes, long long n, int ns,
                       cudaStream_t st) {
  unsigned g = grid_for(n);
  if (g > 8192) g = 8192;
  k_encode_obs<<<g, kThreads, 0, st>>>(encobs, dobs, codes, n, ns);
  note_launch();
}

__global__ void k_f32_to_f64(double *out, const float *in, long long n) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x)
    out[q] = in[q];
}
__global__ void k_f64_to_f32(float *out, const double *in, long long n) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x)
    out[q] = (float)in[q];
}
void launch_f32_to_f64(double *out, const float *in, long long n, cudaStream_t st) {
  unsigned g = grid_for(n);
  if (g > 4096) g = 4096;
  k_f32_to_f64<<<g, kThreads, 0, st>>>(out, in, n);
  note_launch();
}
void launch_f64_to_f32(float *out, const double *in, long long n, cudaStream_t st) {
  unsigned g = grid_for(n);
  if (g > 4096) g = 4096;
  k_f64_to_f32<<<g, kThreads, 0, st>>>(out, in, n);
  note_launch();
}

// explicit instantiations
template void launch_inject<float>(float *, long long, int, PointSet, const float *, long long, int,
                                   int, cudaStream_t);
template void launch_inject<double>(double *, long long, int, PointSet, const double *, long long,
                                    int, int, cudaStream_t);
template void launch_record<float>(float *, long long, const float *, long long, int, PointSet,
                                   cudaStream_t);
template void launch_record<double>(double *, long long, const double *, long long, int, PointSet,
                                    cudaStream_t);
// ---------------------------------------------------------------- trace transpose
__global__ void k_transpose_traces(float *out, const float *in, int nt, int ng) {
  __shared__ float tile[32][33];
  const long long base = (long long)blockIdx.z * nt * ng;
  const int it0 = blockIdx.y * 32, ig0 = blockIdx.x * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    int it = it0 + j, ig = ig0 + threadIdx.x;
    if (it < nt && ig < ng) tile[j][threadIdx.x] = in[base + (long long)it * ng + ig];
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    int ig = ig0 + j, it = it0 + threadIdx.x;
    if (it < nt && ig < ng) out[base + (long long)ig * nt + it] = tile[threadIdx.x][j];
  }
}

void launch_transpose_traces(float *out, const float *in, int nt, int ng, int nslots, cudaStream_t st) {
  if (nt <= 0 || ng <= 0 || nslots <= 0) return;
  dim3 g((ng + 31) / 32, (nt + 31) / 32, nslots);
  k_transpose_traces<<<g, dim3(32, 8), 0, st>>>(out, in, nt, ng);
  note_launch();
}

// ---------------------------------------------------------------- 16-bit strips
namespace {
template <int FMT>
__device__ __forceinline__ uint16_t q_encode(float v) {
  if constexpr (FMT == SWFWI_STRIP_F16) return __half_as_ushort(__float2half_rn(v));
  else return __bfloat16_as_ushort(__float2bfloat16_rn(v));
}
template <int FMT>
__device__ __forceinline__ float q_decode(uint16_t h) {
  if constexpr (FMT == SWFWI_STRIP_F16) return __half2float(__ushort_as_half(h));
  else return __bfloat162float(__ushort_as_bfloat16(h));
}

// One CTA per slot: the step's largest |value|, its power-of-two scale,
// then the scaled 16-bit values.
template <int FMT>
__global__ void __launch_bounds__(1024)
k_strip_write_q(uint16_t *q, long long q_slot_stride, float *scale, long long scale_slot_stride,
                const float *field, long long shot_stride, int bs, int nx, int nz, int bx0, int pitch) {
  __shared__ float wmax[32];
  const int slot = blockIdx.x;
  const float *f = field + (long long)slot * shot_stride;
  float m = 0.f;
  for (int i = threadIdx.x; i < bs; i += blockDim.x)
    m = fmaxf(m, fabsf(f[strip_index(i, nx, nz, bx0, pitch)]));
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = m;
  __syncthreads();
  m = 0.f;
  for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = fmaxf(m, wmax[w]);
  int e = 0;
  if (m > 0.f && m <= 3.0e38f) frexpf(m, &e);   // m < 2^e
  // a step whose largest |value| is subnormal would need a scale of 2^-140
  // or so, whose inverse overflows (and 0 * inf is NaN): such values are
  // kept at the scale 2^-114 (they encode as 0 or as 16-bit subnormals)
  e = max(e, -100);
  const float s = ldexpf(1.0f, e - 14), inv = ldexpf(1.0f, 14 - e);
  if (threadIdx.x == 0) scale[(long long)slot * scale_slot_stride] = s;
  uint16_t *qs = q + (long long)slot * q_slot_stride;
  for (int i = threadIdx.x; i < bs; i += blockDim.x)
    qs[i] = q_encode<FMT>(f[strip_index(i, nx, nz, bx0, pitch)] * inv);
}

template <int FMT>
__global__ void k_strip_read_q(const uint16_t *q, long long q_slot_stride, const float *scale,
                               long long scale_slot_stride, float *field, long long shot_stride, int bs,
                               int nx, int nz, int bx0, int pitch) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, slot = blockIdx.y;
  if (i >= bs) return;
  const float s = scale[(long long)slot * scale_slot_stride];
  field[(long long)slot * shot_stride + strip_index(i, nx, nz, bx0, pitch)] =
      q_decode<FMT>(q[(long long)slot * q_slot_stride + i]) * s;
}
}  // namespace

void launch_strip_write_q(int format, uint16_t *q, long long q_slot_stride, float *scale,
                          long long scale_slot_stride, const float *field, long long shot_stride,
                          int nslots, int nx, int nz, int bx0, int pitch, cudaStream_t st) {
  int bs = strip_size(nx, nz, bx0);
  if (format == SWFWI_STRIP_F16)
    k_strip_write_q<SWFWI_STRIP_F16><<<nslots, 1024, 0, st>>>(q, q_slot_stride, scale, scale_slot_stride,
                                                              field, shot_stride, bs, nx, nz, bx0, pitch);
  else
    k_strip_write_q<SWFWI_STRIP_BF16><<<nslots, 1024, 0, st>>>(q, q_slot_stride, scale, scale_slot_stride,
                                                               field, shot_stride, bs, nx, nz, bx0, pitch);
  note_launch();
}

void launch_strip_read_q(int format, const uint16_t *q, long long q_slot_stride, const float *scale,
                         long long scale_slot_stride, float *field, long long shot_stride, int nslots,
                         int nx, int nz, int bx0, int pitch, cudaStream_t st) {
  int bs = strip_size(nx, nz, bx0);
  dim3 g(grid_for(bs), nslots);
  if (format == SWFWI_STRIP_F16)
    k_strip_read_q<SWFWI_STRIP_F16><<<g, kThreads, 0, st>>>(q, q_slot_stride, scale, scale_slot_stride,
                                                            field, shot_stride, bs, nx, nz, bx0, pitch);
  else
    k_strip_read_q<SWFWI_STRIP_BF16><<<g, kThreads, 0, st>>>(q, q_slot_stride, scale, scale_slot_stride,
                                                             field, shot_stride, bs, nx, nz, bx0, pitch);
  note_launch();
}

// ---------------------------------------------------------------- 16-bit snapshots
namespace {
// Pass 1: each CTA's largest |value| of its part of one slot's field (grid
// x = kSnapParts parts, y = slots) into part_max[slot][part]; pass 2 (the
// encoder) reduces a slot's parts in a fixed order and encodes.
__global__ void __launch_bounds__(1024)
k_field_max(float *part_max, const float *field, long long shot_stride, long long count) {
  __shared__ float wmax[32];
  const int slot = blockIdx.y;
  const float4 *f = reinterpret_cast<const float4 *>(field + (long long)slot * shot_stride);
  const long long n4 = count / 4;
  float m = 0.f;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x) {
    const float4 v = f[i];
    m = fmaxf(m, fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fmaxf(fabsf(v.z), fabsf(v.w))));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = fmaxf(m, wmax[w]);
    part_max[slot * kSnapParts + blockIdx.x] = m;
  }
}

__device__ __forceinline__ void snap_scale_of(float m, float &s, float &inv) {
  int e = 0;
  if (m > 0.f && m <= 3.0e38f) frexpf(m, &e);   // m < 2^e
  e = max(e, -100);                              // as the strips: subnormal-only fields
  s = ldexpf(1.0f, e - 14);
  inv = ldexpf(1.0f, 14 - e);
}

template <int FMT>
__global__ void k_field_write_q(uint16_t *q, float *scale, long long scale_slot_stride, const float *part_max,
                                const float *field, long long shot_stride, long long count) {
  const int slot = blockIdx.y;
  float m = 0.f;
  for (int p = 0; p < kSnapParts; p++) m = fmaxf(m, part_max[slot * kSnapParts + p]);
  float s, inv;
  snap_scale_of(m, s, inv);
  if (blockIdx.x == 0 && threadIdx.x == 0) scale[(long long)slot * scale_slot_stride] = s;
  const float4 *f = reinterpret_cast<const float4 *>(field + (long long)slot * shot_stride);
  ushort4 *qs = reinterpret_cast<ushort4 *>(q + (long long)slot * count);
  const long long n4 = count / 4;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x) {
    const float4 v = f[i];
    qs[i] = make_ushort4(q_encode<FMT>(v.x * inv), q_encode<FMT>(v.y * inv), q_encode<FMT>(v.z * inv),
                         q_encode<FMT>(v.w * inv));
  }
}

template <int FMT>
__global__ void k_field_read_q(const uint16_t *q, const float *scale, long long scale_slot_stride, float *field,
                               long long shot_stride, long long count) {
  const int slot = blockIdx.y;
  const float s = scale[(long long)slot * scale_slot_stride];
  float4 *f = reinterpret_cast<float4 *>(field + (long long)slot * shot_stride);
  const ushort4 *qs = reinterpret_cast<const ushort4 *>(q + (long long)slot * count);
  const long long n4 = count / 4;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x) {
    const ushort4 h = qs[i];
    f[i] = make_float4(q_decode<FMT>(h.x) * s, q_decode<FMT>(h.y) * s, q_decode<FMT>(h.z) * s,
                       q_decode<FMT>(h.w) * s);
  }
}

void check_snap_args(const void *q, const float *field, long long shot_stride, long long count) {
  if (count % 4 != 0 || shot_stride % 4 != 0 ||
      (reinterpret_cast<uintptr_t>(q) | reinterpret_cast<uintptr_t>(field)) % 16 != 0)
    throw Error(SWFWI_ERR_BAD_ARG, "snapshot: sizes and arrays must be 16-byte aligned");
}
}  // namespace

void launch_field_write_q(int format, uint16_t *q, float *scale, long long scale_slot_stride, float *pm,
                          const float *field, long long shot_stride, long long count, int nslots, cudaStream_t st) {
  if (nslots <= 0 || count <= 0) return;
  check_snap_args(q, field, shot_stride, count);
  k_field_max<<<dim3(kSnapParts, nslots), 1024, 0, st>>>(pm, field, shot_stride, count);
  note_launch();
  const dim3 g(grid_for(count / 4, kThreads * 8), nslots);
  if (format == SWFWI_STRIP_F16)
    k_field_write_q<SWFWI_STRIP_F16><<<g, kThreads, 0, st>>>(q, scale, scale_slot_stride, pm, field, shot_stride,
                                                             count);
  else
    k_field_write_q<SWFWI_STRIP_BF16><<<g, kThreads, 0, st>>>(q, scale, scale_slot_stride, pm, field,
                                                              shot_stride, count);
  note_launch();
}

void launch_field_read_q(int format, const uint16_t *q, const float *scale, long long scale_slot_stride,
                         float *field, long long shot_stride, long long count, int nslots, cudaStream_t st) {
  if (nslots <= 0 || count <= 0) return;
  check_snap_args(q, field, shot_stride, count);
  const dim3 g(grid_for(count / 4, kThreads * 8), nslots);
  if (format == SWFWI_STRIP_F16)
    k_field_read_q<SWFWI_STRIP_F16><<<g, kThreads, 0, st>>>(q, scale, scale_slot_stride, field, shot_stride, count);
  else
    k_field_read_q<SWFWI_STRIP_BF16><<<g, kThreads, 0, st>>>(q, scale, scale_slot_stride, field, shot_stride,
                                                             count);
  note_launch();
}

template void launch_after_forward<float>(float *, long long, const float *, PointSet, float *, long long, int,
                                          int, int, int, float *, PointSet, const float *, long long, int,
                                          long long, int, cudaStream_t);
template void launch_after_forward<double>(double *, long long, const double *, PointSet, double *, long long,
                                           int, int, int, int, double *, PointSet, const double *, long long,
                                           int, long long, int, cudaStream_t);
template void launch_inject2<float>(float *, PointSet, const float *, long long, int, int, float *, PointSet,
                                    const float *, long long, int, int, long long, int, cudaStream_t,
                                    const float *, long long, int, int, int, int);
template void launch_inject2<double>(double *, PointSet, const double *, long long, int, int, double *, PointSet,
                                     const double *, long long, int, int, long long, int, cudaStream_t,
                                     const double *, long long, int, int, int, int);
template void launch_strip_write<float>(float *, long long, const float *, long long, int, int, int,
                                        int, int, cudaStream_t);
template void launch_strip_write<double>(double *, long long, const double *, long long, int, int,
                                         int, int, int, cudaStream_t);
template void launch_strip_read<float>(const float *, long long, float *, long long, int, int, int,
                                       int, int, cudaStream_t);
template void launch_strip_read<double>(const double *, long long, double *, long long, int, int,
                                        int, int, int, cudaStream_t);
template void launch_image<float>(float *, long long, const float *, const float *, long long, int,
                                  int, float, cudaStream_t);
template void launch_image<double>(double *, long long, const double *, const double *, long long,
                                   int, int, float, cudaStream_t);

// ---------------------------------------------------------------- regularisation
// ReguFactor (src/unused/ReguFactor.cpp) on p [nx][nz].  Sums: per-block FP64
// partials of the float squares (r * r in float, as :43 and :61) of the x and
// z first differences, added in a fixed order; the reference adds them in
// float in loop order.
namespace {
constexpr int kReguBlocks = 256;

__global__ void k_regu_sums(const float *__restrict__ p, int nx, int nz, double *__restrict__ part) {
  double sx = 0.0, sz = 0.0;
  const long long total = (long long)nx * nz;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(e / nz), iz = (int)(e - (long long)ix * nz);
    const float v = p[e];
    if (ix < nx - 1) {
      const float r = __fsub_rn(p[e + nz], v);
      sx += (double)__fmul_rn(r, r);
    }
    if (iz < nz - 1) {
      const float r = __fsub_rn(p[e + 1], v);
      sz += (double)__fmul_rn(r, r);
    }
  }
  __shared__ double red[2][kThreads / 32];
  for (int o = 16; o > 0; o >>= 1) {
    sx += __shfl_down_sync(0xffffffffu, sx, o);
    sz += __shfl_down_sync(0xffffffffu, sz, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = sx;
    red[1][threadIdx.x >> 5] = sz;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < kThreads / 32; w++) {
      a += red[0][w];
      b += red[1][w];
    }
    part[2 * blockIdx.x] = a;
    part[2 * blockIdx.x + 1] = b;
  }
}

// out: Wx2, Wz2, lx * Wx2 + lz * Wz2 (getReguTerm :19-27)
__global__ void k_regu_final(const double *__restrict__ part, int blocks, float lx, float lz,
                             double *__restrict__ out) {
  double a = 0.0, b = 0.0;
  for (int i = 0; i < blocks; i++) {
    a += part[2 * i];
    b += part[2 * i + 1];
  }
  out[0] = a;
  out[1] = b;
  out[2] = (double)lx * a + (double)lz * b;
}

// getReguGradient (:67-108) element by element as its loops leave it: the z
// loop writes into the x-term array, so every element above the last depth
// holds its z term; the last depth holds the x term (0 on the last row).
// g = (accumulate ? g + term : term), each operation one float rounding.
__global__ void k_regu_grad(const float *__restrict__ p, int nx, int nz, float lx, float lz,
                            float *__restrict__ g, int accumulate) {
  const float cx = __fmul_rn(2.0f, lx), cz = __fmul_rn(2.0f, lz);
  const long long total = (long long)nx * nz;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(e / nz), iz = (int)(e - (long long)ix * nz);
    const float v = p[e];
    float r = 0.0f;
    if (iz < nz - 1) {
      const float d = iz == 0 ? __fsub_rn(v, p[e + 1])
                              : __fsub_rn(__fsub_rn(__fmul_rn(2.0f, v), p[e + 1]), p[e - 1]);
      r = __fmul_rn(cz, d);
    } else if (ix < nx - 1) {
      const float d = ix == 0 ? __fsub_rn(v, p[e + nz])
                              : __fsub_rn(__fsub_rn(__fmul_rn(2.0f, v), p[e + nz]), p[e - nz]);
      r = __fmul_rn(cx, d);
    }
    r = __fadd_rn(r, 0.0f);   // + the (all-zero) second term array
    g[e] = accumulate ? __fadd_rn(g[e], r) : r;
  }
}
}  // namespace

size_t regu_scratch_doubles() { return 3 + 2 * (size_t)kReguBlocks; }

void launch_regu_term(const float *p, int nx, int nz, float lx, float lz, double *scratch, cudaStream_t st) {
  k_regu_sums<<<kReguBlocks, kThreads, 0, st>>>(p, nx, nz, scratch + 3);
  note_launch();
  k_regu_final<<<1, 1, 0, st>>>(scratch + 3, kReguBlocks, lx, lz, scratch);
  note_launch();
}

void launch_regu_grad(const float *p, int nx, int nz, float lx, float lz, float *g, bool accumulate,
                      cudaStream_t st) {
  k_regu_grad<<<grid_for((long long)nx * nz), kThreads, 0, st>>>(p, nx, nz, lx, lz, g, accumulate ? 1 : 0);
  note_launch();
}

}  // namespace swfwi
