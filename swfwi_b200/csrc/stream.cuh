// Shared pieces of the streaming form of the acoustic step for sm_100a (same
// scheme and arithmetics as stencil.cuh): the launch arguments, mbarrier and
// TMA bulk-copy helpers, the per-point u2 and update of each arithmetic,
// their packed FP32x2 FAST forms, and the line cursor of the fused
// epilogues.  The kernels are stream_rq.cuh (register-queue warps) and
// stream_ws.cuh (warp-specialised, with the fused epilogues).
//
// Layout: the field's origin is 8 floats into each slot (coff = 8), rows of
// P floats (P % 8 == 0, P >= nz + 8); depth z of row x sits at origin +
// x*P + z.  Staged windows start at depths that are multiples of 4, so
// every window and every 4-depth group starts on a 16-byte boundary.
// Every mbarrier wait is bounded: on timeout a kernel raises an error flag,
// waits (bounded) for its copies in flight and leaves.
#pragma once
#include <cstdint>
#include "stencil.cuh"

namespace swfwi {

// A regular line of points in padded grid coordinates: point i at
// (x0 + i*jx, z0 + i*jz), i < n (a ShotPosition, shot-position.cpp:11-41).
struct PtLine {
  int x0, z0, jx, jz, n;
};

// Work a streaming step of the backward time loop does at its output points
// besides the update (calgradient, fused):
//   sub:   subSource into the new field at the `src` points,
//          sub[slot*sub_slot_stride + i*sub_stride] (one float subtraction);
//   image: image -= (new * gcurr) * scale at every output point
//          (cross_correlation; gcurr and image laid out as the fields);
//   inj:   addSource of the next step into the new field at the `src`
//          points (one float addition) -- the receiver step's residual.
// `src` lines are per slot and horizontal (or single points); a null
// pointer skips that part; inj is never set with sub or image.
struct Epilogue {
  const PtLine *src;                  // [nslots]
  const float *inj;
  long long inj_slot_stride;
  int inj_stride;
  const float *sub;
  long long sub_slot_stride;
  int sub_stride;
  float *image;
  const float *gcurr;
  float scale;
};

struct StreamArgs {
  float *prev;            // field origins (see layout above)
  float *out = nullptr;   // where the next field goes (same layout); nullptr: in place over prev
  const float2 *coef_x;   // FAST update coefficients of each row's left/right ramp, [nx]
  const float *curr;
  const float *rcp;       // 1/vt, same layout
  const float *damp_x;    // sponge ramp of each row (0 outside), [nx]
  const float *damp_z;    // bottom ramp of each depth, -1 above the sponge, [nz]
  int nx, nz, pitch;
  long long shot_stride;  // floats between shots (multiple of 8)
  long long vel_stride;   // floats between velocity models (0: one model)
  int shots_per_vel;
  int xchunk;             // output rows per CTA
  int shot_major;         // 0: blockIdx = (shot, band, chunk); 1: (band, chunk, shot)
  int *err;               // set to 1 when a bounded wait gives up
  int ramp;               // damp_x is 0 on rows [ramp, nx - ramp): those rows skip its load
  Epilogue epi;           // used by the fused variant of the warp-specialised step
};

constexpr int kStreamCoff = 8;   // floats between a slot's start and its origin

// FAST update coefficients of a sponge ramp distance: next = cf*c + pc*p
// + inc with delta = 0.05 dist^2, cf = 2 - 2 delta + delta^2 (one fma),
// pc = -(1 - 2 delta); (2, -1) where dist is 0 (no damping).
__device__ __forceinline__ float2 fast_damp_coef(float dist) {
  if (dist == 0.0f) return make_float2(2.0f, -1.0f);
  const float delta = __fmul_rn(__fmul_rn(0.05f, dist), dist);
  const float d2 = __fmul_rn(2.0f, delta);
  return make_float2(fmaf(delta, delta, __fsub_rn(2.0f, d2)), -__fsub_rn(1.0f, d2));
}

namespace stream_detail {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// try_wait with a suspend-time hint: a thread whose phase is not complete
// sleeps (up to the hint, in ns) instead of polling, so waiting warps do not
// take issue slots from the warps doing arithmetic.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(100000u)
      : "memory");
  return ok != 0;
}

// Non-blocking test of a phase (acquire on success).
__device__ __forceinline__ bool mbar_test(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: gives up after ~2^31 cycles (about a second).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  long long t0 = clock64();
  while (!mbar_try_wait_sleep(bar, parity)) {
    if (clock64() - t0 > (1LL << 31)) return false;
  }
  return true;
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// The same with the destination and barrier as shared-memory addresses.
__device__ __forceinline__ void bulk_g2s_u32(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ float4 ld4g(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ void st4(float *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }
__device__ __forceinline__ float get(const float4 &v, int i) {
  return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w));
}

// u2 at one point: zn = the 20 staged values around the group (the point's
// z neighbours at zn[8 + i +- k]), xm[k]/xp[k] = the point's value k rows
// before/after; in the reference's order (z-k, z+k, x-k, x+k).
template <int ARITH>
__device__ __forceinline__ float lap_pt(const float (&zn)[20], int i, const float (&xm)[6],
                                        const float (&xp)[6]) {
  const float c = zn[8 + i];
  if constexpr (ARITH == ARITH_REF) {
    double acc = __dmul_rn(-4.0 * (double)SWFWI_A0, (double)c);
#define SWFWI_P_TERM(K, A)                                                                     \
  {                                                                                            \
    float s = __fadd_rn(__fadd_rn(__fadd_rn(zn[8 + i - K], zn[8 + i + K]), xm[K]), xp[K]);     \
    acc = __dadd_rn(acc, (double)__fmul_rn(A, s));                                             \
  }
    SWFWI_P_TERM(1, SWFWI_A1)
    SWFWI_P_TERM(2, SWFWI_A2)
    SWFWI_P_TERM(3, SWFWI_A3)
    SWFWI_P_TERM(4, SWFWI_A4)
    SWFWI_P_TERM(5, SWFWI_A5)
#undef SWFWI_P_TERM
    return __double2float_rn(acc);
  } else {
    float acc = (-4.0f * SWFWI_A0) * c;
    acc = fmaf(SWFWI_A1, (zn[7 + i] + zn[9 + i]) + (xm[1] + xp[1]), acc);
    acc = fmaf(SWFWI_A2, (zn[6 + i] + zn[10 + i]) + (xm[2] + xp[2]), acc);
    acc = fmaf(SWFWI_A3, (zn[5 + i] + zn[11 + i]) + (xm[3] + xp[3]), acc);
    acc = fmaf(SWFWI_A4, (zn[4 + i] + zn[12 + i]) + (xm[4] + xp[4]), acc);
    acc = fmaf(SWFWI_A5, (zn[3 + i] + zn[13 + i]) + (xm[5] + xp[5]), acc);
    return acc;
  }
}

// Time update at one point (Laplacian of u2 summed z-1, z+1, x-1, x+1).
template <int ARITH>
__device__ __forceinline__ float update_pt(float c, float p, float r, float uc, float uzm, float uzp,
                                           float uxm, float uxp, float delta) {
  if constexpr (ARITH == ARITH_REF) {
    float lap = __fsub_rn(__fadd_rn(__fadd_rn(__fadd_rn(uzm, uzp), uxm), uxp), __fmul_rn(4.0f, uc));
    float t4 = __fmul_rn(__fmul_rn(__fmul_rn(1.0f / 12.0f, r), r), lap);
    double acc;
    if (delta == 0.0f) {
      acc = __dsub_rn(__dmul_rn(2.0, (double)c), (double)p);
    } else {
      float d2 = __fmul_rn(2.0f, delta);
      double coef = __dadd_rn(__dsub_rn(2.0, (double)d2), (double)__fmul_rn(delta, delta));
      acc = __dsub_rn(__dmul_rn(coef, (double)c), (double)__fmul_rn(__fsub_rn(1.0f, d2), p));
    }
    acc = __dadd_rn(acc, (double)__fmul_rn(r, uc));
    acc = __dadd_rn(acc, (double)t4);
    return __double2float_rn(acc);
  } else {
    // every rounding spelled out, so each kernel evaluates the same
    // sequence: lap = fma(-4, uc, s), base = fma(coef, c, p * pc)
    const float lap = fmaf(-4.0f, uc, __fadd_rn(__fadd_rn(uzm, uzp), __fadd_rn(uxm, uxp)));
    const float q = __fmul_rn(r, 1.0f / 12.0f);
    const float inc = __fmul_rn(r, fmaf(q, lap, uc));
    float base;
    if (delta == 0.0f) {
      base = fmaf(2.0f, c, __fmul_rn(p, -1.0f));
    } else {
      const float d2 = __fmul_rn(2.0f, delta);
      base = fmaf(fmaf(delta, delta, __fsub_rn(2.0f, d2)), c, __fmul_rn(p, -__fsub_rn(1.0f, d2)));
    }
    return __fadd_rn(base, inc);
  }
}

// FAST arithmetic on a pair of depths with the packed FP32x2 instructions
// of sm_100 (each lane rounded as the scalar instruction would be).
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 lo2(const float4 &v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(const float4 &v) { return make_float2(v.z, v.w); }

// u2 of depths 2p, 2p+1 of the group (lap_pt<ARITH_FAST>'s operations in
// the same order per lane).
template <int P>
__device__ __forceinline__ float2 lap_pair_fast(const float (&zn)[20], const float4 (&xm4)[6],
                                                const float4 (&xp4)[6]) {
  constexpr int i = 2 * P;
  const float a[6] = {-4.0f * SWFWI_A0, SWFWI_A1, SWFWI_A2, SWFWI_A3, SWFWI_A4, SWFWI_A5};
  float2 acc = __fmul2_rn(f2(a[0], a[0]), f2(zn[8 + i], zn[9 + i]));
#pragma unroll
  for (int k = 1; k <= 5; k++) {
    const float2 zs = __fadd2_rn(f2(zn[8 + i - k], zn[9 + i - k]), f2(zn[8 + i + k], zn[9 + i + k]));
    const float2 xs = P == 0 ? __fadd2_rn(lo2(xm4[k]), lo2(xp4[k])) : __fadd2_rn(hi2(xm4[k]), hi2(xp4[k]));
    acc = __ffma2_rn(f2(a[k], a[k]), __fadd2_rn(zs, xs), acc);
  }
  return acc;
}

// Undamped FAST time update of a depth pair: out = 2c - p + r*(uc + (r/12)*lap).
__device__ __forceinline__ float2 update_pair_fast(float2 c, float2 p, float2 r, float2 uc, float2 uzm,
                                                   float2 uzp, float2 uxm, float2 uxp) {
  const float2 s = __fadd2_rn(__fadd2_rn(uzm, uzp), __fadd2_rn(uxm, uxp));
  const float2 lap = __ffma2_rn(f2(-4.0f, -4.0f), uc, s);
  const float2 q = __fmul2_rn(r, f2(1.0f / 12.0f, 1.0f / 12.0f));
  const float2 inc = __fmul2_rn(r, __ffma2_rn(q, lap, uc));
  const float2 base = __ffma2_rn(f2(2.0f, 2.0f), c, __fmul2_rn(p, f2(-1.0f, -1.0f)));
  return __fadd2_rn(base, inc);
}

// FAST time update of a depth pair with sponge coefficients:
// out = cf*c + pc*p + r*(uc + (r/12)*lap), lap = (sz + (uxm + uxp)) - 4 uc,
// sz = uzm + uzp (the z neighbours' sum, formed by the caller).  Each lane
// is evaluated as update_pt<ARITH_FAST> evaluates a point; cf = 2, pc = -1
// where no sponge acts.
__device__ __forceinline__ float2 update_pair_coef(float2 c, float2 p, float2 r, float2 uc, float2 sz, float2 uxm,
                                                   float2 uxp, float2 cf, float2 pc) {
  const float2 s = __fadd2_rn(sz, __fadd2_rn(uxm, uxp));
  const float2 lap = __ffma2_rn(f2(-4.0f, -4.0f), uc, s);
  const float2 q = __fmul2_rn(r, f2(1.0f / 12.0f, 1.0f / 12.0f));
  const float2 inc = __fmul2_rn(r, __ffma2_rn(q, lap, uc));
  const float2 base = __ffma2_rn(cf, c, __fmul2_rn(p, pc));
  return __fadd2_rn(base, inc);
}

// Walks a line's points row by row for a CTA whose output rows increase by
// one per step from xa: at each row, at most one point when jx != 0 (all of
// a vertical line's points sit on row x0).
struct LineCursor {
  int next_x, next_i, step_i, dx, left;
  __device__ __forceinline__ void init(const PtLine &l, int xa) {
    next_x = -1; left = 0; step_i = 0; dx = 0; next_i = 0;
    if (l.n <= 0) return;
    if (l.jx == 0) {   // a single point (vertical lines are visited row-wise below)
      if (l.n == 1 && l.x0 >= xa) {
        next_x = l.x0;
        left = 1;
      }
      return;
    }
    if (l.jx > 0) {
      int i0 = xa <= l.x0 ? 0 : (xa - l.x0 + l.jx - 1) / l.jx;
      if (i0 >= l.n) return;
      next_i = i0; step_i = 1; dx = l.jx; left = l.n - i0;
    } else {
      const int ax = -l.jx;
      if (l.x0 < xa) return;
      int i0 = (l.x0 - xa) / ax;
      if (i0 > l.n - 1) i0 = l.n - 1;
      next_i = i0; step_i = -1; dx = ax; left = i0 + 1;
    }
    next_x = l.x0 + next_i * l.jx;
  }
  // calls f(i, d) for the point on row x at depth zg + d, d < 4
  template <typename F>
  __device__ __forceinline__ void visit(const PtLine &l, int x, int zg, F &&f) {
    if (l.jx != 0) {
      if (left > 0 && x == next_x) {
        const int z = l.z0 + next_i * l.jz;
        if (z >= zg && z < zg + 4) f(next_i, z - zg);
        next_i += step_i;
        next_x += dx;
        left--;
      }
    } else if (x == l.x0 && l.n > 0) {
      if (l.jz == 0) {
        if (l.z0 >= zg && l.z0 < zg + 4) f(0, l.z0 - zg);
      } else {
#pragma unroll
        for (int d = 0; d < 4; d++) {
          const int t = zg + d - l.z0;
          if (t % l.jz == 0 && t / l.jz >= 0 && t / l.jz < l.n) f(t / l.jz, d);
        }
      }
    }
  }
};

}  // namespace stream_detail

}  // namespace swfwi
