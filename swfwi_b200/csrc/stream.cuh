// Streaming form of the acoustic step for sm_100a (same scheme and
// arithmetics as stencil.cuh).
//
// A CTA of NW warps owns a band of BZ = 128*NW - 8 output depths (z,
// contiguous) and a chunk of consecutive rows (x) of one shot, and walks the
// chunk row by row:
//  * thread 0 issues TMA bulk copies (cp.async.bulk global -> shared,
//    completion on an mbarrier) D rows ahead: the current field's row with a
//    12-cell margin each side into a 16-row ring, the previous field's and
//    the velocity reciprocal's rows into (D+1)-row rings;
//  * each thread owns 4 consecutive depths; every shared-memory access is a
//    128-bit vector (z neighbours: 5 loads; x neighbours: 10 loads from the
//    ring; u2 of three rows from a 4-row ring), outputs go out as 128-bit
//    stores in place over prev;
//  * one barrier per row (__syncwarp for a one-warp CTA) between writing u2
//    and reading its z neighbours;
//  * the sponge's damping comes from per-row and per-column ramp tables
//    computed once, not per point.
// Every mbarrier wait is bounded: on timeout the CTA raises an error flag,
// waits (bounded) for its copies in flight and leaves.
//
// Layout: the field's origin is 8 floats into each slot (coff = 8), rows of
// P floats (P % 8 == 0, P >= nz + 8); depth z of row x sits at origin +
// x*P + z.  Band b starts at z0 = 4 + b*BZ, so every staged window
// [z0-12, z0+BZ+12) and [z0-4, z0+BZ+4) and every 4-depth group starts on a
// 16-byte boundary.
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

template <int ARITH, bool DAMPED, int NW, int D>
__global__ void __launch_bounds__(NW * 32)
fd_step_stream(StreamArgs a) {
  using namespace stream_detail;
  constexpr int NT = NW * 32;
  constexpr int BZ = 4 * NT - 8;  // output depths of the band
  constexpr int WC = BZ + 24;     // current-field window [z0-12, z0+BZ+12)
  constexpr int WP = BZ + 8;      // prev / velocity window [z0-4, z0+BZ+4)
  constexpr int NC = 16;          // current-field ring (11 rows in use + D ahead)
  constexpr int NP = D + 1;       // prev/vel ring and mbarriers
  static_assert(D + 11 <= NC, "ring too short");
  __shared__ __align__(128) float cring[NC][WC];
  __shared__ __align__(128) float pring[NP][WP];
  __shared__ __align__(128) float vring[NP][WP];
  __shared__ __align__(16) float u2r[4][4 * NT];
  __shared__ __align__(8) uint64_t bar[NP];
  __shared__ int s_fail;

  const int t = threadIdx.x;
  const int shot = a.shot_major ? blockIdx.z : blockIdx.x;
  const int band = a.shot_major ? blockIdx.x : blockIdx.y;
  const int chunk = a.shot_major ? blockIdx.y : blockIdx.z;
  const int nx = a.nx, nz = a.nz, P = a.pitch;
  const int z0 = 4 + band * BZ;
  const int zg = z0 - 4 + 4 * t;   // first depth of this thread's group
  const int xa = 6 + chunk * a.xchunk;
  const int xb = min(xa + a.xchunk, nx - 6);
  if (xa >= xb) return;
  const int K = xb - xa + 12;      // stages: current rows xa-6 .. xb+5
  // window starts relative to the origin, in floats (>= -8) and byte counts
  const int cz = z0 - 12, pz = z0 - 4;
  const int clen = min(WC, P - kStreamCoff - cz), plen = min(WP, P - kStreamCoff - pz);
  const uint32_t cbytes = (uint32_t)clen * 4u, pbytes = (uint32_t)plen * 4u;

  const float *curr = a.curr + (long long)shot * a.shot_stride + cz;
  float *prev = a.prev + (long long)shot * a.shot_stride;
  const float *prevw = prev + pz;
  const float *rcpw = a.rcp + (long long)(shot / a.shots_per_vel) * a.vel_stride + pz;

  if (t == 0) {
    for (int i = 0; i < NP; i++) mbar_init(&bar[i], 1);
    fence_mbar_init();
    s_fail = 0;
  }
  if constexpr (NW == 1) __syncwarp();
  else __syncthreads();

  auto issue = [&](int k) {
    int slot = k % NP;
    mbar_expect_tx(&bar[slot], cbytes + (k >= 12 ? 2u * pbytes : 0u));
    bulk_g2s(&cring[k & (NC - 1)][0], curr + (long long)(xa - 6 + k) * P, cbytes, &bar[slot]);
    if (k >= 12) {
      long long off = (long long)(xa - 12 + k) * P;
      bulk_g2s(&pring[slot][0], prevw + off, pbytes, &bar[slot]);
      bulk_g2s(&vring[slot][0], rcpw + off, pbytes, &bar[slot]);
    }
  };
  if (t == 0)
    for (int k = 0; k < D && k < K; k++) issue(k);

  // per-depth sponge ramps of this thread's 4 depths
  float dz[4] = {-1.f, -1.f, -1.f, -1.f};
  bool zok[4];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    int z = zg + i;
    zok[i] = z >= 6 && z < nz - 6;
    if constexpr (DAMPED) dz[i] = (z >= 0 && z < nz) ? a.damp_z[z] : -1.f;
  }
  const bool outgroup = t >= 1 && t < NT - 1 && zg < nz - 6 && zg + 3 >= 6;
  const bool fullgroup = zok[0] && zok[1] && zok[2] && zok[3];

  int k = 0;
  for (; k < K; k++) {
    if (!mbar_wait(&bar[k % NP], (uint32_t)((k / NP) & 1))) {
      atomicExch(a.err, 1);
      s_fail = 1;
    }
    if (k >= 10) {
      // u2 of row r = xa - 11 + k: rows r-5 .. r+5 are stages k-10 .. k
      const float *rowc = &cring[(k - 5) & (NC - 1)][0];
      float zn[20];
      {
        float4 v0 = ld4(rowc + 4 * t), v1 = ld4(rowc + 4 * t + 4), v2 = ld4(rowc + 4 * t + 8),
               v3 = ld4(rowc + 4 * t + 12), v4 = ld4(rowc + 4 * t + 16);
        zn[0] = v0.x; zn[1] = v0.y; zn[2] = v0.z; zn[3] = v0.w;
        zn[4] = v1.x; zn[5] = v1.y; zn[6] = v1.z; zn[7] = v1.w;
        zn[8] = v2.x; zn[9] = v2.y; zn[10] = v2.z; zn[11] = v2.w;
        zn[12] = v3.x; zn[13] = v3.y; zn[14] = v3.z; zn[15] = v3.w;
        zn[16] = v4.x; zn[17] = v4.y; zn[18] = v4.z; zn[19] = v4.w;
      }
      float4 xm4[6], xp4[6];
#pragma unroll
      for (int d = 1; d <= 5; d++) {
        xm4[d] = ld4(&cring[(k - 5 - d) & (NC - 1)][8 + 4 * t]);
        xp4[d] = ld4(&cring[(k - 5 + d) & (NC - 1)][8 + 4 * t]);
      }
      float u[4];
#pragma unroll
      for (int i = 0; i < 4; i++) {
        float xm[6], xp[6];
#pragma unroll
        for (int d = 1; d <= 5; d++) {
          xm[d] = get(xm4[d], i);
          xp[d] = get(xp4[d], i);
        }
        xm[0] = xp[0] = 0.f;
        u[i] = lap_pt<ARITH>(zn, i, xm, xp);
      }
      st4(&u2r[k & 3][4 * t], make_float4(u[0], u[1], u[2], u[3]));
    }
    if constexpr (NW == 1) __syncwarp();
    else __syncthreads();
    if (s_fail) break;
    if (t == 0 && k + D < K) {
      fence_proxy_async();
      issue(k + D);
    }
    if (k >= 12 && outgroup) {
      const int j = xa - 12 + k;   // output row; u2 rows j-1, j, j+1 are steps k-2, k-1, k
      const float *um = &u2r[(k - 2) & 3][4 * t];
      const float *uc = &u2r[(k - 1) & 3][4 * t];
      const float *up = &u2r[k & 3][4 * t];
      float4 c4 = ld4(&cring[(k - 6) & (NC - 1)][8 + 4 * t]);
      float4 p4 = ld4(&pring[k % NP][4 * t]);
      float4 r4 = ld4(&vring[k % NP][4 * t]);
      float4 um4 = ld4(um), uc4 = ld4(uc), up4 = ld4(up);
      float ucl = uc[-1], ucr = uc[4];
      float dxr = 0.f;
      if constexpr (DAMPED) dxr = (j < a.ramp || j >= nx - a.ramp) ? a.damp_x[j] : 0.f;
      float o[4];
#pragma unroll
      for (int i = 0; i < 4; i++) {
        float delta = 0.f;
        if constexpr (DAMPED) {
          float dist = dz[i] >= 0.f ? dz[i] : dxr;
          delta = __fmul_rn(__fmul_rn(0.05f, dist), dist);
        }
        float uzm = i == 0 ? ucl : get(uc4, i - 1);
        float uzp = i == 3 ? ucr : get(uc4, i + 1);
        o[i] = update_pt<ARITH>(get(c4, i), get(p4, i), get(r4, i), get(uc4, i), uzm, uzp,
                                get(um4, i), get(up4, i), delta);
      }
      float *dst = prev + (long long)j * P + zg;
      if (fullgroup) {
        st4(dst, make_float4(o[0], o[1], o[2], o[3]));
      } else {
#pragma unroll
        for (int i = 0; i < 4; i++)
          if (zok[i]) dst[i] = o[i];
      }
    }
  }
  if (s_fail && t == 0) {
    // wait (bounded) for this CTA's copies still in flight before leaving
    for (int i = k + 1; i < K && i < k + D; i++) mbar_wait(&bar[i % NP], (uint32_t)((i / NP) & 1));
  }
}

}  // namespace swfwi
