// 4th-order-time / 10th-order-space acoustic step for sm_100a.
//
// The scheme is swfwi's (src/modeling/fd4t10s-damp-zjh.c:14-115 damped,
// src/modeling/fd4t10s-zjh.c:10-56 undamped):
//   pass 1  u2 = -4 a0 c + sum_k a_k (c[z-k] + c[z+k] + c[x-k] + c[x+k]), k = 1..5
//   pass 2  next = (2 - 2d + d^2) c - (1 - 2d) prev + u2/vt
//                  + (1/12)(1/vt)^2 (u2[z-1] + u2[z+1] + u2[x-1] + u2[x+1] - 4 u2)
// with d = 0.05 dist^2 on the left/right/bottom sponge.  Layout p[x*nz + z]
// (z contiguous); outputs on [6, nx-6) x [6, nz-6), in place over prev (or
// into a separate output field, StepArgs::out).
//
// One CTA owns a TX x 32 output tile.  It stages the (TX+12) x 44 halo of
// the current field in shared memory, forms u2 on the (TX+2) x 34 ring in
// shared memory (u2 never reaches HBM: the reference's u2 scratch array and
// its second sweep disappear), then writes TX*32 outputs.  prev and the
// velocity term are fetched into registers before the first barrier so their
// latency overlaps the tile load.  Each warp reads 32 consecutive z values:
// coalesced rows of 128 B.
//
// Three arithmetics (template parameter ARITH):
//   ARITH_REF  float storage; each operation rounded exactly as the
//              reference's C expression is on x86-64 (its 4.0 and 2. literals
//              promote the running sums to double; no FMA contraction).  The
//              result is bit-identical to the reference CPU kernel.
//   ARITH_FAST float storage, FP32 with FMA (tolerance parity).
//   ARITH_F64  double storage and arithmetic: the FP64 oracle of the scheme.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace swfwi {

enum Arith { ARITH_REF = 0, ARITH_FAST = 1, ARITH_F64 = 2 };

// Zhang Jinhai's coefficients (fd4t10s-damp-zjh.c:24-29), float as in the
// reference.
#define SWFWI_A0 (+1.53400796f)
#define SWFWI_A1 (+1.78858721f)
#define SWFWI_A2 (-0.31660756f)
#define SWFWI_A3 (+0.07612173f)
#define SWFWI_A4 (-0.01626042f)
#define SWFWI_A5 (+0.00216736f)

struct StepArgs {
  void *prev;           // [shot][nx][nz] (element type per ARITH)
  void *out = nullptr;  // where the next field goes (same layout); nullptr: in place over prev
  const void *curr;     // same
  const void *vel;      // vt, or 1/vt when VEL_IS_RCP
  int nx, nz;           // padded grid
  int pitch;            // elements between rows (>= nz)
  int bx0;              // sponge width + 6 (damping ramp length)
  long long shot_stride;   // elements between the fields of consecutive shots
  long long vel_stride;    // elements between velocity models
  int shots_per_vel;       // shots sharing one velocity model
};

template <typename T>
struct ArithT;

// Reciprocal of the velocity term; identical to the reference's 1.0f/vt.
__device__ __forceinline__ float rcp_ref(float v) { return __fdiv_rn(1.0f, v); }

// Sponge ramp of fd4t10s-damp-zjh.c:64-80 (the bottom branch overrides).
__device__ __forceinline__ float damp_dist(int ix, int iz, int nx, int nz, int nb) {
  float dist = 0.0f;
  if (ix < nb) dist = __fdiv_rn((float)(nb - ix), (float)nb);
  if (ix >= nx - nb) dist = __fdiv_rn((float)(ix - (nx - nb) + 1), (float)nb);
  if (iz >= nz - nb) dist = __fdiv_rn((float)(iz - (nz - nb) + 1), (float)nb);
  return dist;
}

// ---- pass 1: u2 from a shared-memory tile; c points at the centre -------
template <int ARITH, int CZ, typename T>
__device__ __forceinline__ T lap10(const T *c) {
  if constexpr (ARITH == ARITH_REF) {
    // (-4.0 * a0) * c in double, then + (double)(a_k * S_k) with S_k summed
    // left to right as z-k, z+k, x-k, x+k.
    const double m4a0 = -4.0 * (double)SWFWI_A0;
    double acc = __dmul_rn(m4a0, (double)c[0]);
#define SWFWI_REF_TERM(K, A)                                                  \
  {                                                                           \
    float s = __fadd_rn(__fadd_rn(__fadd_rn(c[-K], c[K]), c[-K * CZ]), c[K * CZ]); \
    acc = __dadd_rn(acc, (double)__fmul_rn(A, s));                            \
  }
    SWFWI_REF_TERM(1, SWFWI_A1)
    SWFWI_REF_TERM(2, SWFWI_A2)
    SWFWI_REF_TERM(3, SWFWI_A3)
    SWFWI_REF_TERM(4, SWFWI_A4)
    SWFWI_REF_TERM(5, SWFWI_A5)
#undef SWFWI_REF_TERM
    return (T)__double2float_rn(acc);
  } else if constexpr (ARITH == ARITH_FAST) {
    float s1 = (c[-1] + c[1]) + (c[-CZ] + c[CZ]);
    float s2 = (c[-2] + c[2]) + (c[-2 * CZ] + c[2 * CZ]);
    float s3 = (c[-3] + c[3]) + (c[-3 * CZ] + c[3 * CZ]);
    float s4 = (c[-4] + c[4]) + (c[-4 * CZ] + c[4 * CZ]);
    float s5 = (c[-5] + c[5]) + (c[-5 * CZ] + c[5 * CZ]);
    float acc = (-4.0f * SWFWI_A0) * c[0];
    acc = fmaf(SWFWI_A1, s1, acc);
    acc = fmaf(SWFWI_A2, s2, acc);
    acc = fmaf(SWFWI_A3, s3, acc);
    acc = fmaf(SWFWI_A4, s4, acc);
    acc = fmaf(SWFWI_A5, s5, acc);
    return (T)acc;
  } else {
    double acc = -4.0 * (double)SWFWI_A0 * c[0];
    acc += (double)SWFWI_A1 * (c[-1] + c[1] + c[-CZ] + c[CZ]);
    acc += (double)SWFWI_A2 * (c[-2] + c[2] + c[-2 * CZ] + c[2 * CZ]);
    acc += (double)SWFWI_A3 * (c[-3] + c[3] + c[-3 * CZ] + c[3 * CZ]);
    acc += (double)SWFWI_A4 * (c[-4] + c[4] + c[-4 * CZ] + c[4 * CZ]);
    acc += (double)SWFWI_A5 * (c[-5] + c[5] + c[-5 * CZ] + c[5 * CZ]);
    return (T)acc;
  }
}

// ---- pass 2: time update at one point ----------------------------------
// u points at u2 of the point inside the u2 tile (row length UZ).
template <int ARITH, int UZ, typename T>
__device__ __forceinline__ T update_point(T c, T p, T r, const T *u, float delta) {
  if constexpr (ARITH == ARITH_REF) {
    float uc = u[0];
    float lap = __fsub_rn(__fadd_rn(__fadd_rn(__fadd_rn(u[-1], u[1]), u[-UZ]), u[UZ]),
                          __fmul_rn(4.0f, uc));
    float t4 = __fmul_rn(__fmul_rn(__fmul_rn(1.0f / 12.0f, r), r), lap);
    double acc;
    if (delta == 0.0f) {
      // (2 - 0 + 0) * c - (1 - 0) * prev: the same bits as the undamped form
      acc = __dsub_rn(__dmul_rn(2.0, (double)c), (double)p);
    } else {
      float d2 = __fmul_rn(2.0f, delta);
      double coef = __dadd_rn(__dsub_rn(2.0, (double)d2), (double)__fmul_rn(delta, delta));
      acc = __dsub_rn(__dmul_rn(coef, (double)c), (double)__fmul_rn(__fsub_rn(1.0f, d2), p));
    }
    acc = __dadd_rn(acc, (double)__fmul_rn(r, uc));
    acc = __dadd_rn(acc, (double)t4);
    return (T)__double2float_rn(acc);
  } else if constexpr (ARITH == ARITH_FAST) {
    float uc = u[0];
    float lap = ((u[-1] + u[1]) + (u[-UZ] + u[UZ])) - 4.0f * uc;
    float q = r * (1.0f / 12.0f);
    float inc = r * fmaf(q, lap, uc);
    float base;
    if (delta == 0.0f) {
      base = fmaf(2.0f, c, -p);
    } else {
      float d2 = 2.0f * delta;
      base = fmaf(2.0f - d2 + delta * delta, c, -(1.0f - d2) * p);
    }
    return (T)(base + inc);
  } else {
    double uc = u[0];
    double lap = u[-1] + u[1] + u[-UZ] + u[UZ] - 4.0 * uc;
    double d = (double)delta;
    return (T)((2.0 - 2.0 * d + d * d) * c - (1.0 - 2.0 * d) * p + r * uc +
               (1.0 / 12.0) * r * r * lap);
  }
}

template <int ARITH>
struct StorageOf { typedef float type; };
template <>
struct StorageOf<ARITH_F64> { typedef double type; };

// The damping value at a point: 0.05 * dist^2, rounded as the reference does
// ((max_delta * dist) * dist in float).  F64 uses the same float dist.
__device__ __forceinline__ float damp_delta(int ix, int iz, int nx, int nz, int nb) {
  float dist = damp_dist(ix, iz, nx, nz, nb);
  return __fmul_rn(__fmul_rn(0.05f, dist), dist);
}

constexpr int kStepThreads = 256;
constexpr int kTZ = 32;

template <int ARITH, bool DAMPED, bool VEL_IS_RCP, int TX>
__global__ void __launch_bounds__(kStepThreads)
fd_step_tile(StepArgs a) {
  typedef typename StorageOf<ARITH>::type T;
  constexpr int H = 6;
  constexpr int CX = TX + 2 * H, CZ = kTZ + 2 * H;
  constexpr int UX = TX + 2, UZ = kTZ + 2;
  constexpr int ROWS = kStepThreads / 32;      // warps, one output row each pass
  constexpr int PER = TX / ROWS;               // outputs per thread
  __shared__ T sc[CX * CZ];
  __shared__ T su[UX * UZ];

  const int nx = a.nx, nz = a.nz, pitch = a.pitch;
  const int shot = blockIdx.z;
  const int x0 = H + blockIdx.y * TX;
  const int z0 = H + blockIdx.x * kTZ;
  const T *curr = (const T *)a.curr + (long long)shot * a.shot_stride;
  T *prev = (T *)a.prev + (long long)shot * a.shot_stride;
  const T *vel = (const T *)a.vel + (long long)(shot / a.shots_per_vel) * a.vel_stride;

  const int tz = threadIdx.x & 31;
  const int ty = threadIdx.x >> 5;
  const int gz = z0 + tz;

  // Early fetch of prev and the velocity term for this thread's outputs.
  T pv[PER], rv[PER];
#pragma unroll
  for (int k = 0; k < PER; k++) {
    int gx = x0 + ty + ROWS * k;
    pv[k] = 0;
    rv[k] = 1;
    if (gx < nx - H && gz < nz - H) {
      long long idx = (long long)gx * pitch + gz;
      pv[k] = prev[idx];
      rv[k] = vel[idx];
    }
  }

  // Stage the current field with its 6-cell halo.
  for (int i = threadIdx.x; i < CX * CZ; i += kStepThreads) {
    int lx = i / CZ, lz = i - lx * CZ;
    int gx = x0 - H + lx, gzz = z0 - H + lz;
    T v = 0;
    if (gx < nx && gzz < nz) v = curr[(long long)gx * pitch + gzz];
    sc[i] = v;
  }
  __syncthreads();

  // u2 on the tile plus a one-cell ring.
  for (int i = threadIdx.x; i < UX * UZ; i += kStepThreads) {
    int ux = i / UZ, uz = i - ux * UZ;
    su[i] = lap10<ARITH, CZ, T>(&sc[(ux + H - 1) * CZ + (uz + H - 1)]);
  }
  __syncthreads();

#pragma unroll
  for (int k = 0; k < PER; k++) {
    int lx = ty + ROWS * k;
    int gx = x0 + lx;
    if (gx < nx - H && gz < nz - H) {
      T r;
      if constexpr (VEL_IS_RCP) {
        r = rv[k];
      } else if constexpr (ARITH == ARITH_F64) {
        r = 1.0 / rv[k];
      } else {
        r = rcp_ref(rv[k]);
      }
      float delta = 0.0f;
      if constexpr (DAMPED) delta = damp_delta(gx, gz, nx, nz, a.bx0);
      T c = sc[(lx + H) * CZ + (tz + H)];
      T *dst = a.out ? (T *)a.out + (long long)shot * a.shot_stride : prev;
      dst[(long long)gx * pitch + gz] = update_point<ARITH, UZ, T>(c, pv[k], r, &su[(lx + 1) * UZ + (tz + 1)], delta);
    }
  }
}

}  // namespace swfwi
