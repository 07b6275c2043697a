// Register-queue streaming step for sm_100a (same scheme, arithmetics and
// layout as stream.cuh; FAST results bit-identical to fd_step_ws).
//
// Every warp is a self-contained pipeline over one task: a 120-deep slice
// of depths [zo, zo+120) and a chunk of consecutive rows of one shot.  No
// producer warp, no CTA barrier:
//  * lane 0 issues TMA bulk copies (cp.async.bulk global -> shared,
//    completion on the warp's own mbarriers) D = 3 or 7 stages ahead; stage
//    k brings current row xa-6+k (depths [zo-12, zo+132)) into an 8- or
//    16-slot ring and, from stage 12 on, previous-field and 1/vt rows
//    xa-12+k (depths [zo, zo+120)) into 4- or 8-slot rings;
//  * lane l owns depths zg = zo-4+4l .. zg+3 and keeps its own values of the
//    11 current rows around the u2 row in registers (a queue shifted by one
//    row per step; the main loop is unrolled by the ring length, so ring
//    slots and barriers are constants and the shift is register renaming
//    but for a rotation at the loop edge), so of the current row only the
//    newly landed row and the z neighbours of the centre row are read from
//    shared memory;
//  * all 32 lanes form u2 (128 depths), lanes 1..30 write the 120 outputs;
//    u2's z neighbours at the group edges come by warp shuffle, its x
//    neighbours are the previous two steps' u2 in registers.
// A slot is refilled only after a __syncwarp that follows its last read.
// Every mbarrier wait is bounded: on timeout the warp raises the error flag,
// waits (bounded) for its own copies in flight and leaves.
#pragma once
#include "stream.cuh"

namespace swfwi {

namespace rq_detail {
using namespace stream_detail;

constexpr int kOutLanes = 30;               // lanes 1..30 write outputs
constexpr int kDepths = 4 * kOutLanes;      // output depths per warp task
constexpr int WC = 4 * 32 + 16;             // current window [zo-12, zo+132)
constexpr int WP = kDepths;                 // previous / 1/vt window [zo, zo+120)

// Rings of one warp: NC current-row slots, NP previous-field / 1/vt slots,
// D stages issued ahead (D + 5 <= NC: a current row is read until 5 steps
// after it lands; D <= NP).  D = 3: 8 + 4 slots, 8.5 KB; D = 7: 16 + 8
// slots, 17 KB.
template <int D>
struct Ring {
  static constexpr int NC = D <= 3 ? 8 : 16;
  static constexpr int NP = D <= 3 ? 4 : 8;
  static_assert(D + 5 <= NC && D <= NP, "ring too short for the lookahead");
};

template <int D>
struct WarpSmem {
  float c[Ring<D>::NC][WC];
  float p[Ring<D>::NP][WP];
  float v[Ring<D>::NP][WP];
  uint64_t full[Ring<D>::NC];
};
static_assert(sizeof(WarpSmem<3>) % 16 == 0 && sizeof(WarpSmem<7>) % 16 == 0,
              "per-warp areas must stay 16-byte aligned");

// slices of 120 output depths covering [6, nz-6) from zo = 4
__host__ __device__ inline int slices(int nz) { return (nz - 10 + kDepths - 1) / kDepths; }

}  // namespace rq_detail

template <int NW, int D>
constexpr size_t rq_smem_bytes() {
  return sizeof(rq_detail::WarpSmem<D>) * NW;
}

// Resident warps per SM the launch bounds aim at: with D = 3, 20 (FAST: 96
// registers a thread; 8.5 KB of rings a warp), 10 for REF; with D = 7, 12
// (17 KB a warp), 8 for REF.
template <int NW, int ARITH, int D>
constexpr int rq_min_blocks() {
  constexpr int warps = D <= 3 ? (ARITH == ARITH_REF ? 10 : 20) : (ARITH == ARITH_REF ? 8 : 12);
  return warps / NW > 0 ? warps / NW : 1;
}

template <int ARITH, bool DAMPED, int NW, int D>
__global__ void __launch_bounds__(NW * 32, rq_min_blocks<NW, ARITH, D>())
fd_step_rq(StreamArgs a, int nslots) {
  using namespace rq_detail;
  constexpr int NC = Ring<D>::NC, NP = Ring<D>::NP;
  constexpr int LNC = NC == 8 ? 3 : 4;   // log2(NC)
  extern __shared__ __align__(128) unsigned char smem[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  WarpSmem<D> &S = reinterpret_cast<WarpSmem<D> *>(smem)[w];

  const int nx = a.nx, nz = a.nz, P = a.pitch;
  const int nsl = slices(nz);
  const int nchunks = (nx - 12 + a.xchunk - 1) / a.xchunk;
  const long long task = (long long)blockIdx.x * NW + w;
  const int slice = (int)(task % nsl);
  const long long rest = task / nsl;
  const int shot = (int)(rest % nslots);
  const int chunk = (int)(rest / nslots);
  if (chunk >= nchunks) return;
  const int zo = 4 + slice * kDepths;
  const int xa = 6 + chunk * a.xchunk;
  const int xb = min(xa + a.xchunk, nx - 6);
  const int K = xb - xa + 12;   // stages: current rows xa-6 .. xb+5

  // windows (floats from the origin; rows of P floats, origin 8 floats in)
  const int cz = zo - 12;
  const uint32_t cbytes = 4u * (uint32_t)min(WC, P - kStreamCoff - cz);
  const uint32_t pbytes = 4u * (uint32_t)min(WP, P - kStreamCoff - zo);
  float *prevb = a.prev + (long long)shot * a.shot_stride;
  // next stage's source rows: current row xa-6+s; previous field and 1/vt
  // row xa-12+s (used from s = 12 on)
  const float *src_c = a.curr + (long long)shot * a.shot_stride + cz + (long long)(xa - 6) * P;
  const float *src_p = prevb + zo + (long long)(xa - 12) * P;
  const float *src_v = a.rcp + (long long)(shot / a.shots_per_vel) * a.vel_stride + zo + (long long)(xa - 12) * P;

  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < NC; i++) mbar_init(&S.full[i], 1);
    fence_mbar_init();
  }
  __syncwarp();

  // lane 0 issues stage s into slot s % NC (current row) and s % NP
  // (previous field and 1/vt, from stage 12 on)
  // Lanes 0..2 each issue one copy of a stage (called by the whole warp):
  // lane 0 the current row and the barrier's arrival with the stage's byte
  // count, lanes 1 and 2 the previous-field and 1/vt rows (from stage 12
  // on).  A lane's source row pointer and ring base are fixed.
  const float *my_src = lane == 0 ? src_c : (lane == 1 ? src_p : src_v);
  const uint32_t my_ring = lane == 0 ? smem_u32(&S.c[0][0]) : (lane == 1 ? smem_u32(&S.p[0][0]) : smem_u32(&S.v[0][0]));
  const uint32_t my_slot_bytes = lane == 0 ? 4u * WC : 4u * WP;
  const uint32_t my_bytes = lane == 0 ? cbytes : pbytes;
  auto issue = [&](int s, int cs, int ps) {
    if (lane < 3) {
      const bool pv = s >= 12;
      const uint32_t bar = smem_u32(&S.full[cs]);
      if (lane == 0) mbar_expect_tx(&S.full[cs], cbytes + (pv ? 2u * pbytes : 0u));
      if (lane == 0 || pv)
        bulk_g2s_u32(my_ring + (uint32_t)(lane == 0 ? cs : ps) * my_slot_bytes, my_src + (long long)s * P, my_bytes,
                     bar);
    }
  };
  for (int s = 0; s < D && s < K; s++) issue(s, s & (NC - 1), s & (NP - 1));

  // ---- this lane's depths
  const int zg = zo - 4 + 4 * lane;
  bool zok[4];
#pragma unroll
  for (int i = 0; i < 4; i++) zok[i] = zg + i >= 6 && zg + i < nz - 6;
  const bool outgroup = lane >= 1 && lane <= kOutLanes && zg < nz - 6 && zg + 3 >= 6;
  const bool fullgroup = zok[0] && zok[1] && zok[2] && zok[3];
  const int zw = 4 * lane;                      // z window (depths zg-8 .. zg+11) in the current window
  const int qo = 4 * lane + 8;                  // own depths in the current window
  const int po = 4 * min(max(lane - 1, 0), kOutLanes - 1);   // own depths in the previous / 1/vt
                                                             // window (lanes 0, 31: a neighbour's)
  float *outp = (a.out ? a.out + (long long)shot * a.shot_stride : prevb) + (long long)xa * P + zg;   // output row xa, a row per output

  // sponge: the bottom ramp (per depth) overrides the left/right one (per
  // row).  REF keeps the depth ramp dz (-1 above the bottom sponge); FAST
  // keeps this lane's update coefficients next = cf*c + pc*p + inc for rows
  // outside the x ramps ((2, -1) undamped; pc > -1 exactly where the bottom
  // ramp acts) and takes the row's, a.coef_x, on ramp rows.
  float dz[4] = {-1.f, -1.f, -1.f, -1.f};
  float2 coefz[2] = {make_float2(2.f, 2.f), make_float2(2.f, 2.f)};
  float2 pcz[2] = {make_float2(-1.f, -1.f), make_float2(-1.f, -1.f)};
  if constexpr (DAMPED) {
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int z = zg + i;
      const float d = (z >= 0 && z < nz) ? a.damp_z[z] : -1.f;
      if constexpr (ARITH == ARITH_FAST) {
        const float2 c = fast_damp_coef(d >= 0.f ? d : 0.0f);
        float2 &cr = i < 2 ? coefz[0] : coefz[1];
        float2 &pr = i < 2 ? pcz[0] : pcz[1];
        if (i & 1) { cr.y = c.x; pr.y = c.y; }
        else { cr.x = c.x; pr.x = c.y; }
      } else {
        dz[i] = d;
      }
    }
  }
  const float *damp_row = a.damp_x + xa - 12;   // damp_x of output row xa-12+k
  const float2 *coef_row = a.coef_x + xa - 12;  // its FAST coefficients
  const int k_ramp_lo = a.ramp - xa + 12, k_ramp_hi = nx - a.ramp - xa + 12;
  // rows k_ramp_lo <= k < k_ramp_lo + ramp_span are off the ramps (none when
  // the ramps overlap)
  const unsigned ramp_span = (unsigned)max(k_ramp_hi - k_ramp_lo, 0);

  float4 q[11];   // own values of current rows (stages k-10 .. k after the push)
  float4 um = make_float4(0.f, 0.f, 0.f, 0.f), uc = um;   // u2 of the two previous rows

  // One step; U = k % NC is a compile-time constant, so every ring slot and
  // barrier is one.  k < 10: fill the queue; k >= 10: u2 of row xa-11+k
  // (centre q[5]); k >= 12: output row xa-12+k (c = q[4]).
  auto step = [&](auto u, int k, uint32_t parity) -> bool {
    constexpr int U = decltype(u)::value;
    constexpr int SC = U, SZ = (U - 5 + NC) % NC, SP = U % NP;
    // warp-uniform outcome: the shuffles and __syncwarp below need every lane
    if (!__all_sync(0xffffffffu, mbar_wait(&S.full[SC], parity))) return false;
#pragma unroll
    for (int j = 0; j < 10; j++) q[j] = q[j + 1];
    q[10] = ld4(&S.c[SC][qo]);
    if (k >= 10) {
      const float *rowc = &S.c[SZ][zw];
      const float4 v0 = ld4(rowc), v1 = ld4(rowc + 4), v3 = ld4(rowc + 12), v4 = ld4(rowc + 16);
      const float4 v2 = q[5];
      const float zn[20] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w, v2.x, v2.y,
                            v2.z, v2.w, v3.x, v3.y, v3.z, v3.w, v4.x, v4.y, v4.z, v4.w};
      float4 up;
      if constexpr (ARITH == ARITH_FAST) {
        const float a5[6] = {-4.0f * SWFWI_A0, SWFWI_A1, SWFWI_A2, SWFWI_A3, SWFWI_A4, SWFWI_A5};
        float2 acc[2];
#pragma unroll
        for (int pr = 0; pr < 2; pr++) {
          const int i = 2 * pr;
          acc[pr] = __fmul2_rn(make_float2(a5[0], a5[0]), pr == 0 ? lo2(v2) : hi2(v2));
#pragma unroll
          for (int kk = 1; kk <= 5; kk++) {
            float2 zs;
            if (kk & 1)   // unaligned depth pairs: two scalar adds
              zs = make_float2(__fadd_rn(zn[8 + i - kk], zn[8 + i + kk]), __fadd_rn(zn[9 + i - kk], zn[9 + i + kk]));
            else
              zs = __fadd2_rn(make_float2(zn[8 + i - kk], zn[9 + i - kk]), make_float2(zn[8 + i + kk], zn[9 + i + kk]));
            const float2 xs = pr == 0 ? __fadd2_rn(lo2(q[5 - kk]), lo2(q[5 + kk]))
                                      : __fadd2_rn(hi2(q[5 - kk]), hi2(q[5 + kk]));
            acc[pr] = __ffma2_rn(make_float2(a5[kk], a5[kk]), __fadd2_rn(zs, xs), acc[pr]);
          }
        }
        up = make_float4(acc[0].x, acc[0].y, acc[1].x, acc[1].y);
      } else {
        float uu[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
          float xm[6], xp[6];
          xm[0] = xp[0] = 0.f;
#pragma unroll
          for (int d = 1; d <= 5; d++) {
            xm[d] = get(q[5 - d], i);
            xp[d] = get(q[5 + d], i);
          }
          uu[i] = lap_pt<ARITH>(zn, i, xm, xp);
        }
        up = make_float4(uu[0], uu[1], uu[2], uu[3]);
      }
      if (k >= 12) {
        // u2 rows: um = xa-13+k, uc = xa-12+k, up = xa-11+k
        const float ucl = __shfl_up_sync(0xffffffffu, uc.w, 1);
        const float ucr = __shfl_down_sync(0xffffffffu, uc.x, 1);
        const float4 c4 = q[4];
        const float4 p4 = ld4(&S.p[SP][po]);
        const float4 r4 = ld4(&S.v[SP][po]);
        // a left/right ramp row: one unsigned compare, marked unlikely (7 %
        // of the rows on the benchmark grid), so the test stays a branch
        const bool ramp_row =
            __builtin_expect(DAMPED && (unsigned)(k - k_ramp_lo) >= ramp_span, 0);
        float4 o;
        if constexpr (ARITH == ARITH_FAST) {
          float2 cf0 = coefz[0], cf1 = coefz[1], pc0 = pcz[0], pc1 = pcz[1];
          if (ramp_row) {   // a left/right ramp row: the row's coefficients where no bottom ramp acts
            const float2 cx = coef_row[k];
            if (pc0.x == -1.f) { cf0.x = cx.x; pc0.x = cx.y; }
            if (pc0.y == -1.f) { cf0.y = cx.x; pc0.y = cx.y; }
            if (pc1.x == -1.f) { cf1.x = cx.x; pc1.x = cx.y; }
            if (pc1.y == -1.f) { cf1.y = cx.x; pc1.y = cx.y; }
          }
          // pair 0: depths zg, zg+1 (z neighbours ucl|uc.x .. uc.y|uc.z)
          const float2 o0 = update_pair_coef(lo2(c4), lo2(p4), lo2(r4), lo2(uc),
                                             make_float2(__fadd_rn(ucl, uc.y), __fadd_rn(uc.x, uc.z)), lo2(um),
                                             lo2(up), cf0, pc0);
          const float2 o1 = update_pair_coef(hi2(c4), hi2(p4), hi2(r4), hi2(uc),
                                             make_float2(__fadd_rn(uc.y, uc.w), __fadd_rn(uc.z, ucr)), hi2(um),
                                             hi2(up), cf1, pc1);
          o = make_float4(o0.x, o0.y, o1.x, o1.y);
        } else {
          const float dxr = ramp_row ? damp_row[k] : 0.f;
          float oo[4];
#pragma unroll
          for (int i = 0; i < 4; i++) {
            float delta = 0.f;
            if constexpr (DAMPED) {
              const float dist = dz[i] >= 0.f ? dz[i] : dxr;
              delta = __fmul_rn(__fmul_rn(0.05f, dist), dist);
            }
            const float uzm = i == 0 ? ucl : get(uc, i - 1);
            const float uzp = i == 3 ? ucr : get(uc, i + 1);
            oo[i] = update_pt<ARITH>(get(c4, i), get(p4, i), get(r4, i), get(uc, i), uzm, uzp,
                                     get(um, i), get(up, i), delta);
          }
          o = make_float4(oo[0], oo[1], oo[2], oo[3]);
        }
        if (outgroup) {
          if (fullgroup) {
            st4(outp, o);
          } else {
            if (zok[0]) outp[0] = o.x;
            if (zok[1]) outp[1] = o.y;
            if (zok[2]) outp[2] = o.z;
            if (zok[3]) outp[3] = o.w;
          }
        }
        outp += P;
      }
      um = uc;
      uc = up;
    }
    // every lane is done with slot (k+D) % NC (its last read, the z window
    // of stage k+D-NC, was this step's or earlier) and with the previous /
    // 1/vt slot of stage k+D-NP: refill them.  Every value read from a slot
    // has fed this step's arithmetic (and its stores) or an earlier step's
    // before the refill is issued, as in a release through an "empty"
    // barrier.
    __syncwarp();
    if (k + D < K) issue(k + D, (U + D) % NC, (U + D) % NP);
    return true;
  };

  bool ok = true;
  int k = 0;
  // the loop is unrolled by the ring length: every step's slot is a
  // constant, the queue's shift is renaming (its period, 11, leaves a
  // rotation at the loop edge)
#define SWFWI_RQ_STEP(U)                                               \
  if constexpr ((U) < NC) {                                            \
    k = k0 + (U);                                                      \
    if (k >= K) break;                                                 \
    if (!step(std::integral_constant<int, (U)>{}, k, parity)) {       \
      ok = false;                                                      \
      break;                                                           \
    }                                                                  \
  }
  for (int k0 = 0;; k0 += NC) {
    const uint32_t parity = (uint32_t)((k0 >> LNC) & 1);
    SWFWI_RQ_STEP(0) SWFWI_RQ_STEP(1) SWFWI_RQ_STEP(2) SWFWI_RQ_STEP(3)
    SWFWI_RQ_STEP(4) SWFWI_RQ_STEP(5) SWFWI_RQ_STEP(6) SWFWI_RQ_STEP(7)
    SWFWI_RQ_STEP(8) SWFWI_RQ_STEP(9) SWFWI_RQ_STEP(10) SWFWI_RQ_STEP(11)
    SWFWI_RQ_STEP(12) SWFWI_RQ_STEP(13) SWFWI_RQ_STEP(14) SWFWI_RQ_STEP(15)
  }
#undef SWFWI_RQ_STEP
  if (!ok) {
    if (lane == 0) {
      atomicExch(a.err, 1);
      // wait (bounded) for the copies this warp already issued: stages k .. k+D-1
      for (int i = k; i < K && i < k + D; i++) mbar_wait(&S.full[i & (NC - 1)], (uint32_t)((i >> LNC) & 1));
    }
    __syncwarp();
  }
}

}  // namespace swfwi
