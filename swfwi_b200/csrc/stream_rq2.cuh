// Two-row register-queue streaming step for sm_100a (kernel 6; FAST
// arithmetic; same scheme, layout and results as fd_step_rq, stream_rq.cuh).
//
// As in fd_step_rq every warp is its own pipeline over one task (120 output
// depths of one shot, a chunk of rows), with no CTA barrier, but a stage
// brings two rows instead of one, so the per-stage work that does not
// depend on the row count (the barrier wait and its vote, the copy issue,
// the queue rotation, the loop's tests) is paid once per two rows:
//  * six lanes issue the stage's TMA bulk copies (cp.async.bulk global ->
//    shared, completion on the stage's mbarrier) two stages (four rows)
//    ahead: current rows A, B (depths [zo-12, zo+132)) into a 6-stage ring,
//    and from stage 6 on the previous-field and 1/vt rows A, B (depths
//    [zo, zo+120)) into 3-stage rings; a row past the task's end is not
//    copied and the barrier expects its bytes only for the rows copied;
//  * lane l owns depths zo-4+4l .. +3 and keeps its own values of 12
//    current rows in registers (the two centre rows of the stage's two u2
//    rows and 5 on each side), shifted two rows a stage; the loop is
//    unrolled by the ring length (6 stages), so ring slots and barriers are
//    constants;
//  * each stage forms two u2 rows (z windows from the ring, x neighbours
//    from the queue, packed FP32x2 arithmetic) and writes two output rows
//    (u2 x neighbours from the two previous and two current u2 rows in
//    registers, z neighbours by shuffle).
// 126 registers a thread at 16 resident warps per SM (the 12-row queue does
// not fit the 96 registers of 20 warps without spilling); with one wave of
// tasks it issues 22 % fewer instructions than fd_step_rq and takes 8-10 %
// less time.  Every mbarrier wait is bounded: on timeout the warp raises the
// error flag, waits (bounded) for its own copies in flight and leaves.
#pragma once
#include "stream.cuh"

namespace swfwi {

namespace rq2_detail {
using namespace stream_detail;

constexpr int kOutLanes = 30;            // lanes 1..30 write outputs
constexpr int kDepths = 4 * kOutLanes;   // output depths per warp task
constexpr int WC = 4 * 32 + 16;          // current window [zo-12, zo+132)
constexpr int WP = kDepths;              // previous / 1/vt window [zo, zo+120)
constexpr int D2 = 2;                    // stages issued ahead
constexpr int NC = D2 + 4;               // a current row pair is read 3 stages after it lands
constexpr int NP = D2 + 1;               // divides NC: U % NP is the slot of stage k
static_assert(NC % NP == 0, "the previous-field ring must divide the current ring");

struct WarpSmem {
  float c[NC][2][WC];
  float p[NP][2][WP];
  float v[NP][2][WP];
  uint64_t full[NC];
};
static_assert(sizeof(float) * 2 * WC % 16 == 0 && sizeof(float) * 2 * WP % 16 == 0 &&
                  sizeof(float) * WP % 16 == 0 && sizeof(float) * WC % 16 == 0,
              "ring rows must stay 16-byte aligned");

__host__ __device__ inline int slices(int nz) { return (nz - 10 + kDepths - 1) / kDepths; }

}  // namespace rq2_detail

constexpr size_t rq2_smem_bytes() { return sizeof(rq2_detail::WarpSmem); }
constexpr int kRq2MinBlocks = 16;   // resident warps per SM the launch bounds aim at

template <bool DAMPED>
__global__ void __launch_bounds__(32, kRq2MinBlocks) fd_step_rq2(StreamArgs a, int nslots) {
  using namespace rq2_detail;
  extern __shared__ __align__(128) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  WarpSmem &S = *reinterpret_cast<WarpSmem *>(smem);

  const int nx = a.nx, nz = a.nz, P = a.pitch;
  const int nsl = slices(nz);
  const int nchunks = (nx - 12 + a.xchunk - 1) / a.xchunk;
  const long long task = blockIdx.x;
  const int slice = (int)(task % nsl);
  const long long rest = task / nsl;
  const int shot = (int)(rest % nslots);
  const int chunk = (int)(rest / nslots);
  if (chunk >= nchunks) return;
  const int zo = 4 + slice * kDepths;
  const int xa = 6 + chunk * a.xchunk;
  const int xb = min(xa + a.xchunk, nx - 6);
  const int R = xb - xa + 12;   // current rows xa-6 .. xb+5
  const int K2 = (R + 1) / 2;   // stages of two rows

  const int cz = zo - 12;
  const uint32_t cbytes = 4u * (uint32_t)min(WC, P - kStreamCoff - cz);
  const uint32_t pbytes = 4u * (uint32_t)min(WP, P - kStreamCoff - zo);
  float *prevb = a.prev + (long long)shot * a.shot_stride;
  // stage s: current rows xa-6+2s (A) and +1 (B); previous-field and 1/vt
  // rows xa-12+2s and +1 (from s = 6 on)
  const float *src_c = a.curr + (long long)shot * a.shot_stride + cz + (long long)(xa - 6) * P;
  const float *src_p = prevb + zo + (long long)(xa - 12) * P;
  const float *src_v = a.rcp + (long long)(shot / a.shots_per_vel) * a.vel_stride + zo + (long long)(xa - 12) * P;

  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < NC; i++) mbar_init(&S.full[i], 1);
    fence_mbar_init();
  }
  __syncwarp();

  // Lanes 0..5 each issue one copy of a stage: current A, B; previous A, B;
  // 1/vt A, B.  Lane 0 also arms the barrier with the stage's byte count.
  // Row B is copied only while it lies in the task (2s + 2 <= R).
  const int role = lane < 6 ? lane : 0;
  const bool is_c = role < 2, rowb = role & 1;
  const float *my_src = (is_c ? src_c : (role < 4 ? src_p : src_v)) + (rowb ? P : 0);
  const uint32_t my_ring = is_c ? smem_u32(&S.c[0][rowb][0])
                                : (role < 4 ? smem_u32(&S.p[0][rowb][0]) : smem_u32(&S.v[0][rowb][0]));
  const uint32_t my_slot_bytes = is_c ? 4u * 2 * WC : 4u * 2 * WP;
  const uint32_t my_bytes = is_c ? cbytes : pbytes;
  // stages are issued in order, so the lane's source row advances two rows
  // a call (a running pointer: no 64-bit multiply per stage)
  const float *run_src = my_src;
  auto issue = [&](int s, int cs, int ps) {
    if (lane < 6) {
      const bool pv = s >= 6;
      const bool b_ok = 2 * s + 2 <= R;
      if (lane == 0) mbar_expect_tx(&S.full[cs], (cbytes + (pv ? 2u * pbytes : 0u)) * (b_ok ? 2u : 1u));
      if ((is_c || pv) && (!rowb || b_ok))
        bulk_g2s_u32(my_ring + (uint32_t)(is_c ? cs : ps) * my_slot_bytes, run_src, my_bytes, smem_u32(&S.full[cs]));
      run_src += 2 * P;
    }
  };
  for (int s = 0; s < D2 && s < K2; s++) issue(s, s % NC, s % NP);

  // ---- this lane's depths
  const int zg = zo - 4 + 4 * lane;
  bool zok[4];
#pragma unroll
  for (int i = 0; i < 4; i++) zok[i] = zg + i >= 6 && zg + i < nz - 6;
  const bool outgroup = lane >= 1 && lane <= kOutLanes && zg < nz - 6 && zg + 3 >= 6;
  const bool fullgroup = zok[0] && zok[1] && zok[2] && zok[3];
  const int zw = 4 * lane;       // z window (depths zg-8 .. zg+11) in the current window
  const int qo = 4 * lane + 8;   // own depths in the current window
  const int po = 4 * min(max(lane - 1, 0), kOutLanes - 1);   // own depths in the previous / 1/vt window
  float *outp = (a.out ? a.out + (long long)shot * a.shot_stride : prevb) + (long long)xa * P + zg;   // output row xa, two rows a stage

  // sponge as in fd_step_rq: this lane's depth coefficients, the row's on
  // left/right ramp rows where no bottom ramp acts
  float2 coefz[2] = {make_float2(2.f, 2.f), make_float2(2.f, 2.f)};
  float2 pcz[2] = {make_float2(-1.f, -1.f), make_float2(-1.f, -1.f)};
  if constexpr (DAMPED) {
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int z = zg + i;
      const float d = (z >= 0 && z < nz) ? a.damp_z[z] : -1.f;
      const float2 c = fast_damp_coef(d >= 0.f ? d : 0.0f);
      float2 &cr = i < 2 ? coefz[0] : coefz[1];
      float2 &pr = i < 2 ? pcz[0] : pcz[1];
      if (i & 1) { cr.y = c.x; pr.y = c.y; }
      else { cr.x = c.x; pr.x = c.y; }
    }
  }
  const float2 *coef_row = a.coef_x + xa;   // coefficients of output row xa + j
  const int j_ramp_lo = a.ramp - xa;        // output rows j < j_ramp_lo, or >= j_ramp_lo + ramp_span: ramp rows
  const unsigned ramp_span = (unsigned)max(nx - 2 * a.ramp, 0);

  float4 q[12];   // own values of current rows xa-16+2k .. xa-5+2k after stage k's push
  float4 w0 = make_float4(0.f, 0.f, 0.f, 0.f), w1 = w0;   // u2 of the previous stage's two rows
  const float a5[6] = {-4.0f * SWFWI_A0, SWFWI_A1, SWFWI_A2, SWFWI_A3, SWFWI_A4, SWFWI_A5};

  // u2 of the row whose own values are q[ci], its z window at rowc
  auto u2_of = [&](const float *rowc, int ci) -> float4 {
    const float4 v0 = ld4(rowc), v1 = ld4(rowc + 4), v3 = ld4(rowc + 12), v4 = ld4(rowc + 16);
    const float4 v2 = q[ci];
    const float zn[20] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w, v2.x, v2.y,
                          v2.z, v2.w, v3.x, v3.y, v3.z, v3.w, v4.x, v4.y, v4.z, v4.w};
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
        const float2 xs = pr == 0 ? __fadd2_rn(lo2(q[ci - kk]), lo2(q[ci + kk]))
                                  : __fadd2_rn(hi2(q[ci - kk]), hi2(q[ci + kk]));
        acc[pr] = __ffma2_rn(make_float2(a5[kk], a5[kk]), __fadd2_rn(zs, xs), acc[pr]);
      }
    }
    return make_float4(acc[0].x, acc[0].y, acc[1].x, acc[1].y);
  };

  // the next field at output row xa + j (u2 rows um, uc, up around it)
  auto out_row = [&](const float4 c4, const float4 p4, const float4 r4, const float4 um, const float4 uc,
                     const float4 up, int j) {
    const float ucl = __shfl_up_sync(0xffffffffu, uc.w, 1);
    const float ucr = __shfl_down_sync(0xffffffffu, uc.x, 1);
    float2 cf0 = coefz[0], cf1 = coefz[1], pc0 = pcz[0], pc1 = pcz[1];
    if (__builtin_expect(DAMPED && (unsigned)(j - j_ramp_lo) >= ramp_span, 0)) {
      const float2 cx = coef_row[j];
      if (pc0.x == -1.f) { cf0.x = cx.x; pc0.x = cx.y; }
      if (pc0.y == -1.f) { cf0.y = cx.x; pc0.y = cx.y; }
      if (pc1.x == -1.f) { cf1.x = cx.x; pc1.x = cx.y; }
      if (pc1.y == -1.f) { cf1.y = cx.x; pc1.y = cx.y; }
    }
    const float2 o0 = update_pair_coef(lo2(c4), lo2(p4), lo2(r4), lo2(uc),
                                       make_float2(__fadd_rn(ucl, uc.y), __fadd_rn(uc.x, uc.z)), lo2(um), lo2(up),
                                       cf0, pc0);
    const float2 o1 = update_pair_coef(hi2(c4), hi2(p4), hi2(r4), hi2(uc),
                                       make_float2(__fadd_rn(uc.y, uc.w), __fadd_rn(uc.z, ucr)), hi2(um), hi2(up),
                                       cf1, pc1);
    return make_float4(o0.x, o0.y, o1.x, o1.y);
  };

  auto store = [&](float *dst, const float4 o) {
    if (outgroup) {
      if (fullgroup) {
        st4(dst, o);
      } else {
        if (zok[0]) dst[0] = o.x;
        if (zok[1]) dst[1] = o.y;
        if (zok[2]) dst[2] = o.z;
        if (zok[3]) dst[3] = o.w;
      }
    }
  };

  // Stage k (U = k % NC, a constant): k >= 5: u2 of rows xa-11+2k (own
  // values q[5], z window = row B of stage k-3) and xa-10+2k (q[6], row A
  // of stage k-2); k >= 6: output rows xa-12+2k and, while in the task,
  // xa-11+2k.
  auto step = [&](auto u, int k, uint32_t parity) -> bool {
    constexpr int U = decltype(u)::value;
    constexpr int SP = U % NP, S3 = (U - 3 + 2 * NC) % NC, S2 = (U - 2 + 2 * NC) % NC;
    // warp-uniform outcome: the shuffles and __syncwarp below need every lane
    if (!__all_sync(0xffffffffu, mbar_wait(&S.full[U], parity))) return false;
#pragma unroll
    for (int j = 0; j < 10; j++) q[j] = q[j + 2];
    q[10] = ld4(&S.c[U][0][qo]);
    q[11] = ld4(&S.c[U][1][qo]);   // not copied past the task's end: used only for rows past it
    if (k >= 5) {
      const float4 w2 = u2_of(&S.c[S3][1][zw], 5);
      const float4 w3 = u2_of(&S.c[S2][0][zw], 6);
      if (k >= 6) {
        const int j = 2 * k - 12;   // output row xa + j
        const float4 pA = ld4(&S.p[SP][0][po]), rA = ld4(&S.v[SP][0][po]);
        store(outp, out_row(q[4], pA, rA, w0, w1, w2, j));
        if (2 * k + 2 <= R) {
          const float4 pB = ld4(&S.p[SP][1][po]), rB = ld4(&S.v[SP][1][po]);
          store(outp + P, out_row(q[5], pB, rB, w1, w2, w3, j + 1));
        }
        outp += 2 * P;
      }
      w0 = w2;
      w1 = w3;
    }
    // every lane is done with the slots stage k+D2 refills (current: stage
    // k-4, last read as a z window at stage k-1; previous / 1/vt: stage k-1)
    __syncwarp();
    if (k + D2 < K2) issue(k + D2, (U + D2) % NC, (U + D2) % NP);
    return true;
  };

  bool ok = true;
  int k = 0;
#define SWFWI_RQ2_STEP(U)                                             \
  {                                                                   \
    k = k0 + (U);                                                     \
    if (k >= K2) break;                                               \
    if (!step(std::integral_constant<int, (U)>{}, k, parity)) {      \
      ok = false;                                                     \
      break;                                                          \
    }                                                                 \
  }
  for (int k0 = 0, it = 0;; k0 += NC, it++) {
    const uint32_t parity = (uint32_t)(it & 1);
    static_assert(NC == 6, "the loop below is unrolled by 6 stages");
    SWFWI_RQ2_STEP(0) SWFWI_RQ2_STEP(1) SWFWI_RQ2_STEP(2) SWFWI_RQ2_STEP(3) SWFWI_RQ2_STEP(4)
    SWFWI_RQ2_STEP(5)
  }
#undef SWFWI_RQ2_STEP
  if (!ok) {
    if (lane == 0) {
      atomicExch(a.err, 1);
      // wait (bounded) for the copies this warp already issued: stages k .. k+D2-1
      for (int i = k; i < K2 && i < k + D2; i++) mbar_wait(&S.full[i % NC], (uint32_t)((i / NC) & 1));
    }
    __syncwarp();
  }
}

}  // namespace swfwi
