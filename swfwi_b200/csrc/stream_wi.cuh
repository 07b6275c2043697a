// Streaming step with independent consumer warps for sm_100a (same scheme,
// arithmetics and layout as stream.cuh).
//
// CTA = NW consumer warps + 1 producer warp.  The producer's lane 0 streams
// rows into shared-memory rings with TMA bulk copies exactly as in
// stream_ws.cuh (16-row current-field ring, NP-row prev / velocity rings,
// full and empty mbarriers, bounded waits).  What differs is the consumer
// side: each consumer warp owns 128 depths of the band, of which lanes
// 1..30 output 120 (lanes 0 and 31 only supply u2 at the edge depths), so a
// warp needs no other warp's results.  A warp keeps the three u2 rows the
// time update reads in registers, gets its z neighbours with shuffles, and
// releases ring slots with one arrival per warp (empty barriers count NW
// arrivals).  There is no CTA-wide barrier in the time loop: warps are
// coupled only through the rings, at most a few rows apart.
#pragma once
#include <utility>
#include "stream.cuh"

namespace swfwi {

namespace wi_detail {
using namespace stream_detail;

constexpr int kWarpDepths = 120;   // output depths of one consumer warp

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

template <typename F, int... I>
__device__ __forceinline__ void static_for(F &&f, std::integer_sequence<int, I...>) {
  (f(std::integral_constant<int, I>{}), ...);
}

template <int NW, int NP>
struct Smem {
  static constexpr int BZ = kWarpDepths * NW, WC = BZ + 24, WP = BZ + 8, NC = 16;
  static constexpr size_t c_off = 0;
  static constexpr size_t p_off = c_off + sizeof(float) * NC * WC;
  static constexpr size_t v_off = p_off + sizeof(float) * NP * WP;
  static constexpr size_t b_off = v_off + sizeof(float) * NP * WP;
  static constexpr size_t bytes = b_off + sizeof(uint64_t) * (2 * NC + NP) + 16;
};

}  // namespace wi_detail

// D rows ahead: the prev/velocity ring has D + 1 slots (D = 3 or 7).
template <int NW, int D>
constexpr size_t wi_smem_bytes() {
  return wi_detail::Smem<NW, D + 1>::bytes;
}

template <int ARITH, bool DAMPED, int NW, int D>
__global__ void __launch_bounds__((NW + 1) * 32)
fd_step_wi(StreamArgs a) {
  using namespace wi_detail;
  constexpr int NP = D + 1;
  static_assert(NP == 4 || NP == 8, "the prev/vel ring must divide the current ring");
  using L = Smem<NW, NP>;
  constexpr int BZ = L::BZ, WC = L::WC, WP = L::WP, NC = L::NC;
  extern __shared__ __align__(128) unsigned char smem[];
  float(*cring)[WC] = reinterpret_cast<float(*)[WC]>(smem + L::c_off);
  float(*pring)[WP] = reinterpret_cast<float(*)[WP]>(smem + L::p_off);
  float(*vring)[WP] = reinterpret_cast<float(*)[WP]>(smem + L::v_off);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + L::b_off);
  uint64_t *emptyc = full + NC;
  uint64_t *emptyp = emptyc + NC;
  int *s_fail = reinterpret_cast<int *>(emptyp + NP);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int shot = a.shot_major ? blockIdx.z : blockIdx.x;
  const int band = a.shot_major ? blockIdx.x : blockIdx.y;
  const int chunk = a.shot_major ? blockIdx.y : blockIdx.z;
  const int nx = a.nx, nz = a.nz, P = a.pitch;
  const int z0 = 4 + band * BZ;
  const int xa = 6 + chunk * a.xchunk;
  const int xb = min(xa + a.xchunk, nx - 6);
  if (xa >= xb) return;
  const int K = xb - xa + 12;

  if (tid == 0) {
    for (int i = 0; i < NC; i++) {
      mbar_init(&full[i], 1);
      mbar_init(&emptyc[i], NW);
    }
    for (int i = 0; i < NP; i++) mbar_init(&emptyp[i], NW);
    fence_mbar_init();
    *s_fail = 0;
  }
  __syncthreads();

  // ---------------------------------------------------------------- producer
  if (warp == NW) {
    if (lane != 0) return;
    const int cz = z0 - 12, pz = z0 - 4;
    const int clen = min(WC, P - kStreamCoff - cz), plen = min(WP, P - kStreamCoff - pz);
    const uint32_t cbytes = (uint32_t)clen * 4u, pbytes = (uint32_t)plen * 4u;
    const float *curr = a.curr + (long long)shot * a.shot_stride + cz;
    const float *prevw = a.prev + (long long)shot * a.shot_stride + pz;
    const float *rcpw = a.rcp + (long long)(shot / a.shots_per_vel) * a.vel_stride + pz;
    for (int k = 0; k < K; k++) {
      if (*(volatile int *)s_fail) break;
      if (k >= NC && !mbar_wait(&emptyc[k & (NC - 1)], (uint32_t)(((k >> 4) + 1) & 1))) {
        atomicExch(a.err, 1);
        *(volatile int *)s_fail = 1;
        break;
      }
      const bool pv = k >= 12;
      const int ps = (k - 12) & (NP - 1);
      if (pv && k - 12 >= NP &&
          !mbar_wait(&emptyp[ps], (uint32_t)((((k - 12) / NP) + 1) & 1))) {
        atomicExch(a.err, 1);
        *(volatile int *)s_fail = 1;
        break;
      }
      uint64_t *fb = &full[k & (NC - 1)];
      mbar_expect_tx(fb, cbytes + (pv ? 2u * pbytes : 0u));
      bulk_g2s(&cring[k & (NC - 1)][0], curr + (long long)(xa - 6 + k) * P, cbytes, fb);
      if (pv) {
        long long off = (long long)(xa - 12 + k) * P;
        bulk_g2s(&pring[ps][0], prevw + off, pbytes, fb);
        bulk_g2s(&vring[ps][0], rcpw + off, pbytes, fb);
      }
    }
    return;
  }

  // ---------------------------------------------------------------- consumers
  const int off = warp * kWarpDepths + 4 * lane;   // this lane's group in the rings
  const int zg = z0 - 4 + off;                      // its first depth
  float *prevg = a.prev + (long long)shot * a.shot_stride + (long long)xa * P + zg;   // row xa
  float dz[4] = {-1.f, -1.f, -1.f, -1.f};
  bool zok[4];
  bool coldamp = false;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    int z = zg + i;
    zok[i] = z >= 6 && z < nz - 6;
    if constexpr (DAMPED) {
      dz[i] = (z >= 0 && z < nz) ? a.damp_z[z] : -1.f;
      coldamp = coldamp || dz[i] >= 0.f;
    }
  }
  const bool outlane = lane >= 1 && lane <= 30 && zg < nz - 6 && zg + 3 >= 6;
  const bool fullgroup = zok[0] && zok[1] && zok[2] && zok[3];
  const float *damp_row = a.damp_x + xa - 12;   // damp_x of output row xa-12+k
  // steps whose output row lies between the x ramps, where damp_x is 0
  const int k_ramp_lo = a.ramp - xa + 12, k_ramp_hi = nx - a.ramp - xa + 12;
  // u2 of rows xa-13+k and xa-12+k at step k (the row made at step k is up)
  float4 um = make_float4(0.f, 0.f, 0.f, 0.f), uc = um;

  // One step.  PH is k & 15 when known at compile time, else -1.
  auto step = [&](auto ph, int k) -> bool {
    constexpr int PH = decltype(ph)::value;
    auto cs = [&](int o) -> int {
      if constexpr (PH >= 0) return (PH + o) & (NC - 1);
      else return (k + o) & (NC - 1);
    };
    // the warp agrees on the wait's outcome, so its lanes never split
    const bool got = __all_sync(0xffffffffu, mbar_wait(&full[cs(0)], (uint32_t)((k >> 4) & 1)));
    if (!got) {
      if (lane == 0) {
        atomicExch(a.err, 1);
        *(volatile int *)s_fail = 1;
      }
      return false;
    }
    const bool has_u2 = PH >= 0 || k >= 10;
    const bool has_out = PH >= 0 || k >= 12;
    float4 up = make_float4(0.f, 0.f, 0.f, 0.f);
    if (has_u2) {
      // u2 of row xa - 11 + k from stages k-10 .. k
      const float *rowc = &cring[cs(-5)][off];
      float zn[20];
      {
        float4 v0 = ld4(rowc), v1 = ld4(rowc + 4), v2 = ld4(rowc + 8), v3 = ld4(rowc + 12),
               v4 = ld4(rowc + 16);
        zn[0] = v0.x; zn[1] = v0.y; zn[2] = v0.z; zn[3] = v0.w;
        zn[4] = v1.x; zn[5] = v1.y; zn[6] = v1.z; zn[7] = v1.w;
        zn[8] = v2.x; zn[9] = v2.y; zn[10] = v2.z; zn[11] = v2.w;
        zn[12] = v3.x; zn[13] = v3.y; zn[14] = v3.z; zn[15] = v3.w;
        zn[16] = v4.x; zn[17] = v4.y; zn[18] = v4.z; zn[19] = v4.w;
      }
      float4 xm4[6], xp4[6];
#pragma unroll
      for (int d = 1; d <= 5; d++) {
        xm4[d] = ld4(&cring[cs(-5 - d)][off + 8]);
        xp4[d] = ld4(&cring[cs(-5 + d)][off + 8]);
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
      up = make_float4(u[0], u[1], u[2], u[3]);
    }
    float4 o4 = make_float4(0.f, 0.f, 0.f, 0.f);
    int ps = 0;
    if (has_out) {
      ps = (PH >= 0) ? ((PH - 12) & (NP - 1)) : ((k - 12) & (NP - 1));
      const float ucl = __shfl_up_sync(0xffffffffu, uc.w, 1);
      const float ucr = __shfl_down_sync(0xffffffffu, uc.x, 1);
      const float4 c4 = ld4(&cring[cs(-6)][off + 8]);
      const float4 p4 = ld4(&pring[ps][off]);
      const float4 r4 = ld4(&vring[ps][off]);
      float o[4];
      bool damp = false;
      float dxr = 0.f;
      if constexpr (DAMPED) {
        dxr = (k < k_ramp_lo || k >= k_ramp_hi) ? damp_row[k] : 0.f;
        damp = coldamp || dxr != 0.f;
      }
      if (!damp) {
#pragma unroll
        for (int i = 0; i < 4; i++) {
          float uzm = i == 0 ? ucl : get(uc, i - 1);
          float uzp = i == 3 ? ucr : get(uc, i + 1);
          o[i] = update_pt<ARITH>(get(c4, i), get(p4, i), get(r4, i), get(uc, i), uzm, uzp,
                                  get(um, i), get(up, i), 0.0f);
        }
      } else {
#pragma unroll
        for (int i = 0; i < 4; i++) {
          float dist = dz[i] >= 0.f ? dz[i] : dxr;
          float delta = __fmul_rn(__fmul_rn(0.05f, dist), dist);
          float uzm = i == 0 ? ucl : get(uc, i - 1);
          float uzp = i == 3 ? ucr : get(uc, i + 1);
          o[i] = update_pt<ARITH>(get(c4, i), get(p4, i), get(r4, i), get(uc, i), uzm, uzp,
                                  get(um, i), get(up, i), delta);
        }
      }
      o4 = make_float4(o[0], o[1], o[2], o[3]);
    }
    // every lane's reads of this step are done: release stage k-10's current
    // row and stage k's prev/velocity rows
    __syncwarp();
    if (lane == 0) {
      if (has_u2) mbar_arrive(&emptyc[cs(-10)]);
      if (has_out) mbar_arrive(&emptyp[ps]);
    }
    if (has_out && outlane) {
      float *dst = prevg + (long long)(k - 12) * P;
      if (fullgroup) {
        st4(dst, o4);
      } else {
        if (zok[0]) dst[0] = o4.x;
        if (zok[1]) dst[1] = o4.y;
        if (zok[2]) dst[2] = o4.z;
        if (zok[3]) dst[3] = o4.w;
      }
    }
    um = uc;
    uc = up;
    return true;
  };

  int k = 0;
  bool ok = true;
  // warm-up: stages 0..11 (u2 from stage 10 on, no output yet)
  for (; ok && k < 12 && k < K; k++) ok = step(std::integral_constant<int, -1>{}, k);
  // main loop: from step 12 in blocks of 16, every ring index is a constant
  for (; ok && k + 16 <= K; k += 16) {
    static_for(
        [&](auto u) {
          constexpr int U = decltype(u)::value;
          if (ok) ok = step(std::integral_constant<int, (12 + U) & 15>{}, k + U);
        },
        std::make_integer_sequence<int, 16>{});
  }
  for (; ok && k < K; k++) ok = step(std::integral_constant<int, -1>{}, k);

  if (!ok && lane == 0) {
    // keep the CTA (and its shared memory) alive until copies the producer
    // already issued have landed (bounded)
    for (int i = k; i < K && i < k + NC; i++) mbar_wait(&full[i & (NC - 1)], (uint32_t)((i >> 4) & 1));
  }
}

}  // namespace swfwi
