// Warp-specialised streaming step with two output rows per consumer step
// (same scheme, arithmetics, producer and rings as stream_ws.cuh).
//
// A consumer step takes stages k and k+1: it reads the 12 staged current
// rows k-10 .. k+1 once for both u2 rows (u2 of rows xa-11+k and xa-10+k),
// stores both in an 8-row u2 ring, synchronises the consumers once, and
// writes output rows xa-12+k and xa-11+k.  Against one row per step this
// halves the barrier, wait and release work per row, shares the x-neighbour
// loads of the two u2 rows and gives each warp two independent rows of
// arithmetic.  Releases run on counters (every current row no u2 needs any
// more, every prev/vel row whose output is stored), so pair steps and a
// single tail step mix freely.  Every wait is bounded.
#pragma once
#include <utility>
#include "stream.cuh"
#include "stream_ws.cuh"

namespace swfwi {

namespace ws2_detail {
// stream_ws.cuh's layout with an 8-row u2 ring: a pair step writes rows
// k, k+1 while slower threads may still read rows k-4 .. k-1.
template <int NT, int NP>
struct Smem2 {
  static constexpr int BZ = 4 * NT - 8, WC = BZ + 24, WP = BZ + 8, NC = 16, NU = 8;
  static constexpr size_t c_off = 0;
  static constexpr size_t p_off = c_off + sizeof(float) * NC * WC;
  static constexpr size_t v_off = p_off + sizeof(float) * NP * WP;
  static constexpr size_t u_off = v_off + sizeof(float) * NP * WP;
  static constexpr size_t b_off = u_off + sizeof(float) * NU * 4 * NT;
  static constexpr size_t bytes = b_off + sizeof(uint64_t) * (2 * NC + NP) + 16;
};
}  // namespace ws2_detail

template <int NW, int D>
constexpr size_t ws2_smem_bytes() {
  return ws2_detail::Smem2<NW * 32, D + 1>::bytes;
}

template <int ARITH, bool DAMPED, int NW, int D>
__global__ void __launch_bounds__((NW + 1) * 32)
fd_step_ws2(StreamArgs a) {
  using namespace ws_detail;
  constexpr int NT = NW * 32;      // consumer threads
  constexpr int NP = D + 1;
  static_assert(NP == 4 || NP == 8, "the prev/vel ring must divide the current ring");
  using L = ws2_detail::Smem2<NT, NP>;
  constexpr int NU = L::NU;
  constexpr int BZ = L::BZ, WC = L::WC, WP = L::WP, NC = L::NC;
  extern __shared__ __align__(128) unsigned char smem[];
  float(*cring)[WC] = reinterpret_cast<float(*)[WC]>(smem + L::c_off);
  float(*pring)[WP] = reinterpret_cast<float(*)[WP]>(smem + L::p_off);
  float(*vring)[WP] = reinterpret_cast<float(*)[WP]>(smem + L::v_off);
  float(*u2r)[4 * NT] = reinterpret_cast<float(*)[4 * NT]>(smem + L::u_off);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + L::b_off);
  uint64_t *emptyc = full + NC;
  uint64_t *emptyp = emptyc + NC;
  int *s_fail = reinterpret_cast<int *>(emptyp + NP);

  const int tid = threadIdx.x;
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
      mbar_init(&emptyc[i], 1);
    }
    for (int i = 0; i < NP; i++) mbar_init(&emptyp[i], 1);
    fence_mbar_init();
    *s_fail = 0;
  }
  __syncthreads();

  // ---------------------------------------------------------------- producer
  if (tid >= NT) {
    if (tid != NT) return;
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
  const int t = tid;
  const int zg = z0 - 4 + 4 * t;
  float *prevg = a.prev + (long long)shot * a.shot_stride + (long long)xa * P + zg;   // output row xa
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
  const bool outgroup = t >= 1 && t < NT - 1 && zg < nz - 6 && zg + 3 >= 6;
  const bool fullgroup = zok[0] && zok[1] && zok[2] && zok[3];
  const float *damp_row = a.damp_x + xa - 12;   // damp_x of output row xa-12+k
  const int k_ramp_lo = a.ramp - xa + 12, k_ramp_hi = nx - a.ramp - xa + 12;
  int rel_c = 0, rel_p = 12;   // next current / prev-vel stage to release

  // u2 at the lane's 4 depths from the staged centre row (zn, 20 values from
  // depth zg-8) and the x neighbours xm/xp (d = 1..5 rows before/after)
  auto lap4 = [&](const float (&zn)[20], const float4 (&xm4)[6], const float4 (&xp4)[6]) -> float4 {
    if constexpr (ARITH == ARITH_FAST) {
      const float2 u01 = lap_pair_fast<0>(zn, xm4, xp4), u23 = lap_pair_fast<1>(zn, xm4, xp4);
      return make_float4(u01.x, u01.y, u23.x, u23.y);
    } else {
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
      return make_float4(u[0], u[1], u[2], u[3]);
    }
  };
  auto load_zn = [&](const float *row, float (&zn)[20]) {
    const float4 v0 = ld4(row + 4 * t), v1 = ld4(row + 4 * t + 4), v2 = ld4(row + 4 * t + 8),
                 v3 = ld4(row + 4 * t + 12), v4 = ld4(row + 4 * t + 16);
    zn[0] = v0.x; zn[1] = v0.y; zn[2] = v0.z; zn[3] = v0.w;
    zn[4] = v1.x; zn[5] = v1.y; zn[6] = v1.z; zn[7] = v1.w;
    zn[8] = v2.x; zn[9] = v2.y; zn[10] = v2.z; zn[11] = v2.w;
    zn[12] = v3.x; zn[13] = v3.y; zn[14] = v3.z; zn[15] = v3.w;
    zn[16] = v4.x; zn[17] = v4.y; zn[18] = v4.z; zn[19] = v4.w;
  };
  // output row xa-12+k from its centre value c4, pv ring slot ps and u2 rows
  // um (row above), uc (own, with its z neighbours ucl / ucr), up (below)
  auto out_row = [&](int k, float4 c4, int ps, float4 um4, float4 uc4, float ucl, float ucr, float4 up4) {
    const float4 p4 = ld4(&pring[ps][4 * t]);
    const float4 r4 = ld4(&vring[ps][4 * t]);
    float o[4];
    bool damp = false;
    float dxr = 0.f;
    if constexpr (DAMPED) {
      dxr = (k < k_ramp_lo || k >= k_ramp_hi) ? damp_row[k] : 0.f;
      damp = coldamp || dxr != 0.f;
    }
    if (!damp) {
      if constexpr (ARITH == ARITH_FAST) {
        const float2 lo = update_pair_fast(lo2(c4), lo2(p4), lo2(r4), lo2(uc4), f2(ucl, uc4.x), f2(uc4.y, uc4.z),
                                           lo2(um4), lo2(up4));
        const float2 hi = update_pair_fast(hi2(c4), hi2(p4), hi2(r4), hi2(uc4), f2(uc4.y, uc4.z), f2(uc4.w, ucr),
                                           hi2(um4), hi2(up4));
        o[0] = lo.x; o[1] = lo.y; o[2] = hi.x; o[3] = hi.y;
      } else {
#pragma unroll
        for (int i = 0; i < 4; i++) {
          const float uzm = i == 0 ? ucl : get(uc4, i - 1);
          const float uzp = i == 3 ? ucr : get(uc4, i + 1);
          o[i] = update_pt<ARITH>(get(c4, i), get(p4, i), get(r4, i), get(uc4, i), uzm, uzp, get(um4, i),
                                  get(up4, i), 0.0f);
        }
      }
    } else {
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const float dist = dz[i] >= 0.f ? dz[i] : dxr;
        const float delta = __fmul_rn(__fmul_rn(0.05f, dist), dist);
        const float uzm = i == 0 ? ucl : get(uc4, i - 1);
        const float uzp = i == 3 ? ucr : get(uc4, i + 1);
        o[i] = update_pt<ARITH>(get(c4, i), get(p4, i), get(r4, i), get(uc4, i), uzm, uzp, get(um4, i),
                                get(up4, i), delta);
      }
    }
    float *dst = prevg + (long long)(k - 12) * P;
    if (fullgroup) {
      st4(dst, make_float4(o[0], o[1], o[2], o[3]));
    } else {
#pragma unroll
      for (int i = 0; i < 4; i++)
        if (zok[i]) dst[i] = o[i];
    }
  };
  // releases after the consumers' barrier of a step whose u2 read stages up
  // to k1 and whose outputs start at stage k0
  auto release = [&](int k0, int k1) {
    if (t == 0) {
      for (; rel_c <= k1 - 10; rel_c++) mbar_arrive(&emptyc[rel_c & (NC - 1)]);
      for (; rel_p < k0; rel_p++) mbar_arrive(&emptyp[(rel_p - 12) & (NP - 1)]);
    }
  };
  auto fail = [&]() {
    atomicExch(a.err, 1);
    *(volatile int *)s_fail = 1;
    return false;
  };

  // Two stages k, k+1 (k even).  PH is k & 15 when known at compile time, else -1.
  auto pair = [&](auto ph, int k) -> bool {
    constexpr int PH = decltype(ph)::value;
    auto cs = [&](int o) -> int {
      if constexpr (PH >= 0) return (PH + o) & (NC - 1);
      else return (k + o) & (NC - 1);
    };
    auto us = [&](int o) -> int {
      if constexpr (PH >= 0) return (PH + o) & (NU - 1);
      else return (k + o) & (NU - 1);
    };
    if (!mbar_wait(&full[cs(0)], (uint32_t)((k >> 4) & 1))) return fail();
    if (!mbar_wait(&full[cs(1)], (uint32_t)(((k + 1) >> 4) & 1))) return fail();
    const bool has_u2 = PH >= 0 || k >= 10;
    const bool has_out = PH >= 0 || k >= 12;
    float4 ca = make_float4(0.f, 0.f, 0.f, 0.f), cb = ca;   // centres of stages k-6, k-5
    if (has_u2) {
      // rows k-10 .. k+1 at the lane's depths: xr[d + 10]
      float za[20], zb[20];
      load_zn(&cring[cs(-5)][0], za);
      load_zn(&cring[cs(-4)][0], zb);
      float4 xr[12];
#pragma unroll
      for (int d = -10; d <= 1; d++) {
        if (d == -5) xr[d + 10] = make_float4(za[8], za[9], za[10], za[11]);
        else if (d == -4) xr[d + 10] = make_float4(zb[8], zb[9], zb[10], zb[11]);
        else xr[d + 10] = ld4(&cring[cs(d)][8 + 4 * t]);
      }
      float4 xm4[6], xp4[6];
#pragma unroll
      for (int d = 1; d <= 5; d++) {
        xm4[d] = xr[-5 - d + 10];
        xp4[d] = xr[-5 + d + 10];
      }
      st4(&u2r[us(0)][4 * t], lap4(za, xm4, xp4));
#pragma unroll
      for (int d = 1; d <= 5; d++) {
        xm4[d] = xr[-4 - d + 10];
        xp4[d] = xr[-4 + d + 10];
      }
      st4(&u2r[us(1)][4 * t], lap4(zb, xm4, xp4));
      ca = xr[4];
      cb = xr[5];
    }
    consumer_sync<NT>();
    if (*(volatile int *)s_fail) return false;
    release(k, has_u2 ? k + 1 : 9);
    if (has_out && outgroup) {
      const float *u0 = &u2r[us(-2)][4 * t], *u1 = &u2r[us(-1)][4 * t];
      const float *u2 = &u2r[us(0)][4 * t], *u3 = &u2r[us(1)][4 * t];
      const float4 a0 = ld4(u0), a1 = ld4(u1), a2 = ld4(u2), a3 = ld4(u3);
      const float l1 = u1[-1], r1 = u1[4], l2 = u2[-1], r2 = u2[4];
      const int ps0 = (PH >= 0) ? ((PH - 12) & (NP - 1)) : ((k - 12) & (NP - 1));
      const int ps1 = (PH >= 0) ? ((PH - 11) & (NP - 1)) : ((k - 11) & (NP - 1));
      out_row(k, ca, ps0, a0, a1, l1, r1, a2);
      out_row(k + 1, cb, ps1, a1, a2, l2, r2, a3);
    }
    return true;
  };

  // One stage k (the odd tail of a chunk).
  auto single = [&](int k) -> bool {
    auto cs = [&](int o) -> int { return (k + o) & (NC - 1); };
    auto us = [&](int o) -> int { return (k + o) & (NU - 1); };
    if (!mbar_wait(&full[cs(0)], (uint32_t)((k >> 4) & 1))) return fail();
    float4 c = make_float4(0.f, 0.f, 0.f, 0.f);
    {
      float zn[20];
      load_zn(&cring[cs(-5)][0], zn);
      float4 xm4[6], xp4[6];
#pragma unroll
      for (int d = 1; d <= 5; d++) {
        xm4[d] = ld4(&cring[cs(-5 - d)][8 + 4 * t]);
        xp4[d] = ld4(&cring[cs(-5 + d)][8 + 4 * t]);
      }
      st4(&u2r[us(0)][4 * t], lap4(zn, xm4, xp4));
      c = xm4[1];   // stage k-6's centre
    }
    consumer_sync<NT>();
    if (*(volatile int *)s_fail) return false;
    release(k, k);
    if (outgroup) {
      const float *u0 = &u2r[us(-2)][4 * t], *u1 = &u2r[us(-1)][4 * t], *u2 = &u2r[us(0)][4 * t];
      out_row(k, c, (k - 12) & (NP - 1), ld4(u0), ld4(u1), u1[-1], u1[4], ld4(u2));
    }
    return true;
  };

  int k = 0;
  bool ok = true;
  // warm-up: stages 0..11 in pairs (u2 from stage 10 on, no output yet)
  for (; ok && k < 12; k += 2) ok = pair(std::integral_constant<int, -1>{}, k);
  // main loop: pairs from stage 12 in blocks of 16 stages, ring indices constant
  for (; ok && k + 16 <= K; k += 16) {
    static_for(
        [&](auto u) {
          constexpr int U = decltype(u)::value;
          if (ok) ok = pair(std::integral_constant<int, (12 + 2 * U) & 15>{}, k + 2 * U);
        },
        std::make_integer_sequence<int, 8>{});
  }
  for (; ok && k + 2 <= K; k += 2) ok = pair(std::integral_constant<int, -1>{}, k);
  if (ok && k < K) {
    ok = single(k);
    k++;
  }

  if (!ok && t == 0) {
    // wait (bounded) for copies the producer already issued
    for (int i = k; i < K && i < k + NC; i++) mbar_wait(&full[i & (NC - 1)], (uint32_t)((i >> 4) & 1));
  }
}

}  // namespace swfwi
