// Warp-specialised streaming step for sm_100a (same scheme, arithmetics and
// layout as stream.cuh).
//
// CTA = NW consumer warps + 1 producer warp.  The producer's lane 0 walks
// the chunk's rows and issues TMA bulk copies into the rings, throttled by
// "empty" mbarriers the consumers release; the consumers wait on "full"
// mbarriers and never touch the copy engine:
//   current-field ring: 16 rows; stage k (row xa-6+k) lands in slot k & 15,
//     is read by u2 at steps k..k+10 and released after step k+10;
//   prev / velocity ring: NP rows (a power of two); stage k >= 12 (row
//     xa-12+k) lands in slot (k-12) & (NP-1), is read by the output at step
//     k and released after step k+1.
// The consumers of one CTA share every staged row: with 3 consumer warps a
// band is 376 deep.  Warm-up rows (no output yet) are peeled off; the main
// loop is unrolled by the ring length from a fixed phase (step 12), so every
// ring slot, barrier and u2-row index is a compile-time constant; rows and
// depths outside the sponge take an undamped fast path.  Every wait is
// bounded; on timeout the CTA raises the error flag and the producer stops.
//
// Fused variants for the backward time loop keep the added work small,
// because the unrolled loop's code must stay in the instruction cache: the
// source back-step also subtracts the source and images (EPI 2), the
// receiver step also injects the next residual (EPI 3); a source or
// receiver line must be horizontal (or one point), so one lane per row adds.
#pragma once
#include <utility>
#include "stream.cuh"

namespace swfwi {

namespace ws_detail {
using namespace stream_detail;

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

template <int NT>
__device__ __forceinline__ void consumer_sync() {
  if constexpr (NT == 32) __syncwarp();
  else asm volatile("bar.sync 1, %0;" ::"r"(NT) : "memory");
}

template <typename F, int... I>
__device__ __forceinline__ void static_for(F &&f, std::integer_sequence<int, I...>) {
  (f(std::integral_constant<int, I>{}), ...);
}

template <int NT, int NP>
struct Smem {
  static constexpr int BZ = 4 * NT - 8, WC = BZ + 24, WP = BZ + 8, NC = 16;
  static constexpr size_t c_off = 0;
  static constexpr size_t p_off = c_off + sizeof(float) * NC * WC;
  static constexpr size_t v_off = p_off + sizeof(float) * NP * WP;
  static constexpr size_t u_off = v_off + sizeof(float) * NP * WP;
  static constexpr size_t b_off = u_off + sizeof(float) * 4 * 4 * NT;
  static constexpr size_t bytes = b_off + sizeof(uint64_t) * (2 * NC + NP) + 16;
};

}  // namespace ws_detail

// D rows ahead: the prev/velocity ring has D + 1 slots (D = 3 or 7).
template <int NW, int D, int EPI = 0>
constexpr size_t ws_smem_bytes() {
  return ws_detail::Smem<NW * 32, D + 1>::bytes;
}

// EPI: also run part of a.epi at the output points with the new values
// before they are stored: 2 = source subtraction and imaging (source
// back-step); 3 = next injection (receiver step).
template <int ARITH, bool DAMPED, int NW, int D, int EPI = 0>
__global__ void __launch_bounds__((NW + 1) * 32, (EPI == 2 || EPI == 3) ? (ARITH == ARITH_REF ? 4 : 5) : 1)
fd_step_ws(StreamArgs a) {
  using namespace ws_detail;
  constexpr int NT = NW * 32;      // consumer threads
  constexpr int NP = D + 1;
  static_assert(NP == 4 || NP == 8, "the prev/vel ring must divide the current ring");
  using L = Smem<NT, NP>;
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
      if (pv && k - 12 >= NP && !mbar_wait(&emptyp[ps], (uint32_t)((((k - 12) / NP) + 1) & 1))) {
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
  float *prevg = (a.out ? a.out : a.prev) + (long long)shot * a.shot_stride + (long long)xa * P + zg;   // output row xa
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
  // FAST sponge coefficients of this thread's depths in the bottom ramp
  float cfz[4] = {2.f, 2.f, 2.f, 2.f}, pcz[4] = {-1.f, -1.f, -1.f, -1.f};
  if constexpr (DAMPED && ARITH == ARITH_FAST) {
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const float2 c = fast_damp_coef(dz[i] >= 0.f ? dz[i] : 0.0f);
      cfz[i] = c.x;
      pcz[i] = c.y;
    }
  }
  const bool outgroup = t >= 1 && t < NT - 1 && zg < nz - 6 && zg + 3 >= 6;
  const bool fullgroup = zok[0] && zok[1] && zok[2] && zok[3];
  const float *damp_row = a.damp_x + xa - 12;   // damp_x of output row xa-12+k
  // steps whose output row lies between the x ramps, where damp_x is 0
  const int k_ramp_lo = a.ramp - xa + 12, k_ramp_hi = nx - a.ramp - xa + 12;
  // fused source work (EPI 3: add; EPI 2: subtract) on a horizontal line or
  // a single point: the lane holding the line's depth, its depth index and
  // the next point's row and index (rows increase by one per step)
  int hit_d = -1, hit_x = -1, hit_i = 0, hit_di = 0, hit_dx = 0, hit_left = 0;
  const float *hit_vals = nullptr;
  int hit_stride = 0;
  if constexpr (EPI == 2 || EPI == 3) {
    const float *vals = EPI == 2 ? a.epi.sub : a.epi.inj;
    if (vals && outgroup) {
      const PtLine l = a.epi.src[shot];
      const int d = l.z0 - zg;
      if (l.n > 0 && (l.jz == 0 || l.n == 1) && d >= 0 && d < 4 && zok[d]) {
        LineCursor c;
        c.init(l, xa);
        hit_d = d;
        hit_x = c.next_x;
        hit_i = c.next_i;
        hit_di = c.step_i;
        hit_dx = c.dx;
        hit_left = c.left;
        hit_vals = vals + (long long)shot * (EPI == 2 ? a.epi.sub_slot_stride : a.epi.inj_slot_stride);
        hit_stride = EPI == 2 ? a.epi.sub_stride : a.epi.inj_stride;
      }
    }
  }

  bool next_ready = false;   // stage k+1 seen complete during step k
  // One step.  PH is k & 15 when known at compile time, else -1.
  auto step = [&](auto ph, int k) -> bool {
    constexpr int PH = decltype(ph)::value;
    auto cs = [&](int off) -> int {
      if constexpr (PH >= 0) return (PH + off) & (NC - 1);
      else return (k + off) & (NC - 1);
    };
    auto us = [&](int off) -> int {
      if constexpr (PH >= 0) return (PH + off) & 3;
      else return (k + off) & 3;
    };
    const int fs = cs(0);
    // the previous step tested this stage already; wait only if it was not in
    if (!next_ready && !mbar_wait(&full[fs], (uint32_t)((k >> 4) & 1))) {
      atomicExch(a.err, 1);
      *(volatile int *)s_fail = 1;
      return false;
    }
    const bool has_u2 = PH >= 0 || k >= 10;
    const bool has_out = PH >= 0 || k >= 12;
    // fused imaging: this step's receiver field and image values, loaded
    // early so their latency overlaps the update
    float4 gimg = make_float4(0.f, 0.f, 0.f, 0.f), vimg = gimg;
    if constexpr (EPI == 2 || EPI == 3) {
      if (EPI == 2 && a.epi.image && has_out && outgroup) {
        const long long o = (long long)shot * a.shot_stride + (long long)(xa - 12 + k) * P + zg;
        if (fullgroup) {
          gimg = ld4g(a.epi.gcurr + o);
          vimg = ld4g(a.epi.image + o);
        } else {
          if (zok[0]) { gimg.x = a.epi.gcurr[o]; vimg.x = a.epi.image[o]; }
          if (zok[1]) { gimg.y = a.epi.gcurr[o + 1]; vimg.y = a.epi.image[o + 1]; }
          if (zok[2]) { gimg.z = a.epi.gcurr[o + 2]; vimg.z = a.epi.image[o + 2]; }
          if (zok[3]) { gimg.w = a.epi.gcurr[o + 3]; vimg.w = a.epi.image[o + 3]; }
        }
      }
    }
    if (has_u2) {
      // u2 of row r = xa - 11 + k from stages k-10 .. k
      const float *rowc = &cring[cs(-5)][0];
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
        xm4[d] = ld4(&cring[cs(-5 - d)][8 + 4 * t]);
        xp4[d] = ld4(&cring[cs(-5 + d)][8 + 4 * t]);
      }
      if constexpr (ARITH == ARITH_FAST) {
        const float2 u01 = lap_pair_fast<0>(zn, xm4, xp4), u23 = lap_pair_fast<1>(zn, xm4, xp4);
        st4(&u2r[us(0)][4 * t], make_float4(u01.x, u01.y, u23.x, u23.y));
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
        st4(&u2r[us(0)][4 * t], make_float4(u[0], u[1], u[2], u[3]));
      }
    }
    // test the next stage now, so the answer is in by the next step
    next_ready = k + 1 < K && mbar_test(&full[cs(1)], (uint32_t)(((k + 1) >> 4) & 1));
    consumer_sync<NT>();
    if (*(volatile int *)s_fail) return false;
    // release stage k-10's current row and stage k-1's prev/vel rows
    if (t == 0) {
      if (has_u2) mbar_arrive(&emptyc[cs(-10)]);
      // (stage 11 carries no prev/vel rows: the first release is at step 13)
      if (k >= 13) {
        if constexpr (PH >= 0) mbar_arrive(&emptyp[(PH - 13) & (NP - 1)]);
        else mbar_arrive(&emptyp[(k - 13) & (NP - 1)]);
      }
    }
    if (has_out && outgroup) {
      const int ps = (PH >= 0) ? ((PH - 12) & (NP - 1)) : ((k - 12) & (NP - 1));
      const float *um = &u2r[us(-2)][4 * t];
      const float *uc = &u2r[us(-1)][4 * t];
      const float *up = &u2r[us(0)][4 * t];
      float4 c4 = ld4(&cring[cs(-6)][8 + 4 * t]);
      const float4 p4 = ld4(&pring[ps][4 * t]);
      const float4 r4 = ld4(&vring[ps][4 * t]);
      float4 um4 = ld4(um), uc4 = ld4(uc), up4 = ld4(up);
      float ucl = uc[-1], ucr = uc[4];
      float o[4];
      bool damp = false;
      float dxr = 0.f;
      if constexpr (DAMPED) {
        dxr = (k < k_ramp_lo || k >= k_ramp_hi) ? damp_row[k] : 0.f;
        damp = coldamp || dxr != 0.f;
      }
      if (!damp) {
        if constexpr (ARITH == ARITH_FAST) {
          const float2 a = update_pair_fast(lo2(c4), lo2(p4), lo2(r4), lo2(uc4), f2(ucl, uc4.x), f2(uc4.y, uc4.z),
                                            lo2(um4), lo2(up4));
          const float2 b = update_pair_fast(hi2(c4), hi2(p4), hi2(r4), hi2(uc4), f2(uc4.y, uc4.z),
                                            f2(uc4.w, ucr), hi2(um4), hi2(up4));
          o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
        } else {
#pragma unroll
          for (int i = 0; i < 4; i++) {
            float uzm = i == 0 ? ucl : get(uc4, i - 1);
            float uzp = i == 3 ? ucr : get(uc4, i + 1);
            o[i] = update_pt<ARITH>(get(c4, i), get(p4, i), get(r4, i), get(uc4, i), uzm, uzp,
                                    get(um4, i), get(up4, i), 0.0f);
          }
        }
      } else if constexpr (ARITH == ARITH_FAST) {
        // sponge coefficients: the bottom ramp overrides the row's
        const float2 cx = a.coef_x[xa - 12 + k];
        float cf[4], pc[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
          cf[i] = dz[i] >= 0.f ? cfz[i] : cx.x;
          pc[i] = dz[i] >= 0.f ? pcz[i] : cx.y;
        }
        const float2 a0 = update_pair_coef(lo2(c4), lo2(p4), lo2(r4), lo2(uc4),
                                           f2(__fadd_rn(ucl, uc4.y), __fadd_rn(uc4.x, uc4.z)), lo2(um4), lo2(up4),
                                           f2(cf[0], cf[1]), f2(pc[0], pc[1]));
        const float2 b0 = update_pair_coef(hi2(c4), hi2(p4), hi2(r4), hi2(uc4),
                                           f2(__fadd_rn(uc4.y, uc4.w), __fadd_rn(uc4.z, ucr)), hi2(um4), hi2(up4),
                                           f2(cf[2], cf[3]), f2(pc[2], pc[3]));
        o[0] = a0.x; o[1] = a0.y; o[2] = b0.x; o[3] = b0.y;
      } else {
#pragma unroll
        for (int i = 0; i < 4; i++) {
          float dist = dz[i] >= 0.f ? dz[i] : dxr;
          float delta = __fmul_rn(__fmul_rn(0.05f, dist), dist);
          float uzm = i == 0 ? ucl : get(uc4, i - 1);
          float uzp = i == 3 ? ucr : get(uc4, i + 1);
          o[i] = update_pt<ARITH>(get(c4, i), get(p4, i), get(r4, i), get(uc4, i), uzm, uzp,
                                  get(um4, i), get(up4, i), delta);
        }
      }
      if constexpr (EPI == 2 || EPI == 3) {
        if (hit_left > 0 && xa - 12 + k == hit_x) {
          const float v = hit_vals[(long long)hit_i * hit_stride];
#pragma unroll
          for (int q = 0; q < 4; q++)
            if (q == hit_d) o[q] = EPI == 2 ? __fsub_rn(o[q], v) : __fadd_rn(o[q], v);
          hit_i += hit_di;
          hit_x += hit_dx;
          hit_left--;
        }
        if (EPI == 2 && a.epi.image) {
          const float sc = a.epi.scale;
          float4 r = vimg;
          r.x = __fsub_rn(r.x, __fmul_rn(__fmul_rn(o[0], gimg.x), sc));
          r.y = __fsub_rn(r.y, __fmul_rn(__fmul_rn(o[1], gimg.y), sc));
          r.z = __fsub_rn(r.z, __fmul_rn(__fmul_rn(o[2], gimg.z), sc));
          r.w = __fsub_rn(r.w, __fmul_rn(__fmul_rn(o[3], gimg.w), sc));
          float *ig = a.epi.image + (long long)shot * a.shot_stride + (long long)(xa - 12 + k) * P + zg;
          if (fullgroup) {
            st4(ig, r);
          } else {
            if (zok[0]) ig[0] = r.x;
            if (zok[1]) ig[1] = r.y;
            if (zok[2]) ig[2] = r.z;
            if (zok[3]) ig[3] = r.w;
          }
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
    }
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

  if (!ok && t == 0) {
    // wait (bounded) for copies the producer already issued
    for (int i = k; i < K && i < k + NC; i++) mbar_wait(&full[i & (NC - 1)], (uint32_t)((i >> 4) & 1));
  }
}

}  // namespace swfwi
