// The prestack LSRTM linear operator of swfwi (src/unused/prtm2d.cpp, never
// built by the reference: its header is missing): Born modelling (adj = 0,
// dat += L mod) and migration by source-wavefield reconstruction (adj = 1,
// mod += L' dat), on the GPU.
//
// Scheme (prtm2d.cpp:82-120): second order in time, fourth order in space,
//   u0 = 2 u1 - u0 + vv (c0 u1 + c11 (u1[z-1] + u1[z+1]) + c12 (u1[z-2] +
//        u1[z+2]) + c21 (u1[x-1] + u1[x+1]) + c22 (u1[x-2] + u1[x+2]))
// with vv = (v dt)^2, c11 = 4/(3 dz^2), c12 = -1/(12 dz^2), c21, c22 the
// same in x, c0 = -2 (c11 + c12 + c21 + c22); the "adjoint" form (used by
// Born) moves vv inside the sums.  Fields are [nxpad][nzpad], nzpad = nz +
// 2 nb, nxpad = nx + 2 nb, updated on [2, n-2).  A Gaussian taper w[ib] =
// exp(-(0.015 (nb-1-ib))^2) multiplies the nb cells along every edge
// (apply_sponge, :123-145); a 2-cell ring just outside the model is saved
// every step for the reconstruction (boundary_rw, :37-80).  Data
// dat[is][ig][it], model mod[ix][iz] (z fastest).
//
// Arithmetic: REF evaluates every expression as the reference's C does on
// x86-64 (its 2. literal makes the time update double; the sums are float,
// left to right, no FMA) and runs the shots one after the other, keeping the
// receiver-side fields between shots and calls as the reference's file-scope
// fields do: its Born branch never clears them (:408-434), so a Born shot
// starts from the fields the previous shot or call left.  REF output is
// bit-identical to the compiled reference.  FAST is FP32 with FMA and runs
// up to a memory budget of shots as one batch, each shot's fields starting
// from zero (per-shot images summed in shot order at the end).
//
// Adjoint modes: SWFWI_PRTM_ADJ_REFERENCE is the reference's migration
// (:371-407).  That pair is not adjoint: it images with the time-advanced
// receiver field and injects the data with the opposite sign to what the
// Born branch's recording implies, so <L m, d> and <m, L' d> differ by order
// one.  SWFWI_PRTM_ADJ_EXACT is the exact transpose of the Born branch (with
// per-shot zero start), derived step by step at k_prtm_born_transpose; it
// passes the dot-product test and is what a least-squares (CG) solver needs.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>
#include "common.hpp"
#include "kernels.cuh"

namespace swfwi {
namespace {

constexpr int kLsZ = 128;  // threads per block, along z

struct PrtmCoef {
  float c0, c11, c12, c21, c22;
};

// Field geometry shared by the kernels.  Per-slot positions: the source
// spos[slot] and the receivers rpos[slot*ng + ig] (padded linear indices).
struct PrtmGeo {
  int nx, nz, nb, nxpad, nzpad, nt, ng;
  long long fsz;             // floats per field slot
  const int *spos, *rpos;
  const float *w;            // sponge taper [nb]
  int serial;                // receivers share a cell: inject in ig order
};

// One time step u0 <- 2 u1 - u0 + (stencil) at the padded point (ix, iz)
// of one slot (ix, iz in [2, n-2)); in place (a point reads only its own
// u0).
template <int ARITH, bool ADJ>
__device__ __forceinline__ void prtm_update(float *o, const float *w, const float *vv, long long p, int nzpad,
                                            const PrtmCoef &c) {
  const float uc = w[p];
  if constexpr (ARITH == ARITH_REF) {
    if constexpr (!ADJ) {
      float s = __fmul_rn(c.c0, uc);
      s = __fadd_rn(s, __fmul_rn(c.c11, __fadd_rn(w[p - 1], w[p + 1])));
      s = __fadd_rn(s, __fmul_rn(c.c12, __fadd_rn(w[p - 2], w[p + 2])));
      s = __fadd_rn(s, __fmul_rn(c.c21, __fadd_rn(w[p - nzpad], w[p + nzpad])));
      s = __fadd_rn(s, __fmul_rn(c.c22, __fadd_rn(w[p - 2 * nzpad], w[p + 2 * nzpad])));
      const double t =
          __dadd_rn(__dsub_rn(__dmul_rn(2.0, (double)uc), (double)o[p]), (double)__fmul_rn(vv[p], s));
      o[p] = __double2float_rn(t);
    } else {
      auto vu = [&](long long k) { return __fmul_rn(vv[k], w[k]); };
      double t = __dsub_rn(__dmul_rn(2.0, (double)uc), (double)o[p]);
      t = __dadd_rn(t, (double)__fmul_rn(__fmul_rn(c.c0, vv[p]), uc));
      t = __dadd_rn(t, (double)__fmul_rn(c.c11, __fadd_rn(vu(p - 1), vu(p + 1))));
      t = __dadd_rn(t, (double)__fmul_rn(c.c12, __fadd_rn(vu(p - 2), vu(p + 2))));
      t = __dadd_rn(t, (double)__fmul_rn(c.c21, __fadd_rn(vu(p - nzpad), vu(p + nzpad))));
      t = __dadd_rn(t, (double)__fmul_rn(c.c22, __fadd_rn(vu(p - 2 * nzpad), vu(p + 2 * nzpad))));
      o[p] = __double2float_rn(t);
    }
  } else {
    float s;
    if constexpr (!ADJ) {
      s = c.c0 * uc;
      s = fmaf(c.c11, w[p - 1] + w[p + 1], s);
      s = fmaf(c.c12, w[p - 2] + w[p + 2], s);
      s = fmaf(c.c21, w[p - nzpad] + w[p + nzpad], s);
      s = fmaf(c.c22, w[p - 2 * nzpad] + w[p + 2 * nzpad], s);
      s *= vv[p];
    } else {
      auto vu = [&](long long k) { return vv[k] * w[k]; };
      s = c.c0 * vu(p);
      s = fmaf(c.c11, vu(p - 1) + vu(p + 1), s);
      s = fmaf(c.c12, vu(p - 2) + vu(p + 2), s);
      s = fmaf(c.c21, vu(p - nzpad) + vu(p + nzpad), s);
      s = fmaf(c.c22, vu(p - 2 * nzpad) + vu(p + 2 * nzpad), s);
    }
    o[p] = fmaf(2.0f, uc, -o[p]) + s;
  }
}

// Receivers of one time step for one slot, receiver ig: dat += field
// (mode 2, record) or field += dat (mode 1, inject); dat[slot*nt*ng + ig*nt
// + it].  With g.serial one thread injects every receiver in ig order.
__device__ __forceinline__ void prtm_receiver(const PrtmGeo &g, int slot, int ig, float *f, float *dat, int it,
                                              int mode) {
  if (ig >= g.ng || (g.serial && mode == 1 && ig > 0)) return;
  const int last = (g.serial && mode == 1) ? g.ng : ig + 1;
  for (int r = ig; r < last; r++) {
    float *q = f + (long long)slot * g.fsz + g.rpos[(long long)slot * g.ng + r];
    float *d = dat + (long long)slot * g.nt * g.ng + (long long)r * g.nt + it;
    if (mode == 2) *d = __fadd_rn(*d, *q);
    else *q = __fadd_rn(*q, *d);
  }
}

// The stencil steps of one time step, in one launch: the receiver-side
// pair (G, kg slots, Born's form when gadj) and the source-side pair (S,
// ks slots), blockIdx.z over kg + ks; blocks with blockIdx.y >= nxpad - 4
// record the receivers of G1 (rec_mode 2), which the G step only reads.
// Grid (z blocks of nzpad - 4, nxpad - 4 + receiver columns, kg + ks).
template <int ARITH, bool GADJ>
__global__ void k_prtm_steps(PrtmGeo g, const float *vv, PrtmCoef c, float *g0, const float *g1, int kg, float *s0,
                             const float *s1, float *dat, int it, int rec_mode) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int z = blockIdx.z;
  if ((int)blockIdx.y >= g.nxpad - 4) {
    if (z < kg && rec_mode)
      prtm_receiver(g, z, (blockIdx.y - (g.nxpad - 4)) * gridDim.x * blockDim.x + t, const_cast<float *>(g1), dat,
                    it, rec_mode);
    return;
  }
  const int iz = 2 + t;
  if (iz >= g.nzpad - 2) return;
  const long long p = (long long)(2 + blockIdx.y) * g.nzpad + iz;
  if (z < kg) {
    const long long off = (long long)z * g.fsz;
    prtm_update<ARITH, GADJ>(g0 + off, g1 + off, vv, p, g.nzpad, c);
  } else {
    const long long off = (long long)(z - kg) * g.fsz;
    prtm_update<ARITH, false>(s0 + off, s1 + off, vv, p, g.nzpad, c);
  }
}

// Index in the boundary_rw store of the padded cell (ix, iz), or -1: the 4
// cells above and below each model column, then the two columns on each
// side of the model (:37-80).
__device__ __forceinline__ int prtm_ring_index(const PrtmGeo &g, int ix, int iz) {
  const int mx = ix - g.nb, mz = iz - g.nb;
  if (mx >= 0 && mx < g.nx) {
    if (mz == -2 || mz == -1) return 4 * mx + mz + 2;
    if (mz == g.nz || mz == g.nz + 1) return 4 * mx + 2 + mz - g.nz;
    return -1;
  }
  if (mz >= 0 && mz < g.nz) {
    if (mx == -2 || mx == -1) return 4 * g.nx + mz + g.nz * (mx + 2);
    if (mx == g.nx || mx == g.nx + 1) return 4 * g.nx + mz + g.nz * (2 + mx - g.nx);
  }
  return -1;
}

// The work of one time step on cells that no stencil step of the same
// launch touches, in one launch.  Four roles, one thread per cell, by the
// thread's index t in its slot:
//  * t < ne, the edge cells (the sponge bands, nb cells from every side;
//    the 2-cell ring lies inside them): apply_sponge (:123-145) to up to
//    four fields, in the reference's order for a point ibz cells from the
//    top or bottom and ibx from the left or right (ib ascending, the z
//    edges before the x edges); then save the ring of ring_f (after its
//    sponge) or overwrite it from the store;
//  * the next nm, the model cells: Born injection g += S mod (cross 1) or
//    imaging img += S g (cross 2);
//  * the next nsrc (0 or 1): add_source (:161-189) at the slot's source;
//  * the rest: receivers (rec_mode 1 inject, 2 record).
// The model interior (W = 1) and the sponge bands are disjoint, so the
// roles never touch the same cell.  Grid (blocks over the roles' cells,
// slots).
struct PrtmAux {
  float *sp[4];
  float *ring_f, *ring;
  long long ring_stride;
  int ring_mode;             // 0 none, 1 save, 2 read
  int cross;                 // 0 none, 1 Born injection, 2 imaging
  float *cg;
  const float *cs, *mod;
  float *img;
  long long img_stride;
  float *src_f;              // null: no source operation
  const float *src_val;
  int src_sign;
  float *rec_f, *dat;
  int rec_it, rec_mode;
};

__global__ void k_prtm_aux(PrtmGeo g, PrtmAux a, int ne, int nm, int nsrc) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x, slot = blockIdx.y;
  if (t < ne) {
    // edge cell t: the nb left columns, the nb right columns, then the nb
    // cells at each end of every column between them
    const int band = g.nb * g.nzpad;
    int ix, iz;
    if (t < 2 * band) {
      const int c = t / g.nzpad;
      ix = c < g.nb ? c : g.nxpad - 2 * g.nb + c;
      iz = t - c * g.nzpad;
    } else {
      const int u = t - 2 * band, r = u % (2 * g.nb);
      ix = g.nb + u / (2 * g.nb);
      iz = r < g.nb ? r : g.nzpad - 2 * g.nb + r;
    }
    const long long p = (long long)slot * g.fsz + (long long)ix * g.nzpad + iz;
    const int ibz = min(iz, g.nzpad - 1 - iz), ibx = min(ix, g.nxpad - 1 - ix);
#pragma unroll
    for (int f = 0; f < 4; f++) {
      if (!a.sp[f]) continue;
      float v = a.sp[f][p];
      if (ibz <= ibx) {
        if (ibz < g.nb) v = __fmul_rn(v, g.w[ibz]);
        if (ibx < g.nb) v = __fmul_rn(v, g.w[ibx]);
      } else {
        if (ibx < g.nb) v = __fmul_rn(v, g.w[ibx]);
        if (ibz < g.nb) v = __fmul_rn(v, g.w[ibz]);
      }
      a.sp[f][p] = v;
    }
    if (a.ring_mode) {
      const int i = prtm_ring_index(g, ix, iz);
      if (i >= 0) {
        float *b = a.ring + (long long)slot * a.ring_stride + i;
        if (a.ring_mode == 1) *b = a.ring_f[p];
        else a.ring_f[p] = *b;
      }
    }
    return;
  }
  int u = t - ne;
  if (u < nm) {
    const int mx = u / g.nz, mz = u - mx * g.nz;
    const long long p = (long long)slot * g.fsz + (long long)(mx + g.nb) * g.nzpad + mz + g.nb;
    if (a.cross == 1) {
      a.cg[p] = __fadd_rn(a.cg[p], __fmul_rn(a.cs[p], a.mod[u]));
    } else {
      float *o = a.img + (long long)slot * a.img_stride + u;
      *o = __fadd_rn(*o, __fmul_rn(a.cs[p], a.cg[p]));
    }
    return;
  }
  u -= nm;
  if (u < nsrc) {
    float *f = a.src_f + (long long)slot * g.fsz + g.spos[slot];
    *f = a.src_sign > 0 ? __fadd_rn(*f, *a.src_val) : __fsub_rn(*f, *a.src_val);
    return;
  }
  u -= nsrc;
  if (a.rec_mode) prtm_receiver(g, slot, u, a.rec_f, a.dat, a.rec_it, a.rec_mode);
}

// mod += the per-slot images, in slot order
__global__ void k_prtm_sum_images(float *mod, const float *img, long long nm, int nslots) {
  for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < nm;
       m += (long long)gridDim.x * blockDim.x) {
    float acc = mod[m];
    for (int s = 0; s < nslots; s++) acc = __fadd_rn(acc, img[(long long)s * nm + m]);
    mod[m] = acc;
  }
}

// vv = (v dt)^2 on the padded grid, the model's edge values repeated
// outwards (prtm2d_init, :302-319).  Grid (z blocks of nzpad, nxpad).
__global__ void k_prtm_vv(float *vv, const float *v, int nx, int nz, int nb, float dt) {
  const int nzpad = nz + 2 * nb;
  const int iz = blockIdx.x * blockDim.x + threadIdx.x, ix = blockIdx.y;
  if (iz >= nzpad) return;
  const int sx = min(max(ix - nb, 0), nx - 1), sz = min(max(iz - nb, 0), nz - 1);
  const float t = __fmul_rn(v[(long long)sx * nz + sz], dt);
  vv[(long long)ix * nzpad + iz] = __fmul_rn(t, t);
}

// One reverse step of the exact transpose of the Born branch.  Forward
// step it (fields a = gp0, b = gp1, source field S_it = sp0 at the start):
//   b1 = b + S_it mod;  a' = P (2 W a - W b1 + D V W a) + Q W b1;
//   b' = W a;  d_it = R W a
// (W the sponge, V = vv, D the stencil, P the update mask [2, n-2), Q = 1 -
// P, R the receivers).  Its transpose, with x = P a^ and the data already
// injected into b^ (b^ += R' d_it):
//   a^_prev = W (2 x + V D x + b^);  b1^ = W (Q a^ - x);  b^_prev = b1^;
//   mod^ += S_it b1^ over the model.
// cn <- a^_prev, bh <- b^_prev (bh is read and written at the same point
// only), ah is read.  Grid (z blocks of nzpad, nxpad, slots).
__global__ void k_prtm_born_transpose(float *cn, float *bh, const float *ah, const float *vv, const float *w,
                                      const float *sf, float *img, long long img_stride, int nx, int nz, int nb,
                                      int nxpad, int nzpad, long long fsz, PrtmCoef c) {
  const int iz = blockIdx.x * blockDim.x + threadIdx.x, ix = blockIdx.y;
  if (iz >= nzpad) return;
  const long long off = (long long)blockIdx.z * fsz;
  const float *A = ah + off;
  auto x = [&](int jx, int jz) -> float {
    return (jx >= 2 && jx < nxpad - 2 && jz >= 2 && jz < nzpad - 2) ? A[(long long)jx * nzpad + jz] : 0.0f;
  };
  const long long q = (long long)ix * nzpad + iz;
  const float xc = x(ix, iz);
  float s = c.c0 * xc;
  s = fmaf(c.c11, x(ix, iz - 1) + x(ix, iz + 1), s);
  s = fmaf(c.c12, x(ix, iz - 2) + x(ix, iz + 2), s);
  s = fmaf(c.c21, x(ix - 1, iz) + x(ix + 1, iz), s);
  s = fmaf(c.c22, x(ix - 2, iz) + x(ix + 2, iz), s);
  const int ibz = min(iz, nzpad - 1 - iz), ibx = min(ix, nxpad - 1 - ix);
  const float wp = (ibz < nb ? w[ibz] : 1.0f) * (ibx < nb ? w[ibx] : 1.0f);
  const long long p = off + q;
  cn[p] = wp * fmaf(vv[q], s, fmaf(2.0f, xc, bh[p]));
  const float a = A[q];
  const bool upd = ix >= 2 && ix < nxpad - 2 && iz >= 2 && iz < nzpad - 2;
  const float b1 = wp * (upd ? -a : a);
  bh[p] = b1;
  const int mx = ix - nb, mz = iz - nb;
  if (mx >= 0 && mx < nx && mz >= 0 && mz < nz) {
    float *o = img + (long long)blockIdx.z * img_stride + (long long)mx * nz + mz;
    *o = fmaf(sf[p], b1, *o);
  }
}

// device bytes the FAST path may use for one batch of shots
constexpr size_t kBatchBudget = size_t(24) << 30;

}  // namespace

// The operator's state (prtm2d_init's file-scope variables, per object).
class Prtm {
 public:
  Prtm(int arith, float dz, float dx, float dt, float amp, float fm, int nz, int nx, int nb, int nt, int ns, int ng,
       int sxbeg, int szbeg, int jsx, int jsz, int gxbeg, int gzbeg, int jgx, int jgz, bool csd, const float *vel,
       cudaStream_t st)
      : arith_(arith), nz_(nz), nx_(nx), nb_(nb), nt_(nt), ns_(ns), ng_(ng) {
    SWFWI_REQUIRE(arith == ARITH_REF || arith == ARITH_FAST, "arithmetic must be REF or FAST");
    SWFWI_REQUIRE(nz > 0 && nx > 0 && nb >= 2 && nt > 0 && ns > 0 && ng > 0, "bad sizes");
    SWFWI_REQUIRE(vel, "null velocity");
    nzpad_ = nz + 2 * nb;
    nxpad_ = nx + 2 * nb;
    SWFWI_REQUIRE((long long)nzpad_ * nxpad_ < (1LL << 31) && nxpad_ + nx_ + ng <= 65535, "grid too large");
    SWFWI_REQUIRE((long long)nt * ng * ns < (1LL << 31) && (long long)nx * nz < (1LL << 31),
                  "data or model too large for the operator's int sizes");
    // prtm2d_init's geometry checks (:326-336), applied to every shot and
    // receiver: the reference checks the first and last only
    const int distx = sxbeg - gxbeg;
    std::vector<int> spos(ns), rpos((size_t)ns * ng);
    for (int is = 0; is < ns; is++) {
      const int sx = sxbeg + is * jsx, sz = szbeg + is * jsz;
      SWFWI_REQUIRE(sx >= 0 && sx < nx && sz >= 0 && sz < nz, "sources exceed the computing zone");
      spos[is] = pidx(sx, sz);
      const int gx0 = csd ? sx - distx : gxbeg;
      for (int ig = 0; ig < ng; ig++) {
        const int gx = gx0 + ig * jgx, gz = gzbeg + ig * jgz;
        SWFWI_REQUIRE(gx >= 0 && gx < nx && gz >= 0 && gz < nz, "geophones exceed the computing zone");
        rpos[(size_t)is * ng + ig] = pidx(gx, gz);
      }
    }
    // coefficients, as prtm2d_init computes them (:254-261)
    float t = (float)(1.0 / (dz * dz));
    c_.c11 = (float)(4.0 * t / 3.0);
    c_.c12 = (float)(-t / 12.0);
    t = (float)(1.0 / (dx * dx));
    c_.c21 = (float)(4.0 * t / 3.0);
    c_.c22 = (float)(-t / 12.0);
    c_.c0 = (float)(-2.0 * (c_.c11 + c_.c12 + c_.c21 + c_.c22));
    // sponge taper and Ricker wavelet (:296-299, :320-323)
    std::vector<float> w(nb), wlt(nt);
    for (int ib = 0; ib < nb; ib++) {
      const float tt = (float)(0.015 * (nb - 1 - ib));
      w[ib] = expf(-tt * tt);
    }
    for (int it = 0; it < nt; it++) {
      float tt = (float)(3.14159265358979323846264338328 * fm * (it * dt - 1.0 / fm));
      tt = tt * tt;
      wlt[it] = (float)(amp * (1.0 - 2.0 * tt) * expf(-tt));
    }
    sponge_.upload(w, st);
    wlt_.upload(wlt, st);
    spos_.upload(spos, st);
    rpos_.upload(rpos, st);
    vv_.resize((size_t)nxpad_ * nzpad_);
    k_prtm_vv<<<dim3((nzpad_ + kLsZ - 1) / kLsZ, nxpad_), kLsZ, 0, st>>>(vv_.get(), vel, nx, nz, nb, dt);
    note_launch();
    SWFWI_CUDA(cudaGetLastError());
    // the shot batch: one shot for REF (the reference's order), else as
    // many as the budget holds; every buffer a call needs, allocated here
    const size_t fsz = (size_t)nxpad_ * nzpad_;
    const size_t per_shot = sizeof(float) * (5 * fsz + (size_t)nt * 4 * (nx + nz) + (size_t)nx * nz);
    kmax_ = arith == ARITH_REF ? 1 : (int)std::max<size_t>(1, std::min<size_t>(ns, kBatchBudget / per_shot));
    kmax_ = std::min(kmax_, 65535);
    for (DevBuf<float> *f : {&sp0_, &sp1_, &gp0_, &gp1_, &gp2_}) {
      f->resize((size_t)kmax_ * fsz);
      f->zero(st);
    }
    ring_.resize((size_t)kmax_ * nt * 4 * (nx + nz));
    if (kmax_ > 1) img_.resize((size_t)kmax_ * nx * nz);
    geo_ = PrtmGeo{nx, nz, nb, nxpad_, nzpad_, nt, ng, (long long)fsz, spos_.get(), rpos_.get(), sponge_.get(),
                   ng > 1 && jgx == 0 && jgz == 0 ? 1 : 0};
  }

  ~Prtm() {
    for (Graph &g : graphs_)
      if (g.exec) cudaGraphExecDestroy(g.exec);
    if (cap_) cudaStreamDestroy(cap_);
  }

  int nx() const { return nx_; }
  int nz() const { return nz_; }
  int nt() const { return nt_; }
  int ng() const { return ng_; }
  int ns() const { return ns_; }
  int batch() const { return kmax_; }
  void set_adjoint_mode(int m) {
    SWFWI_REQUIRE(m == SWFWI_PRTM_ADJ_REFERENCE || m == SWFWI_PRTM_ADJ_EXACT, "unknown adjoint mode");
    adj_mode_ = m;
  }
  void set_graphs(bool on) { use_graphs_ = on; }

  // prtm2d_lop (:354-437) on device arrays.  A call that repeats an earlier
  // one's arrays, direction and mode replays the time loops as one CUDA
  // graph (captured on the second such call).
  void lop(bool adj, bool add, float *mod, float *dat, cudaStream_t st) {
    const std::vector<long long> key = {adj, add, adj_mode_, reinterpret_cast<long long>(mod),
                                        reinterpret_cast<long long>(dat), g_swapped_};
    auto body = [&](cudaStream_t s) {
      const long long nm = (long long)nx_ * nz_, nd = (long long)nt_ * ng_ * ns_;
      // sf_adjnull: without add, the output starts at zero
      if (!add) {
        if (adj) SWFWI_CUDA(cudaMemsetAsync(mod, 0, sizeof(float) * nm, s));
        else SWFWI_CUDA(cudaMemsetAsync(dat, 0, sizeof(float) * nd, s));
      }
      for (int s0 = 0; s0 < ns_; s0 += kmax_) run(adj, mod, dat, s0, std::min(kmax_, ns_ - s0), s);
    };
    if (!use_graphs_) {
      body(st);
      SWFWI_CUDA(cudaGetLastError());
      return;
    }
    for (size_t i = 0; i < graphs_.size(); i++)
      if (graphs_[i].key == key) {
        if (graphs_[i].exec) {
          SWFWI_CUDA(cudaGraphLaunch(graphs_[i].exec, st));
          g_kernel_launches.fetch_add(graphs_[i].kernels);   // the kernels the graph holds
          g_swapped_ = graphs_[i].swapped_after;
          return;
        }
        // second call with these arrays: capture the calls from now on
        if (!cap_) SWFWI_CUDA(cudaStreamCreateWithFlags(&cap_, cudaStreamNonBlocking));
        cudaGraph_t g = nullptr;
        const long long n0 = thread_launches();
        SWFWI_CUDA(cudaStreamBeginCapture(cap_, cudaStreamCaptureModeThreadLocal));
        try {
          body(cap_);
        } catch (...) {
          cudaStreamEndCapture(cap_, &g);
          if (g) cudaGraphDestroy(g);
          throw;
        }
        // the capture launched nothing: its kernels count at each launch
        graphs_[i].kernels = thread_launches() - n0;
        g_kernel_launches.fetch_sub(graphs_[i].kernels);
        SWFWI_CUDA(cudaStreamEndCapture(cap_, &g));
        const cudaError_t err = cudaGraphInstantiate(&graphs_[i].exec, g, 0);
        cudaGraphDestroy(g);
        SWFWI_CUDA(err);
        graphs_[i].swapped_after = g_swapped_;
        SWFWI_CUDA(cudaGraphLaunch(graphs_[i].exec, st));
        g_kernel_launches.fetch_add(graphs_[i].kernels);
        return;
      }
    body(st);
    SWFWI_CUDA(cudaGetLastError());
    if (graphs_.size() >= kGraphs) {
      if (graphs_.front().exec) cudaGraphExecDestroy(graphs_.front().exec);
      graphs_.erase(graphs_.begin());
    }
    graphs_.push_back(Graph{key, nullptr, g_swapped_, 0});
  }

 private:
  struct Graph {
    std::vector<long long> key;
    cudaGraphExec_t exec;
    bool swapped_after;
    long long kernels = 0;   // kernel launches the graph holds
  };
  static constexpr size_t kGraphs = 4;

  int pidx(int x, int z) const { return (x + nb_) * nzpad_ + z + nb_; }
  long long fsz() const { return (long long)nxpad_ * nzpad_; }
  int rec_cols(int zthreads) const { return (ng_ + zthreads - 1) / zthreads; }

  // the stencil steps of one time step (k_prtm_steps); kg, ks slots of the
  // receiver and source pairs, G's in Born's form when gadj
  void steps(const PrtmGeo &geo, bool gadj, float *g0, const float *g1, int kg, float *s0, const float *s1, int ks,
             float *dat, int it, int rec_mode, cudaStream_t st) {
    const int zb = (nzpad_ - 4 + kLsZ - 1) / kLsZ;
    const dim3 grid(zb, nxpad_ - 4 + (rec_mode ? rec_cols(zb * kLsZ) : 0), kg + ks);
    if (arith_ == ARITH_REF) {
      if (gadj) k_prtm_steps<ARITH_REF, true><<<grid, kLsZ, 0, st>>>(geo, vv_.get(), c_, g0, g1, kg, s0, s1, dat, it,
                                                                     rec_mode);
      else k_prtm_steps<ARITH_REF, false><<<grid, kLsZ, 0, st>>>(geo, vv_.get(), c_, g0, g1, kg, s0, s1, dat, it,
                                                                 rec_mode);
    } else {
      if (gadj) k_prtm_steps<ARITH_FAST, true><<<grid, kLsZ, 0, st>>>(geo, vv_.get(), c_, g0, g1, kg, s0, s1, dat,
                                                                      it, rec_mode);
      else k_prtm_steps<ARITH_FAST, false><<<grid, kLsZ, 0, st>>>(geo, vv_.get(), c_, g0, g1, kg, s0, s1, dat, it,
                                                                  rec_mode);
    }
    note_launch();
  }

  void aux(const PrtmGeo &geo, const PrtmAux &a, int k, cudaStream_t st) {
    // the roles a launch needs, one thread per cell: edge cells, model
    // cells, the source, the receivers
    const bool edges = a.sp[0] || a.sp[1] || a.sp[2] || a.sp[3] || a.ring_mode;
    const int ne = edges ? nxpad_ * nzpad_ - (nxpad_ - 2 * nb_) * (nzpad_ - 2 * nb_) : 0;
    const int nm = a.cross ? nx_ * nz_ : 0, nsrc = a.src_f ? 1 : 0, nrec = a.rec_mode ? ng_ : 0;
    const long long total = (long long)ne + nm + nsrc + nrec;
    if (total <= 0) return;
    const dim3 grid((unsigned)((total + 255) / 256), k);
    k_prtm_aux<<<grid, 256, 0, st>>>(geo, a, ne, nm, nsrc);
    note_launch();
  }

  static PrtmAux none() {
    PrtmAux a;
    memset(&a, 0, sizeof(a));
    return a;
  }

  // One batch of k shots from shot s0.  Each time step is two or three
  // launches: the stencil steps of both field pairs in one (k_prtm_steps),
  // and the sponge, ring, imaging or Born injection, source and receivers
  // in one or two (k_prtm_aux), the reference's operations regrouped where
  // they touch disjoint cells and so commute.
  void run(bool adj, float *mod, float *dat, int s0, int k, cudaStream_t st) {
    const long long nm = (long long)nx_ * nz_;
    const size_t fbytes = sizeof(float) * (size_t)k * fsz();
    // the batch's positions
    PrtmGeo g = geo_;
    g.spos = spos_.get() + s0;
    g.rpos = rpos_.get() + (size_t)s0 * ng_;
    // the shot's source fields start at zero (:364-365); the receiver
    // fields do in the migration (:381-382) and, outside REF, in Born
    SWFWI_CUDA(cudaMemsetAsync(sp0_.get(), 0, fbytes, st));
    SWFWI_CUDA(cudaMemsetAsync(sp1_.get(), 0, fbytes, st));
    float *S0 = sp0_.get(), *S1 = sp1_.get();
    float *G0 = gp0_.get(), *G1 = gp1_.get();
    if (g_swapped_) std::swap(G0, G1);
    if (adj || arith_ != ARITH_REF) {
      SWFWI_CUDA(cudaMemsetAsync(G0, 0, fbytes, st));
      SWFWI_CUDA(cudaMemsetAsync(G1, 0, fbytes, st));
    }
    float *d = dat + (long long)s0 * nt_ * ng_;
    const float *wl = wlt_.get();
    if (adj) {
      const int m = 4 * (nx_ + nz_);
      const long long rstride = (long long)nt_ * m;
      // the source field forward, its ring saved every step (:372-379):
      // source at it, step, sponge, swap, save; the next step's source
      // rides with this step's sponge
      PrtmAux a = none();
      a.src_f = S1;
      a.src_val = wl;
      a.src_sign = 1;
      aux(g, a, k, st);
      for (int it = 0; it < nt_; it++) {
        steps(g, false, nullptr, nullptr, 0, S0, S1, k, nullptr, 0, 0, st);
        a = none();
        a.sp[0] = S0;
        a.sp[1] = S1;
        std::swap(S0, S1);
        a.ring_mode = 1;
        a.ring_f = S0;
        a.ring = ring_.get() + (long long)it * m;
        a.ring_stride = rstride;
        if (it + 1 < nt_) {
          a.src_f = S1;
          a.src_val = wl + it + 1;
          a.src_sign = 1;
        }
        aux(g, a, k, st);
      }
      float *img = mod;
      long long img_stride = 0;
      if (k > 1) {
        SWFWI_CUDA(cudaMemsetAsync(img_.get(), 0, sizeof(float) * (size_t)k * nm, st));
        img = img_.get();
        img_stride = nm;
      }
      const bool exact = adj_mode_ == SWFWI_PRTM_ADJ_EXACT;
      float *G2 = gp2_.get();
      const dim3 gfull((nzpad_ + kLsZ - 1) / kLsZ, nxpad_, k);
      for (int it = nt_ - 1; it >= 0; it--) {
        // ring of the source field (:388), the previous step's source
        // subtraction (:391), the data into the receiver field (:394-398)
        a = none();
        a.ring_mode = 2;
        a.ring_f = S0;
        a.ring = ring_.get() + (long long)it * m;
        a.ring_stride = rstride;
        if (it + 1 < nt_) {
          a.src_f = S1;
          a.src_val = wl + it + 1;
          a.src_sign = -1;
        }
        a.rec_f = G1;
        a.dat = d;
        a.rec_it = it;
        a.rec_mode = 1;
        aux(g, a, k, st);
        std::swap(S0, S1);
        if (exact) {
          // G0 = a^, G1 = b^ (data injected), G2 scratch
          steps(g, false, nullptr, nullptr, 0, S0, S1, k, nullptr, 0, 0, st);
          k_prtm_born_transpose<<<gfull, kLsZ, 0, st>>>(G2, G1, G0, vv_.get(), sponge_.get(), S0, img, img_stride,
                                                        nx_, nz_, nb_, nxpad_, nzpad_, fsz(), c_);
          note_launch();
          std::swap(G0, G2);
        } else {
          // reconstruct (:390), back-propagate (:399-402) and image (:404-406)
          steps(g, false, G0, G1, k, S0, S1, k, nullptr, 0, 0, st);
          a = none();
          a.sp[0] = G0;
          a.sp[1] = G1;
          std::swap(G0, G1);
          a.cross = 2;
          a.cs = S0;
          a.cg = G1;
          a.img = img;
          a.img_stride = img_stride;
          aux(g, a, k, st);
        }
      }
      if (k > 1) {
        const long long blocks = std::min<long long>((nm + 255) / 256, 148 * 16);
        k_prtm_sum_images<<<(unsigned)blocks, 256, 0, st>>>(mod, img_.get(), nm, k);
        note_launch();
      }
      if (exact) {
        // the rotation through the scratch field leaves the receiver fields
        // in no order a later REF Born could continue from: clear them
        SWFWI_CUDA(cudaMemsetAsync(gp0_.get(), 0, fbytes, st));
        SWFWI_CUDA(cudaMemsetAsync(gp1_.get(), 0, fbytes, st));
        G0 = gp0_.get();
        G1 = gp1_.get();
      }
    } else {
      // Born modelling (:410-434).  Per step: the injection G1 += S0 mod,
      // the swap, the receiver pair's sponge, the source into S1 and the
      // source pair's sponge of the previous step; then both stencil steps
      // with the receivers recorded from G1
      for (int it = 0; it < nt_; it++) {
        PrtmAux a = none();
        a.cross = 1;
        a.cg = G1;
        a.cs = S0;
        a.mod = mod;
        std::swap(G0, G1);
        a.sp[0] = G0;
        a.sp[1] = G1;
        a.sp[2] = S0;
        a.sp[3] = S1;
        a.src_f = S1;
        a.src_val = wl + it;
        a.src_sign = 1;
        aux(g, a, k, st);
        steps(g, true, G0, G1, k, S0, S1, k, d, it, 2, st);
        std::swap(S0, S1);
      }
    }
    g_swapped_ = G0 != gp0_.get();
  }

  int arith_, nz_, nx_, nb_, nt_, ns_, ng_, nzpad_ = 0, nxpad_ = 0;
  int kmax_ = 1, adj_mode_ = SWFWI_PRTM_ADJ_REFERENCE;
  bool g_swapped_ = false, use_graphs_ = true;
  PrtmCoef c_{};
  PrtmGeo geo_{};
  DevBuf<float> vv_, wlt_, sponge_, sp0_, sp1_, gp0_, gp1_, gp2_, ring_, img_;
  DevBuf<int> spos_, rpos_;
  std::vector<Graph> graphs_;
  cudaStream_t cap_ = nullptr;
};

}  // namespace swfwi

using namespace swfwi;

struct swfwi_prtm {
  std::unique_ptr<Prtm> p;
};

extern "C" int swfwi_prtm2d_create(swfwi_prtm **out, int arith, float dz, float dx, float dt, float amp, float fm,
                                   int nz, int nx, int nb, int nt, int ns, int ng, int sxbeg, int szbeg, int jsx,
                                   int jsz, int gxbeg, int gzbeg, int jgx, int jgz, int csdgather, const float *vel,
                                   void *stream) {
  return guarded([&] {
    SWFWI_REQUIRE(out, "null output");
    *out = nullptr;
    std::unique_ptr<swfwi_prtm> h(new swfwi_prtm);
    h->p.reset(new Prtm(arith, dz, dx, dt, amp, fm, nz, nx, nb, nt, ns, ng, sxbeg, szbeg, jsx, jsz, gxbeg, gzbeg,
                        jgx, jgz, csdgather != 0, vel, reinterpret_cast<cudaStream_t>(stream)));
    *out = h.release();
  });
}

extern "C" int swfwi_prtm2d_set_adjoint(swfwi_prtm *h, int mode) {
  return guarded([&] {
    SWFWI_REQUIRE(h && h->p, "null handle");
    h->p->set_adjoint_mode(mode);
  });
}

extern "C" int swfwi_prtm2d_set_graphs(swfwi_prtm *h, int on) {
  return guarded([&] {
    SWFWI_REQUIRE(h && h->p, "null handle");
    h->p->set_graphs(on != 0);
  });
}

extern "C" int swfwi_prtm2d_batch(swfwi_prtm *h, int *shots) {
  return guarded([&] {
    SWFWI_REQUIRE(h && h->p && shots, "null handle or output");
    *shots = h->p->batch();
  });
}

extern "C" int swfwi_prtm2d_lop(swfwi_prtm *h, int adj, int add, int nm, int nd, float *mod, float *dat,
                                void *stream) {
  return guarded([&] {
    SWFWI_REQUIRE(h && h->p && mod && dat, "null handle or array");
    Prtm &p = *h->p;
    // prtm2d_lop's size checks (:358-359)
    SWFWI_REQUIRE((long long)nm == (long long)p.nx() * p.nz(), "model size mismatch");
    SWFWI_REQUIRE((long long)nd == (long long)p.nt() * p.ng() * p.ns(), "data size mismatch");
    p.lop(adj != 0, add != 0, mod, dat, reinterpret_cast<cudaStream_t>(stream));
  });
}

extern "C" int swfwi_prtm2d_destroy(swfwi_prtm *h) {
  return guarded([&] { delete h; });
}
