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

// One time step of every slot's field: u0 <- 2 u1 - u0 + (stencil) on
// [2, nxpad-2) x [2, nzpad-2), in place (a point reads only its own u0).
// Grid (z blocks, nxpad - 4 columns, slots).
template <int ARITH, bool ADJ>
__global__ void k_prtm_step(float *u0, const float *u1, const float *vv, int nzpad, long long fsz, PrtmCoef c) {
  const int iz = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  if (iz >= nzpad - 2) return;
  const long long off = (long long)blockIdx.z * fsz;
  const long long p = (long long)(2 + blockIdx.y) * nzpad + iz;
  const float *w = u1 + off;
  float *o = u0 + off;
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

// The cells of column ix that the sponge touches: all of an edge column,
// else the nb cells at each end.  Thread t of the column -> iz, or -1.
__device__ __forceinline__ int sponge_iz(int t, int ix, int nxpad, int nzpad, int nb) {
  const bool edge = ix < nb || ix >= nxpad - nb;
  if (edge) return t < nzpad ? t : -1;
  if (t >= 2 * nb) return -1;
  return t < nb ? t : nzpad - 2 * nb + t;
}

// apply_sponge on two sets of fields.  A point ibz cells from the top or
// bottom and ibx cells from the left or right edge is multiplied by w[ibz]
// and w[ibx] (each only when < nb) in the reference's loop order: ib
// ascending, the z edges before the x edges of the same ib.  Grid (z
// blocks of nzpad, nxpad columns, slots).
__global__ void k_prtm_sponge(float *a, float *b, const float *w, int nxpad, int nzpad, int nb, long long fsz) {
  const int ix = blockIdx.y;
  const int iz = sponge_iz(blockIdx.x * blockDim.x + threadIdx.x, ix, nxpad, nzpad, nb);
  if (iz < 0) return;
  const int ibz = min(iz, nzpad - 1 - iz), ibx = min(ix, nxpad - 1 - ix);
  const long long p = (long long)blockIdx.z * fsz + (long long)ix * nzpad + iz;
  float *fs[2] = {a + p, b + p};
#pragma unroll
  for (int f = 0; f < 2; f++) {
    float v = *fs[f];
    if (ibz <= ibx) {
      if (ibz < nb) v = __fmul_rn(v, w[ibz]);
      if (ibx < nb) v = __fmul_rn(v, w[ibx]);
    } else {
      if (ibx < nb) v = __fmul_rn(v, w[ibx]);
      if (ibz < nb) v = __fmul_rn(v, w[ibz]);
    }
    *fs[f] = v;
  }
}

// boundary_rw: the 2-cell ring of one step, 4 (nx + nz) values a slot at
// bnd + slot * bnd_stride, in the reference's order (the 4 cells above and
// below each column, then the two columns left and right of the model).
// Grid (ring blocks, slots).
__global__ void k_prtm_ring(float *p, float *bnd, long long bnd_stride, int nx, int nz, int nb, int nzpad,
                            long long fsz, int read) {
  const int m = 4 * (nx + nz);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  int gx, gz;
  if (i < 4 * nx) {
    const int r = i % 4;
    gx = i / 4 + nb;
    gz = r < 2 ? r - 2 + nb : r - 2 + nz + nb;
  } else {
    const int j = i - 4 * nx, col = j / nz;
    gz = j % nz + nb;
    gx = col < 2 ? col - 2 + nb : col - 2 + nx + nb;
  }
  float *f = p + (long long)blockIdx.y * fsz + (long long)gx * nzpad + gz;
  float *b = bnd + (long long)blockIdx.y * bnd_stride + i;
  if (read) *f = *b;
  else *b = *f;
}

// add_source (:161-189) of the wavelet sample *val at slot s's position
__global__ void k_prtm_source(float *p, const int *pos, const float *val, long long fsz, int nslots, int sign) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslots) return;
  float *f = p + (long long)s * fsz + pos[s];
  *f = sign > 0 ? __fadd_rn(*f, *val) : __fsub_rn(*f, *val);
}

// Receivers of one time step: dat += field (record) or field += dat
// (inject).  rec[s*ng + ig] padded linear index; dat[s*dat_stride + ig*nt
// + it].  serial: receivers that share a cell, injected in ig order by one
// thread.  Grid (receiver blocks, slots).
__global__ void k_prtm_receivers(float *p, float *dat, const int *rec, long long dat_stride, int ng, int nt, int it,
                                 long long fsz, int record, int serial) {
  const int s = blockIdx.y;
  const int first = blockIdx.x * blockDim.x + threadIdx.x;
  if (first >= ng || (serial && first > 0)) return;
  const int last = serial ? ng : first + 1;
  for (int ig = first; ig < last; ig++) {
    float *f = p + (long long)s * fsz + rec[(long long)s * ng + ig];
    float *d = dat + (long long)s * dat_stride + (long long)ig * nt + it;
    if (record) *d = __fadd_rn(*d, *f);
    else *f = __fadd_rn(*f, *d);
  }
}

// Over the model interior: imaging img[s*img_stride + ix*nz + iz] += S g
// (born = 0), or Born injection g += S mod (born = 1).  Grid (z blocks,
// nx, slots).
__global__ void k_prtm_cross(float *img, long long img_stride, float *g, const float *sf, const float *mod, int nz,
                             int nb, int nzpad, long long fsz, int born) {
  const int iz = blockIdx.x * blockDim.x + threadIdx.x;
  if (iz >= nz) return;
  const int ix = blockIdx.y, slot = blockIdx.z;
  const long long m = (long long)ix * nz + iz;
  const long long p = (long long)slot * fsz + (long long)(ix + nb) * nzpad + iz + nb;
  if (born) {
    g[p] = __fadd_rn(g[p], __fmul_rn(sf[p], mod[m]));
  } else {
    float *o = img + (long long)slot * img_stride + m;
    *o = __fadd_rn(*o, __fmul_rn(sf[p], g[p]));
  }
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
    SWFWI_REQUIRE((long long)nzpad_ * nxpad_ < (1LL << 31) && nxpad_ <= 65535, "grid too large");
    SWFWI_REQUIRE((long long)nt * ng * ns < (1LL << 31) && (long long)nx * nz < (1LL << 31),
                  "data or model too large for the operator's int sizes");
    // prtm2d_init's geometry checks (:326-336), applied to every shot and
    // receiver: the reference checks the first and last only
    const int distx = sxbeg - gxbeg;
    spos_h_.resize(ns);
    rpos_h_.resize((size_t)ns * ng);
    for (int is = 0; is < ns; is++) {
      const int sx = sxbeg + is * jsx, sz = szbeg + is * jsz;
      SWFWI_REQUIRE(sx >= 0 && sx < nx && sz >= 0 && sz < nz, "sources exceed the computing zone");
      spos_h_[is] = pidx(sx, sz);
      const int gx0 = csd ? sx - distx : gxbeg;
      for (int ig = 0; ig < ng; ig++) {
        const int gx = gx0 + ig * jgx, gz = gzbeg + ig * jgz;
        SWFWI_REQUIRE(gx >= 0 && gx < nx && gz >= 0 && gz < nz, "geophones exceed the computing zone");
        rpos_h_[(size_t)is * ng + ig] = pidx(gx, gz);
      }
    }
    serial_rec_ = ng > 1 && jgx == 0 && jgz == 0;
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
    vv_.resize((size_t)nxpad_ * nzpad_);
    k_prtm_vv<<<dim3((nzpad_ + kLsZ - 1) / kLsZ, nxpad_), kLsZ, 0, st>>>(vv_.get(), vel, nx, nz, nb, dt);
    note_launch();
    SWFWI_CUDA(cudaGetLastError());
    // the shot batch: one shot for REF (the reference's order), else as
    // many as the budget holds
    const size_t fsz = (size_t)nxpad_ * nzpad_;
    const size_t per_shot =
        sizeof(float) * (5 * fsz + (size_t)nt * 4 * (nx + nz) + (size_t)nx * nz) + sizeof(int) * (1 + ng);
    kmax_ = arith == ARITH_REF ? 1 : (int)std::max<size_t>(1, std::min<size_t>(ns, kBatchBudget / per_shot));
    kmax_ = std::min(kmax_, 65535);
    for (DevBuf<float> *f : {&sp0_, &sp1_, &gp0_, &gp1_}) {
      f->resize((size_t)kmax_ * fsz);
      f->zero(st);
    }
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

  // prtm2d_lop (:354-437) on device arrays
  void lop(bool adj, bool add, float *mod, float *dat, cudaStream_t st) {
    const long long nm = (long long)nx_ * nz_, nd = (long long)nt_ * ng_ * ns_;
    // sf_adjnull: without add, the output starts at zero
    if (!add) {
      if (adj) SWFWI_CUDA(cudaMemsetAsync(mod, 0, sizeof(float) * nm, st));
      else SWFWI_CUDA(cudaMemsetAsync(dat, 0, sizeof(float) * nd, st));
    }
    for (int s0 = 0; s0 < ns_; s0 += kmax_) run(adj, mod, dat, s0, std::min(kmax_, ns_ - s0), st);
    SWFWI_CUDA(cudaGetLastError());
  }

 private:
  int pidx(int x, int z) const { return (x + nb_) * nzpad_ + z + nb_; }
  long long fsz() const { return (long long)nxpad_ * nzpad_; }

  void step(float *u0, const float *u1, bool adj_form, int k, cudaStream_t st) {
    const dim3 g((nzpad_ - 4 + kLsZ - 1) / kLsZ, nxpad_ - 4, k);
    if (arith_ == ARITH_REF) {
      if (adj_form) k_prtm_step<ARITH_REF, true><<<g, kLsZ, 0, st>>>(u0, u1, vv_.get(), nzpad_, fsz(), c_);
      else k_prtm_step<ARITH_REF, false><<<g, kLsZ, 0, st>>>(u0, u1, vv_.get(), nzpad_, fsz(), c_);
    } else {
      if (adj_form) k_prtm_step<ARITH_FAST, true><<<g, kLsZ, 0, st>>>(u0, u1, vv_.get(), nzpad_, fsz(), c_);
      else k_prtm_step<ARITH_FAST, false><<<g, kLsZ, 0, st>>>(u0, u1, vv_.get(), nzpad_, fsz(), c_);
    }
    note_launch();
  }

  void sponge(float *a, float *b, int k, cudaStream_t st) {
    const dim3 g((nzpad_ + kLsZ - 1) / kLsZ, nxpad_, k);
    k_prtm_sponge<<<g, kLsZ, 0, st>>>(a, b, sponge_.get(), nxpad_, nzpad_, nb_, fsz());
    note_launch();
  }

  void source(float *p, int it, int sign, int k, cudaStream_t st) {
    k_prtm_source<<<(k + 127) / 128, 128, 0, st>>>(p, spos_.get(), wlt_.get() + it, fsz(), k, sign);
    note_launch();
  }

  void receivers(float *p, float *d, int it, bool record, int k, cudaStream_t st) {
    const bool serial = serial_rec_ && !record;
    const dim3 g(serial ? 1 : (ng_ + 127) / 128, k);
    k_prtm_receivers<<<g, 128, 0, st>>>(p, d, rpos_.get(), (long long)nt_ * ng_, ng_, nt_, it, fsz(), record,
                                        serial);
    note_launch();
  }

  void ring(float *p, int it, bool read, int k, cudaStream_t st) {
    const int m = 4 * (nx_ + nz_);
    k_prtm_ring<<<dim3((m + 255) / 256, k), 256, 0, st>>>(p, ring_.get() + (long long)it * m, (long long)nt_ * m,
                                                          nx_, nz_, nb_, nzpad_, fsz(), read);
    note_launch();
  }

  void run(bool adj, float *mod, float *dat, int s0, int k, cudaStream_t st) {
    const long long nm = (long long)nx_ * nz_;
    const size_t fbytes = sizeof(float) * (size_t)k * fsz();
    spos_.upload(spos_h_.data() + s0, k, st);
    rpos_.upload(rpos_h_.data() + (size_t)s0 * ng_, (size_t)k * ng_, st);
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
    const dim3 gmod((nz_ + kLsZ - 1) / kLsZ, nx_, k);
    if (adj) {
      // the source field forward, its ring saved every step (:372-379)
      ring_.resize((size_t)k * nt_ * 4 * (nx_ + nz_));
      for (int it = 0; it < nt_; it++) {
        source(S1, it, +1, k, st);
        step(S0, S1, false, k, st);
        sponge(S0, S1, k, st);
        std::swap(S0, S1);
        ring(S0, it, false, k, st);
      }
      float *img = mod;
      long long img_stride = 0;
      if (k > 1) {
        img_.resize((size_t)k * nm);
        img_.zero(st);
        img = img_.get();
        img_stride = nm;
      }
      const bool exact = adj_mode_ == SWFWI_PRTM_ADJ_EXACT;
      float *G2 = nullptr;
      if (exact) {
        gp2_.resize((size_t)k * fsz());
        G2 = gp2_.get();
      }
      const dim3 gfull((nzpad_ + kLsZ - 1) / kLsZ, nxpad_, k);
      for (int it = nt_ - 1; it >= 0; it--) {
        // reconstruct the source field (:388-391)
        ring(S0, it, true, k, st);
        std::swap(S0, S1);
        step(S0, S1, false, k, st);
        source(S1, it, -1, k, st);
        receivers(G1, d, it, false, k, st);
        if (exact) {
          // G0 = a^, G1 = b^ (the data just injected), G2 scratch
          k_prtm_born_transpose<<<gfull, kLsZ, 0, st>>>(G2, G1, G0, vv_.get(), sponge_.get(), S0, img, img_stride,
                                                        nx_, nz_, nb_, nxpad_, nzpad_, fsz(), c_);
          note_launch();
          std::swap(G0, G2);
        } else {
          // back-propagate the receiver field and image (:394-406)
          step(G0, G1, false, k, st);
          sponge(G0, G1, k, st);
          std::swap(G0, G1);
          k_prtm_cross<<<gmod, kLsZ, 0, st>>>(img, img_stride, G1, S0, nullptr, nz_, nb_, nzpad_, fsz(), 0);
          note_launch();
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
      // Born modelling (:410-434)
      for (int it = 0; it < nt_; it++) {
        k_prtm_cross<<<gmod, kLsZ, 0, st>>>(nullptr, 0, G1, S0, mod, nz_, nb_, nzpad_, fsz(), 1);
        note_launch();
        std::swap(G0, G1);
        sponge(G0, G1, k, st);
        step(G0, G1, true, k, st);
        receivers(G1, d, it, true, k, st);
        source(S1, it, +1, k, st);
        step(S0, S1, false, k, st);
        sponge(S0, S1, k, st);
        std::swap(S0, S1);
      }
    }
    g_swapped_ = G0 != gp0_.get();
  }

  int arith_, nz_, nx_, nb_, nt_, ns_, ng_, nzpad_ = 0, nxpad_ = 0;
  int kmax_ = 1, adj_mode_ = SWFWI_PRTM_ADJ_REFERENCE;
  bool serial_rec_ = false, g_swapped_ = false;
  PrtmCoef c_{};
  std::vector<int> spos_h_, rpos_h_;
  DevBuf<float> vv_, wlt_, sponge_, sp0_, sp1_, gp0_, gp1_, gp2_, ring_, img_;
  DevBuf<int> spos_, rpos_;
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
