// Device kernels around the stencil: source injection, receiver sampling,
// boundary strips, imaging, and the per-iteration FWI arithmetic.
// Every launcher is a host function taking a cudaStream_t; none allocates.
#pragma once
#include <atomic>
#include <cstdint>
#include <cuda_runtime.h>
#include "stencil.cuh"
#include "stream.cuh"
#include "stream_ws.cuh"

namespace swfwi {

// Kernel launches issued by this library (all launchers count).
extern std::atomic<long long> g_kernel_launches;
// Counts one launch in g_kernel_launches (and in the calling thread's count).
void note_launch();
// The launches the calling thread has counted (a stream capture's own
// launches are the difference over the capture).
long long thread_launches();

// ---- wavefield point operations (batched over shot slots) --------------
// A "slot" is one wavefield in a batch; slot_shot maps it to a shot id
// (NULL = identity).  Positions are padded linear indices x*nzpad + z, -1
// for an unused entry (uneven receiver spreads).
struct PointSet {
  const int *pos;        // [shot][per_shot]
  int per_shot;
  const int *slot_shot;  // [nslots] or NULL
};

// field[slot][pos] += sign * vals[slot*val_slot_stride + i*val_stride]
// (Damp4t10d::manipSource, damp4t10d.cpp:193-214: float add or subtract).
template <typename T>
void launch_inject(T *field, long long shot_stride, int nslots, PointSet ps, const T *vals,
                   long long val_slot_stride, int val_stride, int sign, cudaStream_t st);

// seis[slot*seis_slot_stride + i] = field[slot][pos]  (recordSeis, :163-180)
template <typename T>
void launch_record(T *seis, long long seis_slot_stride, const T *field, long long shot_stride,
                   int nslots, PointSet ps, cudaStream_t st);

// After a forward step, in one launch: seis[slot*seis_slot_stride + i] =
// cur[slot][rec pos] (record; seis NULL: none), the FP32 strips of cur into
// bndr (NULL: none), and next[slot][src pos] += vals (next NULL: none).  The
// same per-element operations as launch_record, launch_strip_write and
// launch_inject, which they replace when cur and next are different fields.
template <typename T>
void launch_after_forward(T *seis, long long seis_slot_stride, const T *cur, PointSet rec, T *bndr,
                          long long bndr_slot_stride, int nx, int nz, int bx0, int pitch, T *next, PointSet src,
                          const T *vals, long long val_slot_stride, int val_stride, long long shot_stride,
                          int nslots, cudaStream_t st);
// Two launch_inject calls on two different fields in one launch; with
// bndr, also the FP32 strip restore (launch_strip_read) of bndr into fa,
// whose strip cells are disjoint from its source cells.
template <typename T>
void launch_inject2(T *fa, PointSet pa, const T *va, long long va_slot_stride, int va_stride, int sign_a, T *fb,
                    PointSet pb, const T *vb, long long vb_slot_stride, int vb_stride, int sign_b,
                    long long shot_stride, int nslots, cudaStream_t st, const T *bndr = nullptr,
                    long long bndr_slot_stride = 0, int nx = 0, int nz = 0, int bx0 = 0, int pitch = 0);

// Boundary strips (writeBndry/readBndry, damp4t10d.cpp:478-536) for all
// slots at one time step.  bndr layout [slot][bndr_slot_stride], one step's
// strip of strip_size(nx,nz,bx0) values at offset it*strip_size.
int strip_size(int nx, int nz, int bx0);
template <typename T>
void launch_strip_write(T *bndr, long long bndr_slot_stride, const T *field, long long shot_stride,
                        int nslots, int nx, int nz, int bx0, int pitch, cudaStream_t st);
template <typename T>
void launch_strip_read(const T *bndr, long long bndr_slot_stride, T *field, long long shot_stride,
                       int nslots, int nx, int nz, int bx0, int pitch, cudaStream_t st);
// The same strips stored as 16-bit values (format SWFWI_STRIP_F16 or
// SWFWI_STRIP_BF16) with one power-of-two scale per slot and step: value =
// decode(q) * scale, scale chosen so the step's largest |value| / scale is
// below 2^14.  q layout as bndr; scale[slot * scale_slot_stride].
void launch_strip_write_q(int format, uint16_t *q, long long q_slot_stride, float *scale,
                          long long scale_slot_stride, const float *field, long long shot_stride,
                          int nslots, int nx, int nz, int bx0, int pitch, cudaStream_t st);
void launch_strip_read_q(int format, const uint16_t *q, long long q_slot_stride, const float *scale,
                         long long scale_slot_stride, float *field, long long shot_stride, int nslots,
                         int nx, int nz, int bx0, int pitch, cudaStream_t st);
// Whole-field checkpoint snapshots in the same 16-bit formats: the first
// `count` values from each slot's field origin, one power-of-two scale per
// slot (the strips' rule); q is [slot][count], scale[slot * scale_slot_stride];
// part_max is scratch of nslots * kSnapParts floats.
constexpr int kSnapParts = 16;
void launch_field_write_q(int format, uint16_t *q, float *scale, long long scale_slot_stride, float *part_max,
                          const float *field, long long shot_stride, long long count, int nslots, cudaStream_t st);
void launch_field_read_q(int format, const uint16_t *q, const float *scale, long long scale_slot_stride,
                         float *field, long long shot_stride, long long count, int nslots, cudaStream_t st);

// image[slot] -= s[slot] * r[slot] * scale  (cross_correlation,
// fwiframework.cpp:107-112)
template <typename T>
void launch_image(T *image, long long image_stride, const T *s, const T *r, long long shot_stride,
                  int nslots, int n, float scale, cudaStream_t st);

// image -= (sum over slots of s[slot] * r[slot]) * scale: all slots'
// cross-correlations into ONE image (FAST arithmetic; the slot terms are
// added in slot order before the scale, so the bits differ from per-slot
// images summed later), over rows [x0, x1) and depths [z0, z1) of the
// pitched fields (depths widened to whole groups of 4; a caller that masks
// the gradient passes the unmasked region).  16-byte aligned arrays, pitch
// and shot_stride.
void launch_image_sum(float *image, const float *s, const float *r, long long shot_stride, int nslots, int x0,
                      int x1, int z0, int z1, int pitch, float scale, cudaStream_t st);

// One FD step for all slots: the shared-memory tile form (any pitch, any
// arithmetic; stencil.cuh).
void launch_step(int arith, bool damped, bool vel_is_rcp, int tx, const StepArgs &a, int nslots,
                 cudaStream_t st);
// Warp-specialised streaming step (stream_ws.cuh): bz = 120, 248 or 376
// output depths per CTA (1-3 consumer warps), depth = 3 or 7 rows ahead;
// the fused epilogues of a.epi run with 376-deep bands.
void launch_ws_step(int arith, bool damped, int bz, int depth, const StreamArgs &a, int nslots,
                    cudaStream_t st);
// Register-queue streaming step (stream_rq.cuh): one self-contained warp
// pipeline (a one-warp CTA) per task of 120 output depths x a.xchunk rows
// of one slot, depth = 3 or 7 stages ahead.
void launch_rq_step(int arith, bool damped, int depth, const StreamArgs &a, int nslots, cudaStream_t st);
// The two-row register-queue step (kernel 6, stream_rq2.cuh): FAST
// arithmetic only; a.xchunk <= 0 takes the one-wave task length.
void launch_rq2_step(bool damped, const StreamArgs &a, int nslots, cudaStream_t st);
// out[s][ig*nt + it] = in[s][it*ng + ig] for nslots seismograms
// (matrix_transpose of common.cpp:14-24 with n1 = ng, n2 = nt).
void launch_transpose_traces(float *out, const float *in, int nt, int ng, int nslots, cudaStream_t st);
// Per-axis sponge ramps for the streaming step (see stream.cuh), and (if
// coef_x is not null) each row's FAST update coefficients of the left/right
// ramp, fast_damp_coef(dist_x[row]).
void launch_damp_tables(float *dist_x, float *dist_z, float2 *coef_x, int nx, int nz, int nb, cudaStream_t st);

// ---- per-iteration arithmetic --------------------------------------------
// Mute windows of removeDirectArrival (damp4t10d.cpp:321-365) for one
// source position and a receiver list: win[2*i] = start, win[2*i+1] = end.
// The velocity mean over rows [min(sz,gz), max(sz,gz)] is summed in float
// in the reference's order by one thread.
// shot = slot_shot ? slot_shot[slot] : slot; source (src_x[shot],
// src_z[shot]); receivers rec_x/rec_z[shot*rec_row_stride + ig], -1 unused.
void launch_mute_windows(int *win, const float *vel, int nxpad, int nzpad, const int *src_x,
                         const int *src_z, const int *rec_x, const int *rec_z,
                         long long rec_row_stride, int ng, const int *slot_shot, int half_len,
                         int nt, int nslots, cudaStream_t st);
// d[slot][it][ig] = 0 for it in [start, end) of trace ig.
void launch_apply_mute(float *d, long long slot_stride, const int *win, int nt, int ng, int nslots,
                       cudaStream_t st);
// Muted residual in one pass: r = mute(obs) - mute(cal) where obs of slot
// s is obs[slot_shot[s]] (NULL: s), win_obs / win_cal are the mute windows
// of each (the same array when both use one velocity).  Zeroing both inside
// the window and subtracting (removeDirectArrival then vectorMinus) gives
// +0 there, as here.
void launch_muted_residual(float *r, const float *obs, long long obs_shot_stride,
                           const int *slot_shot, const float *cal, const int *win_obs,
                           const int *win_cal, int nt, int ng, int nslots, cudaStream_t st);
// r = obs - cal (vectorMinus, common.h:16-19) and its squared sum in FP64,
// per slot: obj[slot] (FP64, one partial per block, then reduced).
void launch_residual(float *r, const float *obs, long long obs_slot_stride, const float *cal,
                     long long n_per_slot, int nslots, cudaStream_t st);
void launch_sumsq_f64(double *out, const float *x, long long n_per_slot, int nslots,
                      double *partials, int partials_per_slot, cudaStream_t st);
// Time second derivative of fwiframework.cpp:75-105 on [slot][nt][ng].
void launch_trans_vsrc(float *out, const float *in, int nt, int ng, int nslots, cudaStream_t st);
// g2 = sum over slots, in slot order, of mask(scale(g[slot]))
// (scaleGradient :309-319, maskGradient :216-226, std::transform plus).
// accumulate = 1 continues a sum already in g2 (shots processed in chunks).
// gs rows have pitch floats; g2 is [nxpad][nzpad].
void launch_finalize_gradient(float *g2, const float *gs, long long g_stride, int nslots, int nxpad,
                              int nzpad, int bx0, int pitch, int accumulate, cudaStream_t st);
// Dot products for PR+ CG in FP64: out[0]=g.g out[1]=g.g0 out[2]=g0.g0
void launch_cg_dots(double *out, const float *g, const float *g0, int n, double *partials,
                    cudaStream_t st);
// d = g + beta*d; g0 = g  (updateGrad, fwiframework.cpp:42-72)
void launch_cg_update(float *d, float *g0, const float *g, float beta, int n, int first,
                      cudaStream_t st);
// calMaxAlpha2_3 (updatesteplenop.cpp:25-47): min over cells, written as an
// order-independent float min.
void launch_max_alpha(float *out_alpha2, const float *vel, const float *grad, int n, float dt,
                      float dx, float maxdv, cudaStream_t st);
// update_vel (updatevelop.cpp:11-21): new = clamp(v + steplen*g, vmin, vmax)
void launch_update_vel(float *newv, const float *v, const float *g, int n, float steplen,
                       float vmin, float vmax, cudaStream_t st);
// refillBoundary (damp4t10d.cpp:228-252)
void launch_refill_boundary(float *v, int nxpad, int nzpad, int bz0, int bzn, int bx0, int bxn,
                            cudaStream_t st);
// 1/vt, correctly rounded (the reference's 1.0f/curvel, computed once),
// from [nx][nz] into rows of pitch floats (padding columns 1).
void launch_reciprocal(float *out, const float *in, long long n, cudaStream_t st);
void launch_pitched_reciprocal(float *out, const float *in, int nx, int nz, int pitch,
                               cudaStream_t st);
void launch_to_f64_reciprocal(double *out, const float *in, int nx, int nz, int pitch,
                              cudaStream_t st);
// Encoder (encoder.cpp:14-42)
void launch_encode_source(float *encsrc, const float *wlt, const int *codes, int nt, int ns,
                          cudaStream_t st);
void launch_encode_obs(float *encobs, const float *dobs, const int *codes, long long n, int ns,
                       cudaStream_t st);
// float <-> double copies for the FP64 path
void launch_f32_to_f64(double *out, const float *in, long long n, cudaStream_t st);
void launch_f64_to_f32(float *out, const double *in, long long n, cudaStream_t st);

// ReguFactor (src/unused/ReguFactor.cpp) on p [nx][nz] (device):
// scratch[0..2] = Wx2, Wz2, lx Wx2 + lz Wz2 in FP64 (scratch holds
// regu_scratch_doubles()); the gradient written (or added) into g.
size_t regu_scratch_doubles();
void launch_regu_term(const float *p, int nx, int nz, float lx, float lz, double *scratch, cudaStream_t st);
void launch_regu_grad(const float *p, int nx, int nz, float lx, float lz, float *g, bool accumulate,
                      cudaStream_t st);

}  // namespace swfwi
