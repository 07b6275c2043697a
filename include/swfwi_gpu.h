/*
 * swfwi_gpu.h - C ABI of the B200 (sm_100a) implementation of swfwi's 2D
 * acoustic FWI path.
 *
 * Conventions (the reference's, kept so callers can switch):
 *  - Grids are x-major with z contiguous: p[ix*nzpad + iz].
 *  - nxpad = nx + 2*nb + 12, nzpad = nz + nb + 12 (free surface on top,
 *    nb sponge cells left/right/bottom, a 6-cell stencil halo all round).
 *  - Velocities handed to the propagator are padded and transformed,
 *    vt = dx^2 / (v^2 dt^2).
 *  - Seismic data are time-major per shot: d[it*ng + ig]; a set of shots is
 *    [shot][it][ig].
 *  - Field, data and velocity pointers are DEVICE pointers unless a function
 *    says "host"; scalar outputs are host pointers.
 *  - Every entry point returns a status (SWFWI_OK = 0).  swfwi_last_error()
 *    gives the text of the last failure on the calling thread.
 *  - Calls on one handle are ordered on that handle's CUDA stream
 *    (swfwi_damp4t10d_set_stream; a new handle uses the legacy default
 *    stream 0); functions that return host values synchronise that stream.
 */
#ifndef SWFWI_GPU_H
#define SWFWI_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
  SWFWI_OK = 0,
  SWFWI_ERR_BAD_ARG = 1,   /* invalid size, index or pointer */
  SWFWI_ERR_OOM = 2,       /* device or host allocation failed */
  SWFWI_ERR_TIMEOUT = 3,   /* a bounded device wait gave up */
  SWFWI_ERR_NONFINITE = 4, /* NaN/Inf found where a finite value is required */
  SWFWI_ERR_CUDA = 5,      /* CUDA runtime error */
  SWFWI_ERR_STATE = 6      /* call made in the wrong state (e.g. no velocity bound) */
};

/* Arithmetic of the stencil.
 *  REF : float fields, every operation rounded exactly as the reference's C
 *        source is on x86-64 (bit-identical results).
 *  FAST: float fields, FP32 with fused multiply-add (tolerance parity).
 *  F64 : the same scheme in double, used as the FP64 oracle. */
enum { SWFWI_ARITH_REF = 0, SWFWI_ARITH_FAST = 1, SWFWI_ARITH_F64 = 2 };

/* Storage of the boundary strips used to rebuild the source wavefield
 * backwards.  F32 is exact; F16/BF16 keep one scale per strip and step. */
enum { SWFWI_STRIP_F32 = 0, SWFWI_STRIP_F16 = 1, SWFWI_STRIP_BF16 = 2 };

/* How a gradient's backward sweep obtains the source wavefield. */
enum { SWFWI_RECON_STRIPS = 0, SWFWI_RECON_SNAPSHOTS = 1 };

const char *swfwi_status_string(int status);
const char *swfwi_last_error(void);
int swfwi_version(void);

/* ------------------------------------------------------------------------
 * Drop-in stencil steps.  Same arguments and in-place semantics as the
 * reference kernels, on device memory, plus a CUDA stream (NULL = default
 * stream).  nx, nz are padded sizes, vel is transformed, nb is the damping
 * ramp length (the reference passes Damp4t10d::bx0 = sponge + 6).  prev is
 * overwritten on [6, nx-6) x [6, nz-6) with the next field; u2 is accepted
 * for signature compatibility and not touched (the Laplacian stays on chip),
 * so it may be NULL.  REF arithmetic: bit-identical to the reference.
 * ---------------------------------------------------------------------- */

/* replaces fd4t10s_damp_zjh_2d_vtrans, src/modeling/fd4t10s-damp-zjh.h:11 */
int swfwi_fd4t10s_damp_zjh_2d_vtrans(float *prev, const float *curr, const float *vel, float *u2,
                                     int nx, int nz, int nb, void *stream);
/* replaces fd4t10s_zjh_2d_vtrans, src/modeling/fd4t10s-zjh.h:11 */
int swfwi_fd4t10s_zjh_2d_vtrans(float *prev, const float *curr, const float *vel, float *u2, int nx,
                                int nz, void *stream);
/* Either step with a chosen arithmetic (REF or FAST) and nshots fields
 * laid out shot_stride floats apart sharing one velocity (batched form of
 * the two functions above; same per-field semantics). */
int swfwi_fd4t10s_step_batch(float *prev, const float *curr, const float *vel, int nx, int nz,
                             int nb, int damped, int arith, int nshots, long long shot_stride,
                             void *stream);
/* FP64 oracle step (double fields and velocity). */
int swfwi_fd4t10s_step_f64(double *prev, const double *curr, const double *vel, int nx, int nz,
                           int nb, int damped, void *stream);

/* ------------------------------------------------------------------------
 * ShotPosition (src/common/shot-position.h:13-27): a regular line of
 * points, point i at z = szbeg + i*jsz, x = sxbeg + i*jsx (unpadded grid
 * indices).  nz is the unpadded model depth, as in the reference.
 * ---------------------------------------------------------------------- */
typedef struct {
  int szbeg, sxbeg, jsz, jsx, ns, nz;
} swfwi_shot_position;

/* ------------------------------------------------------------------------
 * Damp4t10d (src/modeling/damp4t10d.h:18-87): the propagator object.
 * ---------------------------------------------------------------------- */
typedef struct swfwi_damp4t10d swfwi_damp4t10d;

/* Damp4t10d::Damp4t10d (damp4t10d.cpp:367-376). */
int swfwi_damp4t10d_create(swfwi_damp4t10d **out, const swfwi_shot_position *src,
                           const swfwi_shot_position *geo, float dt, float dx, float fm, int nb,
                           int nt);
int swfwi_damp4t10d_destroy(swfwi_damp4t10d *h);
/* Order this handle's work on a caller stream (cudaStream_t); NULL is the
 * legacy default stream. */
int swfwi_damp4t10d_set_stream(swfwi_damp4t10d *h, void *stream);
int swfwi_damp4t10d_set_arith(swfwi_damp4t10d *h, int arith);
/* Storage of the boundary strips the batched gradients save in the forward
 * sweep and restore in the backward one (SWFWI_STRIP_F32 = the reference's
 * writeBndry/readBndry, bit-exact; F16/BF16 = half the memory, one
 * power-of-two scale per shot and step).  The single-field
 * write_bndry/read_bndry calls always use FP32. */
int swfwi_damp4t10d_set_strip_format(swfwi_damp4t10d *h, int format);
/* Reconstruction of the source wavefield in the gradients' backward sweep.
 * SWFWI_RECON_STRIPS (default): back-propagation with the saved boundary
 * strips, the reference's calgradient (fwiframework.cpp:146-176).
 * SWFWI_RECON_SNAPSHOTS (checkpointing; no counterpart in the reference):
 * the forward sweep saves both wavefields every `every` steps (every >= 2)
 * in `format` (SWFWI_STRIP_F32 = exact; F16/BF16 = one power-of-two scale
 * per field, shot and snapshot); the backward sweep re-runs each segment of
 * `every` steps forward from its snapshot into a ring of every + 1 fields
 * and images with the forward field itself.  With F32 snapshots the imaged
 * source field is the forward's own, bit for bit; the strips' rounding in
 * the back-propagation is gone, so results differ from the reference's
 * within the FP32 gradient tolerance.  Memory per shot: (every + 1) fields
 * plus 2 fields (F32) or 1 field (16-bit) per snapshot. */
int swfwi_damp4t10d_set_reconstruction(swfwi_damp4t10d *h, int mode, int every, int format);
/* Launch shape of the propagator's stencil (results do not depend on it):
 * kernel 6 (default) = two-row register-queue streaming step, one warp a
 * task of 120 output depths x rows_per_cta rows, each warp its own TMA
 * pipeline two rows a stage, two stages ahead (band depth 120; rows in
 * flight accepted but fixed at 4); FAST arithmetic, REF runs kernel 5;
 * kernel 5 = register-queue streaming step, one row a stage (band depth
 * 120, rows ahead 3 or 7); kernel 1 = warp-specialised
 * streaming step (band depth 120, 248 or 376 = 1-3 consumer warps plus a
 * copy warp, rows ahead 3 or 7; the fused time loop always uses it);
 * rows per CTA >= 1, or 0 (default): kernels 5 and 6 take the longest
 * task (at least 8 rows) with which every (shot, depth slice) column's
 * tasks fit in one wave of resident warps, kernel 1 takes 64;
 * shots_slowest = 1 runs the CTAs of one
 * shot together (kernel 1). */
int swfwi_damp4t10d_set_tuning(swfwi_damp4t10d *h, int kernel, int band_depth, int rows_per_cta,
                               int rows_in_flight, int shots_slowest);
/* Fused backward time loop (default off): where sources and receivers form
 * horizontal lines (or single points) and the fields are FP32, the source
 * back-step also subtracts the source and images, and the receiver step
 * also injects the next residual (warp-specialised kernel, 376-deep bands),
 * in place of the separate source, residual and image launches.  Results
 * are bit-identical either way. */
int swfwi_damp4t10d_set_fusion(swfwi_damp4t10d *h, int on);
/* CUDA graphs for the forward and backward time loops: on = 0 never, 1
 * (default) while a step covers at most 8e6 points (fields x nxpad x
 * nzpad), from a loop's second use; 2 for every step size, from its first
 * use.  The loop is captured on a private stream and replayed on the
 * propagator's stream (one graph per loop and setting, stencil timing
 * included).  Same kernels, same results. */
int swfwi_damp4t10d_set_graphs(swfwi_damp4t10d *h, int on);
/* Per-shot receiver lists (uneven spreads; not in the reference, whose
 * ShotPosition is one common line): shot s has receivers
 * [offsets[s], offsets[s+1]) of gx/gz (unpadded, host arrays).  The
 * common line set at creation stays the one the single-shot calls use. */
int swfwi_damp4t10d_set_receivers_per_shot(swfwi_damp4t10d *h, const int *offsets, const int *gx,
                                           const int *gz);
int swfwi_damp4t10d_dims(const swfwi_damp4t10d *h, int *nxpad, int *nzpad, int *ns, int *ng,
                         int *nt);
/* Damp4t10d::expandDomain (damp4t10d.cpp:138-151).  Host arrays:
 * vel [nx][nz] in m/s -> exvel [nxpad][nzpad] transformed.  Also fixes the
 * grid size of the handle (as binding the expanded Velocity does). */
int swfwi_damp4t10d_expand_domain(swfwi_damp4t10d *h, const float *vel, int nx, int nz,
                                  float *exvel);
/* Fix the grid size without expanding (for a velocity expanded
 * elsewhere): nx, nz unpadded. */
int swfwi_damp4t10d_set_model_size(swfwi_damp4t10d *h, int nx, int nz);
/* Damp4t10d::bindVelocity (damp4t10d.cpp:159-161): the padded transformed
 * velocity, device; kept by pointer as the reference keeps a reference.
 * Re-bind after changing it in place. */
int swfwi_damp4t10d_bind_velocity(swfwi_damp4t10d *h, const float *exvel);
/* stepForward (damp4t10d.cpp:153-157): damped step, p0 <- F(p0, p1). */
int swfwi_damp4t10d_step_forward(swfwi_damp4t10d *h, float *p0, float *p1);
/* stepBackward (damp4t10d.cpp:188-191): undamped step. */
int swfwi_damp4t10d_step_backward(swfwi_damp4t10d *h, float *p0, float *p1);
/* addSource/subSource for one shot (curSrcPos = allSrcPos.clip(shot));
 * shot_id = -1: every source, source[is] (addEncodedSource /
 * subEncodedSource, damp4t10d.cpp:193-214, 378-384).  source is device. */
int swfwi_damp4t10d_add_source(swfwi_damp4t10d *h, float *p, const float *source, int shot_id);
int swfwi_damp4t10d_sub_source(swfwi_damp4t10d *h, float *p, const float *source, int shot_id);
/* addSource(p, vsrc_it, allGeoPos): inject one value per receiver. */
int swfwi_damp4t10d_add_receiver_source(swfwi_damp4t10d *h, float *p, const float *vsrc_it);
/* recordSeis (damp4t10d.cpp:163-180, 386-388). */
int swfwi_damp4t10d_record_seis(swfwi_damp4t10d *h, float *seis_it, const float *p);
/* initBndryVector/writeBndry/readBndry (damp4t10d.cpp:447-536): FP32
 * strips, reference layout, bndr holds nt * size floats. */
int swfwi_damp4t10d_bndry_size(const swfwi_damp4t10d *h, int *size);
int swfwi_damp4t10d_write_bndry(swfwi_damp4t10d *h, float *bndr, const float *p, int it);
int swfwi_damp4t10d_read_bndry(swfwi_damp4t10d *h, const float *bndr, float *p, int it);
/* maskGradient :216-226, scaleGradient :309-319, refillBoundary :228-252 */
int swfwi_damp4t10d_mask_gradient(swfwi_damp4t10d *h, float *grad);
int swfwi_damp4t10d_scale_gradient(swfwi_damp4t10d *h, float *grad);
int swfwi_damp4t10d_refill_boundary(swfwi_damp4t10d *h, float *vel);
/* fwiRemoveDirectArrival (shot_id >= 0) / removeDirectArrival (shot_id =
 * -1), damp4t10d.cpp:321-365, 390-394: data [nt][ng] in place. */
int swfwi_damp4t10d_remove_direct_arrival(swfwi_damp4t10d *h, float *data, int shot_id);
/* FwiForwardModeling (damp4t10d.cpp:272-289): wlt [nt] -> dcal [nt][ng]. */
int swfwi_damp4t10d_fwi_forward_modeling(swfwi_damp4t10d *h, const float *wlt, float *dcal,
                                         int shot_id);
/* EssForwardModeling (damp4t10d.cpp:291-307): encsrc [nt][ns]. */
int swfwi_damp4t10d_ess_forward_modeling(swfwi_damp4t10d *h, const float *encsrc, float *dcal);
/* The HA loop of EnkfAnalyze::calGainMatrix (enkfanalyze.cpp:207-236):
 * EssForwardModeling of the encoded supershot (encsrc [nt][ns]) with each of
 * n member velocities vels [n][nxpad*nzpad] (padded, transformed), run as
 * one batch; hona [n][ng*nt] receives each seismogram transposed to the
 * analysis matrix's column order (row ig*nt + it, matrix_transpose).  All
 * device pointers. */
int swfwi_damp4t10d_ess_forward_members(swfwi_damp4t10d *h, const float *encsrc, const float *vels,
                                        int n, float *hona);

/* ------------------------------------------------------------------------
 * Batched whole-shot operations (the fast path): nshots shots of
 * shot_ids[] (host) run as one set of launches per time step.
 * ---------------------------------------------------------------------- */
/* FwiForwardModeling for every listed shot: dcal [nshots][nt][ng]. */
int swfwi_damp4t10d_forward_batch(swfwi_damp4t10d *h, const float *wlt, float *dcal,
                                  const int *shot_ids, int nshots);
/* The per-shot gradient loop of FwiFramework::epoch (fwiframework.cpp:
 * 274-324) for the listed shots: forward modelling, direct-arrival mute of
 * observed and modelled data, residual, objective, time derivative,
 * calgradient (:114-177), scaleGradient, maskGradient, and the sum over
 * shots in list order.  dobs [ns][nt][ng] (device, all shots), grad
 * [nxpad][nzpad] (device, overwritten), obj [nshots] (host, FP64 sums of
 * squared residuals). */
int swfwi_damp4t10d_gradient_batch(swfwi_damp4t10d *h, const float *wlt, const float *dobs,
                                   const int *shot_ids, int nshots, float *grad, double *obj);
/* Same from HOST buffers (copies in and out inside the call): exvel
 * [nxpad][nzpad], wlt [nt], dobs [nshots][nt][ng] for the listed shots,
 * grad [nxpad][nzpad]. */
int swfwi_gradient_host(swfwi_damp4t10d *h, const float *exvel, const float *wlt,
                        const float *dobs, const int *shot_ids, int nshots, float *grad,
                        double *obj);
/* Encoded-source gradient (essfwiframework.cpp:114-173) on device:
 * encsrc [nt][ns], vsrc [nt][ng]; grad accumulates (not scaled). */
int swfwi_damp4t10d_calgradient_ess(swfwi_damp4t10d *h, const float *encsrc, const float *vsrc,
                                    float *grad);
/* Plain per-shot gradient (fwiframework.cpp:114-177) on device; grad
 * accumulates (not scaled). */
int swfwi_damp4t10d_calgradient_fwi(swfwi_damp4t10d *h, const float *wlt, const float *vsrc,
                                    float *grad, int shot_id);
/* FP64 oracle run of the per-shot gradient scheme (double fields, exact
 * strips): vel is the float transformed velocity (device), wlt/vsrc/grad are
 * double (device); grad accumulates. */
int swfwi_damp4t10d_calgradient_fwi_f64(swfwi_damp4t10d *h, const float *vel, const double *wlt,
                                        const double *vsrc, double *grad, int shot_id);
/* FP64 run of the encoded-source gradient scheme (essfwiframework.cpp:
 * 114-173; double fields, exact strips): vel float transformed velocity,
 * encsrc [nt][ns], vsrc [nt][ng] and grad double (device); grad
 * accumulates. */
int swfwi_damp4t10d_calgradient_ess_f64(swfwi_damp4t10d *h, const float *vel, const double *encsrc,
                                        const double *vsrc, double *grad);
/* FP64 forward modelling of one shot (double dcal, device). */
int swfwi_damp4t10d_fwi_forward_modeling_f64(swfwi_damp4t10d *h, const float *vel,
                                             const double *wlt, double *dcal, int shot_id);

/* ------------------------------------------------------------------------
 * Per-iteration arithmetic (device arrays of n = nxpad*nzpad floats).
 * ---------------------------------------------------------------------- */
/* updateGrad (fwiframework.cpp:42-72): PR+ conjugate gradient; the dot
 * products are accumulated in FP64.  pre, dir updated in place. */
int swfwi_update_grad(float *pre_gradient, const float *cur_gradient, float *update_direction,
                      int n, int iter, void *stream);
/* calMaxAlpha2_3 (updatesteplenop.cpp:25-47). */
int swfwi_cal_max_alpha(const float *vel, const float *grad, int n, float dt, float dx, float maxdv,
                        float *alpha2, float *alpha3, void *stream);
/* UpdateVelOp::update (updatevelop.cpp:11-37), vmin/vmax in m/s. */
int swfwi_update_vel(float *new_vel, const float *vel, const float *grad, int n, float steplen,
                     float vmin, float vmax, float dx, float dt, void *stream);
/* second_order_virtual_source_forth_accuracy over [nt][ng] (transVsrc,
 * fwiframework.cpp:75-105), out of place. */
int swfwi_trans_vsrc(float *out, const float *in, int nt, int ng, void *stream);
/* sum of squares of n floats in FP64 (cal_objective, common.cpp:231-241). */
int swfwi_cal_objective(const float *r, long long n, double *obj, void *stream);
/* The sum of squares above for nslots consecutive arrays of n_per_slot
 * floats, written to obj[0..nslots) (DEVICE), without allocating: no
 * counterpart in the reference.  For callers that cannot call cudaMalloc
 * (allocation forbidden inside their callbacks or owned by their own
 * allocator).  Scratch is a static device array of 32 slots x 256 FP64
 * partials (64 KB, held by every GPU that loads the library); nslots > 32
 * is rejected.  The first call on a device looks up that array's address
 * and should come before any stream capture; calls that overlap on the GPU
 * race on the array.  Same results as swfwi_cal_objective per slot. */
int swfwi_cal_objective_static(const float *r, long long n_per_slot, int nslots, double *obj,
                               void *stream);
/* parabolaVertex (parabola-vertex.cpp:12-33), host. */
int swfwi_parabola_vertex(float x1, float y1, float x2, float y2, float x3, float y3,
                          float max_alpha3, float *xv, float *yv);
/* rickerWavelet (ricker-wavelet.cpp:15-31), host. */
int swfwi_ricker_wavelet(float *wlt, int nt, float fm, float dt, float amp);
/* RandomCodes::genPlus1Minus1 (random-code.cpp:2-22): +-1 codes of a
 * minstd_rand stream with the given seed, after skip earlier batches of
 * n codes.  Host. */
int swfwi_random_codes(int seed, int skip, int n, int *codes);

/* ------------------------------------------------------------------------
 * FwiFramework / EssFwiFramework (src/fwi/fwiframework.h:16-53,
 * src/essfwi/essfwiframework.h:16-53) with their step-length and velocity
 * update operators.  encoded = 0: plain FWI over all shots; 1: one
 * +-1-encoded supershot per epoch.  wlt [nt], dobs [ns][nt][ng]: host.
 * ---------------------------------------------------------------------- */
typedef struct swfwi_fwi swfwi_fwi;
int swfwi_fwi_create(swfwi_fwi **out, swfwi_damp4t10d *method, const float *exvel, float vmin,
                     float vmax, int nita, float maxdv, const float *wlt, const float *dobs,
                     int encoded);
/* Destroy a framework before the propagator it was created on. */
int swfwi_fwi_destroy(swfwi_fwi *h);
int swfwi_fwi_epoch(swfwi_fwi *h, int iter);
int swfwi_fwi_get_update_obj(const swfwi_fwi *h, float *obj);
int swfwi_fwi_get_init_obj(const swfwi_fwi *h, float *obj);
/* current padded transformed velocity, host [nxpad][nzpad] */
int swfwi_fwi_get_velocity(swfwi_fwi *h, float *exvel);
/* Replace the framework's velocity (host [nxpad][nzpad], transformed): an
 * EnKF analysis moving the member, as the reference's analysis writes the
 * members' Velocity objects in place (enkfanalyze.cpp:72-108). */
int swfwi_fwi_set_velocity(swfwi_fwi *h, const float *exvel);
/* sfWriteVel (damp4t10d.cpp:254-265) without the file: interior velocity in
 * m/s, host [nx][nz]. */
int swfwi_fwi_write_vel(swfwi_fwi *h, float *vel);
/* EssFwiRegu (src/unused/essfwiregu.cpp:667-776) on an encoded framework:
 * every objective adds lx Wx2 + lz Wz2 of the padded transformed model
 * (ReguFactor, src/unused/ReguFactor.cpp), the gradient adds the factor's
 * gradient before the mask and is not depth-scaled, and the step is taken
 * along the gradient itself.  lx = lz = 0 (default) is the plain encoded
 * epoch. */
int swfwi_fwi_set_regularization(swfwi_fwi *h, float lx, float lz);
/* ReguFactor on a DEVICE model vel [nx][nz]: term (host, FP64 sums of the
 * float squares; the reference sums in float) and the gradient written, or
 * added when accumulate = 1, into grad (DEVICE) exactly as the reference's
 * loops leave it.  Synchronises. */
int swfwi_regu_term(const float *vel, int nx, int nz, float lx, float lz, double *term, void *stream);
int swfwi_regu_gradient(const float *vel, int nx, int nz, float lx, float lz, float *grad, int accumulate,
                        void *stream);

/* ------------------------------------------------------------------------
 * The prestack LSRTM linear operator (src/unused/prtm2d.cpp; the reference
 * never built it: its prtm2d.h is missing).  One handle is one prtm2d_init
 * (:241-338): second-order-time, fourth-order-space propagator with a
 * Gaussian sponge of nb cells on every side, Ricker source of peak
 * frequency fm and amplitude amp, shots at (sxbeg + is jsx, szbeg + is jsz),
 * receivers at (gxbeg + ig jgx, gzbeg + ig jgz), moved with each shot when
 * csdgather = 1 (common-shot gathers).  vel: DEVICE [nx][nz] in m/s.  Every
 * shot and receiver must lie in the model (the reference checks the first
 * and last and exits; here SWFWI_ERR_BAD_ARG).
 * arith SWFWI_ARITH_REF: bit-identical to the compiled prtm2d.cpp, shots
 * in order, the receiver-side fields carried between shots and calls as
 * the reference's Born branch leaves them (it never clears them, :408-434).
 * SWFWI_ARITH_FAST: FP32 with FMA, shots batched, every shot from zero.
 * ---------------------------------------------------------------------- */
typedef struct swfwi_prtm swfwi_prtm;
/* migration: the reference's (:371-407; not the adjoint of its Born
 * branch: <Lm, d> != <m, L'd>), or the exact transpose of the Born branch */
enum { SWFWI_PRTM_ADJ_REFERENCE = 0, SWFWI_PRTM_ADJ_EXACT = 1 };
int swfwi_prtm2d_create(swfwi_prtm **out, int arith, float dz, float dx, float dt, float amp, float fm, int nz,
                        int nx, int nb, int nt, int ns, int ng, int sxbeg, int szbeg, int jsx, int jsz, int gxbeg,
                        int gzbeg, int jgx, int jgz, int csdgather, const float *vel, void *stream);
int swfwi_prtm2d_set_adjoint(swfwi_prtm *h, int mode);
/* on = 1 (default): a call that repeats an earlier call's arrays, direction
 * and adjoint mode replays its time loops as one CUDA graph (captured on
 * the second such call); 0: every call launches its kernels one by one. */
int swfwi_prtm2d_set_graphs(swfwi_prtm *h, int on);
/* shots one launch sequence carries (1 for REF) */
int swfwi_prtm2d_batch(swfwi_prtm *h, int *shots);
/* prtm2d_lop (:354-437): adj = 0: dat += L mod (Born); adj = 1: mod += L'
 * dat; add = 0 zeroes the output first (sf_adjnull).  nm = nx nz, nd = nt
 * ng ns; mod DEVICE [nx][nz], dat DEVICE [ns][ng][nt].  Asynchronous on
 * stream. */
int swfwi_prtm2d_lop(swfwi_prtm *h, int adj, int add, int nm, int nd, float *mod, float *dat, void *stream);
int swfwi_prtm2d_destroy(swfwi_prtm *h);
/* Failure-detection self-test: one thread waits, with the stencil kernels'
 * bounded mbarrier wait (about 2^31 cycles, a second), on a barrier nothing
 * arrives at; the wait gives up, raises the error flag, and the call returns
 * SWFWI_ERR_TIMEOUT as a stalled stencil launch would.  The context stays
 * usable.  Returns SWFWI_OK only if the wait did not give up (a fault). */
int swfwi_selftest_bounded_wait(void *stream);
/* last epoch's step length and trial record: alpha[4], obj[4] (host) */
int swfwi_fwi_last_line_search(const swfwi_fwi *h, float *alpha, float *obj);
/* Trial objectives the last epoch's step-length search evaluated (each a
 * forward sweep over all shots, or over the supershot; refineAlpha and
 * calsteplen of updatesteplenop.cpp:88-265). */
int swfwi_fwi_last_trials(const swfwi_fwi *h, int *trials);

/* ------------------------------------------------------------------------
 * Measurement (no counterpart in the reference, which prints wall-clock
 * timers only, src/common/timer.h:14-29).  Process-wide counters of kernel
 * launches and, when enabled, every stencil launch's algorithmic work
 * (interior point-updates; bytes = 12 per point-update plus 4 per point per
 * velocity model read) with CUDA-event timing, on the launch's own stream,
 * of every on-th stencil launch (on = 1: all of them).
 * kernel_launches counts kernel launches: a time loop replayed as a CUDA
 * graph (swfwi_damp4t10d_set_graphs) counts the kernels it holds at every
 * replay; its timed stencil launches are bracketed by event nodes in the
 * graph, their times added after each replay completes.
 * step_ms is the timed launches' total: their mean is step_ms /
 * step_timed_launches.
 * ---------------------------------------------------------------------- */
typedef struct {
  long long kernel_launches;
  long long step_launches;
  double step_ms;
  double step_point_updates;
  double step_bytes;
  long long step_timed_launches;
} swfwi_stats;
int swfwi_stats_reset(void);
/* on = 0: off; on >= 1: count every stencil launch, time every on-th. */
int swfwi_stats_enable_step_timing(int on);
/* waits for the timed launches to finish */
int swfwi_stats_read(swfwi_stats *out);

/* Encoder::encodeSource (encoder.cpp:14-26): encsrc[it][is] = wlt[it] *
 * codes[is]; codes are +-1 ints.  Device pointers. */
int swfwi_encode_source(float *encsrc, const float *wlt, const int *codes, int nt, int ns, void *stream);
/* Encoder::encodeObsData (encoder.cpp:28-42): encobs[j] = sum over shots in
 * order of dobs[is][j] * codes[is] (float), j < n_per_shot = nt*ng.  Device. */
int swfwi_encode_obs(float *encobs, const float *dobs, const int *codes, long long n_per_shot, int ns,
                     void *stream);

/* ------------------------------------------------------------------------
 * Ensemble Kalman analysis (src/enfwi/enkfanalyze.cpp), FP64 on the GPU.
 * n = 2..64 members; rows = nt*ng data samples in the reference's matrix
 * order (row ig*nt + it); rows*n < 2^32.
 * ---------------------------------------------------------------------- */
/* EnkfAnalyze::calGainMatrix (enkfanalyze.cpp:185-341), serial form.
 * hona [n][rows] DEVICE float: each member's modelled encoded data;
 * dobs [rows] DEVICE float: the encoded observed data (every column of D);
 * z [n][rows] DEVICE double: standard-normal draws, the observation
 *   perturbation being sigma*z (the reference draws normal(0, sigma) from
 *   Boost mt19937 seed 1); NULL draws them on the device (Philox4x32-10 with
 *   `seed`, Box-Muller);
 * sigma (host, in/out): <= 0 on the first call, then set to max|HA'| *
 *   sigfac as initPerturbation does (enkfanalyze.cpp:621-635); pass it back
 *   unchanged on later calls;
 * t4 (host, out): the n x n gain HA'^T U SSqInv U^T (D - HA), column-major
 *   (t4[col*n + row]) like the reference's Matrix;
 * clip (host, out, optional): clipPosition of the singular values.
 * Everything runs on the device: the three n x n products over the rows in
 * one fused FP64 pass, then the SVD through the n x n cross product
 * band^T band (parallel-ordered Jacobi in FP64 in one CTA), clipPosition
 * and the n x n products.  Synchronises the stream. */
int swfwi_enkf_gain_matrix(const float *hona, const float *dobs, const double *z, long long rows,
                           int n, float sigfac, double *sigma, unsigned long long seed, double *t4,
                           int *clip, void *stream);
/* The update of EnkfAnalyze::analyze (enkfanalyze.cpp:57-111): vels [n]
 * [model_size] DEVICE (padded, transformed members, updated in place):
 * A' = members - their float mean, v_i <- velTrans(velRecover(v_i) +
 * (A' t4)_i).  t4 host, column-major as returned above.  Synchronises. */
int swfwi_enkf_update(float *vels, long long model_size, int n, const double *t4, float dx, float dt,
                      void *stream);
/* The analysis in one call (EnkfAnalyze::analyze after calGainMatrix,
 * enkfanalyze.cpp:57-111 and 185-341): the gain of swfwi_enkf_gain_matrix
 * stays in device memory and moves the members vels [n][model_size]
 * (DEVICE) in place as swfwi_enkf_update does; nothing returns to the host
 * between the two.  sigma as above; t4_out (HOST, optional) receives the
 * gain, column-major; clip (host, optional).  A non-finite gain returns
 * SWFWI_ERR_NONFINITE and leaves the members unchanged.  Synchronises. */
int swfwi_enkf_analyze(const float *hona, const float *dobs, const double *z, long long rows, int n,
                       float sigfac, double *sigma, unsigned long long seed, float *vels,
                       long long model_size, float dx, float dt, double *t4_out, int *clip, void *stream);
/* createAMean (enkfanalyze.cpp:568-580): mean [model_size] DEVICE = the
 * members' float sum in member order / n. */
int swfwi_enkf_mean(float *mean, const float *vels, long long model_size, int n, void *stream);

/* ------------------------------------------------------------------------
 * RSF files (Madagascar format), the I/O of the reference's tools
 * (sf_input / sf_output in src/tool/main-*.cpp; ShotDataReader,
 * shotdata-reader.cpp:54-64).  Host buffers; native float32 data only;
 * header keys are key=value tokens, the last occurrence wins; in="stdin"
 * data embedded after the header are read too.
 * ---------------------------------------------------------------------- */
/* The value of one header key (as text) into value[len]. */
int swfwi_rsf_get(const char *path, const char *key, char *value, int len);
/* Axis lengths n[9] (1 where absent), d[9], o[9] (optional) and the number
 * of axes longer than 1. */
int swfwi_rsf_dims(const char *path, int *ndim, int *n, float *d, float *o);
/* count floats starting at element `first`, axis 1 fastest (a velocity
 * n1=nz, n2=nx reads straight into [nx][nz]). */
int swfwi_rsf_read(const char *path, float *out, long long count, long long first);
/* Header at path, data at data_path (NULL: path + "@"); axes n/d/o (d, o
 * optional); extra: more header lines ("\tkey=value\n"), or NULL. */
int swfwi_rsf_write(const char *path, const char *data_path, const float *data, int ndim, const int *n,
                    const float *d, const float *o, const char *extra);
/* Shots n1=nt, n2=ng, n3=ns on disk ([is][ig][it]) -> dobs [ns][nt][ng]
 * (ShotDataReader::serialRead). */
int swfwi_rsf_read_shots(const char *path, float *dobs, int ns, int nt, int ng);
/* dobs [ns][nt][ng] -> a shot file as main-fm-damp.cpp:144-173 writes it
 * (n1=nt d1=dt, n2=ng d2=dgx, n3=ns, labels and units); extra: the
 * acquisition keys (fm, szbeg, ...) as header lines, or NULL. */
int swfwi_rsf_write_shots(const char *path, const char *data_path, const float *dobs, int ns, int nt, int ng,
                          float dt, float dgx, const char *extra);

/* ------------------------------------------------------------------------
 * Learned preconditioner (no counterpart in the reference; it sits beside
 * the plain epoch of src/fwi/fwiframework.cpp:269-356, whose line search
 * accepts or rejects every step it proposes).  A 4-level convolutional
 * encoder-decoder, widths w[4] (multiples of 16, at most 64; default
 * 16/32/64/64), BF16 weights and activations, FP32 accumulation on the
 * tensor cores, FP32 master weights, Adam.  Images are [n][H][W] with H, W
 * multiples of 8; all tensors below are DEVICE pointers.
 * ---------------------------------------------------------------------- */
typedef struct swfwi_precond swfwi_precond;
/* widths NULL: 16/32/64/64.  Weights start from a fixed seeded He-uniform
 * draw. */
int swfwi_precond_create(swfwi_precond **out, const int *widths);
int swfwi_precond_destroy(swfwi_precond *h);
int swfwi_precond_num_params(const swfwi_precond *h, long long *n);
/* Layer l in 0..13 (3x3 convs, weights [cout][3][3][cin] then bias[cout]),
 * 14 = the 1x1 output layer (weights [cin], bias [1]): offsets in floats
 * into the flat parameter vector. */
int swfwi_precond_layer(const swfwi_precond *h, int l, int *cin, int *cout, long long *w_off,
                        long long *b_off);
/* Flat FP32 parameters / last gradient, host.  set resets Adam. */
int swfwi_precond_set_params(swfwi_precond *h, const float *params);
int swfwi_precond_get_params(swfwi_precond *h, float *params);
int swfwi_precond_get_grads(swfwi_precond *h, float *grads);
/* x [n][H][W][3] -> y [n][H][W] (y may be NULL to keep it internal). */
int swfwi_precond_forward(swfwi_precond *h, const float *x, float *y, int n, int H, int W,
                          void *stream);
/* Mean-square loss of the last forward against t [n][H][W] and the
 * parameter gradient; loss (host) may be NULL. */
int swfwi_precond_backward(swfwi_precond *h, const float *t, double *loss, void *stream);
int swfwi_precond_adam_step(swfwi_precond *h, float lr, void *stream);
/* forward + backward + Adam; loss before the step (host, may be NULL). */
int swfwi_precond_train_step(swfwi_precond *h, const float *x, const float *t, int n, int H, int W,
                             float lr, double *loss, void *stream);
/* Network input of one model: the propagator's interior as an image with
 * H = roundup8(nx) rows (x) and W = roundup8(nz) columns (depth), x3
 * [H][W][3]: gradient / RMS, standardised transformed velocity,
 * (log10(illum / max + 1e-6) + 3) / 3 (illum may be NULL: 0).  grad, vel,
 * illum: [nxpad][nzpad]. */
int swfwi_precond_features(swfwi_precond *h, const swfwi_damp4t10d *method, const float *grad,
                           const float *vel, const float *illum, float *x3, void *stream);
/* Training target: the interior of dv [nxpad][nzpad] at unit RMS, t [H][W]. */
int swfwi_precond_target(swfwi_precond *h, const swfwi_damp4t10d *method, const float *dv, float *t,
                         void *stream);
/* features -> forward -> direction dir [nxpad][nzpad] (zero outside the
 * interior). */
int swfwi_precond_propose(swfwi_precond *h, const swfwi_damp4t10d *method, const float *grad,
                          const float *vel, const float *illum, float *dir, void *stream);

/* Attach a network to a plain (encoded = 0) framework (NULL detaches; the
 * network must outlive its use).  Each epoch then tries the network's
 * direction under its own step-length search first and keeps the step only
 * when the search confirms an objective decrease; otherwise the plain CG
 * step is taken.  Source illumination is accumulated every 4 steps of the
 * gradient's forward sweep while a network is attached or collect is on. */
int swfwi_fwi_set_preconditioner(swfwi_fwi *h, swfwi_precond *net);
/* Keep a learned step only if it lowers the objective by at least this
 * fraction (default 0: any decrease the search confirms); in [0, 1). */
int swfwi_fwi_set_learned_min_decrease(swfwi_fwi *h, float frac);
/* Stop proposing learned steps after this many rejected ones (default 0:
 * never stop). */
int swfwi_fwi_set_learned_patience(swfwi_fwi *h, int rejections);
int swfwi_fwi_collect_illumination(swfwi_fwi *h, int on);
/* The last epoch's gradient / illumination, host [nxpad][nzpad]. */
int swfwi_fwi_get_gradient(swfwi_fwi *h, float *grad);
int swfwi_fwi_get_illumination(swfwi_fwi *h, float *illum);
/* last = 1 if the last epoch took the network's step; counts since create. */
int swfwi_fwi_learned_stats(const swfwi_fwi *h, int *last, int *tried, int *accepted);

#ifdef __cplusplus
}
#endif
#endif /* SWFWI_GPU_H */
