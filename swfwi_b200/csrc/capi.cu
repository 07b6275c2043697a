// extern "C" entry points of include/swfwi_gpu.h.
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include "framework.hpp"
#include "precond.hpp"

namespace swfwi {
thread_local std::string g_last_error;
void set_last_error(const std::string &m) { g_last_error = m; }
std::string last_error() { return g_last_error; }
}  // namespace swfwi

using namespace swfwi;

// The handle: the propagator, and the device buffers and copy stream of the
// host-buffer gradient (kept between calls, grown on demand).
struct swfwi_damp4t10d {
  std::unique_ptr<Propagator> p;
  DevBuf<float> hv, hw, hd, hg;
  cudaStream_t copy = nullptr;
  cudaEvent_t copied = nullptr;
  ~swfwi_damp4t10d() {
    if (copied) cudaEventDestroy(copied);
    if (copy) cudaStreamDestroy(copy);
  }
};

struct swfwi_fwi {
  std::unique_ptr<FwiRunner> r;
};

struct swfwi_precond {
  std::unique_ptr<Preconditioner> n;
};

namespace {
cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// After asynchronous launches: surface launch-configuration errors now.
void check_launch() { SWFWI_CUDA(cudaGetLastError()); }

Propagator &P(swfwi_damp4t10d *h) {
  if (!h || !h->p) throw Error(SWFWI_ERR_BAD_ARG, "null propagator handle");
  return *h->p;
}
const Propagator &P(const swfwi_damp4t10d *h) {
  if (!h || !h->p) throw Error(SWFWI_ERR_BAD_ARG, "null propagator handle");
  return *h->p;
}
void need_velocity(Propagator &p) {
  if (!p.velocity()) throw Error(SWFWI_ERR_STATE, "no velocity bound");
}
FwiRunner &R(swfwi_fwi *h) {
  if (!h || !h->r) throw Error(SWFWI_ERR_BAD_ARG, "null framework handle");
  return *h->r;
}
const FwiRunner &R(const swfwi_fwi *h) {
  if (!h || !h->r) throw Error(SWFWI_ERR_BAD_ARG, "null framework handle");
  return *h->r;
}

Preconditioner &NET(swfwi_precond *h, void *stream) {
  if (!h || !h->n) throw Error(SWFWI_ERR_BAD_ARG, "null preconditioner handle");
  h->n->set_stream(as_stream(stream));
  return *h->n;
}

StepArgs drop_in_args(float *prev, const float *curr, const float *vel, int nx, int nz, int nb,
                      long long stride) {
  StepArgs a;
  a.prev = prev;
  a.curr = curr;
  a.vel = vel;
  a.nx = nx;
  a.nz = nz;
  a.pitch = nz;
  a.bx0 = nb;
  a.shot_stride = stride;
  a.vel_stride = 0;
  a.shots_per_vel = 1;
  return a;
}
}  // namespace

extern "C" {

const char *swfwi_status_string(int s) {
  switch (s) {
    case SWFWI_OK: return "ok";
    case SWFWI_ERR_BAD_ARG: return "bad argument";
    case SWFWI_ERR_OOM: return "out of memory";
    case SWFWI_ERR_TIMEOUT: return "timeout";
    case SWFWI_ERR_NONFINITE: return "non-finite value";
    case SWFWI_ERR_CUDA: return "CUDA error";
    case SWFWI_ERR_STATE: return "wrong state";
    default: return "unknown status";
  }
}

const char *swfwi_last_error(void) { return swfwi::g_last_error.c_str(); }

int swfwi_version(void) { return 1; }

// ---------------------------------------------------------------- drop-in
int swfwi_fd4t10s_damp_zjh_2d_vtrans(float *prev, const float *curr, const float *vel, float *u2,
                                     int nx, int nz, int nb, void *stream) {
  (void)u2;
  return guarded([&] {
    SWFWI_REQUIRE(prev && curr && vel, "null field");
    SWFWI_REQUIRE(nx > 12 && nz > 12 && nb >= 1, "grid too small");
    launch_step(ARITH_REF, true, false, 32, drop_in_args(prev, curr, vel, nx, nz, nb, 0), 1,
                as_stream(stream));
    check_launch();
  });
}

int swfwi_fd4t10s_zjh_2d_vtrans(float *prev, const float *curr, const float *vel, float *u2, int nx,
                                int nz, void *stream) {
  (void)u2;
  return guarded([&] {
    SWFWI_REQUIRE(prev && curr && vel, "null field");
    SWFWI_REQUIRE(nx > 12 && nz > 12, "grid too small");
    launch_step(ARITH_REF, false, false, 32, drop_in_args(prev, curr, vel, nx, nz, 1, 0), 1,
                as_stream(stream));
    check_launch();
  });
}

int swfwi_fd4t10s_step_batch(float *prev, const float *curr, const float *vel, int nx, int nz,
                             int nb, int damped, int arith, int nshots, long long shot_stride,
                             void *stream) {
  return guarded([&] {
    SWFWI_REQUIRE(prev && curr && vel, "null field");
    SWFWI_REQUIRE(nx > 12 && nz > 12 && nb >= 1 && nshots >= 1, "bad sizes");
    SWFWI_REQUIRE(arith == SWFWI_ARITH_REF || arith == SWFWI_ARITH_FAST, "arith must be REF or FAST");
    SWFWI_REQUIRE(nshots == 1 || shot_stride >= (long long)nx * nz, "shot stride too small");
    StepArgs a = drop_in_args(prev, curr, vel, nx, nz, nb, shot_stride);
    a.shots_per_vel = nshots;
    launch_step(arith, damped != 0, false, 32, a, nshots, as_stream(stream));
    check_launch();
  });
}

int swfwi_fd4t10s_step_f64(double *prev, const double *curr, const double *vel, int nx, int nz,
                           int nb, int damped, void *stream) {
  return guarded([&] {
    SWFWI_REQUIRE(prev && curr && vel, "null field");
    SWFWI_REQUIRE(nx > 12 && nz > 12 && nb >= 1, "grid too small");
    StepArgs a;
    a.prev = prev;
    a.curr = curr;
    a.vel = vel;
    a.nx = nx;
    a.nz = nz;
    a.pitch = nz;
    a.bx0 = nb;
    a.shot_stride = 0;
    a.vel_stride = 0;
    a.shots_per_vel = 1;
    launch_step(ARITH_F64, damped != 0, false, 32, a, 1, as_stream(stream));
    check_launch();
  });
}

// ---------------------------------------------------------------- Damp4t10d
int swfwi_damp4t10d_create(swfwi_damp4t10d **out, const swfwi_shot_position *src,
                           const swfwi_shot_position *geo, float dt, float dx, float fm, int nb,
                           int nt) {
  return guarded([&] {
    SWFWI_REQUIRE(out && src && geo, "null argument");
    *out = nullptr;
    SWFWI_REQUIRE(src->ns > 0 && geo->ns > 0, "empty source or receiver line");
    Line s{src->szbeg, src->sxbeg, src->jsz, src->jsx, src->ns};
    Line g{geo->szbeg, geo->sxbeg, geo->jsz, geo->jsx, geo->ns};
    std::unique_ptr<swfwi_damp4t10d> h(new swfwi_damp4t10d);
    h->p.reset(new Propagator(s, g, dt, dx, fm, nb, nt));
    *out = h.release();
  });
}

int swfwi_damp4t10d_destroy(swfwi_damp4t10d *h) {
  return guarded([&] { delete h; });
}

int swfwi_damp4t10d_set_stream(swfwi_damp4t10d *h, void *stream) {
  return guarded([&] { P(h).set_stream(as_stream(stream)); });
}

int swfwi_damp4t10d_set_arith(swfwi_damp4t10d *h, int arith) {
  return guarded([&] {
    SWFWI_REQUIRE(arith == SWFWI_ARITH_REF || arith == SWFWI_ARITH_FAST, "arith must be REF or FAST");
    P(h).arith = arith;
  });
}

int swfwi_damp4t10d_set_strip_format(swfwi_damp4t10d *h, int format) {
  return guarded([&] {
    SWFWI_REQUIRE(format == SWFWI_STRIP_F32 || format == SWFWI_STRIP_F16 || format == SWFWI_STRIP_BF16,
                  "strip format must be SWFWI_STRIP_F32, _F16 or _BF16");
    P(h).strip_format = format;
  });
}

int swfwi_damp4t10d_set_reconstruction(swfwi_damp4t10d *h, int mode, int every, int format) {
  return guarded([&] {
    SWFWI_REQUIRE(mode == SWFWI_RECON_STRIPS || mode == SWFWI_RECON_SNAPSHOTS,
                  "reconstruction must be SWFWI_RECON_STRIPS or _SNAPSHOTS");
    SWFWI_REQUIRE(every >= 2, "snapshot interval must be at least 2 steps");
    SWFWI_REQUIRE(format == SWFWI_STRIP_F32 || format == SWFWI_STRIP_F16 || format == SWFWI_STRIP_BF16,
                  "snapshot format must be SWFWI_STRIP_F32, _F16 or _BF16");
    P(h).recon = mode;
    P(h).snap_every = every;
    P(h).snap_format = format;
  });
}

int swfwi_damp4t10d_set_fusion(swfwi_damp4t10d *h, int on) {
  return guarded([&] { P(h).fuse = on != 0; });
}

int swfwi_damp4t10d_set_graphs(swfwi_damp4t10d *h, int on) {
  return guarded([&] {
    SWFWI_REQUIRE(on >= 0 && on <= 2, "graph mode must be 0, 1 or 2");
    P(h).graphs = on;
  });
}

int swfwi_damp4t10d_set_tuning(swfwi_damp4t10d *h, int kernel, int band_depth, int rows_per_cta,
                               int rows_in_flight, int shots_slowest) {
  return guarded([&] {
    SWFWI_REQUIRE(kernel == 1 || kernel == 5 || kernel == 6, "kernel must be 1, 5 or 6");
    if (kernel == 5 || kernel == 6) {
      SWFWI_REQUIRE(band_depth == 120, "band depth must be 120 (one warp a task)");
    } else {
      SWFWI_REQUIRE(band_depth == 120 || band_depth == 248 || band_depth == 376,
                    "band depth must be 120, 248 or 376");
    }
    SWFWI_REQUIRE(rows_in_flight == 3 || rows_in_flight == 7, "rows in flight must be 3 or 7");
    SWFWI_REQUIRE(rows_per_cta >= 0, "rows per CTA must be 0 (automatic) or positive");
    P(h).stream_kernel = kernel;
    P(h).stream_bz = band_depth;
    P(h).stream_xchunk = rows_per_cta;
    P(h).stream_depth = rows_in_flight;
    P(h).stream_shot_major = shots_slowest ? 1 : 0;
  });
}

int swfwi_damp4t10d_set_receivers_per_shot(swfwi_damp4t10d *h, const int *offsets, const int *gx,
                                           const int *gz) {
  return guarded([&] { P(h).set_receivers_per_shot(offsets, gx, gz); });
}

int swfwi_damp4t10d_dims(const swfwi_damp4t10d *h, int *nxpad, int *nzpad, int *ns, int *ng,
                         int *nt) {
  return guarded([&] {
    const Propagator &p = P(h);
    if (nxpad) *nxpad = p.nxpad;
    if (nzpad) *nzpad = p.nzpad;
    if (ns) *ns = p.ns;
    if (ng) *ng = p.ngmax;
    if (nt) *nt = p.nt;
  });
}

int swfwi_damp4t10d_expand_domain(swfwi_damp4t10d *h, const float *vel, int nx, int nz,
                                  float *exvel) {
  return guarded([&] {
    Propagator &p = P(h);
    SWFWI_REQUIRE(vel && exvel, "null array");
    SWFWI_REQUIRE(nx > 0 && nz > 0, "bad model size");
    p.set_dims(nx + 2 * p.nb + 12, nz + p.nb + 12);
    p.expand_domain(vel, exvel);
  });
}

int swfwi_damp4t10d_set_model_size(swfwi_damp4t10d *h, int nx, int nz) {
  return guarded([&] {
    Propagator &p = P(h);
    SWFWI_REQUIRE(nx > 0 && nz > 0, "bad model size");
    p.set_dims(nx + 2 * p.nb + 12, nz + p.nb + 12);
  });
}

int swfwi_damp4t10d_bind_velocity(swfwi_damp4t10d *h, const float *exvel) {
  return guarded([&] {
    Propagator &p = P(h);
    SWFWI_REQUIRE(p.nxpad > 0, "model size unknown: call swfwi_damp4t10d_set_model_size first");
    p.bind_velocity(exvel);
  });
}

int swfwi_damp4t10d_step_forward(swfwi_damp4t10d *h, float *p0, float *p1) {
  return guarded([&] {
    need_velocity(P(h));
    P(h).step_forward(p0, p1);
    check_launch();
  });
}

int swfwi_damp4t10d_step_backward(swfwi_damp4t10d *h, float *p0, float *p1) {
  return guarded([&] {
    need_velocity(P(h));
    P(h).step_backward(p0, p1);
    check_launch();
  });
}

int swfwi_damp4t10d_add_source(swfwi_damp4t10d *h, float *p, const float *source, int shot_id) {
  return guarded([&] {
    P(h).manip_source(p, source, shot_id, +1);
    check_launch();
  });
}

int swfwi_damp4t10d_sub_source(swfwi_damp4t10d *h, float *p, const float *source, int shot_id) {
  return guarded([&] {
    P(h).manip_source(p, source, shot_id, -1);
    check_launch();
  });
}

int swfwi_damp4t10d_add_receiver_source(swfwi_damp4t10d *h, float *p, const float *vsrc_it) {
  return guarded([&] {
    P(h).add_receiver_source(p, vsrc_it);
    check_launch();
  });
}

int swfwi_damp4t10d_record_seis(swfwi_damp4t10d *h, float *seis_it, const float *p) {
  return guarded([&] {
    P(h).record_seis(seis_it, p);
    check_launch();
  });
}

int swfwi_damp4t10d_bndry_size(const swfwi_damp4t10d *h, int *size) {
  return guarded([&] {
    SWFWI_REQUIRE(size, "null output");
    SWFWI_REQUIRE(P(h).nxpad > 0, "model size unknown");
    *size = P(h).bsize;
  });
}

int swfwi_damp4t10d_write_bndry(swfwi_damp4t10d *h, float *bndr, const float *p, int it) {
  return guarded([&] {
    SWFWI_REQUIRE(it < P(h).nt, "time index out of range");
    P(h).write_bndry(bndr, p, it);
    check_launch();
  });
}

int swfwi_damp4t10d_read_bndry(swfwi_damp4t10d *h, const float *bndr, float *p, int it) {
  return guarded([&] {
    SWFWI_REQUIRE(it < P(h).nt, "time index out of range");
    P(h).read_bndry(bndr, p, it);
    check_launch();
  });
}

int swfwi_damp4t10d_mask_gradient(swfwi_damp4t10d *h, float *g) {
  return guarded([&] { P(h).mask_gradient(g); check_launch(); });
}

int swfwi_damp4t10d_scale_gradient(swfwi_damp4t10d *h, float *g) {
  return guarded([&] { P(h).scale_gradient(g); check_launch(); });
}

int swfwi_damp4t10d_refill_boundary(swfwi_damp4t10d *h, float *v) {
  return guarded([&] { P(h).refill_boundary(v); check_launch(); });
}

int swfwi_damp4t10d_remove_direct_arrival(swfwi_damp4t10d *h, float *data, int shot_id) {
  return guarded([&] {
    need_velocity(P(h));
    P(h).remove_direct_arrival(data, shot_id);
    check_launch();
  });
}

int swfwi_damp4t10d_fwi_forward_modeling(swfwi_damp4t10d *h, const float *wlt, float *dcal,
                                         int shot_id) {
  return guarded([&] {
    need_velocity(P(h));
    P(h).fwi_forward(wlt, dcal, shot_id);
    check_launch();
  });
}

int swfwi_damp4t10d_ess_forward_modeling(swfwi_damp4t10d *h, const float *encsrc, float *dcal) {
  return guarded([&] {
    need_velocity(P(h));
    P(h).ess_forward(encsrc, dcal);
    check_launch();
  });
}

int swfwi_encode_source(float *encsrc, const float *wlt, const int *codes, int nt, int ns, void *stream) {
  return guarded([&] {
    SWFWI_REQUIRE(encsrc && wlt && codes && nt > 0 && ns > 0, "bad encoder arguments");
    launch_encode_source(encsrc, wlt, codes, nt, ns, reinterpret_cast<cudaStream_t>(stream));
    check_launch();
  });
}

int swfwi_encode_obs(float *encobs, const float *dobs, const int *codes, long long n_per_shot, int ns,
                     void *stream) {
  return guarded([&] {
    SWFWI_REQUIRE(encobs && dobs && codes && n_per_shot > 0 && ns > 0, "bad encoder arguments");
    launch_encode_obs(encobs, dobs, codes, n_per_shot, ns, reinterpret_cast<cudaStream_t>(stream));
    check_launch();
  });
}

int swfwi_damp4t10d_ess_forward_members(swfwi_damp4t10d *h, const float *encsrc, const float *vels,
                                        int n, float *hona) {
  return guarded([&] {
    P(h).ess_forward_members(encsrc, vels, n, hona);
    check_launch();
  });
}

int swfwi_damp4t10d_forward_batch(swfwi_damp4t10d *h, const float *wlt, float *dcal,
                                  const int *shot_ids, int nshots) {
  return guarded([&] {
    need_velocity(P(h));
    P(h).forward_batch(wlt, dcal, shot_ids, nshots);
    check_launch();
  });
}

int swfwi_damp4t10d_gradient_batch(swfwi_damp4t10d *h, const float *wlt, const float *dobs,
                                   const int *shot_ids, int nshots, float *grad, double *obj) {
  return guarded([&] {
    need_velocity(P(h));
    P(h).gradient_batch(wlt, dobs, shot_ids, nshots, grad, obj);
    check_launch();
  });
}

int swfwi_gradient_host(swfwi_damp4t10d *h, const float *exvel, const float *wlt, const float *dobs,
                        const int *shot_ids, int nshots, float *grad, double *obj) {
  return guarded([&] {
    Propagator &p = P(h);
    SWFWI_REQUIRE(exvel && wlt && dobs && shot_ids && grad && nshots > 0, "null argument");
    SWFWI_REQUIRE(p.nxpad > 0, "model size unknown");
    cudaStream_t st = p.stream();
    long long np = (long long)p.nxpad * p.nzpad, dn = (long long)p.nt * p.ngmax;
    // the host data hold only the listed shots: address them as 0..n-1
    std::vector<int> local(nshots);
    for (int i = 0; i < nshots; i++) {
      SWFWI_REQUIRE(shot_ids[i] >= 0 && shot_ids[i] < p.ns, "shot id out of range");
      local[i] = i;
    }
    if (!h->copy) {
      SWFWI_CUDA(cudaStreamCreateWithFlags(&h->copy, cudaStreamNonBlocking));
      SWFWI_CUDA(cudaEventCreateWithFlags(&h->copied, cudaEventDisableTiming));
    }
    h->hv.upload(exvel, np, st);
    h->hw.upload(wlt, p.nt, st);
    h->hd.resize((size_t)nshots * dn);
    h->hg.resize(np);
    // the observed data are first read by the residual, after the forward
    // sweep: upload them on the copy stream meanwhile
    const size_t dbytes = sizeof(float) * (size_t)nshots * dn;
    std::function<void()> upload = [&] {
      SWFWI_CUDA(cudaStreamWaitEvent(h->copy, h->copied, 0));   // the previous call's reads are done
      SWFWI_CUDA(cudaMemcpyAsync(h->hd.get(), dobs, dbytes, cudaMemcpyHostToDevice, h->copy));
      SWFWI_CUDA(cudaEventRecord(h->copied, h->copy));
      SWFWI_CUDA(cudaStreamWaitEvent(st, h->copied, 0));
    };
    const float *old = p.velocity();
    p.bind_velocity(h->hv.get());
    // slot i models shot_ids[i]; its observed data sit at row i
    p.gradient_batch(h->hw.get(), h->hd.get(), shot_ids, nshots, h->hg.get(), obj, false, local.data(),
                     &upload);
    SWFWI_CUDA(cudaEventRecord(h->copied, st));
    SWFWI_CUDA(cudaMemcpyAsync(grad, h->hg.get(), sizeof(float) * np, cudaMemcpyDeviceToHost, st));
    SWFWI_CUDA(cudaStreamSynchronize(st));
    if (old) p.bind_velocity(old);
    else p.unbind_velocity(h->hv.get());
  });
}

int swfwi_damp4t10d_calgradient_ess(swfwi_damp4t10d *h, const float *encsrc, const float *vsrc,
                                    float *grad) {
  return guarded([&] {
    need_velocity(P(h));
    P(h).calgradient_ess(encsrc, vsrc, grad);
    check_launch();
  });
}

int swfwi_damp4t10d_calgradient_fwi(swfwi_damp4t10d *h, const float *wlt, const float *vsrc,
                                    float *grad, int shot_id) {
  return guarded([&] {
    need_velocity(P(h));
    P(h).calgradient_fwi(wlt, vsrc, grad, shot_id);
    check_launch();
  });
}

int swfwi_damp4t10d_calgradient_fwi_f64(swfwi_damp4t10d *h, const float *vel, const double *wlt,
                                        const double *vsrc, double *grad, int shot_id) {
  return guarded([&] {
    SWFWI_REQUIRE(P(h).nxpad > 0, "model size unknown");
    P(h).calgradient_fwi_f64(vel, wlt, vsrc, grad, shot_id);
  });
}

int swfwi_damp4t10d_calgradient_ess_f64(swfwi_damp4t10d *h, const float *vel, const double *encsrc,
                                        const double *vsrc, double *grad) {
  return guarded([&] {
    SWFWI_REQUIRE(P(h).nxpad > 0, "model size unknown");
    P(h).calgradient_ess_f64(vel, encsrc, vsrc, grad);
  });
}

int swfwi_damp4t10d_fwi_forward_modeling_f64(swfwi_damp4t10d *h, const float *vel,
                                             const double *wlt, double *dcal, int shot_id) {
  return guarded([&] {
    SWFWI_REQUIRE(P(h).nxpad > 0, "model size unknown");
    P(h).fwi_forward_f64(vel, wlt, dcal, shot_id);
  });
}

// ---------------------------------------------------------------- per-iteration
int swfwi_update_grad(float *pre, const float *cur, float *dir, int n, int iter, void *stream) {
  return guarded([&] {
    SWFWI_REQUIRE(pre && cur && dir && n > 0, "bad arguments");
    cudaStream_t st = as_stream(stream);
    if (iter == 0) {
      launch_cg_update(dir, pre, cur, 0.0f, n, 1, st);
    } else {
      DevBuf<double> s(3 + 3 * 256);
      launch_cg_dots(s.get(), cur, pre, n, s.get() + 3, st);
      double d[3];
      SWFWI_CUDA(cudaMemcpyAsync(d, s.get(), sizeof(d), cudaMemcpyDeviceToHost, st));
      SWFWI_CUDA(cudaStreamSynchronize(st));
      float beta = (float)((d[0] - d[1]) / d[2]);
      if (beta < 0.0f) beta = 0.0f;
      launch_cg_update(dir, pre, cur, beta, n, 0, st);
    }
    check_launch();
  });
}

int swfwi_cal_max_alpha(const float *vel, const float *grad, int n, float dt, float dx, float maxdv,
                        float *alpha2, float *alpha3, void *stream) {
  return guarded([&] {
    SWFWI_REQUIRE(vel && grad && n > 0 && alpha2 && alpha3, "bad arguments");
    cudaStream_t st = as_stream(stream);
    DevBuf<float> s(1);
    launch_max_alpha(s.get(), vel, grad, n, dt, dx, maxdv, st);
    float a = 0;
    SWFWI_CUDA(cudaMemcpyAsync(&a, s.get(), sizeof(float), cudaMemcpyDeviceToHost, st));
    SWFWI_CUDA(cudaStreamSynchronize(st));
    *alpha2 = a;
    *alpha3 = 2 * a;
  });
}

int swfwi_update_vel(float *new_vel, const float *vel, const float *grad, int n, float steplen,
                     float vmin, float vmax, float dx, float dt, void *stream) {
  return guarded([&] {
    SWFWI_REQUIRE(new_vel && vel && grad && n > 0, "bad arguments");
    float tmin = (dx / dt / vmax) * (dx / dt / vmax);
    float tmax = (dx / dt / vmin) * (dx / dt / vmin);
    SWFWI_REQUIRE(tmax > tmin, "vmax must exceed vmin");
    launch_update_vel(new_vel, vel, grad, n, steplen, tmin, tmax, as_stream(stream));
    check_launch();
  });
}

int swfwi_trans_vsrc(float *out, const float *in, int nt, int ng, void *stream) {
  return guarded([&] {
    SWFWI_REQUIRE(out && in && nt > 0 && ng > 0 && out != in, "bad arguments");
    launch_trans_vsrc(out, in, nt, ng, 1, as_stream(stream));
    check_launch();
  });
}

int swfwi_cal_objective(const float *r, long long n, double *obj, void *stream) {
  return guarded([&] {
    SWFWI_REQUIRE(r && n > 0 && obj, "bad arguments");
    cudaStream_t st = as_stream(stream);
    DevBuf<double> s(1 + 256);
    launch_sumsq_f64(s.get(), r, n, 1, s.get() + 1, 256, st);
    SWFWI_CUDA(cudaMemcpyAsync(obj, s.get(), sizeof(double), cudaMemcpyDeviceToHost, st));
    SWFWI_CUDA(cudaStreamSynchronize(st));
  });
}

int swfwi_parabola_vertex(float x1, float y1, float x2, float y2, float x3, float y3,
                          float max_alpha3, float *xv, float *yv) {
  return guarded([&] {
    SWFWI_REQUIRE(xv && yv, "null output");
    parabola_vertex(x1, y1, x2, y2, x3, y3, max_alpha3, *xv, *yv);
  });
}

// rickerWavelet (ricker-wavelet.cpp:15-31): tmp = pi*fm*(it*dt - 1/fm) in
// double stored as float, squared in float, amp*(1-2 tmp)*exp(-tmp) in
// double.
int swfwi_ricker_wavelet(float *wlt, int nt, float fm, float dt, float amp) {
  return guarded([&] {
    SWFWI_REQUIRE(wlt && nt > 0 && fm > 0, "bad arguments");
    for (int it = 0; it < nt; it++) {
      float tmp = (float)(M_PI * fm * (it * dt - 1.0 / fm));
      tmp *= tmp;
      wlt[it] = (float)(amp * (1.0 - 2.0 * tmp) * std::exp(-tmp));
    }
  });
}

int swfwi_random_codes(int seed, int skip, int n, int *codes) {
  return guarded([&] {
    SWFWI_REQUIRE(codes && n > 0 && skip >= 0, "bad arguments");
    RandomCodes rc(seed);
    for (int i = 0; i < skip; i++) rc.gen_plus1_minus1(n);
    std::vector<int> c = rc.gen_plus1_minus1(n);
    std::memcpy(codes, c.data(), sizeof(int) * n);
  });
}

// ---------------------------------------------------------------- frameworks
int swfwi_fwi_create(swfwi_fwi **out, swfwi_damp4t10d *method, const float *exvel, float vmin,
                     float vmax, int nita, float maxdv, const float *wlt, const float *dobs,
                     int encoded) {
  return guarded([&] {
    SWFWI_REQUIRE(out, "null output");
    *out = nullptr;
    std::unique_ptr<swfwi_fwi> h(new swfwi_fwi);
    h->r.reset(new FwiRunner(P(method), exvel, vmin, vmax, nita, maxdv, wlt, dobs, encoded != 0));
    *out = h.release();
  });
}

int swfwi_fwi_destroy(swfwi_fwi *h) {
  return guarded([&] { delete h; });
}

int swfwi_fwi_epoch(swfwi_fwi *h, int iter) {
  return guarded([&] {
    SWFWI_REQUIRE(iter >= 0, "negative iteration");
    R(h).epoch(iter);
  });
}

int swfwi_fwi_get_update_obj(const swfwi_fwi *h, float *obj) {
  return guarded([&] { SWFWI_REQUIRE(obj, "null output"); *obj = R(h).update_obj; });
}

int swfwi_fwi_get_init_obj(const swfwi_fwi *h, float *obj) {
  return guarded([&] { SWFWI_REQUIRE(obj, "null output"); *obj = R(h).init_obj; });
}

int swfwi_fwi_get_velocity(swfwi_fwi *h, float *exvel) {
  return guarded([&] { SWFWI_REQUIRE(exvel, "null output"); R(h).get_velocity(exvel); });
}

int swfwi_fwi_set_velocity(swfwi_fwi *h, const float *exvel) {
  return guarded([&] { SWFWI_REQUIRE(exvel, "null input"); R(h).set_velocity(exvel); });
}

int swfwi_fwi_write_vel(swfwi_fwi *h, float *vel) {
  return guarded([&] { SWFWI_REQUIRE(vel, "null output"); R(h).write_vel(vel); });
}

int swfwi_stats_reset(void) {
  return guarded([&] { step_timer().reset(); });
}

int swfwi_stats_enable_step_timing(int on) {
  return guarded([&] {
    SWFWI_REQUIRE(on >= 0, "timing period must be >= 0");
    step_timer().period.store(on > 0 ? on : 1);
    step_timer().enabled.store(on != 0);
  });
}

int swfwi_stats_read(swfwi_stats *out) {
  return guarded([&] {
    SWFWI_REQUIRE(out, "null output");
    double ms = 0, pts = 0, b = 0;
    long long n = 0, timed = 0;
    step_timer().read(ms, n, pts, b, timed);
    out->kernel_launches = g_kernel_launches.load();
    out->step_launches = n;
    out->step_ms = ms;
    out->step_point_updates = pts;
    out->step_bytes = b;
    out->step_timed_launches = timed;
  });
}

int swfwi_fwi_last_trials(const swfwi_fwi *h, int *trials) {
  return guarded([&] {
    SWFWI_REQUIRE(trials, "null output");
    *trials = R(h).search.trials;
  });
}

int swfwi_fwi_last_line_search(const swfwi_fwi *h, float *alpha, float *obj) {
  return guarded([&] {
    SWFWI_REQUIRE(alpha && obj, "null output");
    for (int i = 0; i < 4; i++) {
      alpha[i] = R(h).search.alpha[i];
      obj[i] = R(h).search.obj[i];
    }
  });
}

// ------------------------------------------------------- learned preconditioner
int swfwi_precond_create(swfwi_precond **out, const int *widths) {
  return guarded([&] {
    SWFWI_REQUIRE(out, "null output");
    *out = nullptr;
    const int def[4] = {16, 32, 64, 64};
    std::unique_ptr<swfwi_precond> h(new swfwi_precond);
    h->n.reset(new Preconditioner(widths ? widths : def));
    *out = h.release();
  });
}

int swfwi_precond_destroy(swfwi_precond *h) {
  return guarded([&] { delete h; });
}

int swfwi_precond_num_params(const swfwi_precond *h, long long *n) {
  return guarded([&] {
    SWFWI_REQUIRE(h && h->n && n, "null argument");
    *n = h->n->num_params();
  });
}

int swfwi_precond_layer(const swfwi_precond *h, int l, int *cin, int *cout, long long *w_off,
                        long long *b_off) {
  return guarded([&] {
    SWFWI_REQUIRE(h && h->n && cin && cout && w_off && b_off, "null argument");
    SWFWI_REQUIRE(l >= 0 && l <= Preconditioner::kConvs, "layer out of range");
    if (l < Preconditioner::kConvs) {
      const ConvSpec &c = h->n->convs()[l];
      *cin = c.cin; *cout = c.cout; *w_off = c.w_off; *b_off = c.b_off;
    } else {
      *cin = h->n->convs()[Preconditioner::kConvs - 1].cout; *cout = 1;
      *w_off = h->n->out_w_off(); *b_off = h->n->out_b_off();
    }
  });
}

int swfwi_precond_set_params(swfwi_precond *h, const float *params) {
  return guarded([&] { NET(h, nullptr).set_params(params); });
}

int swfwi_precond_get_params(swfwi_precond *h, float *params) {
  return guarded([&] { SWFWI_REQUIRE(params, "null output"); NET(h, nullptr).get_params(params); });
}

int swfwi_precond_get_grads(swfwi_precond *h, float *grads) {
  return guarded([&] { SWFWI_REQUIRE(grads, "null output"); NET(h, nullptr).get_grads(grads); });
}

int swfwi_precond_forward(swfwi_precond *h, const float *x, float *y, int n, int H, int W,
                          void *stream) {
  return guarded([&] {
    NET(h, stream).forward(x, y, n, H, W);
    check_launch();
  });
}

int swfwi_precond_backward(swfwi_precond *h, const float *t, double *loss, void *stream) {
  return guarded([&] {
    const double l = NET(h, stream).backward(t);
    if (loss) *loss = l;
  });
}

int swfwi_precond_adam_step(swfwi_precond *h, float lr, void *stream) {
  return guarded([&] {
    SWFWI_REQUIRE(lr > 0 && std::isfinite(lr), "bad learning rate");
    NET(h, stream).adam_step(lr);
    check_launch();
  });
}

int swfwi_precond_train_step(swfwi_precond *h, const float *x, const float *t, int n, int H, int W,
                             float lr, double *loss, void *stream) {
  return guarded([&] {
    SWFWI_REQUIRE(lr > 0 && std::isfinite(lr), "bad learning rate");
    const double l = NET(h, stream).train_step(x, t, n, H, W, lr);
    if (loss) *loss = l;
  });
}

int swfwi_precond_features(swfwi_precond *h, const swfwi_damp4t10d *method, const float *grad,
                           const float *vel, const float *illum, float *x3, void *stream) {
  return guarded([&] {
    const Propagator &p = P(method);
    NET(h, stream).features(grad, vel, illum, p.nxpad, p.nzpad, p.bx0, p.bxn, p.bz0, p.bzn, x3);
    check_launch();
  });
}

int swfwi_precond_target(swfwi_precond *h, const swfwi_damp4t10d *method, const float *dv, float *t,
                         void *stream) {
  return guarded([&] {
    const Propagator &p = P(method);
    NET(h, stream).target(dv, p.nxpad, p.nzpad, p.bx0, p.bxn, p.bz0, p.bzn, t);
    check_launch();
  });
}

int swfwi_precond_propose(swfwi_precond *h, const swfwi_damp4t10d *method, const float *grad,
                          const float *vel, const float *illum, float *dir, void *stream) {
  return guarded([&] {
    const Propagator &p = P(method);
    NET(h, stream).propose(grad, vel, illum, p.nxpad, p.nzpad, p.bx0, p.bxn, p.bz0, p.bzn, dir);
    check_launch();
  });
}

int swfwi_fwi_set_preconditioner(swfwi_fwi *h, swfwi_precond *net) {
  return guarded([&] {
    FwiRunner &r = R(h);
    SWFWI_REQUIRE(!net || net->n, "null preconditioner handle");
    r.set_preconditioner(net ? net->n.get() : nullptr);
  });
}

int swfwi_fwi_set_learned_min_decrease(swfwi_fwi *h, float frac) {
  return guarded([&] {
    SWFWI_REQUIRE(frac >= 0.0f && frac < 1.0f, "fraction must be in [0, 1)");
    R(h).learned_min_decrease = frac;
  });
}

int swfwi_fwi_set_learned_patience(swfwi_fwi *h, int rejections) {
  return guarded([&] {
    SWFWI_REQUIRE(rejections >= 0, "negative patience");
    R(h).learned_patience = rejections;
  });
}

int swfwi_fwi_set_regularization(swfwi_fwi *h, float lx, float lz) {
  return guarded([&] { R(h).set_regularization(lx, lz); });
}

int swfwi_regu_term(const float *vel, int nx, int nz, float lx, float lz, double *term, void *stream) {
  return guarded([&] {
    SWFWI_REQUIRE(vel && term && nx > 0 && nz > 0, "bad regularisation arguments");
    DevBuf<double> sc(regu_scratch_doubles());
    launch_regu_term(vel, nx, nz, lx, lz, sc.get(), as_stream(stream));
    check_launch();
    double h[3];
    SWFWI_CUDA(cudaMemcpyAsync(h, sc.get(), sizeof(h), cudaMemcpyDeviceToHost, as_stream(stream)));
    SWFWI_CUDA(cudaStreamSynchronize(as_stream(stream)));
    *term = h[2];
  });
}

int swfwi_regu_gradient(const float *vel, int nx, int nz, float lx, float lz, float *grad, int accumulate,
                        void *stream) {
  return guarded([&] {
    SWFWI_REQUIRE(vel && grad && nx > 0 && nz > 0, "bad regularisation arguments");
    launch_regu_grad(vel, nx, nz, lx, lz, grad, accumulate != 0, as_stream(stream));
    check_launch();
  });
}

int swfwi_fwi_collect_illumination(swfwi_fwi *h, int on) {
  return guarded([&] { R(h).set_collect_illumination(on != 0); });
}

int swfwi_fwi_get_gradient(swfwi_fwi *h, float *grad) {
  return guarded([&] { SWFWI_REQUIRE(grad, "null output"); R(h).get_gradient(grad); });
}

int swfwi_fwi_get_illumination(swfwi_fwi *h, float *illum) {
  return guarded([&] { SWFWI_REQUIRE(illum, "null output"); R(h).get_illumination(illum); });
}

int swfwi_fwi_learned_stats(const swfwi_fwi *h, int *last, int *tried, int *accepted) {
  return guarded([&] {
    SWFWI_REQUIRE(last && tried && accepted, "null output");
    const FwiRunner &r = R(h);
    *last = r.last_step_learned; *tried = r.learned_tried; *accepted = r.learned_accepted;
  });
}

}  // extern "C"
