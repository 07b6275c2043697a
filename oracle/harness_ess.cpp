/* Test infrastructure only (the oracle): C entry points over the reference's
 * own ESS-FWI code.  The reference file src/essfwi/essfwiframework.cpp is
 * compiled into this translation unit so that its file-local helpers
 * (updateGrad :42-72, transVsrc :97-105, calgradient :114-173) are callable.
 * Nothing here is shipped or measured as the product. */
#include "essfwiframework.cpp"
#include "ref_common.h"
#include "parabola-vertex.h"

extern "C" {

/* Silence the reference logger (logger.h:120-123 skips output when the
 * terminal stream is NULL), and size the reference's scratch once.
 *
 * Damp4t10d::stepForward/stepBackward keep their u2 scratch in a
 * function-local static vector sized by the FIRST call's grid
 * (damp4t10d.cpp:154, 189); a later call on a larger grid writes past it.
 * One step on a grid larger than any workload here (3200 x 1100 padded
 * points) sizes both statics before anything else runs. */
void ref_quiet(void) {
  Output2FILE::TerminalStream() = NULL;
  static bool sized = false;
  if (sized) return;
  sized = true;
  const int nxp = 3200, nzp = 1100;
  ShotPosition s(0, 0, 0, 1, 1, nzp), g(0, 0, 0, 1, 1, nzp);
  Damp4t10d fm(s, g, 0.001f, 10.0f, 10.0f, 30, 1);
  Velocity v(std::vector<float>((size_t)nxp * nzp, 1.0f), nxp, nzp);
  fm.bindVelocity(v);
  std::vector<float> p0((size_t)nxp * nzp, 0.0f), p1((size_t)nxp * nzp, 0.0f);
  fm.stepForward(&p0[0], &p1[0]);
  fm.stepBackward(&p0[0], &p1[0]);
}

void *ref_model_create(int nz, int nx, int nb, int nt, float dt, float dx, float fm,
                       int szbeg, int sxbeg, int jsz, int jsx, int ns,
                       int gzbeg, int gxbeg, int jgz, int jgx, int ng) {
  ref_quiet();
  return new RefModel(nz, nx, nb, nt, dt, dx, fm, szbeg, sxbeg, jsz, jsx, ns,
                      gzbeg, gxbeg, jgz, jgx, ng);
}

void ref_model_destroy(void *h) { delete static_cast<RefModel *>(h); }

/* Damp4t10d::expandDomain (damp4t10d.cpp:138-151): physical velocity
 * [nx][nz] -> padded transformed velocity [nxpad][nzpad]; also binds it. */
void ref_expand_domain(void *h, const float *vel, float *exvel_out) {
  RefModel *m = static_cast<RefModel *>(h);
  Velocity v0(std::vector<float>(vel, vel + (size_t)m->nx * m->nz), m->nx, m->nz);
  m->exvel = m->fm_method.expandDomain(v0);
  m->fm_method.bindVelocity(m->exvel);
  std::copy(m->exvel.dat.begin(), m->exvel.dat.end(), exvel_out);
}

/* Bind an already padded, transformed velocity. */
void ref_bind_velocity(void *h, const float *exvel) {
  RefModel *m = static_cast<RefModel *>(h);
  std::copy(exvel, exvel + m->exvel.dat.size(), m->exvel.dat.begin());
  m->fm_method.bindVelocity(m->exvel);
}

void ref_get_velocity(void *h, float *exvel_out) {
  RefModel *m = static_cast<RefModel *>(h);
  std::copy(m->exvel.dat.begin(), m->exvel.dat.end(), exvel_out);
}

void ref_fwi_forward(void *h, const float *wlt, float *dcal, int shot_id) {
  RefModel *m = static_cast<RefModel *>(h);
  std::vector<float> w(wlt, wlt + m->nt), d((size_t)m->nt * m->ng, 0.f);
  m->fm_method.FwiForwardModeling(w, d, shot_id);
  std::copy(d.begin(), d.end(), dcal);
}

void ref_ess_forward(void *h, const float *encsrc, float *dcal) {
  RefModel *m = static_cast<RefModel *>(h);
  std::vector<float> w(encsrc, encsrc + (size_t)m->nt * m->ns), d((size_t)m->nt * m->ng, 0.f);
  m->fm_method.EssForwardModeling(w, d);
  std::copy(d.begin(), d.end(), dcal);
}

/* shot_id >= 0: fwiRemoveDirectArrival; shot_id < 0: removeDirectArrival
 * (all sources, source 0's position). */
void ref_remove_direct_arrival(void *h, float *data, int shot_id) {
  RefModel *m = static_cast<RefModel *>(h);
  if (shot_id >= 0) m->fm_method.fwiRemoveDirectArrival(data, shot_id);
  else m->fm_method.removeDirectArrival(data);
}

void ref_trans_vsrc(float *vsrc, int nt, int ng) {
  std::vector<float> v(vsrc, vsrc + (size_t)nt * ng);
  transVsrc(v, nt, ng);
  std::copy(v.begin(), v.end(), vsrc);
}

/* Encoded-source gradient (essfwiframework.cpp:114-173); g accumulates. */
void ref_calgradient_ess(void *h, const float *encsrc, const float *vsrc, float *g) {
  RefModel *m = static_cast<RefModel *>(h);
  std::vector<float> es(encsrc, encsrc + (size_t)m->nt * m->ns);
  std::vector<float> vs(vsrc, vsrc + (size_t)m->nt * m->ng);
  std::vector<float> gg(g, g + m->exvel.dat.size());
  calgradient(m->fm_method, es, vs, gg, m->nt, m->dt);
  std::copy(gg.begin(), gg.end(), g);
}

void ref_scale_gradient(void *h, float *g) { static_cast<RefModel *>(h)->fm_method.scaleGradient(g); }
void ref_mask_gradient(void *h, float *g) { static_cast<RefModel *>(h)->fm_method.maskGradient(g); }
void ref_refill_boundary(void *h, float *v) { static_cast<RefModel *>(h)->fm_method.refillBoundary(v); }

void ref_write_bndry(void *h, float *bndr, const float *p, int it) {
  static_cast<RefModel *>(h)->fm_method.writeBndry(bndr, p, it);
}
void ref_read_bndry(void *h, const float *bndr, float *p, int it) {
  static_cast<RefModel *>(h)->fm_method.readBndry(bndr, p, it);
}
int ref_bndry_size(void *h) {
  RefModel *m = static_cast<RefModel *>(h);
  return (int)(m->fm_method.initBndryVector(1).size());
}
void ref_add_source(void *h, float *p, const float *src, int shot_id) {
  RefModel *m = static_cast<RefModel *>(h);
  if (shot_id >= 0) m->fm_method.addSource(p, src, m->src.clip(shot_id));
  else m->fm_method.addEncodedSource(p, src);
}
void ref_sub_source(void *h, float *p, const float *src, int shot_id) {
  RefModel *m = static_cast<RefModel *>(h);
  if (shot_id >= 0) m->fm_method.subSource(p, src, m->src.clip(shot_id));
  else m->fm_method.subEncodedSource(p, src);
}
void ref_add_receiver_source(void *h, float *p, const float *vsrc_it) {
  RefModel *m = static_cast<RefModel *>(h);
  m->fm_method.addSource(p, vsrc_it, m->geo);
}
void ref_record_seis(void *h, float *seis_it, const float *p) {
  static_cast<RefModel *>(h)->fm_method.recordSeis(seis_it, p);
}
void ref_step_forward(void *h, float *p0, float *p1) { static_cast<RefModel *>(h)->fm_method.stepForward(p0, p1); }
void ref_step_backward(void *h, float *p0, float *p1) { static_cast<RefModel *>(h)->fm_method.stepBackward(p0, p1); }

void ref_update_grad(float *pre, const float *cur, float *dir, int n, int iter) {
  updateGrad(pre, cur, dir, n, iter);
}

float ref_cal_objective(float *r, int n) { return cal_objective(r, n); }

void ref_parabola_vertex(float x1, float y1, float x2, float y2, float x3, float y3,
                         float maxa3, float *xv, float *yv) {
  float a, b;
  parabolaVertex(x1, y1, x2, y2, x3, y3, maxa3, a, b);
  *xv = a;
  *yv = b;
}

void ref_ricker(float *wlt, int nt, float fm, float dt, float amp) { rickerWavelet(wlt, nt, fm, dt, amp); }

/* +-1 codes from the reference's RandomCodes (random-code.cpp:2-22). */
void ref_random_codes(int seed, int n_draws_before, int ns, int *codes) {
  RandomCodes rc(seed);
  for (int i = 0; i < n_draws_before; i++) rc.genPlus1Minus1(ns);
  std::vector<int> c = rc.genPlus1Minus1(ns);
  std::copy(c.begin(), c.end(), codes);
}

/* Whole EssFwiFramework run (essfwiframework.cpp:191-239), niter epochs
 * with the reference's own UpdateSteplenOp/UpdateVelOp.  dobs is
 * [ns][nt][ng].  Outputs: final padded velocity, per-iteration
 * (initobj, updateobj). */
void ref_ess_fwi_run(void *h, const float *wlt, const float *dobs, int niter, int nita,
                     float maxdv, float vmin, float vmax, float *exvel_out, float *objs_out) {
  RefModel *m = static_cast<RefModel *>(h);
  std::vector<float> w(wlt, wlt + m->nt);
  std::vector<float> d(dobs, dobs + (size_t)m->ns * m->nt * m->ng);
  UpdateVelOp uv(vmin, vmax, m->dx, m->dt);
  UpdateSteplenOp us(m->fm_method, uv, nita, maxdv);
  EssFwiFramework ess(m->fm_method, us, uv, w, d);
  for (int it = 0; it < niter; it++) {
    ess.epoch(it);
    objs_out[2 * it] = ess.getInitObj();
    objs_out[2 * it + 1] = ess.getUpdateObj();
  }
  std::copy(m->exvel.dat.begin(), m->exvel.dat.end(), exvel_out);
}

}  /* extern "C" */
