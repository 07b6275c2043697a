/* Test infrastructure only (the oracle): C entry points over the reference's
 * own plain-FWI code.  src/fwi/fwiframework.cpp and
 * src/fwi/fwiupdatesteplenop.cpp are compiled into this translation unit so
 * that their file-local helpers (calgradient :114-177, updateGrad :42-72,
 * calMaxAlpha2_3 :25-47) are callable.
 *
 * The reference's plain-FWI step length is undefined behaviour: its
 * FwiUpdateSteplenOp::refineAlpha is stubbed (fwiupdatesteplenop.cpp:88-217)
 * and leaves obj_val2/obj_val3 uninitialised.  ref_fwi_run therefore follows
 * the reference's working encoded-source line search
 * (src/essfwi/updatesteplenop.cpp:88-265) with the trial objective summed
 * over shots, each shot modelled with its own source.  This is a documented
 * deviation, restated below with citations. */
#include "fwiframework.cpp"
#include "fwiupdatesteplenop.cpp"
#include "ref_common.h"
#include <set>

extern "C" {

/* Plain per-shot gradient (fwiframework.cpp:114-177); g accumulates. */
void ref_calgradient_fwi(void *h, const float *wlt, const float *vsrc, float *g, int shot_id) {
  RefModel *m = static_cast<RefModel *>(h);
  std::vector<float> w(wlt, wlt + m->nt);
  std::vector<float> vs(vsrc, vsrc + (size_t)m->nt * m->ng);
  std::vector<float> gg(g, g + m->exvel.dat.size());
  calgradient(m->fm_method, w, vs, gg, m->nt, m->dt, shot_id);
  std::copy(gg.begin(), gg.end(), g);
}

/* calMaxAlpha2_3 (fwiupdatesteplenop.cpp:25-47). */
void ref_cal_max_alpha(void *h, const float *grad, float maxdv, float *a2, float *a3) {
  RefModel *m = static_cast<RefModel *>(h);
  float x, y;
  calMaxAlpha2_3(m->exvel, grad, m->dt, m->dx, maxdv, x, y);
  *a2 = x;
  *a3 = y;
}

/* FwiUpdateVelOp::update (fwiupdatevelop.cpp:11-37). */
void ref_update_vel(void *h, float *newv, const float *oldv, const float *dir, float steplen,
                    float vmin, float vmax) {
  RefModel *m = static_cast<RefModel *>(h);
  FwiUpdateVelOp op(vmin, vmax, m->dx, m->dt);
  Velocity nv(m->exvel.nx, m->exvel.nz), ov(std::vector<float>(oldv, oldv + m->exvel.dat.size()),
                                            m->exvel.nx, m->exvel.nz);
  std::vector<float> d(dir, dir + m->exvel.dat.size());
  op.update(nv, ov, d, steplen);
  std::copy(nv.dat.begin(), nv.dat.end(), newv);
}

/* The per-shot gradient loop of FwiFramework::epoch (fwiframework.cpp:
 * 270-324), minus its per-shot gradientNN.bin file write.  dobs is
 * [ns][nt][ng].  g2 receives the summed scaled+masked gradient, *obj the
 * summed objective. */
void ref_fwi_gradient(void *h, const float *wlt, const float *dobs, float *g2_out, float *obj_out) {
  RefModel *m = static_cast<RefModel *>(h);
  Damp4t10d &fmMethod = m->fm_method;
  int nt = m->nt, ng = m->ng, ns = m->ns;
  size_t nxz = m->exvel.dat.size();
  std::vector<float> g2(nxz, 0), encsrc(wlt, wlt + nt), encobs((size_t)ng * nt, 0);
  float obj1 = 0.0f;
  for (int is = 0; is < ns; is++) {
    memcpy(&encobs[0], &dobs[(size_t)is * ng * nt], sizeof(float) * ng * nt);
    std::vector<float> dcal((size_t)nt * ng, 0);
    fmMethod.FwiForwardModeling(encsrc, dcal, is);
    fmMethod.fwiRemoveDirectArrival(&encobs[0], is);
    fmMethod.fwiRemoveDirectArrival(&dcal[0], is);
    std::vector<float> vsrc((size_t)nt * ng, 0);
    vectorMinus(encobs, dcal, vsrc);
    obj1 += cal_objective(&vsrc[0], vsrc.size());
    transVsrc(vsrc, nt, ng);
    std::vector<float> g1(nxz, 0);
    calgradient(fmMethod, encsrc, vsrc, g1, nt, m->dt, is);
    fmMethod.scaleGradient(&g1[0]);
    fmMethod.maskGradient(&g1[0]);
    std::transform(g2.begin(), g2.end(), g1.begin(), g2.begin(), std::plus<float>());
  }
  std::copy(g2.begin(), g2.end(), g2_out);
  *obj_out = obj1;
}

}  /* extern "C" */

namespace {
typedef std::pair<float, float> OPt;
/* Same ordering predicate as updatesteplenop.cpp:19-21. */
bool oLess(const OPt &a, const OPt &b) { return a.second - b.second < 1e-10; }

/* Summed trial objective: every shot forward-modelled on the trial velocity
 * v + alpha*d (FwiUpdateVelOp, no boundary refill, as in
 * updatesteplenop.cpp:59-86), its direct arrival muted with the trial
 * velocity, compared with the muted observed shot. */
struct FwiTrial {
  RefModel *m;
  const std::vector<float> *obs_muted;  /* [ns][nt][ng] */
  const std::vector<float> *wlt;
  const std::vector<float> *dir;
  float vmin, vmax;
  float operator()(float alpha) const {
    int nt = m->nt, ng = m->ng;
    FwiUpdateVelOp uv(vmin, vmax, m->dx, m->dt);
    Velocity nv(m->exvel.nx, m->exvel.nz);
    uv.update(nv, m->exvel, *dir, alpha);
    Damp4t10d trial = m->fm_method;
    trial.bindVelocity(nv);
    float sum = 0.0f;
    for (int is = 0; is < m->ns; is++) {
      std::vector<float> dcal((size_t)nt * ng, 0);
      trial.FwiForwardModeling(*wlt, dcal, is);
      trial.fwiRemoveDirectArrival(&dcal[0], is);
      std::vector<float> ob(obs_muted->begin() + (size_t)is * nt * ng,
                            obs_muted->begin() + (size_t)(is + 1) * nt * ng);
      std::vector<float> r((size_t)nt * ng, 0);
      vectorMinus(ob, dcal, r);
      sum += cal_objective(&r[0], r.size());
    }
    return sum;
  }
};

/* UpdateSteplenOp::refineAlpha (updatesteplenop.cpp:88-214), restated with
 * the summed trial objective, including its quirks (the failure branches
 * re-evaluate the objective at the local alpha3 / alpha2). */
bool refineAlphaSum(const FwiTrial &f, float obj_val1, float maxAlpha3, int nita,
                    float &_alpha2, float &_obj_val2, float &_alpha3, float &_obj_val3) {
  float alpha3 = _alpha3, alpha2 = _alpha2;
  float obj_val2 = f(alpha2), obj_val3 = f(alpha3);
  std::set<OPt, bool (*)(const OPt &, const OPt &)> tuned(oLess);
  tuned.insert(std::make_pair(alpha2, obj_val2));
  for (int iter = 0; iter < nita && obj_val2 > obj_val1; iter++) {
    alpha3 = alpha2;
    obj_val3 = obj_val2;
    alpha2 /= 2;
    obj_val2 = f(alpha2);
    tuned.insert(std::make_pair(alpha2, obj_val2));
  }
  if (obj_val2 > obj_val1) {
    _alpha2 = tuned.begin()->first;
    _obj_val2 = tuned.begin()->second;
    _alpha3 = std::min(_alpha2 * 2, maxAlpha3);
    _obj_val3 = f(alpha3);
    return false;
  }
  const float alpha1 = 0;
  float linear = (obj_val2 - obj_val1) / (alpha2 - alpha1) * (alpha3 - alpha1) + obj_val1;
  tuned.clear();
  tuned.insert(std::make_pair(alpha3, obj_val3));
  while (obj_val3 < linear && obj_val3 < obj_val1 && alpha3 < maxAlpha3) {
    alpha2 = alpha3;
    obj_val2 = obj_val3;
    alpha3 = std::min(alpha3 * 2, maxAlpha3);
    obj_val3 = f(alpha3);
    tuned.insert(std::make_pair(alpha3, obj_val3));
  }
  if (alpha3 > maxAlpha3 + 0.1) {
    _alpha3 = tuned.begin()->first;
    _obj_val3 = tuned.begin()->second;
    _alpha2 = _alpha3 / 2;
    _obj_val2 = f(alpha2);
    return false;
  }
  _alpha2 = alpha2;
  _alpha3 = alpha3;
  _obj_val2 = obj_val2;
  _obj_val3 = obj_val3;
  return true;
}
}  // namespace

extern "C" {
/* Plain FWI, niter epochs: gradient loop as FwiFramework::epoch, PR+ CG
 * (updateGrad), then the summed-objective line search above with
 * calsteplen's initialisation and vertex rule (updatesteplenop.cpp:216-285,
 * preserved alpha across epochs), FwiUpdateVelOp and refillBoundary.
 * objs_out[3*it..] = (obj1, steplen, objval of the chosen step). */
void ref_fwi_run(void *h, const float *wlt, const float *dobs, int niter, int nita, float maxdv,
                 float vmin, float vmax, float *exvel_out, float *objs_out) {
  RefModel *m = static_cast<RefModel *>(h);
  Damp4t10d &fmMethod = m->fm_method;
  int nt = m->nt, ng = m->ng, ns = m->ns;
  size_t nxz = m->exvel.dat.size();
  std::vector<float> g0(nxz, 0), dir(nxz, 0), w(wlt, wlt + nt);
  bool pinit = false;
  float palpha = 0;
  for (int iter = 0; iter < niter; iter++) {
    std::vector<float> g2(nxz, 0);
    float obj1 = 0;
    ref_fwi_gradient(h, wlt, dobs, &g2[0], &obj1);
    updateGrad(&g0[0], &g2[0], &dir[0], (int)nxz, iter);
    /* observed shots muted with the current velocity */
    std::vector<float> obsm(dobs, dobs + (size_t)ns * nt * ng);
    for (int is = 0; is < ns; is++) fmMethod.fwiRemoveDirectArrival(&obsm[(size_t)is * nt * ng], is);
    float maxa2, maxa3;
    calMaxAlpha2_3(m->exvel, &dir[0], m->dt, m->dx, maxdv, maxa2, maxa3);
    if (!pinit) { pinit = true; palpha = maxa3; }
    float a3 = palpha < 1.0E-7f ? 1.0E-4f : palpha;
    float a2 = a3 * 0.5;
    float o2, o3;
    FwiTrial f = {m, &obsm, &w, &dir, vmin, vmax};
    bool para = refineAlphaSum(f, obj1, maxa3, nita, a2, o2, a3, o3);
    float a4, o4;
    if (para) {
      parabolaVertex(0, obj1, a2, o2, a3, o3, maxa3, a4, o4);
      if (a4 > maxa3) a4 = maxa3;
    } else {
      a4 = a3;
      o4 = o3;
    }
    palpha = a4;
    FwiUpdateVelOp uv(vmin, vmax, m->dx, m->dt);
    uv.update(m->exvel, m->exvel, dir, a4);
    fmMethod.refillBoundary(&m->exvel.dat[0]);
    objs_out[3 * iter] = obj1;
    objs_out[3 * iter + 1] = a4;
    objs_out[3 * iter + 2] = o4;
  }
  std::copy(m->exvel.dat.begin(), m->exvel.dat.end(), exvel_out);
}

/* Stubs for the RSF writers the linked reference objects mention but the
 * oracle never calls (Damp4t10d::sfWriteVel). */
void sf_floatwrite(float *, size_t, sf_file) {}
void sf_close(void) {}
}  /* extern "C" */
