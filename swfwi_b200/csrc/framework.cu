// FWI drivers; see framework.hpp for the reference files they follow.
#include <algorithm>
#include <cmath>
#include <numeric>
#include "framework.hpp"
#include "precond.hpp"

namespace swfwi {

// ---------------------------------------------------------------- codes
RandomCodes::RandomCodes(int seed) {
  const int64_t m = 2147483647;
  int64_t s = seed % m;
  if (s < 0) s += m;
  x_ = (uint64_t)(s == 0 ? 1 : s);
}

int RandomCodes::draw() {
  x_ = (x_ * 48271u) % 2147483647u;
  // engine range [1, 2^31-2]: brange = 2^31-3, bucket = (brange+1)/2
  const uint64_t bucket = (2147483645ull + 1) / 2;
  uint64_t b = (x_ - 1) / bucket;   // 0 or 1 (2 is unreachable for this range)
  return (int)b;
}

std::vector<int> RandomCodes::gen_plus1_minus1(int n) {
  std::vector<int> c(n);
  for (int i = 0; i < n; i++) c[i] = draw() * 2 - 1;
  return c;
}

// ---------------------------------------------------------------- vertex
// parabola-vertex.cpp:12-33: the products below are float expressions
// (their operands are float), divided in double.
void parabola_vertex(float x1, float y1, float x2, float y2, float x3, float y3, float max_alpha3,
                     float &xv, float &yv) {
  (void)max_alpha3;
  double k2 = (y3 - y2) / (x3 - x2);
  double k1 = (y2 - y1) / (x2 - x1);
  double denom = (x1 - x2) * (x1 - x3) * (x2 - x3);
  double A = (x3 * (y2 - y1) + x2 * (y1 - y3) + x1 * (y3 - y2)) / denom;
  double B = (x3 * x3 * (y1 - y2) + x2 * x2 * (y3 - y1) + x1 * x1 * (y2 - y3)) / denom;
  double C = (x2 * x3 * (x2 - x3) * y1 + x3 * x1 * (x3 - x1) * y2 + x1 * x2 * (x1 - x2) * y3) / denom;
  xv = (float)(-B / (2 * A));
  yv = (float)(C - B * B / (4 * A));
  if (std::abs(k2 - k1) < 0.001 * (std::max(std::abs(k2), std::abs(k1))) || std::isnan(-xv)) {
    xv = x3;
    yv = y3;
  }
}

// ---------------------------------------------------------------- search
namespace {
// The reference keeps tried (alpha, obj) pairs in a std::set ordered by
// obj (updatesteplenop.cpp:19-21, 107) and takes begin(): the smallest
// objective, the latest insertion first among equal ones.
struct Tried {
  std::vector<std::pair<float, float>> v;
  void insert(float a, float o) { v.emplace_back(a, o); }
  void clear() { v.clear(); }
  std::pair<float, float> best() const {
    std::pair<float, float> b = v.back();
    for (auto it = v.rbegin(); it != v.rend(); ++it)
      if ((double)it->second - (double)b.second < -1e-10) b = *it;
    return b;
  }
};
}  // namespace

float StepSearch::calsteplen(const std::function<float(float)> &fobj, float obj_val1,
                             float max_alpha3, float &objval) {
  trials = 0;
  auto f = [&](float a) {
    trials++;
    return fobj(a);
  };
  // initAlpha23 (updatesteplenop.cpp:273-285)
  const float minAlpha = 1.0E-7f, resetAlpha = 1.0E-4f;
  if (!preserved_init) {
    preserved_init = true;
    preserved_alpha = max_alpha3;
  }
  float alpha3 = preserved_alpha;
  alpha3 = alpha3 < minAlpha ? resetAlpha : alpha3;
  float alpha2 = (float)(alpha3 * 0.5);
  const float alpha1 = 0;
  float obj_val2, obj_val3;
  bool to_parabolic = true;

  // refineAlpha (updatesteplenop.cpp:88-214)
  {
    float a3 = alpha3, a2 = alpha2;
    float o2 = f(a2), o3 = f(a3);
    Tried tuned;
    tuned.insert(a2, o2);
    for (int it = 0; it < nita && o2 > obj_val1; it++) {
      a3 = a2;
      o3 = o2;
      a2 /= 2;
      o2 = f(a2);
      tuned.insert(a2, o2);
    }
    if (o2 > obj_val1) {
      auto b = tuned.best();
      alpha2 = b.first;
      obj_val2 = b.second;
      alpha3 = std::min(alpha2 * 2, max_alpha3);
      obj_val3 = f(a3);   // the reference evaluates its local alpha3 here
      to_parabolic = false;
    } else {
      float linear = (o2 - obj_val1) / (a2 - alpha1) * (a3 - alpha1) + obj_val1;
      tuned.clear();
      tuned.insert(a3, o3);
      while (o3 < linear && o3 < obj_val1 && a3 < max_alpha3) {
        a2 = a3;
        o2 = o3;
        a3 = std::min(a3 * 2, max_alpha3);
        o3 = f(a3);
        tuned.insert(a3, o3);
      }
      if (a3 > max_alpha3 + 0.1) {
        auto b = tuned.best();
        alpha3 = b.first;
        obj_val3 = b.second;
        alpha2 = alpha3 / 2;
        obj_val2 = f(a2);   // the reference evaluates its local alpha2 here
        to_parabolic = false;
      } else {
        alpha2 = a2;
        alpha3 = a3;
        obj_val2 = o2;
        obj_val3 = o3;
      }
    }
  }

  // calsteplen (updatesteplenop.cpp:236-264)
  float alpha4, obj_val4;
  if (to_parabolic) {
    parabola_vertex(alpha1, obj_val1, alpha2, obj_val2, alpha3, obj_val3, max_alpha3, alpha4,
                    obj_val4);
    if (alpha4 > max_alpha3) alpha4 = max_alpha3;
  } else {
    alpha4 = alpha3;
    obj_val4 = obj_val3;
  }
  alpha[0] = alpha1; alpha[1] = alpha2; alpha[2] = alpha3; alpha[3] = alpha4;
  obj[0] = obj_val1; obj[1] = obj_val2; obj[2] = obj_val3; obj[3] = obj_val4;
  preserved_alpha = alpha4;
  objval = obj_val4;
  return alpha4;
}

// ---------------------------------------------------------------- runner
FwiRunner::FwiRunner(Propagator &p, const float *exvel_host, float vmin, float vmax, int nita,
                     float maxdv, const float *wlt_host, const float *dobs_host, bool encoded)
    : p_(p), encoded_(encoded), codes_gen_(1) {
  SWFWI_REQUIRE(p.nxpad > 0, "propagator has no grid: expand or bind a velocity first");
  SWFWI_REQUIRE(exvel_host && wlt_host && dobs_host, "null input");
  SWFWI_REQUIRE(!encoded || p.ngmax == p.ng, "encoded sources need one common receiver line");
  // UpdateVelOp::UpdateVelOp (updatevelop.cpp:23-31)
  vmin_t_ = (p.dx / p.dt / vmax) * (p.dx / p.dt / vmax);
  vmax_t_ = (p.dx / p.dt / vmin) * (p.dx / p.dt / vmin);
  SWFWI_REQUIRE(vmax_t_ > vmin_t_, "vmax must exceed vmin");
  search.nita = nita;
  search.maxdv = maxdv;
  learned_search.nita = nita;
  learned_search.maxdv = maxdv;
  n_ = p.nxpad * p.nzpad;
  cudaStream_t st = p.stream();
  vel_.upload(exvel_host, n_, st);
  trial_.resize(n_);
  g_.resize(n_);
  g0_.resize(n_);
  dir_.resize(n_);
  g0_.zero(st);
  dir_.zero(st);
  wlt_.upload(wlt_host, p.nt, st);
  dobs_.upload(dobs_host, (size_t)p.ns * p.nt * p.ngmax, st);
  scratch_.resize(4096);
  ids_.resize(p.ns);
  std::iota(ids_.begin(), ids_.end(), 0);
  SWFWI_CUDA(cudaStreamSynchronize(st));
}

double FwiRunner::sumsq(const float *x, long long n) {
  launch_sumsq_f64(scratch_.get(), x, n, 1, scratch_.get() + 8, 256, p_.stream());
  double h = 0;
  SWFWI_CUDA(cudaMemcpyAsync(&h, scratch_.get(), sizeof(double), cudaMemcpyDeviceToHost, p_.stream()));
  SWFWI_CUDA(cudaStreamSynchronize(p_.stream()));
  return h;
}

// updateGrad (fwiframework.cpp:42-72), dot products in FP64.
void FwiRunner::update_grad(int iter) {
  cudaStream_t st = p_.stream();
  if (iter == 0) {
    launch_cg_update(dir_.get(), g0_.get(), g_.get(), 0.0f, n_, 1, st);
    return;
  }
  launch_cg_dots(scratch_.get(), g_.get(), g0_.get(), n_, scratch_.get() + 8, st);
  double d[3];
  SWFWI_CUDA(cudaMemcpyAsync(d, scratch_.get(), sizeof(d), cudaMemcpyDeviceToHost, st));
  SWFWI_CUDA(cudaStreamSynchronize(st));
  float beta = (float)((d[0] - d[1]) / d[2]);
  if (beta < 0.0f) beta = 0.0f;
  launch_cg_update(dir_.get(), g0_.get(), g_.get(), beta, n_, 0, st);
}

void FwiRunner::epoch(int iter) {
  if (encoded_ && regu_) regu_epoch(iter);
  else if (encoded_) ess_epoch(iter);
  else plain_epoch(iter);
}

void FwiRunner::set_regularization(float lx, float lz) {
  SWFWI_REQUIRE(encoded_, "regularisation applies to the encoded-source framework");
  SWFWI_REQUIRE(lx >= 0.0f && lz >= 0.0f && std::isfinite(lx) && std::isfinite(lz),
                "regularisation weights must be finite and non-negative");
  regu_lx_ = lx;
  regu_lz_ = lz;
  regu_ = lx > 0.0f || lz > 0.0f;
}

// ReguFactor::getReguTerm of a padded model (FP64 sums, returned as the
// float the reference adds to its objective).
float FwiRunner::regu_term(const float *vel) {
  regu_scratch_.resize(regu_scratch_doubles());
  double *sc = regu_scratch_.get();
  launch_regu_term(vel, p_.nxpad, p_.nzpad, regu_lx_, regu_lz_, sc, p_.stream());
  double h[3];
  SWFWI_CUDA(cudaMemcpyAsync(h, sc, sizeof(h), cudaMemcpyDeviceToHost, p_.stream()));
  SWFWI_CUDA(cudaStreamSynchronize(p_.stream()));
  return (float)h[2];
}

// EssFwiRegu::epoch (src/unused/essfwiregu.cpp:667-776).  The reference
// restores the source field from disk checkpoints every 50 steps (hello,
// :217-349); this restores it from the boundary strips like calgradient.
// The step length is the framework's UpdateSteplenOp search over the
// regularised objective (calculate_obj_val :405-449 adds the trial model's
// term).
void FwiRunner::regu_epoch(int iter) {
  cudaStream_t st = p_.stream();
  p_.bind_velocity(vel_.get());
  const int nt = p_.nt, ns = p_.ns, ng = p_.ng;
  long long dn = (long long)nt * ng;
  std::vector<int> codes = codes_gen_.gen_plus1_minus1(ns);
  codes_.upload(codes, st);
  encsrc_.resize((size_t)nt * ns);
  encobs_.resize(dn);
  dcal_.resize(dn);
  vsrc_.resize(dn);
  res_.resize(dn);
  launch_encode_source(encsrc_.get(), wlt_.get(), codes_.get(), nt, ns, st);
  launch_encode_obs(encobs_.get(), dobs_.get(), codes_.get(), dn, ns, st);
  p_.ess_forward(encsrc_.get(), dcal_.get());
  p_.remove_direct_arrival(encobs_.get(), -1);
  p_.remove_direct_arrival(dcal_.get(), -1);
  launch_residual(res_.get(), encobs_.get(), 0, dcal_.get(), dn, 1, st);
  float obj1 = (float)sumsq(res_.get(), dn);
  obj1 += regu_term(vel_.get());
  if (iter == 0) init_obj = obj1;
  launch_trans_vsrc(vsrc_.get(), res_.get(), nt, ng, 1, st);
  g_.zero(st);
  p_.calgradient_ess(encsrc_.get(), vsrc_.get(), g_.get());
  launch_regu_grad(vel_.get(), p_.nxpad, p_.nzpad, regu_lx_, regu_lz_, g_.get(), true, st);
  p_.mask_gradient(g_.get());
  SWFWI_CUDA(cudaMemcpyAsync(dir_.get(), g_.get(), sizeof(float) * n_, cudaMemcpyDeviceToDevice, st));

  launch_max_alpha(reinterpret_cast<float *>(scratch_.get()), vel_.get(), dir_.get(), n_, p_.dt,
                   p_.dx, search.maxdv, st);
  float a2max = 0;
  SWFWI_CUDA(cudaMemcpyAsync(&a2max, scratch_.get(), sizeof(float), cudaMemcpyDeviceToHost, st));
  SWFWI_CUDA(cudaStreamSynchronize(st));
  float a3max = 2 * a2max;
  auto f = [&](float alpha) -> float {
    launch_update_vel(trial_.get(), vel_.get(), dir_.get(), n_, alpha, vmin_t_, vmax_t_, st);
    p_.ess_forward(encsrc_.get(), dcal_.get(), trial_.get());
    p_.remove_direct_arrival(dcal_.get(), -1, trial_.get());
    launch_residual(res_.get(), encobs_.get(), 0, dcal_.get(), dn, 1, st);
    float v = (float)sumsq(res_.get(), dn);
    return v + regu_term(trial_.get());
  };
  float objv = 0;
  float step = search.calsteplen(f, obj1, a3max, objv);
  update_obj = objv;
  launch_update_vel(vel_.get(), vel_.get(), dir_.get(), n_, step, vmin_t_, vmax_t_, st);
  launch_refill_boundary(vel_.get(), p_.nxpad, p_.nzpad, p_.bz0, p_.bzn, p_.bx0, p_.bxn, st);
  p_.bind_velocity(vel_.get());
  SWFWI_CUDA(cudaStreamSynchronize(st));
}

// FwiFramework::epoch (fwiframework.cpp:269-356) with the documented
// step-length rule: the encoded-source search of updatesteplenop.cpp with
// the trial objective summed over all shots (the reference's plain-FWI
// search reads uninitialised values, fwiupdatesteplenop.cpp:88-217).
void FwiRunner::plain_epoch(int iter) {
  cudaStream_t st = p_.stream();
  p_.bind_velocity(vel_.get());
  std::vector<double> obj(p_.ns);
  const bool want_illum = collect_illum_ || net_;
  if (want_illum) {
    illum_.resize(n_);
    illum_.zero(st);
    p_.illum = illum_.get();
  }
  try {
    p_.gradient_batch(wlt_.get(), dobs_.get(), ids_.data(), p_.ns, g_.get(), obj.data());
  } catch (...) {
    p_.illum = nullptr;
    throw;
  }
  p_.illum = nullptr;
  float obj1 = 0.0f;
  for (double o : obj) obj1 += (float)o;
  if (iter == 0) init_obj = obj1;
  update_grad(restart_cg_ ? 0 : iter);
  restart_cg_ = false;
  last_step_learned = 0;
  if (net_ && (learned_patience == 0 || learned_rejected < learned_patience) && try_learned_step(obj1))
    return;

  launch_max_alpha(reinterpret_cast<float *>(scratch_.get()), vel_.get(), dir_.get(), n_, p_.dt,
                   p_.dx, search.maxdv, st);
  float a2max = 0;
  SWFWI_CUDA(cudaMemcpyAsync(&a2max, scratch_.get(), sizeof(float), cudaMemcpyDeviceToHost, st));
  SWFWI_CUDA(cudaStreamSynchronize(st));
  float a3max = 2 * a2max;
  auto f = [&](float alpha) -> float {
    launch_update_vel(trial_.get(), vel_.get(), dir_.get(), n_, alpha, vmin_t_, vmax_t_, st);
    return (float)p_.trial_objective_fwi(wlt_.get(), dobs_.get(), ids_.data(), p_.ns, trial_.get());
  };
  float objv = 0;
  float step = search.calsteplen(f, obj1, a3max, objv);
  update_obj = objv;
  launch_update_vel(vel_.get(), vel_.get(), dir_.get(), n_, step, vmin_t_, vmax_t_, st);
  launch_refill_boundary(vel_.get(), p_.nxpad, p_.nzpad, p_.bz0, p_.bzn, p_.bx0, p_.bxn, st);
  p_.bind_velocity(vel_.get());
  SWFWI_CUDA(cudaStreamSynchronize(st));
}

bool FwiRunner::try_learned_step(float obj1) {
  cudaStream_t st = p_.stream();
  learned_tried++;
  ldir_.resize(n_);
  net_->set_stream(st);
  net_->propose(g_.get(), vel_.get(), illum_.get(), p_.nxpad, p_.nzpad, p_.bx0, p_.bxn, p_.bz0, p_.bzn,
                ldir_.get());
  launch_max_alpha(reinterpret_cast<float *>(scratch_.get()), vel_.get(), ldir_.get(), n_, p_.dt, p_.dx,
                   learned_search.maxdv, st);
  float a2max = 0;
  SWFWI_CUDA(cudaMemcpyAsync(&a2max, scratch_.get(), sizeof(float), cudaMemcpyDeviceToHost, st));
  SWFWI_CUDA(cudaStreamSynchronize(st));
  if (!(a2max > 0.0f) || !std::isfinite(a2max)) return false;
  auto f = [&](float alpha) -> float {
    launch_update_vel(trial_.get(), vel_.get(), ldir_.get(), n_, alpha, vmin_t_, vmax_t_, st);
    return (float)p_.trial_objective_fwi(wlt_.get(), dobs_.get(), ids_.data(), p_.ns, trial_.get());
  };
  float objv = 0;
  const float step = learned_search.calsteplen(f, obj1, 2 * a2max, objv);
  const float tried_best = std::min(learned_search.obj[1], learned_search.obj[2]);
  const float bar = obj1 * (1.0f - learned_min_decrease);
  if (!(std::isfinite(objv) && objv < bar && tried_best < obj1 && step > 0.0f)) {
    // rejected: the next search along the network starts from scratch
    learned_search.preserved_init = false;
    learned_rejected++;
    return false;
  }
  update_obj = objv;
  launch_update_vel(vel_.get(), vel_.get(), ldir_.get(), n_, step, vmin_t_, vmax_t_, st);
  launch_refill_boundary(vel_.get(), p_.nxpad, p_.nzpad, p_.bz0, p_.bzn, p_.bx0, p_.bxn, st);
  p_.bind_velocity(vel_.get());
  SWFWI_CUDA(cudaStreamSynchronize(st));
  restart_cg_ = true;
  last_step_learned = 1;
  learned_accepted++;
  return true;
}

void FwiRunner::get_gradient(float *host) {
  SWFWI_CUDA(cudaMemcpyAsync(host, g_.get(), sizeof(float) * n_, cudaMemcpyDeviceToHost, p_.stream()));
  SWFWI_CUDA(cudaStreamSynchronize(p_.stream()));
}

void FwiRunner::get_illumination(float *host) {
  SWFWI_REQUIRE(illum_.size() == (size_t)n_, "no illumination recorded: enable collection first");
  SWFWI_CUDA(cudaMemcpyAsync(host, illum_.get(), sizeof(float) * n_, cudaMemcpyDeviceToHost, p_.stream()));
  SWFWI_CUDA(cudaStreamSynchronize(p_.stream()));
}

// EssFwiFramework::epoch (essfwiframework.cpp:191-239).
void FwiRunner::ess_epoch(int iter) {
  cudaStream_t st = p_.stream();
  p_.bind_velocity(vel_.get());
  const int nt = p_.nt, ns = p_.ns, ng = p_.ng;
  long long dn = (long long)nt * ng;
  std::vector<int> codes = codes_gen_.gen_plus1_minus1(ns);
  codes_.upload(codes, st);
  encsrc_.resize((size_t)nt * ns);
  encobs_.resize(dn);
  dcal_.resize(dn);
  vsrc_.resize(dn);
  res_.resize(dn);
  launch_encode_source(encsrc_.get(), wlt_.get(), codes_.get(), nt, ns, st);
  launch_encode_obs(encobs_.get(), dobs_.get(), codes_.get(), dn, ns, st);
  p_.ess_forward(encsrc_.get(), dcal_.get());
  p_.remove_direct_arrival(encobs_.get(), -1);
  p_.remove_direct_arrival(dcal_.get(), -1);
  launch_residual(res_.get(), encobs_.get(), 0, dcal_.get(), dn, 1, st);
  float obj1 = (float)sumsq(res_.get(), dn);
  if (iter == 0) init_obj = obj1;
  launch_trans_vsrc(vsrc_.get(), res_.get(), nt, ng, 1, st);
  g_.zero(st);
  p_.calgradient_ess(encsrc_.get(), vsrc_.get(), g_.get());
  p_.scale_gradient(g_.get());
  p_.mask_gradient(g_.get());
  update_grad(iter);

  launch_max_alpha(reinterpret_cast<float *>(scratch_.get()), vel_.get(), dir_.get(), n_, p_.dt,
                   p_.dx, search.maxdv, st);
  float a2max = 0;
  SWFWI_CUDA(cudaMemcpyAsync(&a2max, scratch_.get(), sizeof(float), cudaMemcpyDeviceToHost, st));
  SWFWI_CUDA(cudaStreamSynchronize(st));
  float a3max = 2 * a2max;
  // calobjval (updatesteplenop.cpp:59-86)
  auto f = [&](float alpha) -> float {
    launch_update_vel(trial_.get(), vel_.get(), dir_.get(), n_, alpha, vmin_t_, vmax_t_, st);
    p_.ess_forward(encsrc_.get(), dcal_.get(), trial_.get());
    p_.remove_direct_arrival(dcal_.get(), -1, trial_.get());
    launch_residual(res_.get(), encobs_.get(), 0, dcal_.get(), dn, 1, st);
    return (float)sumsq(res_.get(), dn);
  };
  float objv = 0;
  float step = search.calsteplen(f, obj1, a3max, objv);
  update_obj = objv;
  launch_update_vel(vel_.get(), vel_.get(), dir_.get(), n_, step, vmin_t_, vmax_t_, st);
  launch_refill_boundary(vel_.get(), p_.nxpad, p_.nzpad, p_.bz0, p_.bzn, p_.bx0, p_.bxn, st);
  p_.bind_velocity(vel_.get());
  SWFWI_CUDA(cudaStreamSynchronize(st));
}

void FwiRunner::get_velocity(float *host) {
  SWFWI_CUDA(cudaMemcpyAsync(host, vel_.get(), sizeof(float) * n_, cudaMemcpyDeviceToHost, p_.stream()));
  SWFWI_CUDA(cudaStreamSynchronize(p_.stream()));
}

void FwiRunner::set_velocity(const float *host) {
  SWFWI_CUDA(cudaMemcpyAsync(vel_.get(), host, sizeof(float) * n_, cudaMemcpyHostToDevice, p_.stream()));
  SWFWI_CUDA(cudaStreamSynchronize(p_.stream()));
  p_.bind_velocity(vel_.get());   // contents changed: recompute 1/vt
}

// sfWriteVel (damp4t10d.cpp:254-265): recoverVel v = sqrt(dx^2/(dt^2 vt))
// then the interior columns from depth 6.
void FwiRunner::write_vel(float *host) {
  std::vector<float> v(n_);
  get_velocity(v.data());
  float dx = p_.dx, dt = p_.dt;
  int nzpad = p_.nzpad, nz = nzpad - p_.bz0 - p_.bzn;
  for (int ix = p_.bx0; ix < p_.nxpad - p_.bxn; ix++)
    for (int iz = 0; iz < nz; iz++) {
      float t = v[(size_t)ix * nzpad + 6 + iz];
      host[(size_t)(ix - p_.bx0) * nz + iz] = std::sqrt(dx * dx / (dt * dt * t));
    }
}

}  // namespace swfwi
