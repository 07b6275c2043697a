/* Damp4t10d (src/modeling/damp4t10d.h:18-87) over the C ABI of
 * swfwi_gpu.h: the reference's class name, constructor and method names,
 * so its drivers (src/tool/main-fwi-damp.cpp:145-212,
 * main-essfwi-damp.cpp:145-211) compile against this directory unchanged and
 * run on the GPU.  Header-only; link libswfwi_b200.so and the CUDA runtime.
 *
 * Arrays the reference passes as host pointers stay host pointers here: the
 * per-call methods copy to the device and back (correct, not fast: a whole
 * time loop belongs in FwiForwardModeling / the frameworks, which keep
 * everything on the device).  Errors throw std::runtime_error with the
 * library's message. */
#ifndef SWFWI_CPP_DAMP4T10D_H
#define SWFWI_CPP_DAMP4T10D_H

#include <cuda_runtime_api.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "shot-position.h"
#include "../swfwi_gpu.h"
#include "velocity.h"

namespace swfwi_cpp {

inline void check(int status) {
  if (status != SWFWI_OK) throw std::runtime_error(std::string("swfwi: ") + swfwi_last_error());
}

inline void cuda_check(cudaError_t e) {
  if (e != cudaSuccess) throw std::runtime_error(std::string("swfwi: ") + cudaGetErrorString(e));
}

/* a device copy of host floats, copied back on request */
class DeviceFloats {
 public:
  DeviceFloats() = default;
  explicit DeviceFloats(size_t n) { resize(n); }
  DeviceFloats(const float *h, size_t n) {
    resize(n);
    put(h);
  }
  ~DeviceFloats() {
    if (p_) cudaFree(p_);
  }
  DeviceFloats(const DeviceFloats &) = delete;
  DeviceFloats &operator=(const DeviceFloats &) = delete;
  void resize(size_t n) {
    if (n == n_) return;
    if (p_) cudaFree(p_);
    p_ = nullptr;
    n_ = n;
    if (n) cuda_check(cudaMalloc(reinterpret_cast<void **>(&p_), n * sizeof(float)));
  }
  void put(const float *h) { cuda_check(cudaMemcpy(p_, h, n_ * sizeof(float), cudaMemcpyHostToDevice)); }
  void get(float *h) const { cuda_check(cudaMemcpy(h, p_, n_ * sizeof(float), cudaMemcpyDeviceToHost)); }
  float *ptr() const { return p_; }

 private:
  float *p_ = nullptr;
  size_t n_ = 0;
};

}  // namespace swfwi_cpp

class Damp4t10d {
 public:
  Damp4t10d(const ShotPosition &allSrcPos, const ShotPosition &allGeoPos, float dt, float dx, float fm, int nb,
            int nt)
      : src_(allSrcPos), geo_(allGeoPos), dt_(dt), dx_(dx), fm_(fm), nb_(nb), nt_(nt) {
    const swfwi_shot_position s = src_.raw(), g = geo_.raw();
    swfwi_cpp::check(swfwi_damp4t10d_create(&h_, &s, &g, dt, dx, fm, nb, nt));
  }
  ~Damp4t10d() { swfwi_damp4t10d_destroy(h_); }
  Damp4t10d(const Damp4t10d &) = delete;
  Damp4t10d &operator=(const Damp4t10d &) = delete;

  /* expandDomain (damp4t10d.cpp:138-151): sponge and stencil padding,
   * velocity transformed to dx^2 / (v^2 dt^2) */
  Velocity expandDomain(const Velocity &vel) {
    Velocity ret(vel.nx + 2 * nb_ + 12, vel.nz + nb_ + 12);
    swfwi_cpp::check(swfwi_damp4t10d_expand_domain(h_, vel.dat.data(), vel.nx, vel.nz, ret.dat.data()));
    return ret;
  }

  /* bindVelocity (:159-161): keeps a reference to the expanded model, as
   * the reference does, and a device copy of it */
  void bindVelocity(const Velocity &vel) {
    vel_ = &vel;
    swfwi_cpp::check(swfwi_damp4t10d_set_model_size(h_, vel.nx - 2 * nb_ - 12, vel.nz - nb_ - 12));
    dvel_.resize(vel.dat.size());
    dvel_.put(vel.dat.data());
    swfwi_cpp::check(swfwi_damp4t10d_bind_velocity(h_, dvel_.ptr()));
  }

  /* stepForward (:153-157, damped) / stepBackward (:188-191): p0 <- F(p0,
   * p1) on host fields of nxpad x nzpad */
  void stepForward(float *p0, float *p1) const { step(p0, p1, true); }
  void stepBackward(float *p0, float *p1) const { step(p0, p1, false); }

  /* FwiForwardModeling (:272-289): shot shot_id, wavelet encsrc [nt] ->
   * dcal [nt][ng] */
  void FwiForwardModeling(const std::vector<float> &encsrc, std::vector<float> &dcal, int shot_id) const {
    swfwi_cpp::DeviceFloats w(encsrc.data(), (size_t)nt_), d((size_t)nt_ * getng());
    swfwi_cpp::check(swfwi_damp4t10d_fwi_forward_modeling(h_, w.ptr(), d.ptr(), shot_id));
    dcal.resize((size_t)nt_ * getng());
    d.get(dcal.data());
  }

  /* EssForwardModeling (:291-307): encoded sources encsrc [nt][ns] ->
   * dcal [nt][ng] */
  void EssForwardModeling(const std::vector<float> &encsrc, std::vector<float> &dcal) const {
    swfwi_cpp::DeviceFloats w(encsrc.data(), (size_t)nt_ * getns()), d((size_t)nt_ * getng());
    swfwi_cpp::check(swfwi_damp4t10d_ess_forward_modeling(h_, w.ptr(), d.ptr()));
    dcal.resize((size_t)nt_ * getng());
    d.get(dcal.data());
  }

  /* fwiRemoveDirectArrival (:390-394) / removeDirectArrival (:321-365):
   * data [nt][ng] in place */
  void fwiRemoveDirectArrival(float *data, int shot_id) const { data_op(data, shot_id); }
  void removeDirectArrival(float *data) const { data_op(data, -1); }

  /* maskGradient (:216-226), scaleGradient (:309-319), refillBoundary
   * (:228-252) on host arrays of nxpad x nzpad */
  void maskGradient(float *grad) const { model_op(grad, swfwi_damp4t10d_mask_gradient); }
  void scaleGradient(float *grad) const { model_op(grad, swfwi_damp4t10d_scale_gradient); }
  void refillBoundary(float *vel) const { model_op(vel, swfwi_damp4t10d_refill_boundary); }

  /* getVelocity (:184-186, :443-445): the bound model; the reference
   * hands it out writable too */
  const Velocity &getVelocity() const { return *vel_; }
  Velocity &getVelocity() { return const_cast<Velocity &>(*vel_); }
  const ShotPosition &getAllSrcPos() const { return src_; }
  const ShotPosition &getAllGeoPos() const { return geo_; }
  int getns() const { return src_.ns; }
  int getng() const { return geo_.ns; }
  float getdt() const { return dt_; }
  float getdx() const { return dx_; }
  int getnt() const { return nt_; }
  int getnx() const { return vel_->nx; }
  int getnz() const { return vel_->nz; }
  /* sponge width given to the constructor (not in the reference's class) */
  int getnb() const { return nb_; }

  /* the C ABI handle, for the swfwi_damp4t10d_* calls this class does not
   * wrap (batched gradients, arithmetic, strips, tuning) */
  swfwi_damp4t10d *handle() const { return h_; }

 private:
  size_t model_size() const { return (size_t)vel_->nx * vel_->nz; }

  void step(float *p0, float *p1, bool damped) const {
    swfwi_cpp::DeviceFloats a(p0, model_size()), b(p1, model_size());
    swfwi_cpp::check(damped ? swfwi_damp4t10d_step_forward(h_, a.ptr(), b.ptr())
                            : swfwi_damp4t10d_step_backward(h_, a.ptr(), b.ptr()));
    a.get(p0);
  }

  void data_op(float *data, int shot_id) const {
    swfwi_cpp::DeviceFloats d(data, (size_t)nt_ * getng());
    swfwi_cpp::check(swfwi_damp4t10d_remove_direct_arrival(h_, d.ptr(), shot_id));
    d.get(data);
  }

  void model_op(float *a, int (*op)(swfwi_damp4t10d *, float *)) const {
    swfwi_cpp::DeviceFloats d(a, model_size());
    swfwi_cpp::check(op(h_, d.ptr()));
    d.get(a);
  }

  ShotPosition src_, geo_;
  float dt_, dx_, fm_;
  int nb_, nt_;
  const Velocity *vel_ = nullptr;
  swfwi_damp4t10d *h_ = nullptr;
  swfwi_cpp::DeviceFloats dvel_;
};

#endif
