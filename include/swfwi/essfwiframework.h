/* EssFwiFramework (src/essfwi/essfwiframework.h:16-53) and FwiFramework
 * (src/fwi/fwiframework.h:16-53) over swfwi_fwi_*: the reference's
 * constructors and methods.  epoch() runs the whole iteration on the GPU
 * (gradient over all shots or the encoded supershot, conjugate direction,
 * step-length search, velocity update) and then writes the updated model
 * into the Velocity bound to the Damp4t10d, as the reference's epoch
 * updates it in place (fwiframework.cpp:352-355). */
#ifndef SWFWI_CPP_ESSFWIFRAMEWORK_H
#define SWFWI_CPP_ESSFWIFRAMEWORK_H

#include <vector>

#include "damp4t10d.h"
#include "updatesteplenop.h"
#include "updatevelop.h"

namespace swfwi_cpp {

class FrameworkBase {
 public:
  FrameworkBase(Damp4t10d &fmMethod, const UpdateSteplenOp &sl, const UpdateVelOp &uv, const std::vector<float> &wlt,
                const std::vector<float> &dobs, int encoded)
      : fm_(fmMethod) {
    check(swfwi_fwi_create(&h_, fm_.handle(), fm_.getVelocity().dat.data(), uv.vmin, uv.vmax, sl.nita, sl.maxdv,
                           wlt.data(), dobs.data(), encoded));
  }
  ~FrameworkBase() { swfwi_fwi_destroy(h_); }
  FrameworkBase(const FrameworkBase &) = delete;
  FrameworkBase &operator=(const FrameworkBase &) = delete;

  void epoch(int iter) {
    check(swfwi_fwi_epoch(h_, iter));
    Velocity &v = fm_.getVelocity();
    check(swfwi_fwi_get_velocity(h_, v.dat.data()));
  }
  float getUpdateObj() const {
    float o;
    check(swfwi_fwi_get_update_obj(h_, &o));
    return o;
  }
  float getInitObj() const {
    float o;
    check(swfwi_fwi_get_init_obj(h_, &o));
    return o;
  }
  /* the interior model in m/s, [nx][nz] (what sfWriteVel writes,
   * damp4t10d.cpp:254-265) */
  std::vector<float> writeVel() const {
    const Velocity &v = fm_.getVelocity();
    const int nb = fm_.getnb();
    std::vector<float> out((size_t)(v.nx - 2 * nb - 12) * (v.nz - nb - 12));
    check(swfwi_fwi_write_vel(h_, out.data()));
    return out;
  }
  /* writeVel(sf_file) (fwiframework.cpp:358-361): the same floats to an RSF
   * file (sf_floatwrite, found where the caller's rsf.h declares it) */
  template <class File>
  void writeVel(File file) const {
    std::vector<float> v = writeVel();
    sf_floatwrite(v.data(), v.size(), file);
  }
  swfwi_fwi *handle() const { return h_; }

 private:
  Damp4t10d &fm_;
  swfwi_fwi *h_ = nullptr;
};

}  // namespace swfwi_cpp

class EssFwiFramework : public swfwi_cpp::FrameworkBase {
 public:
  EssFwiFramework(Damp4t10d &fmMethod, const UpdateSteplenOp &updateSteplenOp, const UpdateVelOp &updateVelOp,
                  const std::vector<float> &wlt, const std::vector<float> &dobs)
      : FrameworkBase(fmMethod, updateSteplenOp, updateVelOp, wlt, dobs, 1) {}
};

#endif
