/* FwiFramework (src/fwi/fwiframework.h:16-53): plain FWI over all shots,
 * one batched gradient per epoch; see essfwiframework.h. */
#ifndef SWFWI_CPP_FWIFRAMEWORK_H
#define SWFWI_CPP_FWIFRAMEWORK_H

#include "essfwiframework.h"
#include "fwiupdatesteplenop.h"
#include "fwiupdatevelop.h"

class FwiFramework : public swfwi_cpp::FrameworkBase {
 public:
  FwiFramework(Damp4t10d &fmMethod, const FwiUpdateSteplenOp &updateSteplenOp, const FwiUpdateVelOp &updateVelOp,
               const std::vector<float> &wlt, const std::vector<float> &dobs)
      : FrameworkBase(fmMethod, updateSteplenOp, updateVelOp, wlt, dobs, 0) {}
};

#endif
