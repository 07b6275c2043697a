/* UpdateSteplenOp (src/essfwi/updatesteplenop.h:15-45) and
 * FwiUpdateSteplenOp (src/fwi/fwiupdatesteplenop.h:15-45): the step-length
 * search's settings (trial budget nita, largest velocity change maxdv); the
 * search itself (calMaxAlpha, the parabola vertex, refineAlpha) runs inside
 * the frameworks' epoch. */
#ifndef SWFWI_CPP_UPDATESTEPLENOP_H
#define SWFWI_CPP_UPDATESTEPLENOP_H

#include "damp4t10d.h"
#include "updatevelop.h"

class UpdateSteplenOp {
 public:
  UpdateSteplenOp(const Damp4t10d &fmMethod_, const UpdateVelOp &updateVelOp_, int max_iter_select_alpha3,
                  float maxdv_)
      : fmMethod(fmMethod_), updateVelOp(updateVelOp_), nita(max_iter_select_alpha3), maxdv(maxdv_) {}
  const Damp4t10d &fmMethod;
  const UpdateVelOp &updateVelOp;
  int nita;
  float maxdv;
};

class FwiUpdateSteplenOp : public UpdateSteplenOp {
 public:
  FwiUpdateSteplenOp(const Damp4t10d &fmMethod_, const FwiUpdateVelOp &updateVelOp_, int max_iter_select_alpha3,
                     float maxdv_)
      : UpdateSteplenOp(fmMethod_, updateVelOp_, max_iter_select_alpha3, maxdv_) {}
};

#endif
