/* UpdateVelOp (src/essfwi/updatevelop.h:13-24) and FwiUpdateVelOp
 * (src/fwi/fwiupdatevelop.h:13-24): the velocity bounds and grid steps the
 * frameworks' velocity update uses (the update itself runs on the GPU,
 * swfwi_update_vel). */
#ifndef SWFWI_CPP_UPDATEVELOP_H
#define SWFWI_CPP_UPDATEVELOP_H

class UpdateVelOp {
 public:
  UpdateVelOp(float vmin_, float vmax_, float dx_, float dt_) : vmin(vmin_), vmax(vmax_), dx(dx_), dt(dt_) {}
  float vmin, vmax, dx, dt;
};

class FwiUpdateVelOp : public UpdateVelOp {
 public:
  using UpdateVelOp::UpdateVelOp;
};

#endif
