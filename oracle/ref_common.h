/* Test infrastructure only: shared declarations for the two harness
 * translation units that wrap the compiled reference (swfwi) sources.
 * Only tests/, the smoke check and bench.py's CPU-baseline leg load the
 * resulting library; the product never does. */
#ifndef ORACLE_REF_COMMON_H
#define ORACLE_REF_COMMON_H
#include <vector>
#include "damp4t10d.h"
#include "shot-position.h"
#include "velocity.h"

/* One modelling set-up as the reference's drivers build it
 * (src/tool/main-fwi-damp.cpp:170-178): regular source and receiver
 * lines, a Damp4t10d bound to an expanded, transformed velocity. */
struct RefModel {
  int nz, nx, nb, nt, ns, ng;
  float dt, dx, fm;
  ShotPosition src;
  ShotPosition geo;
  Damp4t10d fm_method;
  Velocity exvel;
  RefModel(int nz_, int nx_, int nb_, int nt_, float dt_, float dx_, float fm_,
           int szbeg, int sxbeg, int jsz, int jsx, int ns_,
           int gzbeg, int gxbeg, int jgz, int jgx, int ng_)
      : nz(nz_), nx(nx_), nb(nb_), nt(nt_), ns(ns_), ng(ng_), dt(dt_), dx(dx_), fm(fm_),
        src(szbeg, sxbeg, jsz, jsx, ns_, nz_),
        geo(gzbeg, gxbeg, jgz, jgx, ng_, nz_),
        fm_method(src, geo, dt_, dx_, fm_, nb_, nt_),
        exvel(nx_ + 2 * nb_ + 12, nz_ + nb_ + 12) {}
  int nxpad() const { return nx + 2 * nb + 12; }
  int nzpad() const { return nz + nb + 12; }
};

/* Line search shared by both harnesses: the reference's working
 * UpdateSteplenOp logic (src/essfwi/updatesteplenop.cpp:88-265) with the
 * trial objective supplied by the caller. */
struct RefObjFn {
  virtual float operator()(float alpha) = 0;
  virtual ~RefObjFn() {}
};
#endif
