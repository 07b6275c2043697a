/* Velocity (src/common/velocity.h:12-20): a model of nx x nz floats,
 * x-major (dat[ix*nz + iz]).  The same members as the reference's class, so
 * its readers and drivers compile against this header unchanged. */
#ifndef SWFWI_CPP_VELOCITY_H
#define SWFWI_CPP_VELOCITY_H

#include <vector>

class Velocity {
 public:
  Velocity(int nx_, int nz_) : dat((size_t)nx_ * nz_), nx(nx_), nz(nz_) {}
  Velocity(const std::vector<float> &d, int nx_, int nz_) : dat(d), nx(nx_), nz(nz_) {}

  std::vector<float> dat;
  int nx;
  int nz;
};

#endif
