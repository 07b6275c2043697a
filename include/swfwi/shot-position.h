/* ShotPosition (src/common/shot-position.h:13-27): a regular line of ns
 * points, point i at z = szbeg + i jsz, x = sxbeg + i jsx (unpadded grid
 * indices), nz the model depth.  The reference's interface, so its drivers
 * compile against this header unchanged. */
#ifndef SWFWI_CPP_SHOT_POSITION_H
#define SWFWI_CPP_SHOT_POSITION_H

#include <stdexcept>

#include "../swfwi_gpu.h"

class ShotPosition {
 public:
  ShotPosition(int szbeg, int sxbeg, int jsz, int jsx, int ns_, int nz_)
      : ns(ns_), szbeg_(szbeg), sxbeg_(sxbeg), jsz_(jsz), jsx_(jsx), nz_(nz_) {}

  /* points [begin, end] (inclusive, as the reference's clipRange) */
  ShotPosition clipRange(int begin, int end) const {
    if (begin < 0 || end >= ns || begin > end) throw std::out_of_range("ShotPosition::clipRange");
    return ShotPosition(getz(begin), getx(begin), jsz_, jsx_, end - begin + 1, nz_);
  }
  ShotPosition clip(int idx) const { return clipRange(idx, idx); }
  int getx(int idx) const { return sxbeg_ + idx * jsx_; }
  int getz(int idx) const { return szbeg_ + idx * jsz_; }

  /* the C ABI's description of the line */
  swfwi_shot_position raw() const { return swfwi_shot_position{szbeg_, sxbeg_, jsz_, jsx_, ns, nz_}; }

  int ns;

 private:
  int szbeg_, sxbeg_, jsz_, jsx_, nz_;
};

#endif
