/* rickerWavelet (src/common/ricker-wavelet.h:13, 15): nt samples of a
 * Ricker wavelet of peak frequency fm, sample interval dt, amplitude amp. */
#ifndef SWFWI_CPP_RICKER_WAVELET_H
#define SWFWI_CPP_RICKER_WAVELET_H

#include <stdexcept>
#include <vector>

#include "../swfwi_gpu.h"

inline void rickerWavelet(float *wlt, int nt, float fm, float dt, float amp) {
  if (swfwi_ricker_wavelet(wlt, nt, fm, dt, amp) != SWFWI_OK) throw std::runtime_error(swfwi_last_error());
}

inline std::vector<float> rickerWavelet(int nt, float fm, float dt, float amp) {
  std::vector<float> w(nt);
  rickerWavelet(w.data(), nt, fm, dt, amp);
  return w;
}

#endif
