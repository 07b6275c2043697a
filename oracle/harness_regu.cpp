/* Test infrastructure only (the oracle): a C entry point over the
 * reference's own regularisation factor (src/unused/ReguFactor.cpp,
 * compiled in place).  Nothing here is shipped or measured as the product. */
#include <algorithm>
#include "ReguFactor.h"

extern "C" {

/* ReguFactor(vel, nx, nz, lx, lz): term = getReguTerm() (:19-27), grad
 * [nx*nz] = getReguGradient() (:67-108). */
void ref_regu(const float *vel, int nx, int nz, float lx, float lz, float *term, float *grad) {
  ReguFactor f(vel, nx, nz, lx, lz);
  *term = f.getReguTerm();
  const float *g = f.getReguGradient();
  std::copy(g, g + (size_t)nx * nz, grad);
}

}  // extern "C"
