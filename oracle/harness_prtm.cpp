/* Test infrastructure only (the oracle): the reference's prestack LSRTM
 * operator (src/unused/prtm2d.cpp) compiled in place, in this translation
 * unit so that its file-scope state is reachable, behind C entry points.
 * The reference never built this file; shim/prtm2d.h supplies the header it
 * includes and sf_adjnull below the one library function its tree lacks.
 * Nothing here is shipped or measured as the product. */
#include <float.h>
#include <math.h>
#include <stdbool.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/types.h>
#include <unistd.h>
/* rsf.h declares most of the library outside its extern "C" blocks; the
 * library (the C files of src/rsf) is C, so the header is read as C here.  The
 * system headers it pulls in come first, under their own linkage. */
extern "C" {
#include <rsf.h>
}

/* sf_adjnull (declared at src/rsf/rsf.h:417, not defined in the tree): a
 * linear operator's output starts at zero unless add is set. */
void sf_adjnull(bool adj, bool add, int nx, int ny, float *x, float *y) {
  if (add) return;
  if (adj) memset(x, 0, sizeof(float) * (size_t)nx);
  else memset(y, 0, sizeof(float) * (size_t)ny);
}

#include "prtm2d.cpp"

extern "C" {

/* prtm2d_init (:241-338) with the velocity as vel[ix*nz + iz].  The
 * receiver-side fields gp0/gp1 come from malloc and the Born branch never
 * clears them (:408-434); they are cleared here so that a first Born call
 * is defined. */
void ref_prtm_init(int csdgather, float dz, float dx, float dt, float amp, float fm, int nz, int nx, int nb,
                   int nt, int ns, int ng, int sxbeg, int szbeg, int jsx, int jsz, int gxbeg, int gzbeg, int jgx,
                   int jgz, const float *vel) {
  float **v0 = (float **)malloc(sizeof(float *) * (size_t)nx);
  for (int ix = 0; ix < nx; ix++) v0[ix] = (float *)vel + (size_t)ix * nz;
  prtm2d_init(false, csdgather != 0, dz, dx, dt, amp, fm, nz, nx, nb, nt, ns, ng, sxbeg, szbeg, jsx, jsz, gxbeg,
              gzbeg, jgx, jgz, v0, NULL, NULL);
  free(v0);
  memset(gp0[0], 0, sizeof(float) * (size_t)nzpad * nxpad);
  memset(gp1[0], 0, sizeof(float) * (size_t)nzpad * nxpad);
}

/* prtm2d_lop (:354-437) */
void ref_prtm_lop(int adj, int add, int nm, int nd, float *mod_, float *dat_) {
  prtm2d_lop(adj != 0, add != 0, nm, nd, mod_, dat_);
}

/* zero the receiver-side fields (what a per-shot operator starts from) */
void ref_prtm_clear() {
  memset(gp0[0], 0, sizeof(float) * (size_t)nzpad * nxpad);
  memset(gp1[0], 0, sizeof(float) * (size_t)nzpad * nxpad);
}

/* error.c's sf_error closes the RSF files; this library opens none */
void sf_close(void) {}


/* prtm2d_close (:340-352), plus the boundary store it does not free */
void ref_prtm_close() {
  prtm2d_close();
  free(rwbndr);
  rwbndr = NULL;
}

}  // extern "C"
