/* The oracle (test infrastructure only; never linked into the product).
 *
 * Plain-C restatement of swfwi's 4th-order-time / 10th-order-space acoustic
 * step, written from the reference's formulas:
 *   src/modeling/fd4t10s-damp-zjh.c:14-115  (damped, sponge on left/right/bottom)
 *   src/modeling/fd4t10s-zjh.c:10-56        (undamped)
 * Layout p[ix*nz + iz], z fastest; nx, nz are padded sizes; vel is the
 * transformed velocity vt = dx^2/(v^2 dt^2); nb is the sponge width plus the
 * 6-cell halo (Damp4t10d's bx0).  prev is overwritten in place with the next
 * field on [6, n-6); everything outside keeps its old value.
 *
 * Two arithmetics:
 *  - fdo_step_ref: float storage with the reference's own mixed float/double
 *    expression order (its literals 4.0, 2. promote the running sums to
 *    double).  Compiled with -ffp-contract=off this reproduces the reference
 *    bit for bit, which the tests check against the compiled reference.
 *  - fdo_step_f64: the same scheme entirely in double, the FP64 oracle.
 *
 * Also: fdo_forward_f64 / fdo_gradient_f64, double-precision restatements of
 * Damp4t10d::FwiForwardModeling (damp4t10d.cpp:272-289) and the per-shot
 * calgradient (src/fwi/fwiframework.cpp:114-177) for one source and a
 * receiver list, used to state errors against FP64. */
#include <math.h>
#include <stdlib.h>
#include <string.h>

static const float ZA[6] = {+1.53400796f, +1.78858721f, -0.31660756f,
                            +0.07612173f, -0.01626042f, +0.00216736f};

/* Sponge ramp of fd4t10s-damp-zjh.c:64-80 (bottom overrides left/right). */
static float damp_dist(int ix, int iz, int nx, int nz, int nb) {
  float dist = 0.0f;
  if (ix < nb) dist = (float)(nb - ix) / (float)nb;
  if (ix >= nx - nb) dist = (float)(ix - (nx - nb) + 1) / (float)nb;
  if (iz >= nz - nb) dist = (float)(iz - (nz - nb) + 1) / (float)nb;
  return dist;
}

void fdo_step_ref(float *prev, const float *curr, const float *vel, int nx, int nz, int nb,
                  int damped) {
  float *u2 = (float *)calloc((size_t)nx * nz, sizeof(float));
  for (int ix = 5; ix < nx - 5; ix++) {
    for (int iz = 5; iz < nz - 5; iz++) {
      const float *c = curr + (size_t)ix * nz + iz;
      double acc = (-4.0 * (double)ZA[0]) * (double)c[0];
      for (int k = 1; k <= 5; k++) {
        float s = c[-k] + c[k];
        s = s + c[-k * nz];
        s = s + c[k * nz];
        acc = acc + (double)(ZA[k] * s);
      }
      u2[(size_t)ix * nz + iz] = (float)acc;
    }
  }
  for (int ix = 6; ix < nx - 6; ix++) {
    for (int iz = 6; iz < nz - 6; iz++) {
      size_t p = (size_t)ix * nz + iz;
      float r = 1.0f / vel[p];
      float lap = u2[p - 1] + u2[p + 1];
      lap = lap + u2[p - nz];
      lap = lap + u2[p + nz];
      lap = lap - 4.0f * u2[p];
      float t4 = ((1.0f / 12.0f) * r) * r;
      t4 = t4 * lap;
      double acc;
      if (damped) {
        float delta = (0.05f * damp_dist(ix, iz, nx, nz, nb));
        delta = delta * damp_dist(ix, iz, nx, nz, nb);
        double coef = (2.0 - (double)(2.0f * delta)) + (double)(delta * delta);
        acc = coef * (double)curr[p];
        acc = acc - (double)((1.0f - 2.0f * delta) * prev[p]);
      } else {
        acc = 2.0 * (double)curr[p];
        acc = acc - (double)prev[p];
      }
      acc = acc + (double)(r * u2[p]);
      acc = acc + (double)t4;
      prev[p] = (float)acc;
    }
  }
  free(u2);
}

void fdo_step_f64(double *prev, const double *curr, const double *vel, int nx, int nz, int nb,
                  int damped) {
  double *u2 = (double *)calloc((size_t)nx * nz, sizeof(double));
  for (int ix = 5; ix < nx - 5; ix++) {
    for (int iz = 5; iz < nz - 5; iz++) {
      const double *c = curr + (size_t)ix * nz + iz;
      double acc = -4.0 * (double)ZA[0] * c[0];
      for (int k = 1; k <= 5; k++) acc += (double)ZA[k] * (c[-k] + c[k] + c[-k * nz] + c[k * nz]);
      u2[(size_t)ix * nz + iz] = acc;
    }
  }
  for (int ix = 6; ix < nx - 6; ix++) {
    for (int iz = 6; iz < nz - 6; iz++) {
      size_t p = (size_t)ix * nz + iz;
      double r = 1.0 / vel[p];
      double lap = u2[p - 1] + u2[p + 1] + u2[p - nz] + u2[p + nz] - 4.0 * u2[p];
      double delta = 0.0;
      if (damped) {
        double d = (double)damp_dist(ix, iz, nx, nz, nb);
        delta = 0.05 * d * d;
      }
      prev[p] = (2.0 - 2.0 * delta + delta * delta) * curr[p] - (1.0 - 2.0 * delta) * prev[p] +
                r * u2[p] + (1.0 / 12.0) * r * r * lap;
    }
  }
  free(u2);
}

/* Single-shot forward modelling in double.  Source at padded index src_pos,
 * receivers at padded indices rec_pos[0..ng).  Records the current field
 * (with this step's source added) at every step, as
 * Damp4t10d::FwiForwardModeling does after its swap. */
void fdo_forward_f64(const double *vel, int nx, int nz, int nb, int nt, const double *wlt,
                     int src_pos, const int *rec_pos, int ng, double *dcal) {
  size_t n = (size_t)nx * nz;
  double *p0 = (double *)calloc(n, sizeof(double));
  double *p1 = (double *)calloc(n, sizeof(double));
  for (int it = 0; it < nt; it++) {
    p1[src_pos] += wlt[it];
    fdo_step_f64(p0, p1, vel, nx, nz, nb, 1);
    double *t = p0; p0 = p1; p1 = t;
    for (int ig = 0; ig < ng; ig++) dcal[(size_t)it * ng + ig] = p0[rec_pos[ig]];
  }
  free(p0);
  free(p1);
}

/* Boundary strips of Damp4t10d::writeBndry/readBndry (damp4t10d.cpp:478-536):
 * a 6-wide ring just outside the interior, bottom [ix][iz] then left then
 * right.  bx0 = sponge width + 6; bz0 = 6; the strip has
 * 6*((nx - 2*(bx0-6)) + 2*(nz - 6 - bx0)) values. */
static void strip_io_f64(double *bndr, double *p, int nx, int nz, int bx0, int write) {
  int w = 6, nxs = nx - 2 * (bx0 - w), nzs = nz - 6 - bx0;
  for (int ix = 0; ix < nxs; ix++)
    for (int iz = 0; iz < w; iz++) {
      double *q = p + (size_t)(ix + bx0 - w) * nz + (nz - bx0 + iz);
      if (write) bndr[iz + w * ix] = *q; else *q = bndr[iz + w * ix];
    }
  for (int iz = 0; iz < nzs; iz++)
    for (int ix = 0; ix < w; ix++) {
      double *l = p + (size_t)(bx0 - w + ix) * nz + (6 + iz);
      double *r = p + (size_t)(nx - bx0 + ix) * nz + (6 + iz);
      double *bl = bndr + w * nxs + iz + nzs * ix;
      double *br = bndr + w * nxs + iz + nzs * (ix + w);
      if (write) { *bl = *l; *br = *r; } else { *l = *bl; *r = *br; }
    }
}

int fdo_strip_size(int nx, int nz, int bx0) { return 6 * ((nx - 2 * (bx0 - 6)) + 2 * (nz - 6 - bx0)); }

/* Per-shot adjoint gradient in double: the scheme of
 * src/fwi/fwiframework.cpp:114-177 step for step (strip save on the way
 * forward, undamped back-stepping with strip restore, the reference's
 * subSource on the reconstructed field, damped receiver propagation,
 * g -= s*r*w with w = 1 above 0.4 s, a ramp on (0.3, 0.4] s, stop at or
 * below 0.3 s). */
void fdo_gradient_f64(const double *vel, int nx, int nz, int nb, int nt, double dt,
                      const double *wlt, int src_pos, const int *rec_pos, int ng,
                      const double *vsrc, double *g) {
  size_t n = (size_t)nx * nz;
  int bs = fdo_strip_size(nx, nz, nb);
  double *bndr = (double *)calloc((size_t)bs * nt, sizeof(double));
  double *sp0 = (double *)calloc(n, sizeof(double));
  double *sp1 = (double *)calloc(n, sizeof(double));
  double *gp0 = (double *)calloc(n, sizeof(double));
  double *gp1 = (double *)calloc(n, sizeof(double));
  double *t;
  for (int it = 0; it < nt; it++) {
    sp1[src_pos] += wlt[it];
    fdo_step_f64(sp0, sp1, vel, nx, nz, nb, 1);
    t = sp0; sp0 = sp1; sp1 = t;
    strip_io_f64(bndr + (size_t)bs * it, sp0, nx, nz, nb, 1);
  }
  for (int it = nt - 1; it >= 0; it--) {
    strip_io_f64(bndr + (size_t)bs * it, sp0, nx, nz, nb, 0);
    t = sp0; sp0 = sp1; sp1 = t;
    fdo_step_f64(sp0, sp1, vel, nx, nz, nb, 0);
    sp0[src_pos] -= wlt[it];
    for (int ig = 0; ig < ng; ig++) gp1[rec_pos[ig]] += vsrc[(size_t)it * ng + ig];
    fdo_step_f64(gp0, gp1, vel, nx, nz, nb, 1);
    t = gp0; gp0 = gp1; gp1 = t;
    /* the reference passes the taper as a float (cross_correlation's
     * scale parameter): t = dt*it in float, the ramp rounded to float */
    double tt = (double)(float)((float)dt * (float)it), w;
    if (tt > 0.4) w = 1.0;
    else if (tt > 0.3) w = (double)(float)((tt - 0.3) / 0.1);
    else break;
    for (size_t i = 0; i < n; i++) g[i] -= sp0[i] * gp0[i] * w;
  }
  free(bndr); free(sp0); free(sp1); free(gp0); free(gp1);
}
