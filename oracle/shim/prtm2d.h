/* Declarations of src/unused/prtm2d.cpp's functions.  The reference tree
 * does not carry this header (the operator was never built there); the
 * oracle's harness compiles prtm2d.cpp in place against it.  Test
 * infrastructure only. */
#ifndef SWFWI_ORACLE_PRTM2D_H
#define SWFWI_ORACLE_PRTM2D_H

void boundary_rw(float **p, float *spo, bool read);
void step_forward(float **u0, float **u1, float **vv, bool adj);
void apply_sponge(float **p0);
void sg_init(int *sxz, int szbeg, int sxbeg, int jsz, int jsx, int ns);
void add_source(int *sxz, float **p, int ns, float *source, bool add);
void expand2d(float **b, float **a);
void window2d(float **a, float **b);
void prtm2d_init(bool verb_, bool csdgather_, float dz_, float dx_, float dt_, float amp, float fm, int nz_,
                 int nx_, int nb_, int nt_, int ns_, int ng_, int sxbeg_, int szbeg_, int jsx_, int jsz_,
                 int gxbeg_, int gzbeg_, int jgx_, int jgz_, float **v0, float *mod_, float *dat_);
void prtm2d_close();
void prtm2d_lop(bool adj, bool add, int nm, int nd, float *mod, float *dat);

#endif
