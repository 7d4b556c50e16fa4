/*
 * gp_oracle.h -- CPU restatement of the reference's serial grand-potential
 * step.  TEST INFRASTRUCTURE: used only by tests/, by __graft_entry__.smoke()
 * as the checker, and by bench.py's cpu_baseline leg.  The product (libgp)
 * never links or calls it.
 */
#ifndef GP_ORACLE_H_
#define GP_ORACLE_H_

#include "gp.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gpo gpo;

/* recip_div = 0: reciprocals inside matinvnew use pow(x,-1) like the reference
 * (matrix.h:121,127); recip_div = 1: IEEE division 1.0/x (what the CUDA path
 * does, since a correctly rounded division is the only reciprocal a GPU can
 * reproduce exactly).  Only the smoothing pass and the K>2 general inversion
 * use matinvnew per cell. */
gpo *gpo_create(const gp_params *p, int recip_div, char *err, int errlen);
void gpo_destroy(gpo *o);
void gpo_dims(const gpo *o, long *rows_x, long *rows_y);
int gpo_set(gpo *o, const double *phi, const double *mu);      /* interior; applies BCs */
void gpo_get(const gpo *o, double *phi, double *mu);           /* interior */
void gpo_get_full(const gpo *o, double *phi, double *mu, double *dphi); /* ghosted */
/* interior temperature field [mx][my] (gridinfo[].temperature); T when isothermal */
void gpo_temperature(const gpo *o, double *T);
void gpo_smooth(gpo *o, long nsteps);
void gpo_step(gpo *o, long nsteps);
void gpo_stats(const gpo *o, gp_stats *s);
/* derived constants, for pinning the host derivation: cmu[a][i][j] (N*K*K),
 * B[a][i] (N*K), C[a] (N), Beq (N*K), dBbdT (N*K), R (N*N*9), Rinv (N*N*9) */
void gpo_consts(const gpo *o, double *cmu, double *B, double *C, double *Beq,
                double *dBbdT, double *R, double *Rinv);

#ifdef __cplusplus
}
#endif
#endif
