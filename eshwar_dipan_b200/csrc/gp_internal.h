/*
 * gp_internal.h -- definitions shared by the host C code and the CUDA side of
 * libgp (not part of the public ABI).
 */
#ifndef GP_INTERNAL_H_
#define GP_INTERNAL_H_

#include "gp.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Kernel limits. */
#define GPK_MAXN 4
#define GPK_MAXK 2

/* Mode of the interface dc/dmu inversion (calculate_divergence_concentration.h:238-270). */
enum { GP_INV_BINARY = 1, GP_INV_TERNARY = 2, GP_INV_DILUTE = 3, GP_INV_GENERAL = 4 };

/*
 * Constants the step needs, derived once on the host from gp_params exactly as
 * the reference derives them (init_propertymatrices, functionF_01.h:169-230;
 * initialize_variables.h:4-28; populate_rotation_matrix,
 * utility_functions.h:700-774).  Products of constants that the reference
 * evaluates in the same order on every call are folded here; each fold keeps the
 * reference's operation order so the folded value is bit-identical.
 */
typedef struct gp_derived {
  int N, K;
  long mx, my;                            /* MESH_X, MESH_Y */
  double dx, dy, dt;
  double eps, inv_eps;                    /* epsilon, 1.0/epsilon */
  double tau;                             /* scalar tau of FunctionTau */
  double c16pi2;                          /* 16.0/(M_PI*M_PI)  functionW_01.h:22 */
  double jat_obst;                        /* -0.25*M_PI*epsilon calculate_divergence_concentration.h:53 */
  double jat_well;                        /* -1.0*epsilon               ...:57 */
  double well_half;                       /* 0.5/sqrt(2.0)  calculate_fluxes_concentration.h:89 */
  int obstacle, well, aniso, inv_mode;
  double gamma[GPK_MAXN][GPK_MAXN];
  double gamma_abc[GPK_MAXN][GPK_MAXN][GPK_MAXN];
  double tau_ab[GPK_MAXN][GPK_MAXN];
  double dab16[GPK_MAXN][GPK_MAXN];       /* 16.0*dab  anisotropy_01.h:20 */
  double dab[GPK_MAXN][GPK_MAXN];
  double rot[GPK_MAXN][GPK_MAXN][2][2];   /* Rotation_matrix[a][b] (after the LU round trip) */
  double rinv[GPK_MAXN][GPK_MAXN][2][2];  /* Inv_Rotation_matrix[a][b] */
  int rot_identity;                       /* all pairs rotate by the identity */
  double cmu[GPK_MAXN][GPK_MAXK][GPK_MAXK];
  double E[GPK_MAXN][GPK_MAXK];           /* Beq + dBbdT*(T-Teq)  functionF_01.h:22,34 */
  double twoA[GPK_MAXN][GPK_MAXK];        /* 2.0*A[a][i][i]  functionF_01.h:22 */
  double A[GPK_MAXN][GPK_MAXK][GPK_MAXK];
  double B[GPK_MAXN][GPK_MAXK];           /* B at T  */
  double C[GPK_MAXN];                     /* C at T  */
  double DC[GPK_MAXN][GPK_MAXK][GPK_MAXK][GPK_MAXK]; /* Diffusivity[b][i][k]*cmu[b][k][j] -> [b][i][j][k] */
  double atf[GPK_MAXN][GPK_MAXK];         /* 1.0 - D[a][k][k]/D[N-1][k][k] */
  double Dbulk[GPK_MAXN][GPK_MAXK][GPK_MAXK]; /* D_kl of a cell with phi = e_p, summed as functionD.h does */
  /* boundary index maps along x and y: ghosted index -> ghosted index; per field */
  int bc_x[2][2], bc_y[2][2];             /* [field phi/mu][low/high side] type (1 or 3) */
  /* non-isothermal runs (ISOTHERMAL = 0): the temperature field
   * T = temp_bottom + y*GRADIENT of apply_temperature_gradientY
   * (Temperature_gradient.h:4-29) and what a cell needs at its temperature:
   * E = Beq + dBbdT*(T-Teq) (functionF_01.h:22,34) and B, C of
   * function_B/function_C (functionF_01.h:62-104) */
  int tgrad;
  double Teq;
  double Beq[GPK_MAXN][GPK_MAXK], dBbdT[GPK_MAXN][GPK_MAXK];
  double ceql[GPK_MAXN][GPK_MAXK], ceqs[GPK_MAXN][GPK_MAXK], DCk[GPK_MAXN][GPK_MAXK];
  double DTl[GPK_MAXN], DTs[GPK_MAXN];
  double tg_base, tg_dT, tg_dist, tg_off, tg_vel;   /* Tempgrady = {base, DeltaT, Distance, OFFSET, velocity} */
  int bc_t[2];                                       /* T's boundary types along y [low/high side] */
  /* moving frame (Shift = 1, shift.h:4-66) */
  int shift;
  long shiftj;
  double mu_fill[GPK_MAXK];                         /* Mu(cfill of the liquid, Tfill) of the cells shifted in */
} gp_derived;

/* Host restatement of matinvnew (matrix.h:50-218): LU with the reference's
 * partial pivoting, inverse by forward/back substitution with pow(x,-1), and the
 * reference's write-back of the reconstructed product into m.  n <= 3. */
void gp_host_matinv(double m[3][3], double inv[3][3], int n);

/* Derive constants; returns GP_OK or GP_EINVAL with a message in err. */
int gp_host_derive(const gp_params *p, gp_derived *d, char *err, size_t errlen);

/* Reference Mu() at temperature Tc (functionF_01.h:19-29) with the property
 * matrices evaluated at Tq (the filling evaluates both at Teq). */
void gp_host_property_matrices(const gp_params *p, double Tq,
                               double B[GP_MAX_PHASES][GP_MAX_COMP], double C[GP_MAX_PHASES],
                               double cmu[GP_MAX_PHASES][GP_MAX_COMP][GP_MAX_COMP],
                               double Beq[GP_MAX_PHASES][GP_MAX_COMP],
                               double dBbdT[GP_MAX_PHASES][GP_MAX_COMP]);

/* The reference's temperature of each interior column [MESH_Y] of a
 * non-isothermal run after `steps` steps, laid down with shift_OFFSET =
 * shift_off and then moved by a frame shift of dshift cells (0: none). */
void gp_host_temperature_column(const gp_derived *d, long long steps, long long shift_off, long dshift, double *Ty);

void gp_set_thread_error(const char *fmt, ...);

#ifdef __cplusplus
}
#endif
#endif
