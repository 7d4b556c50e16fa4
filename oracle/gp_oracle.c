/*
 * gp_oracle.c -- CPU restatement of the reference's serial grand-potential
 * finite-difference step (Grand_potential_Finite_difference_2D_serial).
 *
 * TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA path (tests/,
 * __graft_entry__.smoke()) and the "port" CPU baseline of bench.py.  Nothing in
 * the product links or calls this file.
 *
 * The reference sweeps rows with a rolling 4-row gradient ring and updates the
 * grid in place, but every value it reads is either precomputed from the old
 * state or belongs to a row not yet updated, so the step is a pure Jacobi
 * update.  This restatement computes the same quantities as whole-grid arrays:
 *   1. face quantities of every cell (the reference's struct gradlayer),
 *   2. delta-phi of every cell the reference updates,
 *   3. anti-trapping fluxes, then mu and phi of every cell it updates,
 *   4. the boundary copies.
 * Entries the reference never writes (ring slots read before they are filled)
 * are set to NaN here, so any result that depended on them would show up as NaN
 * in the interior; only ghost cells read them, and the boundary copies overwrite
 * those.  Arithmetic follows the reference expression by expression (same
 * operands, same association); it must be compiled without FMA contraction.
 */
#include "gp_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define MAXN GP_MAX_PHASES
#define MAXK GP_MAX_COMP

struct gpo {
  int N, K;
  long mx, my, rx, ry, n;
  int obstacle, well, aniso, inv_mode, recip_div;
  double dx, dy, dt, eps, tau;
  double T, Teq;
  /* non-isothermal runs (ISOTHERMAL = 0, Tempgrady): the temperature of every
   * ghosted cell, its gradient parameters and the phase-diagram constants of
   * function_B/function_C at a temperature (functionF_01.h:62-104) */
  int tgrad;
  double *Tc, *Tstep;   /* the field now, and the field the last step used */
  double tg_base, tg_dT, tg_dist, tg_off, tg_vel;
  double ceq_l[MAXN][MAXK], ceq_s[MAXN][MAXK], DT_l[MAXN], DT_s[MAXN], DC[MAXN][MAXK];
  /* moving frame (Shift = 1): shift every 100 steps when the interface passes
   * column shiftj (microsim_gp.c:115-126, shift.h:4-66) */
  int shift;
  long shiftj, shift_off, last_shift;
  double Tfill, cfill_l[MAXK];
  long tstep;   /* time steps since gpo_create: the reference main's t */
  double gamma[MAXN][MAXN], gabc[MAXN][MAXN][MAXN], tau_ab[MAXN][MAXN], dab[MAXN][MAXN];
  double diff[MAXN][MAXK][MAXK], A[MAXN][MAXK][MAXK];
  double cmu[MAXN][MAXK][MAXK], B[MAXN][MAXK], C[MAXN], Beq[MAXN][MAXK], dBbdT[MAXN][MAXK];
  double R[MAXN][MAXN][3][3], Rinv[MAXN][MAXN][3][3];
  int bctype[3][4];          /* [phi/mu/T][face X-, X+, Y+, Y-] */
  /* state, ghosted [field][x*ry+y] */
  double *phi, *mu, *dphi;
  /* face quantities */
  double *gx, *sx, *gy, *sy, *gcx, *gcy;   /* [N][n] */
  double *gmx, *gmy;                       /* [K][n] */
  double *Dmx, *Dmy;                       /* [K*K][n] */
  double *jx, *jy;                         /* [K][n] */
  double *sdphi;                           /* smoothing delta-phi [N][n] */
  double *nphi, *nmu;                      /* next state */
  /* progress record over the interior (see gp_stats) */
  double phi_max[MAXN], phi_min[MAXN], mu_max[MAXK], mu_min[MAXK];
  double rel_phi[MAXN], rel_mu[MAXK];
  long long steps;
};

#define I(o, x, y) ((long)(x) * (o)->ry + (y))
#define F(arr, o, a) ((arr) + (long)(a) * (o)->n)

/* ------------------------------------------------------------ matinvnew */

/* matinvnew (matrix.h:50-218) for n <= 3, with the reference's pivot rule,
 * its write-back of the reconstructed product into m, and pow(x,-1) or 1.0/x
 * as the reciprocal. */
static void o_matinv(double m[3][3], double inv[3][3], int n, int recip_div) {
  double fac[3][3] = {{0}}, inv1[3][3], prod[3][3], v1[3], v[3];
  int tag[3], i, j, k;
  for (k = 0; k < n; k++) tag[k] = k;
  for (k = 0; k < n; k++) {
    double big = fabs(m[k][k]);
    int t1 = k, s;
    for (i = k + 1; i < n; i++)
      if (fabs(m[i][k]) > big) { t1 = i; big = m[i][k]; }       /* matrix.h:169-173 */
    s = tag[k]; tag[k] = tag[t1]; tag[t1] = s;
    for (i = 0; i < n; i++) { double w = m[k][i]; m[k][i] = m[t1][i]; m[t1][i] = w; }
    for (i = 0; i < k; i++) { double w = fac[k][i]; fac[k][i] = fac[t1][i]; fac[t1][i] = w; }
    for (i = k + 1; i < n; i++) {
      double f = -m[i][k] / m[k][k];                            /* matrix.h:67-71 */
      fac[i][k] = -f;
      for (j = k; j <= n - 1; j++) m[i][j] = f * m[k][j] + m[i][j];
    }
  }
  for (i = 0; i < n; i++)
    for (j = 0; j < n; j++) {
      if (i == j) fac[i][j] = 1;
      if (j > i) fac[i][j] = 0;
    }
  for (i = 0; i < n; i++) {
    int r;
    double s;
    v1[0] = (i == 0) ? 1.0 : 0.0;                                /* substitutef */
    for (r = 1; r < n; r++) {
      s = 0;
      for (j = 0; j < r; j++) s = s - fac[r][j] * v1[j];
      v1[r] = ((r == i) ? 1.0 : 0.0) + s;
    }
    v[n - 1] = v1[n - 1] * (recip_div ? 1.0 / m[n - 1][n - 1] : pow(m[n - 1][n - 1], -1));
    for (r = n - 2; r >= 0; r--) {                              /* substituteb */
      s = 0;
      for (j = r + 1; j < n; j++) s = s - m[r][j] * v[j];
      v[r] = (v1[r] + s) * (recip_div ? 1.0 / m[r][r] : pow(m[r][r], -1));
    }
    for (j = 0; j < n; j++) inv1[j][i] = v[j];
  }
  for (j = 0; j < n; j++)                                        /* colswap */
    for (i = 0; i < n; i++) inv[i][tag[j]] = inv1[i][j];
  for (k = 0; k < n; k++)                                        /* multiply2d */
    for (i = 0; i < n; i++) {
      double s = 0;
      for (j = 0; j < n; j++) s = s + fac[k][j] * m[j][i];
      prod[k][i] = s;
    }
  for (j = 0; j < n; j++)                                        /* rowswap */
    for (i = 0; i < n; i++) m[tag[j]][i] = prod[j][i];
}

/* ------------------------------------------------------- constants */

static void o_rotation(const double ang[3], double R[3][3], double Ri[3][3]) {
  /* get_Rotation_Matrix x3, multiply2d twice, matinvnew
   * (utility_functions.h:655-751) */
  double Rm[3][3][3], M[3][3];
  int ax, i, j, k;
  for (ax = 0; ax < 3; ax++) {
    double c = cos(ang[ax] * M_PI / 180.0), s = sin(ang[ax] * M_PI / 180.0);
    double (*r)[3] = Rm[ax];
    for (i = 0; i < 3; i++)
      for (j = 0; j < 3; j++) r[i][j] = 0.0;
    if (ax == 0) { r[0][0] = 1.0; r[1][1] = c; r[1][2] = -s; r[2][1] = s; r[2][2] = c; }
    if (ax == 1) { r[0][0] = c; r[0][2] = s; r[2][0] = -s; r[1][1] = 1.0; r[2][2] = c; }
    if (ax == 2) { r[0][0] = c; r[0][1] = -s; r[1][0] = s; r[1][1] = c; r[2][2] = 1.0; }
  }
  for (k = 0; k < 3; k++)
    for (i = 0; i < 3; i++) {
      double s = 0;
      for (j = 0; j < 3; j++) s = s + Rm[0][k][j] * Rm[1][j][i];
      M[k][i] = s;
    }
  for (k = 0; k < 3; k++)
    for (i = 0; i < 3; i++) {
      double s = 0;
      for (j = 0; j < 3; j++) s = s + M[k][j] * Rm[2][j][i];
      R[k][i] = s;
    }
  o_matinv(R, Ri, 3, 0);
}

/* cmu = inverse of muc (initialize_variables.h:6-17, functionF_01.h:184-197) */
static void o_props(gpo *o) {
  int a, i, j, K = o->K;
  for (a = 0; a < o->N; a++) {
    double m[3][3] = {{0}}, v[3][3] = {{0}};
    for (i = 0; i < K; i++)
      for (j = 0; j < K; j++) m[i][j] = (i == j) ? 2.0 * o->A[a][i][j] : o->A[a][i][j];
    o_matinv(m, v, K, 0);
    for (i = 0; i < K; i++)
      for (j = 0; j < K; j++) o->cmu[a][i][j] = v[i][j];
  }
}

static void o_props_full(gpo *o, const gp_params *p) {
  int N = o->N, K = o->K, L = N - 1, a, i, j, k, pass;
  double DT[MAXN][MAXN] = {{0}}, DC[MAXN][MAXK] = {{0}}, dcb_s[MAXN][MAXK] = {{0}}, dcb_l[MAXN][MAXK] = {{0}};
  o_props(o);
  for (a = 0; a < L; a++) {
    DT[a][L] = 0.0;
    DT[a][a] = 0.0;
    for (k = 0; k < K; k++) {
      DT[a][a] += p->slopes[a][a][k] * (p->ceq[a][L][k] - p->ceq[a][a][k]);
      DT[a][L] += p->slopes[a][L][k] * (p->ceq[a][L][k] - p->ceq[a][a][k]);
      DC[a][k] = p->ceq[a][L][k] - p->ceq[a][a][k];
    }
    for (k = 0; k < K; k++) {
      dcb_s[a][k] = DC[a][k] / DT[a][a];
      dcb_l[a][k] = DC[a][k] / DT[a][L];
    }
    for (k = 0; k < K; k++) {
      o->dBbdT[a][k] = 2.0 * (o->A[L][k][k] * dcb_l[a][k] - o->A[a][k][k] * dcb_s[a][k]);
      for (i = 0; i < K; i++)
        if (k != i) o->dBbdT[a][k] += (o->A[L][k][i] * dcb_l[a][i] - o->A[a][k][i] * dcb_s[a][i]);
    }
  }
  for (k = 0; k < K; k++) o->dBbdT[L][k] = 0.0;
  for (pass = 0; pass < 2; pass++) {          /* function_B at Teq, then B, C at T */
    double Tb = pass == 0 ? o->Teq : o->T;
    for (a = 0; a < N; a++) {
      double cl[MAXK] = {0}, cs[MAXK] = {0}, sc;
      if (a != L)
        for (k = 0; k < K; k++) {
          cl[k] = p->ceq[a][L][k] - (DC[a][k]) * (o->Teq - Tb) / (DT[a][L]);
          cs[k] = p->ceq[a][a][k] - (DC[a][k]) * (o->Teq - Tb) / (DT[a][a]);
        }
      for (i = 0; i < K; i++) {
        double bai = 0.0;
        sc = 0.0;
        if (a != L) {
          for (k = 0; k < K; k++)
            if (k != i) sc += o->A[L][k][i] * cl[k] - o->A[a][k][i] * cs[k];
          bai = (2.0 * (o->A[L][i][i] * cl[i] - o->A[a][i][i] * cs[i]) + sc);
        }
        if (pass == 0) o->Beq[a][i] = bai; else o->B[a][i] = bai;
      }
      if (pass == 1) {
        sc = 0.0;
        if (a != L)
          for (i = 0; i < K; i++)
            for (j = 0; j < K; j++)
              if (i <= j) sc += (o->A[a][i][j] * cs[i] * cs[j] - o->A[L][i][j] * cl[i] * cl[j]);
        o->C[a] = sc;
      }
    }
  }
}

/* --------------------------------------------------- thermodynamics */

/* hphi, dhphi (functionH.h:1-36).  o_dh(ph, b, a) = d h_b / d phi_a. */
static double o_h(const gpo *o, const double *ph, int a) {
  int b, c;
  double s1 = 0.0, s = 3.0 * ph[a] * ph[a] - 2.0 * ph[a] * ph[a] * ph[a];
  for (b = 0; b < o->N; b++)
    for (c = 0; c < o->N; c++)
      if (b != a && c != a && b < c) s1 += ph[b] * ph[c];
  s1 *= 2.0 * ph[a];
  return s + s1;
}

static double o_dh(const gpo *o, const double *ph, int b, int a) {
  int e, f;
  double s = 0.0;
  if (a == b) {
    s = 6.0 * ph[a] * (1.0 - ph[a]);
    for (e = 0; e < o->N; e++)
      for (f = 0; f < o->N; f++)
        if (e != b && f != b && e < f) s += 2.0 * ph[e] * ph[f];
  } else {
    for (e = 0; e < o->N; e++)
      if (e != b && e != a) s += 2.0 * ph[e];
    s *= ph[b];
  }
  return s;
}

/* c_mu, Mu, free_energy (functionF_01.h:5-37) at temperature T */
static double o_cmu(const gpo *o, const double *m, double T, int a, int i) {
  int k;
  double s = 0.0;
  for (k = 0; k < o->K; k++) s += o->cmu[a][i][k] * (m[k] - (o->Beq[a][k] + o->dBbdT[a][k] * (T - o->Teq)));
  return s;
}

static double o_Mu(const gpo *o, const double *c, double T, int a, int i) {
  int j;
  double s = 2.0 * o->A[a][i][i] * c[i] + (o->Beq[a][i] + o->dBbdT[a][i] * (T - o->Teq));
  for (j = 0; j < o->K; j++)
    if (i != j) s += o->A[a][i][j] * c[j];
  return s;
}

static double o_fe(const gpo *o, const double *c, int a, const double B[][MAXK], const double *C) {
  int i, j;
  double s = 0.0;
  for (i = 0; i < o->K; i++) {
    for (j = 0; j < o->K; j++)
      if (i <= j) s += o->A[a][i][j] * c[i] * c[j];
    s += B[a][i] * c[i];
  }
  s += C[a];
  return s;
}

/* B and C of every phase at temperature T: function_B / function_C
 * (functionF_01.h:62-104), as init_propertymatrices(T) sets them
 * (functionF_01.h:169-230) */
static void o_BC(const gpo *o, double T, double B[][MAXK], double *C) {
  int a, i, j, k, L = o->N - 1;
  for (a = 0; a < o->N; a++) {
    double cl[MAXK] = {0}, cs[MAXK] = {0}, sc;
    for (i = 0; i < o->K; i++) {
      sc = 0.0;
      B[a][i] = 0.0;
      if (a != L) {
        for (k = 0; k < o->K; k++) {
          cl[k] = o->ceq_l[a][k] - (o->DC[a][k]) * (o->Teq - T) / (o->DT_l[a]);
          cs[k] = o->ceq_s[a][k] - (o->DC[a][k]) * (o->Teq - T) / (o->DT_s[a]);
          if (k != i) sc += o->A[L][k][i] * cl[k] - o->A[a][k][i] * cs[k];
        }
        B[a][i] = (2.0 * (o->A[L][i][i] * cl[i] - o->A[a][i][i] * cs[i]) + sc);
      }
    }
    sc = 0.0;
    if (a != L) {
      for (k = 0; k < o->K; k++) {
        cl[k] = o->ceq_l[a][k] - (o->DC[a][k]) * (o->Teq - T) / (o->DT_l[a]);
        cs[k] = o->ceq_s[a][k] - (o->DC[a][k]) * (o->Teq - T) / (o->DT_s[a]);
      }
      for (i = 0; i < o->K; i++)
        for (j = 0; j < o->K; j++)
          if (i <= j) sc += (o->A[a][i][j] * cs[i] * cs[j] - o->A[L][i][j] * cl[i] * cl[j]);
    }
    C[a] = sc;
  }
}

/* temperature of a ghosted cell: the field of a non-isothermal run, else T */
static double o_Tcell(const gpo *o, long c) { return o->tgrad ? o->Tc[c] : o->T; }

/* dpsi (functionF_01.h:41-57) at temperature T with B, C at T */
static double o_dpsi(const gpo *o, const double *m, double T, const double *ph, int a, const double B[][MAXK],
                     const double *C) {
  int b, k;
  double s = 0.0;
  for (b = 0; b < o->N; b++) {
    double c[MAXK], psi = 0.0;
    for (k = 0; k < o->K; k++) {
      c[k] = o_cmu(o, m, T, b, k);
      psi -= m[k] * c[k];
    }
    psi += o_fe(o, c, b, B, C);
    s += psi * o_dh(o, ph, b, a);
  }
  return s;
}

/* D(i,j) of one cell (functionD.h:1-16) */
static double o_D(const gpo *o, const double *ph, int i, int j) {
  int b, k;
  double s = 0.0;
  for (b = 0; b < o->N; b++)
    for (k = 0; k < o->K; k++) s += o->diff[b][i][k] * o->cmu[b][k][j] * ph[b];
  return s;
}

/* FunctionTau (functionTau.h:1-17) */
static double o_tau(const gpo *o, const double *ph) {
  int a, b;
  double s = 0.0, s1 = 0.0;
  for (a = 0; a < o->N; a++)
    for (b = 0; b < o->N; b++)
      if (a < b) {
        s += o->tau_ab[a][b] * ph[a] * ph[b];
        s1 += ph[a] * ph[b];
      }
  if (s1) return s / s1;
  return o->tau;
}

/* ----------------------------------------------------------- faces */

static void gather_phi(const gpo *o, long idx, double *ph) {
  int a;
  for (a = 0; a < o->N; a++) ph[a] = F(o->phi, o, a)[idx];
}

static void gather_mu(const gpo *o, long idx, double *m) {
  int k;
  for (k = 0; k < o->K; k++) m[k] = F(o->mu, o, k)[idx];
}

/* calculate_gradients_phasefield_2D (calculate_gradients.h:92-131) and the
 * phase-field half of calculate_gradients_2D (:4-91), for all rows.  smooth=1
 * selects the calculate_gradients_2D variant, whose row-0 centred x-gradient
 * reads a ring slot that holds data from an earlier sweep (NaN here). */
static void o_phi_faces(gpo *o) {
  long x, y;
  int a;
  for (a = 0; a < o->N; a++) {
    double *p = F(o->phi, o, a);
    double *gx = F(o->gx, o, a), *sx = F(o->sx, o, a), *gy = F(o->gy, o, a), *sy = F(o->sy, o, a);
    double *gcx = F(o->gcx, o, a), *gcy = F(o->gcy, o, a);
    for (x = 0; x < o->rx; x++) {
      for (y = 0; y <= o->ry - 2; y++) {
        long c = I(o, x, y);
        if (x <= o->rx - 2) {
          gx[c] = (p[c + o->ry] - p[c]) / o->dx;
          sx[c] = 0.5 * (p[c + o->ry] + p[c]);
        } else {
          gx[c] = 0.0;
          sx[c] = (p[c]);
        }
        gy[c] = (p[c + 1] - p[c]) / o->dy;
        sy[c] = 0.5 * (p[c + 1] + p[c]);
      }
      for (y = 0; y <= o->ry - 2; y++) {
        long c = I(o, x, y);
        if (y > 0 && y <= o->ry - 2) gcy[c] = (p[c + 1] - p[c - 1]) / (2.0 * o->dy);
        else gcy[c] = gy[c];
        gcx[c] = (x > 0) ? 0.5 * (gx[c] + gx[c - o->ry]) : NAN;
      }
      /* column rows_y-1 is never computed by the reference */
      gx[I(o, x, o->ry - 1)] = sx[I(o, x, o->ry - 1)] = NAN;
      gy[I(o, x, o->ry - 1)] = sy[I(o, x, o->ry - 1)] = NAN;
      gcx[I(o, x, o->ry - 1)] = gcy[I(o, x, o->ry - 1)] = NAN;
    }
  }
}

/* concentration half of calculate_gradients_2D / calculate_gradients_concentration_2D
 * (calculate_gradients.h:132-185) */
static void o_mu_faces(gpo *o) {
  long x, y;
  int k, l, K = o->K;
  for (x = 0; x < o->rx; x++)
    for (y = 0; y <= o->ry - 2; y++) {
      long c = I(o, x, y), f = c + o->ry, r = c + 1;
      double phc[MAXN], phf[MAXN], phr[MAXN];
      gather_phi(o, c, phc);
      gather_phi(o, r, phr);
      if (x <= o->rx - 2) gather_phi(o, f, phf);
      for (k = 0; k < K; k++) {
        double *m = F(o->mu, o, k);
        F(o->gmx, o, k)[c] = (x <= o->rx - 2) ? (m[f] - m[c]) / o->dx : 0.0;
        F(o->gmy, o, k)[c] = (m[r] - m[c]) / o->dy;
        for (l = 0; l < K; l++) {
          F(o->Dmx, o, k * K + l)[c] = (x <= o->rx - 2) ? (o_D(o, phf, k, l) + o_D(o, phc, k, l)) * 0.5
                                                        : o_D(o, phc, k, l);
          F(o->Dmy, o, k * K + l)[c] = (o_D(o, phr, k, l) + o_D(o, phc, k, l)) * 0.5;
        }
      }
    }
  for (x = 0; x < o->rx; x++)
    for (k = 0; k < K; k++) {
      long c = I(o, x, o->ry - 1);
      F(o->gmx, o, k)[c] = F(o->gmy, o, k)[c] = NAN;
      for (l = 0; l < K; l++) F(o->Dmx, o, k * K + l)[c] = F(o->Dmy, o, k * K + l)[c] = NAN;
    }
}

/* --------------------------------------------------------- anisotropy */

/* multiply(Rotation_matrix[a][b], q, out, DIMENSION=2) (matrix.h:10-20) */
static void rot2(const double M[3][3], const double *q, double *out) {
  int i, j;
  for (i = 0; i < 2; i++) {
    double s = 0;
    for (j = 0; j < 2; j++) s = s + M[i][j] * q[j];
    out[i] = s;
  }
}

/* anisotropy_01_dAdq / _function_ac (anisotropy_01.h:9-48) */
static void o_dadq(const gpo *o, const double *q, double *d, int a, int b) {
  double qx3 = q[0] * q[0] * q[0], qy3 = q[1] * q[1] * q[1], qz3 = q[2] * q[2] * q[2];
  double q2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
  double q22 = q2 * q2, q23 = q2 * q2 * q2;
  double q4 = qx3 * q[0] + qy3 * q[1] + qz3 * q[2];
  if (fabs(q2) > 1.0e-15) {
    d[0] = 16.0 * o->dab[a][b] * (qx3 / q22 - q[0] * q4 / q23);
    d[1] = 16.0 * o->dab[a][b] * (qy3 / q22 - q[1] * q4 / q23);
    d[2] = 16.0 * o->dab[a][b] * (qz3 / q22 - q[2] * q4 / q23);
  } else {
    d[0] = d[1] = d[2] = 0.0;
  }
}

static double o_ac(const gpo *o, const double *q, int a, int b) {
  double qx2 = q[0] * q[0], qx4 = qx2 * qx2, qy2 = q[1] * q[1], qy4 = qy2 * qy2;
  double qz2 = q[2] * q[2], qz4 = qz2 * qz2, q2 = qx2 + qy2 + qz2;
  if (fabs(q2) > 1.0e-15) return 1.0 - o->dab[a][b] * (3.0 - 4.0 * (qx4 + qy4 + qz4) / (q2 * q2));
  return 1.0;
}

/* q_divx (functionQ.h:4-21): face between cell c and its +x neighbour f */
static void o_qdivx(const gpo *o, long c, long f, int a, int b, double *q) {
  double t[3], r[2];
  t[0] = (F(o->sx, o, a)[c] * F(o->gx, o, b)[c] - F(o->sx, o, b)[c] * F(o->gx, o, a)[c]);
  t[1] = 0.5 * (F(o->sx, o, a)[c] * (F(o->gcy, o, b)[c] + F(o->gcy, o, b)[f]) -
                F(o->sx, o, b)[c] * (F(o->gcy, o, a)[c] + F(o->gcy, o, a)[f]));
  t[2] = 0.0;
  rot2(o->R[a][b], t, r);
  q[0] = r[0]; q[1] = r[1]; q[2] = t[2];
}

/* q_divy (functionQ.h:22-40): face between cell c and its +y neighbour r */
static void o_qdivy(const gpo *o, long c, long r, int a, int b, double *q) {
  double t[3], w[2];
  t[0] = 0.5 * (F(o->sy, o, a)[c] * (F(o->gcx, o, b)[c] + F(o->gcx, o, b)[r]) -
                F(o->sy, o, b)[c] * (F(o->gcx, o, a)[c] + F(o->gcx, o, a)[r]));
  t[1] = (F(o->sy, o, a)[c] * F(o->gy, o, b)[c] - F(o->sy, o, b)[c] * F(o->gy, o, a)[c]);
  t[2] = 0.0;
  rot2(o->R[a][b], t, w);
  q[0] = w[0]; q[1] = w[1]; q[2] = t[2];
}

/* function_A_01_dAdphi (function_A_01.h:4-71) */
static double o_dAdphi_aniso(const gpo *o, const double *ph, long c, int a) {
  int b, dir;
  double s1 = 0.0, s2 = 0.0;
  for (b = 0; b < o->N; b++) {
    double t[3], q[3], d[3], dq[3], rdq[2], q2, ac1, ac2, sp1 = 0.0, sp2 = 0.0;
    if (b == a) continue;
    t[0] = (ph[a] * F(o->gcx, o, b)[c] - ph[b] * F(o->gcx, o, a)[c]);
    t[1] = (ph[a] * F(o->gcy, o, b)[c] - ph[b] * F(o->gcy, o, a)[c]);
    rot2(o->R[a][b], t, q);
    q[2] = 0.0;
    o_dadq(o, q, d, a, b);
    q2 = (q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
    ac1 = o_ac(o, q, a, b);
    ac2 = ac1 * ac1;
    dq[0] = F(o->gcx, o, b)[c];
    dq[1] = F(o->gcy, o, b)[c];
    dq[2] = 0.0;
    rot2(o->R[a][b], dq, rdq);
    dq[0] = rdq[0]; dq[1] = rdq[1];
    for (dir = 0; dir < 2; dir++) sp1 += q[dir] * dq[dir];
    for (dir = 0; dir < 2; dir++) sp2 += (d[dir]) * dq[dir];
    sp1 *= o->gamma[a][b] * ac2;
    sp2 *= o->gamma[a][b] * ac1 * q2;
    s1 += sp1;
    s2 += sp2;
  }
  return 2.0 * (s1 + s2);
}

/* function_A_01_divdAdgradphi (function_A_01.h:101-219) */
static double o_divdA_aniso(const gpo *o, long c, int a) {
  long bk = c - o->ry, fr = c + o->ry, lf = c - 1, rt = c + 1;
  int b;
  double s1 = 0.0, s2 = 0.0;
  for (b = 0; b < o->N; b++) {
    double qf[3], qb[3], qr[3], ql[3], df[3], db[3], dr[3], dl[3];
    double rdf[2], rdb[2], rdr[2], rdl[2];
    double acf, acb, acr, acl, d1, d2, qf2, qb2, qr2, ql2;
    const double *sxa = F(o->sx, o, a), *sxb = F(o->sx, o, b), *gxa = F(o->gx, o, a), *gxb = F(o->gx, o, b);
    const double *sya = F(o->sy, o, a), *syb = F(o->sy, o, b), *gya = F(o->gy, o, a), *gyb = F(o->gy, o, b);
    if (b == a) continue;
    o_qdivx(o, c, fr, a, b, qf);  acf = o_ac(o, qf, a, b);
    o_qdivx(o, bk, c, a, b, qb);  acb = o_ac(o, qb, a, b);
    o_qdivy(o, c, rt, a, b, qr);  acr = o_ac(o, qr, a, b);
    o_qdivy(o, lf, c, a, b, ql);  acl = o_ac(o, ql, a, b);
    d1 = ((acf * acf * (sxa[c] * gxb[c] - sxb[c] * gxa[c]) * (-sxb[c])) -
          (acb * acb * (sxa[bk] * gxb[bk] - sxb[bk] * gxa[bk]) * (-sxb[bk]))) / o->dx;
    d1 += ((acr * acr * (sya[c] * gyb[c] - syb[c] * gya[c]) * (-syb[c])) -
           (acl * acl * (sya[lf] * gyb[lf] - syb[lf] * gya[lf]) * (-syb[lf]))) / o->dy;
    d1 *= o->gamma[a][b];
    s1 += d1;
    o_dadq(o, qf, df, a, b); rot2(o->Rinv[a][b], df, rdf);
    qf2 = qf[0] * qf[0] + qf[1] * qf[1] + qf[2] * qf[2];
    o_dadq(o, qb, db, a, b); rot2(o->Rinv[a][b], db, rdb);
    qb2 = qb[0] * qb[0] + qb[1] * qb[1] + qb[2] * qb[2];
    o_dadq(o, qr, dr, a, b); rot2(o->Rinv[a][b], dr, rdr);
    qr2 = qr[0] * qr[0] + qr[1] * qr[1] + qr[2] * qr[2];
    o_dadq(o, ql, dl, a, b); rot2(o->Rinv[a][b], dl, rdl);
    ql2 = ql[0] * ql[0] + ql[1] * ql[1] + ql[2] * ql[2];
    d2 = (acf * qf2 * rdf[0] * (-sxb[c]) - acb * qb2 * rdb[0] * (-sxb[bk])) / o->dx;
    d2 += (acr * qr2 * rdr[1] * (-syb[c]) - acl * ql2 * rdl[1] * (-syb[lf])) / o->dy;
    d2 *= o->gamma[a][b];
    s2 += d2;
  }
  return (2.0 * (s1 + s2) + 0.0);
}

/* function_A_00_dAdphi / A_01_dAdphi_smooth (function_A_00.h:4-21, function_A_01.h:73-100) */
static double o_dAdphi_iso(const gpo *o, const double *ph, long c, int a) {
  int b;
  double s = 0.0;
  for (b = 0; b < o->N; b++) {
    double sp = 0.0;
    if (b == a) continue;
    sp += (ph[a] * F(o->gcx, o, b)[c] - ph[b] * F(o->gcx, o, a)[c]) * F(o->gcx, o, b)[c];
    sp += (ph[a] * F(o->gcy, o, b)[c] - ph[b] * F(o->gcy, o, a)[c]) * F(o->gcy, o, b)[c];
    sp *= o->gamma[a][b];
    s += sp;
  }
  return 2.0 * s;
}

/* function_A_00_divdAdgradphi / A_01_divdAdgradphi_smooth (function_A_00.h:22-58,
 * function_A_01.h:220-259) */
static double o_divdA_iso(const gpo *o, long c, int a) {
  long bk = c - o->ry, lf = c - 1;
  int b;
  double s = 0.0;
  for (b = 0; b < o->N; b++) {
    const double *sxa = F(o->sx, o, a), *sxb = F(o->sx, o, b), *gxa = F(o->gx, o, a), *gxb = F(o->gx, o, b);
    const double *sya = F(o->sy, o, a), *syb = F(o->sy, o, b), *gya = F(o->gy, o, a), *gyb = F(o->gy, o, b);
    double d;
    if (b == a) continue;
    d = ((sxa[c] * gxb[c] - sxb[c] * gxa[c]) * (-sxb[c]) - ((sxa[bk] * gxb[bk] - sxb[bk] * gxa[bk]) * (-sxb[bk]))) / o->dx;
    d += ((sya[c] * gyb[c] - syb[c] * gya[c]) * (-syb[c]) - ((sya[lf] * gyb[lf] - syb[lf] * gya[lf]) * (-syb[lf]))) / o->dy;
    d *= o->gamma[a][b];
    s += d;
  }
  return 2.0 * s;
}

/* function_W_01_dwdphi (functionW_01.h:6-39), W_02 (functionW_02.h:4-33) and
 * their _smooth variants (functionW_01.h:41-64, functionW_02.h:35-59) */
static double o_dwdphi(const gpo *o, const double *ph, const double *dv, int a, int smooth) {
  int b, c, N = o->N;
  double s = 0.0;
  for (b = 0; b < N; b++) {
    if (b == a || !(fabs(dv[b]) > 0.0)) continue;
    if (o->well) {
      s += 2.0 * o->gamma[a][b] * (ph[b] * ph[b] * ph[a]);
    } else if (smooth) {
      s += o->gamma[a][b] * ph[b];
    } else {
      if ((ph[a] * ph[b]) >= 0.00000) s += o->gamma[a][b] * (ph[b]);
      else s += -o->gamma[a][b] * (ph[b]);
    }
  }
  if (o->well) s *= 9.0;
  else s *= 16.0 / (M_PI * M_PI);
  for (b = 0; b < N; b++)
    for (c = 0; c < N; c++)
      if (b != a && c != a && b < c && fabs(dv[b]) > 0.0 && fabs(dv[c]) > 0.0) {
        if (smooth) {
          s += o->gabc[a][b][c] * ph[b] * ph[c];
        } else {
          double bc = ph[b] * ph[c];
          if (ph[a] * bc >= 0.00000) s += o->gabc[a][b][c] * bc;
          else s += -o->gabc[a][b][c] * bc;
        }
      }
  return s;
}

/* projection_on_simplex (simplex_projection.h:1-49) */
static void o_project(const gpo *o, const double *ph, const double *dv, double *d) {
  int a, b, N = o->N;
  double Dphi = 0.0, sum_phib = 0.0;
  long count = 0;
  for (a = 0; a < N; a++)
    if ((fabs(dv[a]) > 0.0) && (ph[a] + d[a]) > 0.0 && (ph[a] + d[a]) < 1.0) {
      count++;
      sum_phib += ph[a];
    }
  for (a = 0; a < N; a++)
    if ((ph[a] + d[a]) < 0.0) {
      double da = fabs(d[a] + ph[a]);
      d[a] += da;
      Dphi += da;
    }
  if (Dphi > 0.0)
    for (b = 0; b < N; b++)
      if ((fabs(dv[b]) > 0.0) && ((ph[b] + d[b]) > 0.0) && ((ph[b] + d[b]) < 1.0)) {
        if (fabs(sum_phib) > 0.0) d[b] -= Dphi * (ph[b]) / (sum_phib);
        else d[b] -= Dphi / (count);
      }
  for (a = 0; a < N; a++)
    if (fabs(dv[a]) > 0.0 && (ph[a] + d[a]) > 1.0) {
      d[a] = (1.0 - ph[a]);
      for (b = 0; b < N; b++)
        if ((fabs(dv[b]) > 0.0) && b != a) d[b] = -ph[b];
      break;
    }
}

/* projection_on_simplex_without_weights (simplex_projection.h:50-91) */
static void o_project_nw(const gpo *o, const double *ph, const double *dv, double *d) {
  int a, b, N = o->N;
  long count = 0;
  for (a = 0; a < N; a++)
    if ((fabs(dv[a]) > 0.0) && (ph[a] + d[a]) > 0.0 && (ph[a] + d[a]) < 1.0) count++;
  for (a = 0; a < N; a++) {
    if (!(fabs(dv[a]) > 0.0)) continue;
    if ((ph[a] + d[a]) > 1.0) {
      d[a] = (1.0 - ph[a]);
      for (b = 0; b < N; b++)
        if ((fabs(dv[b]) > 0.0) && b != a) d[b] = -ph[b];
      break;
    }
    if ((ph[a] + d[a]) < 0.0) {
      double Dphi = fabs(d[a] + ph[a]);
      d[a] += Dphi;
      for (b = 0; b < N; b++)
        if (((fabs(dv[b]) > 0.0) && b != a) && (ph[b] + d[b]) > 0.0 && (ph[b] + d[b]) < 1.0) d[b] -= Dphi / (count);
    }
  }
}

/* calculate_divergence_phasefield_2D (calculate_divergence_phasefield.h:4-62)
 * and its _smooth variant (:63-158) for one cell. */
static void o_dphi_cell(const gpo *o, long c, int smooth, double *out) {
  int a, N = o->N;
  double ph[MAXN], m[MAXK], dv[MAXN], lam[MAXN], sl = 0.0;
  long act = 0;
  const double T = o_Tcell(o, c);
  double Bt[MAXN][MAXK], Ct[MAXN];
  gather_phi(o, c, ph);
  gather_mu(o, c, m);
  for (a = 0; a < N; a++) {
    dv[a] = (F(o->gx, o, a)[c] - F(o->gx, o, a)[c - o->ry]) / o->dx;
    dv[a] += (F(o->gy, o, a)[c] - F(o->gy, o, a)[c - 1]) / o->dy;
  }
  /* init_propertymatrices(T) before each active phase's dpsi
   * (calculate_divergence_phasefield.h:21-29): B, C at the cell's T */
  if (o->tgrad) o_BC(o, T, Bt, Ct);
  else memcpy(Bt, o->B, sizeof Bt), memcpy(Ct, o->C, sizeof Ct);
  for (a = 0; a < N; a++) {
    if (!(fabs(dv[a]) > 0.0)) continue;
    if (!smooth) {
      double dA = o->aniso ? o_dAdphi_aniso(o, ph, c, a) : o_dAdphi_iso(o, ph, c, a);
      double dd = o->aniso ? o_divdA_aniso(o, c, a) : o_divdA_iso(o, c, a);
      lam[a] = o->eps * (-dA + dd) - (1.0 / o->eps) * o_dwdphi(o, ph, dv, a, 0) - o_dpsi(o, m, T, ph, a, Bt, Ct);
    } else if (o->aniso) {
      /* A_01 _smooth variants return 2.0*(sum1 + 0.0): the same value as the
       * isotropic A_00 forms, since sum1 (a sum started at 0.0) is never -0 */
      lam[a] = o->eps * (-o_dAdphi_iso(o, ph, c, a) + o_divdA_iso(o, c, a)) -
               (1.0 / o->eps) * o_dwdphi(o, ph, dv, a, 1);
    } else {
      lam[a] = o->eps * (-o_dAdphi_iso(o, ph, c, a) + o_divdA_iso(o, c, a)) -
               (1.0 / o->eps) * o_dwdphi(o, ph, dv, a, 0);
    }
    sl += lam[a];
    act++;
  }
  if (act) sl /= act;
  for (a = 0; a < N; a++) {
    if (fabs(dv[a]) > 0.0) out[a] = o->dt * (lam[a] - sl) / (o_tau(o, ph) * o->eps);
    else out[a] = 0.0;
  }
  if (smooth) o_project_nw(o, ph, dv, out);
  else o_project(o, ph, dv, out);
}

/* calculate_fluxes_concentration_2D (calculate_fluxes_concentration.h:4-145) */
static void o_fluxes(gpo *o) {
  long x, y;
  int a, k, N = o->N, K = o->K, L = N - 1;
  for (k = 0; k < K; k++)
    for (y = 0; y < o->n; y++) F(o->jx, o, k)[y] = F(o->jy, o, k)[y] = NAN;
  for (x = 1; x <= o->rx - 3; x++)
    for (y = 0; y <= o->ry - 2; y++) {
      long c = I(o, x, y), r = c + 1, f = c + o->ry;
      double mc[MAXK], mr[MAXK], mf[MAXK], pc[MAXN], pr[MAXN], pf[MAXN];
      double gpx_l, ngy_l, gpy_l, ngx_l;
      gather_mu(o, c, mc); gather_mu(o, r, mr); gather_mu(o, f, mf);
      gather_phi(o, c, pc); gather_phi(o, r, pr); gather_phi(o, f, pf);
      gpx_l = 0.5 * (F(o->gcx, o, L)[c] + F(o->gcx, o, L)[r]);
      ngy_l = sqrt(gpx_l * gpx_l + F(o->gy, o, L)[c] * F(o->gy, o, L)[c]);
      gpy_l = 0.5 * (F(o->gcy, o, L)[c] + F(o->gcy, o, L)[f]);
      ngx_l = sqrt(gpy_l * gpy_l + F(o->gx, o, L)[c] * F(o->gx, o, L)[c]);
      for (k = 0; k < K; k++) { F(o->jx, o, k)[c] = 0.0; F(o->jy, o, k)[c] = 0.0; }
      for (a = 0; a < N - 1; a++) {
        double gpx, gpy, ng, s_r = 0, s_c = 0, s_f = 0;
        double gya = F(o->gy, o, a)[c], gxa = F(o->gx, o, a)[c];
        gpx = 0.5 * (F(o->gcx, o, a)[c] + F(o->gcx, o, a)[r]);
        ng = sqrt(gpx * gpx + gya * gya);
        if (o->obstacle) {
          s_r = (pr[a] * (1.0 - pr[a]) > 0.0) ? pr[a] * (1.0 - o_h(o, pr, a)) / (sqrt(pr[a] * (1.0 - pr[a]))) : 0.0;
          s_c = (pc[a] * (1.0 - pc[a]) > 0.0) ? pc[a] * (1.0 - o_h(o, pc, a)) / (sqrt(pc[a] * (1.0 - pc[a]))) : 0.0;
          s_f = (pf[a] * (1.0 - pf[a]) > 0.0) ? pf[a] * (1.0 - o_h(o, pf, a)) / (sqrt(pf[a] * (1.0 - pf[a]))) : 0.0;
        }
        for (k = 0; k < K; k++) {
          if (ng != 0.0 && y != 0 && y != o->my - 2) {
            /* non-isothermal: each cell's own temperature (calculate_fluxes_concentration.h:66-77) */
            double Tr = o_Tcell(o, r), Tcc = o_Tcell(o, c);
            double cl_r = o_cmu(o, mr, Tr, L, k), cl_c = o_cmu(o, mc, Tcc, L, k);
            double cs_r = o_cmu(o, mr, Tr, a, k), cs_c = o_cmu(o, mc, Tcc, a, k);
            double sp = gya * F(o->gy, o, L)[c];
            double atf = (1.0 - o->diff[a][k][k] / o->diff[L][k][k]);
            sp += gpx * gpx_l;
            if (ngy_l > 0.0) sp /= (ngy_l * ng);
            if (o->well)
              F(o->jy, o, k)[c] += atf * fabs(sp) * (0.5 / sqrt(2.0)) *
                                   ((cl_r - cs_r) * F(o->dphi, o, a)[r] + (cl_c - cs_c) * F(o->dphi, o, a)[c]) * gya / ng;
            if (o->obstacle)
              F(o->jy, o, k)[c] += atf * fabs(sp) * 0.5 *
                                   (s_r * (cl_r - cs_r) * F(o->dphi, o, a)[r] + s_c * (cl_c - cs_c) * F(o->dphi, o, a)[c]) * gya / ng;
          }
        }
        gpy = 0.5 * (F(o->gcy, o, a)[c] + F(o->gcy, o, a)[f]);
        ng = sqrt(gpy * gpy + gxa * gxa);
        for (k = 0; k < K; k++) {
          if (ng != 0.0) {
            double Tf = o_Tcell(o, f), Tcc = o_Tcell(o, c);
            double cl_f = o_cmu(o, mf, Tf, L, k), cl_c = o_cmu(o, mc, Tcc, L, k);
            double cs_f = o_cmu(o, mf, Tf, a, k), cs_c = o_cmu(o, mc, Tcc, a, k);
            double sp = gxa * F(o->gx, o, L)[c];
            double atf = (1.0 - o->diff[a][k][k] / o->diff[L][k][k]);
            sp += gpy * gpy_l;
            if (ngx_l > 0.0) sp /= (ngx_l * ng);
            if (o->well)
              F(o->jx, o, k)[c] += atf * fabs(sp) * (0.5 / sqrt(2.0)) *
                                   ((cl_f - cs_f) * F(o->dphi, o, a)[f] + (cl_c - cs_c) * F(o->dphi, o, a)[c]) * (gxa) / ng;
            if (o->obstacle)
              F(o->jx, o, k)[c] += atf * fabs(sp) * 0.5 *
                                   (s_f * (cl_f - cs_f) * F(o->dphi, o, a)[f] + s_c * (cl_c - cs_c) * F(o->dphi, o, a)[c]) * (gxa) / ng;
          }
        }
      }
    }
}

/* --------------------------------------------------------- boundaries */

/* apply_boundary_conditions (boundary_serial.h:176-203) with the copy tables of
 * assign_buffer_points_conditions / assign_boundary_points_values
 * (utility_functions.h:471-654): X faces copy whole rows, then Y faces copy
 * whole columns, three ghost layers each, phi then mu per face. */
static void o_bc(gpo *o) {
  int face, field, j;
  long rx = o->rx, ry = o->ry;
  for (face = 0; face < 4; face++)
    for (field = 0; field < (o->tgrad ? 3 : 2); field++) {
      int t = o->bctype[field][face], nf = field == 2 ? 1 : field ? o->K : o->N, a;
      double *arr = field == 2 ? o->Tc : field ? o->mu : o->phi;
      long pts[3], prx[3];
      if (t != 1 && t != 3) continue;
      for (j = 0; j < 3; j++) {
        if (face == 0) { pts[j] = 2 - j; prx[j] = (t == 1) ? 4 + j : rx - 5 - j; }
        if (face == 1) { pts[j] = rx - 3 + j; prx[j] = (t == 1) ? rx - 5 - j : 4 + j; }
        if (face == 2) { pts[j] = ry - 3 + j; prx[j] = (t == 1) ? ry - 5 - j : 4 + j; }
        if (face == 3) { pts[j] = 2 - j; prx[j] = (t == 1) ? 4 + j : ry - 5 - j; }
      }
      for (j = 0; j < 3; j++)
        for (a = 0; a < nf; a++) {
          double *p = F(arr, o, a);
          long u;
          if (face < 2)
            for (u = 0; u < ry; u++) p[I(o, pts[j], u)] = p[I(o, prx[j], u)];
          else
            for (u = 0; u < rx; u++) p[I(o, u, pts[j])] = p[I(o, u, prx[j])];
        }
    }
}

/* ------------------------------------------------------------ stats */

static void o_track(gpo *o, const double *dmu_cells) {
  long x, y;
  int a, k;
  for (a = 0; a < o->N; a++) o->rel_phi[a] = 0.0;
  for (k = 0; k < o->K; k++) o->rel_mu[k] = 0.0;
  for (x = 3; x < o->mx + 3; x++)
    for (y = 3; y < o->my + 3; y++) {
      long c = I(o, x, y);
      for (a = 0; a < o->N; a++) {
        double v = F(o->phi, o, a)[c], d = F(o->dphi, o, a)[c];
        if (v > o->phi_max[a]) o->phi_max[a] = v;
        if (v < o->phi_min[a]) o->phi_min[a] = v;
        o->rel_phi[a] += d * d;
      }
      for (k = 0; k < o->K; k++) {
        double v = F(o->mu, o, k)[c], d = dmu_cells[(long)k * o->n + c];
        if (v > o->mu_max[k]) o->mu_max[k] = v;
        if (v < o->mu_min[k]) o->mu_min[k] = v;
        o->rel_mu[k] += d * d;
      }
    }
}

/* ------------------------------------------------------------- passes */

/* mu update + phi commit of one cell; calculate_divergence_concentration_2D
 * (calculate_divergence_concentration.h:4-153) when smooth=0, the _smooth_2D
 * variant (:154-253) when smooth=1.  Writes nphi/nmu and the cell's delta-mu. */
static void o_conc_cell(gpo *o, long c, int smooth, double *dmu_out, double *deltamu) {
  int a, b, k, l, N = o->N, K = o->K;
  double ph[MAXN], m[MAXK], sum[MAXK], divflux[MAXK], divjat[MAXK] = {0};
  double dcdmu[3][3] = {{0}}, inv[3][3] = {{0}}, deltac[MAXK], cold[MAXK], cnew[MAXK];
  const double *dph = smooth ? o->sdphi : o->dphi;
  int interface = 1, bulk = 0;
  long bk = c - o->ry, lf = c - 1;
  const double T = o_Tcell(o, c);
  double sum_dcbdT[MAXK];
  gather_phi(o, c, ph);
  gather_mu(o, c, m);
  for (k = 0; k < K; k++) sum[k] = sum_dcbdT[k] = 0.0;
  if (!smooth)
    for (a = 0; a < N; a++) {
      double sdh = 0.0;
      for (b = 0; b < N; b++) sdh += o_dh(o, ph, a, b) * F(dph, o, b)[c];
      for (k = 0; k < K; k++) {
        sum[k] += o_cmu(o, m, T, a, k) * sdh;
        /* dcbdT_phase is allocated but never filled by the reference
         * (reading_input_parameters.h:85): taken as 0 */
        sum_dcbdT[k] += 0.0 * o_h(o, ph, a);
      }
    }
  for (k = 0; k < K; k++) {
    divflux[k] = 0.0;
    for (l = 0; l < K; l++) {
      divflux[k] += (F(o->Dmx, o, k * K + l)[c] * F(o->gmx, o, l)[c] - F(o->Dmx, o, k * K + l)[bk] * F(o->gmx, o, l)[bk]) / o->dx;
      divflux[k] += (F(o->Dmy, o, k * K + l)[c] * F(o->gmy, o, l)[c] - F(o->Dmy, o, k * K + l)[lf] * F(o->gmy, o, l)[lf]) / o->dy;
    }
    if (!smooth) {
      double cst = o->obstacle ? (-0.25 * M_PI * o->eps) : (-1.0 * o->eps);
      divjat[k] = (F(o->jx, o, k)[c] - F(o->jx, o, k)[bk]) * cst / o->dx;
      divjat[k] += (F(o->jy, o, k)[c] - F(o->jy, o, k)[lf]) * cst / o->dy;
    }
  }
  for (a = 0; a < N; a++)
    if (ph[a] == 1.0) { bulk = a; interface = 0; break; }
  if (!interface) {
    for (k = 0; k < K; k++) {
      cold[k] = o_cmu(o, m, T, bulk, k);
      cnew[k] = smooth ? cold[k] + o->dt * (divflux[k]) : cold[k] + o->dt * (divflux[k]) - divjat[k];
    }
    for (k = 0; k < K; k++) {
      double nv = o_Mu(o, cnew, T, bulk, k);
      deltamu[k] = nv - m[k];
      F(o->nmu, o, k)[c] = nv;
    }
  } else {
    double nm[MAXK];
    for (k = 0; k < K; k++) {
      deltac[k] = smooth ? o->dt * (divflux[k]) : o->dt * (divflux[k]) - divjat[k] - sum[k];
      /* calculate_divergence_concentration.h:85: the struct member GRADIENT
       * of temperature_gradientY is never set, so the term is a signed zero */
      if (!smooth && o->tgrad) deltac[k] = deltac[k] - sum_dcbdT[k] * o->dt * (-0.0 * o->tg_vel);
      for (l = 0; l < K; l++)
        for (a = 0; a < N; a++) dcdmu[k][l] += o->cmu[a][k][l] * o_h(o, ph, a);
    }
    for (k = 0; k < K; k++) nm[k] = m[k];
    if (!smooth && o->inv_mode == 1) {          /* BINARY */
      double i00 = 1.0 / dcdmu[0][0];
      deltamu[0] = deltac[0] * i00;
      nm[0] += deltamu[0];
    } else if (!smooth && o->inv_mode == 2) {   /* TERNARY */
      double det = dcdmu[0][0] * dcdmu[1][1] - dcdmu[0][1] * dcdmu[1][0];
      inv[0][0] = dcdmu[1][1] / det;
      inv[1][1] = dcdmu[0][0] / det;
      inv[0][1] = -dcdmu[0][1] / det;
      inv[1][0] = -dcdmu[1][0] / det;
      for (k = 0; k < K; k++) {
        deltamu[k] = 0.0;
        for (l = 0; l < K; l++) deltamu[k] += inv[k][l] * deltac[l];
      }
      for (k = 0; k < K; k++) nm[k] = deltamu[k] + nm[k];
    } else if (!smooth && o->inv_mode == 3) {   /* DILUTE */
      for (k = 0; k < K; k++) {
        double ikk = 1.0 / dcdmu[k][k];
        deltamu[k] = deltac[k] * ikk;
        nm[k] += deltamu[k];
      }
    } else {                                    /* matinvnew */
      o_matinv(dcdmu, inv, K, o->recip_div);
      for (k = 0; k < K; k++) {
        double s = 0;
        for (l = 0; l < K; l++) s = s + inv[k][l] * deltac[l];
        deltamu[k] = s;
      }
      for (k = 0; k < K; k++) nm[k] = deltamu[k] + nm[k];
    }
    for (k = 0; k < K; k++) F(o->nmu, o, k)[c] = nm[k];
  }
  for (b = 0; b < N; b++) F(o->nphi, o, b)[c] = ph[b] + F(dph, o, b)[c];
  for (k = 0; k < K; k++) dmu_out[(long)k * o->n + c] = deltamu[k];
}

/* apply_temperature_gradientY (Temperature_gradient.h:4-29) after the
 * reference main's BASE_POS / GRADIENT / temp_bottom for step t
 * (microsim_gp.c:77-82 for t = 0, :108-113 after step t): every ghosted cell */
static void o_temperature(gpo *o, long t) {
  long x, y;
  double base_pos, grad, tb;
  if (t == 0) base_pos = (o->tg_off / o->dy) - o->shift_off;
  else base_pos = (o->tg_off / o->dy) - o->shift_off + ((o->tg_vel / o->dy) * (t * o->dt));
  grad = (o->tg_dT) * o->dy / (o->tg_dist);
  tb = o->tg_base - base_pos * grad;
  for (x = 0; x < o->rx; x++)
    for (y = 0; y < o->ry; y++) o->Tc[I(o, x, y)] = tb + y * grad;
}

/* check_SHIFT (shift.h:47-65) over the rows the concentration pass updated,
 * on the values it left (updated cells new, the others as before): the
 * largest column y with liquid below one half at y-1 and above at y */
static long o_interface_pos(const gpo *o) {
  long x, y, best = 0;
  const double *pl = F(o->phi, o, o->N - 1);
  for (x = 1; x <= o->rx - 3; x++)
    for (y = 1; y <= o->ry - 1; y++) {
      double a = pl[I(o, x, y - 1)], b = pl[I(o, x, y)];
      if ((a - (1.0 - a) < 0.0) && (b - (1.0 - b) > 0.0) && y > best) best = y;
    }
  return best;
}

/* apply_shiftY (shift.h:4-45): every row moves down by d = pos - shiftj
 * cells; the top d cells become liquid at cfill with Mu at Tfill (their
 * temperature is left as it was) */
static void o_shift(gpo *o, long pos) {
  long x, y, d = pos - o->shiftj;
  int a, k, L = o->N - 1;
  for (x = 0; x < o->rx; x++) {
    for (y = 0; y <= (o->ry - 1 - d); y++) {
      long c = I(o, x, y);
      for (a = 0; a < o->N; a++) F(o->phi, o, a)[c] = F(o->phi, o, a)[c + d];
      for (k = 0; k < o->K; k++) F(o->mu, o, k)[c] = F(o->mu, o, k)[c + d];
      if (o->tgrad) o->Tc[c] = o->Tc[c + d];
    }
    for (y = o->ry - d; y <= o->ry - 1; y++) {
      long c = I(o, x, y);
      for (a = 0; a < L; a++) F(o->phi, o, a)[c] = 0.0;
      F(o->phi, o, L)[c] = 1.0;
      for (k = 0; k < o->K; k++) F(o->mu, o, k)[c] = o_Mu(o, o->cfill_l, o->Tfill, L, k);
    }
  }
}

static void o_commit(gpo *o) {
  double *t;
  t = o->phi; o->phi = o->nphi; o->nphi = t;
  t = o->mu; o->mu = o->nmu; o->nmu = t;
}

void gpo_step(gpo *o, long nsteps) {
  long s, x, y;
  double *dmu = malloc(sizeof(double) * (size_t)o->K * o->n);
  double deltamu[MAXK] = {0};
  for (s = 0; s < nsteps; s++) {
    /* phase-field pass: solverloop_phasefield (solverloop.h:21-34) */
    o_phi_faces(o);
    for (x = 1; x <= o->rx - 2; x++)
      for (y = 1; y <= o->ry - 2; y++) {
        long c = I(o, x, y);
        double d[MAXN];
        int a;
        o_dphi_cell(o, c, 0, d);
        for (a = 0; a < o->N; a++) F(o->dphi, o, a)[c] = d[a];
      }
    o_bc(o);
    /* concentration pass: solverloop_concentration (solverloop.h:35-71) */
    o_mu_faces(o);
    o_fluxes(o);
    memcpy(o->nphi, o->phi, sizeof(double) * (size_t)o->N * o->n);
    memcpy(o->nmu, o->mu, sizeof(double) * (size_t)o->K * o->n);
    memset(dmu, 0, sizeof(double) * (size_t)o->K * o->n);
    for (x = 1; x <= o->rx - 3; x++)
      for (y = 1; y <= o->ry - 2; y++) o_conc_cell(o, I(o, x, y), 0, dmu, deltamu);
    o_commit(o);
    {
      long pos = o->shift ? o_interface_pos(o) : 0;
      o_bc(o);
      o_track(o, dmu);
      o->steps++;
      o->tstep++;
      if (o->tgrad) {
        memcpy(o->Tstep, o->Tc, sizeof(double) * (size_t)o->n);
        o_temperature(o, o->tstep);
      }
      o->last_shift = 0;
      if (o->shift && o->tstep % 100 == 0 && pos > o->shiftj) {
        o_shift(o, pos);
        o->last_shift = pos - o->shiftj;
        o->shift_off += pos - o->shiftj;
      }
    }
  }
  free(dmu);
}

void gpo_smooth(gpo *o, long nsteps) {
  long s, x, y;
  double *dmu = malloc(sizeof(double) * (size_t)o->K * o->n);
  double deltamu[MAXK] = {0};
  for (s = 0; s < nsteps; s++) {
    /* smooth (solverloop.h:72-90) */
    o_phi_faces(o);
    for (y = 0; y < o->ry; y++) {
      int a;
      for (a = 0; a < o->N; a++) F(o->gcx, o, a)[I(o, 0, y)] = NAN;   /* stale ring slot */
    }
    o_mu_faces(o);
    for (x = 1; x <= o->rx - 2; x++)
      for (y = 1; y <= o->ry - 2; y++) {
        long c = I(o, x, y);
        double d[MAXN];
        int a;
        o_dphi_cell(o, c, 1, d);
        for (a = 0; a < o->N; a++) F(o->sdphi, o, a)[c] = d[a];
      }
    memcpy(o->nphi, o->phi, sizeof(double) * (size_t)o->N * o->n);
    memcpy(o->nmu, o->mu, sizeof(double) * (size_t)o->K * o->n);
    for (x = 1; x <= o->rx - 3; x++)
      for (y = 1; y <= o->ry - 2; y++) o_conc_cell(o, I(o, x, y), 1, dmu, deltamu);
    o_commit(o);
    o_bc(o);
  }
  free(dmu);
}

/* ------------------------------------------------------------ public */

gpo *gpo_create(const gp_params *p, int recip_div, char *err, int errlen) {
  gpo *o;
  int a, b, c, i, j, f;
  long n;
  if (p->dimension != 2 || p->numphases < 2 || p->numphases > MAXN || p->numcomponents < 2 ||
      p->numcomponents - 1 > 3 || p->mesh_x < 5 || p->mesh_y < 5) {
    snprintf(err, errlen, "oracle: unsupported parameters");
    return NULL;
  }
  for (f = 0; f < (p->isothermal ? 2 : 3); f++)
    for (i = 0; i < 4; i++)
      if (p->bc_type[f][i] != 1 && p->bc_type[f][i] != 3) {
        snprintf(err, errlen, "oracle: only Neumann/periodic boundaries");
        return NULL;
      }
  o = calloc(1, sizeof *o);
  o->N = p->numphases;
  o->K = p->numcomponents - 1;
  o->mx = p->mesh_x; o->my = p->mesh_y;
  o->rx = o->mx + 6; o->ry = o->my + 6;
  o->n = n = o->rx * o->ry;
  o->well = (p->function_w == 2);
  o->obstacle = !o->well;
  o->aniso = (p->function_anisotropy == 1);
  o->inv_mode = p->binary ? 1 : p->ternary ? 2 : p->dilute ? 3 : 4;
  o->recip_div = recip_div;
  o->dx = p->deltax; o->dy = p->deltay; o->dt = p->deltat;
  o->eps = p->epsilon; o->tau = p->tau;
  o->T = p->T; o->Teq = p->Teq;
  for (a = 0; a < o->N; a++)
    for (b = 0; b < o->N; b++) {
      static const double zero[3] = {0, 0, 0};
      o->gamma[a][b] = p->gamma[a][b];
      o->tau_ab[a][b] = p->tau_ab[a][b];
      o->dab[a][b] = p->dab[a][b];
      for (c = 0; c < o->N; c++) o->gabc[a][b][c] = p->gamma_abc[a][b][c];
      if (a != b) o_rotation(p->rot_set[a][b] ? p->rot_angles[a][b] : zero, o->R[a][b], o->Rinv[a][b]);
    }
  for (a = 0; a < o->N; a++)
    for (i = 0; i < o->K; i++)
      for (j = 0; j < o->K; j++) {
        o->diff[a][i][j] = p->diffusivity[a][i][j];
        o->A[a][i][j] = p->A[a][i][j];
      }
  o_props_full(o, p);
  for (f = 0; f < 3; f++)
    for (i = 0; i < 4; i++) o->bctype[f][i] = p->bc_type[f][i];
  {
    int L = o->N - 1, k;
    o->tgrad = !p->isothermal;
    o->tg_base = p->tempgrady_v[0];
    o->tg_dT = p->tempgrady_v[1];
    o->tg_dist = p->tempgrady_v[2];
    o->tg_off = p->tempgrady_v[3];
    o->tg_vel = p->tempgrady_v[4];
    for (a = 0; a < o->N; a++)
      for (k = 0; k < o->K; k++) {
        o->ceq_l[a][k] = p->ceq[a][L][k];
        o->ceq_s[a][k] = p->ceq[a][a][k];
      }
    for (a = 0; a < L; a++) {
      o->DT_l[a] = 0.0;
      o->DT_s[a] = 0.0;
      for (k = 0; k < o->K; k++) {
        o->DT_s[a] += p->slopes[a][a][k] * (p->ceq[a][L][k] - p->ceq[a][a][k]);
        o->DT_l[a] += p->slopes[a][L][k] * (p->ceq[a][L][k] - p->ceq[a][a][k]);
        o->DC[a][k] = p->ceq[a][L][k] - p->ceq[a][a][k];
      }
    }
    o->shift = p->shift != 0;
    o->shiftj = p->shiftj;
    o->Tfill = p->Tfill;
    for (k = 0; k < o->K; k++) o->cfill_l[k] = p->cfill[L][L][k];
  }
  o->phi = calloc((size_t)o->N * n, 8); o->nphi = calloc((size_t)o->N * n, 8);
  o->dphi = calloc((size_t)o->N * n, 8); o->sdphi = calloc((size_t)o->N * n, 8);
  o->mu = calloc((size_t)o->K * n, 8); o->nmu = calloc((size_t)o->K * n, 8);
  o->gx = calloc((size_t)o->N * n, 8); o->sx = calloc((size_t)o->N * n, 8);
  o->gy = calloc((size_t)o->N * n, 8); o->sy = calloc((size_t)o->N * n, 8);
  o->gcx = calloc((size_t)o->N * n, 8); o->gcy = calloc((size_t)o->N * n, 8);
  o->gmx = calloc((size_t)o->K * n, 8); o->gmy = calloc((size_t)o->K * n, 8);
  o->Dmx = calloc((size_t)o->K * o->K * n, 8); o->Dmy = calloc((size_t)o->K * o->K * n, 8);
  o->jx = calloc((size_t)o->K * n, 8); o->jy = calloc((size_t)o->K * n, 8);
  o->Tc = calloc((size_t)n, 8);
  o->Tstep = calloc((size_t)n, 8);
  if (o->tgrad) o_temperature(o, 0);
  for (a = 0; a < o->N; a++) { o->phi_max[a] = 1.0; o->phi_min[a] = 0.0; }
  for (i = 0; i < o->K; i++) { o->mu_max[i] = 1.0; o->mu_min[i] = 1.0; }
  return o;
}

void gpo_destroy(gpo *o) {
  if (!o) return;
  free(o->phi); free(o->nphi); free(o->dphi); free(o->sdphi); free(o->mu); free(o->nmu);
  free(o->gx); free(o->sx); free(o->gy); free(o->sy); free(o->gcx); free(o->gcy);
  free(o->gmx); free(o->gmy); free(o->Dmx); free(o->Dmy); free(o->jx); free(o->jy);
  free(o->Tc);
  free(o->Tstep);
  free(o);
}

void gpo_dims(const gpo *o, long *rows_x, long *rows_y) { *rows_x = o->rx; *rows_y = o->ry; }

int gpo_set(gpo *o, const double *phi, const double *mu) {
  long x, y;
  int a, k;
  for (a = 0; a < o->N; a++)
    for (x = 0; x < o->mx; x++)
      for (y = 0; y < o->my; y++) F(o->phi, o, a)[I(o, x + 3, y + 3)] = phi[((long)a * o->mx + x) * o->my + y];
  for (k = 0; k < o->K; k++)
    for (x = 0; x < o->mx; x++)
      for (y = 0; y < o->my; y++) F(o->mu, o, k)[I(o, x + 3, y + 3)] = mu[((long)k * o->mx + x) * o->my + y];
  o_bc(o);
  return 0;
}

void gpo_get(const gpo *o, double *phi, double *mu) {
  long x, y;
  int a, k;
  for (a = 0; a < o->N; a++)
    for (x = 0; x < o->mx; x++)
      for (y = 0; y < o->my; y++) phi[((long)a * o->mx + x) * o->my + y] = F(o->phi, o, a)[I(o, x + 3, y + 3)];
  for (k = 0; k < o->K; k++)
    for (x = 0; x < o->mx; x++)
      for (y = 0; y < o->my; y++) mu[((long)k * o->mx + x) * o->my + y] = F(o->mu, o, k)[I(o, x + 3, y + 3)];
}

void gpo_temperature(const gpo *o, double *T) {
  long x, y;
  for (x = 0; x < o->mx; x++)
    for (y = 0; y < o->my; y++) T[x * o->my + y] = o->tgrad ? o->Tc[I(o, x + 3, y + 3)] : o->T;
}

void gpo_get_full(const gpo *o, double *phi, double *mu, double *dphi) {
  if (phi) memcpy(phi, o->phi, sizeof(double) * (size_t)o->N * o->n);
  if (mu) memcpy(mu, o->mu, sizeof(double) * (size_t)o->K * o->n);
  if (dphi) memcpy(dphi, o->dphi, sizeof(double) * (size_t)o->N * o->n);
}

void gpo_stats(const gpo *o, gp_stats *s) {
  long x, y;
  int a, k, b;
  memset(s, 0, sizeof *s);
  for (a = 0; a < o->N; a++) {
    s->phi_max[a] = o->phi_max[a]; s->phi_min[a] = o->phi_min[a]; s->rel_change_phi[a] = o->rel_phi[a];
  }
  for (k = 0; k < o->K; k++) {
    s->mu_max[k] = o->mu_max[k]; s->mu_min[k] = o->mu_min[k]; s->rel_change_mu[k] = o->rel_mu[k];
  }
  for (x = 3; x < o->mx + 3; x++)
    for (y = 3; y < o->my + 3; y++) {
      long c = I(o, x, y);
      double ph[MAXN], m[MAXK];
      int bad = 0;
      gather_phi(o, c, ph);
      gather_mu(o, c, m);
      for (a = 0; a < o->N; a++) { s->phi_sum[a] += ph[a]; if (!isfinite(ph[a])) bad = 1; }
      for (k = 0; k < o->K; k++) {
        double comp = 0.0;
        if (!isfinite(m[k])) bad = 1;
        /* at the temperature the last step used (the field before its update) */
        for (b = 0; b < o->N; b++) comp += o_cmu(o, m, o->tgrad ? o->Tstep[c] : o->T, b, k) * o_h(o, ph, b);
        s->comp_sum[k] += comp;
      }
      s->nonfinite += bad;
    }
  s->steps_done = o->steps;
  s->shift_offset = o->shift_off;
}

void gpo_consts(const gpo *o, double *cmu, double *B, double *C, double *Beq,
                double *dBbdT, double *R, double *Rinv) {
  int N = o->N, K = o->K, a, b, i, j;
  for (a = 0; a < N; a++) {
    for (i = 0; i < K; i++) {
      for (j = 0; j < K; j++) cmu[(a * K + i) * K + j] = o->cmu[a][i][j];
      B[a * K + i] = o->B[a][i];
      Beq[a * K + i] = o->Beq[a][i];
      dBbdT[a * K + i] = o->dBbdT[a][i];
    }
    C[a] = o->C[a];
    for (b = 0; b < N; b++)
      for (i = 0; i < 3; i++)
        for (j = 0; j < 3; j++) {
          R[((a * N + b) * 3 + i) * 3 + j] = a == b ? 0.0 : o->R[a][b][i][j];
          Rinv[((a * N + b) * 3 + i) * 3 + j] = a == b ? 0.0 : o->Rinv[a][b][i][j];
        }
  }
}
