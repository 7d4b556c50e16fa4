/*
 * gp_host.c -- host surface of libgp in C: Input.in / Filling.in parsing,
 * filling, legacy-VTK output, and the host-side derivation of the constants the
 * CUDA step uses.  It keeps the reference's file formats and their quirks
 * (line grammar, defaults, ordering rules) so existing MicroSim input decks work
 * unchanged; each routine cites the reference code whose behaviour it follows.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gp_internal.h"

/* ------------------------------------------------------------------ errors */

static __thread char g_thread_err[256];

void gp_set_thread_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_thread_err, sizeof g_thread_err, fmt, ap);
  va_end(ap);
}

const char *gp_host_thread_error(void) { return g_thread_err; }

/* ---------------------------------------------------------------- tokens */

/* Split a "{a, b, c}" value on the characters "{,}" the way strtok_r does in
 * the reference's populate_* helpers (utility_functions.h:84-341).  Tokens keep
 * their leading blanks (atof/atol skip them; names keep them). */
#define MAXTOK 64
typedef struct { int n; char tok[MAXTOK][104]; } toklist;

static void split_tokens(const char *s, toklist *tl) {
  char buf[512], *save = NULL, *t;
  size_t len = strlen(s);
  if (len >= sizeof buf) len = sizeof buf - 1;
  memcpy(buf, s, len);
  buf[len] = 0;
  tl->n = 0;
  for (t = strtok_r(buf, "{,}", &save); t && tl->n < MAXTOK; t = strtok_r(NULL, "{,}", &save)) {
    snprintf(tl->tok[tl->n], sizeof tl->tok[0], "%s", t);
    tl->n++;
  }
}

static double tokd(const toklist *tl, int i) { return i < tl->n ? atof(tl->tok[i]) : 0.0; }
static long tokl(const toklist *tl, int i) { return i < tl->n ? atol(tl->tok[i]) : 0; }

/* ------------------------------------------------------------ line reader */

/* The reference reads every line with sscanf("%100s = %100[^;];") into two
 * buffers that keep their previous contents when a line does not match
 * (reading_input_parameters.h:24-25), so a blank line repeats the previous
 * key.  This reader keeps that behaviour. */
typedef struct { FILE *f; char key[128]; char val[128]; } linereader;

static int next_line(linereader *lr) {
  char buf[1000];
  if (!fgets(buf, sizeof buf, lr->f)) return 0;
  sscanf(buf, "%100s = %100[^;];", lr->key, lr->val);
  return 1;
}

/* ------------------------------------------------------------- populate */

static void pop_pair_matrix(double m[GP_MAX_PHASES][GP_MAX_PHASES], const char *v, int N) {
  /* populate_matrix (utility_functions.h:84-117): upper-triangle pairs in order */
  toklist tl;
  int i, j, k = 0;
  split_tokens(v, &tl);
  for (i = 0; i < N; i++)
    for (j = i + 1; j < N; j++) {
      m[i][i] = 0.0;
      m[i][j] = tokd(&tl, k);
      m[j][i] = m[i][j];
      k++;
    }
}

static void pop_triple(double m[GP_MAX_PHASES][GP_MAX_PHASES][GP_MAX_PHASES], const char *v, int N) {
  /* populate_matrix3M (utility_functions.h:119-162) */
  toklist tl;
  int i, j, k, l = 0;
  split_tokens(v, &tl);
  for (i = 0; i < N; i++)
    for (j = i + 1; j < N; j++)
      for (k = j + 1; k < N; k++) {
        double g = tokd(&tl, l);
        m[i][i][i] = 0.0; m[i][j][j] = 0.0; m[i][k][k] = 0.0;
        m[i][j][k] = g; m[i][k][j] = g; m[j][i][k] = g;
        m[j][k][i] = g; m[k][i][j] = g; m[k][j][i] = g;
        l++;
      }
}

static void pop_diffusivity(gp_params *p, const char *v) {
  /* populate_diffusivity_matrix (utility_functions.h:163-218).  The
   * non-diagonal form reads past the reference's token array; here a missing
   * token reads as 0. */
  toklist tl;
  int i, j, l, K = p->numcomponents - 1;
  long ph;
  split_tokens(v, &tl);
  if (tl.n < 2) return;
  ph = tokl(&tl, 1);
  if (ph < 0 || ph >= GP_MAX_PHASES) return;
  l = 1;
  for (i = 0; i < K; i++) { p->diffusivity[ph][i][i] = tokd(&tl, 1 + l); l++; }
  if (strcmp(tl.tok[0], "1") == 0) {
    for (i = 0; i < K; i++)
      for (j = i + 1; j < K; j++) { p->diffusivity[ph][i][j] = 0.0; p->diffusivity[ph][j][i] = 0.0; }
  } else {
    for (i = 0; i < K; i++)
      for (j = 0; j < K; j++) { p->diffusivity[ph][i][j] = tokd(&tl, 1 + l); l++; }
  }
}

static void pop_A(gp_params *p, const char *v) {
  /* populate_A_matrix (utility_functions.h:219-257) */
  toklist tl;
  int i, j, l = 1, K = p->numcomponents - 1;
  long ph;
  split_tokens(v, &tl);
  ph = tokl(&tl, 0);
  if (ph < 0 || ph >= GP_MAX_PHASES) return;
  for (i = 0; i < K; i++) { p->A[ph][i][i] = tokd(&tl, l); l++; }
  for (i = 0; i < K; i++)
    for (j = i + 1; j < K; j++) {
      p->A[ph][i][j] = tokd(&tl, l);
      p->A[ph][j][i] = p->A[ph][i][j];
      l++;
    }
}

static void pop_thermo(double m[GP_MAX_PHASES][GP_MAX_PHASES][GP_MAX_COMP], const char *v, int K) {
  /* populate_thermodynamic_matrix (utility_functions.h:259-292) */
  toklist tl;
  int i;
  long p1, p2;
  split_tokens(v, &tl);
  p1 = tokl(&tl, 0); p2 = tokl(&tl, 1);
  if (p1 < 0 || p2 < 0 || p1 >= GP_MAX_PHASES || p2 >= GP_MAX_PHASES) return;
  for (i = 0; i < K; i++) m[p1][p2][i] = tokd(&tl, 2 + i);
}

static void pop_names(char names[][GP_NAME_LEN], int cap, const char *v) {
  /* populate_string_array (utility_functions.h:328-341): tokens as they are */
  toklist tl;
  int i;
  split_tokens(v, &tl);
  for (i = 0; i < tl.n && i < cap; i++) snprintf(names[i], GP_NAME_LEN, "%s", tl.tok[i]);
}

/* ---------------------------------------------------------------- parser */

static void params_defaults(gp_params *p) {
  memset(p, 0, sizeof *p);
  /* initial values of the reference's globals (global_vars.h) */
  p->function_w = 1;
  p->function_anisotropy = 1;
  p->function_f = 1;
  p->obstacle_key = -1;
  p->isothermal = 0;
  p->tempgrady = 0;
  {
    int f, s;
    for (f = 0; f < 3; f++)
      for (s = 0; s < 6; s++) p->bc_type[f][s] = -1;
  }
}

static int bc_field(const char *name) {
  if (strcmp(name, "phi") == 0) return 0;
  if (strcmp(name, "mu") == 0) return 1;
  if (strcmp(name, "T") == 0) return 2;
  return -1;
}

int gp_params_load(gp_params *p, const char *input_path) {
  linereader lr;
  int N, K;
  if (!p || !input_path) { gp_set_thread_error("gp_params_load: NULL argument"); return GP_EINVAL; }
  params_defaults(p);
  memset(&lr, 0, sizeof lr);
  lr.f = fopen(input_path, "rt");
  if (!lr.f) { gp_set_thread_error("cannot open %s", input_path); return GP_EIO; }

  /* pass 1: reading_input_parameters.h:24-307 */
  while (next_line(&lr)) {
    const char *k = lr.key, *v = lr.val;
    N = p->numphases;
    K = p->numcomponents - 1;
    if (k[0] == '#') continue;
    if (!strcmp(k, "DIMENSION")) p->dimension = atoi(v);
    else if (!strcmp(k, "MESH_X")) p->mesh_x = atol(v);
    else if (!strcmp(k, "MESH_Y")) p->mesh_y = atol(v);
    else if (!strcmp(k, "MESH_Z")) p->mesh_z = atol(v);
    else if (!strcmp(k, "DELTA_X")) p->deltax = atof(v);
    else if (!strcmp(k, "DELTA_Y")) p->deltay = atof(v);
    else if (!strcmp(k, "DELTA_Z")) p->deltaz = atof(v);
    else if (!strcmp(k, "DELTA_t")) p->deltat = atof(v);
    else if (!strcmp(k, "NUMPHASES")) {
      p->numphases = atoi(v);
      if (p->numphases < 1 || p->numphases > GP_MAX_PHASES) {
        fclose(lr.f);
        gp_set_thread_error("NUMPHASES=%d outside 1..%d", p->numphases, GP_MAX_PHASES);
        return GP_EINVAL;
      }
    } else if (!strcmp(k, "NUMCOMPONENTS")) {
      p->numcomponents = atoi(v);
      if (p->numcomponents < 1 || p->numcomponents - 1 > GP_MAX_COMP) {
        fclose(lr.f);
        gp_set_thread_error("NUMCOMPONENTS=%d outside 1..%d", p->numcomponents, GP_MAX_COMP + 1);
        return GP_EINVAL;
      }
    }
    else if (!strcmp(k, "epsilon")) p->epsilon = atof(v);
    else if (!strcmp(k, "tau")) p->tau = atof(v);
    else if (!strcmp(k, "NTIMESTEPS")) p->ntimesteps = atol(v);
    else if (!strcmp(k, "SAVET")) p->savet = atol(v);
    else if (!strcmp(k, "NSMOOTH")) p->nsmooth = atol(v);
    else if (!strcmp(k, "STARTTIME")) p->starttime = atol(v);
    else if (!strcmp(k, "RESTART")) p->restart = atol(v);
    else if (!strcmp(k, "R")) p->R = atof(v);
    else if (!strcmp(k, "V")) p->V = atof(v);
    else if (!strcmp(k, "WRITEFORMAT")) {
      if (!strcmp(v, "ASCII")) p->ascii = 1;
      else if (!strcmp(v, "BINARY")) p->ascii = 0;
    }
    else if (!strcmp(k, "TRACK_PROGRESS")) p->track_progress = atol(v);
    else if (!strcmp(k, "TEMPERATURE_SCALE")) p->temperature_scale = atof(v);
    else if (!strcmp(k, "Equilibrium_temperature")) p->Teq = atof(v);
    else if (!strcmp(k, "Filling_temperature")) p->Tfill = atof(v);
    else if (!strcmp(k, "T")) p->T = atof(v);
    else if (!strcmp(k, "tilt_angle")) p->tilt_angle = atof(v);
    else if (!strcmp(k, "Rtheta")) p->Rtheta = atof(v);
    else if (!strcmp(k, "COMPONENTS")) pop_names(p->components, GP_MAX_COMP + 1, v);
    else if (!strcmp(k, "PHASES")) pop_names(p->phases, GP_MAX_PHASES, v);
    else if (!strcmp(k, "Function_anisotropy") && N > 0 && K > 0) p->function_anisotropy = atoi(v);
    else if (!strcmp(k, "Anisotropy_type") && p->function_anisotropy != 0) p->anisotropy_type = atoi(v);
    else if (!strcmp(k, "Rotation_matrix") && p->function_anisotropy != 0) {
      toklist tl;
      long p1, p2;
      split_tokens(v, &tl);
      p1 = tokl(&tl, 0); p2 = tokl(&tl, 1);
      if (p1 >= 0 && p2 >= 0 && p1 < GP_MAX_PHASES && p2 < GP_MAX_PHASES) {
        int i;
        for (i = 0; i < 3; i++) {
          p->rot_angles[p1][p2][i] = tokd(&tl, 2 + i);
          p->rot_angles[p2][p1][i] = tokd(&tl, 2 + i);
        }
        p->rot_set[p1][p2] = p->rot_set[p2][p1] = 1;
      }
    }
    else if (!strcmp(k, "OBSTACLE")) p->obstacle_key = atoi(v);
    else if (!strcmp(k, "Function_W") && N > 0 && K > 0) p->function_w = atoi(v);
    else if (!strcmp(k, "ISOTHERMAL")) {
      p->isothermal = atoi(v);
      if (!p->isothermal) p->tempgrady = 1;
    }
    else if (!strcmp(k, "Tempgrady") && p->tempgrady) {
      toklist tl;
      int i;
      split_tokens(v, &tl);
      for (i = 0; i < 5; i++) p->tempgrady_v[i] = tokd(&tl, i);
    }
    else if (!strcmp(k, "Shift")) p->shift = atoi(v);
    else if (!strcmp(k, "Shiftj")) { if (p->shift) p->shiftj = (int)atol(v); }
    else if (!strcmp(k, "BINARY")) { p->binary = atoi(v); p->ternary = 0; p->dilute = 0; }
    else if (!strcmp(k, "TERNARY")) { p->ternary = atoi(v); p->binary = 0; p->dilute = 0; }
    else if (!strcmp(k, "DILUTE")) { p->dilute = atoi(v); p->binary = 0; p->ternary = 0; }
    else if (!strcmp(k, "Writecomposition")) p->writecomposition = atoi(v);
    else if (!strcmp(k, "Noise_phasefield")) p->noise_phasefield = atoi(v);
    else if (!strcmp(k, "Amp_Noise_Phase")) { if (p->noise_phasefield) p->amp_noise_phase = atof(v); }
    else if (!strcmp(k, "GAMMA") && N > 0) { pop_pair_matrix(p->gamma, v, N); p->have_gamma = 1; }
    else if (!strcmp(k, "Tau") && N > 0) { pop_pair_matrix(p->tau_ab, v, N); p->have_tau_ab = 1; }
    else if (!strcmp(k, "dab") && N > 0) { pop_pair_matrix(p->dab, v, N); p->have_dab = 1; }
    else if ((!strcmp(k, "ec") || !strcmp(k, "e2") || !strcmp(k, "e4") || !strcmp(k, "beta")) && N > 0) { /* unused */ }
    else if (!strcmp(k, "Gamma_abc") && N > 0) { pop_triple(p->gamma_abc, v, N); p->have_gamma_abc = 1; }
    else if (!strcmp(k, "DIFFUSIVITY") && N > 0 && K > 0) pop_diffusivity(p, v);
    else if (!strcmp(k, "ceq") && N > 0 && K > 0) pop_thermo(p->ceq, v, K);
    else if (!strcmp(k, "cfill") && N > 0 && K > 0) pop_thermo(p->cfill, v, K);
    else if (!strcmp(k, "Function_F") && N > 0 && K > 0) p->function_f = atoi(v);
    else if (!strcmp(k, "A") && N > 0 && K > 0) pop_A(p, v);
    else if (!strcmp(k, "slopes") && N > 0 && K > 0) pop_thermo(p->slopes, v, K);
    /* EIGEN_STRAIN / VOIGT_ISOTROPIC and unknown keys: not used by this solver */
  }

  /* pass 2: read_boundary_conditions.h:29-41 with initialize_boundary_conditions /
   * initialize_boundary_points_values (utility_functions.h:376-470) */
  rewind(lr.f);
  lr.key[0] = lr.val[0] = 0;
  while (next_line(&lr)) {
    toklist tl;
    int f, s;
    if (lr.key[0] == '#' || p->numphases <= 0) continue;
    if (!strcmp(lr.key, "BOUNDARY")) {
      int t[6];
      split_tokens(lr.val, &tl);
      if (tl.n < 1 || (f = bc_field(tl.tok[0])) < 0) continue;
      /* {field, X+, X-, Y+, Y-, Z+, Z-} -> boundary[0]=X- .. [5]=Z- */
      t[0] = (int)tokl(&tl, 2); t[1] = (int)tokl(&tl, 1);
      t[2] = (int)tokl(&tl, 3); t[3] = (int)tokl(&tl, 4);
      t[4] = (int)tokl(&tl, 5); t[5] = (int)tokl(&tl, 6);
      if (t[0] == 3 || t[1] == 3) t[0] = t[1] = 3;
      if (t[2] == 3 || t[3] == 3) t[2] = t[3] = 3;
      if (t[4] == 3 || t[5] == 3) t[4] = t[5] = 3;
      if (p->dimension == 2) t[4] = t[5] = 0;
      for (s = 0; s < 6; s++) p->bc_type[f][s] = t[s];
    } else if (!strcmp(lr.key, "BOUNDARY_VALUE")) {
      split_tokens(lr.val, &tl);
      if (tl.n < 1 || (f = bc_field(tl.tok[0])) < 0) continue;
      p->bc_value[f][0] = tokd(&tl, 2); p->bc_value[f][1] = tokd(&tl, 1);
      p->bc_value[f][2] = tokd(&tl, 3); p->bc_value[f][3] = tokd(&tl, 4);
      p->bc_value[f][4] = tokd(&tl, 5); p->bc_value[f][5] = tokd(&tl, 6);
      /* the copy sources (proxies) are fixed from the types known now */
      for (s = 0; s < 6; s++) p->bc_proxy_type[f][s] = p->bc_type[f][s];
      p->bc_value_set[f] = 1;
    }
  }
  fclose(lr.f);
  return GP_OK;
}

/* ------------------------------------------------------- linear algebra */

/* matinvnew (matrix.h:50-218), restated for n <= 3 on fixed arrays.  Keeps the
 * reference's pivot rule (it compares |a[i][k]| against the SIGNED value of the
 * last pivot candidate, matrix.h:169-173), its reciprocal pow(x,-1) and its
 * final write-back of the row-permuted L*U product into m. */
void gp_host_matinv(double m[3][3], double inv[3][3], int n) {
  double fac[3][3] = {{0}}, inv1[3][3], prod[3][3], vec1[3], vec[3];
  int tag[3], i, j, k;
  for (k = 0; k < n; k++) tag[k] = k;
  for (k = 0; k < n; k++) {
    double big = fabs(m[k][k]);
    int t1 = k, ts;
    for (i = k + 1; i < n; i++)
      if (fabs(m[i][k]) > big) { t1 = i; big = m[i][k]; }
    ts = tag[k]; tag[k] = tag[t1]; tag[t1] = ts;
    for (i = 0; i < n; i++) { double s = m[k][i]; m[k][i] = m[t1][i]; m[t1][i] = s; }
    for (i = 0; i < k; i++) { double s = fac[k][i]; fac[k][i] = fac[t1][i]; fac[t1][i] = s; }
    for (i = k + 1; i < n; i++) {
      double f = -m[i][k] / m[k][k];
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
    /* forward substitution of unit column i (substitutef, matrix.h:143-160) */
    double s;
    int r;
    vec1[0] = (i == 0) ? 1.0 : 0.0;
    for (r = 1; r < n; r++) {
      s = 0;
      for (j = 0; j < r; j++) s = s - fac[r][j] * vec1[j];
      vec1[r] = ((r == i) ? 1.0 : 0.0) + s;
    }
    /* back substitution (substituteb, matrix.h:128-141) */
    vec[n - 1] = vec1[n - 1] * pow(m[n - 1][n - 1], -1);
    for (r = n - 2; r >= 0; r--) {
      s = 0;
      for (j = r + 1; j < n; j++) s = s - m[r][j] * vec[j];
      vec[r] = (vec1[r] + s) * pow(m[r][r], -1);
    }
    for (j = 0; j < n; j++) inv1[j][i] = vec[j];
  }
  for (j = 0; j < n; j++)
    for (i = 0; i < n; i++) inv[i][tag[j]] = inv1[i][j];
  for (k = 0; k < n; k++)
    for (i = 0; i < n; i++) {
      double s = 0;
      for (j = 0; j < n; j++) s = s + fac[k][j] * m[j][i];
      prod[k][i] = s;
    }
  for (j = 0; j < n; j++)
    for (i = 0; i < n; i++) m[tag[j]][i] = prod[j][i];
}

/* Rotation_matrix[a][b] and its inverse for the Euler angles of one pair
 * (get_Rotation_Matrix + populate_rotation_matrix, utility_functions.h:655-774). */
static void rotation_pair(const double ang[3], double R[3][3], double Rinv[3][3]) {
  double Rx[3][3], Ry[3][3], Rz[3][3], M[3][3];
  int axis, i, j, k;
  for (axis = 0; axis < 3; axis++) {
    double c = cos(ang[axis] * M_PI / 180.0), s = sin(ang[axis] * M_PI / 180.0);
    double (*r)[3] = axis == 0 ? Rx : axis == 1 ? Ry : Rz;
    if (axis == 0) {
      r[0][0] = 1.0; r[0][1] = 0.0; r[0][2] = 0.0; r[1][0] = 0.0; r[2][0] = 0.0;
      r[1][1] = c; r[1][2] = -s; r[2][1] = s; r[2][2] = c;
    } else if (axis == 1) {
      r[0][0] = c; r[0][1] = 0.0; r[0][2] = s; r[1][0] = 0.0; r[2][0] = -s;
      r[1][1] = 1.0; r[1][2] = 0.0; r[2][1] = 0.0; r[2][2] = c;
    } else {
      r[0][0] = c; r[0][1] = -s; r[0][2] = 0.0; r[1][0] = s; r[2][0] = 0.0;
      r[1][1] = c; r[1][2] = 0.0; r[2][1] = 0.0; r[2][2] = 1.0;
    }
  }
  for (k = 0; k < 3; k++)                      /* multiply2d, matrix.h:22-34 */
    for (i = 0; i < 3; i++) {
      double s = 0;
      for (j = 0; j < 3; j++) s = s + Rx[k][j] * Ry[j][i];
      M[k][i] = s;
    }
  for (k = 0; k < 3; k++)
    for (i = 0; i < 3; i++) {
      double s = 0;
      for (j = 0; j < 3; j++) s = s + M[k][j] * Rz[j][i];
      R[k][i] = s;
    }
  gp_host_matinv(R, Rinv, 3);
}

/* --------------------------------------------------- property matrices */

/* init_propertymatrices(Tq) (functionF_01.h:169-230) with function_B/_C
 * (functionF_01.h:62-104).  Only the values it leaves behind are returned. */
void gp_host_property_matrices(const gp_params *p, double Tq,
                               double B[GP_MAX_PHASES][GP_MAX_COMP], double C[GP_MAX_PHASES],
                               double cmu[GP_MAX_PHASES][GP_MAX_COMP][GP_MAX_COMP],
                               double Beq[GP_MAX_PHASES][GP_MAX_COMP],
                               double dBbdT[GP_MAX_PHASES][GP_MAX_COMP]) {
  int N = p->numphases, K = p->numcomponents - 1, L = N - 1;
  double DT[GP_MAX_PHASES][GP_MAX_PHASES] = {{0}}, DC[GP_MAX_PHASES][GP_MAX_COMP] = {{0}};
  double dcbdT[GP_MAX_PHASES][GP_MAX_PHASES][GP_MAX_COMP] = {{{0}}};
  int a, i, j, k;
  for (a = 0; a < N; a++) {
    double muc[3][3] = {{0}}, inv[3][3] = {{0}};
    for (i = 0; i < K; i++)
      for (j = 0; j < K; j++) muc[i][j] = (i == j) ? 2.0 * p->A[a][i][j] : p->A[a][i][j];
    gp_host_matinv(muc, inv, K);
    for (i = 0; i < K; i++)
      for (j = 0; j < K; j++) cmu[a][i][j] = inv[i][j];
  }
  for (a = 0; a < L; a++) {
    DT[a][L] = 0.0;
    DT[a][a] = 0.0;
    for (k = 0; k < K; k++) {
      DT[a][a] += p->slopes[a][a][k] * (p->ceq[a][L][k] - p->ceq[a][a][k]);
      DT[a][L] += p->slopes[a][L][k] * (p->ceq[a][L][k] - p->ceq[a][a][k]);
      DC[a][k] = p->ceq[a][L][k] - p->ceq[a][a][k];
    }
    for (k = 0; k < K; k++) {
      dcbdT[a][a][k] = DC[a][k] / DT[a][a];
      dcbdT[a][L][k] = DC[a][k] / DT[a][L];
    }
    for (k = 0; k < K; k++) {
      dBbdT[a][k] = 2.0 * (p->A[L][k][k] * dcbdT[a][L][k] - p->A[a][k][k] * dcbdT[a][a][k]);
      for (i = 0; i < K; i++)
        if (k != i) dBbdT[a][k] += (p->A[L][k][i] * dcbdT[a][L][i] - p->A[a][k][i] * dcbdT[a][a][i]);
    }
  }
  for (k = 0; k < K; k++) dBbdT[L][k] = 0.0;
  /* function_B at Teq, then B and C at Tq */
  for (int pass = 0; pass < 2; pass++) {
    double Tb = pass == 0 ? p->Teq : Tq;
    for (a = 0; a < N; a++) {
      double cl[GP_MAX_COMP], cs[GP_MAX_COMP];
      if (a != L)
        for (k = 0; k < K; k++) {
          cl[k] = p->ceq[a][L][k] - (DC[a][k]) * (p->Teq - Tb) / (DT[a][L]);
          cs[k] = p->ceq[a][a][k] - (DC[a][k]) * (p->Teq - Tb) / (DT[a][a]);
        }
      for (i = 0; i < K; i++) {
        double bai = 0.0, sum_c = 0.0;
        if (a != L) {
          for (k = 0; k < K; k++)
            if (k != i) sum_c += p->A[L][k][i] * cl[k] - p->A[a][k][i] * cs[k];
          bai = (2.0 * (p->A[L][i][i] * cl[i] - p->A[a][i][i] * cs[i]) + sum_c);
        }
        if (pass == 0) Beq[a][i] = bai; else B[a][i] = bai;
      }
      if (pass == 1) {
        double sum_c = 0.0;
        if (a != L)
          for (i = 0; i < K; i++)
            for (j = 0; j < K; j++)
              if (i <= j) sum_c += (p->A[a][i][j] * cs[i] * cs[j] - p->A[L][i][j] * cl[i] * cl[j]);
        C[a] = sum_c;
      }
    }
  }
}

/* --------------------------------------------------------------- derive */

int gp_host_derive(const gp_params *p, gp_derived *d, char *err, size_t errlen) {
  int N = p->numphases, K = p->numcomponents - 1, a, b, c, i, j, k, f;
  double B[GP_MAX_PHASES][GP_MAX_COMP], C[GP_MAX_PHASES], cmu[GP_MAX_PHASES][GP_MAX_COMP][GP_MAX_COMP];
  double Beq[GP_MAX_PHASES][GP_MAX_COMP], dBbdT[GP_MAX_PHASES][GP_MAX_COMP];
#define FAIL(...) do { snprintf(err, errlen, __VA_ARGS__); return GP_EINVAL; } while (0)
  memset(d, 0, sizeof *d);
  if (p->dimension != 2) FAIL("DIMENSION=%d: only 2-D is implemented", p->dimension);
  if (N < 2 || N > GPK_MAXN) FAIL("NUMPHASES=%d: kernels take 2..%d", N, GPK_MAXN);
  if (K < 1 || K > GPK_MAXK) FAIL("NUMCOMPONENTS=%d: kernels take 2..%d", p->numcomponents, GPK_MAXK + 1);
  if (p->mesh_x < 5 || p->mesh_y < 5) FAIL("MESH_X/MESH_Y must be >= 5");
  if (!p->isothermal && !p->tempgrady) FAIL("ISOTHERMAL=0 without Tempgrady");
  if (!p->isothermal && (p->tempgrady_v[2] == 0.0))
    FAIL("Tempgrady: Distance must be non-zero");
  if (p->noise_phasefield) FAIL("Noise_phasefield uses rand(); not reproducible, not implemented");
  if (p->function_f != 1) FAIL("Function_F=%d: only 1 (parabolic) exists", p->function_f);
  if (p->function_w != 1 && p->function_w != 2) FAIL("Function_W=%d: only 1 or 2", p->function_w);
  if (p->function_anisotropy != 0 && p->function_anisotropy != 1) FAIL("Function_anisotropy must be 0 or 1");
  if (p->function_anisotropy == 1 && p->anisotropy_type != 4) FAIL("Anisotropy_type must be 4 with Function_anisotropy=1");
  if (!p->have_gamma || !p->have_tau_ab) FAIL("GAMMA and Tau are required");
  if (p->function_anisotropy == 1 && !p->have_dab) FAIL("dab is required with Function_anisotropy=1");
  if (N > 2 && !p->have_gamma_abc) FAIL("Gamma_abc is required with NUMPHASES>2");
  if (p->deltax == 0.0 || p->deltay == 0.0) FAIL("DELTA_X/DELTA_Y must be non-zero");
  for (f = 0; f < 2; f++) {
    if (!p->bc_value_set[f]) FAIL("BOUNDARY_VALUE missing for %s", f ? "mu" : "phi");
    for (i = 0; i < 4; i++) {
      int t = p->bc_type[f][i];
      if (t != GP_BC_NEUMANN && t != GP_BC_PERIODIC)
        FAIL("boundary type %d on face %d of %s: the reference leaves those ghost cells "
             "to stale buffer contents; only Neumann(1) and Periodic(3) are implemented", t, i, f ? "mu" : "phi");
      if (p->bc_proxy_type[f][i] != t) FAIL("BOUNDARY_VALUE for %s precedes its BOUNDARY line", f ? "mu" : "phi");
    }
    d->bc_x[f][0] = p->bc_type[f][0]; d->bc_x[f][1] = p->bc_type[f][1];
    d->bc_y[f][0] = p->bc_type[f][3]; d->bc_y[f][1] = p->bc_type[f][2];
  }
  if (p->binary) d->inv_mode = GP_INV_BINARY;
  else if (p->ternary) d->inv_mode = GP_INV_TERNARY;
  else if (p->dilute) d->inv_mode = GP_INV_DILUTE;
  else d->inv_mode = GP_INV_GENERAL;
  if (d->inv_mode == GP_INV_TERNARY && K != 2) FAIL("TERNARY needs NUMCOMPONENTS=3");

  d->N = N; d->K = K;
  d->mx = p->mesh_x; d->my = p->mesh_y;
  d->dx = p->deltax; d->dy = p->deltay; d->dt = p->deltat;
  d->eps = p->epsilon; d->inv_eps = 1.0 / p->epsilon;
  d->tau = p->tau;
  d->c16pi2 = 16.0 / (M_PI * M_PI);
  d->jat_obst = -0.25 * M_PI * p->epsilon;
  d->jat_well = -1.0 * p->epsilon;
  d->well_half = 0.5 / sqrt(2.0);
  d->well = (p->function_w == 2);
  d->obstacle = !d->well;
  d->aniso = (p->function_anisotropy == 1);

  gp_host_property_matrices(p, p->T, B, C, cmu, Beq, dBbdT);
  for (a = 0; a < N; a++) {
    for (b = 0; b < N; b++) {
      d->gamma[a][b] = p->gamma[a][b];
      d->tau_ab[a][b] = p->tau_ab[a][b];
      d->dab[a][b] = p->dab[a][b];
      d->dab16[a][b] = 16.0 * p->dab[a][b];
      for (c = 0; c < N; c++) d->gamma_abc[a][b][c] = p->gamma_abc[a][b][c];
    }
    for (i = 0; i < K; i++) {
      d->E[a][i] = Beq[a][i] + dBbdT[a][i] * (p->T - p->Teq);
      d->twoA[a][i] = 2.0 * p->A[a][i][i];
      d->B[a][i] = B[a][i];
      for (j = 0; j < K; j++) {
        d->cmu[a][i][j] = cmu[a][i][j];
        d->A[a][i][j] = p->A[a][i][j];
        for (k = 0; k < K; k++) d->DC[a][i][j][k] = p->diffusivity[a][i][k] * cmu[a][k][j];
      }
      d->atf[a][i] = 1.0 - p->diffusivity[a][i][i] / p->diffusivity[N - 1][i][i];
    }
    d->C[a] = C[a];
  }
  /* D of a pure-phase cell: the same products and sum order as D()
   * (functionD.h:10-14) with phi_b = 1.0 for b == p and 0.0 otherwise */
  for (int q = 0; q < N; q++)
    for (i = 0; i < K; i++)
      for (j = 0; j < K; j++) {
        double s = 0.0;
        for (b = 0; b < N; b++)
          for (k = 0; k < K; k++) s += d->DC[b][i][j][k] * (b == q ? 1.0 : 0.0);
        d->Dbulk[q][i][j] = s;
      }
  /* the temperature field of a non-isothermal run, and the moving frame */
  d->tgrad = !p->isothermal;
  d->Teq = p->Teq;
  for (a = 0; a < N; a++)
    for (i = 0; i < K; i++) {
      d->Beq[a][i] = Beq[a][i];
      d->dBbdT[a][i] = dBbdT[a][i];
      d->ceql[a][i] = p->ceq[a][N - 1][i];
      d->ceqs[a][i] = p->ceq[a][a][i];
    }
  for (a = 0; a < N - 1; a++) {
    d->DTl[a] = 0.0;
    d->DTs[a] = 0.0;
    for (k = 0; k < K; k++) {
      d->DTs[a] += p->slopes[a][a][k] * (p->ceq[a][N - 1][k] - p->ceq[a][a][k]);
      d->DTl[a] += p->slopes[a][N - 1][k] * (p->ceq[a][N - 1][k] - p->ceq[a][a][k]);
      d->DCk[a][k] = p->ceq[a][N - 1][k] - p->ceq[a][a][k];
    }
  }
  d->tg_base = p->tempgrady_v[0];
  d->tg_dT = p->tempgrady_v[1];
  d->tg_dist = p->tempgrady_v[2];
  d->tg_off = p->tempgrady_v[3];
  d->tg_vel = p->tempgrady_v[4];
  d->bc_t[0] = p->bc_type[2][3];
  d->bc_t[1] = p->bc_type[2][2];
  d->shift = p->shift != 0;
  d->shiftj = p->shiftj;
  if (d->shift && (p->shiftj < 1 || p->shiftj >= p->mesh_y + 5)) FAIL("Shiftj=%ld outside the grid", (long)p->shiftj);
  for (i = 0; i < K; i++) {
    /* Mu(c, Tfill, N-1, i) with c = cfill of the liquid (shift.h:28-35, functionF_01.h:19-29) */
    int L = N - 1;
    double sm = 2.0 * p->A[L][i][i] * p->cfill[L][L][i] + (Beq[L][i] + dBbdT[L][i] * (p->Tfill - p->Teq));
    for (j = 0; j < K; j++)
      if (i != j) sm += p->A[L][i][j] * p->cfill[L][L][j];
    d->mu_fill[i] = sm;
  }
  d->rot_identity = 1;
  for (a = 0; a < N; a++)
    for (b = 0; b < N; b++) {
      double R[3][3], Ri[3][3];
      static const double zero[3] = {0.0, 0.0, 0.0};
      if (a == b) continue;
      /* a pair without a Rotation_matrix line rotates by the identity (the
       * reference would read uninitialised memory there) */
      rotation_pair(p->rot_set[a][b] ? p->rot_angles[a][b] : zero, R, Ri);
      for (i = 0; i < 2; i++)
        for (j = 0; j < 2; j++) {
          d->rot[a][b][i][j] = R[i][j];
          d->rinv[a][b][i][j] = Ri[i][j];
          if (R[i][j] != (i == j ? 1.0 : 0.0) || Ri[i][j] != (i == j ? 1.0 : 0.0)) d->rot_identity = 0;
        }
    }
  return GP_OK;
#undef FAIL
}
