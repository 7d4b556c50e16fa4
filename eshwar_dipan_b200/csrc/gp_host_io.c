/*
 * gp_host_io.c -- Filling.in and legacy-VTK I/O of libgp, host side, in C.
 * Keeps the reference's formats byte for byte (file_writer.h) and its filling
 * semantics (fill_domain.h, filling.h), including the coordinate offsets of the
 * three ghost layers.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gp_internal.h"

typedef struct {
  int N, K;
  long rx, ry, mx, my;
  double *phi;   /* [N][rx*ry] ghosted, as gridinfo[].phia */
  double *mu;    /* [K][rx*ry] */
} ggrid;

#define GI(g, x, y) ((long)(x) * (g)->ry + (y))

/* ---------------------------------------------------------------- fills */

/* Liquid pass shared by every fill (filling.h:29-46 and siblings). */
static void fill_liquid_cell(ggrid *g, long idx, int b) {
  int a;
  double sum = 0.0;
  for (a = 0; a < g->N - 1; a++) sum += g->phi[(long)a * g->rx * g->ry + idx];
  if (sum > 1.0) {
    g->phi[(long)b * g->rx * g->ry + idx] = 1.0;
    for (a = 0; a < g->N - 1; a++)
      if (a != b) g->phi[(long)a * g->rx * g->ry + idx] = 0.0;
  } else {
    g->phi[(long)b * g->rx * g->ry + idx] = 1.0 - sum;
  }
}

/* Solid pass: cell inside the shape -> phase b alone; outside -> clear b
 * unless it is already 1 (filling.h:17-27). */
static void fill_solid_cell(ggrid *g, long idx, int b, int inside) {
  long n = g->rx * g->ry;
  int a;
  if (inside) {
    g->phi[(long)b * n + idx] = 1.0;
    for (a = 0; a < g->N; a++)
      if (a != b) g->phi[(long)a * n + idx] = 0.0;
  } else if (g->phi[(long)b * n + idx] != 1.0) {
    g->phi[(long)b * n + idx] = 0.0;
  }
}

/* fill_phase_cube (filling.h:6-51); z is the single 2-D layer z=0. */
static void fill_cube(ggrid *g, long xs, long xe, long ys, long ye, long zs, long ze, int b) {
  long x, y, z = 0;
  for (x = 0; x < g->rx; x++)
    for (y = 0; y < g->ry; y++) {
      long idx = GI(g, x, y);
      if (b < g->N - 1)
        fill_solid_cell(g, idx, b, x >= xs && x <= xe && y >= ys && y <= ye && z >= zs && z <= ze);
      else
        fill_liquid_cell(g, idx, b);
    }
}

/* fill_phase_cylinder (filling.h:117-168): integer squared distance against
 * radius*radius in double. */
static void fill_cylinder(ggrid *g, long xc, long yc, long zs, long ze, double r, int b) {
  long x, y, z = 0;
  for (x = 0; x < g->rx; x++)
    for (y = 0; y < g->ry; y++) {
      long idx = GI(g, x, y);
      if (b < g->N - 1)
        fill_solid_cell(g, idx, b, ((x - xc) * (x - xc) + (y - yc) * (y - yc) <= r * r) && z >= zs && z <= ze);
      else
        fill_liquid_cell(g, idx, b);
    }
}

/* fill_phase_sphere (filling.h:169-219) */
static void fill_sphere(ggrid *g, long xc, long yc, long zc, double r, int b) {
  long x, y, z = 0;
  for (x = 0; x < g->rx; x++)
    for (y = 0; y < g->ry; y++) {
      long idx = GI(g, x, y);
      if (b < g->N - 1)
        fill_solid_cell(g, idx, b, (x - xc) * (x - xc) + (y - yc) * (y - yc) + (z - zc) * (z - zc) <= r * r);
      else
        fill_liquid_cell(g, idx, b);
    }
}

/* fill_phase_ellipse (filling.h:54-116).  Keeps the reference's indexing
 * (loops over 0..MESH-1 and addresses the ghosted array as x*MESH_Y+y).  The
 * reference evaluates its rotation from a variable read before it is set
 * (filling.h:62 uses `angle` before :69 assigns it); here the angle from the
 * Filling.in line is used. */
static void fill_ellipse(ggrid *g, long xc, long yc, double l, double e, double angle, int b) {
  long x, y;
  long n = g->rx * g->ry;
  double angle_rad = angle * M_PI / 180.0;
  for (x = 0; x <= g->mx - 1; x++)
    for (y = 0; y <= g->my - 1; y++) {
      if (b < g->N - 1) {
        double x_, y_;
        long gidy;
        int inside = (double)(x - xc) * (x - xc) / (l * l) + ((double)(y - yc) * (y - yc)) / (e * e * l * l) <= 1.0;
        if (inside) {
          x_ = xc + floor((double)(x - xc) * cos(angle_rad) + (double)(y - yc) * sin(angle_rad));
          y_ = yc + floor(-(double)(x - xc) * sin(angle_rad) + (double)(y - yc) * cos(angle_rad));
        } else {
          x_ = x;
          y_ = y;
        }
        gidy = (long)(x_ * g->my + y_);
        if (gidy < g->mx * g->my && gidy > 0) fill_solid_cell(g, gidy, b, inside);
      } else {
        long gidy = x * g->my + y;
        if (gidy < n) fill_liquid_cell(g, gidy, b);
      }
    }
}

/* Mu(c, Teq, a, i) with the property matrices at Teq (functionF_01.h:19-29). */
static double mu_of_c(const gp_params *p, const double *c, int a, int i,
                      double Beq[GP_MAX_PHASES][GP_MAX_COMP], double dBbdT[GP_MAX_PHASES][GP_MAX_COMP]) {
  int j, K = p->numcomponents - 1;
  double sum = 2.0 * p->A[a][i][i] * c[i] + (Beq[a][i] + dBbdT[a][i] * (p->Teq - p->Teq));
  for (j = 0; j < K; j++)
    if (i != j) sum += p->A[a][i][j] * c[j];
  return sum;
}

int gp_fill(const gp_params *p, const char *filling_path, double *phi, double *mu) {
  ggrid g;
  FILE *f;
  char buf[1000], key[128] = "", val[128] = "";
  double Bq[GP_MAX_PHASES][GP_MAX_COMP], Cq[GP_MAX_PHASES], cmu[GP_MAX_PHASES][GP_MAX_COMP][GP_MAX_COMP];
  double Beq[GP_MAX_PHASES][GP_MAX_COMP], dBbdT[GP_MAX_PHASES][GP_MAX_COMP];
  long x, y, n;
  int a, k;
  if (!p || !filling_path || !phi || !mu) { gp_set_thread_error("gp_fill: NULL argument"); return GP_EINVAL; }
  if (p->numphases < 2 || p->numcomponents < 2 || p->mesh_x < 1 || p->mesh_y < 1) {
    gp_set_thread_error("gp_fill: parameters not loaded");
    return GP_EINVAL;
  }
  g.N = p->numphases; g.K = p->numcomponents - 1;
  g.mx = p->mesh_x; g.my = p->mesh_y;
  g.rx = g.mx + 6; g.ry = g.my + 6;
  n = g.rx * g.ry;
  g.phi = calloc((size_t)g.N * n, sizeof(double));
  g.mu = calloc((size_t)g.K * n, sizeof(double));
  if (!g.phi || !g.mu) { free(g.phi); free(g.mu); gp_set_thread_error("gp_fill: out of memory"); return GP_ENOMEM; }
  f = fopen(filling_path, "rt");
  if (!f) { free(g.phi); free(g.mu); gp_set_thread_error("cannot open %s", filling_path); return GP_EIO; }
  while (fgets(buf, sizeof buf, f)) {
    char tmp[8][104];
    int nt = 0;
    char vb[128], *save = NULL, *t;
    sscanf(buf, "%100s = %100[^;];", key, val);
    if (key[0] == '#') continue;
    snprintf(vb, sizeof vb, "%s", val);
    for (t = strtok_r(vb, "{,}", &save); t && nt < 8; t = strtok_r(NULL, "{,}", &save))
      snprintf(tmp[nt++], sizeof tmp[0], "%s", t);
    for (; nt < 8; nt++) tmp[nt][0] = 0;
    /* coordinates are offset by the ghost width start[X]=start[Y]=3, start[Z]=0
     * (fill_domain.h:46-51,75-79,103-106,130-135) */
    if (!strcmp(key, "FILLCUBE")) {
      int ph = atoi(tmp[0]);
      if (ph < 0 || ph >= g.N) continue;
      fill_cube(&g, atol(tmp[1]) + 3, atol(tmp[4]) + 3, atol(tmp[2]) + 3, atol(tmp[5]) + 3,
                atol(tmp[3]), atol(tmp[6]), ph);
      fill_cube(&g, atol(tmp[1]) + 3, atol(tmp[4]) + 3, atol(tmp[2]) + 3, atol(tmp[5]) + 3,
                atol(tmp[3]), atol(tmp[6]), g.N - 1);
    } else if (!strcmp(key, "FILLCYLINDER")) {
      int ph = atoi(tmp[0]);
      if (ph < 0 || ph >= g.N) continue;
      fill_cylinder(&g, atol(tmp[1]) + 3, atol(tmp[2]) + 3, atol(tmp[3]), atol(tmp[4]), atof(tmp[5]), ph);
      fill_cylinder(&g, atol(tmp[1]) + 3, atol(tmp[2]) + 3, atol(tmp[3]), atol(tmp[4]), atof(tmp[5]), g.N - 1);
    } else if (!strcmp(key, "FILLSPHERE")) {
      int ph = atoi(tmp[0]);
      if (ph < 0 || ph >= g.N) continue;
      fill_sphere(&g, atol(tmp[1]) + 3, atol(tmp[2]) + 3, atol(tmp[3]), atof(tmp[4]), ph);
      fill_sphere(&g, atol(tmp[1]) + 3, atol(tmp[2]) + 3, atol(tmp[3]), atof(tmp[4]), g.N - 1);
    } else if (!strcmp(key, "FILLELLIPSE")) {
      int ph = atoi(tmp[0]);
      if (ph < 0 || ph >= g.N) continue;
      /* major axis, eccentricity and angle are read with atol (fill_domain.h:133-135) */
      fill_ellipse(&g, atol(tmp[1]) + 3, atol(tmp[2]) + 3, (double)atol(tmp[4]), (double)atol(tmp[5]),
                   (double)atol(tmp[6]), ph);
      fill_ellipse(&g, atol(tmp[1]) + 3, atol(tmp[2]) + 3, (double)atol(tmp[4]), (double)atol(tmp[5]),
                   (double)atol(tmp[6]), g.N - 1);
    }
  }
  fclose(f);
  /* fill_composition_cube (filling.h:221-270) */
  gp_host_property_matrices(p, p->Teq, Bq, Cq, cmu, Beq, dBbdT);
  for (x = 0; x < g.rx; x++)
    for (y = 0; y < g.ry; y++) {
      long idx = GI(&g, x, y);
      double c[GP_MAX_COMP];
      int filled = 0;
      for (a = 0; a < g.N - 1; a++) {
        if (g.phi[(long)a * n + idx] == 1.0) {
          for (k = 0; k < g.K; k++) c[k] = p->ceq[a][a][k];
          for (k = 0; k < g.K; k++) g.mu[(long)k * n + idx] = mu_of_c(p, c, a, k, Beq, dBbdT);
          filled = 1;
          break;
        }
      }
      if (!filled) {
        for (k = 0; k < g.K; k++) c[k] = p->cfill[g.N - 1][g.N - 1][k];
        for (k = 0; k < g.K; k++) g.mu[(long)k * n + idx] = mu_of_c(p, c, g.N - 1, k, Beq, dBbdT);
      }
    }
  for (a = 0; a < g.N; a++)
    for (x = 0; x < g.mx; x++)
      for (y = 0; y < g.my; y++)
        phi[((long)a * g.mx + x) * g.my + y] = g.phi[(long)a * n + GI(&g, x + 3, y + 3)];
  for (k = 0; k < g.K; k++)
    for (x = 0; x < g.mx; x++)
      for (y = 0; y < g.my; y++)
        mu[((long)k * g.mx + x) * g.my + y] = g.mu[(long)k * n + GI(&g, x + 3, y + 3)];
  free(g.phi);
  free(g.mu);
  return GP_OK;
}

/* ------------------------------------------------------------------ VTK */

/* hphi (functionH.h:24-36) */
static double host_hphi(const double *ph, int N, int a) {
  int b, c;
  double sum1 = 0.0;
  double sum = 3.0 * ph[a] * ph[a] - 2.0 * ph[a] * ph[a] * ph[a];
  for (b = 0; b < N; b++)
    for (c = 0; c < N; c++)
      if (b != a && c != a && b < c) sum1 += ph[b] * ph[c];
  sum1 *= 2.0 * ph[a];
  return sum + sum1;
}

static double be_double(double v) {
  uint64_t u;
  memcpy(&u, &v, 8);
  u = __builtin_bswap64(u);
  memcpy(&v, &u, 8);
  return v;
}

/* One row of MY values: lines of `fmt` (ASCII) or big-endian doubles
 * (binary), in one fwrite. */
static int put_row(FILE *f, const double *v, long MY, int ascii, const char *fmt, char *buf, size_t bufn) {
  long y;
  size_t n = 0;
  if (!ascii) {
    uint64_t *u = (uint64_t *)buf;
    for (y = 0; y < MY; y++) {
      memcpy(&u[y], &v[y], 8);
      u[y] = __builtin_bswap64(u[y]);
    }
    return fwrite(buf, 8, (size_t)MY, f) == (size_t)MY ? 0 : -1;
  }
  for (y = 0; y < MY; y++) {
    int w = snprintf(buf + n, bufn - n, fmt, v[y]);
    if (w < 0 || (size_t)w >= bufn - n) return -1;
    n += (size_t)w;
  }
  return fwrite(buf, 1, n, f) == n ? 0 : -1;
}

/* The temperature of each interior column y of a non-isothermal run after
 * `steps` time steps: temp_bottom + y_g*GRADIENT over the ghosted column y_g =
 * y + 3 (apply_temperature_gradientY, Temperature_gradient.h:4-29), with
 * BASE_POS and temp_bottom of microsim_gp.c:77-82 at steps = 0 and of
 * microsim_gp.c:108-113 after step `steps`.  shift_off is shift_OFFSET when
 * the field was laid down; when the frame then moved by dshift > 0 cells
 * (apply_shiftY, shift.h:4-45) column y_g holds the value laid at y_g + dshift,
 * the top dshift ghosted columns keep their own. */
void gp_host_temperature_column(const gp_derived *d, long long steps, long long shift_off, long dshift, double *Ty) {
  long y;
  const long ry = d->my + 6;
  double base_pos, grad, tb;
  if (steps == 0) base_pos = (d->tg_off / d->dy) - (double)shift_off;
  else base_pos = (d->tg_off / d->dy) - (double)shift_off + ((d->tg_vel / d->dy) * ((double)steps * d->dt));
  grad = (d->tg_dT) * d->dy / (d->tg_dist);
  tb = d->tg_base - base_pos * grad;
  for (y = 0; y < d->my; y++) {
    const long yg = y + 3;
    Ty[y] = yg <= ry - 1 - dshift ? tb + (double)(yg + dshift) * grad : tb + (double)yg * grad;
  }
}

int gp_vtk_write(const gp_params *p, const char *path, const double *phi, const double *mu, int ascii) {
  return gp_vtk_write_temperature(p, path, phi, mu, NULL, ascii);
}

/* write_cells_vtk_2D / write_cells_vtk_2D_binary (file_writer.h:71-255):
 * the same bytes, written a row at a time. */
int gp_vtk_write_temperature(const gp_params *p, const char *path, const double *phi, const double *mu,
                             const double *temperature, int ascii) {
  FILE *f;
  long x, y, MX, MY;
  int a, k, N, K, bad = 0;
  gp_derived d;
  char err[256];
  int have_d = 0;
  char *buf;
  double *row, *tcol = NULL;
  const double *T = temperature;
  size_t bufn;
  if (!p || !path || !phi || !mu) { gp_set_thread_error("gp_vtk_write: NULL argument"); return GP_EINVAL; }
  N = p->numphases; K = p->numcomponents - 1; MX = p->mesh_x; MY = p->mesh_y;
  if (p->writecomposition || (!p->isothermal && !T)) {
    if (gp_host_derive(p, &d, err, sizeof err) != GP_OK) {
      gp_set_thread_error("gp_vtk_write: %s", err);
      return GP_EINVAL;
    }
    have_d = 1;
  }
  if (!p->isothermal && !T) {
    /* the field laid down at start-up (microsim_gp.c:77-82) */
    tcol = malloc(sizeof(double) * (size_t)MY);
    if (!tcol) { gp_set_thread_error("gp_vtk_write: out of host memory"); return GP_ENOMEM; }
    gp_host_temperature_column(&d, 0, 0, 0, tcol);
  }
  bufn = (size_t)MY * 32 + 64;   /* "%le" is at most 13 characters plus sign and separators */
  buf = malloc(bufn);
  row = malloc(sizeof(double) * (size_t)MY);
  if (!buf || !row) {
    free(buf);
    free(row);
    free(tcol);
    gp_set_thread_error("gp_vtk_write: out of host memory");
    return GP_ENOMEM;
  }
  f = fopen(path, ascii ? "w" : "wb");
  if (!f) {
    free(buf);
    free(row);
    free(tcol);
    gp_set_thread_error("cannot write %s", path);
    return GP_EIO;
  }
  setvbuf(f, NULL, _IOFBF, (size_t)1 << 22);
  fprintf(f, "# vtk DataFile Version 3.0\n");
  fprintf(f, "Microsim_fields\n");
  fprintf(f, ascii ? "ASCII\n" : "BINARY\n");
  fprintf(f, "DATASET STRUCTURED_POINTS\n");
  fprintf(f, "DIMENSIONS %ld %ld %ld\n", MY, MX, (long)1);
  fprintf(f, "ORIGIN 0 0 0\n");
  fprintf(f, "SPACING %le %le %le\n", p->deltax, p->deltay, p->deltaz);
  fprintf(f, "POINT_DATA %ld\n", (long)MX * (long)MY);
  for (a = 0; a < N; a++) {
    fprintf(f, "SCALARS %s double 1\n", p->phases[a]);
    fprintf(f, "LOOKUP_TABLE default\n");
    for (x = 0; x < MX && !bad; x++) bad = put_row(f, phi + ((long)a * MX + x) * MY, MY, ascii, "%le\n", buf, bufn);
    if (ascii) fprintf(f, "\n");
  }
  for (k = 0; k < K; k++) {
    fprintf(f, "SCALARS Mu_%s double 1\n", p->components[k]);
    fprintf(f, "LOOKUP_TABLE default\n");
    for (x = 0; x < MX && !bad; x++) bad = put_row(f, mu + ((long)k * MX + x) * MY, MY, ascii, "%le\n", buf, bufn);
    if (ascii) fprintf(f, "\n");
  }
  if (p->writecomposition && have_d) {
    for (k = 0; k < K; k++) {
      fprintf(f, "SCALARS Composition_%s double 1\n", p->components[k]);
      fprintf(f, "LOOKUP_TABLE default\n");
      for (x = 0; x < MX && !bad; x++) {
        for (y = 0; y < MY; y++) {
          double ph[GP_MAX_PHASES], m[GP_MAX_COMP], comp = 0.0;
          int b, l;
          for (b = 0; b < N; b++) ph[b] = phi[((long)b * MX + x) * MY + y];
          for (l = 0; l < K; l++) m[l] = mu[((long)l * MX + x) * MY + y];
          for (b = 0; b < N; b++) {
            double cmu_v = 0.0;   /* c_mu (functionF_01.h:30-37), at the cell's temperature when not isothermal */
            if (p->isothermal)
              for (l = 0; l < K; l++) cmu_v += d.cmu[b][k][l] * (m[l] - d.E[b][l]);
            else {
              const double Tc = T ? T[x * MY + y] : tcol[y];
              for (l = 0; l < K; l++) cmu_v += d.cmu[b][k][l] * (m[l] - (d.Beq[b][l] + d.dBbdT[b][l] * (Tc - d.Teq)));
            }
            comp += cmu_v * host_hphi(ph, N, b);
          }
          row[y] = comp;
        }
        bad = put_row(f, row, MY, ascii, "%le \n", buf, bufn);
      }
      if (ascii) fprintf(f, "\n");
    }
  }
  if (!p->isothermal) {
    /* the temperature block, without a closing blank line (file_writer.h:138-148, 238-250) */
    fprintf(f, "SCALARS Temperature double 1\n");
    fprintf(f, "LOOKUP_TABLE default\n");
    for (x = 0; x < MX && !bad; x++) bad = put_row(f, T ? T + x * MY : tcol, MY, ascii, "%le \n", buf, bufn);
  }
  free(buf);
  free(row);
  free(tcol);
  if (fclose(f) != 0 || bad) { gp_set_thread_error("error writing %s", path); return GP_EIO; }
  return GP_OK;
}

/* Read one '\n'-terminated line; returns 0 at EOF. */
static int read_line(FILE *f, char *buf, size_t n) {
  size_t i = 0;
  int c;
  while ((c = fgetc(f)) != EOF) {
    if (c == '\n') { buf[i] = 0; return 1; }
    if (i + 1 < n) buf[i++] = (char)c;
  }
  buf[i] = 0;
  return i > 0;
}

/* read_cells_vtk_2D / read_cells_vtk_2D_binary (file_writer.h:256-416).  Header
 * lines are consumed one line at a time; the reference's fscanf("...\n") can
 * also swallow leading bytes of binary data that happen to be white space. */
int gp_vtk_read(const gp_params *p, const char *path, double *phi, double *mu, int ascii) {
  FILE *f;
  char line[512];
  long x, y, MX, MY;
  int a, k, i, N, K;
  if (!p || !path || !phi || !mu) { gp_set_thread_error("gp_vtk_read: NULL argument"); return GP_EINVAL; }
  N = p->numphases; K = p->numcomponents - 1; MX = p->mesh_x; MY = p->mesh_y;
  f = fopen(path, ascii ? "r" : "rb");
  if (!f) { gp_set_thread_error("cannot open %s", path); return GP_EIO; }
  for (i = 0; i < 8; i++)
    if (!read_line(f, line, sizeof line)) goto bad;
  for (a = 0; a < N + K; a++) {
    double *dst = a < N ? phi + (long)a * MX * MY : mu + (long)(a - N) * MX * MY;
    if (ascii) {
      /* a blank separator line follows each ASCII block */
      do { if (!read_line(f, line, sizeof line)) goto bad; } while (line[0] == 0);
    } else if (!read_line(f, line, sizeof line)) goto bad;
    if (strncmp(line, "SCALARS", 7) != 0) goto bad;
    if (!read_line(f, line, sizeof line)) goto bad;
    for (x = 0; x < MX; x++)
      for (y = 0; y < MY; y++) {
        double v;
        if (ascii) {
          if (fscanf(f, "%le", &v) != 1) goto bad;
        } else {
          if (fread(&v, 8, 1, f) != 1) goto bad;
          v = be_double(v);
        }
        dst[x * MY + y] = v;
      }
    if (ascii) { int c; while ((c = fgetc(f)) != EOF && c != '\n') {} }
  }
  (void)k;
  fclose(f);
  return GP_OK;
bad:
  fclose(f);
  gp_set_thread_error("malformed VTK file %s", path);
  return GP_EIO;
}
