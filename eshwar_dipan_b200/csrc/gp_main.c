/*
 * gp_main.c -- command-line driver with the reference's surface:
 *
 *     gp_microsim Input.in Filling.in NAME
 *
 * Same flow and files as main() of the serial solver (microsim_gp.c:41-151):
 * parse the input, fill (or restart from DATA/NAME_<STARTTIME>.vtk), write the
 * t=0 VTK, run NSMOOTH-1 smoothing sweeps, then NTIMESTEPS steps on the GPU,
 * writing DATA/NAME_<t>.vtk every SAVET steps (in the background, while the
 * next steps run; plus the frame position in DATA/shift.dat) and the progress
 * record every TRACK_PROGRESS steps.  A restart (STARTTIME, RESTART) reads the
 * state from DATA/NAME_<STARTTIME>.vtk and, with the moving frame, its
 * position from DATA/shift.dat.  The progress sums cover the interior cells
 * only (see gp_stats in gp.h).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include "gp.h"

static int die(const char *what, int rc, const gp_ctx *c) {
  fprintf(stderr, "gp_microsim: %s failed (%d): %s\n", what, rc, gp_last_error(c));
  return 1;
}

static long lgcd(long a, long b) {
  while (b) {
    long t = a % b;
    a = b;
    b = t;
  }
  return a;
}

int main(int argc, char **argv) {
  gp_params p;
  gp_ctx *c = NULL;
  gp_stats st;
  char path[1200];
  int rc, a, k, N, K, max_length;
  long t, chunk, shift_position = 0;
  double *phi, *mu;
  if (argc < 4) {
    fprintf(stderr, "usage: %s Input.in Filling.in NAME\n", argv[0]);
    return 2;
  }
  mkdir("DATA", 0777);
  if ((rc = gp_params_load(&p, argv[1])) != GP_OK) return die("reading the input file", rc, NULL);
  N = p.numphases;
  K = p.numcomponents - 1;
  phi = malloc(sizeof(double) * (size_t)N * p.mesh_x * p.mesh_y);
  mu = malloc(sizeof(double) * (size_t)K * p.mesh_x * p.mesh_y);
  if (!phi || !mu) return die("allocation", GP_ENOMEM, NULL);
  if (p.starttime == 0 && p.restart == 0) {
    if ((rc = gp_fill(&p, argv[2], phi, mu)) != GP_OK) return die("filling", rc, NULL);
  } else {
    snprintf(path, sizeof path, "DATA/%s_%ld.vtk", argv[3], p.starttime);
    if ((rc = gp_vtk_read(&p, path, phi, mu, p.ascii)) != GP_OK) return die("reading the restart file", rc, NULL);
    if (p.shift) {
      /* the frame position at STARTTIME: line STARTTIME/SAVET of DATA/shift.dat (microsim_gp.c:58-66) */
      FILE *fs = fopen("DATA/shift.dat", "r");
      long i, tf = 0, pos = 0;
      if (!fs) return die("reading DATA/shift.dat", GP_EIO, NULL);
      for (i = 0; i <= p.starttime / (p.savet > 0 ? p.savet : 1); i++)
        if (fscanf(fs, "%ld %ld\n", &tf, &pos) != 2) break;
      fclose(fs);
      shift_position = pos;
    }
    if (!p.isothermal) {
      /* the temperature field resumes where it was (microsim_gp.c:67-73) */
      if (p.shift)
        p.tempgrady_v[3] = (p.tempgrady_v[3]) + floor((p.tempgrady_v[4]) * (p.starttime * p.deltat)) -
                           shift_position * p.deltay;
      else
        p.tempgrady_v[3] = (p.tempgrady_v[3]) + floor((p.tempgrady_v[4]) * (p.starttime * p.deltat));
    }
  }
  if ((rc = gp_init(&c, &p, phi, mu, GP_FP64)) != GP_OK) return die("gp_init", rc, NULL);
  if (p.restart == 0 || p.starttime == 0) {
    snprintf(path, sizeof path, "DATA/%s_%ld.vtk", argv[3], 0L);
    if ((rc = gp_vtk_write(&p, path, phi, mu, p.ascii)) != GP_OK) return die("writing VTK", rc, c);
  }
  if (p.nsmooth > 1 && (rc = gp_smooth(c, p.nsmooth - 1)) != GP_OK) return die("gp_smooth", rc, c);
  max_length = 0;
  for (a = 0; a < N; a++)
    if ((int)strlen(p.phases[a]) > max_length) max_length = (int)strlen(p.phases[a]);
  for (k = 0; k < K; k++)
    if ((int)strlen(p.components[k]) > max_length) max_length = (int)strlen(p.components[k]);
  /* advance in chunks that end on every SAVET and TRACK_PROGRESS boundary */
  {
    long s = p.savet > 0 ? p.savet : p.ntimesteps, q = p.track_progress > 0 ? p.track_progress : p.ntimesteps;
    chunk = s > 0 && q > 0 ? lgcd(s, q) : 1;
    if (chunk <= 0) chunk = 1;
  }
  for (t = 0; t < p.ntimesteps;) {
    long n = chunk - (t % chunk);
    if (t + n > p.ntimesteps) n = p.ntimesteps - t;
    /* non-finite cells do not stop the run (the reference keeps stepping);
     * they are reported with the progress record */
    if ((rc = gp_step(c, n, &st)) != GP_OK && rc != GP_ENONFINITE) return die("gp_step", rc, c);
    t += n;
    if (p.savet > 0 && t % p.savet == 0) {
      FILE *f;
      /* written in the background while the next steps run */
      snprintf(path, sizeof path, "DATA/%s_%ld.vtk", argv[3], t + p.starttime);
      if ((rc = gp_vtk_write_async(c, path, p.ascii)) != GP_OK) return die("writing VTK", rc, c);
      f = fopen("DATA/shift.dat", "a");
      if (f) {
        fprintf(f, "%ld %ld\n", t + p.starttime, (long)st.shift_offset + shift_position);
        fclose(f);
      }
    }
    if (p.track_progress > 0 && t % p.track_progress == 0) {
      fprintf(stdout, "Time=%le\n", t * p.deltat);
      for (a = 0; a < N; a++)
        fprintf(stdout, "%*s, Max = %le, Min = %le, Relative_Change=%le\n", max_length, p.phases[a], st.phi_max[a],
                st.phi_min[a], sqrt(st.rel_change_phi[a]));
      for (k = 0; k < K; k++)
        fprintf(stdout, "%*s, Max = %le, Min = %le, Relative_Change=%le\n", max_length, p.components[k],
                st.mu_max[k], st.mu_min[k], sqrt(st.rel_change_mu[k]));
      fprintf(stdout, "\n");
      if (st.nonfinite) fprintf(stderr, "gp_microsim: %lld cells are not finite\n", st.nonfinite);
    }
  }
  if ((rc = gp_vtk_wait(c)) != GP_OK) return die("writing VTK", rc, c);
  gp_destroy(c);
  free(phi);
  free(mu);
  return 0;
}
