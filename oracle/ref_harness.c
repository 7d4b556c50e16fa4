/*
 * ref_harness.c -- test infrastructure, not product code.
 *
 * Drives the UNMODIFIED reference serial grand-potential solver
 * (Grand_potential_Finite_difference_2D_serial) one pass at a time so that its
 * full state can be dumped and compared with the oracle restatement and with
 * the CUDA path.  The reference sources are #included from where they lie (the
 * include path is given by oracle/Makefile); nothing of the reference is
 * copied.  The include list mirrors microsim_gp.c:7-39 of the reference.
 *
 * Differences from the reference main (microsim_gp.c:41-151), all outside the
 * time loop:
 *   - boundary conditions are read with the reference's own
 *     initialize_boundary_conditions / initialize_boundary_points_values, but
 *     without PRINT_BOUNDARY_CONDITIONS, whose 10-byte key buffers overflow
 *     (utility_functions.h:880-891) and crash the reference at random;
 *   - no VTK files are written unless asked for (mode "vtk");
 *   - the state can be loaded from a raw binary file instead of filled.
 * Mode "main" runs the sequence of the reference's main() (microsim_gp.c:48-150)
 * with the reference's own routines: fill or read the restart file
 * DATA/NAME_<STARTTIME>.vtk, boundary copies, the t=0 file, NSMOOTH-1
 * smoothing sweeps, then NTIMESTEPS steps writing DATA/NAME_<t>.vtk and a
 * DATA/shift.dat line every SAVET steps and the progress record every
 * TRACK_PROGRESS steps on stdout, with the temperature field of a
 * non-isothermal run and the moving frame (Shift).
 *
 * Usage:
 *   gp_ref_harness IN FILL run   NSMOOTH NSTEPS OUT.bin   (NSMOOTH<0: from IN)
 *   gp_ref_harness IN FILL load  STATE.bin NSMOOTH NSTEPS OUT.bin
 *   gp_ref_harness IN FILL time  NSTEPS                   (prints seconds)
 *   gp_ref_harness IN FILL consts OUT.txt
 *   gp_ref_harness IN FILL vtk   NSTEPS NAME              (reference writer)
 *   gp_ref_harness IN FILL main  NAME                     (main()'s flow: see below)
 *
 * OUT.bin layout (little endian): "GPRF", int32 rows_x, rows_y, N, K, then
 * float64 phi[N][rows_x][rows_y], mu[K][..], dphi[N][..], then the reference's
 * progress record phi_max[N], phi_min[N], mu_max[K], mu_min[K],
 * rel_change_phi[N], rel_change_mu[K].
 * STATE.bin layout: "GPST", int32 MESH_X, MESH_Y, N, K, then interior
 * float64 phi[N][MESH_X][MESH_Y], mu[K][MESH_X][MESH_Y].
 */
#include <stdio.h>
#include <math.h>
#include <string.h>
#include <stdlib.h>
#include <stdbool.h>
#include <sys/stat.h>
#include <time.h>
#include "functions/global_vars.h"
#include "functions/functions.h"
#include "functions/matrix.h"
#include "functions/utility_functions.h"
#include "functions/functionH.h"
#include "functions/functionF_01.h"
#include "functions/functionQ.h"
#include "functions/functionW_01.h"
#include "functions/functionW_02.h"
#include "functions/function_A_00.h"
#include "functions/function_A_01.h"
#include "functions/anisotropy_01.h"
#include "functions/functionTau.h"
#include "functions/functionD.h"
#include "functions/filling.h"
#include "functions/reading_input_parameters.h"
#include "functions/read_boundary_conditions.h"
#include "functions/initialize_variables.h"
#include "functions/free_variables.h"
#include "functions/fill_domain.h"
#include "functions/shift.h"
#include "functions/Temperature_gradient.h"
#include "solverloop/serialinfo_xy.h"
#include "solverloop/gradients.h"
#include "solverloop/simplex_projection.h"
#include "solverloop/calculate_gradients.h"
#include "solverloop/calculate_fluxes_concentration.h"
#include "solverloop/calculate_divergence_phasefield.h"
#include "solverloop/calculate_divergence_concentration.h"
#include "solverloop/initialize_functions_solverloop.h"
#include "solverloop/solverloop.h"
#include "solverloop/boundary_serial.h"
#include "solverloop/file_writer.h"

/* Boundary-condition reader: the loop of read_boundary_conditions.h:29-41
 * without the echo file. */
static void harness_read_bc(const char *path) {
  char buf[1000], k1[128], v1[128];
  FILE *fr = fopen(path, "rt");
  if (!fr) { fprintf(stderr, "cannot open %s\n", path); exit(2); }
  k1[0] = v1[0] = 0;
  while (fgets(buf, sizeof buf, fr)) {
    sscanf(buf, "%100s = %100[^;];", k1, v1);
    if (k1[0] != '#') {
      if (strcmp(k1, "BOUNDARY") == 0 && NUMPHASES > 0) {
        initialize_boundary_conditions(v1);
      } else if (strcmp(k1, "BOUNDARY_VALUE") == 0 && NUMPHASES > 0) {
        initialize_boundary_points_values(v1);
      }
    }
  }
  fclose(fr);
}

static void setup(char **argv) {
  char *av[4];
  av[0] = argv[0]; av[1] = argv[1]; av[2] = argv[2]; av[3] = "harness";
  reading_input_parameters(av);
  initialize_variables();
  serialinfo_xy();
  initialize_functions_solverloop();
  harness_read_bc(argv[1]);
}

static void fill(char **argv) {
  char *av[4];
  av[0] = argv[0]; av[1] = argv[1]; av[2] = argv[2]; av[3] = "harness";
  fill_domain(av);
}

static void put_i32(FILE *f, int v) { fwrite(&v, 4, 1, f); }

static void dump_state(const char *path) {
  long a, k, i, n = rows_x * rows_y;
  FILE *f = fopen(path, "wb");
  if (!f) { fprintf(stderr, "cannot write %s\n", path); exit(2); }
  fwrite("GPRF", 1, 4, f);
  put_i32(f, (int)rows_x); put_i32(f, (int)rows_y);
  put_i32(f, NUMPHASES); put_i32(f, NUMCOMPONENTS - 1);
  for (a = 0; a < NUMPHASES; a++)
    for (i = 0; i < n; i++) fwrite(&gridinfo[i].phia[a], 8, 1, f);
  for (k = 0; k < NUMCOMPONENTS - 1; k++)
    for (i = 0; i < n; i++) fwrite(&gridinfo[i].compi[k], 8, 1, f);
  for (a = 0; a < NUMPHASES; a++)
    for (i = 0; i < n; i++) fwrite(&gridinfo[i].deltaphi[a], 8, 1, f);
  fwrite(global_max_min.phi_max, 8, NUMPHASES, f);
  fwrite(global_max_min.phi_min, 8, NUMPHASES, f);
  fwrite(global_max_min.mu_max, 8, NUMCOMPONENTS - 1, f);
  fwrite(global_max_min.mu_min, 8, NUMCOMPONENTS - 1, f);
  fwrite(global_max_min.rel_change_phi, 8, NUMPHASES, f);
  fwrite(global_max_min.rel_change_mu, 8, NUMCOMPONENTS - 1, f);
  fclose(f);
}

static void load_state(const char *path) {
  char magic[4];
  int hdr[4];
  long a, k, x, y;
  FILE *f = fopen(path, "rb");
  if (!f || fread(magic, 1, 4, f) != 4 || memcmp(magic, "GPST", 4) != 0 ||
      fread(hdr, 4, 4, f) != 4) {
    fprintf(stderr, "bad state file %s\n", path); exit(2);
  }
  if (hdr[0] != MESH_X || hdr[1] != MESH_Y || hdr[2] != NUMPHASES ||
      hdr[3] != NUMCOMPONENTS - 1) {
    fprintf(stderr, "state shape does not match the input file\n"); exit(2);
  }
  for (a = 0; a < NUMPHASES; a++)
    for (x = 0; x < MESH_X; x++)
      for (y = 0; y < MESH_Y; y++) {
        double v;
        if (fread(&v, 8, 1, f) != 1) { fprintf(stderr, "short state\n"); exit(2); }
        gridinfo[(x + 3) * layer_size + (y + 3)].phia[a] = v;
      }
  for (k = 0; k < NUMCOMPONENTS - 1; k++)
    for (x = 0; x < MESH_X; x++)
      for (y = 0; y < MESH_Y; y++) {
        double v;
        if (fread(&v, 8, 1, f) != 1) { fprintf(stderr, "short state\n"); exit(2); }
        gridinfo[(x + 3) * layer_size + (y + 3)].compi[k] = v;
      }
  fclose(f);
  for (x = 0; x < rows_x * rows_y; x++)
    for (a = 0; a < NUMPHASES; a++) gridinfo[x].deltaphi[a] = 0.0;
  /* the filled path leaves the property matrices at T (filling.h:269) */
  init_propertymatrices(T);
}

/* microsim_gp.c:77-82: the temperature field of a non-isothermal run at t = 0 */
static void temp_init(void) {
  if (TEMPGRADY) {
    BASE_POS = (temperature_gradientY.gradient_OFFSET / deltay) - shift_OFFSET;
    GRADIENT = (temperature_gradientY.DeltaT) * deltay / (temperature_gradientY.Distance);
    temp_bottom = temperature_gradientY.base_temp - BASE_POS * GRADIENT;
    apply_temperature_gradientY(gridinfo, shift_OFFSET, 0);
  }
}

/* microsim_gp.c:108-126: after step t, the temperature field moves with the
 * gradient and, with Shift, every 100 steps the frame follows the interface */
static void after_step(long tt) {
  if (TEMPGRADY) {
    BASE_POS = (temperature_gradientY.gradient_OFFSET / deltay) - shift_OFFSET +
               ((temperature_gradientY.velocity / deltay) * (tt * deltat));
    GRADIENT = (temperature_gradientY.DeltaT) * deltay / (temperature_gradientY.Distance);
    temp_bottom = temperature_gradientY.base_temp - BASE_POS * GRADIENT;
    apply_temperature_gradientY(gridinfo, shift_OFFSET, tt);
  }
  if (tt % 100 == 0) {
    if (SHIFT) {
      if (MAX_INTERFACE_POS > shiftj) shift_ON = 1;
      if (shift_ON) {
        apply_shiftY(gridinfo, MAX_INTERFACE_POS);
        shift_OFFSET += (MAX_INTERFACE_POS - shiftj);
        shift_ON = 0;
      }
    }
  }
}

static void smooth_steps(long ns) {
  long s;
  for (s = 1; s < ns; s++) {           /* microsim_gp.c:97-100 */
    smooth(start, end);
    apply_boundary_conditions(0);
  }
}

static void time_steps(long nsteps) {
  long s;
  for (s = 1; s <= nsteps; s++) {      /* microsim_gp.c:102-126 */
    t = (int)s;
    solverloop_phasefield(start, end);
    apply_boundary_conditions(0);
    solverloop_concentration(start, end);
    apply_boundary_conditions(0);
    after_step(s);
  }
}

static void dump_consts(const char *path) {
  long a, b, i, j;
  FILE *f = fopen(path, "w");
  if (!f) exit(2);
  for (a = 0; a < NUMPHASES; a++) {
    for (i = 0; i < NUMCOMPONENTS - 1; i++) {
      fprintf(f, "B %ld %ld %a\n", a, i, B[a][i]);
      fprintf(f, "Beq %ld %ld %a\n", a, i, Beq[a][i]);
      fprintf(f, "dBbdT %ld %ld %a\n", a, i, dBbdT[a][i]);
      for (j = 0; j < NUMCOMPONENTS - 1; j++)
        fprintf(f, "cmu %ld %ld %ld %a\n", a, i, j, cmu[a][i][j]);
    }
    fprintf(f, "C %ld %a\n", a, C[a]);
  }
  if (FUNCTION_ANISOTROPY)
    for (a = 0; a < NUMPHASES; a++)
      for (b = 0; b < NUMPHASES; b++)
        if (a != b)
          for (i = 0; i < 3; i++)
            for (j = 0; j < 3; j++) {
              fprintf(f, "R %ld %ld %ld %ld %a\n", a, b, i, j, Rotation_matrix[a][b][i][j]);
              fprintf(f, "Rinv %ld %ld %ld %ld %a\n", a, b, i, j, Inv_Rotation_matrix[a][b][i][j]);
            }
  fclose(f);
}

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

int main(int argc, char *argv[]) {
  if (argc < 4) {
    fprintf(stderr, "usage: %s IN FILL run|load|time|consts|vtk ...\n", argv[0]);
    return 2;
  }
  const char *mode = argv[3];
  setup(argv);
  if (strcmp(mode, "run") == 0 && argc == 7) {
    long ns = atol(argv[4]);
    fill(argv);
    temp_init();
    apply_boundary_conditions(0);
    smooth_steps(ns < 0 ? nsmooth : ns);
    time_steps(atol(argv[5]));
    dump_state(argv[6]);
  } else if (strcmp(mode, "load") == 0 && argc == 8) {
    long ns = atol(argv[5]);
    load_state(argv[4]);
    temp_init();
    apply_boundary_conditions(0);
    smooth_steps(ns < 0 ? nsmooth : ns);
    time_steps(atol(argv[6]));
    dump_state(argv[7]);
  } else if (strcmp(mode, "time") == 0 && argc == 5) {
    double t0, t1;
    fill(argv);
    temp_init();
    apply_boundary_conditions(0);
    smooth_steps(nsmooth);
    t0 = now_s();
    time_steps(atol(argv[4]));
    t1 = now_s();
    printf("%.9f\n", t1 - t0);
  } else if (strcmp(mode, "consts") == 0 && argc == 5) {
    fill(argv);
    dump_consts(argv[4]);
  } else if (strcmp(mode, "vtk") == 0 && argc == 6) {
    char *av[4];
    av[0] = argv[0]; av[1] = argv[1]; av[2] = argv[2]; av[3] = argv[5];
    mkdir("DATA", 0777);
    fill(argv);
    temp_init();
    apply_boundary_conditions(0);
    smooth_steps(nsmooth);
    time_steps(atol(argv[4]));
    if (ASCII) writetofile_serial2D(gridinfo, av, atol(argv[4]));
    else writetofile_serial2D_binary(gridinfo, av, atol(argv[4]));
  } else if (strcmp(mode, "main") == 0 && argc == 5) {
    char *av[4];
    FILE *fs;
    av[0] = argv[0]; av[1] = argv[1]; av[2] = argv[2]; av[3] = argv[4];
    mkdir("DATA", 0777);
    if ((STARTTIME == 0) && (RESTART == 0)) {
      fill(argv);
    } else {
      if (ASCII) readfromfile_serial2D(gridinfo, av, STARTTIME);
      else readfromfile_serial2D_binary(gridinfo, av, STARTTIME);
      init_propertymatrices(T);
      if (SHIFT) {
        FILE *fp = fopen("DATA/shift.dat", "r");
        for (file_iter = 0; file_iter <= STARTTIME / saveT; file_iter++) fscanf(fp, "%ld %ld\n", &time_file, &position);
        fclose(fp);
        shift_position = position;
      }
      if (!ISOTHERMAL) {
        if (SHIFT)
          temperature_gradientY.gradient_OFFSET = (temperature_gradientY.gradient_OFFSET) +
                                                  floor((temperature_gradientY.velocity) * (STARTTIME * deltat)) -
                                                  shift_position * deltay;
        else
          temperature_gradientY.gradient_OFFSET = (temperature_gradientY.gradient_OFFSET) +
                                                  floor((temperature_gradientY.velocity) * (STARTTIME * deltat));
      }
    }
    temp_init();
    apply_boundary_conditions(0);
    if ((RESTART == 0) || (STARTTIME == 0)) {
      if (ASCII == 0) writetofile_serial2D_binary(gridinfo, av, 0);
      else writetofile_serial2D(gridinfo, av, 0);
    }
    smooth_steps(nsmooth);
    for (t = 1; t <= ntimesteps; t++) {
      solverloop_phasefield(start, end);
      apply_boundary_conditions(0);
      solverloop_concentration(start, end);
      apply_boundary_conditions(0);
      after_step(t);
      if (t % saveT == 0) {
        if (ASCII == 0) writetofile_serial2D_binary(gridinfo, av, t + STARTTIME);
        else writetofile_serial2D(gridinfo, av, t + STARTTIME);
        fs = fopen("DATA/shift.dat", "a");
        if (fs) {
          fprintf(fs, "%ld %ld\n", t + STARTTIME, shift_OFFSET + shift_position);
          fclose(fs);
        }
      }
      if (t % time_output == 0) {
        fprintf(stdout, "Time=%le\n", t * deltat);
        for (b = 0; b < NUMPHASES; b++)
          fprintf(stdout, "%*s, Max = %le, Min = %le, Relative_Change=%le\n", max_length, Phases[b],
                  global_max_min.phi_max[b], global_max_min.phi_min[b], sqrt(global_max_min.rel_change_phi[b]));
        for (k = 0; k < NUMCOMPONENTS - 1; k++)
          fprintf(stdout, "%*s, Max = %le, Min = %le, Relative_Change=%le\n", max_length, Components[k],
                  global_max_min.mu_max[k], global_max_min.mu_min[k], sqrt(global_max_min.rel_change_mu[k]));
        fprintf(stdout, "\n");
      }
    }
  } else {
    fprintf(stderr, "bad arguments for mode %s\n", mode);
    return 2;
  }
  return 0;
}
