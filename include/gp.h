/*
 * gp.h -- C ABI of libgp, a B200 (sm_100a) implementation of MicroSim's 2D
 * grand-potential finite-difference time step (serial solver,
 * Grand_potential_Finite_difference_2D_serial of the reference).
 *
 * The reference has no library boundary: main() (microsim_gp.c:41-151) calls
 * the solver passes directly on global state.  Each entry point below names the
 * reference routine(s) it replaces.  Conventions:
 *   - every call returns 0 (GP_OK) or a negative GP_E* code; gp_last_error()
 *     gives a message for the last failure on a context (or, with NULL, for
 *     the calling thread's last context-free failure);
 *   - the caller owns all host buffers; the library owns all device buffers;
 *   - fields cross the boundary as interior-only planes in the reference's
 *     order: phi[a][x][y] (a < NUMPHASES), mu[k][x][y] (k < NUMCOMPONENTS-1),
 *     x < MESH_X, y < MESH_Y, y contiguous (file_writer.h:172-183);
 *   - one host thread per context; work is ordered on the context's stream and
 *     every call that returns data synchronises before returning.
 * Plain C types only: no CUDA or torch types cross this boundary.
 */
#ifndef GP_H_
#define GP_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GP_MAX_PHASES 6   /* parsing limit; the CUDA kernels take N <= 4 */
#define GP_MAX_COMP   4   /* independent components K = NUMCOMPONENTS-1; kernels take K <= 2 */
#define GP_NAME_LEN   52

enum {
  GP_OK = 0,
  GP_EINVAL = -1,        /* bad argument or unsupported parameter combination */
  GP_ENOMEM = -2,        /* host or device allocation failed */
  GP_ECUDA = -3,         /* CUDA runtime error (no device, launch failure, ...) */
  GP_ETIMEOUT = -4,      /* a bounded device-side wait gave up */
  GP_ENONFINITE = -5,    /* the state holds non-finite values */
  GP_EIO = -6,           /* file could not be read or written */
  GP_EUNSUPPORTED = -7   /* the reference path exists but is not built here */
};

typedef enum { GP_FP64 = 0, GP_FP32 = 1 } gp_precision;

/* Boundary types as in the reference (utility_functions.h:471-654,
 * Input.in "0: Free, 1: Neumann, 2: Dirichlet, 3: Periodic"). */
enum { GP_BC_FREE = 0, GP_BC_NEUMANN = 1, GP_BC_DIRICHLET = 2, GP_BC_PERIODIC = 3 };
/* Faces, in the reference's boundary[] order: 0 X-, 1 X+, 2 Y+, 3 Y-, 4 Z+, 5 Z-.
 * Fields: 0 phi, 1 mu, 2 T (assign_buffer_points_conditions, utility_functions.h:471). */

/*
 * Parameters of one simulation: the reference's globals after
 * reading_input_parameters() (reading_input_parameters.h:1-307) and
 * read_boundary_conditions() (read_boundary_conditions.h:4-57).  Field names
 * follow the Input.in keys.  Arrays are indexed as in the reference:
 * gamma[a][b], diffusivity[phase][i][j], A[phase][i][j],
 * ceq/cfill/slopes[phase1][phase2][comp].
 */
typedef struct gp_params {
  int dimension;
  long mesh_x, mesh_y, mesh_z;
  double deltax, deltay, deltaz, deltat;
  int numphases, numcomponents;           /* as in Input.in: K = numcomponents-1 */
  long ntimesteps, savet, nsmooth, starttime, restart, track_progress;
  double R, V, T, Teq, Tfill, temperature_scale, tilt_angle, Rtheta;
  double epsilon, tau;
  int function_f, function_w, function_anisotropy, anisotropy_type;
  int obstacle_key;                       /* OBSTACLE key if present (-1 absent) */
  int isothermal, tempgrady, binary, ternary, dilute;
  int shift, shiftj, writecomposition, noise_phasefield, ascii;
  double amp_noise_phase;
  double tempgrady_v[5];                  /* base, DeltaT, Distance, OFFSET, velocity */
  double gamma[GP_MAX_PHASES][GP_MAX_PHASES];
  double tau_ab[GP_MAX_PHASES][GP_MAX_PHASES];
  double dab[GP_MAX_PHASES][GP_MAX_PHASES];
  double gamma_abc[GP_MAX_PHASES][GP_MAX_PHASES][GP_MAX_PHASES];
  double diffusivity[GP_MAX_PHASES][GP_MAX_COMP][GP_MAX_COMP];
  double A[GP_MAX_PHASES][GP_MAX_COMP][GP_MAX_COMP];
  double ceq[GP_MAX_PHASES][GP_MAX_PHASES][GP_MAX_COMP];
  double cfill[GP_MAX_PHASES][GP_MAX_PHASES][GP_MAX_COMP];
  double slopes[GP_MAX_PHASES][GP_MAX_PHASES][GP_MAX_COMP];
  /* Rotation_matrix = {p1, p2, theta_x, theta_y, theta_z}: Euler angles in
   * degrees per unordered phase pair (utility_functions.h:700-774). */
  double rot_angles[GP_MAX_PHASES][GP_MAX_PHASES][3];
  int rot_set[GP_MAX_PHASES][GP_MAX_PHASES];
  int bc_type[3][6];                      /* [field][face]; -1 = no BOUNDARY line */
  double bc_value[3][6];
  int bc_value_set[3];                    /* BOUNDARY_VALUE line seen per field */
  int bc_proxy_type[3][6];                /* type in force when BOUNDARY_VALUE fixed the copy sources */
  int have_gamma, have_tau_ab, have_dab, have_gamma_abc;
  char phases[GP_MAX_PHASES][GP_NAME_LEN];
  char components[GP_MAX_COMP + 1][GP_NAME_LEN];
} gp_params;

/* Diagnostics after gp_step / gp_smooth.  phi/mu extremes follow the
 * reference's progress record (calculate_divergence_concentration.h:273-296):
 * running extremes since gp_init (starting from phi 1/0 and mu 1/1 as in
 * serialinfo_xy.h:59-66), never reset.  rel_change_* are sum(delta^2) of the
 * last step (printed as sqrt by microsim_gp.c:139-148).  All sums run over the
 * interior cells only (the reference also adds ghost cells whose values depend
 * on stale buffer contents).  phi_sum/comp_sum are FP64 sums of phi_a and of
 * c_k = sum_a c_a,k(mu) h_a(phi) over the interior after the last step. */
typedef struct gp_stats {
  double phi_max[GP_MAX_PHASES], phi_min[GP_MAX_PHASES];
  double mu_max[GP_MAX_COMP], mu_min[GP_MAX_COMP];
  double rel_change_phi[GP_MAX_PHASES], rel_change_mu[GP_MAX_COMP];
  double phi_sum[GP_MAX_PHASES];
  double comp_sum[GP_MAX_COMP];
  long long nonfinite;                    /* interior cells with a non-finite field */
  long long steps_done;                   /* time steps taken since gp_init */
  long long shift_offset;                 /* moving frame: cells the fields have moved down since gp_init
                                             (shift_OFFSET, microsim_gp.c:122) */
} gp_stats;

typedef struct gp_ctx gp_ctx;

/* ---- host surface (no GPU needed) ------------------------------------- */

/* Parse Input.in.  Replaces reading_input_parameters (reading_input_parameters.h:1-307)
 * and read_boundary_conditions (read_boundary_conditions.h:4-41); the echo files
 * <in>.out/<in>.bd are not written.  Returns GP_EIO if the file cannot be read,
 * GP_EINVAL if a size/count exceeds GP_MAX_*. */
int gp_params_load(gp_params *p, const char *input_path);

/* Fill the interior from Filling.in.  Replaces fill_domain (fill_domain.h:4-151)
 * with fill_phase_cube/cylinder/sphere/ellipse and fill_composition_cube
 * (filling.h:6-270).  phi: [N][MESH_X][MESH_Y], mu: [K][MESH_X][MESH_Y]. */
int gp_fill(const gp_params *p, const char *filling_path, double *phi, double *mu);

/* Legacy-VTK writer/reader of the interior.  Replaces writetofile_serial2D[_binary]
 * and readfromfile_serial2D[_binary] (file_writer.h:23-70,71-416).
 * ascii=1: "%le" text; ascii=0: big-endian float64.  A non-isothermal run
 * (ISOTHERMAL = 0) also writes the Temperature field, and its optional
 * composition fields are taken at each cell's temperature: gp_vtk_write uses
 * the field laid down at start-up (microsim_gp.c:77-82), as a file written
 * before the first step holds; gp_vtk_write_temperature takes the field
 * [MESH_X][MESH_Y] (gp_temperature gives a context's; NULL = the start-up
 * field; ignored when isothermal).  The reader reads phi and mu and skips the
 * fields after them (the reference lays the temperature field down again
 * after reading, microsim_gp.c:75-82). */
int gp_vtk_write(const gp_params *p, const char *path, const double *phi, const double *mu, int ascii);
int gp_vtk_write_temperature(const gp_params *p, const char *path, const double *phi, const double *mu,
                             const double *temperature, int ascii);
int gp_vtk_read(const gp_params *p, const char *path, double *phi, double *mu, int ascii);

/* Write the context's current state to `path` as gp_vtk_write does, in the
 * background: the state is copied on the device (ordered after the steps
 * already queued), and a host thread brings the copy down through pinned
 * memory and writes the file while the caller keeps stepping.  Replaces the
 * periodic writetofile_serial2D[_binary] of the time loop
 * (microsim_gp.c:129-134) without stopping the GPU.  One write is in flight
 * per context: a call first waits for the previous one and returns its error,
 * if any.  The file is complete after gp_vtk_wait or gp_destroy. */
int gp_vtk_write_async(gp_ctx *ctx, const char *path, int ascii);
/* Wait for the context's background write; its result. */
int gp_vtk_wait(gp_ctx *ctx);

/* ---- device path ------------------------------------------------------- */

/* Create a context on the current CUDA device, upload the interior state and
 * the derived constants (init_propertymatrices, functionF_01.h:169-230, and
 * initialize_variables, initialize_variables.h:4-28, evaluated on the host).
 * Replaces serialinfo_xy (serialinfo_xy.h:1-66) + initialize_functions_solverloop
 * (initialize_functions_solverloop.h:4-58) + apply_boundary_conditions(0) at
 * microsim_gp.c:84.  GP_EINVAL for combinations the kernels do not cover
 * (N>4, K>2, noise, free/Dirichlet BCs, 3-D).  A non-isothermal run
 * (ISOTHERMAL = 0) carries the temperature gradient along y of Tempgrady and,
 * with Shift = 1, the moving frame. */
int gp_init(gp_ctx **ctx, const gp_params *p, const double *phi, const double *mu,
            gp_precision prec);

/* nsteps preconditioning sweeps; replaces the loop
 * "for(t=1; t<nsmooth; t++) { smooth(); apply_boundary_conditions(0); }"
 * (microsim_gp.c:97-100, solverloop.h:72-90), i.e. call with nsmooth-1. */
int gp_smooth(gp_ctx *ctx, long nsteps);

/* nsteps explicit time steps; each replaces solverloop_phasefield +
 * apply_boundary_conditions + solverloop_concentration + apply_boundary_conditions
 * (microsim_gp.c:103-106, solverloop.h:21-71, boundary_serial.h:176-203).
 * stats may be NULL.  Besides GP_EINVAL/GP_ECUDA it returns
 *   GP_ETIMEOUT    when a bounded device-side wait of the step kernels gave up
 *                  (a tile's staged fields did not arrive); the state is then
 *                  not valid and the error flag is cleared for the next call;
 *   GP_ENONFINITE  when stats were asked for and the state after the steps
 *                  holds interior cells with a non-finite phi or mu: the steps
 *                  are done and *stats is filled (stats->nonfinite counts the
 *                  cells), as the reference, which keeps stepping, would have
 *                  them.  Without stats the count is not made. */
int gp_step(gp_ctx *ctx, long nsteps, gp_stats *stats);

/* Copy the interior state out / in (host buffers, layouts as above). */
int gp_get(gp_ctx *ctx, double *phi, double *mu);
int gp_set(gp_ctx *ctx, const double *phi, const double *mu);

/* Same as gp_get/gp_set with device pointers (FP64, same layouts) on the
 * context's device; used by the Python integrator to exchange CUDA tensors. */
int gp_get_dev(gp_ctx *ctx, double *phi_dev, double *mu_dev);
int gp_set_dev(gp_ctx *ctx, const double *phi_dev, const double *mu_dev);

int gp_get_stats(gp_ctx *ctx, gp_stats *stats);

/* The temperature of every interior cell [MESH_X][MESH_Y] as the reference
 * holds it after the steps taken so far (gridinfo[].temperature: laid down by
 * apply_temperature_gradientY after each step, Temperature_gradient.h:4-29 and
 * microsim_gp.c:108-113, then moved with the frame by apply_shiftY,
 * shift.h:4-45).  An isothermal run has T everywhere. */
int gp_temperature(gp_ctx *ctx, double *temperature);

/* gp_step with CUDA events recorded on the context's stream: total_ms is the
 * device time of the nsteps steps.  A step is two kernels: the bulk-tile
 * kernel (tiles with one pure phase everywhere within reach of their stencil,
 * which only move mu) and the interface-tile kernel (everything else);
 * ms_bulk / ms_iface, when not NULL, receive their summed device times, and
 * the steps then run one by one instead of as CUDA graphs.  Each may be NULL.
 * Measurement entry point; results are those of gp_step. */
int gp_step_timed(gp_ctx *ctx, long nsteps, gp_stats *stats, double *total_ms,
                  double *ms_bulk, double *ms_iface);

/* Per-kernel device times of nsteps steps launched one by one (no graphs) in
 * the launch shape the context uses, CUDA events around each launch.  Fused
 * shape: kf_classify then kf_step (interface tiles, then bulk tiles, in one
 * launch); two-launch shape: kf_classify + kf_bulk, then kf_general.
 * Measurement entry point with no counterpart in the reference; the state
 * advances by nsteps as with gp_step. */
typedef struct gp_kernel_times {
  double classify_ms;          /* fused shape: kf_classify, summed over the steps */
  double step_ms;              /* fused shape: kf_step, summed */
  double bulk_ms;              /* two-launch shape: kf_classify + kf_bulk, summed */
  double iface_ms;             /* two-launch shape: kf_general, summed */
  int launches_per_step;       /* kernels of one step in this shape (2 or 3) */
  int fused;                   /* 1: fused shape */
} gp_kernel_times;
int gp_step_kernel_times(gp_ctx *ctx, long nsteps, gp_kernel_times *t);

/* ---- batches of simulations ------------------------------------------- */

/* Many independent simulations stepped together: grids of different sizes,
 * different physical parameters, one launch per pass over all of them
 * (persistent CTAs pulling (simulation, tile) items from a work queue), steps
 * replayed as CUDA graphs of 100 steps.  All simulations share NUMPHASES,
 * NUMCOMPONENTS and Function_anisotropy.  The reference runs one simulation
 * per process (microsim_gp.c); there is no batch call to replace.
 * prec = GP_FP64: each simulation is bit-identical to gp_step on its own.
 * prec = GP_FP32: fields stored and stepped in float; the dc/dmu inversion and
 * every reduction in FP64.
 * params: nsims structs; phi[s], mu[s]: host interior planes of simulation s. */
typedef struct gp_batch gp_batch;
int gp_batch_create(gp_batch **b, int nsims, const gp_params *params, const double *const *phi,
                    const double *const *mu, gp_precision prec);
int gp_batch_smooth(gp_batch *b, long nsteps);
/* stats: NULL or nsims records, in simulation order; return codes as gp_step
 * (GP_ENONFINITE names the first simulation with non-finite cells) */
int gp_batch_step(gp_batch *b, long nsteps, gp_stats *stats);
int gp_batch_step_timed(gp_batch *b, long nsteps, gp_stats *stats, double *total_ms);
int gp_batch_get(gp_batch *b, int sim, double *phi, double *mu);
int gp_batch_set(gp_batch *b, int sim, const double *phi, const double *mu);
int gp_batch_size(const gp_batch *b);
const char *gp_batch_last_error(const gp_batch *b);
void gp_batch_destroy(gp_batch *b);

/* One FP64 time step that allocates nothing.  This entry point has no
 * counterpart in the reference; it exists for callers that cannot call
 * cudaMalloc -- applications that own all device memory through their own pool
 * or arena, run under a fixed memory budget, or sit on a path where a failed
 * allocation cannot be handled.  They pass their own device buffers:
 * phi_in/mu_in (read) and phi_out/mu_out (written), contiguous planes
 * [N][MESH_X][MESH_Y] and [K][MESH_X][MESH_Y] on the current device; neither
 * output may share a byte with an input or with the other output (GP_EINVAL
 * otherwise); stream is a cudaStream_t (NULL = default stream).
 * The step's scratch (delta-phi over the interior plus a one-cell ring) lives
 * in a fixed 32 MiB array inside the library that every GPU which loads the
 * library keeps until exit; grids needing more (about 1.3 million cells with
 * 3 phases) are rejected with GP_EINVAL and a message.  The first call on a
 * device looks up that array's device address (cudaGetSymbolAddress).  No
 * call may be recorded by stream capture: each one copies the step's constant
 * block from host (pageable) memory into the library's __constant__ block,
 * which a captured graph could not replay.  All calls share the array, so
 * calls that overlap on the GPU (other streams, other host threads) race; the
 * same holds for the constant block its kernels read.  The call is
 * asynchronous on `stream`; no progress record is produced.  Results are those
 * of gp_step. */
int gp_step_noalloc(const gp_params *p, const double *phi_in, const double *mu_in,
                    double *phi_out, double *mu_out, void *stream);

/* ---- adjoint --------------------------------------------------------- */

/* Gradients of a loss of the final state with respect to the start state and
 * four parameters, through nsteps FP64 time steps of a context: the discrete
 * adjoint of the step, i.e. exact derivatives of the computed trajectory.  The
 * reference has no adjoint.  Contexts with NUMPHASES = 2, NUMCOMPONENTS = 2
 * (one independent component, BINARY) and FP64 only; others get
 * GP_EUNSUPPORTED.  The step is not differentiated where it branches (active
 * phases, simplex projection, bulk test): derivatives are those of the branch
 * the trajectory took.
 * The forward pass runs from the context's current state and leaves the
 * context at the final state (as gp_step would).  Steps are reversed in the
 * order of binomial checkpointing: with s states kept on the device besides
 * the start state, the schedule recomputes the fewest forward steps any
 * schedule with s snapshots can (none when s = nsteps-1, the default whenever
 * that many states fit in half the free device memory). */
typedef struct gp_adj_req {
  long nsteps;                 /* time steps, >= 1 */
  const double *phi_bar;       /* NULL, or [N][X][Y]: dL/dphi of the final state */
  const double *mu_bar;        /* NULL (zero), or [K][X][Y]: dL/dmu of the final state */
  const double *target_phi;    /* used when phi_bar is NULL: L = 1/2 sum over phases and
                                  cells of (phi_final - target)^2 */
  long checkpoint_every;       /* > 0 (and snapshots 0): keep nsteps/checkpoint_every states */
  long snapshots;              /* states kept besides the start state (binomial checkpointing);
                                  0 and checkpoint_every 0: as many as half the free device memory
                                  holds, at most nsteps-1 (every state: nothing is recomputed, and
                                  when it fits each step's delta-phi is kept as well) */
  int device;                  /* 1: phi_bar, mu_bar, target_phi and the phi0_bar / mu0_bar of the
                                  result are device pointers on the context's device */
} gp_adj_req;

typedef struct gp_adj_out {
  double loss;                 /* L with target_phi, else 0 */
  double d_tau;                /* dL/dTau of phases (0,1); the mobility is 1/Tau */
  double d_dab;                /* dL/d dab of phases (0,1): anisotropy strength */
  double d_epsilon;            /* dL/d epsilon: interface width */
  double d_gamma;              /* dL/d GAMMA of phases (0,1): interface energy */
  double *phi0_bar;            /* NULL, or [N][X][Y]: receives dL/dphi of the start state */
  double *mu0_bar;             /* NULL, or [K][X][Y]: receives dL/dmu of the start state */
  double ms_forward;           /* device time of the forward pass */
  double ms_reverse;           /* device time of the recomputation and reverse sweep (with every
                                  state kept, both sweeps run as CUDA graphs of 100 steps; the
                                  first graph of each is captured before these times start) */
  long snapshots;              /* states kept besides the start state */
  long recomputed;             /* forward steps taken again in the reverse sweep */
} gp_adj_out;

int gp_adjoint(gp_ctx *ctx, const gp_adj_req *req, gp_adj_out *out);

/* Verification of the adjoint's cell functions: nsteps steps evaluated with
 * them (one thread per cell, no tiles) against gp_step's kernels from the same
 * start state; *max_abs_diff receives the largest difference of any field
 * value and *n_diff the number of values whose bits differ.  The context
 * advances by nsteps. */
int gp_adjoint_replay(gp_ctx *ctx, long nsteps, double *max_abs_diff, long long *n_diff);

/* ---- slabs: one grid split along x over several contexts ----------------
 * Each context (one per GPU rank) holds its own rows of the global grid plus
 * halo rows above and below (3 rows, the reference's ghost width) that
 * another rank owns, or, at a periodic edge, the rows the reference's ghost
 * copy maps there.  A step of the local grid leaves its own rows exactly as a
 * step of the whole grid does (the step reads no further than two rows), so
 * one halo exchange per step keeps every rank exact.  Replaces the MPI slab
 * exchange of the reference's MPI variant (mpiinfo_xyz.h:739-787). */

/* Rows [x0, x1) of the context's grid are counted by the progress statistics
 * (gp_stats): the context's own rows.  Default: every row.  Not with the
 * moving frame (GP_EUNSUPPORTED). */
int gp_set_stat_rows(gp_ctx *ctx, long x0, long x1);

/* Gather rows of the current state into a contiguous device buffer (pack) or
 * scatter them from one (unpack): item i is row rows[i] of field fields[i]
 * (0..N-1: phi_a, N..N+K-1: mu_k), MESH_Y values of the context's precision,
 * in item order; 1 <= n <= 64.  Ordered on the context's stream (gp_stream),
 * without a host wait; unpack also renews the tiles' phase flags. */
int gp_rows_pack(gp_ctx *ctx, int n, const int *fields, const int *rows, void *dev_buf);
int gp_rows_unpack(gp_ctx *ctx, int n, const int *fields, const int *rows, const void *dev_buf);

/* Stream the context's work is ordered on (a cudaStream_t as an opaque pointer). */
void *gp_stream(gp_ctx *ctx);

void gp_destroy(gp_ctx *ctx);
const char *gp_last_error(const gp_ctx *ctx);
const char *gp_version(void);

#ifdef __cplusplus
}
#endif
#endif /* GP_H_ */
