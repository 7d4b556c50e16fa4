/*
 * gp_adjoint_launch.h -- launcher table of the adjoint kernels (gp_adjoint.cu)
 * for the host driver in gp_device.cu.
 */
#pragma once
#include <cuda_runtime.h>

#include "gp_tiles.cuh"

namespace gpd {

enum { ADJ_TAU = 0, ADJ_DAB = 1, ADJ_EPS = 2, ADJ_GAMMA = 3, ADJ_NPARAM = 4 };

/* values of the differentiable parameters */
struct AdjParams {
  double v[ADJ_NPARAM];   /* Tau_01, dab_01, epsilon, GAMMA_01 */
};

struct AdjLaunch {
  /* delta-phi of the interior plus ring of a state (dplane layout) */
  cudaError_t (*dphi)(cudaStream_t s, const void *consts, AdjParams p, Grid g, const double *state, double *dphi);
  /* the same values from a sweep that lists the active cells and a pass over
   * the list (cells/count: scratch list as below) */
  cudaError_t (*dphi_sparse)(cudaStream_t s, const void *consts, AdjParams p, Grid g, const double *state,
                             double *dphi, int2 *cells, int *count);
  /* the step from a state and its delta-phi, by the adjoint's cell functions */
  cudaError_t (*update)(cudaStream_t s, const void *consts, AdjParams p, Grid g, const double *state,
                        const double *dphi, double *next);
  /* reverse of the concentration pass: ybar -> xbar, dphibar, pbar
   * (accumulated); cells/count: scratch list of (mx+2)*(my+2) cells, the
   * count zero on entry (each pass takes a counter of its own) */
  cudaError_t (*rev_update)(cudaStream_t s, const void *consts, AdjParams p, Grid g, const double *state,
                            const double *dphi, const double *ybar, double *xbar, double *dphibar, double *pbar,
                            int2 *cells, int *count);
  /* reverse of the phase-field pass: dphibar -> xbar, pbar (accumulated);
   * count zero on entry */
  cudaError_t (*rev_dphi)(cudaStream_t s, const void *consts, AdjParams p, Grid g, const double *state,
                          const double *dphibar, double *xbar, double *pbar, int2 *cells, int *count);
};
}  // namespace gpd

bool gp_adjoint_launch(int N, int K, bool aniso, gpd::AdjLaunch *out);
