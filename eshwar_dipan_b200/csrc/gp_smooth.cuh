/*
 * gp_smooth.cuh -- the preconditioning sweeps run before the time loop
 * (smooth(), solverloop.h:72-90; microsim_gp.c:97-100): no dpsi, no
 * anti-trapping, isotropic gradient terms, and the unweighted simplex
 * projection.  They run NSMOOTH-1 times per simulation, so they are plain
 * one-thread-per-cell kernels reading through the boundary remap; constants
 * come from a Consts<R> block in global memory.
 */
#pragma once
#include "gp_tiles.cuh"

namespace gpd {

/* Offsets of the cells (x-1..x+1, y-1..y+1) of interior cell (x, y) in a
 * field's planes, ghosts through the boundary remap of that field (0 phi,
 * 1 mu): o(u, v) = row[u] + col[v].  Computed once per cell; 32 bits hold
 * any offset inside a plane (a plane of 2^32 FP64 cells is 32 GB). */
struct Nbr3 {
  unsigned row[3], col[3];
  __device__ __forceinline__ unsigned o(int u, int v) const { return row[u] + col[v]; }
};
template <typename R>
__device__ __forceinline__ Nbr3 nbr3(const Consts<R> &D, const Grid &g, int field, int x, int y) {
  Nbr3 n;
  const int bx0 = D.bc_x[field][0], bx1 = D.bc_x[field][1], by0 = D.bc_y[field][0], by1 = D.bc_y[field][1];
#pragma unroll
  for (int u = 0; u < 3; u++) {
    n.row[u] = (unsigned)remap(x - 1 + u, g.mx, bx0, bx1) * (unsigned)g.pitch;
    n.col[u] = (unsigned)remap(y - 1 + u, g.my, by0, by1);
  }
  return n;
}

/* calculate_divergence_phasefield_smooth_2D (calculate_divergence_phasefield.h:63-158)
 * at interior cell (x, y): its delta-phi into d. */
template <typename R, int N, bool ANISO>
__device__ __forceinline__ void sdphi_cell(const Consts<R> &D, const R *__restrict__ phi, const Grid &g,
                                           const Nbr3 &np, R (&d)[N]) {
  R S[N][3][3];
#pragma unroll
  for (int a = 0; a < N; a++)
#pragma unroll
    for (int u = 0; u < 3; u++)
#pragma unroll
      for (int v = 0; v < 3; v++) S[a][u][v] = __ldg(phi + a * g.plane + np.o(u, v));
  R ph[N], dv[N], gcx[N], gcy[N], lam[N];
  bool act[N];
#pragma unroll
  for (int a = 0; a < N; a++) {
    ph[a] = S[a][1][1];
    R gxf = divx(S[a][2][1] - S[a][1][1], D), gxb = divx(S[a][1][1] - S[a][0][1], D);
    R gyr = divy(S[a][1][2] - S[a][1][1], D), gyl = divy(S[a][1][1] - S[a][1][0], D);
    dv[a] = divx(gxf - gxb, D);
    dv[a] += divy(gyr - gyl, D);
    act[a] = fabs(dv[a]) > R(0.0);
    gcx[a] = R(0.5) * (gxf + gxb);
    gcy[a] = div2y(S[a][1][2] - S[a][1][0], D);
  }
  R sl = R(0.0);
  long nact = 0;
#pragma unroll
  for (int a = 0; a < N; a++) {
    if (!act[a]) continue;
    R s = R(0.0), t = R(0.0);
#pragma unroll
    for (int b = 0; b < N; b++) {
      if (b == a) continue;
      R sp = R(0.0);
      sp += (ph[a] * gcx[b] - ph[b] * gcx[a]) * gcx[b];
      sp += (ph[a] * gcy[b] - ph[b] * gcy[a]) * gcy[b];
      sp *= D.gamma[a][b];
      s += sp;
      R pa = S[a][1][1], pb = S[b][1][1];
      R sxa = R(0.5) * (S[a][2][1] + pa), sxb = R(0.5) * (S[b][2][1] + pb);
      R gxa = divx(S[a][2][1] - pa, D), gxb = divx(S[b][2][1] - pb, D);
      R bxa = R(0.5) * (pa + S[a][0][1]), bxb = R(0.5) * (pb + S[b][0][1]);
      R hxa = divx(pa - S[a][0][1], D), hxb = divx(pb - S[b][0][1], D);
      R sya = R(0.5) * (S[a][1][2] + pa), syb = R(0.5) * (S[b][1][2] + pb);
      R gya = divy(S[a][1][2] - pa, D), gyb = divy(S[b][1][2] - pb, D);
      R lya = R(0.5) * (pa + S[a][1][0]), lyb = R(0.5) * (pb + S[b][1][0]);
      R hya = divy(pa - S[a][1][0], D), hyb = divy(pb - S[b][1][0], D);
      R dvg = divx((sxa * gxb - sxb * gxa) * (-sxb) - ((bxa * hxb - bxb * hxa) * (-bxb)), D);
      dvg += divy((sya * gyb - syb * gya) * (-syb) - ((lya * hyb - lyb * hya) * (-lyb)), D);
      dvg *= D.gamma[a][b];
      t += dvg;
    }
    /* A_01 *_smooth and A_00 give the same values here (sums started at 0.0
     * are never -0, so 2*(s+0.0) == 2*s) */
    lam[a] = D.eps * (-(R(2.0) * s) + (R(2.0) * t)) - D.inv_eps * dwdphi<R, N>(D, ph, act, a, ANISO);
    sl += lam[a];
    nact++;
  }
  if (nact) sl /= (R)nact;
  const R tau = tau_of<R, N>(D, ph);
#pragma unroll
  for (int a = 0; a < N; a++) d[a] = act[a] ? D.dt * (lam[a] - sl) / (tau * D.eps) : R(0.0);
  project_nw<R, N>(ph, act, d);
}

/* calculate_divergence_concentration_smooth_2D (calculate_divergence_concentration.h:154-253)
 * at interior cell (x, y), given the cell's delta-phi of the sweep (the pass
 * reads no other cell's) */
template <typename R, int N, int K>
__device__ __forceinline__ void supd_cell(const Consts<R> &D, const R *__restrict__ phi, const R *__restrict__ mu,
                                          const R (&dph)[N], R *__restrict__ phin, R *__restrict__ mun,
                                          const Grid &g, const double *__restrict__ tcc, const Nbr3 &np,
                                          const Nbr3 &nq, int x, int y) {
  /* cells: 0 centre, 1 front (x+1), 2 back (x-1), 3 right (y+1), 4 left (y-1) */
  const int cu[5] = {1, 2, 0, 1, 1}, cv[5] = {1, 1, 1, 2, 0};
  R P[5][N], M[5][K], Dv[5][K][K];
#pragma unroll
  for (int q = 0; q < 5; q++) {
#pragma unroll
    for (int a = 0; a < N; a++) P[q][a] = __ldg(phi + a * g.plane + np.o(cu[q], cv[q]));
#pragma unroll
    for (int k = 0; k < K; k++) M[q][k] = __ldg(mu + k * g.plane + nq.o(cu[q], cv[q]));
#pragma unroll
    for (int k = 0; k < K; k++)
#pragma unroll
      for (int l = 0; l < K; l++) Dv[q][k][l] = Dcell<R, N, K>(D, P[q], k, l);
  }
  R divflux[K];
#pragma unroll
  for (int k = 0; k < K; k++) {
    divflux[k] = R(0.0);
#pragma unroll
    for (int l = 0; l < K; l++) {
      R fx = ((Dv[1][k][l] + Dv[0][k][l]) * R(0.5)) * divx(M[1][l] - M[0][l], D);
      R bx = ((Dv[0][k][l] + Dv[2][k][l]) * R(0.5)) * divx(M[0][l] - M[2][l], D);
      R fy = ((Dv[3][k][l] + Dv[0][k][l]) * R(0.5)) * divy(M[3][l] - M[0][l], D);
      R by = ((Dv[0][k][l] + Dv[4][k][l]) * R(0.5)) * divy(M[0][l] - M[4][l], D);
      divflux[k] += divx(fx - bx, D);
      divflux[k] += divy(fy - by, D);
    }
  }
  const R *ph = P[0], *m = M[0];
  R nm[K];
  int bulk = -1;
#pragma unroll
  for (int a = 0; a < N; a++)
    if (bulk < 0 && ph[a] == R(1.0)) bulk = a;
  if (bulk >= 0) {
    R cn[K], E[N][K];
    /* the cell's temperature in a non-isothermal run
     * (calculate_divergence_concentration.h:167-170) */
    if (D.tgrad) e_at<R, N, K>(D, tcc[y + 3], E);
#pragma unroll
    for (int k = 0; k < K; k++)
      cn[k] = (D.tgrad ? c_muE<R, K>(D, E[bulk], m, bulk, k) : c_mu<R, K>(D, m, bulk, k)) + D.dt * (divflux[k]);
#pragma unroll
    for (int k = 0; k < K; k++) nm[k] = D.tgrad ? MuE<R, K>(D, E[bulk], cn, bulk, k) : Mu<R, K>(D, cn, bulk, k);
  } else {
    double dc[K], dcdmu[K][K], iv[K][K];
#pragma unroll
    for (int k = 0; k < K; k++) {
      dc[k] = (double)(D.dt * (divflux[k]));
#pragma unroll
      for (int l = 0; l < K; l++) {
        dcdmu[k][l] = 0.0;
#pragma unroll
        for (int a = 0; a < N; a++) dcdmu[k][l] += D.cmu64[a][k][l] * (double)h<R, N>(ph, a);
      }
    }
    matinv_div<double, K>(dcdmu, iv);
#pragma unroll
    for (int k = 0; k < K; k++) {
      double s = 0;
#pragma unroll
      for (int l = 0; l < K; l++) s = s + iv[k][l] * dc[l];
      nm[k] = (R)(s + (double)m[k]);
    }
  }
  const long long o = (long long)x * g.pitch + y;
#pragma unroll
  for (int a = 0; a < N; a++) phin[a * g.plane + o] = ph[a] + dph[a];
#pragma unroll
  for (int k = 0; k < K; k++) mun[k * g.plane + o] = nm[k];
}

/* One smoothing sweep (smooth(), solverloop.h:72-90), one thread per interior
 * cell: the phase-field pass's delta-phi of the cell, then the concentration
 * pass's update, which reads the delta-phi of no other cell (the two passes
 * in one launch, without a delta-phi buffer between them). */
template <typename R, int N, int K, bool ANISO>
__global__ void __launch_bounds__(128, N <= 3 ? 4 : 3) k_smooth(const Consts<R> *__restrict__ Dp, const R *__restrict__ phi, const R *__restrict__ mu,
                         R *__restrict__ phin, R *__restrict__ mun, Grid g, const double *__restrict__ tcc) {
  const Consts<R> &D = *Dp;
  const int y = blockIdx.x * blockDim.x + threadIdx.x, x = blockIdx.y;
  if (y >= g.my) return;
  const Nbr3 np = nbr3(D, g, 0, x, y), nq = nbr3(D, g, 1, x, y);
  R d[N];
  sdphi_cell<R, N, ANISO>(D, phi, g, np, d);
  supd_cell<R, N, K>(D, phi, mu, d, phin, mun, g, tcc, np, nq, x, y);
}

}  // namespace gpd
