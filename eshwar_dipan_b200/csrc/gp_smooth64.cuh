/*
 * gp_smooth64.cuh -- the preconditioning sweeps run before the time loop
 * (smooth(), solverloop.h:72-90; microsim_gp.c:97-100): no dpsi, no
 * anti-trapping, isotropic gradient terms, and the unweighted simplex
 * projection.  They run NSMOOTH-1 times per simulation, so they are plain
 * one-thread-per-cell kernels reading through the boundary remap.
 */
#pragma once
#include "gp_step64.cuh"

namespace gpd {

/* phi of interior cell (x,y) (coordinates may lie in the ghost layers) */
__device__ __forceinline__ double ld_phi(const double *__restrict__ f, const Grid &g, int a, int x, int y) {
  int sx = remap(x, g.mx, cD.bc_x[0][0], cD.bc_x[0][1]), sy = remap(y, g.my, cD.bc_y[0][0], cD.bc_y[0][1]);
  return __ldg(f + a * g.plane + (long long)sx * g.pitch + sy);
}
__device__ __forceinline__ double ld_mu(const double *__restrict__ f, const Grid &g, int k, int x, int y) {
  int sx = remap(x, g.mx, cD.bc_x[1][0], cD.bc_x[1][1]), sy = remap(y, g.my, cD.bc_y[1][0], cD.bc_y[1][1]);
  return __ldg(f + k * g.plane + (long long)sx * g.pitch + sy);
}

/* calculate_divergence_phasefield_smooth_2D (calculate_divergence_phasefield.h:63-158)
 * for the interior; result into the delta-phi buffer. */
template <int N, bool ANISO>
__global__ void k_sdphi(const double *__restrict__ phi, double *__restrict__ dphi, Grid g) {
  const int y = blockIdx.x * blockDim.x + threadIdx.x, x = blockIdx.y;
  if (y >= g.my) return;
  double S[N][3][3];
#pragma unroll
  for (int a = 0; a < N; a++)
#pragma unroll
    for (int u = 0; u < 3; u++)
#pragma unroll
      for (int v = 0; v < 3; v++) S[a][u][v] = ld_phi(phi, g, a, x - 1 + u, y - 1 + v);
  double ph[N], dv[N], gcx[N], gcy[N], d[N], lam[N];
  bool act[N];
#pragma unroll
  for (int a = 0; a < N; a++) {
    ph[a] = S[a][1][1];
    double gxf = divx(S[a][2][1] - S[a][1][1], g), gxb = divx(S[a][1][1] - S[a][0][1], g);
    double gyr = divy(S[a][1][2] - S[a][1][1], g), gyl = divy(S[a][1][1] - S[a][1][0], g);
    dv[a] = divx(gxf - gxb, g);
    dv[a] += divy(gyr - gyl, g);
    act[a] = fabs(dv[a]) > 0.0;
    gcx[a] = 0.5 * (gxf + gxb);
    gcy[a] = div2y(S[a][1][2] - S[a][1][0], g);
  }
  double sl = 0.0;
  long nact = 0;
#pragma unroll
  for (int a = 0; a < N; a++) {
    if (!act[a]) continue;
    double s = 0.0, t = 0.0;
#pragma unroll
    for (int b = 0; b < N; b++) {
      if (b == a) continue;
      double sp = 0.0;
      sp += (ph[a] * gcx[b] - ph[b] * gcx[a]) * gcx[b];
      sp += (ph[a] * gcy[b] - ph[b] * gcy[a]) * gcy[b];
      sp *= cD.gamma[a][b];
      s += sp;
      double pa = S[a][1][1], pb = S[b][1][1];
      double sxa = 0.5 * (S[a][2][1] + pa), sxb = 0.5 * (S[b][2][1] + pb);
      double gxa = divx(S[a][2][1] - pa, g), gxb = divx(S[b][2][1] - pb, g);
      double bxa = 0.5 * (pa + S[a][0][1]), bxb = 0.5 * (pb + S[b][0][1]);
      double hxa = divx(pa - S[a][0][1], g), hxb = divx(pb - S[b][0][1], g);
      double sya = 0.5 * (S[a][1][2] + pa), syb = 0.5 * (S[b][1][2] + pb);
      double gya = divy(S[a][1][2] - pa, g), gyb = divy(S[b][1][2] - pb, g);
      double lya = 0.5 * (pa + S[a][1][0]), lyb = 0.5 * (pb + S[b][1][0]);
      double hya = divy(pa - S[a][1][0], g), hyb = divy(pb - S[b][1][0], g);
      double dvg = divx((sxa * gxb - sxb * gxa) * (-sxb) - ((bxa * hxb - bxb * hxa) * (-bxb)), g);
      dvg += divy((sya * gyb - syb * gya) * (-syb) - ((lya * hyb - lyb * hya) * (-lyb)), g);
      dvg *= cD.gamma[a][b];
      t += dvg;
    }
    /* A_01 *_smooth and A_00 give the same values here (sums started at 0.0
     * are never -0, so 2*(s+0.0) == 2*s) */
    lam[a] = cD.eps * (-(2.0 * s) + (2.0 * t)) - cD.inv_eps * dwdphi<N>(ph, act, a, ANISO);
    sl += lam[a];
    nact++;
  }
  if (nact) sl /= (double)nact;
  const double tau = tau_of<N>(ph);
#pragma unroll
  for (int a = 0; a < N; a++) d[a] = act[a] ? cD.dt * (lam[a] - sl) / (tau * cD.eps) : 0.0;
  project_nw<N>(ph, act, d);
  const long long o = (long long)(x + 1) * g.dpitch + (y + 1);
#pragma unroll
  for (int a = 0; a < N; a++) dphi[a * g.dplane + o] = d[a];
}

/* calculate_divergence_concentration_smooth_2D (calculate_divergence_concentration.h:154-253) */
template <int N, int K>
__global__ void k_supdate(const double *__restrict__ phi, const double *__restrict__ mu,
                          const double *__restrict__ dphi, double *__restrict__ phin,
                          double *__restrict__ mun, Grid g) {
  const int y = blockIdx.x * blockDim.x + threadIdx.x, x = blockIdx.y;
  if (y >= g.my) return;
  /* cells: 0 centre, 1 front (x+1), 2 back (x-1), 3 right (y+1), 4 left (y-1) */
  const int cx[5] = {x, x + 1, x - 1, x, x}, cy[5] = {y, y, y, y + 1, y - 1};
  double P[5][N], M[5][K], Dv[5][K][K];
#pragma unroll
  for (int q = 0; q < 5; q++) {
#pragma unroll
    for (int a = 0; a < N; a++) P[q][a] = ld_phi(phi, g, a, cx[q], cy[q]);
#pragma unroll
    for (int k = 0; k < K; k++) M[q][k] = ld_mu(mu, g, k, cx[q], cy[q]);
#pragma unroll
    for (int k = 0; k < K; k++)
#pragma unroll
      for (int l = 0; l < K; l++) Dv[q][k][l] = Dcell<N, K>(P[q], k, l);
  }
  double divflux[K];
#pragma unroll
  for (int k = 0; k < K; k++) {
    divflux[k] = 0.0;
#pragma unroll
    for (int l = 0; l < K; l++) {
      double fx = ((Dv[1][k][l] + Dv[0][k][l]) * 0.5) * divx(M[1][l] - M[0][l], g);
      double bx = ((Dv[0][k][l] + Dv[2][k][l]) * 0.5) * divx(M[0][l] - M[2][l], g);
      double fy = ((Dv[3][k][l] + Dv[0][k][l]) * 0.5) * divy(M[3][l] - M[0][l], g);
      double by = ((Dv[0][k][l] + Dv[4][k][l]) * 0.5) * divy(M[0][l] - M[4][l], g);
      divflux[k] += divx(fx - bx, g);
      divflux[k] += divy(fy - by, g);
    }
  }
  const double *ph = P[0], *m = M[0];
  double nm[K];
  int bulk = -1;
#pragma unroll
  for (int a = 0; a < N; a++)
    if (bulk < 0 && ph[a] == 1.0) bulk = a;
  if (bulk >= 0) {
    double cn[K];
#pragma unroll
    for (int k = 0; k < K; k++) cn[k] = c_mu<K>(m, bulk, k) + cD.dt * (divflux[k]);
#pragma unroll
    for (int k = 0; k < K; k++) nm[k] = Mu<K>(cn, bulk, k);
  } else {
    double dc[K], dcdmu[K][K], iv[K][K];
#pragma unroll
    for (int k = 0; k < K; k++) {
      dc[k] = cD.dt * (divflux[k]);
#pragma unroll
      for (int l = 0; l < K; l++) {
        dcdmu[k][l] = 0.0;
#pragma unroll
        for (int a = 0; a < N; a++) dcdmu[k][l] += cD.cmu[a][k][l] * h<N>(ph, a);
      }
    }
    matinv_div<K>(dcdmu, iv);
#pragma unroll
    for (int k = 0; k < K; k++) {
      double s = 0;
#pragma unroll
      for (int l = 0; l < K; l++) s = s + iv[k][l] * dc[l];
      nm[k] = s + m[k];
    }
  }
  const long long o = (long long)x * g.pitch + y, od = (long long)(x + 1) * g.dpitch + (y + 1);
#pragma unroll
  for (int a = 0; a < N; a++) phin[a * g.plane + o] = ph[a] + dphi[a * g.dplane + od];
#pragma unroll
  for (int k = 0; k < K; k++) mun[k * g.plane + o] = nm[k];
}

}  // namespace gpd
