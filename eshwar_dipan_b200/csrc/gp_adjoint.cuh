/*
 * gp_adjoint.cuh -- the FP64 step as per-cell functions of a generic scalar,
 * for the adjoint (gp_adjoint in gp.h).
 *
 * The time step is written here as two cell functions:
 *   dphi_cell    delta-phi of one cell of the interior plus its ring from the
 *                phi of its 3x3 neighbourhood and its own mu
 *                (calculate_divergence_phasefield_2D, calculate_divergence_phasefield.h:4-62);
 *   update_cell  new phi and mu of one interior cell from the phi of its 3x3
 *                neighbourhood and the mu and delta-phi of its 5-point
 *                neighbourhood (calculate_fluxes_concentration_2D +
 *                calculate_divergence_concentration_2D,
 *                calculate_fluxes_concentration.h:4-145, calculate_divergence_concentration.h:4-153).
 * Every expression is the FP64 kernel's (gp_tiles.cuh / gp_fused.cuh) in the
 * same order, so with T = double the functions reproduce the production step
 * bit for bit (the replay check in gp_adjoint_replay), and with T = Dual<W>
 * they also return exact partial derivatives along W seeded inputs.
 *
 * Differentiable parameters (AdjParams): Tau of the pair (0,1) (mobility is
 * 1/Tau), dab of the pair (0,1) (anisotropy strength), epsilon (interface
 * width) and GAMMA of the pair (0,1) (interface energy).  Everything else comes
 * from the simulation's FP64 constant block.
 */
#pragma once
#include "gp_adjoint_launch.h"
#include "gp_dual.cuh"
#include "gp_tiles.cuh"

namespace gpd {


/* The constants of one step, the differentiable ones in T. */
template <typename T>
struct AK {
  const Consts<double> *c;
  T tau01, dab01, dab16_01, eps, inv_eps, jat_obst, jat_well, gamma01;
  __host__ __device__ bool pair01(int a, int b) const { return (a == 0 && b == 1) || (a == 1 && b == 0); }
  __host__ __device__ T gamma(int a, int b) const { return pair01(a, b) ? gamma01 : T(c->gamma[a][b]); }
  __host__ __device__ T tau_ab(int a, int b) const { return pair01(a, b) ? tau01 : T(c->tau_ab[a][b]); }
  __host__ __device__ T dab(int a, int b) const { return pair01(a, b) ? dab01 : T(c->dab[a][b]); }
  __host__ __device__ T dab16(int a, int b) const { return pair01(a, b) ? dab16_01 : T(c->dab16[a][b]); }
};

/* derived constants as gp_host_derive computes them (gp_host.c) */
template <typename T>
__device__ __forceinline__ AK<T> make_ak(const Consts<double> *c, const T (&p)[ADJ_NPARAM]) {
  AK<T> k;
  k.c = c;
  k.tau01 = p[ADJ_TAU];
  k.dab01 = p[ADJ_DAB];
  k.dab16_01 = 16.0 * p[ADJ_DAB];
  k.eps = p[ADJ_EPS];
  k.inv_eps = 1.0 / p[ADJ_EPS];
  k.jat_obst = (-0.25 * M_PI) * p[ADJ_EPS];
  k.jat_well = -1.0 * p[ADJ_EPS];
  k.gamma01 = p[ADJ_GAMMA];
  return k;
}

template <typename T>
__device__ __forceinline__ T adivx(T v, const AK<T> &D) { return D.c->mul_dx ? v * D.c->inv_dx : v / D.c->dx; }
template <typename T>
__device__ __forceinline__ T adivy(T v, const AK<T> &D) { return D.c->mul_dy ? v * D.c->inv_dy : v / D.c->dy; }
template <typename T>
__device__ __forceinline__ T adiv2y(T v, const AK<T> &D) {
  return D.c->mul_dy ? v * D.c->inv_2dy : v / (2.0 * D.c->dy);
}

/* ---- free-energy, interpolation and kinetic functions (gp_math.cuh, same order) */

template <typename T, int N>
__device__ __forceinline__ T ah(const T *ph, int a) {
  T s1 = T(0.0);
  T s = 3.0 * ph[a] * ph[a] - 2.0 * ph[a] * ph[a] * ph[a];
#pragma unroll
  for (int b = 0; b < N; b++)
#pragma unroll
    for (int c = 0; c < N; c++)
      if (b != a && c != a && b < c) s1 += ph[b] * ph[c];
  s1 *= 2.0 * ph[a];
  return s + s1;
}

template <typename T, int N>
__device__ __forceinline__ T adh(const T *ph, int b, int a) {
  T s = T(0.0);
  if (a == b) {
    s = 6.0 * ph[a] * (1.0 - ph[a]);
#pragma unroll
    for (int e = 0; e < N; e++)
#pragma unroll
      for (int f = 0; f < N; f++)
        if (e != b && f != b && e < f) s += 2.0 * ph[e] * ph[f];
  } else {
#pragma unroll
    for (int e = 0; e < N; e++)
      if (e != b && e != a) s += 2.0 * ph[e];
    s *= ph[b];
  }
  return s;
}

template <typename T, int K>
__device__ __forceinline__ T ac_mu(const AK<T> &D, const T *m, int a, int i) {
  T s = T(0.0);
#pragma unroll
  for (int k = 0; k < K; k++) s += D.c->cmu[a][i][k] * (m[k] - D.c->E[a][k]);
  return s;
}

template <typename T, int K>
__device__ __forceinline__ T aMu(const AK<T> &D, const T *c, int a, int i) {
  T s = D.c->twoA[a][i] * c[i] + D.c->E[a][i];
#pragma unroll
  for (int j = 0; j < K; j++)
    if (i != j) s += D.c->A[a][i][j] * c[j];
  return s;
}

template <typename T, int K>
__device__ __forceinline__ T afe(const AK<T> &D, const T *c, int a) {
  T s = T(0.0);
#pragma unroll
  for (int i = 0; i < K; i++) {
#pragma unroll
    for (int j = 0; j < K; j++)
      if (i <= j) s += D.c->A[a][i][j] * c[i] * c[j];
    s += D.c->B[a][i] * c[i];
  }
  s += D.c->C[a];
  return s;
}

template <typename T, int N>
__device__ __forceinline__ T atau(const AK<T> &D, const T *ph) {
  T s = T(0.0), s1 = T(0.0);
#pragma unroll
  for (int a = 0; a < N; a++)
#pragma unroll
    for (int b = 0; b < N; b++)
      if (a < b) {
        s += D.tau_ab(a, b) * ph[a] * ph[b];
        s1 += ph[a] * ph[b];
      }
  if (s1 != 0.0) return s / s1;
  return T(D.c->tau);
}

template <typename T, int N, int K>
__device__ __forceinline__ T aDcell(const AK<T> &D, const T *ph, int i, int j) {
  T s = T(0.0);
#pragma unroll
  for (int b = 0; b < N; b++)
#pragma unroll
    for (int k = 0; k < K; k++) s += D.c->DC[b][i][j][k] * ph[b];
  return s;
}

template <typename T, int N>
__device__ __forceinline__ T adwdphi(const AK<T> &D, const T *ph, const bool *act, int a) {
  T s = T(0.0);
#pragma unroll
  for (int b = 0; b < N; b++) {
    if (b == a || !act[b]) continue;
    if (D.c->well) {
      s += 2.0 * D.gamma(a, b) * (ph[b] * ph[b] * ph[a]);
    } else {
      if ((ph[a] * ph[b]) >= 0.00000) s += D.gamma(a, b) * (ph[b]);
      else s += -D.gamma(a, b) * (ph[b]);
    }
  }
  if (D.c->well) s *= 9.0;
  else s *= D.c->c16pi2;
#pragma unroll
  for (int b = 0; b < N; b++)
#pragma unroll
    for (int c = 0; c < N; c++)
      if (b != a && c != a && b < c && act[b] && act[c]) {
        T bc = ph[b] * ph[c];
        if (ph[a] * bc >= 0.00000) s += D.c->gamma_abc[a][b][c] * bc;
        else s += -D.c->gamma_abc[a][b][c] * bc;
      }
  return s;
}

template <typename T, int N>
__device__ __forceinline__ void aproject(const T *ph, const bool *act, T *d) {
  T Dphi = T(0.0), sum_phib = T(0.0);
  long count = 0;
#pragma unroll
  for (int a = 0; a < N; a++)
    if (act[a] && (ph[a] + d[a]) > 0.0 && (ph[a] + d[a]) < 1.0) {
      count++;
      sum_phib += ph[a];
    }
#pragma unroll
  for (int a = 0; a < N; a++)
    if ((ph[a] + d[a]) < 0.0) {
      T da = fabs(d[a] + ph[a]);
      d[a] += da;
      Dphi += da;
    }
  if (Dphi > 0.0) {
#pragma unroll
    for (int b = 0; b < N; b++)
      if (act[b] && ((ph[b] + d[b]) > 0.0) && ((ph[b] + d[b]) < 1.0)) {
        if (fabs(sum_phib) > 0.0) d[b] -= Dphi * (ph[b]) / (sum_phib);
        else d[b] -= Dphi / (double)(count);
      }
  }
  int hit = -1;
#pragma unroll
  for (int a = 0; a < N; a++)
    if (hit < 0 && act[a] && (ph[a] + d[a]) > 1.0) hit = a;
  if (hit >= 0) {
    /* d[hit] = 1 - ph[hit], the other active phases -ph (by compile-time indices) */
#pragma unroll
    for (int b = 0; b < N; b++) {
      if (b == hit) d[b] = (1.0 - ph[b]);
      else if (act[b]) d[b] = -ph[b];
    }
  }
}

template <typename T>
__device__ __forceinline__ void arot2(const AK<T> &D, const double (&M)[2][2], T q0, T q1, T &r0, T &r1) {
  if (D.c->rot_identity) {
    r0 = q0 + 0.0;
    r1 = q1 + 0.0;
  } else {
    T s = T(0.0);
    s = s + M[0][0] * q0;
    s = s + M[0][1] * q1;
    r0 = s;
    s = T(0.0);
    s = s + M[1][0] * q0;
    s = s + M[1][1] * q1;
    r1 = s;
  }
}

template <typename T>
__device__ __forceinline__ T aac(T qx, T qy, T dab) {
  T qx2 = qx * qx, qx4 = qx2 * qx2, qy2 = qy * qy, qy4 = qy2 * qy2;
  double qz2 = 0.0 * 0.0, qz4 = qz2 * qz2;
  T q2 = qx2 + qy2 + qz2;
  if (fabs(q2) > 1.0e-15) return 1.0 - dab * (3.0 - 4.0 * (qx4 + qy4 + qz4) / (q2 * q2));
  return T(1.0);
}

template <typename T>
struct AQPow {
  T q2, q22, q23, q4;
};
template <typename T>
__device__ __forceinline__ AQPow<T> aqpow(T qx, T qy) {
  AQPow<T> r;
  T qx3 = qx * qx * qx, qy3 = qy * qy * qy;
  const double qz3 = 0.0;
  r.q2 = qx * qx + qy * qy + 0.0 * 0.0;
  r.q22 = r.q2 * r.q2;
  r.q23 = r.q2 * r.q2 * r.q2;
  r.q4 = qx3 * qx + qy3 * qy + qz3 * 0.0;
  return r;
}
template <typename T>
__device__ __forceinline__ T adadq(T qi, const AQPow<T> &p, T dab16) {
  if (fabs(p.q2) > 1.0e-15) return dab16 * (qi * qi * qi / p.q22 - qi * p.q4 / p.q23);
  return T(0.0);
}


/* ---- phase-field pass ------------------------------------------------- */

/* Anisotropy terms of one face of the 3x3 window S (rows i, columns j): the
 * arithmetic of face_terms (gp_tiles.cuh).  xface: between (i,j) and (i+1,j);
 * else between (i,j) and (i,j+1).  T4[p][0..3] as in the tile face cache. */
template <typename T, int N>
__device__ __forceinline__ void aface(const AK<T> &D, const T (&S)[N][3][3], bool xface, int i, int j,
                                      T (&F)[NP<N>::v][4]) {
  T s[N], gr[N], c0[N], c1[N];
#pragma unroll
  for (int a = 0; a < N; a++) {
    if (xface) {
      T p0 = S[a][i][j], p1 = S[a][i + 1][j];
      s[a] = 0.5 * (p1 + p0);
      gr[a] = adivx(p1 - p0, D);
      c0[a] = adiv2y(S[a][i][j + 1] - S[a][i][j - 1], D);
      c1[a] = adiv2y(S[a][i + 1][j + 1] - S[a][i + 1][j - 1], D);
    } else {
      T p0 = S[a][i][j], p1 = S[a][i][j + 1];
      s[a] = 0.5 * (p1 + p0);
      gr[a] = adivy(p1 - p0, D);
      c0[a] = 0.5 * (adivx(S[a][i + 1][j] - S[a][i][j], D) + adivx(S[a][i][j] - S[a][i - 1][j], D));
      c1[a] = 0.5 * (adivx(S[a][i + 1][j + 1] - S[a][i][j + 1], D) + adivx(S[a][i][j + 1] - S[a][i - 1][j + 1], D));
    }
  }
#pragma unroll
  for (int a = 0; a < N; a++)
#pragma unroll
    for (int b = a + 1; b < N; b++) {
      const int p = pidx<N>(a, b);
      T Pab = s[a] * gr[b] - s[b] * gr[a];
      T Pba = s[b] * gr[a] - s[a] * gr[b];
      T tq = 0.5 * (s[a] * (c0[b] + c1[b]) - s[b] * (c0[a] + c1[a]));
      T q0, q1;
      if (xface) arot2(D, D.c->rot[a][b], Pab, tq, q0, q1);
      else arot2(D, D.c->rot[a][b], tq, Pab, q0, q1);
      T acv = aac(q0, q1, D.dab(a, b));
      AQPow<T> qp = aqpow(q0, q1);
      T rd;
      if (D.c->rot_identity) {
        rd = (xface ? adadq(q0, qp, D.dab16(a, b)) : adadq(q1, qp, D.dab16(a, b))) + 0.0;
      } else {
        T d0 = adadq(q0, qp, D.dab16(a, b)), d1 = adadq(q1, qp, D.dab16(a, b));
        T r0, r1;
        arot2(D, D.c->rinv[a][b], d0, d1, r0, r1);
        rd = xface ? r0 : r1;
      }
      T ac2 = acv * acv, acq = acv * qp.q2;
      F[p][0] = ac2 * Pab * (-s[b]);
      F[p][1] = ac2 * Pba * (-s[a]);
      F[p][2] = acq * rd * (-s[b]);
      F[p][3] = acq * (0.0 - rd) * (-s[a]);
    }
}

/* delta-phi of the centre cell of the 3x3 window S with mu m (ring_dphi). */
template <typename T, int N, int K, bool ANISO>
__device__ __forceinline__ void dphi_cell(const AK<T> &D, const T (&S)[N][3][3], const T (&m)[K], T (&d)[N]) {
  T ph[N];
  bool act[N];
  bool any = false;
#pragma unroll
  for (int a = 0; a < N; a++) {
    ph[a] = S[a][1][1];
    T gxf = adivx(S[a][2][1] - S[a][1][1], D), gxb = adivx(S[a][1][1] - S[a][0][1], D);
    T gyr = adivy(S[a][1][2] - S[a][1][1], D), gyl = adivy(S[a][1][1] - S[a][1][0], D);
    T dv = adivx(gxf - gxb, D);
    dv += adivy(gyr - gyl, D);
    act[a] = fabs(dv) > 0.0;
    any |= act[a];
  }
  if (!any) {
#pragma unroll
    for (int a = 0; a < N; a++) {
      d[a] = T(0.0);
      if ((ph[a] + d[a]) < 0.0) d[a] += fabs(d[a] + ph[a]);
    }
    return;
  }
  T gcx[N], gcy[N];
#pragma unroll
  for (int a = 0; a < N; a++) {
    gcx[a] = 0.5 * (adivx(S[a][2][1] - S[a][1][1], D) + adivx(S[a][1][1] - S[a][0][1], D));
    gcy[a] = adiv2y(S[a][1][2] - S[a][1][0], D);
  }
  T psi[N];
#pragma unroll
  for (int b = 0; b < N; b++) {
    T c[K], ps = T(0.0);
#pragma unroll
    for (int k = 0; k < K; k++) {
      c[k] = ac_mu<T, K>(D, m, b, k);
      ps -= m[k] * c[k];
    }
    ps += afe<T, K>(D, c, b);
    psi[b] = ps;
  }
  /* the four faces of the cell: forward/backward x, right/left y */
  T Fxf[NP<N>::v][4], Fxb[NP<N>::v][4], Fyr[NP<N>::v][4], Fyl[NP<N>::v][4];
  T cq0[NP<N>::v], cq1[NP<N>::v], cd0[NP<N>::v], cd1[NP<N>::v], cac[NP<N>::v], cq2[NP<N>::v];
  if (ANISO) {
    aface<T, N>(D, S, true, 1, 1, Fxf);
    aface<T, N>(D, S, true, 0, 1, Fxb);
    aface<T, N>(D, S, false, 1, 1, Fyr);
    aface<T, N>(D, S, false, 1, 0, Fyl);
#pragma unroll
    for (int a = 0; a < N; a++)
#pragma unroll
      for (int b = a + 1; b < N; b++) {
        const int p = pidx<N>(a, b);
        T q0, q1;
        arot2(D, D.c->rot[a][b], (ph[a] * gcx[b] - ph[b] * gcx[a]), (ph[a] * gcy[b] - ph[b] * gcy[a]), q0, q1);
        AQPow<T> qp = aqpow(q0, q1);
        cq0[p] = q0;
        cq1[p] = q1;
        cd0[p] = adadq(q0, qp, D.dab16(a, b));
        cd1[p] = adadq(q1, qp, D.dab16(a, b));
        cq2[p] = (q0 * q0 + q1 * q1 + 0.0 * 0.0);
        cac[p] = aac(q0, q1, D.dab(a, b));
      }
  }
  const T tau = atau<T, N>(D, ph);
  T lam[N], sl = T(0.0);
  long nact = 0;
#pragma unroll
  for (int a = 0; a < N; a++) {
    if (!act[a]) continue;
    T dA, div;
    if (ANISO) {
      T s1 = T(0.0), s2 = T(0.0), t1 = T(0.0), t2 = T(0.0);
#pragma unroll
      for (int b = 0; b < N; b++) {
        if (b == a) continue;
        const int p = a < b ? pidx<N>(a, b) : pidx<N>(b, a);
        const double sg = 0.0;
        T q0 = a < b ? cq0[p] : sg - cq0[p], q1 = a < b ? cq1[p] : sg - cq1[p];
        T d0 = a < b ? cd0[p] : sg - cd0[p], d1 = a < b ? cd1[p] : sg - cd1[p];
        T w0, w1;
        arot2(D, D.c->rot[a][b], gcx[b], gcy[b], w0, w1);
        T sp1 = T(0.0), sp2 = T(0.0);
        sp1 += q0 * w0;
        sp1 += q1 * w1;
        sp2 += (d0) * w0;
        sp2 += (d1) * w1;
        sp1 *= D.gamma(a, b) * (cac[p] * cac[p]);
        sp2 *= D.gamma(a, b) * cac[p] * cq2[p];
        s1 += sp1;
        s2 += sp2;
        const int o = a < b ? 0 : 1;
        T d1v = adivx((Fxf[p][o]) - (Fxb[p][o]), D);
        d1v += adivy((Fyr[p][o]) - (Fyl[p][o]), D);
        d1v *= D.gamma(a, b);
        t1 += d1v;
        T d2v = adivx(Fxf[p][2 + o] - Fxb[p][2 + o], D);
        d2v += adivy(Fyr[p][2 + o] - Fyl[p][2 + o], D);
        d2v *= D.gamma(a, b);
        t2 += d2v;
      }
      dA = 2.0 * (s1 + s2);
      div = (2.0 * (t1 + t2) + 0.0);
    } else {
      T s = T(0.0), t = T(0.0);
#pragma unroll
      for (int b = 0; b < N; b++) {
        if (b == a) continue;
        T sp = T(0.0);
        sp += (ph[a] * gcx[b] - ph[b] * gcx[a]) * gcx[b];
        sp += (ph[a] * gcy[b] - ph[b] * gcy[a]) * gcy[b];
        sp *= D.gamma(a, b);
        s += sp;
        T pa = S[a][1][1], pb = S[b][1][1];
        T sxa = 0.5 * (S[a][2][1] + pa), sxb = 0.5 * (S[b][2][1] + pb);
        T gxa = adivx(S[a][2][1] - pa, D), gxb = adivx(S[b][2][1] - pb, D);
        T bxa = 0.5 * (pa + S[a][0][1]), bxb = 0.5 * (pb + S[b][0][1]);
        T hxa = adivx(pa - S[a][0][1], D), hxb = adivx(pb - S[b][0][1], D);
        T sya = 0.5 * (S[a][1][2] + pa), syb = 0.5 * (S[b][1][2] + pb);
        T gya = adivy(S[a][1][2] - pa, D), gyb = adivy(S[b][1][2] - pb, D);
        T lya = 0.5 * (pa + S[a][1][0]), lyb = 0.5 * (pb + S[b][1][0]);
        T hya = adivy(pa - S[a][1][0], D), hyb = adivy(pb - S[b][1][0], D);
        T dvg = adivx((sxa * gxb - sxb * gxa) * (-sxb) - ((bxa * hxb - bxb * hxa) * (-bxb)), D);
        dvg += adivy((sya * gyb - syb * gya) * (-syb) - ((lya * hyb - lyb * hya) * (-lyb)), D);
        dvg *= D.gamma(a, b);
        t += dvg;
      }
      dA = 2.0 * s;
      div = 2.0 * t;
    }
    T dpsi = T(0.0);
#pragma unroll
    for (int b = 0; b < N; b++) dpsi += psi[b] * adh<T, N>(ph, b, a);
    lam[a] = D.eps * (-dA + div) - D.inv_eps * adwdphi<T, N>(D, ph, act, a) - dpsi;
    sl += lam[a];
    nact++;
  }
  if (nact) sl /= (double)nact;
#pragma unroll
  for (int a = 0; a < N; a++) d[a] = act[a] ? D.c->dt * (lam[a] - sl) / (tau * D.eps) : T(0.0);
  aproject<T, N>(ph, act, d);
}

/* ---- concentration pass ----------------------------------------------- */

/* Quantities of one cell (update_tile's per-cell loop). */
template <typename T, int N, int K>
struct ACell {
  T H[N], CM[N][K], SP[N], DD[K][K];
};
template <typename T, int N, int K>
__device__ __forceinline__ void acell(const AK<T> &D, const T *p, const T *mm, ACell<T, N, K> &q) {
  constexpr int L = N - 1;
#pragma unroll
  for (int a = 0; a < N; a++) {
    T hv = ah<T, N>(p, a);
    q.H[a] = hv;
#pragma unroll
    for (int k = 0; k < K; k++) q.CM[a][k] = ac_mu<T, K>(D, mm, a, k);
    if (a < L) q.SP[a] = (p[a] * (1.0 - p[a]) > 0.0) ? p[a] * (1.0 - hv) / (sqrt(p[a] * (1.0 - p[a]))) : T(0.0);
  }
#pragma unroll
  for (int k = 0; k < K; k++)
#pragma unroll
    for (int l = 0; l < K; l++) q.DD[k][l] = aDcell<T, N, K>(D, p, k, l);
}

/* Anti-trapping current and diffusion flux products through one face of the
 * window (faces loop of update_tile).  xface: between (i,j) and (i+1,j);
 * else between (i,j) and (i,j+1).  q0/q1: the two cells' quantities; ylo: the
 * interior y of the face's lower cell (y-faces only). */
template <typename T, int N, int K>
__device__ __forceinline__ void aflux(const AK<T> &D, const T (&S)[N][3][3], const T (&M)[K][3][3],
                                      const T (&DP)[N][3][3], const ACell<T, N, K> &q0, const ACell<T, N, K> &q1,
                                      bool xface, int fi, int fj, int ylo, int my, T (&jat)[K], T (&F)[K][K]) {
  constexpr int L = N - 1;
  const int i1 = xface ? fi + 1 : fi, j1 = xface ? fj : fj + 1;
  T gr[N], cn[N];
#pragma unroll
  for (int a = 0; a < N; a++) {
    if (xface) {
      gr[a] = adivx(S[a][i1][j1] - S[a][fi][fj], D);
      cn[a] = 0.5 * (adiv2y(S[a][fi][fj + 1] - S[a][fi][fj - 1], D) + adiv2y(S[a][i1][fj + 1] - S[a][i1][fj - 1], D));
    } else {
      gr[a] = adivy(S[a][i1][j1] - S[a][fi][fj], D);
      T gc0 = 0.5 * (adivx(S[a][fi + 1][fj] - S[a][fi][fj], D) + adivx(S[a][fi][fj] - S[a][fi - 1][fj], D));
      T gc1 = 0.5 * (adivx(S[a][fi + 1][j1] - S[a][i1][j1], D) + adivx(S[a][i1][j1] - S[a][fi - 1][j1], D));
      cn[a] = 0.5 * (gc0 + gc1);
    }
  }
#pragma unroll
  for (int k = 0; k < K; k++) jat[k] = T(0.0);
  const bool yskip = !xface && (ylo + 3 == my - 2);
  T nl = T(-1.0);
#pragma unroll
  for (int a = 0; a < L; a++) {
    const T s2 = cn[a] * cn[a] + gr[a] * gr[a];
    if (s2 != 0.0 && !yskip) {
      const T ng = sqrt(s2);
      if (nl < 0.0) nl = sqrt(cn[L] * cn[L] + gr[L] * gr[L]);
      T sp = gr[a] * gr[L];
      sp += cn[a] * cn[L];
      if (nl > 0.0) sp /= (nl * ng);
#pragma unroll
      for (int k = 0; k < K; k++) {
        T cl1 = q1.CM[L][k], cl0 = q0.CM[L][k];
        T cs1 = q1.CM[a][k], cs0 = q0.CM[a][k];
        T bracket;
        if (D.c->obstacle)
          bracket = q1.SP[a] * (cl1 - cs1) * DP[a][i1][j1] + q0.SP[a] * (cl0 - cs0) * DP[a][fi][fj];
        else
          bracket = (cl1 - cs1) * DP[a][i1][j1] + (cl0 - cs0) * DP[a][fi][fj];
        jat[k] += D.c->atf[a][k] * fabs(sp) * (D.c->obstacle ? 0.5 : D.c->well_half) * bracket * gr[a] / ng;
      }
    }
  }
#pragma unroll
  for (int k = 0; k < K; k++)
#pragma unroll
    for (int l = 0; l < K; l++) {
      T dm = (q1.DD[k][l] + q0.DD[k][l]) * 0.5;
      T gm = xface ? adivx(M[l][i1][j1] - M[l][fi][fj], D) : adivy(M[l][i1][j1] - M[l][fi][fj], D);
      F[k][l] = dm * gm;
    }
}

/* New phi and mu of the centre cell of the window (interior coordinates x, y):
 * S phi 3x3; M mu and DP delta-phi, of which the 5-point stencil is used. */
template <typename T, int N, int K>
__device__ __forceinline__ void update_cell(const AK<T> &D, const T (&S)[N][3][3], const T (&M)[K][3][3],
                                            const T (&DP)[N][3][3], int y, int my, T (&nph)[N], T (&nm)[K]) {
  /* cells: centre, x-1, x+1, y-1, y+1 */
  const int ci[5] = {1, 0, 2, 1, 1}, cj[5] = {1, 1, 1, 0, 2};
  ACell<T, N, K> q[5];
#pragma unroll
  for (int e = 0; e < 5; e++) {
    T p[N], mm[K];
#pragma unroll
    for (int a = 0; a < N; a++) p[a] = S[a][ci[e]][cj[e]];
#pragma unroll
    for (int k = 0; k < K; k++) mm[k] = M[k][ci[e]][cj[e]];
    acell<T, N, K>(D, p, mm, q[e]);
  }
  T jxf[K], jxb[K], jyr[K], jyl[K], fxf[K][K], fxb[K][K], fyr[K][K], fyl[K][K];
  aflux<T, N, K>(D, S, M, DP, q[0], q[2], true, 1, 1, 0, my, jxf, fxf);
  aflux<T, N, K>(D, S, M, DP, q[1], q[0], true, 0, 1, 0, my, jxb, fxb);
  aflux<T, N, K>(D, S, M, DP, q[0], q[4], false, 1, 1, y, my, jyr, fyr);
  aflux<T, N, K>(D, S, M, DP, q[3], q[0], false, 1, 0, y - 1, my, jyl, fyl);
  const T cst = D.c->obstacle ? D.jat_obst : D.jat_well;
  T ph[N], dp[N], m[K];
#pragma unroll
  for (int a = 0; a < N; a++) { ph[a] = S[a][1][1]; dp[a] = DP[a][1][1]; }
#pragma unroll
  for (int k = 0; k < K; k++) m[k] = M[k][1][1];
  T divflux[K], divjat[K];
#pragma unroll
  for (int k = 0; k < K; k++) {
    divflux[k] = T(0.0);
#pragma unroll
    for (int l = 0; l < K; l++) {
      divflux[k] += adivx(fxf[k][l] - fxb[k][l], D);
      divflux[k] += adivy(fyr[k][l] - fyl[k][l], D);
    }
    divjat[k] = adivx((jxf[k] - jxb[k]) * cst, D);
    divjat[k] += adivy((jyr[k] - jyl[k]) * cst, D);
  }
  int bulk = -1;
#pragma unroll
  for (int a = 0; a < N; a++)
    if (bulk < 0 && ph[a] == 1.0) bulk = a;
  if (bulk >= 0) {
    /* the bulk phase's c_mu, picked by compile-time indices (q stays in registers) */
    T cb[K];
#pragma unroll
    for (int k = 0; k < K; k++) cb[k] = q[0].CM[0][k];
#pragma unroll
    for (int a = 1; a < N; a++)
      if (a == bulk)
#pragma unroll
        for (int k = 0; k < K; k++) cb[k] = q[0].CM[a][k];
    T cn[K];
#pragma unroll
    for (int k = 0; k < K; k++) cn[k] = cb[k] + D.c->dt * (divflux[k]) - divjat[k];
#pragma unroll
    for (int k = 0; k < K; k++) nm[k] = aMu<T, K>(D, cn, bulk, k);
  } else {
    T sum[K], dc[K], dcdmu[K][K];
#pragma unroll
    for (int k = 0; k < K; k++) sum[k] = T(0.0);
#pragma unroll
    for (int a = 0; a < N; a++) {
      T sdh = T(0.0);
#pragma unroll
      for (int b = 0; b < N; b++) sdh += adh<T, N>(ph, a, b) * dp[b];
#pragma unroll
      for (int k = 0; k < K; k++) sum[k] += q[0].CM[a][k] * sdh;
    }
#pragma unroll
    for (int k = 0; k < K; k++) {
      dc[k] = D.c->dt * (divflux[k]) - divjat[k] - sum[k];
#pragma unroll
      for (int l = 0; l < K; l++) {
        dcdmu[k][l] = T(0.0);
#pragma unroll
        for (int a = 0; a < N; a++) dcdmu[k][l] += D.c->cmu64[a][k][l] * q[0].H[a];
      }
    }
    T m64[K];
#pragma unroll
    for (int k = 0; k < K; k++) m64[k] = m[k];
    if (K == 1 || D.c->inv_mode == GP_INV_BINARY) {
      T i00 = 1.0 / dcdmu[0][0];
      T dmu = dc[0] * i00;
      m64[0] += dmu;
    } else if (D.c->inv_mode == GP_INV_TERNARY) {
      T det = dcdmu[0][0] * dcdmu[K - 1][K - 1] - dcdmu[0][K - 1] * dcdmu[K - 1][0];
      T iv[K][K];
      iv[0][0] = dcdmu[K - 1][K - 1] / det;
      iv[K - 1][K - 1] = dcdmu[0][0] / det;
      iv[0][K - 1] = -dcdmu[0][K - 1] / det;
      iv[K - 1][0] = -dcdmu[K - 1][0] / det;
      T dmu[K];
#pragma unroll
      for (int k = 0; k < K; k++) {
        dmu[k] = T(0.0);
#pragma unroll
        for (int l = 0; l < K; l++) dmu[k] += iv[k][l] * dc[l];
      }
#pragma unroll
      for (int k = 0; k < K; k++) m64[k] = dmu[k] + m64[k];
    } else {
#pragma unroll
      for (int k = 0; k < K; k++) {
        T ikk = 1.0 / dcdmu[k][k];
        T dmu = dc[k] * ikk;
        m64[k] += dmu;
      }
    }
#pragma unroll
    for (int k = 0; k < K; k++) nm[k] = m64[k];
  }
#pragma unroll
  for (int a = 0; a < N; a++) nph[a] = ph[a] + dp[a];
}

}  // namespace gpd
