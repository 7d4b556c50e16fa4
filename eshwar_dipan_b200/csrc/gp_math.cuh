/*
 * gp_math.cuh -- per-cell thermodynamics and phase-field terms of the
 * grand-potential model on the device (FP64), in the reference's arithmetic
 * order so results are bit-identical to the CPU code (compile with
 * --fmad=false; '/' and sqrt are IEEE correctly rounded in CUDA).
 * Constants come from the __constant__ gp_derived block cD.
 */
#pragma once
#include "gp_internal.h"

/* one translation unit (gp_device.cu) includes this header */
__constant__ gp_derived cD;

namespace gpd {

/* h_a(phi) (functionH.h:24-36) */
template <int N>
__device__ __forceinline__ double h(const double *ph, int a) {
  double s1 = 0.0;
  double s = 3.0 * ph[a] * ph[a] - 2.0 * ph[a] * ph[a] * ph[a];
#pragma unroll
  for (int b = 0; b < N; b++)
#pragma unroll
    for (int c = 0; c < N; c++)
      if (b != a && c != a && b < c) s1 += ph[b] * ph[c];
  s1 *= 2.0 * ph[a];
  return s + s1;
}

/* d h_b / d phi_a (functionH.h:1-23, dhphi(phi, b, a)) */
template <int N>
__device__ __forceinline__ double dh(const double *ph, int b, int a) {
  double s = 0.0;
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

/* c_a,i(mu) (functionF_01.h:30-37) */
template <int K>
__device__ __forceinline__ double c_mu(const double *m, int a, int i) {
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < K; k++) s += cD.cmu[a][i][k] * (m[k] - cD.E[a][k]);
  return s;
}

/* Mu_a,i(c) (functionF_01.h:19-29) */
template <int K>
__device__ __forceinline__ double Mu(const double *c, int a, int i) {
  double s = cD.twoA[a][i] * c[i] + cD.E[a][i];
#pragma unroll
  for (int j = 0; j < K; j++)
    if (i != j) s += cD.A[a][i][j] * c[j];
  return s;
}

/* f_a(c) (functionF_01.h:5-18) */
template <int K>
__device__ __forceinline__ double fe(const double *c, int a) {
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < K; i++) {
#pragma unroll
    for (int j = 0; j < K; j++)
      if (i <= j) s += cD.A[a][i][j] * c[i] * c[j];
    s += cD.B[a][i] * c[i];
  }
  s += cD.C[a];
  return s;
}

/* FunctionTau (functionTau.h:1-17) */
template <int N>
__device__ __forceinline__ double tau_of(const double *ph) {
  double s = 0.0, s1 = 0.0;
#pragma unroll
  for (int a = 0; a < N; a++)
#pragma unroll
    for (int b = 0; b < N; b++)
      if (a < b) {
        s += cD.tau_ab[a][b] * ph[a] * ph[b];
        s1 += ph[a] * ph[b];
      }
  if (s1 != 0.0) return s / s1;
  return cD.tau;
}

/* D_ij of one cell (functionD.h:1-16); DC = Diffusivity*cmu folded on the host */
template <int N, int K>
__device__ __forceinline__ double Dcell(const double *ph, int i, int j) {
  double s = 0.0;
#pragma unroll
  for (int b = 0; b < N; b++)
#pragma unroll
    for (int k = 0; k < K; k++) s += cD.DC[b][i][j][k] * ph[b];
  return s;
}

/* dw/dphi_a, obstacle (functionW_01.h:6-39) or well (functionW_02.h:4-33);
 * smooth selects the _smooth variants (no sign test, other association). */
template <int N>
__device__ __forceinline__ double dwdphi(const double *ph, const bool *act, int a, bool smooth) {
  double s = 0.0;
#pragma unroll
  for (int b = 0; b < N; b++) {
    if (b == a || !act[b]) continue;
    if (cD.well) {
      s += 2.0 * cD.gamma[a][b] * (ph[b] * ph[b] * ph[a]);
    } else if (smooth) {
      s += cD.gamma[a][b] * ph[b];
    } else {
      if ((ph[a] * ph[b]) >= 0.00000) s += cD.gamma[a][b] * (ph[b]);
      else s += -cD.gamma[a][b] * (ph[b]);
    }
  }
  if (cD.well) s *= 9.0;
  else s *= cD.c16pi2;
#pragma unroll
  for (int b = 0; b < N; b++)
#pragma unroll
    for (int c = 0; c < N; c++)
      if (b != a && c != a && b < c && act[b] && act[c]) {
        if (smooth) {
          s += cD.gamma_abc[a][b][c] * ph[b] * ph[c];
        } else {
          double bc = ph[b] * ph[c];
          if (ph[a] * bc >= 0.00000) s += cD.gamma_abc[a][b][c] * bc;
          else s += -cD.gamma_abc[a][b][c] * bc;
        }
      }
  return s;
}

/* projection_on_simplex (simplex_projection.h:1-49) */
template <int N>
__device__ __forceinline__ void project(const double *ph, const bool *act, double *d) {
  double Dphi = 0.0, sum_phib = 0.0;
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
      double da = fabs(d[a] + ph[a]);
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
    d[hit] = (1.0 - ph[hit]);
#pragma unroll
    for (int b = 0; b < N; b++)
      if (act[b] && b != hit) d[b] = -ph[b];
  }
}

/* projection_on_simplex_without_weights (simplex_projection.h:50-91) */
template <int N>
__device__ __forceinline__ void project_nw(const double *ph, const bool *act, double *d) {
  long count = 0;
#pragma unroll
  for (int a = 0; a < N; a++)
    if (act[a] && (ph[a] + d[a]) > 0.0 && (ph[a] + d[a]) < 1.0) count++;
  bool done = false;
#pragma unroll
  for (int a = 0; a < N; a++) {
    if (done || !act[a]) continue;
    if ((ph[a] + d[a]) > 1.0) {
      d[a] = (1.0 - ph[a]);
#pragma unroll
      for (int b = 0; b < N; b++)
        if (act[b] && b != a) d[b] = -ph[b];
      done = true;
      continue;
    }
    if ((ph[a] + d[a]) < 0.0) {
      double Dphi = fabs(d[a] + ph[a]);
      d[a] += Dphi;
#pragma unroll
      for (int b = 0; b < N; b++)
        if ((act[b] && b != a) && (ph[b] + d[b]) > 0.0 && (ph[b] + d[b]) < 1.0) d[b] -= Dphi / (double)(count);
    }
  }
}

/* multiply(M, q, out, 2) (matrix.h:10-20); the identity case reduces to q+0.0
 * bit for bit (the leading 0.0 turns -0 into +0, the other term adds +-0). */
__device__ __forceinline__ void rot2(const double M[2][2], double q0, double q1, double &r0, double &r1) {
  if (cD.rot_identity) {
    r0 = q0 + 0.0;
    r1 = q1 + 0.0;
  } else {
    double s = 0;
    s = s + M[0][0] * q0;
    s = s + M[0][1] * q1;
    r0 = s;
    s = 0;
    s = s + M[1][0] * q0;
    s = s + M[1][1] * q1;
    r1 = s;
  }
}

/* anisotropy_01_function_ac (anisotropy_01.h:30-48), q_z = 0 */
__device__ __forceinline__ double ac(double qx, double qy, double dab) {
  double qx2 = qx * qx, qx4 = qx2 * qx2, qy2 = qy * qy, qy4 = qy2 * qy2;
  double qz2 = 0.0 * 0.0, qz4 = qz2 * qz2;
  double q2 = qx2 + qy2 + qz2;
  if (fabs(q2) > 1.0e-15) return 1.0 - dab * (3.0 - 4.0 * (qx4 + qy4 + qz4) / (q2 * q2));
  return 1.0;
}

/* one component of anisotropy_01_dAdq (anisotropy_01.h:9-29), q_z = 0:
 * 16*dab*(q_i^3/|q|^4 - q_i*sum q^4/|q|^6) */
struct QPow {
  double q2, q22, q23, q4;
};
__device__ __forceinline__ QPow qpow(double qx, double qy) {
  QPow r;
  double qx3 = qx * qx * qx, qy3 = qy * qy * qy, qz3 = 0.0;
  r.q2 = qx * qx + qy * qy + 0.0 * 0.0;
  r.q22 = r.q2 * r.q2;
  r.q23 = r.q2 * r.q2 * r.q2;
  r.q4 = qx3 * qx + qy3 * qy + qz3 * 0.0;
  return r;
}
__device__ __forceinline__ double dadq_c(double qi, const QPow &p, double dab16) {
  if (fabs(p.q2) > 1.0e-15) return dab16 * (qi * qi * qi / p.q22 - qi * p.q4 / p.q23);
  return 0.0;
}

}  // namespace gpd

namespace gpd {
/* matinvnew (matrix.h:50-218) for n = K <= 2 with 1.0/x as the reciprocal
 * (pow(x,-1) of the host library cannot be reproduced on the device; the
 * reference uses it only in the smoothing sweeps and for K>2 without
 * BINARY/TERNARY/DILUTE). */
template <int K>
__device__ __forceinline__ void matinv_div(double (&m)[K][K], double (&inv)[K][K]) {
  double fac[K][K], inv1[K][K], v1[K], v[K];
  int tag[K];
#pragma unroll
  for (int i = 0; i < K; i++) {
    tag[i] = i;
#pragma unroll
    for (int j = 0; j < K; j++) fac[i][j] = 0.0;
  }
#pragma unroll
  for (int k = 0; k < K; k++) {
    double big = fabs(m[k][k]);
    int t1 = k;
#pragma unroll
    for (int i = k + 1; i < K; i++)
      if (fabs(m[i][k]) > big) { t1 = i; big = m[i][k]; }
    if (t1 != k) {
      int s = tag[k]; tag[k] = tag[t1]; tag[t1] = s;
#pragma unroll
      for (int i = 0; i < K; i++) { double w = m[k][i]; m[k][i] = m[t1][i]; m[t1][i] = w; }
#pragma unroll
      for (int i = 0; i < k; i++) { double w = fac[k][i]; fac[k][i] = fac[t1][i]; fac[t1][i] = w; }
    }
#pragma unroll
    for (int i = k + 1; i < K; i++) {
      double f = -m[i][k] / m[k][k];
      fac[i][k] = -f;
#pragma unroll
      for (int j = k; j <= K - 1; j++) m[i][j] = f * m[k][j] + m[i][j];
    }
  }
#pragma unroll
  for (int i = 0; i < K; i++)
#pragma unroll
    for (int j = 0; j < K; j++) {
      if (i == j) fac[i][j] = 1;
      if (j > i) fac[i][j] = 0;
    }
#pragma unroll
  for (int i = 0; i < K; i++) {
    v1[0] = (i == 0) ? 1.0 : 0.0;
#pragma unroll
    for (int r = 1; r < K; r++) {
      double s = 0;
#pragma unroll
      for (int j = 0; j < r; j++) s = s - fac[r][j] * v1[j];
      v1[r] = ((r == i) ? 1.0 : 0.0) + s;
    }
    v[K - 1] = v1[K - 1] * (1.0 / m[K - 1][K - 1]);
#pragma unroll
    for (int r = K - 2; r >= 0; r--) {
      double s = 0;
#pragma unroll
      for (int j = r + 1; j < K; j++) s = s - m[r][j] * v[j];
      v[r] = (v1[r] + s) * (1.0 / m[r][r]);
    }
#pragma unroll
    for (int j = 0; j < K; j++) inv1[j][i] = v[j];
  }
#pragma unroll
  for (int j = 0; j < K; j++)
#pragma unroll
    for (int i = 0; i < K; i++) inv[i][tag[j]] = inv1[i][j];
}
}  // namespace gpd
