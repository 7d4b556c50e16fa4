/*
 * gp_math.cuh -- per-cell thermodynamics and phase-field terms of the
 * grand-potential model on the device, templated on the field type R (double
 * for the plain form, float for the FP32 storage form) and reading the
 * constants of one simulation from a Consts<R> block.
 *
 * With R = double and --fmad=false the arithmetic follows the reference
 * expression by expression (same operands, same association; '/' and sqrt
 * are IEEE correctly rounded in CUDA), so results are bit-identical to the CPU
 * code.  Literal constants are written R(...) so that the float form stays in
 * float.
 */
#pragma once
#include "gp_internal.h"

namespace gpd {

/* Constants of one simulation in the field type (see gp_derived for their
 * meaning), plus FP64 copies of cmu (dc/dmu of each phase, for the inversion
 * of the FP32 form) and of its inverse muc (dmu/dc of each phase: 2A on the
 * diagonal, A off it; the FP32 form's bulk update). */
template <typename R>
struct Consts {
  R dx, dy, dt, eps, inv_eps, tau, c16pi2, jat_obst, jat_well, well_half;
  R inv_dx, inv_dy, inv_2dy;   /* used instead of dividing when mul_dx/mul_dy are set */
  int mul_dx, mul_dy;          /* FP64: dx (dy) is a power of two, so x*(1/dx) == x/dx exactly */
  int obstacle, well, aniso, inv_mode, rot_identity;
  int bc_x[2][2], bc_y[2][2];
  R gamma[GPK_MAXN][GPK_MAXN];
  R gamma_abc[GPK_MAXN][GPK_MAXN][GPK_MAXN];
  R tau_ab[GPK_MAXN][GPK_MAXN];
  R dab16[GPK_MAXN][GPK_MAXN];
  R dab[GPK_MAXN][GPK_MAXN];
  R rot[GPK_MAXN][GPK_MAXN][2][2];
  R rinv[GPK_MAXN][GPK_MAXN][2][2];
  R cmu[GPK_MAXN][GPK_MAXK][GPK_MAXK];
  R E[GPK_MAXN][GPK_MAXK];
  R twoA[GPK_MAXN][GPK_MAXK];
  R A[GPK_MAXN][GPK_MAXK][GPK_MAXK];
  R B[GPK_MAXN][GPK_MAXK];
  R C[GPK_MAXN];
  R DC[GPK_MAXN][GPK_MAXK][GPK_MAXK][GPK_MAXK];
  R atf[GPK_MAXN][GPK_MAXK];
  R Dbulk[GPK_MAXN][GPK_MAXK][GPK_MAXK];
  double cmu64[GPK_MAXN][GPK_MAXK][GPK_MAXK];
  double muc64[GPK_MAXN][GPK_MAXK][GPK_MAXK];
  /* non-isothermal runs: E, B and C of a cell are functions of its
   * temperature (see gp_derived); FP64 whatever the field type */
  int tgrad;
  int bc_t[2];
  double Teq64;
  double Beq64[GPK_MAXN][GPK_MAXK], dBbdT64[GPK_MAXN][GPK_MAXK];
  double ceql[GPK_MAXN][GPK_MAXK], ceqs[GPK_MAXN][GPK_MAXK], DCk[GPK_MAXN][GPK_MAXK];
  double DTl[GPK_MAXN], DTs[GPK_MAXN];
  double A64[GPK_MAXN][GPK_MAXK][GPK_MAXK];
  double tg_base, tg_dT, tg_dist, tg_off, tg_vel, dx64, dy64, dt64;
  /* moving frame */
  int shift, shiftj;
  R mu_fill[GPK_MAXK];
};

/* h_a(phi) (functionH.h:24-36) */
template <typename R, int N>
__device__ __forceinline__ R h(const R *ph, int a) {
  R s1 = R(0.0);
  R s = R(3.0) * ph[a] * ph[a] - R(2.0) * ph[a] * ph[a] * ph[a];
#pragma unroll
  for (int b = 0; b < N; b++)
#pragma unroll
    for (int c = 0; c < N; c++)
      if (b != a && c != a && b < c) s1 += ph[b] * ph[c];
  s1 *= R(2.0) * ph[a];
  return s + s1;
}

/* d h_b / d phi_a (functionH.h:1-23, dhphi(phi, b, a)) */
template <typename R, int N>
__device__ __forceinline__ R dh(const R *ph, int b, int a) {
  R s = R(0.0);
  if (a == b) {
    s = R(6.0) * ph[a] * (R(1.0) - ph[a]);
#pragma unroll
    for (int e = 0; e < N; e++)
#pragma unroll
      for (int f = 0; f < N; f++)
        if (e != b && f != b && e < f) s += R(2.0) * ph[e] * ph[f];
  } else {
#pragma unroll
    for (int e = 0; e < N; e++)
      if (e != b && e != a) s += R(2.0) * ph[e];
    s *= ph[b];
  }
  return s;
}

/* c_a,i(mu) (functionF_01.h:30-37) */
template <typename R, int K>
__device__ __forceinline__ R c_mu(const Consts<R> &D, const R *m, int a, int i) {
  R s = R(0.0);
#pragma unroll
  for (int k = 0; k < K; k++) s += D.cmu[a][i][k] * (m[k] - D.E[a][k]);
  return s;
}

/* Mu_a,i(c) (functionF_01.h:19-29) */
template <typename R, int K>
__device__ __forceinline__ R Mu(const Consts<R> &D, const R *c, int a, int i) {
  R s = D.twoA[a][i] * c[i] + D.E[a][i];
#pragma unroll
  for (int j = 0; j < K; j++)
    if (i != j) s += D.A[a][i][j] * c[j];
  return s;
}

/* f_a(c) (functionF_01.h:5-18) */
template <typename R, int K>
__device__ __forceinline__ R fe(const Consts<R> &D, const R *c, int a) {
  R s = R(0.0);
#pragma unroll
  for (int i = 0; i < K; i++) {
#pragma unroll
    for (int j = 0; j < K; j++)
      if (i <= j) s += D.A[a][i][j] * c[i] * c[j];
    s += D.B[a][i] * c[i];
  }
  s += D.C[a];
  return s;
}

/* ---- the thermodynamics of a cell at its own temperature (non-isothermal
 * runs, where init_propertymatrices(T) runs per cell: calculate_divergence_
 * phasefield.h:21-29; c_mu and Mu take the cell's T: functionF_01.h:19-37) */

/* E_a,k = Beq + dBbdT (T - Teq) of every phase at temperature T */
template <typename R, int N, int K, typename CT>
__device__ __forceinline__ void e_at(const CT &D, double T, R (&E)[N][K]) {
#pragma unroll
  for (int a = 0; a < N; a++)
#pragma unroll
    for (int k = 0; k < K; k++) E[a][k] = (R)(D.Beq64[a][k] + D.dBbdT64[a][k] * (T - D.Teq64));
}

/* B and C of every phase at temperature T: function_B and function_C
 * (functionF_01.h:62-104), their expressions in their order */
template <typename R, int N, int K, typename CT>
__device__ __forceinline__ void bc_at(const CT &D, double T, R (&B)[N][K], R (&C)[N]) {
  constexpr int L = N - 1;
#pragma unroll
  for (int a = 0; a < N; a++) {
    double cl[K], cs[K];
#pragma unroll
    for (int i = 0; i < K; i++) {
      double sc = 0.0, bai = 0.0;
      if (a != L) {
#pragma unroll
        for (int k = 0; k < K; k++) {
          cl[k] = D.ceql[a][k] - (D.DCk[a][k]) * (D.Teq64 - T) / (D.DTl[a]);
          cs[k] = D.ceqs[a][k] - (D.DCk[a][k]) * (D.Teq64 - T) / (D.DTs[a]);
          if (k != i) sc += D.A64[L][k][i] * cl[k] - D.A64[a][k][i] * cs[k];
        }
        bai = (2.0 * (D.A64[L][i][i] * cl[i] - D.A64[a][i][i] * cs[i]) + sc);
      }
      B[a][i] = (R)bai;
    }
    double sc = 0.0;
    if (a != L) {
#pragma unroll
      for (int k = 0; k < K; k++) {
        cl[k] = D.ceql[a][k] - (D.DCk[a][k]) * (D.Teq64 - T) / (D.DTl[a]);
        cs[k] = D.ceqs[a][k] - (D.DCk[a][k]) * (D.Teq64 - T) / (D.DTs[a]);
      }
#pragma unroll
      for (int i = 0; i < K; i++)
#pragma unroll
        for (int j = 0; j < K; j++)
          if (i <= j) sc += (D.A64[a][i][j] * cs[i] * cs[j] - D.A64[L][i][j] * cl[i] * cl[j]);
    }
    C[a] = (R)sc;
  }
}

/* c_a,i(mu), Mu_a,i(c) and f_a(c) with the phase's E (and B, C) given */
template <typename R, int K, typename CT>
__device__ __forceinline__ R c_muE(const CT &D, const R *E, const R *m, int a, int i) {
  R s = R(0.0);
#pragma unroll
  for (int k = 0; k < K; k++) s += D.cmu[a][i][k] * (m[k] - E[k]);
  return s;
}
template <typename R, int K, typename CT>
__device__ __forceinline__ R MuE(const CT &D, const R *E, const R *c, int a, int i) {
  R s = D.twoA[a][i] * c[i] + E[i];
#pragma unroll
  for (int j = 0; j < K; j++)
    if (i != j) s += D.A[a][i][j] * c[j];
  return s;
}
template <typename R, int K, typename CT>
__device__ __forceinline__ R feBC(const CT &D, const R *B, R C, const R *c, int a) {
  R s = R(0.0);
#pragma unroll
  for (int i = 0; i < K; i++) {
#pragma unroll
    for (int j = 0; j < K; j++)
      if (i <= j) s += D.A[a][i][j] * c[i] * c[j];
    s += B[i] * c[i];
  }
  s += C;
  return s;
}

/* FunctionTau (functionTau.h:1-17) */
template <typename R, int N>
__device__ __forceinline__ R tau_of(const Consts<R> &D, const R *ph) {
  R s = R(0.0), s1 = R(0.0);
#pragma unroll
  for (int a = 0; a < N; a++)
#pragma unroll
    for (int b = 0; b < N; b++)
      if (a < b) {
        s += D.tau_ab[a][b] * ph[a] * ph[b];
        s1 += ph[a] * ph[b];
      }
  if (s1 != R(0.0)) return s / s1;
  return D.tau;
}

/* D_ij of one cell (functionD.h:1-16); DC = Diffusivity*cmu folded on the host */
template <typename R, int N, int K>
__device__ __forceinline__ R Dcell(const Consts<R> &D, const R *ph, int i, int j) {
  R s = R(0.0);
#pragma unroll
  for (int b = 0; b < N; b++)
#pragma unroll
    for (int k = 0; k < K; k++) s += D.DC[b][i][j][k] * ph[b];
  return s;
}

/* dw/dphi_a, obstacle (functionW_01.h:6-39) or well (functionW_02.h:4-33);
 * smooth selects the _smooth variants (no sign test, other association). */
template <typename R, int N>
__device__ __forceinline__ R dwdphi(const Consts<R> &D, const R *ph, const bool *act, int a, bool smooth) {
  R s = R(0.0);
#pragma unroll
  for (int b = 0; b < N; b++) {
    if (b == a || !act[b]) continue;
    if (D.well) {
      s += R(2.0) * D.gamma[a][b] * (ph[b] * ph[b] * ph[a]);
    } else if (smooth) {
      s += D.gamma[a][b] * ph[b];
    } else {
      if ((ph[a] * ph[b]) >= R(0.00000)) s += D.gamma[a][b] * (ph[b]);
      else s += -D.gamma[a][b] * (ph[b]);
    }
  }
  if (D.well) s *= R(9.0);
  else s *= D.c16pi2;
#pragma unroll
  for (int b = 0; b < N; b++)
#pragma unroll
    for (int c = 0; c < N; c++)
      if (b != a && c != a && b < c && act[b] && act[c]) {
        if (smooth) {
          s += D.gamma_abc[a][b][c] * ph[b] * ph[c];
        } else {
          R bc = ph[b] * ph[c];
          if (ph[a] * bc >= R(0.00000)) s += D.gamma_abc[a][b][c] * bc;
          else s += -D.gamma_abc[a][b][c] * bc;
        }
      }
  return s;
}

/* projection_on_simplex (simplex_projection.h:1-49) */
template <typename R, int N>
__device__ __forceinline__ void project(const R *ph, const bool *act, R *d) {
  R Dphi = R(0.0), sum_phib = R(0.0);
  long count = 0;
#pragma unroll
  for (int a = 0; a < N; a++)
    if (act[a] && (ph[a] + d[a]) > R(0.0) && (ph[a] + d[a]) < R(1.0)) {
      count++;
      sum_phib += ph[a];
    }
#pragma unroll
  for (int a = 0; a < N; a++)
    if ((ph[a] + d[a]) < R(0.0)) {
      R da = fabs(d[a] + ph[a]);
      d[a] += da;
      Dphi += da;
    }
  if (Dphi > R(0.0)) {
#pragma unroll
    for (int b = 0; b < N; b++)
      if (act[b] && ((ph[b] + d[b]) > R(0.0)) && ((ph[b] + d[b]) < R(1.0))) {
        if (fabs(sum_phib) > R(0.0)) d[b] -= Dphi * (ph[b]) / (sum_phib);
        else d[b] -= Dphi / (R)(count);
      }
  }
  int hit = -1;
#pragma unroll
  for (int a = 0; a < N; a++)
    if (hit < 0 && act[a] && (ph[a] + d[a]) > R(1.0)) hit = a;
  if (hit >= 0) {
    d[hit] = (R(1.0) - ph[hit]);
#pragma unroll
    for (int b = 0; b < N; b++)
      if (act[b] && b != hit) d[b] = -ph[b];
  }
}

/* projection_on_simplex_without_weights (simplex_projection.h:50-91) */
template <typename R, int N>
__device__ __forceinline__ void project_nw(const R *ph, const bool *act, R *d) {
  long count = 0;
#pragma unroll
  for (int a = 0; a < N; a++)
    if (act[a] && (ph[a] + d[a]) > R(0.0) && (ph[a] + d[a]) < R(1.0)) count++;
  bool done = false;
#pragma unroll
  for (int a = 0; a < N; a++) {
    if (done || !act[a]) continue;
    if ((ph[a] + d[a]) > R(1.0)) {
      d[a] = (R(1.0) - ph[a]);
#pragma unroll
      for (int b = 0; b < N; b++)
        if (act[b] && b != a) d[b] = -ph[b];
      done = true;
      continue;
    }
    if ((ph[a] + d[a]) < R(0.0)) {
      R Dphi = fabs(d[a] + ph[a]);
      d[a] += Dphi;
#pragma unroll
      for (int b = 0; b < N; b++)
        if ((act[b] && b != a) && (ph[b] + d[b]) > R(0.0) && (ph[b] + d[b]) < R(1.0)) d[b] -= Dphi / (R)(count);
    }
  }
}

/* multiply(M, q, out, 2) (matrix.h:10-20); the identity case reduces to q+0.0
 * bit for bit (the leading 0.0 turns -0 into +0, the other term adds +-0). */
template <typename R>
__device__ __forceinline__ void rot2(const Consts<R> &D, const R (&M)[2][2], R q0, R q1, R &r0, R &r1) {
  if (D.rot_identity) {
    r0 = q0 + R(0.0);
    r1 = q1 + R(0.0);
  } else {
    R s = R(0);
    s = s + M[0][0] * q0;
    s = s + M[0][1] * q1;
    r0 = s;
    s = R(0);
    s = s + M[1][0] * q0;
    s = s + M[1][1] * q1;
    r1 = s;
  }
}

/* Anisotropy functions.  For FP64 fields the expressions are exactly the
 * reference's.  The FP32 form evaluates them in float on the normalised
 * gradient (below): written as the reference writes them, |q|^6 of a gradient
 * just above the reference's |q|^2 > 1e-15 guard is about 1e-45 and
 * underflows in float, which turns dA/dq into inf or NaN. */

/* anisotropy_01_function_ac (anisotropy_01.h:30-48), q_z = 0 */
template <typename R>
__device__ __forceinline__ R ac(R qx_, R qy_, R dab) {
  const double qx = qx_, qy = qy_;
  double qx2 = qx * qx, qx4 = qx2 * qx2, qy2 = qy * qy, qy4 = qy2 * qy2;
  double qz2 = 0.0 * 0.0, qz4 = qz2 * qz2;
  double q2 = qx2 + qy2 + qz2;
  if (fabs(q2) > 1.0e-15) return (R)(1.0 - (double)dab * (3.0 - 4.0 * (qx4 + qy4 + qz4) / (q2 * q2)));
  return R(1.0);
}

/* one component of anisotropy_01_dAdq (anisotropy_01.h:9-29), q_z = 0:
 * 16*dab*(q_i^3/|q|^4 - q_i*sum q^4/|q|^6) */
template <typename R>
struct QPow {
  double q2, q22, q23, q4;
};
template <typename R>
__device__ __forceinline__ QPow<R> qpow(R qx_, R qy_) {
  const double qx = qx_, qy = qy_;
  QPow<R> r;
  double qx3 = qx * qx * qx, qy3 = qy * qy * qy, qz3 = 0.0;
  r.q2 = qx * qx + qy * qy + 0.0 * 0.0;
  r.q22 = r.q2 * r.q2;
  r.q23 = r.q2 * r.q2 * r.q2;
  r.q4 = qx3 * qx + qy3 * qy + qz3 * 0.0;
  return r;
}
template <typename R>
__device__ __forceinline__ R dadq_c(R qi_, const QPow<R> &p, R dab16) {
  const double qi = qi_;
  if (fabs(p.q2) > 1.0e-15) return (R)((double)dab16 * (qi * qi * qi / p.q22 - qi * p.q4 / p.q23));
  return R(0.0);
}

/* The FP32 form: with r2 = 1/|q|^2 and s4 = sum q^4 r2^2 (the sum of the
 * fourth powers of the unit vector q/|q|, between 1/2 and 1),
 *   a_c   = 1 - dab (3 - 4 s4),
 *   dA/dq_i = 16 dab (q_i r2) (q_i^2 r2 - s4),
 * the same functions as above, with no intermediate below about 1e-30. */
template <>
struct QPow<float> {
  float q2, r2, s4;
};
template <>
__device__ __forceinline__ QPow<float> qpow<float>(float qx, float qy) {
  QPow<float> r;
  r.q2 = qx * qx + qy * qy;
  r.r2 = r.q2 > 0.0f ? 1.0f / r.q2 : 0.0f;
  const float nx = qx * qx * r.r2, ny = qy * qy * r.r2;
  r.s4 = nx * nx + ny * ny;
  return r;
}
template <>
__device__ __forceinline__ float dadq_c<float>(float qi, const QPow<float> &p, float dab16) {
  if (fabsf(p.q2) > 1.0e-15f) return dab16 * (qi * p.r2) * (qi * qi * p.r2 - p.s4);
  return 0.0f;
}
template <>
__device__ __forceinline__ float ac<float>(float qx, float qy, float dab) {
  const QPow<float> p = qpow<float>(qx, qy);
  if (fabsf(p.q2) > 1.0e-15f) return 1.0f - dab * (3.0f - 4.0f * p.s4);
  return 1.0f;
}

/* matinvnew (matrix.h:50-218) for n = K <= 2 with 1.0/x as the reciprocal
 * (pow(x,-1) of the host library cannot be reproduced on the device; the
 * reference uses it only in the smoothing sweeps and for K>2 without
 * BINARY/TERNARY/DILUTE). */
template <typename T, int K>
__device__ __forceinline__ void matinv_div(T (&m)[K][K], T (&inv)[K][K]) {
  T fac[K][K], inv1[K][K], v1[K], v[K];
  int tag[K];
#pragma unroll
  for (int i = 0; i < K; i++) {
    tag[i] = i;
#pragma unroll
    for (int j = 0; j < K; j++) fac[i][j] = T(0.0);
  }
#pragma unroll
  for (int k = 0; k < K; k++) {
    T big = fabs(m[k][k]);
    int t1 = k;
#pragma unroll
    for (int i = k + 1; i < K; i++)
      if (fabs(m[i][k]) > big) { t1 = i; big = m[i][k]; }
    if (t1 != k) {
      int s = tag[k]; tag[k] = tag[t1]; tag[t1] = s;
#pragma unroll
      for (int i = 0; i < K; i++) { T w = m[k][i]; m[k][i] = m[t1][i]; m[t1][i] = w; }
#pragma unroll
      for (int i = 0; i < k; i++) { T w = fac[k][i]; fac[k][i] = fac[t1][i]; fac[t1][i] = w; }
    }
#pragma unroll
    for (int i = k + 1; i < K; i++) {
      T f = -m[i][k] / m[k][k];
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
    v1[0] = (i == 0) ? T(1.0) : T(0.0);
#pragma unroll
    for (int r = 1; r < K; r++) {
      T s = 0;
#pragma unroll
      for (int j = 0; j < r; j++) s = s - fac[r][j] * v1[j];
      v1[r] = ((r == i) ? T(1.0) : T(0.0)) + s;
    }
    v[K - 1] = v1[K - 1] * (T(1.0) / m[K - 1][K - 1]);
#pragma unroll
    for (int r = K - 2; r >= 0; r--) {
      T s = 0;
#pragma unroll
      for (int j = r + 1; j < K; j++) s = s - m[r][j] * v[j];
      v[r] = (v1[r] + s) * (T(1.0) / m[r][r]);
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
