/*
 * gp_step64.cuh -- plain FP64 step kernels (the drop-in for the reference's
 * solverloop_phasefield / solverloop_concentration / smooth).
 *
 * Data layout in HBM: one plane per field (phi_a, mu_k), interior cells only,
 * row x, column y contiguous, row pitch a multiple of 32 doubles.  The
 * reference's three ghost layers are never stored: after every boundary copy a
 * ghost cell holds an interior cell, so loads map ghost coordinates through the
 * copy tables (remap) instead.  delta-phi lives in its own buffer over the
 * interior plus a one-cell ring, because the anti-trapping flux at a boundary
 * face reads delta-phi computed at the ghost cell beyond it
 * (calculate_fluxes_concentration.h:93,135 read gridinfo[right/front].deltaphi).
 *
 * Kernel k_dphi (phase-field pass) and k_update (concentration pass) each work
 * on TX x TY tiles staged in shared memory.  Quantities that belong to a cell
 * face (anisotropy of every phase pair, anti-trapping flux, diffusion flux) are
 * computed once per face into shared memory and used by both cells of the face;
 * the reference evaluates every face from both sides and every anisotropy term
 * twice.  Pair (b,a) reuses the work of pair (a,b): its rotated q and dA/dq are
 * 0.0 minus those of (a,b) bit for bit (rotation results are never -0, and
 * negation is exact).
 */
#pragma once
#include "gp_math.cuh"

namespace gpd {

constexpr int TX = 8;    /* rows per tile    */
constexpr int TY = 32;   /* columns per tile */
constexpr int NT = TX * TY;
constexpr int SW = TY + 2, SH = TX + 2, SS = SW * SH;
constexpr int NXF = (TX + 1) * TY;       /* x-faces of a tile */
constexpr int NYF = TX * (TY + 1);       /* y-faces of a tile */

struct Grid {
  int mx, my;            /* interior size */
  int pitch;             /* row pitch of state planes (elements) */
  long long plane;       /* elements per state plane */
  int dpitch;            /* row pitch of the delta-phi buffer */
  long long dplane;      /* elements per delta-phi plane ((mx+2) rows) */
  int dx_pow2, dy_pow2;  /* division by dx/dy is an exact multiply */
  double inv_dx, inv_dy, inv_2dy;
};

/* interior coordinate v in [-3, m+2] -> interior coordinate it is a copy of
 * (assign_buffer_points_conditions / assign_boundary_points_values,
 * utility_functions.h:471-654): Neumann mirrors about the boundary cell,
 * periodic wraps with period m-1. */
__device__ __forceinline__ int remap(int v, int m, int tlo, int thi) {
  int g = v + 3, r = m + 6, src = g;
  if (g < 3) {
    int j = 2 - g;
    src = (tlo == GP_BC_NEUMANN) ? 4 + j : r - 5 - j;
  } else if (g >= r - 3) {
    int j = g - (r - 3);
    src = (thi == GP_BC_NEUMANN) ? r - 5 - j : 4 + j;
  }
  return src - 3;
}

__device__ __forceinline__ double divx(double v, const Grid &g) { return g.dx_pow2 ? v * g.inv_dx : v / cD.dx; }
__device__ __forceinline__ double divy(double v, const Grid &g) { return g.dy_pow2 ? v * g.inv_dy : v / cD.dy; }
__device__ __forceinline__ double div2y(double v, const Grid &g) { return g.dy_pow2 ? v * g.inv_2dy : v / (2.0 * cD.dy); }

/* pair index of a<b among N phases */
template <int N>
__device__ __forceinline__ constexpr int pidx(int a, int b) {
  return a * N - a * (a + 1) / 2 + (b - a - 1);
}
template <int N>
struct NP { static constexpr int v = N * (N - 1) / 2; };

/* ------------------------------------------------------------------ */
/* phase-field pass                                                    */
/* ------------------------------------------------------------------ */

template <int N>
struct DphiSmem {
  double S[N][SS];                                   /* phi tile with a 1-cell halo */
  double T[NP<N>::v > 0 ? NP<N>::v : 1][4][NXF + NYF]; /* face terms: T1ab, T1ba, T2ab, T2ba */
};

/* Load the phi tile whose local (i,j) is interior (x0-1+i, y0-1+j); entries
 * outside [-2, m+1] are not needed by any valid cell and are zeroed. */
/* Source row offsets and columns of a tile's SH staged rows and SW staged
 * columns after the boundary remap, one field; -1 where the row/column lies
 * outside [lo, hi] (not needed by any valid cell).  Filled by threads
 * 0..SH+SW-1; the caller synchronises before use. */
struct RemapTab {
  int row[SH], col[SW];
};
__device__ __forceinline__ void remap_tab(RemapTab &t, const Grid &g, int x0, int y0, int field, int lo_x,
                                          int hi_x, int lo_y, int hi_y) {
  const int u = threadIdx.x;
  if (u < SH) {
    const int x = x0 - 1 + u;
    t.row[u] = (x >= lo_x && x <= hi_x) ? remap(x, g.mx, cD.bc_x[field][0], cD.bc_x[field][1]) * g.pitch : -1;
  } else if (u < SH + SW) {
    const int y = y0 - 1 + (u - SH);
    t.col[u - SH] = (y >= lo_y && y <= hi_y) ? remap(y, g.my, cD.bc_y[field][0], cD.bc_y[field][1]) : -1;
  }
}

template <int NF>
__device__ __forceinline__ void load_tile(double (*S)[SS], const double *__restrict__ f, const Grid &g,
                                          const RemapTab &t) {
  for (int e = threadIdx.x; e < SS; e += NT) {
    const int i = e / SW, j = e - i * SW;
    const int r = t.row[i], cc = t.col[j];
    if (r >= 0 && cc >= 0) {
      const double *src = f + (r + cc);
#pragma unroll
      for (int a = 0; a < NF; a++) S[a][e] = __ldg(src + a * g.plane);
    } else {
#pragma unroll
      for (int a = 0; a < NF; a++) S[a][e] = 0.0;
    }
  }
}

#define LI(i, j) ((i) * SW + (j))

/* anisotropy terms of one face for all pairs.  xface: face between local
 * (i,j) and (i+1,j); else between (i,j) and (i,j+1).  Follows q_divx/q_divy
 * (functionQ.h:4-40), function_ac, dAdq (anisotropy_01.h) and the divergence
 * sums of function_A_01_divdAdgradphi (function_A_01.h:163-215). */
template <int N>
__device__ __forceinline__ void face_terms(DphiSmem<N> &sm, bool xface, int i, int j, int fidx, const Grid &g) {
  double s[N], gr[N], c0[N], c1[N];
#pragma unroll
  for (int a = 0; a < N; a++) {
    const double *S = sm.S[a];
    if (xface) {
      double p0 = S[LI(i, j)], p1 = S[LI(i + 1, j)];
      s[a] = 0.5 * (p1 + p0);
      gr[a] = divx(p1 - p0, g);
      c0[a] = div2y(S[LI(i, j + 1)] - S[LI(i, j - 1)], g);
      c1[a] = div2y(S[LI(i + 1, j + 1)] - S[LI(i + 1, j - 1)], g);
    } else {
      double p0 = S[LI(i, j)], p1 = S[LI(i, j + 1)];
      s[a] = 0.5 * (p1 + p0);
      gr[a] = divy(p1 - p0, g);
      c0[a] = 0.5 * (divx(S[LI(i + 1, j)] - S[LI(i, j)], g) + divx(S[LI(i, j)] - S[LI(i - 1, j)], g));
      c1[a] = 0.5 * (divx(S[LI(i + 1, j + 1)] - S[LI(i, j + 1)], g) + divx(S[LI(i, j + 1)] - S[LI(i - 1, j + 1)], g));
    }
  }
#pragma unroll
  for (int a = 0; a < N; a++)
#pragma unroll
    for (int b = a + 1; b < N; b++) {
      const int p = pidx<N>(a, b);
      double Pab = s[a] * gr[b] - s[b] * gr[a];
      double Pba = s[b] * gr[a] - s[a] * gr[b];
      double tq = 0.5 * (s[a] * (c0[b] + c1[b]) - s[b] * (c0[a] + c1[a]));
      double q0, q1;
      if (xface) rot2(cD.rot[a][b], Pab, tq, q0, q1);
      else rot2(cD.rot[a][b], tq, Pab, q0, q1);
      double acv = ac(q0, q1, cD.dab[a][b]);
      QPow qp = qpow(q0, q1);
      double rd;
      if (cD.rot_identity) {
        rd = (xface ? dadq_c(q0, qp, cD.dab16[a][b]) : dadq_c(q1, qp, cD.dab16[a][b])) + 0.0;
      } else {
        double d0 = dadq_c(q0, qp, cD.dab16[a][b]), d1 = dadq_c(q1, qp, cD.dab16[a][b]);
        double r0, r1;
        rot2(cD.rinv[a][b], d0, d1, r0, r1);
        rd = xface ? r0 : r1;
      }
      double ac2 = acv * acv, acq = acv * qp.q2;
      sm.T[p][0][fidx] = ac2 * Pab * (-s[b]);
      sm.T[p][1][fidx] = ac2 * Pba * (-s[a]);
      sm.T[p][2][fidx] = acq * rd * (-s[b]);
      sm.T[p][3][fidx] = acq * (0.0 - rd) * (-s[a]);
    }
}

/* delta-phi of the interior plus a one-cell ring (calculate_divergence_phasefield_2D,
 * calculate_divergence_phasefield.h:4-62).  Grid: x tiles over rows -1..mx,
 * y tiles over columns -1..my. */
template <int N, int K, bool ANISO>
__global__ void __launch_bounds__(NT) k_dphi(const double *__restrict__ phi, const double *__restrict__ mu,
                                             double *__restrict__ dphi, Grid g) {
  extern __shared__ __align__(16) unsigned char smraw[];
  DphiSmem<N> &sm = *reinterpret_cast<DphiSmem<N> *>(smraw);
  const int x0 = blockIdx.y * TX - 1, y0 = blockIdx.x * TY - 1;
  __shared__ RemapTab rt;
  remap_tab(rt, g, x0, y0, 0, -2, g.mx + 1, -2, g.my + 1);
  __syncthreads();
  load_tile<N>(sm.S, phi, g, rt);
  __syncthreads();

  const int tx = threadIdx.x / TY, ty = threadIdx.x - (threadIdx.x / TY) * TY;
  const int x = x0 + tx, y = y0 + ty, i = tx + 1, j = ty + 1;
  const bool valid = (x <= g.mx) && (y <= g.my);
  double ph[N], dv[N];
  bool act[N];
  bool anyact = false;
#pragma unroll
  for (int a = 0; a < N; a++) {
    const double *S = sm.S[a];
    ph[a] = S[LI(i, j)];
    double gxf = divx(S[LI(i + 1, j)] - S[LI(i, j)], g), gxb = divx(S[LI(i, j)] - S[LI(i - 1, j)], g);
    double gyr = divy(S[LI(i, j + 1)] - S[LI(i, j)], g), gyl = divy(S[LI(i, j)] - S[LI(i, j - 1)], g);
    dv[a] = divx(gxf - gxb, g);
    dv[a] += divy(gyr - gyl, g);
    act[a] = fabs(dv[a]) > 0.0;
    anyact |= act[a];
  }
  anyact = anyact && valid;
  const bool blockact = __syncthreads_or(anyact);

  if (ANISO && blockact) {
    for (int e = threadIdx.x; e < NXF + NYF; e += NT) {
      if (e < NXF) {
        int fi = e / TY, fj = e - fi * TY + 1;
        face_terms<N>(sm, true, fi, fj, e, g);
      } else {
        int f = e - NXF;
        int fi = f / (TY + 1) + 1, fj = f - (fi - 1) * (TY + 1);
        face_terms<N>(sm, false, fi, fj, e, g);
      }
    }
  }
  __syncthreads();
  if (!valid) return;

  double d[N];
  if (!anyact) {
    /* no active phase: delta-phi is 0 except where the simplex projection lifts
     * a negative phi back to 0 (simplex_projection.h:16-22) */
#pragma unroll
    for (int a = 0; a < N; a++) {
      d[a] = 0.0;
      if ((ph[a] + d[a]) < 0.0) d[a] += fabs(d[a] + ph[a]);
    }
  } else {
    double m[K];
    const int sxm = remap(x, g.mx, cD.bc_x[1][0], cD.bc_x[1][1]);
    const int sym = remap(y, g.my, cD.bc_y[1][0], cD.bc_y[1][1]);
#pragma unroll
    for (int k = 0; k < K; k++) m[k] = __ldg(mu + k * g.plane + (long long)sxm * g.pitch + sym);
    /* centred gradients of the cell */
    double gcx[N], gcy[N];
#pragma unroll
    for (int a = 0; a < N; a++) {
      const double *S = sm.S[a];
      gcx[a] = 0.5 * (divx(S[LI(i + 1, j)] - S[LI(i, j)], g) + divx(S[LI(i, j)] - S[LI(i - 1, j)], g));
      gcy[a] = div2y(S[LI(i, j + 1)] - S[LI(i, j - 1)], g);
    }
    /* psi_b (functionF_01.h:41-57): independent of the phase differentiated */
    double psi[N];
#pragma unroll
    for (int b = 0; b < N; b++) {
      double c[K], ps = 0.0;
#pragma unroll
      for (int k = 0; k < K; k++) {
        c[k] = c_mu<K>(m, b, k);
        ps -= m[k] * c[k];
      }
      ps += fe<K>(c, b);
      psi[b] = ps;
    }
    /* centre anisotropy per unordered pair (function_A_01_dAdphi, function_A_01.h:4-71) */
    double cq0[NP<N>::v > 0 ? NP<N>::v : 1], cq1[NP<N>::v > 0 ? NP<N>::v : 1];
    double cd0[NP<N>::v > 0 ? NP<N>::v : 1], cd1[NP<N>::v > 0 ? NP<N>::v : 1];
    double cac[NP<N>::v > 0 ? NP<N>::v : 1], cq2[NP<N>::v > 0 ? NP<N>::v : 1];
    if (ANISO) {
#pragma unroll
      for (int a = 0; a < N; a++)
#pragma unroll
        for (int b = a + 1; b < N; b++) {
          const int p = pidx<N>(a, b);
          double q0, q1;
          rot2(cD.rot[a][b], (ph[a] * gcx[b] - ph[b] * gcx[a]), (ph[a] * gcy[b] - ph[b] * gcy[a]), q0, q1);
          QPow qp = qpow(q0, q1);
          cq0[p] = q0;
          cq1[p] = q1;
          cd0[p] = dadq_c(q0, qp, cD.dab16[a][b]);
          cd1[p] = dadq_c(q1, qp, cD.dab16[a][b]);
          cq2[p] = (q0 * q0 + q1 * q1 + 0.0 * 0.0);
          cac[p] = ac(q0, q1, cD.dab[a][b]);
        }
    }
    const double tau = tau_of<N>(ph);
    double lam[N], sl = 0.0;
    long nact = 0;
#pragma unroll
    for (int a = 0; a < N; a++) {
      if (!act[a]) continue;
      double dA, div;
      if (ANISO) {
        double s1 = 0.0, s2 = 0.0, t1 = 0.0, t2 = 0.0;
#pragma unroll
        for (int b = 0; b < N; b++) {
          if (b == a) continue;
          const int p = a < b ? pidx<N>(a, b) : pidx<N>(b, a);
          const double sg = 0.0;
          double q0 = a < b ? cq0[p] : sg - cq0[p], q1 = a < b ? cq1[p] : sg - cq1[p];
          double d0 = a < b ? cd0[p] : sg - cd0[p], d1 = a < b ? cd1[p] : sg - cd1[p];
          double w0, w1;
          rot2(cD.rot[a][b], gcx[b], gcy[b], w0, w1);
          double sp1 = 0.0, sp2 = 0.0;
          sp1 += q0 * w0;
          sp1 += q1 * w1;
          sp2 += (d0) * w0;
          sp2 += (d1) * w1;
          sp1 *= cD.gamma[a][b] * (cac[p] * cac[p]);
          sp2 *= cD.gamma[a][b] * cac[p] * cq2[p];
          s1 += sp1;
          s2 += sp2;
          /* divergence terms from the face cache */
          const int o = a < b ? 0 : 1;
          const int xf = (i) * TY + (j - 1), xb = (i - 1) * TY + (j - 1);
          const int yr = NXF + (i - 1) * (TY + 1) + j, yl = NXF + (i - 1) * (TY + 1) + (j - 1);
          double d1v = divx((sm.T[p][o][xf]) - (sm.T[p][o][xb]), g);
          d1v += divy((sm.T[p][o][yr]) - (sm.T[p][o][yl]), g);
          d1v *= cD.gamma[a][b];
          t1 += d1v;
          double d2v = divx(sm.T[p][2 + o][xf] - sm.T[p][2 + o][xb], g);
          d2v += divy(sm.T[p][2 + o][yr] - sm.T[p][2 + o][yl], g);
          d2v *= cD.gamma[a][b];
          t2 += d2v;
        }
        dA = 2.0 * (s1 + s2);
        div = (2.0 * (t1 + t2) + 0.0);
      } else {
        /* function_A_00 (function_A_00.h:4-58) */
        double s = 0.0, t = 0.0;
        const double *Sa = sm.S[a];
#pragma unroll
        for (int b = 0; b < N; b++) {
          if (b == a) continue;
          const double *Sb = sm.S[b];
          double sp = 0.0;
          sp += (ph[a] * gcx[b] - ph[b] * gcx[a]) * gcx[b];
          sp += (ph[a] * gcy[b] - ph[b] * gcy[a]) * gcy[b];
          sp *= cD.gamma[a][b];
          s += sp;
          /* staggered values and one-sided gradients of the four faces */
          double pa = Sa[LI(i, j)], pb = Sb[LI(i, j)];
          double sxa = 0.5 * (Sa[LI(i + 1, j)] + pa), sxb = 0.5 * (Sb[LI(i + 1, j)] + pb);
          double gxa = divx(Sa[LI(i + 1, j)] - pa, g), gxb = divx(Sb[LI(i + 1, j)] - pb, g);
          double bxa = 0.5 * (pa + Sa[LI(i - 1, j)]), bxb = 0.5 * (pb + Sb[LI(i - 1, j)]);
          double hxa = divx(pa - Sa[LI(i - 1, j)], g), hxb = divx(pb - Sb[LI(i - 1, j)], g);
          double sya = 0.5 * (Sa[LI(i, j + 1)] + pa), syb = 0.5 * (Sb[LI(i, j + 1)] + pb);
          double gya = divy(Sa[LI(i, j + 1)] - pa, g), gyb = divy(Sb[LI(i, j + 1)] - pb, g);
          double lya = 0.5 * (pa + Sa[LI(i, j - 1)]), lyb = 0.5 * (pb + Sb[LI(i, j - 1)]);
          double hya = divy(pa - Sa[LI(i, j - 1)], g), hyb = divy(pb - Sb[LI(i, j - 1)], g);
          double dvg = divx((sxa * gxb - sxb * gxa) * (-sxb) - ((bxa * hxb - bxb * hxa) * (-bxb)), g);
          dvg += divy((sya * gyb - syb * gya) * (-syb) - ((lya * hyb - lyb * hya) * (-lyb)), g);
          dvg *= cD.gamma[a][b];
          t += dvg;
        }
        dA = 2.0 * s;
        div = 2.0 * t;
      }
      double dpsi = 0.0;
#pragma unroll
      for (int b = 0; b < N; b++) dpsi += psi[b] * dh<N>(ph, b, a);
      lam[a] = cD.eps * (-dA + div) - cD.inv_eps * dwdphi<N>(ph, act, a, false) - dpsi;
      sl += lam[a];
      nact++;
    }
    if (nact) sl /= (double)nact;
#pragma unroll
    for (int a = 0; a < N; a++) d[a] = act[a] ? cD.dt * (lam[a] - sl) / (tau * cD.eps) : 0.0;
    project<N>(ph, act, d);
  }
  const long long o = (long long)(x + 1) * g.dpitch + (y + 1);
#pragma unroll
  for (int a = 0; a < N; a++) dphi[a * g.dplane + o] = d[a];
}

/* ------------------------------------------------------------------ */
/* concentration pass                                                  */
/* ------------------------------------------------------------------ */

template <int N, int K>
struct UpdSmem {
  double P[N][SS], M[K][SS], DP[N][SS];
  double CM[N][K][SS];     /* c_a,k(mu) per cell */
  double H[N][SS];         /* h_a(phi) per cell */
  double SP[N][SS];        /* s_phi of the obstacle anti-trapping (solid phases) */
  double DD[K][K][SS];     /* D_kl per cell */
  double JX[K][NXF], JY[K][NYF];
  double FX[K][K][NXF], FY[K][K][NYF];
};

/* Block-wide reduction helpers (deterministic order). */
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

/* total order on doubles as signed 64-bit integers, for atomic max/min */
__device__ __forceinline__ long long ord(double v) {
  long long i = __double_as_longlong(v);
  return i < 0 ? i ^ 0x7fffffffffffffffLL : i;
}

struct StatBufs {
  long long *ext;      /* per-block running extremes [blocks][2*(N+K)] (ordered ints), or NULL */
  double *partials;    /* [blocks][2N+2K+1] sums when want_sums */
  int want_sums;
};

/* Per-block running extremes and (on request) sums of the cells a block owns.
 * Each block owns its slots, so no atomics are needed and results are
 * deterministic; gp_step folds the slots when it reports. */
/* UNI: every valid cell of the block holds the same phi (uniform tile), so
 * the phi extremes are thread 0's values and only mu is reduced. */
template <int N, int K, bool UNI = false>
__device__ __forceinline__ void block_stats(bool valid, const double *nph, const double *nm, const double *dp,
                                            const double *dmu, const StatBufs &st) {
  constexpr int NE = 2 * (N + K), NS = 2 * N + 2 * K + 1, NW = NT / 32;
  __shared__ double red[NW][NE > NS ? NE : NS];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const long long blk = (long long)blockIdx.y * gridDim.x + blockIdx.x;
  if (st.ext) {
#pragma unroll
    for (int f = 0; f < NE; f++) {
      const int fld = f >> 1;
      const bool isMax = !(f & 1);
      if (UNI && fld < N) {
        if (threadIdx.x == 0) red[0][f] = nph[fld];
        continue;
      }
      double v = isMax ? -INFINITY : INFINITY;
      if (valid) {
        double w = fld < N ? nph[fld] : nm[fld - N];
        if (w == w) v = w;
      }
      v = isMax ? warp_max(v) : warp_min(v);
      if (lane == 0) red[wid][f] = v;
    }
    __syncthreads();
    if (threadIdx.x < NE) {
      const int f = threadIdx.x, fld = f >> 1;
      const bool isMax = !(f & 1);
      double r = red[0][f];
      if (!(UNI && fld < N))
        for (int w = 1; w < NW; w++) r = isMax ? fmax(r, red[w][f]) : fmin(r, red[w][f]);
      /* slot layout: max phi[N], min phi[N], max mu[K], min mu[K] */
      const int slot = fld < N ? (isMax ? fld : N + fld) : (isMax ? 2 * N + (fld - N) : 2 * N + K + (fld - N));
      long long *p = st.ext + blk * NE + slot;
      if (isMax && r > -INFINITY && ord(r) > *p) *p = ord(r);
      if (!isMax && r < INFINITY && ord(r) < *p) *p = ord(r);
    }
    __syncthreads();
  }
  if (st.want_sums) {
    for (int f = 0; f < NS; f++) {
      double v = 0.0;
      if (valid) {
        if (f < N) v = dp[f] * dp[f];
        else if (f < N + K) v = dmu[f - N] * dmu[f - N];
        else if (f < 2 * N + K) v = nph[f - N - K];
        else if (f < 2 * N + 2 * K) {
          int k = f - 2 * N - K;
          double comp = 0.0;
#pragma unroll
          for (int b = 0; b < N; b++) comp += c_mu<K>(nm, b, k) * h<N>(nph, b);
          v = comp;
        } else {
          bool bad = false;
#pragma unroll
          for (int a = 0; a < N; a++) bad |= !isfinite(nph[a]);
#pragma unroll
          for (int k = 0; k < K; k++) bad |= !isfinite(nm[k]);
          v = bad ? 1.0 : 0.0;
        }
      }
      v = warp_sum(v);
      if (lane == 0) red[wid][f] = v;
    }
    __syncthreads();
    if (threadIdx.x < NS) {
      double r = 0.0;
      for (int w = 0; w < NW; w++) r += red[w][threadIdx.x];
      st.partials[blk * NS + threadIdx.x] = r;
    }
  }
}

/* mu update and phi commit of the interior
 * (calculate_fluxes_concentration_2D + calculate_divergence_concentration_2D,
 * calculate_fluxes_concentration.h:4-145, calculate_divergence_concentration.h:4-153). */
template <int N, int K>
__global__ void __launch_bounds__(NT) k_update(const double *__restrict__ phi, const double *__restrict__ mu,
                                               const double *__restrict__ dphi, double *__restrict__ phin,
                                               double *__restrict__ mun, Grid g, StatBufs st) {
  extern __shared__ __align__(16) unsigned char smraw[];
  UpdSmem<N, K> &sm = *reinterpret_cast<UpdSmem<N, K> *>(smraw);
  const int x0 = blockIdx.y * TX, y0 = blockIdx.x * TY;
  constexpr int L = N - 1;
  const double cst = cD.obstacle ? cD.jat_obst : cD.jat_well;

  /* A tile whose staged cells (in the domain) all hold the same one-hot phi
   * and no delta-phi has no interface in reach: every anti-trapping current is
   * 0.0 (all gradients vanish, calculate_fluxes_concentration.h:64,103), every
   * cell takes the bulk branch, and D is the same everywhere.  The fast path
   * evaluates exactly the expressions of the general path that remain.  The
   * reference cell is the tile's first cell (x0, y0), always in the domain. */
  double refp[N];
  int ref_phase = -1;
  {
    int ones = 0, zeros = 0;
#pragma unroll
    for (int a = 0; a < N; a++) {
      refp[a] = __ldg(phi + a * g.plane + (long long)x0 * g.pitch + y0);
      if (refp[a] == 1.0) { if (ref_phase < 0) ref_phase = a; ones++; }
      else if (refp[a] == 0.0) zeros++;
    }
    if (!(ones == 1 && zeros == N - 1)) ref_phase = -1;
  }

  /* stage phi, mu (remapped) and delta-phi; check uniformity on the way */
  __shared__ RemapTab rtp, rtm;
  remap_tab(rtp, g, x0, y0, 0, -1, g.mx, -1, g.my);
  remap_tab(rtm, g, x0, y0, 1, -1, g.mx, -1, g.my);
  __syncthreads();
  bool uni = ref_phase >= 0;
  for (int e = threadIdx.x; e < SS; e += NT) {
    const int i = e / SW, j = e - i * SW;
    const int rp = rtp.row[i], cp = rtp.col[j];
    if (rp >= 0 && cp >= 0) {
      const double *sp_ = phi + (rp + cp), *sm_ = mu + (rtm.row[i] + rtm.col[j]);
      const double *sd_ = dphi + ((long long)(x0 + i) * g.dpitch + (y0 + j));
#pragma unroll
      for (int a = 0; a < N; a++) {
        const double pv = __ldg(sp_ + a * g.plane), dv = __ldg(sd_ + a * g.dplane);
        sm.P[a][e] = pv;
        sm.DP[a][e] = dv;
        uni = uni && pv == refp[a] && dv == 0.0;
      }
#pragma unroll
      for (int k = 0; k < K; k++) sm.M[k][e] = __ldg(sm_ + k * g.plane);
    } else {
#pragma unroll
      for (int a = 0; a < N; a++) { sm.P[a][e] = 0.0; sm.DP[a][e] = 0.0; }
#pragma unroll
      for (int k = 0; k < K; k++) sm.M[k][e] = 0.0;
    }
  }
  const bool uniform = __syncthreads_and(uni);

  const int tx = threadIdx.x / TY, ty = threadIdx.x - (threadIdx.x / TY) * TY;
  const int x = x0 + tx, y = y0 + ty, i = tx + 1, j = ty + 1, c = LI(i, j);
  const bool valid = x < g.mx && y < g.my;
  double ph[N], m[K], dp[N], nph[N], nm[K], dmu[K];

  if (uniform) {
    if (valid) {
#pragma unroll
      for (int a = 0; a < N; a++) { ph[a] = sm.P[a][c]; dp[a] = sm.DP[a][c]; }
#pragma unroll
      for (int k = 0; k < K; k++) m[k] = sm.M[k][c];
      double Dv[K][K];
#pragma unroll
      for (int k = 0; k < K; k++)
#pragma unroll
        for (int l = 0; l < K; l++) Dv[k][l] = cD.Dbulk[ref_phase][k][l];   /* == Dcell(ph) */
      double cn[K];
#pragma unroll
      for (int k = 0; k < K; k++) {
        double divflux = 0.0;
#pragma unroll
        for (int l = 0; l < K; l++) {
          const double *M = sm.M[l];
          const double dm = (Dv[k][l] + Dv[k][l]) * 0.5;
          double fx = dm * divx(M[LI(i + 1, j)] - M[c], g), bx = dm * divx(M[c] - M[LI(i - 1, j)], g);
          double fy = dm * divy(M[LI(i, j + 1)] - M[c], g), by = dm * divy(M[c] - M[LI(i, j - 1)], g);
          divflux += divx(fx - bx, g);
          divflux += divy(fy - by, g);
        }
        double divjat = divx((0.0 - 0.0) * cst, g);
        divjat += divy((0.0 - 0.0) * cst, g);
        cn[k] = c_mu<K>(m, ref_phase, k) + cD.dt * (divflux) - divjat;
      }
#pragma unroll
      for (int k = 0; k < K; k++) {
        nm[k] = Mu<K>(cn, ref_phase, k);
        dmu[k] = nm[k] - m[k];
      }
#pragma unroll
      for (int a = 0; a < N; a++) nph[a] = ph[a] + dp[a];
      const long long o = (long long)x * g.pitch + y;
#pragma unroll
      for (int a = 0; a < N; a++) phin[a * g.plane + o] = nph[a];
#pragma unroll
      for (int k = 0; k < K; k++) mun[k * g.plane + o] = nm[k];
    }
    block_stats<N, K, true>(valid, nph, nm, dp, dmu, st);
    return;
  }

  /* general path: per-cell quantities */
  for (int e = threadIdx.x; e < SS; e += NT) {
    double p[N], mm[K];
#pragma unroll
    for (int a = 0; a < N; a++) p[a] = sm.P[a][e];
#pragma unroll
    for (int k = 0; k < K; k++) mm[k] = sm.M[k][e];
#pragma unroll
    for (int a = 0; a < N; a++) {
      double hv = h<N>(p, a);
      sm.H[a][e] = hv;
#pragma unroll
      for (int k = 0; k < K; k++) sm.CM[a][k][e] = c_mu<K>(mm, a, k);
      if (a < L)
        sm.SP[a][e] = (p[a] * (1.0 - p[a]) > 0.0) ? p[a] * (1.0 - hv) / (sqrt(p[a] * (1.0 - p[a]))) : 0.0;
    }
#pragma unroll
    for (int k = 0; k < K; k++)
#pragma unroll
      for (int l = 0; l < K; l++) sm.DD[k][l][e] = Dcell<N, K>(p, k, l);
  }
  __syncthreads();

  /* faces: anti-trapping current and diffusion flux products */
  for (int e = threadIdx.x; e < NXF + NYF; e += NT) {
    const bool xface = e < NXF;
    int fi, fj, i1, j1, fidx;
    if (xface) { fi = e / TY; fj = e - fi * TY + 1; i1 = fi + 1; j1 = fj; fidx = e; }
    else { int f = e - NXF; fi = f / (TY + 1) + 1; fj = f - (fi - 1) * (TY + 1); i1 = fi; j1 = fj + 1; fidx = f; }
    const int c0 = LI(fi, fj), c1 = LI(i1, j1);
    double gr[N], cn[N];   /* one-sided gradient across the face, mean of the centred tangential gradient */
#pragma unroll
    for (int a = 0; a < N; a++) {
      const double *S = sm.P[a];
      if (xface) {
        gr[a] = divx(S[c1] - S[c0], g);
        cn[a] = 0.5 * (div2y(S[LI(fi, fj + 1)] - S[LI(fi, fj - 1)], g) + div2y(S[LI(i1, fj + 1)] - S[LI(i1, fj - 1)], g));
      } else {
        gr[a] = divy(S[c1] - S[c0], g);
        double gc0 = 0.5 * (divx(S[LI(fi + 1, fj)] - S[c0], g) + divx(S[c0] - S[LI(fi - 1, fj)], g));
        double gc1 = 0.5 * (divx(S[LI(fi + 1, j1)] - S[c1], g) + divx(S[c1] - S[LI(fi - 1, j1)], g));
        cn[a] = 0.5 * (gc0 + gc1);
      }
    }
    double jat[K];
#pragma unroll
    for (int k = 0; k < K; k++) jat[k] = 0.0;
    /* calculate_fluxes_concentration.h:65: no y-current where gidy is 0 or MESH_Y-2 */
    const bool yskip = !xface && ((y0 - 1 + fj) + 3 == g.my - 2);
    double nl = -1.0;   /* |grad phi_liquid| on the face, computed on first use */
#pragma unroll
    for (int a = 0; a < L; a++) {
      /* sqrt(s2) != 0 exactly when s2 != 0 (s2 >= 0, or NaN on both sides) */
      const double s2 = cn[a] * cn[a] + gr[a] * gr[a];
      if (s2 != 0.0 && !yskip) {
        const double ng = sqrt(s2);
        if (nl < 0.0) nl = sqrt(cn[L] * cn[L] + gr[L] * gr[L]);
        double sp = gr[a] * gr[L];
        sp += cn[a] * cn[L];
        if (nl > 0.0) sp /= (nl * ng);
#pragma unroll
        for (int k = 0; k < K; k++) {
          double cl1 = sm.CM[L][k][c1], cl0 = sm.CM[L][k][c0];
          double cs1 = sm.CM[a][k][c1], cs0 = sm.CM[a][k][c0];
          double bracket;
          if (cD.obstacle)
            bracket = sm.SP[a][c1] * (cl1 - cs1) * sm.DP[a][c1] + sm.SP[a][c0] * (cl0 - cs0) * sm.DP[a][c0];
          else
            bracket = (cl1 - cs1) * sm.DP[a][c1] + (cl0 - cs0) * sm.DP[a][c0];
          jat[k] += cD.atf[a][k] * fabs(sp) * (cD.obstacle ? 0.5 : cD.well_half) * bracket * gr[a] / ng;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < K; k++) {
      if (xface) sm.JX[k][fidx] = jat[k];
      else sm.JY[k][fidx] = jat[k];
#pragma unroll
      for (int l = 0; l < K; l++) {
        double dm = (sm.DD[k][l][c1] + sm.DD[k][l][c0]) * 0.5;
        double gm = xface ? divx(sm.M[l][c1] - sm.M[l][c0], g) : divy(sm.M[l][c1] - sm.M[l][c0], g);
        if (xface) sm.FX[k][l][fidx] = dm * gm;
        else sm.FY[k][l][fidx] = dm * gm;
      }
    }
  }
  __syncthreads();

  if (valid) {
#pragma unroll
    for (int a = 0; a < N; a++) { ph[a] = sm.P[a][c]; dp[a] = sm.DP[a][c]; }
#pragma unroll
    for (int k = 0; k < K; k++) m[k] = sm.M[k][c];
    double divflux[K], divjat[K];
    const int xf = i * TY + (j - 1), xb = (i - 1) * TY + (j - 1);
    const int yr = (i - 1) * (TY + 1) + j, yl = (i - 1) * (TY + 1) + (j - 1);
#pragma unroll
    for (int k = 0; k < K; k++) {
      divflux[k] = 0.0;
#pragma unroll
      for (int l = 0; l < K; l++) {
        divflux[k] += divx(sm.FX[k][l][xf] - sm.FX[k][l][xb], g);
        divflux[k] += divy(sm.FY[k][l][yr] - sm.FY[k][l][yl], g);
      }
      divjat[k] = divx((sm.JX[k][xf] - sm.JX[k][xb]) * cst, g);
      divjat[k] += divy((sm.JY[k][yr] - sm.JY[k][yl]) * cst, g);
    }
    int bulk = -1;
#pragma unroll
    for (int a = 0; a < N; a++)
      if (bulk < 0 && ph[a] == 1.0) bulk = a;
    if (bulk >= 0) {
      double cn[K];
#pragma unroll
      for (int k = 0; k < K; k++) cn[k] = sm.CM[bulk][k][c] + cD.dt * (divflux[k]) - divjat[k];
#pragma unroll
      for (int k = 0; k < K; k++) {
        nm[k] = Mu<K>(cn, bulk, k);
        dmu[k] = nm[k] - m[k];
      }
    } else {
      /* sum_a c_a(mu) sum_b dh_a/dphi_b dphi_b (calculate_divergence_concentration.h:23-31) */
      double sum[K], dc[K], dcdmu[K][K];
#pragma unroll
      for (int k = 0; k < K; k++) sum[k] = 0.0;
#pragma unroll
      for (int a = 0; a < N; a++) {
        double sdh = 0.0;
#pragma unroll
        for (int b = 0; b < N; b++) sdh += dh<N>(ph, a, b) * dp[b];
#pragma unroll
        for (int k = 0; k < K; k++) sum[k] += sm.CM[a][k][c] * sdh;
      }
#pragma unroll
      for (int k = 0; k < K; k++) {
        dc[k] = cD.dt * (divflux[k]) - divjat[k] - sum[k];
#pragma unroll
        for (int l = 0; l < K; l++) {
          dcdmu[k][l] = 0.0;
#pragma unroll
          for (int a = 0; a < N; a++) dcdmu[k][l] += cD.cmu[a][k][l] * sm.H[a][c];
        }
      }
#pragma unroll
      for (int k = 0; k < K; k++) { nm[k] = m[k]; dmu[k] = 0.0; }
      if (cD.inv_mode == GP_INV_BINARY) {
        double i00 = 1.0 / dcdmu[0][0];
        dmu[0] = dc[0] * i00;
        nm[0] += dmu[0];
      } else if (cD.inv_mode == GP_INV_TERNARY && K == 2) {
        double det = dcdmu[0][0] * dcdmu[K - 1][K - 1] - dcdmu[0][K - 1] * dcdmu[K - 1][0];
        double iv[K][K];
        iv[0][0] = dcdmu[K - 1][K - 1] / det;
        iv[K - 1][K - 1] = dcdmu[0][0] / det;
        iv[0][K - 1] = -dcdmu[0][K - 1] / det;
        iv[K - 1][0] = -dcdmu[K - 1][0] / det;
#pragma unroll
        for (int k = 0; k < K; k++) {
          dmu[k] = 0.0;
#pragma unroll
          for (int l = 0; l < K; l++) dmu[k] += iv[k][l] * dc[l];
        }
#pragma unroll
        for (int k = 0; k < K; k++) nm[k] = dmu[k] + nm[k];
      } else if (cD.inv_mode == GP_INV_DILUTE) {
#pragma unroll
        for (int k = 0; k < K; k++) {
          double ikk = 1.0 / dcdmu[k][k];
          dmu[k] = dc[k] * ikk;
          nm[k] += dmu[k];
        }
      } else {
        double iv[K][K];
        matinv_div<K>(dcdmu, iv);
#pragma unroll
        for (int k = 0; k < K; k++) {
          double s = 0;
#pragma unroll
          for (int l = 0; l < K; l++) s = s + iv[k][l] * dc[l];
          dmu[k] = s;
        }
#pragma unroll
        for (int k = 0; k < K; k++) nm[k] = dmu[k] + nm[k];
      }
    }
#pragma unroll
    for (int a = 0; a < N; a++) nph[a] = ph[a] + dp[a];
    const long long o = (long long)x * g.pitch + y;
#pragma unroll
    for (int a = 0; a < N; a++) phin[a * g.plane + o] = nph[a];
#pragma unroll
    for (int k = 0; k < K; k++) mun[k * g.plane + o] = nm[k];
  }
  block_stats<N, K>(valid, nph, nm, dp, dmu, st);
}

}  // namespace gpd
