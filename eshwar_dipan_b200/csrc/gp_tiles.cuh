/*
 * gp_tiles.cuh -- the time-step kernels, generic in the field type R.
 *
 * Data layout in HBM: one plane per field (phi_a, mu_k), interior cells only,
 * row x, column y contiguous.  The reference's three ghost layers are never
 * stored: after every boundary copy a ghost cell holds an interior cell, so
 * loads map ghost coordinates through the copy tables (remap) instead.
 * delta-phi lives in its own buffer over the interior plus a one-cell ring,
 * because the anti-trapping flux at a boundary face reads delta-phi computed at
 * the ghost cell beyond it (calculate_fluxes_concentration.h:93,135 read
 * gridinfo[right/front].deltaphi).
 *
 * dphi_tile (phase-field pass) and update_tile (concentration pass) each work
 * on a TX x TY tile staged in shared memory.  Quantities that belong to a cell
 * face (anisotropy of every phase pair, anti-trapping current, diffusion flux)
 * are computed once per face and used by both cells of the face; the reference
 * evaluates every face from both sides and every anisotropy term twice.  Pair
 * (b,a) reuses the work of pair (a,b): its rotated q and dA/dq are 0.0 minus
 * those of (a,b) bit for bit (rotation results are never -0, negation is exact).
 *
 * dphi_tile / update_tile drive k_dphi / k_update (gp_device.cu), one CTA
 * per tile of one simulation with its constants in __constant__ memory: the
 * two-pass step of gp_step_noalloc.  The stepping engine of gp_ctx and
 * gp_batch is in gp_fused.cuh and shares this file's staging, face, commit
 * and statistics code.
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
  int sx0, sx1;          /* rows the progress statistics cover (a slab's own rows; all by default) */
};

/* rows moved by one gp_rows_pack / gp_rows_unpack call: item i is row
 * row[i] of state field field[i] */
constexpr int ROW_ITEMS_MAX = 64;
struct RowItems {
  int field[ROW_ITEMS_MAX];
  int row[ROW_ITEMS_MAX];
};

/* the cell's row is counted by the progress statistics */
__device__ __forceinline__ bool stat_row(const Grid &g, int x) { return x >= g.sx0 && x < g.sx1; }

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

template <typename R>
__device__ __forceinline__ R divx(R v, const Consts<R> &D) { return D.mul_dx ? v * D.inv_dx : v / D.dx; }
template <typename R>
__device__ __forceinline__ R divy(R v, const Consts<R> &D) { return D.mul_dy ? v * D.inv_dy : v / D.dy; }
template <typename R>
__device__ __forceinline__ R div2y(R v, const Consts<R> &D) { return D.mul_dy ? v * D.inv_2dy : v / (R(2.0) * D.dy); }

/* The same constants when every spacing is known to be a power of two (or
 * the field type is float): the divisions are multiplications by the exact
 * reciprocals and no division code is emitted.  Kernels view their Consts
 * through this type when the launch says so. */
template <typename R>
struct ConstsMul : Consts<R> {};
template <typename R>
__device__ __forceinline__ R divx(R v, const ConstsMul<R> &D) { return v * D.inv_dx; }
template <typename R>
__device__ __forceinline__ R divy(R v, const ConstsMul<R> &D) { return v * D.inv_dy; }
template <typename R>
__device__ __forceinline__ R div2y(R v, const ConstsMul<R> &D) { return v * D.inv_2dy; }

/* pair index of a<b among N phases */
template <int N>
__device__ __forceinline__ constexpr int pidx(int a, int b) {
  return a * N - a * (a + 1) / 2 + (b - a - 1);
}
template <int N>
struct NP { static constexpr int v = N * (N - 1) / 2 > 0 ? N * (N - 1) / 2 : 1; };

/* Source row offsets and columns of a tile's SH staged rows and SW staged
 * columns after the boundary remap, one field; -1 where the row/column lies
 * outside [lo, hi] (not needed by any valid cell).  Filled by threads
 * 0..SH+SW-1; the caller synchronises before use. */
struct RemapTab {
  int row[SH], col[SW];
};
template <typename R>
__device__ __forceinline__ void remap_tab(RemapTab &t, const Consts<R> &D, const Grid &g, int x0, int y0, int field,
                                          int lo_x, int hi_x, int lo_y, int hi_y) {
  const int u = threadIdx.x;
  if (u < SH) {
    const int x = x0 - 1 + u;
    t.row[u] = (x >= lo_x && x <= hi_x) ? remap(x, g.mx, D.bc_x[field][0], D.bc_x[field][1]) * g.pitch : -1;
  } else if (u < SH + SW) {
    const int y = y0 - 1 + (u - SH);
    t.col[u - SH] = (y >= lo_y && y <= hi_y) ? remap(y, g.my, D.bc_y[field][0], D.bc_y[field][1]) : -1;
  }
}

template <typename R, int NF>
__device__ __forceinline__ void load_tile(R (*S)[SS], const R *__restrict__ f, const Grid &g, const RemapTab &t) {
  for (int e = threadIdx.x; e < SS; e += NT) {
    const int i = e / SW, j = e - i * SW;
    const int r = t.row[i], cc = t.col[j];
    if (r >= 0 && cc >= 0) {
      const R *src = f + (r + cc);
#pragma unroll
      for (int a = 0; a < NF; a++) S[a][e] = __ldg(src + a * g.plane);
    } else {
#pragma unroll
      for (int a = 0; a < NF; a++) S[a][e] = R(0.0);
    }
  }
}

#define LI(i, j) ((i) * SW + (j))

/* ------------------------------------------------------------------ */
/* phase-field pass                                                    */
/* ------------------------------------------------------------------ */

template <typename R, int N>
struct DphiSmem {
  R S[N][SS];                      /* phi tile with a 1-cell halo */
  R T[NP<N>::v][4][NXF + NYF];     /* face terms: T1ab, T1ba, T2ab, T2ba */
  RemapTab rt;
};

/* anisotropy terms of one face for all pairs.  xface: face between local
 * (i,j) and (i+1,j); else between (i,j) and (i,j+1).  Follows q_divx/q_divy
 * (functionQ.h:4-40), function_ac, dAdq (anisotropy_01.h) and the divergence
 * sums of function_A_01_divdAdgradphi (function_A_01.h:163-215). */
template <typename R, int N>
__device__ __forceinline__ void face_terms(const Consts<R> &D, DphiSmem<R, N> &sm, bool xface, int i, int j,
                                           int fidx) {
  R s[N], gr[N], c0[N], c1[N];
#pragma unroll
  for (int a = 0; a < N; a++) {
    const R *S = sm.S[a];
    if (xface) {
      R p0 = S[LI(i, j)], p1 = S[LI(i + 1, j)];
      s[a] = R(0.5) * (p1 + p0);
      gr[a] = divx(p1 - p0, D);
      c0[a] = div2y(S[LI(i, j + 1)] - S[LI(i, j - 1)], D);
      c1[a] = div2y(S[LI(i + 1, j + 1)] - S[LI(i + 1, j - 1)], D);
    } else {
      R p0 = S[LI(i, j)], p1 = S[LI(i, j + 1)];
      s[a] = R(0.5) * (p1 + p0);
      gr[a] = divy(p1 - p0, D);
      c0[a] = R(0.5) * (divx(S[LI(i + 1, j)] - S[LI(i, j)], D) + divx(S[LI(i, j)] - S[LI(i - 1, j)], D));
      c1[a] = R(0.5) * (divx(S[LI(i + 1, j + 1)] - S[LI(i, j + 1)], D) + divx(S[LI(i, j + 1)] - S[LI(i - 1, j + 1)], D));
    }
  }
#pragma unroll
  for (int a = 0; a < N; a++)
#pragma unroll
    for (int b = a + 1; b < N; b++) {
      const int p = pidx<N>(a, b);
      R Pab = s[a] * gr[b] - s[b] * gr[a];
      R Pba = s[b] * gr[a] - s[a] * gr[b];
      R tq = R(0.5) * (s[a] * (c0[b] + c1[b]) - s[b] * (c0[a] + c1[a]));
      R q0, q1;
      if (xface) rot2(D, D.rot[a][b], Pab, tq, q0, q1);
      else rot2(D, D.rot[a][b], tq, Pab, q0, q1);
      R acv = ac(q0, q1, D.dab[a][b]);
      QPow<R> qp = qpow(q0, q1);
      R rd;
      if (D.rot_identity) {
        rd = (xface ? dadq_c(q0, qp, D.dab16[a][b]) : dadq_c(q1, qp, D.dab16[a][b])) + R(0.0);
      } else {
        R d0 = dadq_c(q0, qp, D.dab16[a][b]), d1 = dadq_c(q1, qp, D.dab16[a][b]);
        R r0, r1;
        rot2(D, D.rinv[a][b], d0, d1, r0, r1);
        rd = xface ? r0 : r1;
      }
      R ac2 = acv * acv, acq = acv * qp.q2;
      sm.T[p][0][fidx] = ac2 * Pab * (-s[b]);
      sm.T[p][1][fidx] = ac2 * Pba * (-s[a]);
      sm.T[p][2][fidx] = acq * rd * (-s[b]);
      sm.T[p][3][fidx] = acq * (R(0.0) - rd) * (-s[a]);
    }
}

/* delta-phi of one tile (calculate_divergence_phasefield_2D,
 * calculate_divergence_phasefield.h:4-62).  The tile's cells are interior
 * (x0+tx, y0+ty) for x in [-1, mx], y in [-1, my] (interior plus ring). */
template <typename R, int N, int K, bool ANISO>
__device__ __forceinline__ void dphi_tile(const Consts<R> &D, const Grid &g, const R *__restrict__ phi,
                                          const R *__restrict__ mu, R *__restrict__ dphi, int x0, int y0,
                                          DphiSmem<R, N> &sm) {
  remap_tab(sm.rt, D, g, x0, y0, 0, -2, g.mx + 1, -2, g.my + 1);
  __syncthreads();
  load_tile<R, N>(sm.S, phi, g, sm.rt);
  __syncthreads();

  const int tx = threadIdx.x / TY, ty = threadIdx.x - (threadIdx.x / TY) * TY;
  const int x = x0 + tx, y = y0 + ty, i = tx + 1, j = ty + 1;
  const bool valid = (x <= g.mx) && (y <= g.my);
  R ph[N], dv[N];
  bool act[N];
  bool anyact = false;
#pragma unroll
  for (int a = 0; a < N; a++) {
    const R *S = sm.S[a];
    ph[a] = S[LI(i, j)];
    R gxf = divx(S[LI(i + 1, j)] - S[LI(i, j)], D), gxb = divx(S[LI(i, j)] - S[LI(i - 1, j)], D);
    R gyr = divy(S[LI(i, j + 1)] - S[LI(i, j)], D), gyl = divy(S[LI(i, j)] - S[LI(i, j - 1)], D);
    dv[a] = divx(gxf - gxb, D);
    dv[a] += divy(gyr - gyl, D);
    act[a] = fabs(dv[a]) > R(0.0);
    anyact |= act[a];
  }
  anyact = anyact && valid;
  const bool blockact = __syncthreads_or(anyact);

  if (ANISO && blockact) {
    for (int e = threadIdx.x; e < NXF + NYF; e += NT) {
      if (e < NXF) {
        int fi = e / TY, fj = e - fi * TY + 1;
        face_terms<R, N>(D, sm, true, fi, fj, e);
      } else {
        int f = e - NXF;
        int fi = f / (TY + 1) + 1, fj = f - (fi - 1) * (TY + 1);
        face_terms<R, N>(D, sm, false, fi, fj, e);
      }
    }
  }
  __syncthreads();
  if (!valid) return;

  R d[N];
  if (!anyact) {
    /* no active phase: delta-phi is 0 except where the simplex projection lifts
     * a negative phi back to 0 (simplex_projection.h:16-22) */
#pragma unroll
    for (int a = 0; a < N; a++) {
      d[a] = R(0.0);
      if ((ph[a] + d[a]) < R(0.0)) d[a] += fabs(d[a] + ph[a]);
    }
  } else {
    R m[K];
    const int sxm = remap(x, g.mx, D.bc_x[1][0], D.bc_x[1][1]);
    const int sym = remap(y, g.my, D.bc_y[1][0], D.bc_y[1][1]);
#pragma unroll
    for (int k = 0; k < K; k++) m[k] = __ldg(mu + k * g.plane + (long long)sxm * g.pitch + sym);
    R gcx[N], gcy[N];
#pragma unroll
    for (int a = 0; a < N; a++) {
      const R *S = sm.S[a];
      gcx[a] = R(0.5) * (divx(S[LI(i + 1, j)] - S[LI(i, j)], D) + divx(S[LI(i, j)] - S[LI(i - 1, j)], D));
      gcy[a] = div2y(S[LI(i, j + 1)] - S[LI(i, j - 1)], D);
    }
    /* psi_b (functionF_01.h:41-57): independent of the phase differentiated */
    R psi[N];
#pragma unroll
    for (int b = 0; b < N; b++) {
      R c[K], ps = R(0.0);
#pragma unroll
      for (int k = 0; k < K; k++) {
        c[k] = c_mu<R, K>(D, m, b, k);
        ps -= m[k] * c[k];
      }
      ps += fe<R, K>(D, c, b);
      psi[b] = ps;
    }
    /* centre anisotropy per unordered pair (function_A_01_dAdphi, function_A_01.h:4-71) */
    R cq0[NP<N>::v], cq1[NP<N>::v], cd0[NP<N>::v], cd1[NP<N>::v], cac[NP<N>::v], cq2[NP<N>::v];
    if (ANISO) {
#pragma unroll
      for (int a = 0; a < N; a++)
#pragma unroll
        for (int b = a + 1; b < N; b++) {
          const int p = pidx<N>(a, b);
          R q0, q1;
          rot2(D, D.rot[a][b], (ph[a] * gcx[b] - ph[b] * gcx[a]), (ph[a] * gcy[b] - ph[b] * gcy[a]), q0, q1);
          QPow<R> qp = qpow(q0, q1);
          cq0[p] = q0;
          cq1[p] = q1;
          cd0[p] = dadq_c(q0, qp, D.dab16[a][b]);
          cd1[p] = dadq_c(q1, qp, D.dab16[a][b]);
          cq2[p] = (q0 * q0 + q1 * q1 + R(0.0) * R(0.0));
          cac[p] = ac(q0, q1, D.dab[a][b]);
        }
    }
    const R tau = tau_of<R, N>(D, ph);
    R lam[N], sl = R(0.0);
    long nact = 0;
#pragma unroll
    for (int a = 0; a < N; a++) {
      if (!act[a]) continue;
      R dA, div;
      if (ANISO) {
        R s1 = R(0.0), s2 = R(0.0), t1 = R(0.0), t2 = R(0.0);
#pragma unroll
        for (int b = 0; b < N; b++) {
          if (b == a) continue;
          const int p = a < b ? pidx<N>(a, b) : pidx<N>(b, a);
          const R sg = R(0.0);
          R q0 = a < b ? cq0[p] : sg - cq0[p], q1 = a < b ? cq1[p] : sg - cq1[p];
          R d0 = a < b ? cd0[p] : sg - cd0[p], d1 = a < b ? cd1[p] : sg - cd1[p];
          R w0, w1;
          rot2(D, D.rot[a][b], gcx[b], gcy[b], w0, w1);
          R sp1 = R(0.0), sp2 = R(0.0);
          sp1 += q0 * w0;
          sp1 += q1 * w1;
          sp2 += (d0) * w0;
          sp2 += (d1) * w1;
          sp1 *= D.gamma[a][b] * (cac[p] * cac[p]);
          sp2 *= D.gamma[a][b] * cac[p] * cq2[p];
          s1 += sp1;
          s2 += sp2;
          /* divergence terms from the face cache */
          const int o = a < b ? 0 : 1;
          const int xf = (i) * TY + (j - 1), xb = (i - 1) * TY + (j - 1);
          const int yr = NXF + (i - 1) * (TY + 1) + j, yl = NXF + (i - 1) * (TY + 1) + (j - 1);
          R d1v = divx((sm.T[p][o][xf]) - (sm.T[p][o][xb]), D);
          d1v += divy((sm.T[p][o][yr]) - (sm.T[p][o][yl]), D);
          d1v *= D.gamma[a][b];
          t1 += d1v;
          R d2v = divx(sm.T[p][2 + o][xf] - sm.T[p][2 + o][xb], D);
          d2v += divy(sm.T[p][2 + o][yr] - sm.T[p][2 + o][yl], D);
          d2v *= D.gamma[a][b];
          t2 += d2v;
        }
        dA = R(2.0) * (s1 + s2);
        div = (R(2.0) * (t1 + t2) + R(0.0));
      } else {
        /* function_A_00 (function_A_00.h:4-58) */
        R s = R(0.0), t = R(0.0);
        const R *Sa = sm.S[a];
#pragma unroll
        for (int b = 0; b < N; b++) {
          if (b == a) continue;
          const R *Sb = sm.S[b];
          R sp = R(0.0);
          sp += (ph[a] * gcx[b] - ph[b] * gcx[a]) * gcx[b];
          sp += (ph[a] * gcy[b] - ph[b] * gcy[a]) * gcy[b];
          sp *= D.gamma[a][b];
          s += sp;
          /* staggered values and one-sided gradients of the four faces */
          R pa = Sa[LI(i, j)], pb = Sb[LI(i, j)];
          R sxa = R(0.5) * (Sa[LI(i + 1, j)] + pa), sxb = R(0.5) * (Sb[LI(i + 1, j)] + pb);
          R gxa = divx(Sa[LI(i + 1, j)] - pa, D), gxb = divx(Sb[LI(i + 1, j)] - pb, D);
          R bxa = R(0.5) * (pa + Sa[LI(i - 1, j)]), bxb = R(0.5) * (pb + Sb[LI(i - 1, j)]);
          R hxa = divx(pa - Sa[LI(i - 1, j)], D), hxb = divx(pb - Sb[LI(i - 1, j)], D);
          R sya = R(0.5) * (Sa[LI(i, j + 1)] + pa), syb = R(0.5) * (Sb[LI(i, j + 1)] + pb);
          R gya = divy(Sa[LI(i, j + 1)] - pa, D), gyb = divy(Sb[LI(i, j + 1)] - pb, D);
          R lya = R(0.5) * (pa + Sa[LI(i, j - 1)]), lyb = R(0.5) * (pb + Sb[LI(i, j - 1)]);
          R hya = divy(pa - Sa[LI(i, j - 1)], D), hyb = divy(pb - Sb[LI(i, j - 1)], D);
          R dvg = divx((sxa * gxb - sxb * gxa) * (-sxb) - ((bxa * hxb - bxb * hxa) * (-bxb)), D);
          dvg += divy((sya * gyb - syb * gya) * (-syb) - ((lya * hyb - lyb * hya) * (-lyb)), D);
          dvg *= D.gamma[a][b];
          t += dvg;
        }
        dA = R(2.0) * s;
        div = R(2.0) * t;
      }
      R dpsi = R(0.0);
#pragma unroll
      for (int b = 0; b < N; b++) dpsi += psi[b] * dh<R, N>(ph, b, a);
      lam[a] = D.eps * (-dA + div) - D.inv_eps * dwdphi<R, N>(D, ph, act, a, false) - dpsi;
      sl += lam[a];
      nact++;
    }
    if (nact) sl /= (R)nact;
#pragma unroll
    for (int a = 0; a < N; a++) d[a] = act[a] ? D.dt * (lam[a] - sl) / (tau * D.eps) : R(0.0);
    project<R, N>(ph, act, d);
  }
  const long long o = (long long)(x + 1) * g.dpitch + (y + 1);
#pragma unroll
  for (int a = 0; a < N; a++) dphi[a * g.dplane + o] = d[a];
}

/* ------------------------------------------------------------------ */
/* concentration pass                                                  */
/* ------------------------------------------------------------------ */

template <typename R, int N, int K>
struct UpdSmem {
  R P[N][SS], M[K][SS], DP[N][SS];
  R CM[N][K][SS];     /* c_a,k(mu) per cell */
  R H[N][SS];         /* h_a(phi) per cell */
  R SP[N][SS];        /* s_phi of the obstacle anti-trapping (solid phases) */
  R DD[K][K][SS];     /* D_kl per cell */
  R JX[K][NXF], JY[K][NYF];
  R FX[K][K][NXF], FY[K][K][NYF];
  RemapTab rtp, rtm;
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

/* total order on doubles as signed 64-bit integers */
__device__ __forceinline__ long long ord(double v) {
  long long i = __double_as_longlong(v);
  return i < 0 ? i ^ 0x7fffffffffffffffLL : i;
}

struct StatBufs {
  long long *ext;      /* running extremes [simulations][2*(N+K)] (ordered ints, atomic max/min), or NULL */
  double *partials;    /* [tiles][2N+2K+1] sums when want_sums */
  int want_sums;
  const unsigned *round_step;  /* FP32 form: device step counter keying the rounding stream */
  int mbar_tries;      /* polls of a TMA box's barrier before kf_bulk gives up (MBAR_TRIES) */
  int bch_max, bch_div;  /* bulk chunks: at most bch_max (<= 16) entries, left / (bch_div * warps) */
  int mixed;           /* kf_step: odd CTAs take bulk tiles first, then interface tiles */
  const double *trows; /* non-isothermal simulations: per simulation the temperature of each ghosted column y
                          as the phase-field pass reads it, then as the concentration pass reads it */
  unsigned tma_extra;  /* bytes a box's barrier expects beyond the box: 0, or more to test the give-up path */
  double *dphi_out;    /* NULL, or (a batch of one) the step's delta-phi of every interface tile and its ring in
                          the delta-phi layout (Grid dpitch/dplane); cells no interface tile covers are left as
                          they are (their delta-phi is +0.0) */
};

/* ---- FP32 storage rounding ------------------------------------------------
 * The FP32 form adds each step's increment in FP64 and rounds the sum to float
 * stochastically: up with probability (distance to the float below) / ulp.
 * Round-to-nearest would drop every increment below half an ulp (a slowly
 * diffusing far field stops moving and solute is lost); stochastic rounding
 * keeps every stored value unbiased, so the solute-mass error is a random walk
 * of size ulp*sqrt(steps/cells) instead of a systematic drift.  The random
 * bits are a counter-based hash of (step, cell, field): deterministic, and the
 * same for a simulation alone or inside a batch.  Values exactly
 * representable in float (pure phases 0/1, unchanged cells) are stored as is. */
__device__ __forceinline__ unsigned mix32(unsigned v) {
  /* a 32-bit avalanche hash (xor-shift / multiply rounds) */
  v ^= v >> 16;
  v *= 0x7feb352du;
  v ^= v >> 15;
  v *= 0x846ca68bu;
  v ^= v >> 16;
  return v;
}

__device__ __forceinline__ unsigned round_key(unsigned step, int x, int y) {
  return mix32(mix32(step * 0x9e3779b9u + 0x632be5abu) ^ ((unsigned)x * 0x85ebca6bu + (unsigned)y * 0xc2b2ae35u));
}

__device__ __forceinline__ float round_stochastic(double v, unsigned key, int field) {
  const float lo = __double2float_rz(v);              /* toward zero */
  const double rem = v - (double)lo;                   /* exact, same sign as v */
  if (rem == 0.0) return lo;
  const float hi = __uint_as_float(__float_as_uint(lo) + 1u);  /* next float away from zero */
  const double span = (double)hi - (double)lo;
  const double u = (double)(mix32(key + (unsigned)field * 0x27d4eb2fu) >> 8) * 0x1p-24;
  return fabs(rem) > u * fabs(span) ? hi : lo;
}

/* a + b rounded to float stochastically without leaving float: TwoSum gives
 * the round-to-nearest sum s and the exact remainder e (s + e = a + b); the
 * neighbour t of s on the side of e is taken with probability |e| / |t - s|,
 * decided by the 16-bit uniform r16 (the probability is exact to 2^-16). */
__device__ __forceinline__ float add_stochastic(float a, float b, unsigned r16) {
  const float s = a + b;
  const float bb = s - a;
  const float e = (a - (s - bb)) + (b - bb);
  if (e == 0.0f) return s;
  const float t = nextafterf(s, e > 0.0f ? INFINITY : -INFINITY);
  const float u = (float)r16 * (1.0f / 65536.0f);
  return fabsf(e) > u * fabsf(t - s) ? t : s;
}

/* FP32 commit of a pure-phase cell: mu += muc_a * dc in FP64, phi += dphi,
 * both rounded stochastically. */
template <typename R, int N, int K>
__device__ __forceinline__ void bulk_commit_f32(const Consts<R> &D, int a, const R *dc, const R *ph, const R *dp,
                                                const R *m, R *nph, R *nm, double *dmu, unsigned key) {
#pragma unroll
  for (int k = 0; k < K; k++) {
    double s = 0.0;
#pragma unroll
    for (int l = 0; l < K; l++) s += D.muc64[a][k][l] * (double)dc[l];
    dmu[k] = s;
    nm[k] = (R)round_stochastic((double)m[k] + s, key, N + k);
  }
#pragma unroll
  for (int a2 = 0; a2 < N; a2++) nph[a2] = (R)round_stochastic((double)ph[a2] + (double)dp[a2], key, a2);
}

/* Running extremes and (on request) FP64 sums of the cells a tile owns.
 * Extremes go to the simulation's slots (ext_slot) by atomic max/min on the
 * ordered integer image (exact and order-free, so deterministic); the sums go
 * to the tile's own slot (sum_slot) and the host folds the slots in a fixed
 * order.  UNI: every valid cell of the tile holds the same phi (uniform tile),
 * so the phi extremes are thread 0's values and only mu is reduced. */
template <typename R, int N, int K, bool UNI = false>
__device__ __forceinline__ void block_stats(const Consts<R> &D, bool valid, const R *nph, const R *nm, const R *dp,
                                            const double *dmu, const StatBufs &st, long long ext_slot,
                                            long long sum_slot, double Tc = 0.0) {
  constexpr int NE = 2 * (N + K), NS = 2 * N + 2 * K + 1, NW = NT / 32;
  __shared__ double red[NW][NE > NS ? NE : NS];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (st.ext) {
#pragma unroll
    for (int f = 0; f < NE; f++) {
      const int fld = f >> 1;
      const bool isMax = !(f & 1);
      if (UNI && fld < N) {
        if (threadIdx.x == 0) red[0][f] = (double)nph[fld];
        continue;
      }
      double v = isMax ? -INFINITY : INFINITY;
      if (valid) {
        double w = fld < N ? (double)nph[fld] : (double)nm[fld - N];
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
      const int sl = fld < N ? (isMax ? fld : N + fld) : (isMax ? 2 * N + (fld - N) : 2 * N + K + (fld - N));
      long long *p = st.ext + ext_slot * NE + sl;
      if (isMax && r > -INFINITY) atomicMax(p, ord(r));
      if (!isMax && r < INFINITY) atomicMin(p, ord(r));
    }
    __syncthreads();
  }
  if (st.want_sums) {
    for (int f = 0; f < NS; f++) {
      double v = 0.0;
      if (valid) {
        if (f < N) v = (double)dp[f] * (double)dp[f];
        else if (f < N + K) v = dmu[f - N] * dmu[f - N];
        else if (f < 2 * N + K) v = (double)nph[f - N - K];
        else if (f < 2 * N + 2 * K) {
          int k = f - 2 * N - K;
          R comp = R(0.0);
#pragma unroll
          if (D.tgrad) {
            R E[N][K];
            e_at<R, N, K>(D, Tc, E);
#pragma unroll
            for (int b = 0; b < N; b++) comp += c_muE<R, K>(D, E[b], nm, b, k) * h<R, N>(nph, b);
          } else {
#pragma unroll
            for (int b = 0; b < N; b++) comp += c_mu<R, K>(D, nm, b, k) * h<R, N>(nph, b);
          }
          v = (double)comp;
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
      st.partials[sum_slot * NS + threadIdx.x] = r;
    }
    __syncthreads();
  }
}

/* mu update and phi commit of one tile cell from the tile's face fluxes
 * (calculate_divergence_concentration.h:24-140): divergences, then the bulk
 * branch (mu = Mu_a(c_a(mu) + dc)) or the interface branch (dmu = (dc/dmu)^-1 dc,
 * inverted in FP64), then phi += delta-phi.  i, j: the cell's position in the
 * one-cell-halo tile layout; x, y: its interior coordinates. */
template <typename R, int N, int K, typename CT>
__device__ __forceinline__ void commit_cell(const CT &D, const R (&FX)[K][K][NXF], const R (&FY)[K][K][NYF],
                                            const R (&JX)[K][NXF], const R (&JY)[K][NYF], const R (&CM)[N][K][SS],
                                            const R (&H)[N][SS], int i, int j, int x, int y, const R *ph,
                                            const R *dp, const R *m, R *nph, R *nm, double *dmu,
                                            const StatBufs &st, double Tc = 0.0) {
  const R cst = D.obstacle ? D.jat_obst : D.jat_well;
  const int c = LI(i, j);
  R divflux[K], divjat[K];
  const int xf = i * TY + (j - 1), xb = (i - 1) * TY + (j - 1);
  const int yr = (i - 1) * (TY + 1) + j, yl = (i - 1) * (TY + 1) + (j - 1);
#pragma unroll
  for (int k = 0; k < K; k++) {
    divflux[k] = R(0.0);
#pragma unroll
    for (int l = 0; l < K; l++) {
      divflux[k] += divx(FX[k][l][xf] - FX[k][l][xb], D);
      divflux[k] += divy(FY[k][l][yr] - FY[k][l][yl], D);
    }
    divjat[k] = divx((JX[k][xf] - JX[k][xb]) * cst, D);
    divjat[k] += divy((JY[k][yr] - JY[k][yl]) * cst, D);
  }
  int bulk = -1;
#pragma unroll
  for (int a = 0; a < N; a++)
    if (bulk < 0 && ph[a] == R(1.0)) bulk = a;
  if (bulk >= 0 && sizeof(R) == 4) {
    R cn[K];
#pragma unroll
    for (int k = 0; k < K; k++) cn[k] = D.dt * (divflux[k]) - divjat[k];
    bulk_commit_f32<R, N, K>(D, bulk, cn, ph, dp, m, nph, nm, dmu, round_key(__ldg(st.round_step), x, y));
  } else if (bulk >= 0) {
    R cn[K];
#pragma unroll
    for (int k = 0; k < K; k++) cn[k] = CM[bulk][k][c] + D.dt * (divflux[k]) - divjat[k];
    if (D.tgrad) {
      R E[N][K];
      e_at<R, N, K>(D, Tc, E);
#pragma unroll
      for (int k = 0; k < K; k++) {
        nm[k] = MuE<R, K>(D, E[bulk], cn, bulk, k);
        dmu[k] = (double)nm[k] - (double)m[k];
      }
    } else {
#pragma unroll
      for (int k = 0; k < K; k++) {
        nm[k] = Mu<R, K>(D, cn, bulk, k);
        dmu[k] = (double)nm[k] - (double)m[k];
      }
    }
#pragma unroll
    for (int a = 0; a < N; a++) nph[a] = ph[a] + dp[a];
  } else {
    /* sum_a c_a(mu) sum_b dh_a/dphi_b dphi_b (calculate_divergence_concentration.h:23-31) */
    R sum[K];
    double dc[K], dcdmu[K][K];
#pragma unroll
    for (int k = 0; k < K; k++) sum[k] = R(0.0);
#pragma unroll
    for (int a = 0; a < N; a++) {
      R sdh = R(0.0);
#pragma unroll
      for (int b = 0; b < N; b++) sdh += dh<R, N>(ph, a, b) * dp[b];
#pragma unroll
      for (int k = 0; k < K; k++) sum[k] += CM[a][k][c] * sdh;
    }
    /* non-isothermal (calculate_divergence_concentration.h:85): minus
     * sum_a dcbdT_phase h_a * dt * (-GRADIENT * velocity); dcbdT_phase is
     * allocated but never filled by the reference (taken as 0) and the struct
     * member GRADIENT is never set, so the term is a signed zero */
    R sdc = R(0.0);
    if (D.tgrad) {
#pragma unroll
      for (int a = 0; a < N; a++) sdc += R(0.0) * H[a][c];
    }
#pragma unroll
    for (int k = 0; k < K; k++) {
      if (D.tgrad) dc[k] = (double)(D.dt * (divflux[k]) - divjat[k] - sum[k] - sdc * D.dt * (R(-0.0) * (R)D.tg_vel));
      else dc[k] = (double)(D.dt * (divflux[k]) - divjat[k] - sum[k]);
#pragma unroll
      for (int l = 0; l < K; l++) {
        dcdmu[k][l] = 0.0;
#pragma unroll
        for (int a = 0; a < N; a++) dcdmu[k][l] += D.cmu64[a][k][l] * (double)H[a][c];
      }
    }
    double m64[K];
#pragma unroll
    for (int k = 0; k < K; k++) { m64[k] = (double)m[k]; dmu[k] = 0.0; }
    if (D.inv_mode == GP_INV_BINARY) {
      double i00 = 1.0 / dcdmu[0][0];
      dmu[0] = dc[0] * i00;
      m64[0] += dmu[0];
    } else if (D.inv_mode == GP_INV_TERNARY && K == 2) {
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
      for (int k = 0; k < K; k++) m64[k] = dmu[k] + m64[k];
    } else if (D.inv_mode == GP_INV_DILUTE) {
#pragma unroll
      for (int k = 0; k < K; k++) {
        double ikk = 1.0 / dcdmu[k][k];
        dmu[k] = dc[k] * ikk;
        m64[k] += dmu[k];
      }
    } else {
      double iv[K][K];
      matinv_div<double, K>(dcdmu, iv);
#pragma unroll
      for (int k = 0; k < K; k++) {
        double s = 0;
#pragma unroll
        for (int l = 0; l < K; l++) s = s + iv[k][l] * dc[l];
        dmu[k] = s;
      }
#pragma unroll
      for (int k = 0; k < K; k++) m64[k] = dmu[k] + m64[k];
    }
    if constexpr (sizeof(R) == 8) {
#pragma unroll
      for (int k = 0; k < K; k++) nm[k] = (R)m64[k];
#pragma unroll
      for (int a = 0; a < N; a++) nph[a] = ph[a] + dp[a];
    } else {
      const unsigned key = round_key(__ldg(st.round_step), x, y);
#pragma unroll
      for (int k = 0; k < K; k++) nm[k] = round_stochastic(m64[k], key, N + k);
#pragma unroll
      for (int a = 0; a < N; a++) nph[a] = round_stochastic((double)ph[a] + (double)dp[a], key, a);
    }
  }
}

/* mu update and phi commit of one interior tile
 * (calculate_fluxes_concentration_2D + calculate_divergence_concentration_2D,
 * calculate_fluxes_concentration.h:4-145, calculate_divergence_concentration.h:4-153).
 * The dc/dmu inversion is done in FP64 for both field types. */
template <typename R, int N, int K>
__device__ __forceinline__ void update_tile(const Consts<R> &D, const Grid &g, const R *__restrict__ phi,
                                            const R *__restrict__ mu, const R *__restrict__ dphi,
                                            R *__restrict__ phin, R *__restrict__ mun, int x0, int y0,
                                            const StatBufs &st, long long slot, UpdSmem<R, N, K> &sm) {
  constexpr int L = N - 1;
  const R cst = D.obstacle ? D.jat_obst : D.jat_well;

  /* A tile whose staged cells (in the domain) all hold the same one-hot phi
   * and no delta-phi has no interface in reach: every anti-trapping current is
   * 0.0 (all gradients vanish, calculate_fluxes_concentration.h:64,103), every
   * cell takes the bulk branch, and D is the same everywhere.  The fast path
   * evaluates exactly the expressions of the general path that remain.  The
   * reference cell is the tile's first cell (x0, y0), always in the domain. */
  R refp[N];
  int ref_phase = -1;
  {
    int ones = 0, zeros = 0;
#pragma unroll
    for (int a = 0; a < N; a++) {
      refp[a] = __ldg(phi + a * g.plane + (long long)x0 * g.pitch + y0);
      if (refp[a] == R(1.0)) { if (ref_phase < 0) ref_phase = a; ones++; }
      else if (refp[a] == R(0.0)) zeros++;
    }
    if (!(ones == 1 && zeros == N - 1)) ref_phase = -1;
  }

  /* stage phi, mu (remapped) and delta-phi; check uniformity on the way */
  remap_tab(sm.rtp, D, g, x0, y0, 0, -1, g.mx, -1, g.my);
  remap_tab(sm.rtm, D, g, x0, y0, 1, -1, g.mx, -1, g.my);
  __syncthreads();
  bool uni = ref_phase >= 0;
  for (int e = threadIdx.x; e < SS; e += NT) {
    const int i = e / SW, j = e - i * SW;
    const int rp = sm.rtp.row[i], cp = sm.rtp.col[j];
    if (rp >= 0 && cp >= 0) {
      const R *sp_ = phi + (rp + cp), *sm_ = mu + (sm.rtm.row[i] + sm.rtm.col[j]);
      const R *sd_ = dphi + ((long long)(x0 + i) * g.dpitch + (y0 + j));
#pragma unroll
      for (int a = 0; a < N; a++) {
        const R pv = __ldg(sp_ + a * g.plane), dv = __ldg(sd_ + a * g.dplane);
        sm.P[a][e] = pv;
        sm.DP[a][e] = dv;
        uni = uni && pv == refp[a] && dv == R(0.0);
      }
#pragma unroll
      for (int k = 0; k < K; k++) sm.M[k][e] = __ldg(sm_ + k * g.plane);
    } else {
#pragma unroll
      for (int a = 0; a < N; a++) { sm.P[a][e] = R(0.0); sm.DP[a][e] = R(0.0); }
#pragma unroll
      for (int k = 0; k < K; k++) sm.M[k][e] = R(0.0);
    }
  }
  const bool uniform = __syncthreads_and(uni);

  const int tx = threadIdx.x / TY, ty = threadIdx.x - (threadIdx.x / TY) * TY;
  const int x = x0 + tx, y = y0 + ty, i = tx + 1, j = ty + 1, c = LI(i, j);
  const bool valid = x < g.mx && y < g.my;
  R ph[N], m[K], dp[N], nph[N], nm[K];
  double dmu[K];

  if (uniform) {
    if (valid) {
#pragma unroll
      for (int a = 0; a < N; a++) { ph[a] = sm.P[a][c]; dp[a] = sm.DP[a][c]; }
#pragma unroll
      for (int k = 0; k < K; k++) m[k] = sm.M[k][c];
      R cn[K];
#pragma unroll
      for (int k = 0; k < K; k++) {
        R divflux = R(0.0);
#pragma unroll
        for (int l = 0; l < K; l++) {
          const R *M = sm.M[l];
          const R Dv = D.Dbulk[ref_phase][k][l];   /* == Dcell(ph) */
          const R dm = (Dv + Dv) * R(0.5);
          R fx = dm * divx(M[LI(i + 1, j)] - M[c], D), bx = dm * divx(M[c] - M[LI(i - 1, j)], D);
          R fy = dm * divy(M[LI(i, j + 1)] - M[c], D), by = dm * divy(M[c] - M[LI(i, j - 1)], D);
          divflux += divx(fx - bx, D);
          divflux += divy(fy - by, D);
        }
        R divjat = divx((R(0.0) - R(0.0)) * cst, D);
        divjat += divy((R(0.0) - R(0.0)) * cst, D);
        if constexpr (sizeof(R) == 8) cn[k] = c_mu<R, K>(D, m, ref_phase, k) + D.dt * (divflux) - divjat;
        else cn[k] = D.dt * divflux - divjat;   /* FP32: the composition increment */
      }
      if constexpr (sizeof(R) == 8) {
#pragma unroll
        for (int k = 0; k < K; k++) {
          nm[k] = Mu<R, K>(D, cn, ref_phase, k);
          dmu[k] = (double)nm[k] - (double)m[k];
        }
#pragma unroll
        for (int a = 0; a < N; a++) nph[a] = ph[a] + dp[a];
      } else {
        /* mu += (dmu/dc) dc of the pure phase, in FP64: the same update as
         * Mu(c(mu) + dc) without the float c -> mu round trip, whose matrix
         * product is not exactly the identity and would drift every step */
        bulk_commit_f32<R, N, K>(D, ref_phase, cn, ph, dp, m, nph, nm, dmu, round_key(__ldg(st.round_step), x, y));
      }
      const long long o = (long long)x * g.pitch + y;
#pragma unroll
      for (int a = 0; a < N; a++) phin[a * g.plane + o] = nph[a];
#pragma unroll
      for (int k = 0; k < K; k++) mun[k * g.plane + o] = nm[k];
    }
    block_stats<R, N, K, true>(D, valid && stat_row(g, x), nph, nm, dp, dmu, st, 0, slot);
    return;
  }

  /* general path: per-cell quantities */
  for (int e = threadIdx.x; e < SS; e += NT) {
    R p[N], mm[K];
#pragma unroll
    for (int a = 0; a < N; a++) p[a] = sm.P[a][e];
#pragma unroll
    for (int k = 0; k < K; k++) mm[k] = sm.M[k][e];
#pragma unroll
    for (int a = 0; a < N; a++) {
      R hv = h<R, N>(p, a);
      sm.H[a][e] = hv;
#pragma unroll
      for (int k = 0; k < K; k++) sm.CM[a][k][e] = c_mu<R, K>(D, mm, a, k);
      if (a < L)
        sm.SP[a][e] = (p[a] * (R(1.0) - p[a]) > R(0.0)) ? p[a] * (R(1.0) - hv) / (sqrt(p[a] * (R(1.0) - p[a]))) : R(0.0);
    }
#pragma unroll
    for (int k = 0; k < K; k++)
#pragma unroll
      for (int l = 0; l < K; l++) sm.DD[k][l][e] = Dcell<R, N, K>(D, p, k, l);
  }
  __syncthreads();

  /* faces: anti-trapping current and diffusion flux products */
  for (int e = threadIdx.x; e < NXF + NYF; e += NT) {
    const bool xface = e < NXF;
    int fi, fj, i1, j1, fidx;
    if (xface) { fi = e / TY; fj = e - fi * TY + 1; i1 = fi + 1; j1 = fj; fidx = e; }
    else { int f = e - NXF; fi = f / (TY + 1) + 1; fj = f - (fi - 1) * (TY + 1); i1 = fi; j1 = fj + 1; fidx = f; }
    const int c0 = LI(fi, fj), c1 = LI(i1, j1);
    R gr[N], cn[N];   /* one-sided gradient across the face, mean of the centred tangential gradient */
#pragma unroll
    for (int a = 0; a < N; a++) {
      const R *S = sm.P[a];
      if (xface) {
        gr[a] = divx(S[c1] - S[c0], D);
        cn[a] = R(0.5) * (div2y(S[LI(fi, fj + 1)] - S[LI(fi, fj - 1)], D) + div2y(S[LI(i1, fj + 1)] - S[LI(i1, fj - 1)], D));
      } else {
        gr[a] = divy(S[c1] - S[c0], D);
        R gc0 = R(0.5) * (divx(S[LI(fi + 1, fj)] - S[c0], D) + divx(S[c0] - S[LI(fi - 1, fj)], D));
        R gc1 = R(0.5) * (divx(S[LI(fi + 1, j1)] - S[c1], D) + divx(S[c1] - S[LI(fi - 1, j1)], D));
        cn[a] = R(0.5) * (gc0 + gc1);
      }
    }
    R jat[K];
#pragma unroll
    for (int k = 0; k < K; k++) jat[k] = R(0.0);
    /* calculate_fluxes_concentration.h:65: no y-current where gidy is 0 or MESH_Y-2 */
    const bool yskip = !xface && ((y0 - 1 + fj) + 3 == g.my - 2);
    R nl = R(-1.0);   /* |grad phi_liquid| on the face, computed on first use */
#pragma unroll
    for (int a = 0; a < L; a++) {
      /* sqrt(s2) != 0 exactly when s2 != 0 (s2 >= 0, or NaN on both sides) */
      const R s2 = cn[a] * cn[a] + gr[a] * gr[a];
      if (s2 != R(0.0) && !yskip) {
        const R ng = sqrt(s2);
        if (nl < R(0.0)) nl = sqrt(cn[L] * cn[L] + gr[L] * gr[L]);
        R sp = gr[a] * gr[L];
        sp += cn[a] * cn[L];
        if (nl > R(0.0)) sp /= (nl * ng);
#pragma unroll
        for (int k = 0; k < K; k++) {
          R cl1 = sm.CM[L][k][c1], cl0 = sm.CM[L][k][c0];
          R cs1 = sm.CM[a][k][c1], cs0 = sm.CM[a][k][c0];
          R bracket;
          if (D.obstacle)
            bracket = sm.SP[a][c1] * (cl1 - cs1) * sm.DP[a][c1] + sm.SP[a][c0] * (cl0 - cs0) * sm.DP[a][c0];
          else
            bracket = (cl1 - cs1) * sm.DP[a][c1] + (cl0 - cs0) * sm.DP[a][c0];
          jat[k] += D.atf[a][k] * fabs(sp) * (D.obstacle ? R(0.5) : D.well_half) * bracket * gr[a] / ng;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < K; k++) {
      if (xface) sm.JX[k][fidx] = jat[k];
      else sm.JY[k][fidx] = jat[k];
#pragma unroll
      for (int l = 0; l < K; l++) {
        R dm = (sm.DD[k][l][c1] + sm.DD[k][l][c0]) * R(0.5);
        R gm = xface ? divx(sm.M[l][c1] - sm.M[l][c0], D) : divy(sm.M[l][c1] - sm.M[l][c0], D);
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
    commit_cell<R, N, K>(D, sm.FX, sm.FY, sm.JX, sm.JY, sm.CM, sm.H, i, j, x, y, ph, dp, m, nph, nm, dmu, st);
    const long long o = (long long)x * g.pitch + y;
#pragma unroll
    for (int a = 0; a < N; a++) phin[a * g.plane + o] = nph[a];
#pragma unroll
    for (int k = 0; k < K; k++) mun[k * g.plane + o] = nm[k];
  }
  block_stats<R, N, K>(D, valid && stat_row(g, x), nph, nm, dp, dmu, st, 0, slot);
}

/* ------------------------------------------------------------------ */
/* batched simulations                                                 */
/* ------------------------------------------------------------------ */

/* One simulation of a batch: its geometry, where its planes start in the
 * pooled buffers, and its tiles in the batch's tile numbering. */
struct SimDesc {
  Grid g;
  long long off_state;   /* N phi planes then K mu planes */
  int tiles_x, tile0;    /* tiles per row, first tile */
  int off_T;             /* non-isothermal: the step's temperature rows (two of MESH_Y+6) in StatBufs::trows */
};

template <typename R>
__device__ __forceinline__ void load_consts(Consts<R> &dst, const Consts<R> *__restrict__ src) {
  const int *s = reinterpret_cast<const int *>(src);
  int *d = reinterpret_cast<int *>(&dst);
  for (int w = threadIdx.x; w < (int)(sizeof(Consts<R>) / sizeof(int)); w += NT) d[w] = __ldg(s + w);
}

}  // namespace gpd
