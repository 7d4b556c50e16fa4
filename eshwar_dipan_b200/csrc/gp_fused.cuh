/*
 * gp_fused.cuh -- the time step as two kernels over classified tiles.
 *
 * Every TX x TY tile of every simulation carries a phase flag per state
 * buffer: p >= 0 when each of its cells holds exactly the one-hot phi of phase
 * p (bits of 1.0 and +0.0), -1 otherwise, -2 when not known.  A tile whose own
 * flag and the flags of every tile its two-cell phi halo reaches (through the
 * boundary copy tables) are the same p >= 0 is a bulk tile: no phase is
 * active anywhere on its delta-phi ring (every Laplacian is 0.0), so delta-phi
 * is +0.0 there, no anti-trapping current flows, every cell takes the bulk
 * branch of the mu update with the pure-phase D, and phi stays as it is
 * (calculate_divergence_phasefield.h:19-22, calculate_fluxes_concentration.h:64,
 * calculate_divergence_concentration.h:43-57).
 *
 *  kf_classify one thread per tile: the bulk test; bulk and interface lists.
 *  kf_bulk     persistent warps over contiguous ranges of the bulk list, the
 *              next tile's mu in flight (one TMA box) while one is stepped.  Bulk
 *              tiles read and write mu only (phi is rewritten only when the
 *              output buffer does not already hold the same one-hot tile).
 *  kf_general  persistent CTAs over the interface list.  Stages phi with a
 *              two-cell halo and mu with one, computes delta-phi on the tile
 *              plus its one-cell ring in shared memory (the ring is recomputed
 *              by each neighbour instead of going through HBM), then the mu
 *              update and the phi commit, and the tile's new flag.
 *
 * The arithmetic of each cell is the reference's, in its order (FP64 results
 * are bit-identical to the reference step); the FP32 form differs only where
 * gp_tiles.cuh says.
 */
#pragma once
#include <climits>
#include <type_traits>

#include "gp_tiles.cuh"

namespace gpd {

constexpr int W2 = TY + 4, H2 = TX + 4, S2 = W2 * H2;   /* phi with a two-cell halo */
constexpr int RXF = (TX + 3) * (TY + 2);                 /* x-faces around the ring cells */
constexpr int RYF = (TX + 2) * (TY + 3);                 /* y-faces around the ring cells */
#define L2I(i, j) ((i) * W2 + (j))

constexpr signed char FLAG_MIXED = -1, FLAG_UNKNOWN = -2;

/* A pair of floats in one 64-bit register pair, for sm_100's packed FP32
 * arithmetic (add/sub/mul/fma .rn.f32x2: two IEEE single-precision results,
 * round to nearest, per instruction). */
typedef unsigned long long f2;
__device__ __forceinline__ f2 f2pack(float lo, float hi) {
  f2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ float f2lo(f2 v) {
  float lo, hi;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
  return lo;
}
__device__ __forceinline__ float f2hi(f2 v) {
  float lo, hi;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
  return hi;
}
__device__ __forceinline__ f2 f2add(f2 a, f2 b) {
  f2 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2 f2sub(f2 a, f2 b) {
  f2 d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2 f2mul(f2 a, f2 b) {
  f2 d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2 f2fma(f2 a, f2 b, f2 c) {
  f2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
/* three-operand max/min (a NaN operand is ignored, as by fmaxf) */
__device__ __forceinline__ float fmax3f(float a, float b, float c) {
  float d;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
  return d;
}
__device__ __forceinline__ float fmin3f(float a, float b, float c) {
  float d;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
  return d;
}
/* spacing of the floats at |v| (2^(e-23) for a normal v of exponent e; the
 * subnormal spacing below) */
__device__ __forceinline__ float ulpf(float v) {
  const unsigned e = max(__float_as_uint(v) & 0x7f800000u, 24u << 23);
  return __uint_as_float(e - (23u << 23));
}

/* Phase flags of one tile in one state buffer: for the whole tile and for its
 * four two-cell-deep edge bands (top = first two rows, bot = last two rows,
 * left/right = first/last two columns, over the tile's cells inside the
 * domain): the phase p whose exact one-hot phi every cell of the region holds,
 * FLAG_MIXED, or FLAG_UNKNOWN.  8 bytes, read as one word. */
struct __align__(8) TileFlags {
  signed char whole, top, bot, left, right, pad0, pad1, pad2;
};

struct RemapTab2 {
  int row[H2], col[W2];
};

/* rows/columns of the two-cell phi halo (origin x0-2, y0-2) after the remap;
 * -1 outside [-2, m+1] (not needed by any delta-phi ring cell). */
template <typename R>
__device__ __forceinline__ void remap_tab2(RemapTab2 &t, const Consts<R> &D, const Grid &g, int x0, int y0) {
  const int u = threadIdx.x;
  if (u < H2) {
    const int x = x0 - 2 + u;
    t.row[u] = (x >= -2 && x <= g.mx + 1) ? remap(x, g.mx, D.bc_x[0][0], D.bc_x[0][1]) * g.pitch : -1;
  } else if (u < H2 + W2) {
    const int y = y0 - 2 + (u - H2);
    t.col[u - H2] = (y >= -2 && y <= g.my + 1) ? remap(y, g.my, D.bc_y[0][0], D.bc_y[0][1]) : -1;
  }
}

/* one-hot test on exact bits: phase index, or -1 */
template <typename R, int N>
__device__ __forceinline__ int one_hot(const R *ph) {
  int p = -1, ones = 0, zeros = 0;
#pragma unroll
  for (int a = 0; a < N; a++) {
    if (sizeof(R) == 8) {
      const long long b = __double_as_longlong((double)ph[a]);
      if (b == 0x3ff0000000000000LL) { p = a; ones++; }
      else if (b == 0) zeros++;
    } else {
      const unsigned b = __float_as_uint((float)ph[a]);
      if (b == 0x3f800000u) { p = a; ones++; }
      else if (b == 0u) zeros++;
    }
  }
  return (ones == 1 && zeros == N - 1) ? p : -1;
}

/* Flags of a tile from its new phi, one one-hot phase (or -1) per thread
 * (cell (tx, ty) of the tile, valid cells only; rows x cols cells are in the
 * domain).  Call with all threads; the result is valid in every thread. */
__device__ __forceinline__ TileFlags tile_flags(bool valid, int p, int tx, int ty, int rows, int cols) {
  __shared__ int s_lo[NT / 32][5], s_hi[NT / 32][5];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const bool in[5] = {true, tx < 2, tx >= rows - 2, ty < 2, ty >= cols - 2};
  int lo[5], hi[5];
#pragma unroll
  for (int r = 0; r < 5; r++) {
    lo[r] = (valid && in[r]) ? p : INT_MAX;
    hi[r] = (valid && in[r]) ? p : INT_MIN;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo[r] = min(lo[r], __shfl_xor_sync(0xffffffffu, lo[r], o));
      hi[r] = max(hi[r], __shfl_xor_sync(0xffffffffu, hi[r], o));
    }
  }
  if (lane == 0) {
#pragma unroll
    for (int r = 0; r < 5; r++) { s_lo[wid][r] = lo[r]; s_hi[wid][r] = hi[r]; }
  }
  __syncthreads();
  signed char f[5];
#pragma unroll
  for (int r = 0; r < 5; r++) {
    int l2 = INT_MAX, h2 = INT_MIN;
#pragma unroll
    for (int w = 0; w < NT / 32; w++) { l2 = min(l2, s_lo[w][r]); h2 = max(h2, s_hi[w][r]); }
    f[r] = (l2 >= 0 && l2 == h2) ? (signed char)l2 : FLAG_MIXED;
  }
  __syncthreads();
  TileFlags t;
  t.whole = f[0]; t.top = f[1]; t.bot = f[2]; t.left = f[3]; t.right = f[4];
  t.pad0 = t.pad1 = t.pad2 = 0;
  return t;
}

__device__ __forceinline__ TileFlags uniform_flags(int p) {
  TileFlags t;
  t.whole = t.top = t.bot = t.left = t.right = (signed char)p;
  t.pad0 = t.pad1 = t.pad2 = 0;
  return t;
}

/* Bulk test of tile (tile rows by, columns bx) of a simulation, by one
 * thread: every cell of the tile and of its two-cell phi halo holds the exact
 * one-hot phi of one phase.  Returns the phase or -1.  When the halo stays
 * inside the domain it is covered by the facing edge bands of the eight
 * neighbour tiles (a corner by either band that contains it); otherwise by the
 * whole-tile flags of the tiles that hold the halo cells after the boundary
 * remap. */
template <typename R>
__device__ __forceinline__ int bulk_phase(const Consts<R> &D, const Grid &g, const TileFlags *__restrict__ flags,
                                          int tile0, int tiles_x, int by, int bx) {
  const int x0 = by * TX, y0 = bx * TY;
  const int xl = min(x0 + TX, g.mx) - 1, yl = min(y0 + TY, g.my) - 1;
  if (x0 >= 2 && xl + 2 < g.mx && y0 >= 2 && yl + 2 < g.my) {
    const TileFlags *f = flags + tile0 + by * tiles_x + bx;
    const TileFlags ul = f[-tiles_x - 1], u = f[-tiles_x], ur = f[-tiles_x + 1];
    const TileFlags l = f[-1], c = f[0], r = f[1];
    const TileFlags dl = f[tiles_x - 1], d = f[tiles_x], dr = f[tiles_x + 1];
    const int p = c.whole;
    const bool ok = p >= 0 && u.bot == p && d.top == p && l.right == p && r.left == p &&
                    (ul.bot == p || ul.right == p) && (ur.bot == p || ur.left == p) &&
                    (dl.top == p || dl.right == p) && (dr.top == p || dr.left == p);
    return ok ? p : -1;
  }
  /* the tiles of rows x0-2, x0-1, xl+1, xl+2 and columns y0-2, y0-1, yl+1, yl+2 */
  int rows[5], cols[5];
  {
    const int xs[4] = {x0 - 2, x0 - 1, xl + 1, xl + 2};
    const int ys[4] = {y0 - 2, y0 - 1, yl + 1, yl + 2};
    rows[0] = by;
    cols[0] = bx;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      int x = xs[q], y = ys[q];
      if (x < 0 || x >= g.mx) x = remap(x, g.mx, D.bc_x[0][0], D.bc_x[0][1]);
      if (y < 0 || y >= g.my) y = remap(y, g.my, D.bc_y[0][0], D.bc_y[0][1]);
      rows[q + 1] = x / TX;
      cols[q + 1] = y / TY;
    }
  }
  const int p = flags[tile0 + by * tiles_x + bx].whole;
  bool ok = p >= 0;
#pragma unroll
  for (int q = 0; q < 25; q++) ok = ok && flags[tile0 + rows[q / 5] * tiles_x + cols[q % 5]].whole == p;
  return ok ? p : -1;
}


/* ------------------------------------------------------------------ */
/* interface tiles                                                     */
/* ------------------------------------------------------------------ */

template <typename R, int N, int K>
struct GenSmem {
  R P[N][S2];              /* phi, two-cell halo, origin (x0-2, y0-2) */
  R M[K][SS];              /* mu, one-cell halo, origin (x0-1, y0-1)  */
  R DP[N][SS];             /* delta-phi of the ring region (same origin as M) */
  unsigned char ACT[SS];   /* active phases of each ring cell (bit a) */
  short LIST[SS];          /* ring cells with an active phase, in no particular order */
  short FLIST[RXF + RYF];  /* anisotropy faces those cells read */
  int nlist, nflist;
  union {
    R T[NP<N>::v][4][RXF + RYF];   /* anisotropy face terms of the ring region */
    struct {
      R CM[N][K][SS];      /* c_a,k(mu) per cell */
      R H[N][SS];          /* h_a(phi) per cell */
      R SP[N][SS];         /* s_phi of the obstacle anti-trapping (solid phases) */
      R DD[K][K][SS];      /* D_kl per cell */
      R JX[K][NXF], JY[K][NYF];
      R FX[K][K][NXF], FY[K][K][NYF];
    } u;
  } w;
  RemapTab2 rtp;
  RemapTab rtm;
};

/* Anisotropy terms of one face of the ring region for all pairs: the same
 * arithmetic as face_terms (function_A_01.h:163-215 through functionQ.h and
 * anisotropy_01.h) on the two-cell-halo layout.  xface: face between P rows
 * i and i+1 at column j; else between columns j and j+1 of row i. */
template <typename R, int N, typename CT>
__device__ __forceinline__ void ring_face_terms(const CT &D, const R (*P)[S2], R (*T)[4][RXF + RYF],
                                                bool xface, int i, int j, int fidx) {
  R s[N], gr[N], c0[N], c1[N];
#pragma unroll
  for (int a = 0; a < N; a++) {
    const R *S = P[a];
    if (xface) {
      R p0 = S[L2I(i, j)], p1 = S[L2I(i + 1, j)];
      s[a] = R(0.5) * (p1 + p0);
      gr[a] = divx(p1 - p0, D);
      c0[a] = div2y(S[L2I(i, j + 1)] - S[L2I(i, j - 1)], D);
      c1[a] = div2y(S[L2I(i + 1, j + 1)] - S[L2I(i + 1, j - 1)], D);
    } else {
      R p0 = S[L2I(i, j)], p1 = S[L2I(i, j + 1)];
      s[a] = R(0.5) * (p1 + p0);
      gr[a] = divy(p1 - p0, D);
      c0[a] = R(0.5) * (divx(S[L2I(i + 1, j)] - S[L2I(i, j)], D) + divx(S[L2I(i, j)] - S[L2I(i - 1, j)], D));
      c1[a] = R(0.5) * (divx(S[L2I(i + 1, j + 1)] - S[L2I(i, j + 1)], D) +
                        divx(S[L2I(i, j + 1)] - S[L2I(i - 1, j + 1)], D));
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
      T[p][0][fidx] = ac2 * Pab * (-s[b]);
      T[p][1][fidx] = ac2 * Pba * (-s[a]);
      T[p][2][fidx] = acq * rd * (-s[b]);
      T[p][3][fidx] = acq * (R(0.0) - rd) * (-s[a]);
    }
}

/* delta-phi of one ring cell (ring coordinates ri, rj; its phi at P row ri+1,
 * column rj+1) from the staged tile: calculate_divergence_phasefield_2D
 * (calculate_divergence_phasefield.h:4-62) in the same arithmetic as dphi_tile.
 * Not inlined: as a call of its own it gets its own register allocation, and
 * the interface tiles spill far less under the 128-register cap of two CTAs
 * per SM (FP64 ternary 3-phase: 732 bytes of spill stores inlined, about 200
 * not; FP32: none), which made whole steps 3-8 % faster. */
template <typename R, int N, int K, bool ANISO, typename CT>
__device__ __noinline__ void ring_dphi(const CT &D, const GenSmem<R, N, K> &sm, int ri, int rj,
                                          unsigned mask, R *d, double Tpf) {
  const int i = ri + 1, j = rj + 1, e = LI(ri, rj);
  R ph[N];
  bool act[N];
#pragma unroll
  for (int a = 0; a < N; a++) {
    ph[a] = sm.P[a][L2I(i, j)];
    act[a] = (mask >> a) & 1u;
  }
  if (!mask) {
#pragma unroll
    for (int a = 0; a < N; a++) {
      d[a] = R(0.0);
      if ((ph[a] + d[a]) < R(0.0)) d[a] += fabs(d[a] + ph[a]);
    }
    return;
  }
  R m[K];
#pragma unroll
  for (int k = 0; k < K; k++) m[k] = sm.M[k][e];
  R gcx[N], gcy[N];
#pragma unroll
  for (int a = 0; a < N; a++) {
    const R *S = sm.P[a];
    gcx[a] = R(0.5) * (divx(S[L2I(i + 1, j)] - S[L2I(i, j)], D) + divx(S[L2I(i, j)] - S[L2I(i - 1, j)], D));
    gcy[a] = div2y(S[L2I(i, j + 1)] - S[L2I(i, j - 1)], D);
  }
  R psi[N];
  if (D.tgrad) {
    /* init_propertymatrices(T) at the cell's temperature before dpsi
     * (calculate_divergence_phasefield.h:21-29) */
    R E[N][K], Bt[N][K], Ct[N];
    e_at<R, N, K>(D, Tpf, E);
    bc_at<R, N, K>(D, Tpf, Bt, Ct);
#pragma unroll
    for (int b = 0; b < N; b++) {
      R c[K], ps = R(0.0);
#pragma unroll
      for (int k = 0; k < K; k++) {
        c[k] = c_muE<R, K>(D, E[b], m, b, k);
        ps -= m[k] * c[k];
      }
      ps += feBC<R, K>(D, Bt[b], Ct[b], c, b);
      psi[b] = ps;
    }
  } else {
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
  }
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
  /* face indices of this cell in the ring face cache */
  const int xf = i * (TY + 2) + (j - 1), xb = (i - 1) * (TY + 2) + (j - 1);
  const int yr = RXF + (i - 1) * (TY + 3) + j, yl = RXF + (i - 1) * (TY + 3) + (j - 1);
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
        const int o = a < b ? 0 : 1;
        const R(*T)[RXF + RYF] = sm.w.T[p];
        R d1v = divx((T[o][xf]) - (T[o][xb]), D);
        d1v += divy((T[o][yr]) - (T[o][yl]), D);
        d1v *= D.gamma[a][b];
        t1 += d1v;
        R d2v = divx(T[2 + o][xf] - T[2 + o][xb], D);
        d2v += divy(T[2 + o][yr] - T[2 + o][yl], D);
        d2v *= D.gamma[a][b];
        t2 += d2v;
      }
      dA = R(2.0) * (s1 + s2);
      div = (R(2.0) * (t1 + t2) + R(0.0));
    } else {
      R s = R(0.0), t = R(0.0);
      const R *Sa = sm.P[a];
#pragma unroll
      for (int b = 0; b < N; b++) {
        if (b == a) continue;
        const R *Sb = sm.P[b];
        R sp = R(0.0);
        sp += (ph[a] * gcx[b] - ph[b] * gcx[a]) * gcx[b];
        sp += (ph[a] * gcy[b] - ph[b] * gcy[a]) * gcy[b];
        sp *= D.gamma[a][b];
        s += sp;
        R pa = Sa[L2I(i, j)], pb = Sb[L2I(i, j)];
        R sxa = R(0.5) * (Sa[L2I(i + 1, j)] + pa), sxb = R(0.5) * (Sb[L2I(i + 1, j)] + pb);
        R gxa = divx(Sa[L2I(i + 1, j)] - pa, D), gxb = divx(Sb[L2I(i + 1, j)] - pb, D);
        R bxa = R(0.5) * (pa + Sa[L2I(i - 1, j)]), bxb = R(0.5) * (pb + Sb[L2I(i - 1, j)]);
        R hxa = divx(pa - Sa[L2I(i - 1, j)], D), hxb = divx(pb - Sb[L2I(i - 1, j)], D);
        R sya = R(0.5) * (Sa[L2I(i, j + 1)] + pa), syb = R(0.5) * (Sb[L2I(i, j + 1)] + pb);
        R gya = divy(Sa[L2I(i, j + 1)] - pa, D), gyb = divy(Sb[L2I(i, j + 1)] - pb, D);
        R lya = R(0.5) * (pa + Sa[L2I(i, j - 1)]), lyb = R(0.5) * (pb + Sb[L2I(i, j - 1)]);
        R hya = divy(pa - Sa[L2I(i, j - 1)], D), hyb = divy(pb - Sb[L2I(i, j - 1)], D);
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

/* One interface tile (cells (x0+tx, y0+ty)): delta-phi on the tile and its
 * ring, then the concentration pass (calculate_fluxes_concentration_2D +
 * calculate_divergence_concentration_2D, calculate_fluxes_concentration.h:4-145,
 * calculate_divergence_concentration.h:4-153) and the phi commit, in the
 * arithmetic of update_tile's general path.  Returns the tile's new flags. */
template <typename R, int N, int K, bool ANISO, typename CT>
__device__ __forceinline__ TileFlags general_tile(const CT &D, const Grid &g, const R *__restrict__ phi,
                                                    const R *__restrict__ mu, R *__restrict__ phin,
                                                    R *__restrict__ mun, int x0, int y0, const StatBufs &st,
                                                    long long ext_slot, long long slot, GenSmem<R, N, K> &sm,
                                                    const double *__restrict__ tpf, const double *__restrict__ tcc) {
  constexpr int L = N - 1;
  const R cst = D.obstacle ? D.jat_obst : D.jat_well;

  /* ---- stage phi (two-cell halo) and mu (one-cell halo) through the copy tables */
  remap_tab2(sm.rtp, D, g, x0, y0);
  remap_tab(sm.rtm, D, g, x0, y0, 1, -1, g.mx, -1, g.my);
  __syncthreads();
  for (int e = threadIdx.x; e < S2; e += NT) {
    const int i = e / W2, j = e - i * W2;
    const int r = sm.rtp.row[i], c = sm.rtp.col[j];
    if (r >= 0 && c >= 0) {
      const R *src = phi + (r + c);
#pragma unroll
      for (int a = 0; a < N; a++) sm.P[a][e] = __ldg(src + a * g.plane);
    } else {
#pragma unroll
      for (int a = 0; a < N; a++) sm.P[a][e] = R(0.0);
    }
  }
  for (int e = threadIdx.x; e < SS; e += NT) {
    const int i = e / SW, j = e - i * SW;
    const int r = sm.rtm.row[i], c = sm.rtm.col[j];
    if (r >= 0 && c >= 0) {
      const R *src = mu + (r + c);
#pragma unroll
      for (int k = 0; k < K; k++) sm.M[k][e] = __ldg(src + k * g.plane);
    } else {
#pragma unroll
      for (int k = 0; k < K; k++) sm.M[k][e] = R(0.0);
    }
  }
  __syncthreads();

  /* ---- active phases of the ring cells (interior plus ring: x <= mx, y <= my).
   * A cell with no active phase gets its delta-phi here (no phase active:
   * 0, then the projection's clamp of a negative phi; outside the needed
   * region: 0); the others go on a list, so that the expensive delta-phi
   * work is spread over every thread of the CTA wherever the active cells
   * lie in the tile. */
  for (int e = threadIdx.x; e < SS; e += NT) {
    const int ri = e / SW, rj = e - ri * SW, i = ri + 1, j = rj + 1;
    const bool vd = (x0 - 1 + ri <= g.mx) && (y0 - 1 + rj <= g.my);
    unsigned mask = 0;
#pragma unroll
    for (int a = 0; a < N; a++) {
      const R *S = sm.P[a];
      R gxf = divx(S[L2I(i + 1, j)] - S[L2I(i, j)], D), gxb = divx(S[L2I(i, j)] - S[L2I(i - 1, j)], D);
      R gyr = divy(S[L2I(i, j + 1)] - S[L2I(i, j)], D), gyl = divy(S[L2I(i, j)] - S[L2I(i, j - 1)], D);
      R dv = divx(gxf - gxb, D);
      dv += divy(gyr - gyl, D);
      if (fabs(dv) > R(0.0)) mask |= 1u << a;
    }
    if (!vd) mask = 0;
    sm.ACT[e] = (unsigned char)mask;
    if (mask) {
      sm.LIST[atomicAdd(&sm.nlist, 1)] = (short)e;
    } else {
#pragma unroll
      for (int a = 0; a < N; a++) {
        R d = R(0.0);
        if (vd) {
          const R ph = sm.P[a][L2I(i, j)];
          if ((ph + d) < R(0.0)) d += fabs(d + ph);
        }
        sm.DP[a][e] = d;
      }
    }
  }
  __syncthreads();
  const int nact = sm.nlist;
  if (ANISO && nact > 0) {
    /* only the faces of active ring cells are read by ring_dphi: list them,
     * then compute them spread over the CTA */
    for (int e = threadIdx.x; e < RXF + RYF; e += NT) {
      bool need;
      if (e < RXF) {
        const int fi = e / (TY + 2), fj = e - fi * (TY + 2) + 1;
        /* ring cells (fi-1, fj-1) and (fi, fj-1) */
        need = (fi >= 1 && sm.ACT[LI(fi - 1, fj - 1)]) || (fi < SH && sm.ACT[LI(fi, fj - 1)]);
      } else {
        const int f = e - RXF, fi = f / (TY + 3) + 1, fj = f - (fi - 1) * (TY + 3);
        /* ring cells (fi-1, fj-1) and (fi-1, fj) */
        need = (fj >= 1 && sm.ACT[LI(fi - 1, fj - 1)]) || (fj < SW && sm.ACT[LI(fi - 1, fj)]);
      }
      if (need) sm.FLIST[atomicAdd(&sm.nflist, 1)] = (short)e;
    }
    __syncthreads();
    const int nf = sm.nflist;
    for (int q = threadIdx.x; q < nf; q += NT) {
      const int e = sm.FLIST[q];
      if (e < RXF) {
        const int fi = e / (TY + 2), fj = e - fi * (TY + 2) + 1;
        ring_face_terms<R, N>(D, sm.P, sm.w.T, true, fi, fj, e);
      } else {
        const int f = e - RXF, fi = f / (TY + 3) + 1, fj = f - (fi - 1) * (TY + 3);
        ring_face_terms<R, N>(D, sm.P, sm.w.T, false, fi, fj, e);
      }
    }
    __syncthreads();
  }
  for (int q = threadIdx.x; q < nact; q += NT) {
    const int e = sm.LIST[q];
    const int ri = e / SW, rj = e - ri * SW;
    R d[N];
    ring_dphi<R, N, K, ANISO>(D, sm, ri, rj, sm.ACT[e], d, D.tgrad ? tpf[y0 - 1 + rj + 3] : 0.0);
#pragma unroll
    for (int a = 0; a < N; a++) sm.DP[a][e] = d[a];
  }
  __syncthreads();   /* the face-term cache is dead from here: its space holds the update's arrays */
  if (st.dphi_out) {
    /* the adjoint's tape: the delta-phi of the tile and of its ring cells
     * (the domain's ring included), as the reverse sweep reads it */
    for (int e = threadIdx.x; e < SS; e += NT) {
      const int x = x0 - 1 + e / SW, y = y0 - 1 + e % SW;
      if (x <= g.mx && y <= g.my) {
#pragma unroll
        for (int a = 0; a < N; a++)
          st.dphi_out[a * g.dplane + (long long)(x + 1) * g.dpitch + (y + 1)] = (double)sm.DP[a][e];
      }
    }
  }
  if (threadIdx.x == 0) {
    sm.nlist = 0;    /* for the CTA's next tile */
    sm.nflist = 0;
  }

#define PR(a, e) sm.P[a][L2I((e) / SW + 1, (e) % SW + 1)]
  /* ---- per-cell quantities of the ring region */
  for (int e = threadIdx.x; e < SS; e += NT) {
    R p[N], mm[K];
#pragma unroll
    for (int a = 0; a < N; a++) p[a] = PR(a, e);
#pragma unroll
    for (int k = 0; k < K; k++) mm[k] = sm.M[k][e];
    R Ec[N][K];
    /* the ghosted column of ring cell e (cells past my+1 are not needed: clamped) */
    if (D.tgrad) e_at<R, N, K>(D, tcc[min(y0 - 1 + e % SW + 3, g.my + 5)], Ec);
#pragma unroll
    for (int a = 0; a < N; a++) {
      R hv = h<R, N>(p, a);
      sm.w.u.H[a][e] = hv;
#pragma unroll
      for (int k = 0; k < K; k++)
        sm.w.u.CM[a][k][e] = D.tgrad ? c_muE<R, K>(D, Ec[a], mm, a, k) : c_mu<R, K>(D, mm, a, k);
      if (a < L)
        sm.w.u.SP[a][e] =
            (p[a] * (R(1.0) - p[a]) > R(0.0)) ? p[a] * (R(1.0) - hv) / (sqrt(p[a] * (R(1.0) - p[a]))) : R(0.0);
    }
#pragma unroll
    for (int k = 0; k < K; k++)
#pragma unroll
      for (int l = 0; l < K; l++) sm.w.u.DD[k][l][e] = Dcell<R, N, K>(D, p, k, l);
  }
  __syncthreads();

#define PRIJ(a, i, j) sm.P[a][L2I((i) + 1, (j) + 1)]
  /* ---- faces of the tile: anti-trapping current and diffusion flux products */
  for (int e = threadIdx.x; e < NXF + NYF; e += NT) {
    const bool xface = e < NXF;
    int fi, fj, i1, j1, fidx;
    if (xface) { fi = e / TY; fj = e - fi * TY + 1; i1 = fi + 1; j1 = fj; fidx = e; }
    else { int f = e - NXF; fi = f / (TY + 1) + 1; fj = f - (fi - 1) * (TY + 1); i1 = fi; j1 = fj + 1; fidx = f; }
    const int c0 = LI(fi, fj), c1 = LI(i1, j1);
    R gr[N], cn[N];
#pragma unroll
    for (int a = 0; a < N; a++) {
      if (xface) {
        gr[a] = divx(PRIJ(a, i1, j1) - PRIJ(a, fi, fj), D);
        cn[a] = R(0.5) * (div2y(PRIJ(a, fi, fj + 1) - PRIJ(a, fi, fj - 1), D) +
                          div2y(PRIJ(a, i1, fj + 1) - PRIJ(a, i1, fj - 1), D));
      } else {
        gr[a] = divy(PRIJ(a, i1, j1) - PRIJ(a, fi, fj), D);
        R gc0 = R(0.5) * (divx(PRIJ(a, fi + 1, fj) - PRIJ(a, fi, fj), D) + divx(PRIJ(a, fi, fj) - PRIJ(a, fi - 1, fj), D));
        R gc1 = R(0.5) * (divx(PRIJ(a, fi + 1, j1) - PRIJ(a, i1, j1), D) + divx(PRIJ(a, i1, j1) - PRIJ(a, fi - 1, j1), D));
        cn[a] = R(0.5) * (gc0 + gc1);
      }
    }
    R jat[K];
#pragma unroll
    for (int k = 0; k < K; k++) jat[k] = R(0.0);
    /* calculate_fluxes_concentration.h:65: no y-current where gidy is 0 or MESH_Y-2 */
    const bool yskip = !xface && ((y0 - 1 + fj) + 3 == g.my - 2);
    R nl = R(-1.0);
#pragma unroll
    for (int a = 0; a < L; a++) {
      const R s2 = cn[a] * cn[a] + gr[a] * gr[a];
      if (s2 != R(0.0) && !yskip) {
        const R ng = sqrt(s2);
        if (nl < R(0.0)) nl = sqrt(cn[L] * cn[L] + gr[L] * gr[L]);
        R sp = gr[a] * gr[L];
        sp += cn[a] * cn[L];
        if (nl > R(0.0)) sp /= (nl * ng);
#pragma unroll
        for (int k = 0; k < K; k++) {
          R cl1 = sm.w.u.CM[L][k][c1], cl0 = sm.w.u.CM[L][k][c0];
          R cs1 = sm.w.u.CM[a][k][c1], cs0 = sm.w.u.CM[a][k][c0];
          R bracket;
          if (D.obstacle)
            bracket = sm.w.u.SP[a][c1] * (cl1 - cs1) * sm.DP[a][c1] + sm.w.u.SP[a][c0] * (cl0 - cs0) * sm.DP[a][c0];
          else
            bracket = (cl1 - cs1) * sm.DP[a][c1] + (cl0 - cs0) * sm.DP[a][c0];
          jat[k] += D.atf[a][k] * fabs(sp) * (D.obstacle ? R(0.5) : D.well_half) * bracket * gr[a] / ng;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < K; k++) {
      if (xface) sm.w.u.JX[k][fidx] = jat[k];
      else sm.w.u.JY[k][fidx] = jat[k];
#pragma unroll
      for (int l = 0; l < K; l++) {
        R dm = (sm.w.u.DD[k][l][c1] + sm.w.u.DD[k][l][c0]) * R(0.5);
        R gm = xface ? divx(sm.M[l][c1] - sm.M[l][c0], D) : divy(sm.M[l][c1] - sm.M[l][c0], D);
        if (xface) sm.w.u.FX[k][l][fidx] = dm * gm;
        else sm.w.u.FY[k][l][fidx] = dm * gm;
      }
    }
  }
  __syncthreads();

  /* ---- per cell: mu update, phi commit */
  const int tx = threadIdx.x / TY, ty = threadIdx.x - (threadIdx.x / TY) * TY;
  const int x = x0 + tx, y = y0 + ty, i = tx + 1, j = ty + 1, c = LI(i, j);
  const bool valid = (x < g.mx) && (y < g.my);
  R ph[N], dp[N], m[K], nph[N], nm[K];
  double dmu[K];
  int oh = -1;
  if (valid) {
#pragma unroll
    for (int a = 0; a < N; a++) { ph[a] = PRIJ(a, i, j); dp[a] = sm.DP[a][c]; }
#pragma unroll
    for (int k = 0; k < K; k++) m[k] = sm.M[k][c];
    commit_cell<R, N, K>(D, sm.w.u.FX, sm.w.u.FY, sm.w.u.JX, sm.w.u.JY, sm.w.u.CM, sm.w.u.H, i, j, x, y, ph, dp, m,
                         nph, nm, dmu, st, D.tgrad ? tcc[y + 3] : 0.0);
    const long long o = (long long)x * g.pitch + y;
#pragma unroll
    for (int a = 0; a < N; a++) phin[a * g.plane + o] = nph[a];
#pragma unroll
    for (int k = 0; k < K; k++) mun[k * g.plane + o] = nm[k];
    oh = one_hot<R, N>(nph);
  }
#undef PRIJ
#undef PR
  block_stats<R, N, K>(D, valid && stat_row(g, x), nph, nm, dp, dmu, st, ext_slot, slot,
                       (D.tgrad && valid) ? tcc[y + 3] : 0.0);
  return tile_flags(valid, oh, tx, ty, min(TX, g.mx - x0), min(TY, g.my - y0));
}

/* ------------------------------------------------------------------ */
/* kernels                                                             */
/* ------------------------------------------------------------------ */

/* Work-list counters of a batch: [0] interface tiles listed by kf_classify,
 * [1] next interface entry to take, [2] CTAs of kf_bulk and kf_general
 * finished, [3] step number (keys the FP32 rounding stream), [4] bulk tiles
 * listed, [5] error flag (a TMA box of kf_bulk did not arrive; the host reads
 * and clears it).  The last CTA of the two kernels resets [0..2] and [4] and
 * advances [3], so a step is exactly the three launches kf_classify, then
 * kf_bulk and kf_general (in either order or side by side). */
enum { CTR_LIST = 0, CTR_HEAD = 1, CTR_DONE = 2, CTR_STEP = 3, CTR_BULK = 4, CTR_ERR = 5, CTR_BHEAD = 6,
       CTR_COUNT = 8 };

/* End of one CTA of the step's bulk or interface kernel (they may run
 * concurrently): the last of the step's ndone CTAs empties the lists and
 * advances the step counter.  Call with all threads. */
__device__ __forceinline__ void step_finish(int *ctr, int ndone) {
  __shared__ int s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(ctr + CTR_DONE, 1) == ndone - 1;
  }
  __syncthreads();
  if (s_last && threadIdx.x == 0) {
    ctr[CTR_LIST] = 0;
    ctr[CTR_HEAD] = 0;
    ctr[CTR_DONE] = 0;
    ctr[CTR_BULK] = 0;
    ctr[CTR_BHEAD] = 0;
    ctr[CTR_STEP] = (int)((unsigned)ctr[CTR_STEP] + 1u);
    __threadfence();
  }
}

/* One thread per tile: the bulk test, then the tile goes on the bulk list
 * or the interface list; one atomic per warp and list.  A bulk entry holds
 * everything kf_bulk needs to start the tile: {t | phase << 28, simulation |
 * flag of the output buffer << 24, tile row << 16 | tile column, 0}.  Small CTAs (NTC threads) spread the flag reads over every SM. */
constexpr int NTC = 64;
template <typename R>
__global__ void __launch_bounds__(NTC) kf_classify(const SimDesc *__restrict__ sims,
                                                  const Consts<R> *__restrict__ consts, const int *__restrict__ tsim,
                                                  int ntiles, const TileFlags *__restrict__ flag_in,
                                                  const TileFlags *__restrict__ flag_outbuf,
                                                  int *__restrict__ glist, int4 *__restrict__ blist,
                                                  int *__restrict__ ctr) {
  const int t = blockIdx.x * NTC + threadIdx.x, lane = threadIdx.x & 31;
  int p = -1, s = 0, by = 0, bx = 0;
  if (t < ntiles) {
    s = __ldg(tsim + t);
    const SimDesc &sd = sims[s];
    const int lt = t - sd.tile0;
    by = lt / sd.tiles_x;
    bx = lt - by * sd.tiles_x;
    /* a non-isothermal simulation steps every tile as an interface tile
     * (whose pure-phase cells take the bulk update at their temperature) */
    if (!consts[s].tgrad) p = bulk_phase<R>(consts[s], sd.g, flag_in, sd.tile0, sd.tiles_x, by, bx);
  }
  const unsigned mb = __ballot_sync(0xffffffffu, t < ntiles && p >= 0);
  const unsigned mg = __ballot_sync(0xffffffffu, t < ntiles && p < 0);
  int bb = 0, bg = 0;
  if (lane == 0) {
    if (mb) bb = atomicAdd(ctr + CTR_BULK, __popc(mb));
    if (mg) bg = atomicAdd(ctr + CTR_LIST, __popc(mg));
  }
  bb = __shfl_sync(0xffffffffu, bb, 0);
  bg = __shfl_sync(0xffffffffu, bg, 0);
  const unsigned below = (1u << lane) - 1u;
  if (t < ntiles) {
    if (p >= 0)
      blist[bb + __popc(mb & below)] =
          make_int4(t | (p << 28), s | (((int)flag_outbuf[t].whole & 0xff) << 24), (by << 16) | bx, 0);
    else glist[bg + __popc(mg & below)] = t;
  }
}

/* ---- TMA and mbarrier primitives (one CTA, no cluster, no multicast) ---- */
__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
/* make barrier initialisation and earlier generic shared-memory writes
 * visible to the async (TMA) proxy */
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
/* tiled 3-D tensor copy global -> this CTA's shared memory, completion
 * counted in bytes on bar; c0 is the innermost coordinate */
__device__ __forceinline__ void tma_load_3d(unsigned dst, const void *tmap, int c0, int c1, int c2, unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];\n" ::"r"(dst),
      "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
      : "memory");
}
__device__ __forceinline__ bool mbar_test(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
/* wait for phase `parity` of bar to complete, at most `tries` polls (each
 * poll may suspend the thread for a short while); false when it did not */
constexpr int MBAR_TRIES = 1 << 20;
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, int tries) {
  for (int it = 0; it < tries; it++)
    if (mbar_test(bar, parity)) return true;
  return false;
}

/* x/dx and y/dy of the bulk kernel: a multiplication by the reciprocal when
 * the spacing is a power of two (MUL, chosen at launch), else the division */
template <bool MUL, typename R>
__device__ __forceinline__ R bdiv(R v, R inv, R d) {
  if constexpr (MUL) return v * inv;
  else return v / d;
}

/* A tensor map (CUtensorMap, 128 bytes) of the K mu planes of one simulation
 * in one state buffer: dimensions {pitch, mx, K}, box {BW, SH, K}. */
struct alignas(64) TensorMapSlot {
  unsigned long long w[16];
};

/* Shared memory of one warp of kf_bulk: NST stages of mu with a one-cell halo,
 * each filled by one TMA box.  A box starts CO columns left of the halo
 * column so that its first column is 16-byte aligned (y0 - 1 - CO is a
 * multiple of 16 bytes / sizeof(R)); stage column c holds y = y0 - 1 - CO + c. */
template <typename R, int K>
struct BulkGeom {
  static constexpr int CO = sizeof(R) == 8 ? 1 : 3;
  static constexpr int BW = SW + 2 * CO;   /* 36 doubles or 40 floats: a multiple of 16 bytes */
  /* boxes in flight per warp: 4 of FP32 or 2 of FP64 (the same bytes) */
  static constexpr int NST = sizeof(R) == 4 ? 4 : 2;
  static constexpr unsigned BOX_BYTES = (unsigned)(K * SH * BW * sizeof(R));
};
template <typename R, int K>
struct alignas(128) BulkStage {
  R M[K][SH][BulkGeom<R, K>::BW];
};
/* list entry of a tile in flight: tile | phase << 28, simulation, first
 * cell, the flag of its output buffer */
struct BulkEntry {
  int item, s, x0, y0, have;
};
template <typename R, int K>
struct alignas(128) BulkWarpSmem {
  BulkStage<R, K> st[BulkGeom<R, K>::NST];
  unsigned long long bar[BulkGeom<R, K>::NST];
  BulkEntry meta[BulkGeom<R, K>::NST];
};
/* dynamic shared memory of kf_bulk (the base is rounded up to 128 bytes in
 * the kernel) */
template <typename R, int K>
constexpr size_t bulk_smem_bytes() {
  return (NT / 32) * sizeof(BulkWarpSmem<R, K>) + 128;
}

/* The FP64 bulk update of one cell (stage row i, column j) of phase p with
 * every term of the K x K matrices: the expressions of a non-DIAG kernel in
 * their order (calculate_divergence_concentration.h:43-57 through
 * functionF_01.h:19-37).  A DIAG kernel calls it, after a tile's rows, for
 * the rare cells whose result was not finite. */
template <int K, bool MUL>
__device__ __forceinline__ void bulk_cell_full_f64(const double *__restrict__ st, int i, int j,
                                                const Consts<double> *__restrict__ Dp, int p, const double *m,
                                                double *nm, double *dmu) {
  constexpr int BW = BulkGeom<double, K>::BW;
  const Consts<double> &D = *Dp;
  const double idx = D.inv_dx, idy = D.inv_dy, ddx = D.dx, ddy = D.dy, dt = D.dt;
  const double cst = D.obstacle ? D.jat_obst : D.jat_well;
  double divjat = bdiv<MUL>((0.0 - 0.0) * cst, idx, ddx);
  divjat += bdiv<MUL>((0.0 - 0.0) * cst, idy, ddy);
#define BM(l, r, c) st[((l) * SH + (r)) * BW + (c)]
  double cn[K];
#pragma unroll
  for (int k = 0; k < K; k++) {
    double divflux = 0.0;
#pragma unroll
    for (int l = 0; l < K; l++) {
      const double Dv = D.Dbulk[p][k][l];
      const double dm = (Dv + Dv) * 0.5, c = BM(l, i, j);
      const double fx = dm * bdiv<MUL>(BM(l, i + 1, j) - c, idx, ddx);
      const double bx_ = dm * bdiv<MUL>(c - BM(l, i - 1, j), idx, ddx);
      const double fy = dm * bdiv<MUL>(BM(l, i, j + 1) - c, idy, ddy);
      const double by_ = dm * bdiv<MUL>(c - BM(l, i, j - 1), idy, ddy);
      divflux += bdiv<MUL>(fx - bx_, idx, ddx);
      divflux += bdiv<MUL>(fy - by_, idy, ddy);
    }
    double cm = 0.0;   /* c_mu (functionF_01.h:30-37) */
#pragma unroll
    for (int l = 0; l < K; l++) cm += D.cmu[p][k][l] * (m[l] - D.E[p][l]);
    cn[k] = cm + dt * (divflux) - divjat;
  }
#undef BM
#pragma unroll
  for (int k = 0; k < K; k++) {
    double sm = D.twoA[p][k] * cn[k] + D.E[p][k];   /* Mu (functionF_01.h:19-29) */
#pragma unroll
    for (int l = 0; l < K; l++)
      if (k != l) sm += D.A[p][k][l] * cn[l];
    nm[k] = sm;
    dmu[k] = sm - m[k];
  }
}

/* Bulk tiles, one warp per tile.  Warps take contiguous ranges of the bulk
 * list.  Lane 0 issues one TMA box per tile (the K mu planes of the tile with
 * a one-cell halo, rows x0-1..x0+TX) into the warp's next stage while the warp
 * steps the current one; an mbarrier per stage counts the bytes in.  Halo
 * cells outside the domain (tiles on the boundary) are then overwritten with
 * the cells the boundary copy tables name.  Lane j steps column y0+j row by
 * row.  No block-wide barrier anywhere.  The running mu extremes of the cells
 * a warp steps stay in registers and are merged into the simulation's slots
 * (atomic max/min) when the warp moves to another simulation or finishes;
 * bulk tiles cannot move the phi extremes (their phi is 0 or 1, inside the
 * initial [0, 1]).  A stage whose bytes do not arrive within the poll limit
 * sets ctr[CTR_ERR]; the warp then stops taking tiles. */
template <typename R, int N, int K, bool SUMS, bool MUL, bool DIAG>
__device__ __forceinline__ void bulk_tiles(const SimDesc *__restrict__ sims, const Consts<R> *__restrict__ consts,
                                           const int *__restrict__ tsim, const int4 *__restrict__ blist,
                                           const TensorMapSlot *__restrict__ tmaps, int buf,
                                           const R *__restrict__ state, R *__restrict__ next,
                                           TileFlags *__restrict__ flag_out, int *__restrict__ ctr, StatBufs st,
                                           unsigned char *smraw) {
  using G = BulkGeom<R, K>;
  constexpr int NS = 2 * N + 2 * K + 1, NST = G::NST, CO = G::CO;
  unsigned char *sbase = (unsigned char *)(((size_t)smraw + 127) & ~(size_t)127);
  BulkWarpSmem<R, K> &ws = reinterpret_cast<BulkWarpSmem<R, K> *>(sbase)[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int nbulk = *(const volatile int *)(ctr + CTR_BULK);

  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < NST; q++) mbar_init(smem_addr(&ws.bar[q]), 1);
    fence_barrier_init();
    fence_proxy_async_smem();
  }
  __syncwarp();

  R emax[K], emin[K];   /* running mu extremes of the cells this warp stepped */
#pragma unroll
  for (int k = 0; k < K; k++) { emax[k] = -INFINITY; emin[k] = INFINITY; }
  int cur_sim = -1;
  auto flush = [&](int s) {
#pragma unroll
    for (int k = 0; k < K; k++) {
      const double a = warp_max(emax[k]), c = warp_min(emin[k]);
      if (lane == 0 && st.ext) {
        long long *slot = st.ext + (long long)s * (2 * (N + K));
        if (a > -INFINITY) atomicMax(slot + 2 * N + k, ord(a));
        if (c < INFINITY) atomicMin(slot + 2 * N + K + k, ord(c));
      }
      emax[k] = -INFINITY;
      emin[k] = INFINITY;
    }
  };

  /* Work comes in chunks of list entries taken from the bulk head counter
   * (one atomic per warp and chunk), so warps that run faster take more; the
   * chunk size shrinks as the list drains (a few chunks per warp in all; the
   * batch's launch shape sets the largest chunk and the divisor).
   * Two chunks are held: A (being issued) and B (next).  Lane h*16+r holds
   * entry r of the chunk in half h; B's entries are loaded when it is taken,
   * one 16-byte load per lane, and used one tile later. */
  constexpr int BCH = 16;
  const int nwarps = gridDim.x * (NT / 32);
  int q_item = 0, q_s = 0, q_xy = 0;   /* q_s: simulation | output flag << 24; q_xy: tile row << 16 | column */
  auto grab = [&](int half, int &start, int &n) {
    int v = 0, c = 0;
    if (lane == 0) {
      const int left = nbulk - *(volatile int *)(ctr + CTR_BHEAD);
      c = max(2, min(min(BCH, st.bch_max), left / (st.bch_div * nwarps)));
      v = atomicAdd(ctr + CTR_BHEAD, c);
    }
    start = __shfl_sync(0xffffffffu, v, 0);
    c = __shfl_sync(0xffffffffu, c, 0);
    n = max(0, min(c, nbulk - start));
    const int r = lane - 16 * half;
    if (r >= 0 && r < n) {
      const int4 e = __ldg(blist + start + r);
      q_item = e.x;
      q_s = e.y;
      q_xy = e.z;
    }
  };
  int ha = 0, na = 0, pa = 0;   /* chunk A: half, entries, next to issue */
  int cb = 0, nb = 0;           /* chunk B (half ha ^ 1) */
  {
    int ca = 0;
    grab(0, ca, na);
  }
  if (na > 0) grab(1, cb, nb);
  /* the next entry in issue order; false when the list is used up */
  auto next_entry = [&](BulkEntry &en) {
    if (pa == na) {
      if (nb == 0) return false;
      ha ^= 1;
      na = nb;
      pa = 0;
      grab(ha ^ 1, cb, nb);
    }
    const int r = 16 * ha + pa;
    en.item = __shfl_sync(0xffffffffu, q_item, r);
    const int sh = __shfl_sync(0xffffffffu, q_s, r), xy = __shfl_sync(0xffffffffu, q_xy, r);
    en.s = sh & 0xffffff;
    en.have = (signed char)(sh >> 24);
    en.x0 = (xy >> 16) * TX;
    en.y0 = (xy & 0xffff) * TY;
    pa++;
    return true;
  };
  /* lane 0: start the TMA box of a tile into stage b and note its entry */
  auto issue = [&](const BulkEntry &en, int b) {
    if (lane == 0) {
      ws.meta[b] = en;
      const unsigned bar = smem_addr(&ws.bar[b]);
      mbar_expect_tx(bar, G::BOX_BYTES + st.tma_extra);
      tma_load_3d(smem_addr(&ws.st[b]), tmaps + 2 * en.s + buf, en.y0 - 1 - CO, en.x0 - 1, 0, bar);
    }
  };

  /* the current simulation's layout and the current (simulation, phase)'s
   * constants stay in registers while consecutive tiles share them */
  Grid g = {};
  long long off_state = 0;
  int cur_key = -1;
  R idx = R(0), idy = R(0), ddx = R(1), ddy = R(1), dt = R(0), divjat = R(0);
  /* the K x K constants of a phase: diffusive flux factor, c_mu, A and
   * dmu/dc */
  struct MatC {
    R dm[K][K], cmu[K][K], A[K][K], muc[K][K];
  };
  auto load_mat = [&](MatC &c, const Consts<R> &D, int p) {
#pragma unroll
    for (int k = 0; k < K; k++)
#pragma unroll
      for (int l = 0; l < K; l++) {
        const R Dv = D.Dbulk[p][k][l];
        c.dm[k][l] = (Dv + Dv) * R(0.5);
        c.cmu[k][l] = D.cmu[p][k][l];
        c.A[k][l] = D.A[p][k][l];
        c.muc[k][l] = (R)D.muc64[p][k][l];
      }
  };
  R E[K], twoA[K];
  MatC mc;
  /* FP32: flux-divergence coefficients of the bulk update (x and y) */
  f2 CX2[K][K], CY2[K][K];
  /* FP32: the step's part of the rounding key */
  const unsigned skey = sizeof(R) == 4 ? mix32(__ldg(st.round_step) * 0x9e3779b9u + 0x632be5abu) : 0u;

  /* the qi-th box a warp issues goes to stage qi % NST and completes phase
   * (qi / NST) & 1 of that stage's barrier; NST-1 boxes are in flight while a
   * tile is stepped */
  int qi = 0, ci = 0;
  for (int q = 0; q < NST - 1; q++) {
    BulkEntry en;
    if (!next_entry(en)) break;
    issue(en, qi % NST);
    qi++;
  }
  __syncwarp();
  while (ci < qi) {
    {
      BulkEntry en;
      if (next_entry(en)) {   /* into the stage of tile ci-1, stepped already */
        issue(en, qi % NST);
        qi++;
      }
    }
    const int b = ci % NST;
    if (!mbar_wait(smem_addr(&ws.bar[b]), (ci / NST) & 1, st.mbar_tries)) {
      /* bytes missing: record it, wait (bounded) for the other boxes in
       * flight, step nothing more */
      if (lane == 0) atomicExch(ctr + CTR_ERR, 1);
      for (int q = ci + 1; q < qi; q++) mbar_wait(smem_addr(&ws.bar[q % NST]), (q / NST) & 1, st.mbar_tries);
      break;
    }
    ci++;
    /* ---- step bulk tile t (phase p) from stage b */
    const BulkEntry cur = ws.meta[b];
    const int t = cur.item & 0x0fffffff, p = cur.item >> 28, s = cur.s;
    const int x0 = cur.x0, y0 = cur.y0, have = cur.have;
    const Consts<R> &D = consts[s];
    if (s != cur_sim) {
      if (cur_sim >= 0) flush(cur_sim);
      cur_sim = s;
      g = sims[s].g;
      off_state = sims[s].off_state;
    }
    if (cur_key != s * 16 + p) {
      cur_key = s * 16 + p;
      idx = D.inv_dx; idy = D.inv_dy; ddx = D.dx; ddy = D.dy; dt = D.dt;
      const R cst = D.obstacle ? D.jat_obst : D.jat_well;
      /* the anti-trapping divergence of a bulk cell: no phi gradient, the
       * same value for every cell */
      divjat = bdiv<MUL>((R(0.0) - R(0.0)) * cst, idx, ddx);
      divjat += bdiv<MUL>((R(0.0) - R(0.0)) * cst, idy, ddy);
#pragma unroll
      for (int k = 0; k < K; k++) {
        E[k] = D.E[p][k];
        twoA[k] = D.twoA[p][k];
      }
      /* a DIAG kernel keeps only the diagonals live */
      load_mat(mc, D, p);
      if constexpr (sizeof(R) == 4) {
        /* dt * sum_l (dmu/dc)_kl D_lm / dx^2 (and / dy^2), from the FP64
         * constants, rounded once */
        const double dtd = (double)D.dt, ix = 1.0 / (double)D.dx, iy = 1.0 / (double)D.dy;
#pragma unroll
        for (int k = 0; k < K; k++)
#pragma unroll
          for (int m = 0; m < K; m++) {
            double sv = 0.0;
#pragma unroll
            for (int l = 0; l < K; l++) sv += D.muc64[p][k][l] * (double)D.Dbulk[p][l][m];
            const float cx = (float)(sv * dtd * ix * ix), cy = (float)(sv * dtd * iy * iy);
            CX2[k][m] = f2pack(cx, cx);
            CY2[k][m] = f2pack(cy, cy);
          }
      }
    }
    BulkStage<R, K> &sg = ws.st[b];
    const int rows = min(TX, g.mx - x0), ncols = min(TY, g.my - y0);
    if (x0 == 0 || x0 + TX >= g.mx || y0 == 0 || y0 + TY >= g.my) {
      /* boundary tile: halo cells outside the domain are copies of interior
       * cells (the box read zeros there) */
      const R *mu = state + off_state + (long long)N * g.plane;
      const int bx0 = D.bc_x[1][0], bx1 = D.bc_x[1][1], by0 = D.bc_y[1][0], by1 = D.bc_y[1][1];
      for (int e = lane; e < 2 * SW + 2 * SH; e += 32) {
        int i, j;
        bool need;
        if (e < 2 * SW) {   /* halo rows x0-1 (top) and x0+rows (bottom) */
          const int side = e >= SW;
          j = e - side * SW;
          i = side ? rows + 1 : 0;
          need = side ? x0 + TX >= g.mx : x0 == 0;
        } else {            /* halo columns y0-1 (left) and y0+ncols (right) */
          const int side = e >= 2 * SW + SH;
          i = e - 2 * SW - side * SH;
          j = side ? ncols + 1 : 0;
          need = side ? y0 + TY >= g.my : y0 == 0;
        }
        int x = x0 - 1 + i, y = y0 - 1 + j;
        if (need && x <= g.mx && y <= g.my) {
          if (x < 0 || x >= g.mx) x = remap(x, g.mx, bx0, bx1);
          if (y < 0 || y >= g.my) y = remap(y, g.my, by0, by1);
          const R *src = mu + (long long)x * g.pitch + y;
#pragma unroll
          for (int k = 0; k < K; k++) sg.M[k][i][j + CO] = __ldg(src + (long long)k * g.plane);
        }
      }
      fence_proxy_async_smem();   /* before a later box overwrites this stage */
      __syncwarp();
    }
    R *phin = next + off_state;
    R *mun = phin + (long long)N * g.plane;
    /* lane 16h + q steps tile rows 4h..4h+3 at columns 2q and 2q+1: stage
     * columns c and c+1 (c = 2q + 1 + CO, so the pair is 16-byte aligned in
     * FP64 and 8-byte aligned in FP32); the y-face between the two cells is
     * computed once, and the x-face below a row is carried to the next */
    const int hh = lane >> 4, qq = lane & 15;
    const int jc = 2 * qq, c = jc + 1 + CO, y = y0 + jc;
    const bool v0 = y < g.my, v1 = y + 1 < g.my;
    const int r0 = 4 * hh, nr = max(0, min(4, rows - r0));
    double acc[SUMS ? NS : 1];
#pragma unroll
    for (int f = 0; f < (SUMS ? NS : 1); f++) acc[f] = 0.0;
    /* the progress sums of one new cell of phase p */
    auto sum_cell = [&](const R (&nm)[K], const double (&dmu)[K]) {
      if constexpr (SUMS) {
        R nph[N];
#pragma unroll
        for (int a = 0; a < N; a++) nph[a] = a == p ? R(1.0) : R(0.0);
#pragma unroll
        for (int k = 0; k < K; k++) acc[N + k] += dmu[k] * dmu[k];
#pragma unroll
        for (int a = 0; a < N; a++) acc[N + K + a] += (double)nph[a];
#pragma unroll
        for (int k = 0; k < K; k++) {
          R comp = R(0.0);
#pragma unroll
          for (int b2 = 0; b2 < N; b2++) comp += c_mu<R, K>(D, nm, b2, k) * h<R, N>(nph, b2);
          acc[2 * N + K + k] += (double)comp;
        }
        bool bad = false;
#pragma unroll
        for (int k = 0; k < K; k++) bad |= !isfinite(nm[k]);
        acc[NS - 1] += bad ? 1.0 : 0.0;
      }
    };
    /* FP64: the new mu of a cell from its old mu and the flux divergences,
     * every term of the K x K matrices (non-DIAG kernels) */
    auto commit_mu = [&](const MatC &mt, const R (&m)[K], const R (&df)[K], R (&nm)[K], double (&dmu)[K]) {
      R cn[K];
#pragma unroll
      for (int k = 0; k < K; k++) {
        R cm = R(0.0);   /* c_mu (functionF_01.h:30-37) */
#pragma unroll
        for (int l = 0; l < K; l++) cm += mt.cmu[k][l] * (m[l] - E[l]);
        cn[k] = cm + dt * (df[k]) - divjat;
      }
#pragma unroll
      for (int k = 0; k < K; k++) {
        R sm = twoA[k] * cn[k] + E[k];   /* Mu (functionF_01.h:19-29) */
#pragma unroll
        for (int l = 0; l < K; l++)
          if (k != l) sm += mt.A[k][l] * cn[l];
        nm[k] = sm;
        dmu[k] = (double)nm[k] - (double)m[k];
      }
    };
    if (v0 && nr > 0) {
      if constexpr (sizeof(R) == 8) {
        /* ---- FP64: the reference's bulk expressions (update_tile's uniform
         * path) in their order, two cells at a time */
        double2 P[K], FXP[K][K];
        unsigned redo = 0;   /* DIAG: bit 2 rr + e, cell e of row rr to redo with every term */
#pragma unroll
        for (int l = 0; l < K; l++) {
          const double2 pp = *reinterpret_cast<const double2 *>(&sg.M[l][r0][c]);
          P[l] = *reinterpret_cast<const double2 *>(&sg.M[l][r0 + 1][c]);
          const R g0 = bdiv<MUL>(P[l].x - pp.x, idx, ddx), g1 = bdiv<MUL>(P[l].y - pp.y, idx, ddx);
#pragma unroll
          for (int k = 0; k < K; k++)
            if (!DIAG || l == k) FXP[k][l] = make_double2(mc.dm[k][l] * g0, mc.dm[k][l] * g1);
        }
        for (int rr = 0; rr < nr; rr++) {
          const int i = r0 + 1 + rr, x = x0 + i - 1;
          double2 Pn[K];
          R m0[K], m1[K], n0[K], n1[K];
          double d0[K], d1[K];
#pragma unroll
          for (int k = 0; k < K; k++) { m0[k] = P[k].x; m1[k] = P[k].y; }
          if constexpr (DIAG) {
            /* only the diagonal terms: one component at a time */
#pragma unroll
            for (int k = 0; k < K; k++) {
              Pn[k] = *reinterpret_cast<const double2 *>(&sg.M[k][i + 1][c]);
              const R L = sg.M[k][i][c - 1], Rn = sg.M[k][i][c + 2];
              const R dm = mc.dm[k][k];
              const R fx0 = dm * bdiv<MUL>(Pn[k].x - P[k].x, idx, ddx);
              const R fx1 = dm * bdiv<MUL>(Pn[k].y - P[k].y, idx, ddx);
              const R fl = dm * bdiv<MUL>(P[k].x - L, idy, ddy);
              const R fm = dm * bdiv<MUL>(P[k].y - P[k].x, idy, ddy);
              const R fr = dm * bdiv<MUL>(Rn - P[k].y, idy, ddy);
              R a0 = R(0.0), a1 = R(0.0);
              a0 += bdiv<MUL>(fx0 - FXP[k][k].x, idx, ddx);
              a0 += bdiv<MUL>(fm - fl, idy, ddy);
              a1 += bdiv<MUL>(fx1 - FXP[k][k].y, idx, ddx);
              a1 += bdiv<MUL>(fr - fm, idy, ddy);
              FXP[k][k] = make_double2(fx0, fx1);
              /* c_mu, the bulk update and Mu (functionF_01.h:19-37) of the
               * pure phase, diagonal terms only */
              R cm0 = R(0.0), cm1 = R(0.0);
              cm0 += mc.cmu[k][k] * (m0[k] - E[k]);
              cm1 += mc.cmu[k][k] * (m1[k] - E[k]);
              const R cn0 = cm0 + dt * (a0) - divjat, cn1 = cm1 + dt * (a1) - divjat;
              n0[k] = twoA[k] * cn0 + E[k];
              n1[k] = twoA[k] * cn1 + E[k];
              d0[k] = (double)n0[k] - (double)m0[k];
              d1[k] = (double)n1[k] - (double)m1[k];
            }
          } else {
            R gx0[K], gx1[K], gl[K], gm[K], gr[K];
#pragma unroll
            for (int l = 0; l < K; l++) {
              Pn[l] = *reinterpret_cast<const double2 *>(&sg.M[l][i + 1][c]);
              const R L = sg.M[l][i][c - 1], Rn = sg.M[l][i][c + 2];
              gx0[l] = bdiv<MUL>(Pn[l].x - P[l].x, idx, ddx);
              gx1[l] = bdiv<MUL>(Pn[l].y - P[l].y, idx, ddx);
              gl[l] = bdiv<MUL>(P[l].x - L, idy, ddy);
              gm[l] = bdiv<MUL>(P[l].y - P[l].x, idy, ddy);
              gr[l] = bdiv<MUL>(Rn - P[l].y, idy, ddy);
            }
            R df0[K], df1[K];
#pragma unroll
            for (int k = 0; k < K; k++) {
              R a0 = R(0.0), a1 = R(0.0);
#pragma unroll
              for (int l = 0; l < K; l++) {
                const R dm = mc.dm[k][l];
                const R fx0 = dm * gx0[l], fx1 = dm * gx1[l];
                const R fl = dm * gl[l], fm = dm * gm[l], fr = dm * gr[l];
                a0 += bdiv<MUL>(fx0 - FXP[k][l].x, idx, ddx);
                a0 += bdiv<MUL>(fm - fl, idy, ddy);
                a1 += bdiv<MUL>(fx1 - FXP[k][l].y, idx, ddx);
                a1 += bdiv<MUL>(fr - fm, idy, ddy);
                FXP[k][l] = make_double2(fx0, fx1);
              }
              df0[k] = a0;
              df1[k] = a1;
            }
            commit_mu(mc, m0, df0, n0, d0);
            commit_mu(mc, m1, df1, n1, d1);
          }
          /* a left-out term is +-0 only when the values it multiplies are
           * finite, and they are when every new mu is; otherwise (DIAG) the
           * cell is redone with every term after the rows (its extremes and
           * sums are taken then) */
          bool f0 = true, f1 = v1;
          if constexpr (DIAG) {
#pragma unroll
            for (int k = 0; k < K; k++) { f0 &= fabs(n0[k]) < R(INFINITY); f1 &= fabs(n1[k]) < R(INFINITY); }
            redo |= (f0 ? 0u : 1u) << (2 * rr);
            redo |= (v1 && !f1 ? 2u : 0u) << (2 * rr);
          }
          const long long o = (long long)x * g.pitch + y;
          /* the statistics take the cells of their rows */
          const bool srow = stat_row(g, x);
          f0 = f0 && srow;
          f1 = f1 && srow;
#pragma unroll
          for (int k = 0; k < K; k++) {
            if (v1) *reinterpret_cast<double2 *>(mun + k * g.plane + o) = make_double2(n0[k], n1[k]);
            else mun[k * g.plane + o] = n0[k];
            /* NaN is ignored by fmax/fmin; a cell to be redone is left out */
            const R x0 = f0 ? n0[k] : R(NAN), x1 = f1 ? n1[k] : R(NAN);
            emax[k] = fmax(emax[k], fmax(x0, x1));
            emin[k] = fmin(emin[k], fmin(x0, x1));
          }
          if (have != p) {
#pragma unroll
            for (int a = 0; a < N; a++) {
              const R v = a == p ? R(1.0) : R(0.0);
              if (v1) *reinterpret_cast<double2 *>(phin + a * g.plane + o) = make_double2(v, v);
              else phin[a * g.plane + o] = v;
            }
          }
          if (f0) sum_cell(n0, d0);
          if (f1) sum_cell(n1, d1);
#pragma unroll
          for (int l = 0; l < K; l++) P[l] = Pn[l];
        }
        if constexpr (DIAG) {
          while (redo) {
            const int bit = __ffs(redo) - 1;
            redo &= redo - 1;
            const int i = r0 + 1 + (bit >> 1), cc = c + (bit & 1), x = x0 + i - 1;
            R m[K], nm[K];
            double dmu[K];
#pragma unroll
            for (int k = 0; k < K; k++) m[k] = sg.M[k][i][cc];
            bulk_cell_full_f64<K, MUL>(&sg.M[0][0][0], i, cc, &D, p, m, nm, dmu);
            const long long o = (long long)x * g.pitch + y + (bit & 1);
            const bool srow = stat_row(g, x);
#pragma unroll
            for (int k = 0; k < K; k++) {
              mun[k * g.plane + o] = nm[k];
              if (srow) {
                emax[k] = fmax(emax[k], nm[k]);
                emin[k] = fmin(emin[k], nm[k]);
              }
            }
            if (srow) sum_cell(nm, dmu);
          }
        }
      } else {
        /* ---- FP32: the new mu of a bulk cell is mu + sum_m (CX[k][m] lapx(mu_m)
         * + CY[k][m] lapy(mu_m)) -- the flux divergence of the pure phase's
         * constant D times dt and dmu/dc folded into one coefficient per
         * direction -- in packed f32x2 arithmetic on the cell pair, rounded
         * stochastically by dithering: RN(mu + (s + w ulp(mu))) with w
         * uniform in [-1/2, 1/2) takes the upper neighbour with probability
         * equal to the fraction of the ulp. */
        f2 P[K], DXP[K];
#pragma unroll
        for (int m = 0; m < K; m++) {
          const f2 pp = *reinterpret_cast<const f2 *>(&sg.M[m][r0][c]);
          P[m] = *reinterpret_cast<const f2 *>(&sg.M[m][r0 + 1][c]);
          DXP[m] = f2sub(P[m], pp);
        }
        unsigned rng = mix32(skey ^ ((unsigned)(x0 + r0) * 0x85ebca6bu + (unsigned)y * 0xc2b2ae35u));
        for (int rr = 0; rr < nr; rr++) {
          const int i = r0 + 1 + rr, x = x0 + i - 1;
          f2 Pn[K], LX[K], LY[K];
#pragma unroll
          for (int m = 0; m < K; m++) {
            Pn[m] = *reinterpret_cast<const f2 *>(&sg.M[m][i + 1][c]);
            const float L = (float)sg.M[m][i][c - 1], Rn = (float)sg.M[m][i][c + 2];
            const f2 dxn = f2sub(Pn[m], P[m]);
            LX[m] = f2sub(dxn, DXP[m]);
            DXP[m] = dxn;
            const float px = f2lo(P[m]), py = f2hi(P[m]);
            const f2 o = f2sub(f2pack(px, Rn), f2pack(L, py));   /* (yl, yr) */
            const float ym = __fsub_rn(py, px);
            LY[m] = f2sub(f2pack(ym, f2hi(o)), f2pack(f2lo(o), ym));
          }
          const long long o = (long long)x * g.pitch + y;
          const bool srow = stat_row(g, x);
          R n0[K], n1[K];
          double d0[K], d1[K];
#pragma unroll
          for (int k = 0; k < K; k++) {
            f2 sdm = f2mul(CY2[k][k], LY[k]);
            sdm = f2fma(CX2[k][k], LX[k], sdm);
            if constexpr (!DIAG) {
#pragma unroll
              for (int m = 0; m < K; m++) {
                if (m == k) continue;
                sdm = f2fma(CY2[k][m], LY[m], sdm);
                sdm = f2fma(CX2[k][m], LX[m], sdm);
              }
            }
            const float m0 = f2lo(P[k]), m1 = f2hi(P[k]);
            rng = rng * 1664525u + 1013904223u;
            const float w0 = __uint_as_float(0x3f800000u | (rng >> 9)) - 1.5f;
            rng = rng * 1664525u + 1013904223u;
            const float w1 = __uint_as_float(0x3f800000u | (rng >> 9)) - 1.5f;
            const f2 nm = f2add(P[k], f2fma(f2pack(w0, w1), f2pack(ulpf(m0), ulpf(m1)), sdm));
            n0[k] = f2lo(nm);
            n1[k] = f2hi(nm);
            d0[k] = (double)f2lo(sdm);
            d1[k] = (double)f2hi(sdm);
            if (v1) {
              *reinterpret_cast<f2 *>(mun + k * g.plane + o) = nm;
              if (srow) {
                emax[k] = fmax3f(emax[k], n0[k], n1[k]);
                emin[k] = fmin3f(emin[k], n0[k], n1[k]);
              }
            } else {
              mun[k * g.plane + o] = n0[k];
              if (srow) {
                emax[k] = fmaxf(emax[k], n0[k]);
                emin[k] = fminf(emin[k], n0[k]);
              }
            }
          }
          if (have != p) {
#pragma unroll
            for (int a = 0; a < N; a++) {
              const R v = a == p ? R(1.0) : R(0.0);
              if (v1) *reinterpret_cast<f2 *>(phin + a * g.plane + o) = f2pack(v, v);
              else phin[a * g.plane + o] = v;
            }
          }
          if (srow) {
            sum_cell(n0, d0);
            if (v1) sum_cell(n1, d1);
          }
#pragma unroll
          for (int m = 0; m < K; m++) P[m] = Pn[m];
        }
      }
    }
    if constexpr (SUMS) {
#pragma unroll
      for (int f = 0; f < NS; f++) {
        const double r = warp_sum(acc[f]);
        if (lane == 0) st.partials[(long long)t * NS + f] = r;
      }
    }
    if (lane == 0) flag_out[t] = uniform_flags(p);
    __syncwarp();   /* stage b is refilled by a later issue */
  }
  if (cur_sim >= 0) flush(cur_sim);
}

/* End of a warp's bulk tiles when the same shared memory is used otherwise
 * afterwards: its stage barriers are invalidated (every box it issued has
 * completed or been waited for). */
template <typename R, int K>
__device__ __forceinline__ void bulk_release_warp(unsigned char *smraw) {
  unsigned char *sbase = (unsigned char *)(((size_t)smraw + 127) & ~(size_t)127);
  BulkWarpSmem<R, K> &ws = reinterpret_cast<BulkWarpSmem<R, K> *>(sbase)[threadIdx.x >> 5];
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int q = 0; q < BulkGeom<R, K>::NST; q++)
      asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smem_addr(&ws.bar[q])) : "memory");
  }
  __syncwarp();
}

template <typename R, int N, int K, bool SUMS, bool MUL, bool DIAG>
__global__ void __launch_bounds__(NT, sizeof(R) == 4 && K == 1 ? 3 : 2) kf_bulk(const SimDesc *__restrict__ sims, const Consts<R> *__restrict__ consts,
                                                 const int *__restrict__ tsim, const int4 *__restrict__ blist,
                                                 const TensorMapSlot *__restrict__ tmaps, int buf,
                                                 const R *__restrict__ state, R *__restrict__ next,
                                                 TileFlags *__restrict__ flag_out, int *__restrict__ ctr,
                                                 int ndone, StatBufs st) {
  extern __shared__ __align__(16) unsigned char smraw[];
  bulk_tiles<R, N, K, SUMS, MUL, DIAG>(sims, consts, tsim, blist, tmaps, buf, state, next, flag_out, ctr, st, smraw);
  step_finish(ctr, ndone);
}

/* Interface tiles of one step: the CTA takes tiles from the interface list
 * until it is empty.  Each simulation's constants are copied into shared
 * memory when the CTA moves to it.  Not inlined: the step kernel and the
 * interface-only kernel share one copy of this code. */
template <typename R, int N, int K, bool ANISO, bool MUL>
__device__ __noinline__ void general_tiles(const SimDesc *__restrict__ sims, const Consts<R> *__restrict__ consts,
                                           const int *__restrict__ tsim, const R *__restrict__ state,
                                           R *__restrict__ next, TileFlags *__restrict__ flag_out,
                                           const int *__restrict__ glist, int *__restrict__ ctr, StatBufs st,
                                           unsigned char *smraw) {
  GenSmem<R, N, K> &sm = *reinterpret_cast<GenSmem<R, N, K> *>(smraw);
  __shared__ Consts<R> sc;
  __shared__ int s_item;
  const int nlist = *(volatile int *)(ctr + CTR_LIST);
  int cur_sim = -1;
  if (threadIdx.x == 0) {   /* the tile's list counters (reset again after each tile) */
    sm.nlist = 0;
    sm.nflist = 0;
  }
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(ctr + CTR_HEAD, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= nlist) break;
    const int t = __ldg(glist + item);
    const int s = __ldg(tsim + t);
    if (s != cur_sim) {
      load_consts(sc, consts + s);
      cur_sim = s;
      __syncthreads();
    }
    const SimDesc sd = sims[s];
    const int lt = t - sd.tile0, by = lt / sd.tiles_x, bx = lt - by * sd.tiles_x;
    const R *ph = state + sd.off_state;
    R *nx = next + sd.off_state;
    using CT = typename std::conditional<MUL, ConstsMul<R>, Consts<R>>::type;
    const double *tpf = st.trows ? st.trows + sd.off_T : nullptr;
    const double *tcc = tpf ? tpf + (sd.g.my + 6) : nullptr;
    const TileFlags f = general_tile<R, N, K, ANISO>(static_cast<const CT &>(sc), sd.g, ph, ph + (long long)N * sd.g.plane, nx,
                                                       nx + (long long)N * sd.g.plane, by * TX, bx * TY, st, s, t,
                                                       sm, tpf, tcc);
    if (threadIdx.x == 0) flag_out[t] = f;
    __syncthreads();
  }
}

template <typename R, int N, int K, bool ANISO, bool MUL>
__global__ void __launch_bounds__(NT, (N <= 3 ? 2 : 1)) kf_general(const SimDesc *__restrict__ sims,
                                                 const Consts<R> *__restrict__ consts, const int *__restrict__ tsim,
                                                 const R *__restrict__ state, R *__restrict__ next,
                                                 TileFlags *__restrict__ flag_out, const int *__restrict__ glist,
                                                 int *__restrict__ ctr, int ndone, StatBufs st) {
  extern __shared__ __align__(16) unsigned char smraw[];
  general_tiles<R, N, K, ANISO, MUL>(sims, consts, tsim, state, next, flag_out, glist, ctr, st, smraw);
  step_finish(ctr, ndone);
}

/* One step in one persistent launch: each CTA takes interface tiles while
 * the interface list lasts, then its warps take bulk tiles, so the two kinds
 * of work share the SMs and the step ends with one tail instead of two. */
template <typename R, int N, int K, bool ANISO, bool MUL, bool DIAG>
__global__ void __launch_bounds__(NT, (N <= 3 ? 2 : 1)) kf_step(const SimDesc *__restrict__ sims,
                                                 const Consts<R> *__restrict__ consts, const int *__restrict__ tsim,
                                                 const int4 *__restrict__ blist, const int *__restrict__ glist,
                                                 const TensorMapSlot *__restrict__ tmaps, int buf,
                                                 const R *__restrict__ state, R *__restrict__ next,
                                                 TileFlags *__restrict__ flag_out, int *__restrict__ ctr,
                                                 int ndone, StatBufs st) {
  extern __shared__ __align__(16) unsigned char smraw[];
  if (st.mixed && (blockIdx.x & 1)) {
    /* bulk tiles first, then whatever is left of the interface list: the two
     * kinds of work share every SM from the start of the step */
    bulk_tiles<R, N, K, false, MUL, DIAG>(sims, consts, tsim, blist, tmaps, buf, state, next, flag_out, ctr, st,
                                          smraw);
    bulk_release_warp<R, K>(smraw);
    __syncthreads();   /* the bulk stages' shared memory becomes the interface tile's */
    general_tiles<R, N, K, ANISO, MUL>(sims, consts, tsim, state, next, flag_out, glist, ctr, st, smraw);
  } else {
    general_tiles<R, N, K, ANISO, MUL>(sims, consts, tsim, state, next, flag_out, glist, ctr, st, smraw);
    __syncthreads();   /* the interface tiles' shared memory becomes the bulk stages */
    bulk_tiles<R, N, K, false, MUL, DIAG>(sims, consts, tsim, blist, tmaps, buf, state, next, flag_out, ctr, st,
                                          smraw);
  }
  step_finish(ctr, ndone);
}

/* Per simulation, the moving-frame state the temperature rows need: the
 * offset of the frame, and after a shift the offset and distance the
 * shifted temperature field was laid down with (consumed by the next step). */
struct SimDyn {
  long long shift_off;   /* shift_OFFSET (microsim_gp.c:122) */
  long long shift_T;     /* the offset of the temperature field being shifted */
  int dlast;             /* its shift distance */
  int fresh;             /* a shift happened at the end of the last step */
  int pos;               /* MAX_INTERFACE_POS of the last check */
  int pad;
};

/* The temperature of every ghosted column y of a non-isothermal simulation
 * during the coming step, one CTA per simulation.  The reference's field is
 * temp_bottom + y*GRADIENT (apply_temperature_gradientY, Temperature_gradient.h:4-29),
 * laid down after each step with the step's BASE_POS (microsim_gp.c:108-113;
 * at t = 0 without the velocity term, :77-82) and copied into the ghost
 * columns only by the next boundary copy: the phase-field pass of step t+1
 * reads the field as laid down (as copied at t = 0, where the start-up copy
 * came after it), the concentration pass reads it copied.  After a moving-
 * frame shift the field holds the shifted columns (shift.h:20) until the
 * next step lays it down again.  Rows: [0, MESH_Y+6) as the phase-field pass
 * reads them, then [0, MESH_Y+6) as the concentration pass reads them. */
template <typename R>
__global__ void __launch_bounds__(128) kt_rows(const SimDesc *__restrict__ sims, const Consts<R> *__restrict__ consts,
                                               const int *__restrict__ ctr, SimDyn *__restrict__ dyn,
                                               double *__restrict__ trows) {
  const int s = blockIdx.x;
  const Consts<R> &D = consts[s];
  if (!D.tgrad) return;
  const SimDesc sd = sims[s];
  const int my = sd.g.my, ry = my + 6;
  const long t0 = (long)(unsigned)ctr[CTR_STEP];
  const SimDyn dd = dyn[s];
  const long long shT = dd.fresh ? dd.shift_T : dd.shift_off;
  const long d = dd.fresh ? dd.dlast : 0;
  double base_pos;
  if (t0 == 0) base_pos = (D.tg_off / D.dy64) - (double)shT;
  else base_pos = (D.tg_off / D.dy64) - (double)shT + ((D.tg_vel / D.dy64) * ((double)t0 * D.dt64));
  const double grad = (D.tg_dT) * D.dy64 / (D.tg_dist);
  const double tb = D.tg_base - base_pos * grad;
  double *tpf = trows + sd.off_T, *tcc = tpf + ry;
  for (int y = threadIdx.x; y < ry; y += blockDim.x) {
    /* the column a ghost column is a copy of (T's own boundary types; other
     * types copy nothing) */
    int yr = y;
    if (y < 3 && (D.bc_t[0] == GP_BC_NEUMANN || D.bc_t[0] == GP_BC_PERIODIC))
      yr = remap(y - 3, my, D.bc_t[0], D.bc_t[1]) + 3;
    else if (y >= my + 3 && (D.bc_t[1] == GP_BC_NEUMANN || D.bc_t[1] == GP_BC_PERIODIC))
      yr = remap(y - 3, my, D.bc_t[0], D.bc_t[1]) + 3;
    const double laid = y <= ry - 1 - d ? tb + (double)(y + d) * grad : tb + (double)y * grad;
    const double copied = yr <= ry - 1 - d ? tb + (double)(yr + d) * grad : tb + (double)yr * grad;
    tcc[y] = copied;
    tpf[y] = t0 == 0 ? copied : laid;
  }
  __syncthreads();
  if (threadIdx.x == 0 && dd.fresh) dyn[s].fresh = 0;
}

/* ---- moving frame (Shift = 1) --------------------------------------------
 * Every 100 steps the reference finds MAX_INTERFACE_POS, the largest column y
 * where the liquid crosses one half upwards (check_SHIFT, shift.h:47-65, run
 * over the rows its concentration sweep has just updated), and when it is
 * past Shiftj moves every row down by d = MAX_INTERFACE_POS - Shiftj cells,
 * the top d cells becoming liquid at cfill (apply_shiftY, shift.h:4-45;
 * microsim_gp.c:115-123).  Columns are ghosted indices (interior y + 3). */

/* MAX_INTERFACE_POS over the interior (pairs of interior columns y-1, y),
 * one CTA per tile, atomic max into pos[simulation] */
template <typename R, int N>
__global__ void __launch_bounds__(NT) ks_pos(const SimDesc *__restrict__ sims, const Consts<R> *__restrict__ consts,
                                             const int *__restrict__ tsim, const R *__restrict__ state,
                                             int *__restrict__ pos) {
  __shared__ int s_best[NT / 32];
  const int t = blockIdx.x, s = __ldg(tsim + t);
  if (!consts[s].shift) return;
  const SimDesc sd = sims[s];
  const int lt = t - sd.tile0, by = lt / sd.tiles_x, bx = lt - by * sd.tiles_x;
  const int x = by * TX + threadIdx.x / TY, y = bx * TY + threadIdx.x % TY;
  int best = 0;
  if (x < sd.g.mx && y >= 1 && y < sd.g.my) {
    const R *pl = state + sd.off_state + (long long)(N - 1) * sd.g.plane + (long long)x * sd.g.pitch;
    const R a = pl[y - 1], b = pl[y];
    if ((a - (R(1.0) - a) < R(0.0)) && (b - (R(1.0) - b) > R(0.0))) best = y + 3;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0) s_best[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    int b = 0;
#pragma unroll
    for (int w = 0; w < NT / 32; w++) b = max(b, s_best[w]);
    if (b > 0) atomicMax(pos + s, b);
  }
}

/* The state after the check into the other buffer: shifted by d rows where
 * pos > Shiftj, else copied.  A cell takes the cell d columns up (through
 * the boundary copy tables past the last interior column), or the liquid
 * fill beyond the ghost columns.  The first tile's thread 0 records the
 * shift for the temperature rows of the next step. */
template <typename R, int N, int K>
__global__ void __launch_bounds__(NT) ks_shift(const SimDesc *__restrict__ sims,
                                               const Consts<R> *__restrict__ consts, const int *__restrict__ tsim,
                                               const R *__restrict__ state, R *__restrict__ next,
                                               const int *__restrict__ pos, SimDyn *__restrict__ dyn) {
  const int t = blockIdx.x, s = __ldg(tsim + t);
  const Consts<R> &D = consts[s];
  const SimDesc sd = sims[s];
  const int lt = t - sd.tile0, by = lt / sd.tiles_x, bx = lt - by * sd.tiles_x;
  const int x = by * TX + threadIdx.x / TY, y = bx * TY + threadIdx.x % TY;
  const int p = pos[s];
  const int d = (D.shift && p > D.shiftj) ? p - D.shiftj : 0;
  if (lt == 0 && threadIdx.x == 0 && d > 0) {
    SimDyn &dd = dyn[s];
    dd.shift_T = dd.shift_off;
    dd.dlast = d;
    dd.fresh = 1;
    dd.shift_off += d;
    dd.pos = p;
  }
  if (x >= sd.g.mx || y >= sd.g.my) return;
  const R *src = state + sd.off_state;
  R *dst = next + sd.off_state;
  const long long row = (long long)x * sd.g.pitch, o = row + y;
  const int sy = y + d;
  if (d == 0) {
#pragma unroll
    for (int f = 0; f < N + K; f++) dst[f * sd.g.plane + o] = src[f * sd.g.plane + o];
  } else if (sy <= sd.g.my + 2) {
    const int yp = sy < sd.g.my ? sy : remap(sy, sd.g.my, D.bc_y[0][0], D.bc_y[0][1]);
    const int ym = sy < sd.g.my ? sy : remap(sy, sd.g.my, D.bc_y[1][0], D.bc_y[1][1]);
#pragma unroll
    for (int a = 0; a < N; a++) dst[a * sd.g.plane + o] = src[a * sd.g.plane + row + yp];
#pragma unroll
    for (int k = 0; k < K; k++) dst[(N + k) * sd.g.plane + o] = src[(N + k) * sd.g.plane + row + ym];
  } else {
#pragma unroll
    for (int a = 0; a < N; a++) dst[a * sd.g.plane + o] = a == N - 1 ? R(1.0) : R(0.0);
#pragma unroll
    for (int k = 0; k < K; k++) dst[(N + k) * sd.g.plane + o] = D.mu_fill[k];
  }
}

/* Flags of every tile of a state buffer from its phi (after an upload,
 * smoothing or gp_batch_set). */
template <typename R, int N>
__global__ void __launch_bounds__(NT) kf_flags(const SimDesc *__restrict__ sims, const int *__restrict__ tsim,
                                               const R *__restrict__ state, TileFlags *__restrict__ flags) {
  const int t = blockIdx.x;
  const SimDesc sd = sims[__ldg(tsim + t)];
  const int lt = t - sd.tile0, by = lt / sd.tiles_x, bx = lt - by * sd.tiles_x;
  const int tx = threadIdx.x / TY, ty = threadIdx.x - (threadIdx.x / TY) * TY;
  const int x = by * TX + tx, y = bx * TY + ty;
  const bool valid = (x < sd.g.mx) && (y < sd.g.my);
  int oh = -1;
  if (valid) {
    R ph[N];
#pragma unroll
    for (int a = 0; a < N; a++) ph[a] = __ldg(state + sd.off_state + a * sd.g.plane + (long long)x * sd.g.pitch + y);
    oh = one_hot<R, N>(ph);
  }
  const TileFlags f = tile_flags(valid, oh, tx, ty, min(TX, sd.g.mx - by * TX), min(TY, sd.g.my - bx * TY));
  if (threadIdx.x == 0) flags[t] = f;
}

}  // namespace gpd
