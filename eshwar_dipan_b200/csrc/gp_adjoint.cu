/*
 * gp_adjoint.cu -- kernels of the adjoint of the FP64 step (gp_adjoint).
 * Compiled without FMA contraction, like the FP64 step, so that the cell
 * functions of gp_adjoint.cuh evaluated in double reproduce it bit for bit.
 *
 * One reverse step maps the adjoint of the state after a step (ybar) to the
 * adjoint of the state before it (xbar):
 *   ka_rev_update  for every interior cell, the transposed local Jacobian of
 *                  update_cell applied to the cell's ybar, scattered onto the
 *                  phi / mu of its stencil (through the boundary copy tables:
 *                  a ghost cell is a copy of an interior cell, so its adjoint
 *                  belongs to that cell), onto the delta-phi of its 5-point
 *                  stencil (dphibar, interior plus ring) and onto the four
 *                  parameters;
 *   ka_rev_dphi    for every interior or ring cell, the transposed local
 *                  Jacobian of dphi_cell applied to its dphibar, scattered the
 *                  same way.
 * The local Jacobians are exact: the cell functions are evaluated on
 * Dual<ADJ_W> numbers seeded on ADJ_W of the stencil inputs at a time.
 * Each reverse pass runs in two launches: a sort over the grid that handles
 * the cheap cells (pure-phase windows: bulk_rev; no active phase: nothing)
 * and lists the others, then one thread per (listed cell, dual pass), so the
 * expensive work fills every SM with whole warps of it instead of a few
 * lanes per warp along the interface.
 * Scatter-adds are atomic (FP64), so the last bits of a gradient may differ
 * between runs; values are exact derivatives up to summation order.
 */
#include <cuda_runtime.h>

#include <cstdlib>

#include "gp_adjoint.cuh"
#include "gp_adjoint_launch.h"

namespace gpd {

/* seeded inputs per dual pass: of the concentration pass (ADJ_W) and of the
 * phase-field pass (ADJ_WD).  With a thread per (cell, pass) the leanest pass
 * of the concentration update is the fastest (wider ones spill); the
 * phase-field pass takes GP_ADJ_WD */
#ifndef GP_ADJ_W
#define GP_ADJ_W 1
#endif
#ifndef GP_ADJ_WD
#define GP_ADJ_WD 1
#endif
constexpr int ADJ_W = GP_ADJ_W;
constexpr int ADJ_WD = GP_ADJ_WD;
constexpr int AB = 128;   /* threads per block along y */

__device__ __forceinline__ int rmx(int x, const Grid &g, const Consts<double> *c, int f) {
  return (x < 0 || x >= g.mx) ? remap(x, g.mx, c->bc_x[f][0], c->bc_x[f][1]) : x;
}
__device__ __forceinline__ int rmy(int y, const Grid &g, const Consts<double> *c, int f) {
  return (y < 0 || y >= g.my) ? remap(y, g.my, c->bc_y[f][0], c->bc_y[f][1]) : y;
}

/* phi of the 3x3 window around (x, y) and mu of its 5-point stencil (corners
 * of the mu window are filled too; update_cell does not read them) */
template <int N, int K>
__device__ __forceinline__ void gather(const Consts<double> *c, const Grid &g, const double *st, int x, int y,
                                       double (&S)[N][3][3], double (&M)[K][3][3]) {
#pragma unroll
  for (int di = 0; di < 3; di++) {
    const int xp = rmx(x + di - 1, g, c, 0), xm = rmx(x + di - 1, g, c, 1);
#pragma unroll
    for (int dj = 0; dj < 3; dj++) {
      const int yp = rmy(y + dj - 1, g, c, 0), ym = rmy(y + dj - 1, g, c, 1);
#pragma unroll
      for (int a = 0; a < N; a++) S[a][di][dj] = st[a * g.plane + (long long)xp * g.pitch + yp];
#pragma unroll
      for (int k = 0; k < K; k++) M[k][di][dj] = st[(N + k) * g.plane + (long long)xm * g.pitch + ym];
    }
  }
}

/* phase whose exact one-hot phi (1.0 and +0.0) the values hold, or -1 */
template <int N>
__device__ __forceinline__ int one_hot_bits(const double *v) {
  int p = -1, ones = 0, zeros = 0;
#pragma unroll
  for (int a = 0; a < N; a++) {
    const long long b = __double_as_longlong(v[a]);
    if (b == 0x3ff0000000000000LL) { p = a; ones++; }
    else if (b == 0) zeros++;
  }
  return (ones == 1 && zeros == N - 1) ? p : -1;
}

__device__ __forceinline__ long long didx(const Grid &g, int a, int x, int y) {
  return a * g.dplane + (long long)(x + 1) * g.dpitch + (y + 1);
}

/* ---- forward ------------------------------------------------------------ */

template <int N, int K, bool A>
__global__ void __launch_bounds__(AB) ka_dphi(const Consts<double> *__restrict__ c, AdjParams prm, Grid g,
                                              const double *__restrict__ st, double *__restrict__ dphi) {
  const int y = blockIdx.x * AB + threadIdx.x - 1, x = (int)blockIdx.y - 1;
  if (y > g.my) return;
  double S[N][3][3], M[K][3][3];
  gather<N, K>(c, g, st, x, y, S, M);
  double p[ADJ_NPARAM];
#pragma unroll
  for (int j = 0; j < ADJ_NPARAM; j++) p[j] = prm.v[j];
  const AK<double> D = make_ak<double>(c, p);
  double m[K], d[N];
#pragma unroll
  for (int k = 0; k < K; k++) m[k] = M[k][1][1];
  dphi_cell<double, N, K, A>(D, S, m, d);
#pragma unroll
  for (int a = 0; a < N; a++) dphi[didx(g, a, x, y)] = d[a];
}

/* A ring or interior cell whose delta-phi can differ from +0.0: a phase with
 * a non-zero discrete Laplacian there, or a negative phi (dphi_cell returns
 * +0.0 first for every other cell). */
template <int N, int K>
__device__ __forceinline__ bool dphi_active(const Consts<double> *c, const Grid &g, const double *st, int x, int y) {
  const int xm = rmx(x - 1, g, c, 0), xc = rmx(x, g, c, 0), xp = rmx(x + 1, g, c, 0);
  const int ym = rmy(y - 1, g, c, 0), yc = rmy(y, g, c, 0), yp = rmy(y + 1, g, c, 0);
  bool active = false;
#pragma unroll
  for (int a = 0; a < N; a++) {
    const double *f = st + a * g.plane;
    const double cc = f[(long long)xc * g.pitch + yc];
    const double gxf = f[(long long)xp * g.pitch + yc] - cc, gxb = cc - f[(long long)xm * g.pitch + yc];
    const double gyr = f[(long long)xc * g.pitch + yp] - cc, gyl = cc - f[(long long)xc * g.pitch + ym];
    active |= (gxf - gxb) != 0.0 || (gyr - gyl) != 0.0 || cc < 0.0;
  }
  return active;
}

/* delta-phi in two launches: the grid is swept for the active cells (the
 * others keep the +0.0 the buffer was cleared to), then one thread per
 * listed cell evaluates dphi_cell */
template <int N, int K>
__global__ void __launch_bounds__(AB) ka_dphi_sort(const Consts<double> *__restrict__ c, Grid g,
                                                   const double *__restrict__ st, int2 *__restrict__ cells,
                                                   int *__restrict__ count);

template <int N, int K, bool A>
__global__ void __launch_bounds__(AB) ka_dphi_list(const Consts<double> *__restrict__ c, AdjParams prm, Grid g,
                                                   const double *__restrict__ st, double *__restrict__ dphi,
                                                   const int2 *__restrict__ cells, const int *__restrict__ count) {
  double p[ADJ_NPARAM];
#pragma unroll
  for (int j = 0; j < ADJ_NPARAM; j++) p[j] = prm.v[j];
  const AK<double> D = make_ak<double>(c, p);
  const int n = *count;
  for (int i = blockIdx.x * AB + threadIdx.x; i < n; i += gridDim.x * AB) {
    const int2 e = cells[i];
    double S[N][3][3], M[K][3][3];
    gather<N, K>(c, g, st, e.x, e.y, S, M);
    double m[K], d[N];
#pragma unroll
    for (int k = 0; k < K; k++) m[k] = M[k][1][1];
    dphi_cell<double, N, K, A>(D, S, m, d);
#pragma unroll
    for (int a = 0; a < N; a++) dphi[didx(g, a, e.x, e.y)] = d[a];
  }
}

template <int N, int K>
__global__ void __launch_bounds__(AB) ka_update(const Consts<double> *__restrict__ c, AdjParams prm, Grid g,
                                                const double *__restrict__ st, const double *__restrict__ dphi,
                                                double *__restrict__ next) {
  const int y = blockIdx.x * AB + threadIdx.x, x = blockIdx.y;
  if (y >= g.my) return;
  double S[N][3][3], M[K][3][3], DP[N][3][3];
  gather<N, K>(c, g, st, x, y, S, M);
#pragma unroll
  for (int a = 0; a < N; a++)
#pragma unroll
    for (int di = 0; di < 3; di++)
#pragma unroll
      for (int dj = 0; dj < 3; dj++) DP[a][di][dj] = dphi[didx(g, a, x + di - 1, y + dj - 1)];
  double p[ADJ_NPARAM];
#pragma unroll
  for (int j = 0; j < ADJ_NPARAM; j++) p[j] = prm.v[j];
  const AK<double> D = make_ak<double>(c, p);
  double nph[N], nm[K];
  update_cell<double, N, K>(D, S, M, DP, y, g.my, nph, nm);
  const long long o = (long long)x * g.pitch + y;
#pragma unroll
  for (int a = 0; a < N; a++) next[a * g.plane + o] = nph[a];
#pragma unroll
  for (int k = 0; k < K; k++) next[(N + k) * g.plane + o] = nm[k];
}

/* ---- reverse ------------------------------------------------------------ */

/* parameter adjoints: one atomic per warp */
__device__ __forceinline__ void flush_params(double (&pacc)[ADJ_NPARAM], double *pbar) {
#pragma unroll
  for (int j = 0; j < ADJ_NPARAM; j++) {
    double v = pacc[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(pbar + j, v);
  }
}

/* Transposed update of a bulk cell (phase p one-hot over its 3x3 window, one
 * independent component): nm = twoA*(cmu*(m - E) + dt*divflux - divjat) + E,
 * divflux = (Fxf - Fxb)/dx + (Fyr - Fyl)/dy, F = (D(lower)+D(upper))/2 *
 * (m(upper) - m(lower))/h with D(e) = sum_b DC_b phi_b(e), divjat constant;
 * nphi = phi + dphi. */
template <int N>
__device__ __forceinline__ void bulk_rev(const Consts<double> *c, const Grid &g, int x, int y, int p,
                                         const double (&S)[N][3][3], const double (&M)[1][3][3], const double *yb,
                                         double *xbar, double *dphibar) {
  const double idx = c->mul_dx ? c->inv_dx : 1.0 / c->dx, idy = c->mul_dy ? c->inv_dy : 1.0 / c->dy;
  /* phi passes through, and so does the cell's own delta-phi */
  const long long oc = (long long)x * g.pitch + y;
#pragma unroll
  for (int a = 0; a < N; a++) {
    if (yb[a] == 0.0) continue;
    atomicAdd(xbar + a * g.plane + oc, yb[a]);
    atomicAdd(dphibar + didx(g, a, x, y), yb[a]);
  }
  const double ym = yb[N];
  if (ym == 0.0) return;
  const double cnb = ym * c->twoA[p][0];
  /* the cell's own mu through c_mu */
  double mbar_c = cnb * c->cmu[p][0][0];
  const double dfb = cnb * c->dt;
  /* faces: lower/upper cells in the window, the face's gradient scale, sign in divflux */
  const int li[4] = {1, 0, 1, 1}, lj[4] = {1, 1, 1, 0}, ui[4] = {2, 1, 1, 1}, uj[4] = {1, 1, 2, 1};
  const double sc[4] = {idx, idx, idy, idy}, sg[4] = {1.0, -1.0, 1.0, -1.0};
  double Dw[3][3];
#pragma unroll
  for (int di = 0; di < 3; di++)
#pragma unroll
    for (int dj = 0; dj < 3; dj++) {
      double d = 0.0;
#pragma unroll
      for (int b = 0; b < N; b++) d += c->DC[b][0][0][0] * S[b][di][dj];
      Dw[di][dj] = d;
    }
  double Dbar[3][3] = {}, Mbar[3][3] = {};
  Mbar[1][1] = mbar_c;
#pragma unroll
  for (int f = 0; f < 4; f++) {
    const double Fb = dfb * sg[f] * sc[f];
    const double dm = (Dw[ui[f]][uj[f]] + Dw[li[f]][lj[f]]) * 0.5;
    const double gr = (M[0][ui[f]][uj[f]] - M[0][li[f]][lj[f]]) * sc[f];
    const double gb = Fb * dm, dmb = Fb * gr;
    Mbar[ui[f]][uj[f]] += gb * sc[f];
    Mbar[li[f]][lj[f]] -= gb * sc[f];
    Dbar[ui[f]][uj[f]] += 0.5 * dmb;
    Dbar[li[f]][lj[f]] += 0.5 * dmb;
  }
  const int pi[5] = {1, 0, 2, 1, 1}, pj[5] = {1, 1, 1, 0, 2};
#pragma unroll
  for (int r = 0; r < 5; r++) {
    const int di = pi[r], dj = pj[r];
    if (Mbar[di][dj] != 0.0) {
      const int xs = rmx(x + di - 1, g, c, 1), ys = rmy(y + dj - 1, g, c, 1);
      atomicAdd(xbar + N * g.plane + (long long)xs * g.pitch + ys, Mbar[di][dj]);
    }
    if (Dbar[di][dj] != 0.0) {
      const int xs = rmx(x + di - 1, g, c, 0), ys = rmy(y + dj - 1, g, c, 0);
#pragma unroll
      for (int b = 0; b < N; b++) {
        const double v = Dbar[di][dj] * c->DC[b][0][0][0];
        if (v != 0.0) atomicAdd(xbar + b * g.plane + (long long)xs * g.pitch + ys, v);
      }
    }
  }
}

/* The inputs of update_cell, in seeding order (phi 3x3 per phase, mu and
 * delta-phi 5-point per field, the four parameters), less those it does not
 * read: the liquid's delta-phi enters only at the centre (the commit and the
 * dh/dphi coupling; the anti-trapping current reads the solids'), and of the
 * parameters only epsilon (the anti-trapping factor).  upd_inputs: how many
 * remain; upd_input(u): the seeding index of the u-th. */
template <int N, int K>
__host__ __device__ constexpr int upd_inputs() {
  return 9 * N + 5 * K + 5 * (N - 1) + 1 + 1;
}
template <int N, int K>
__device__ __forceinline__ int upd_input(int u) {
  constexpr int NPHI = 9 * N, NMU = 5 * K, NDP = 5 * N, LIQ = NPHI + NMU + 5 * (N - 1);
  return u <= LIQ ? u : NPHI + NMU + NDP + ADJ_EPS;
}

/* Reverse of the concentration pass at cell (x, y).  SORT: cells whose 3x3
 * window is one pure phase take bulk_rev here; the others are returned
 * (true) for the dual passes, which run with SORT false over the list of
 * such cells, so that a warp's lanes all take the expensive path together. */
template <int N, int K, bool SORT>
__device__ __forceinline__ bool rev_update_cell(const Consts<double> *__restrict__ c, const AdjParams &prm,
                                                const Grid &g, const double *__restrict__ st,
                                                const double *__restrict__ dphi, const double *__restrict__ ybar,
                                                double *__restrict__ xbar, double *__restrict__ dphibar, int x, int y,
                                                bool live, double (&pacc)[ADJ_NPARAM], int pass = -1) {
  using DT = Dual<ADJ_W>;
  constexpr int NPHI = 9 * N, NMU = 5 * K, NDP = 5 * N, NIN = NPHI + NMU + NDP + ADJ_NPARAM;
  /* pass >= 0: only the dual pass seeding inputs pass*ADJ_W .. (one input
   * per pass: the pass-th input update_cell depends on, upd_input) */
  const int b0 = pass < 0 ? 0 : (ADJ_W == 1 ? upd_input<N, K>(pass) : pass * ADJ_W);
  const int b1 = pass < 0 ? NIN : min(NIN, b0 + ADJ_W);
  double yb[N + K];
  bool any = false;
  if (live) {
    const long long o = (long long)x * g.pitch + y;
#pragma unroll
    for (int f = 0; f < N + K; f++) {
      yb[f] = ybar[f * g.plane + o];
      any |= yb[f] != 0.0;
    }
  }
  if (live && any) {
    double S[N][3][3], M[K][3][3], DP[N][3][3];
    gather<N, K>(c, g, st, x, y, S, M);
#pragma unroll
    for (int a = 0; a < N; a++)
#pragma unroll
      for (int di = 0; di < 3; di++)
#pragma unroll
        for (int dj = 0; dj < 3; dj++) DP[a][di][dj] = dphi[didx(g, a, x + di - 1, y + dj - 1)];
    const int pi[5] = {1, 0, 2, 1, 1}, pj[5] = {1, 1, 1, 0, 2};
    /* A cell whose 3x3 phi window holds one phase's exact one-hot phi has
     * every face phi gradient 0.0 (no anti-trapping current is evaluated) and
     * takes the bulk branch: its update is linear diffusion of mu with the
     * face means of D(phi), transposed here directly (bulk_rev). */
    int ph = -1;
    bool uni;
    {
      double c0[N];
#pragma unroll
      for (int a = 0; a < N; a++) c0[a] = S[a][1][1];
      ph = one_hot_bits<N>(c0);
      uni = ph >= 0;
#pragma unroll
      for (int di = 0; di < 3; di++)
#pragma unroll
        for (int dj = 0; dj < 3; dj++) {
          double v[N];
#pragma unroll
          for (int a = 0; a < N; a++) v[a] = S[a][di][dj];
          uni = uni && one_hot_bits<N>(v) == ph;
        }
    }
    if (SORT) {
      if (uni && K == 1) bulk_rev<N>(c, g, x, y, ph, S, M, yb, xbar, dphibar);
      else return true;
    } else
    for (int base = b0; base < b1; base += ADJ_W) {
      DT Sd[N][3][3], Md[K][3][3], DPd[N][3][3], pd[ADJ_NPARAM];
      /* seed inputs base .. base+W-1: every element compares its own
       * (compile-time) input number, so the dual arrays stay in registers */
#pragma unroll
      for (int a = 0; a < N; a++)
#pragma unroll
        for (int di = 0; di < 3; di++)
#pragma unroll
          for (int dj = 0; dj < 3; dj++) {
            Sd[a][di][dj] = DT(S[a][di][dj]);
            DPd[a][di][dj] = DT(DP[a][di][dj]);
#pragma unroll
            for (int w = 0; w < ADJ_W; w++) Sd[a][di][dj].d[w] = (a * 9 + di * 3 + dj == base + w) ? 1.0 : 0.0;
          }
#pragma unroll
      for (int k = 0; k < K; k++)
#pragma unroll
        for (int di = 0; di < 3; di++)
#pragma unroll
          for (int dj = 0; dj < 3; dj++) Md[k][di][dj] = DT(M[k][di][dj]);
#pragma unroll
      for (int r = 0; r < 5; r++) {
#pragma unroll
        for (int k = 0; k < K; k++)
#pragma unroll
          for (int w = 0; w < ADJ_W; w++)
            Md[k][pi[r]][pj[r]].d[w] = (NPHI + k * 5 + r == base + w) ? 1.0 : 0.0;
#pragma unroll
        for (int a = 0; a < N; a++)
#pragma unroll
          for (int w = 0; w < ADJ_W; w++)
            DPd[a][pi[r]][pj[r]].d[w] = (NPHI + NMU + a * 5 + r == base + w) ? 1.0 : 0.0;
      }
#pragma unroll
      for (int j = 0; j < ADJ_NPARAM; j++) {
        pd[j] = DT(prm.v[j]);
#pragma unroll
        for (int w = 0; w < ADJ_W; w++) pd[j].d[w] = (NPHI + NMU + NDP + j == base + w) ? 1.0 : 0.0;
      }
      const AK<DT> D = make_ak<DT>(c, pd);
      DT nph[N], nm[K];
      update_cell<DT, N, K>(D, Sd, Md, DPd, y, g.my, nph, nm);
      for (int w = 0; w < ADJ_W && base + w < NIN; w++) {
        const int id = base + w;
        double gsum = 0.0;
#pragma unroll
        for (int a = 0; a < N; a++) gsum += yb[a] * nph[a].d[w];
#pragma unroll
        for (int k = 0; k < K; k++) gsum += yb[N + k] * nm[k].d[w];
        if (gsum == 0.0) continue;
        if (id < NPHI) {
          const int a = id / 9, r = id % 9;
          const int xs = rmx(x + r / 3 - 1, g, c, 0), ys = rmy(y + r % 3 - 1, g, c, 0);
          atomicAdd(xbar + a * g.plane + (long long)xs * g.pitch + ys, gsum);
        } else if (id < NPHI + NMU) {
          const int k = (id - NPHI) / 5, r = (id - NPHI) % 5;
          const int xs = rmx(x + pi[r] - 1, g, c, 1), ys = rmy(y + pj[r] - 1, g, c, 1);
          atomicAdd(xbar + (N + k) * g.plane + (long long)xs * g.pitch + ys, gsum);
        } else if (id < NPHI + NMU + NDP) {
          const int a = (id - NPHI - NMU) / 5, r = (id - NPHI - NMU) % 5;
          atomicAdd(dphibar + didx(g, a, x + pi[r] - 1, y + pj[r] - 1), gsum);
        } else {
#pragma unroll
          for (int j = 0; j < ADJ_NPARAM; j++)
            if (id - NPHI - NMU - NDP == j) pacc[j] += gsum;
        }
      }
    }
  }
  return false;
}

/* warp-aggregated append of (x, y) to a cell list; call with the whole warp */
__device__ __forceinline__ void push_cell(bool want, int x, int y, int2 *__restrict__ cells, int *__restrict__ count) {
  const unsigned m = __ballot_sync(0xffffffffu, want);
  if (!m) return;
  const int lane = threadIdx.x & 31, lead = __ffs(m) - 1;
  int base = 0;
  if (lane == lead) base = atomicAdd(count, __popc(m));
  base = __shfl_sync(0xffffffffu, base, lead);
  if (want) cells[base + __popc(m & ((1u << lane) - 1u))] = make_int2(x, y);
}

template <int N, int K>
__global__ void __launch_bounds__(AB) ka_dphi_sort(const Consts<double> *__restrict__ c, Grid g,
                                                   const double *__restrict__ st, int2 *__restrict__ cells,
                                                   int *__restrict__ count) {
  const int y = blockIdx.x * AB + threadIdx.x - 1, x = (int)blockIdx.y - 1;
  const bool want = y <= g.my && dphi_active<N, K>(c, g, st, x, y);
  push_cell(want, x, y, cells, count);
}

template <int N, int K>
__global__ void __launch_bounds__(AB) ka_rev_update(const Consts<double> *__restrict__ c, AdjParams prm, Grid g,
                                                    const double *__restrict__ st, const double *__restrict__ dphi,
                                                    const double *__restrict__ ybar, double *__restrict__ xbar,
                                                    double *__restrict__ dphibar, int2 *__restrict__ cells,
                                                    int *__restrict__ count) {
  const int y = blockIdx.x * AB + threadIdx.x, x = blockIdx.y;
  double pacc[ADJ_NPARAM] = {};
  const bool want = rev_update_cell<N, K, true>(c, prm, g, st, dphi, ybar, xbar, dphibar, x, y, y < g.my, pacc);
  push_cell(want, x, y, cells, count);
}

template <int N, int K>
__global__ void __launch_bounds__(AB) ka_rev_update_list(const Consts<double> *__restrict__ c, AdjParams prm, Grid g,
                                                         const double *__restrict__ st,
                                                         const double *__restrict__ dphi,
                                                         const double *__restrict__ ybar, double *__restrict__ xbar,
                                                         double *__restrict__ dphibar, double *__restrict__ pbar,
                                                         const int2 *__restrict__ cells,
                                                         const int *__restrict__ count) {
  /* one thread per (cell, dual pass): every SM gets work */
  constexpr int NIN = 9 * N + 5 * K + 5 * N + ADJ_NPARAM;
  constexpr int NPASS = ADJ_W == 1 ? upd_inputs<N, K>() : (NIN + ADJ_W - 1) / ADJ_W;
  double pacc[ADJ_NPARAM] = {};
  const long long n = (long long)*count * NPASS;
  for (long long i = (long long)blockIdx.x * AB + threadIdx.x; i < n; i += (long long)gridDim.x * AB) {
    const int2 e = cells[i / NPASS];
    rev_update_cell<N, K, false>(c, prm, g, st, dphi, ybar, xbar, dphibar, e.x, e.y, true, pacc, (int)(i % NPASS));
  }
  flush_params(pacc, pbar);
}

/* ---- hand-derived reverse of the concentration update ---------------------
 * For two phases and one component (the adjoint's scope) the transposed
 * local Jacobian of update_cell written out, beside its evaluation by dual
 * passes (the default, which is faster: thirty threads per listed cell hide
 * latency better than five); the two cross-check each other.  Five parts per
 * listed cell: part 0 the cell's own terms (the phi commit, its mu, the
 * dh/dphi * delta-phi coupling and the dc/dmu inversion), parts 1-4 one face
 * each (x+, x-, y+, y-: the diffusion flux and the anti-trapping current
 * through it).  Every derivative is that of the expressions update_cell
 * evaluates, on the branch the step took (bulk or interface cell, current
 * evaluated or not); only the rounding of the derivative arithmetic differs
 * from the dual passes. */

/* d(v / h)/dv in the step's arithmetic for spacing h (mul: v * (1/h)) */
__device__ __forceinline__ double rdx(const Consts<double> *c) { return c->mul_dx ? c->inv_dx : 1.0 / c->dx; }
__device__ __forceinline__ double rdy(const Consts<double> *c) { return c->mul_dy ? c->inv_dy : 1.0 / c->dy; }
__device__ __forceinline__ double r2dy(const Consts<double> *c) { return c->mul_dy ? c->inv_2dy : 1.0 / (2.0 * c->dy); }

/* obstacle anti-trapping weight s(p) = p (1 - h(p)) / sqrt(p (1 - p)) and ds/dp */
__device__ __forceinline__ void sp_weight(double p, double &s, double &ds) {
  const double w = p * (1.0 - p);
  if (!(w > 0.0)) {
    s = 0.0;
    ds = 0.0;
    return;
  }
  const double h = 3.0 * p * p - 2.0 * p * p * p, dh = 6.0 * p - 6.0 * p * p;
  const double sq = sqrt(w), u = p * (1.0 - h);
  s = u / sq;
  ds = ((1.0 - h) - p * dh) / sq - u * (1.0 - 2.0 * p) / (2.0 * sq * w);
}

/* One face of the 3x3 window (xface: between (fi,fj) and (fi+1,fj); else
 * between (fi,fj) and (fi,fj+1)) for two phases, one component: its primal
 * current j and flux F, then, given their adjoints jb and Fb, the adjoints
 * of the phi window (Sb), the mu window (Mb) and the solid's delta-phi window
 * (Db).  ylo: interior y of the face's lower cell (y-faces). */
__device__ __forceinline__ void face_rev(const AK<double> &D, const double (&S)[2][3][3], const double (&M)[1][3][3],
                                         const double (&DP)[2][3][3], bool xface, int fi, int fj, int ylo, int my,
                                         double &j, double &F, double jb, double Fb, bool want_j, double (&Sb)[2][3][3],
                                         double (&Mb)[3][3], double (&Db)[3][3]) {
  const Consts<double> *c = D.c;
  const int i1 = xface ? fi + 1 : fi, j1 = xface ? fj : fj + 1;
  double gr[2], cn[2];
#pragma unroll
  for (int a = 0; a < 2; a++) {
    if (xface) {
      gr[a] = adivx(S[a][i1][j1] - S[a][fi][fj], D);
      cn[a] = 0.5 * (adiv2y(S[a][fi][fj + 1] - S[a][fi][fj - 1], D) + adiv2y(S[a][i1][fj + 1] - S[a][i1][fj - 1], D));
    } else {
      gr[a] = adivy(S[a][i1][j1] - S[a][fi][fj], D);
      const double gc0 = 0.5 * (adivx(S[a][fi + 1][fj] - S[a][fi][fj], D) + adivx(S[a][fi][fj] - S[a][fi - 1][fj], D));
      const double gc1 = 0.5 * (adivx(S[a][fi + 1][j1] - S[a][i1][j1], D) + adivx(S[a][i1][j1] - S[a][fi - 1][j1], D));
      cn[a] = 0.5 * (gc0 + gc1);
    }
  }
  const double hg = xface ? rdx(c) : rdy(c);   /* d gr / d(difference) */
  /* ---- diffusion flux F = (D(cell 1) + D(cell 0)) / 2 * (mu1 - mu0) / h */
  double DD0 = 0.0, DD1 = 0.0;
#pragma unroll
  for (int b = 0; b < 2; b++) {
    DD0 += c->DC[b][0][0][0] * S[b][fi][fj];
    DD1 += c->DC[b][0][0][0] * S[b][i1][j1];
  }
  const double dm = (DD1 + DD0) * 0.5;
  const double gm = xface ? adivx(M[0][i1][j1] - M[0][fi][fj], D) : adivy(M[0][i1][j1] - M[0][fi][fj], D);
  F = dm * gm;
  {
    const double dmb = Fb * gm, gmb = Fb * dm;
    Mb[i1][j1] += gmb * hg;
    Mb[fi][fj] -= gmb * hg;
#pragma unroll
    for (int b = 0; b < 2; b++) {
      Sb[b][i1][j1] += 0.5 * dmb * c->DC[b][0][0][0];
      Sb[b][fi][fj] += 0.5 * dmb * c->DC[b][0][0][0];
    }
  }
  /* ---- anti-trapping current of the solid (phase 0) */
  j = 0.0;
  const bool yskip = !xface && (ylo + 3 == my - 2);
  const double s2 = cn[0] * cn[0] + gr[0] * gr[0];
  if (s2 == 0.0 || yskip) return;
  const double ng = sqrt(s2), nl = sqrt(cn[1] * cn[1] + gr[1] * gr[1]);
  double sp = gr[0] * gr[1];
  sp += cn[0] * cn[1];
  const double sp0 = sp;
  if (nl > 0.0) sp /= (nl * ng);
  const double m0 = M[0][fi][fj], m1 = M[0][i1][j1];
  const double cl0 = 0.0 + c->cmu[1][0][0] * (m0 - c->E[1][0]), cs0 = 0.0 + c->cmu[0][0][0] * (m0 - c->E[0][0]);
  const double cl1 = 0.0 + c->cmu[1][0][0] * (m1 - c->E[1][0]), cs1 = 0.0 + c->cmu[0][0][0] * (m1 - c->E[0][0]);
  const double dp0 = DP[0][fi][fj], dp1 = DP[0][i1][j1];
  double w0 = 1.0, w1 = 1.0, dw0 = 0.0, dw1 = 0.0;
  if (c->obstacle) {
    sp_weight(S[0][fi][fj], w0, dw0);
    sp_weight(S[0][i1][j1], w1, dw1);
  }
  const double t0 = w0 * (cl0 - cs0), t1 = w1 * (cl1 - cs1);
  const double br = t1 * dp1 + t0 * dp0;
  const double half = c->obstacle ? 0.5 : c->well_half, atf = c->atf[0][0];
  const double A1 = atf * fabs(sp) * half, A2 = A1 * br, A3 = A2 * gr[0];
  j = A3 / ng;
  if (!want_j || jb == 0.0) return;
  /* reverse */
  const double A3b = jb / ng;
  double ngb = -jb * A3 / (ng * ng);
  const double A2b = A3b * gr[0];
  double gr0b = A3b * A2;
  const double A1b = A2b * br, brb = A2b * A1;
  const double spb = A1b * half * atf * (sp > 0.0 ? 1.0 : (sp < 0.0 ? -1.0 : 0.0));
  double sp0b = spb, nlb = 0.0;
  if (nl > 0.0) {
    const double den = nl * ng;
    sp0b = spb / den;
    const double denb = -spb * sp / den;
    nlb = denb * ng;
    ngb += denb * nl;
  }
  (void)sp0;
  gr0b += sp0b * gr[1];
  double grLb = sp0b * gr[0], cn0b = sp0b * cn[1], cnLb = sp0b * cn[0];
  gr0b += ngb * gr[0] / ng;
  cn0b += ngb * cn[0] / ng;
  if (nl > 0.0) {
    grLb += nlb * gr[1] / nl;
    cnLb += nlb * cn[1] / nl;
  }
  /* bracket: t1 dp1 + t0 dp0, t = w (cl - cs), cl - cs linear in mu */
  const double t1b = brb * dp1, t0b = brb * dp0;
  Db[i1][j1] += brb * t1;
  Db[fi][fj] += brb * t0;
  const double dcm = c->cmu[1][0][0] - c->cmu[0][0][0];
  Mb[i1][j1] += t1b * w1 * dcm;
  Mb[fi][fj] += t0b * w0 * dcm;
  if (c->obstacle) {
    Sb[0][i1][j1] += t1b * (cl1 - cs1) * dw1;
    Sb[0][fi][fj] += t0b * (cl0 - cs0) * dw0;
  }
  /* gradients to the phi window */
  const double grb[2] = {gr0b, grLb}, cnb[2] = {cn0b, cnLb};
#pragma unroll
  for (int a = 0; a < 2; a++) {
    Sb[a][i1][j1] += grb[a] * hg;
    Sb[a][fi][fj] -= grb[a] * hg;
    if (xface) {
      const double q = 0.5 * cnb[a] * r2dy(c);
      Sb[a][fi][fj + 1] += q;
      Sb[a][fi][fj - 1] -= q;
      Sb[a][i1][fj + 1] += q;
      Sb[a][i1][fj - 1] -= q;
    } else {
      const double q = 0.25 * cnb[a] * rdx(c);
      Sb[a][fi + 1][fj] += q;
      Sb[a][fi - 1][fj] -= q;
      Sb[a][fi + 1][j1] += q;
      Sb[a][fi - 1][j1] -= q;
    }
  }
}

/* One warp takes six listed cells, five lanes each: lane 5i is cell i's own
 * part, lanes 5i+1 .. 5i+4 its faces x+, x-, y+, y-.  A face lane reverses its
 * face (its adjoints depend on the cell's adjoint of mu and on the cell's
 * multiplier only) and hands the face's current and flux to the cell lane,
 * which needs all four for the dc of the dc/dmu term; the five lanes' window
 * adjoints are then summed by shuffles and the cell lane scatters them. */
__global__ void __launch_bounds__(AB) ka_rev_update_hand(const Consts<double> *__restrict__ c, AdjParams prm, Grid g,
                                                         const double *__restrict__ st,
                                                         const double *__restrict__ dphi,
                                                         const double *__restrict__ ybar, double *__restrict__ xbar,
                                                         double *__restrict__ dphibar, double *__restrict__ pbar,
                                                         const int2 *__restrict__ cells,
                                                         const int *__restrict__ count) {
  constexpr unsigned FULL = 0xffffffffu;
  double pacc[ADJ_NPARAM] = {};
  const int lane = threadIdx.x & 31, slot = lane / 5, part = lane - slot * 5, base = slot * 5;
  const long long ncell = *count, nwarps = (long long)gridDim.x * (AB / 32);
  double p[ADJ_NPARAM];
#pragma unroll
  for (int k = 0; k < ADJ_NPARAM; k++) p[k] = prm.v[k];
  const AK<double> D = make_ak<double>(c, p);
  const double cst = c->obstacle ? D.jat_obst : D.jat_well;
  for (long long w0 = ((long long)blockIdx.x * (AB / 32) + (threadIdx.x >> 5)) * 6; w0 < ncell; w0 += nwarps * 6) {
    const long long ci = w0 + slot;
    const bool live = slot < 6 && ci < ncell;
    int x = 0, y = 0;
    double S[2][3][3] = {}, M[1][3][3] = {}, DP[2][3][3] = {};
    double yb0 = 0.0, yb1 = 0.0, ybm = 0.0;
    if (live) {
      const int2 e = cells[ci];
      x = e.x;
      y = e.y;
      const long long o = (long long)x * g.pitch + y;
      yb0 = ybar[o];
      yb1 = ybar[g.plane + o];
      ybm = ybar[2 * g.plane + o];
      gather<2, 1>(c, g, st, x, y, S, M);
#pragma unroll
      for (int a = 0; a < 2; a++)
#pragma unroll
        for (int di = 0; di < 3; di++)
#pragma unroll
          for (int dj = 0; dj < 3; dj++) DP[a][di][dj] = dphi[didx(g, a, x + di - 1, y + dj - 1)];
    }
    double Sb[2][3][3] = {}, Mb[3][3] = {}, Db[3][3] = {};
    const double ph0 = S[0][1][1], ph1 = S[1][1][1], m = M[0][1][1];
    const int bulk = ph0 == 1.0 ? 0 : (ph1 == 1.0 ? 1 : -1);
    const double H0 = 3.0 * ph0 * ph0 - 2.0 * ph0 * ph0 * ph0, H1 = 3.0 * ph1 * ph1 - 2.0 * ph1 * ph1 * ph1;
    const double dcdmu = (0.0 + c->cmu64[0][0][0] * H0) + c->cmu64[1][0][0] * H1;
    /* d nm / d(dt*divflux - divjat) */
    const double kap = bulk >= 0 ? (bulk == 0 ? c->twoA[0][0] : c->twoA[1][0]) : (live ? 1.0 / dcdmu : 0.0);
    const double dcb = ybm * kap;   /* adjoint of the update's dc (of cn in a bulk cell) */
    /* ---- face lanes: the face's current and flux, and their reverse */
    double jf = 0.0, Ff = 0.0;
    if (live && part > 0) {
      const int f = part - 1;
      const bool xf = f < 2;
      const double sg = (f == 0 || f == 2) ? 1.0 : -1.0, hh = xf ? rdx(c) : rdy(c);
      const double divfluxb = dcb * c->dt, divjatb = -dcb;
      const double jb = sg * cst * divjatb * hh, Fb = sg * divfluxb * hh;
      const bool rev = ybm != 0.0;
      switch (f) {   /* window coordinates as constants: the window arrays stay in registers */
        case 0: face_rev(D, S, M, DP, true, 1, 1, 0, g.my, jf, Ff, jb, Fb, rev, Sb, Mb, Db); break;
        case 1: face_rev(D, S, M, DP, true, 0, 1, 0, g.my, jf, Ff, jb, Fb, rev, Sb, Mb, Db); break;
        case 2: face_rev(D, S, M, DP, false, 1, 1, y, g.my, jf, Ff, jb, Fb, rev, Sb, Mb, Db); break;
        default: face_rev(D, S, M, DP, false, 1, 0, y - 1, g.my, jf, Ff, jb, Fb, rev, Sb, Mb, Db); break;
      }
      /* cst = jat_obst or jat_well = (-0.25 pi or -1) * epsilon */
      pacc[ADJ_EPS] += sg * jf * divjatb * hh * (c->obstacle ? (-0.25 * M_PI) : -1.0);
    }
    double jx[4], fx[4];
#pragma unroll
    for (int f = 0; f < 4; f++) {
      jx[f] = __shfl_sync(FULL, jf, base + 1 + f);
      fx[f] = __shfl_sync(FULL, Ff, base + 1 + f);
    }
    /* ---- the cell lane: the phi commit and the cell's own terms */
    if (live && part == 0) {
      const long long o = (long long)x * g.pitch + y;
      if (yb0 != 0.0) {
        atomicAdd(xbar + o, yb0);
        atomicAdd(dphibar + didx(g, 0, x, y), yb0);
      }
      if (yb1 != 0.0) {
        atomicAdd(xbar + g.plane + o, yb1);
        atomicAdd(dphibar + didx(g, 1, x, y), yb1);
      }
      if (ybm != 0.0) {
        if (bulk >= 0) {
          Mb[1][1] += dcb * c->cmu[bulk][0][0];   /* cn = c_mu(m) + ... */
        } else {
          /* nm = m + dc / dcdmu, dc = dt*divflux - divjat - sum */
          Mb[1][1] += ybm;
          double divflux = 0.0;
          divflux += adivx(fx[0] - fx[1], D);
          divflux += adivy(fx[2] - fx[3], D);
          double divjat = adivx((jx[0] - jx[1]) * cst, D);
          divjat += adivy((jx[2] - jx[3]) * cst, D);
          const double dp0 = DP[0][1][1], dp1 = DP[1][1][1];
          const double g0 = 6.0 * ph0 * (1.0 - ph0), g1 = 6.0 * ph1 * (1.0 - ph1);
          const double sdh0 = (0.0 + g0 * dp0) + (0.0 * ph0) * dp1, sdh1 = (0.0 + (0.0 * ph1) * dp0) + g1 * dp1;
          const double cm0 = 0.0 + c->cmu[0][0][0] * (m - c->E[0][0]), cm1 = 0.0 + c->cmu[1][0][0] * (m - c->E[1][0]);
          const double sum = (0.0 + cm0 * sdh0) + cm1 * sdh1;
          const double dc = c->dt * divflux - divjat - sum;
          const double i00 = 1.0 / dcdmu;
          /* dc / dcdmu */
          const double dcdmub = -ybm * dc * i00 * i00;
          Sb[0][1][1] += dcdmub * c->cmu64[0][0][0] * (6.0 * ph0 - 6.0 * ph0 * ph0);
          Sb[1][1][1] += dcdmub * c->cmu64[1][0][0] * (6.0 * ph1 - 6.0 * ph1 * ph1);
          /* - sum */
          const double sumb = -dcb;
          Mb[1][1] += sumb * (sdh0 * c->cmu[0][0][0] + sdh1 * c->cmu[1][0][0]);
          const double s0b = sumb * cm0, s1b = sumb * cm1;
          Db[1][1] += s0b * g0;
          if (s1b * g1 != 0.0) atomicAdd(dphibar + didx(g, 1, x, y), s1b * g1);
          Sb[0][1][1] += s0b * dp0 * (6.0 - 12.0 * ph0);
          Sb[1][1][1] += s1b * dp1 * (6.0 - 12.0 * ph1);
        }
      }
    }
    /* ---- the five lanes' window adjoints, summed on the cell lane, scattered
     * through the boundary copy tables */
#pragma unroll
    for (int di = 0; di < 3; di++)
#pragma unroll
      for (int dj = 0; dj < 3; dj++) {
        double v[4] = {Sb[0][di][dj], Sb[1][di][dj], Mb[di][dj], Db[di][dj]};
#pragma unroll
        for (int q = 0; q < 4; q++) {
          double t = v[q];
#pragma unroll
          for (int k = 1; k < 5; k++) t += __shfl_sync(FULL, v[q], base + k);
          v[q] = t;
        }
        if (live && part == 0) {
          const int xs = rmx(x + di - 1, g, c, 0), ys = rmy(y + dj - 1, g, c, 0);
#pragma unroll
          for (int a = 0; a < 2; a++)
            if (v[a] != 0.0) atomicAdd(xbar + a * g.plane + (long long)xs * g.pitch + ys, v[a]);
          if (v[2] != 0.0) {
            const int xm = rmx(x + di - 1, g, c, 1), ym = rmy(y + dj - 1, g, c, 1);
            atomicAdd(xbar + 2 * g.plane + (long long)xm * g.pitch + ym, v[2]);
          }
          if (v[3] != 0.0) atomicAdd(dphibar + didx(g, 0, x + di - 1, y + dj - 1), v[3]);
        }
      }
  }
  flush_params(pacc, pbar);
}

/* Reverse of the phase-field pass at ring or interior cell (x, y).  SORT:
 * returns whether the cell has an active phase (the only cells with a
 * derivative); the dual passes run with SORT false over the list of those. */
template <int N, int K, bool A, bool SORT>
__device__ __forceinline__ bool rev_dphi_cell(const Consts<double> *__restrict__ c, const AdjParams &prm,
                                              const Grid &g, const double *__restrict__ st,
                                              const double *__restrict__ dphibar, double *__restrict__ xbar, int x,
                                              int y, bool live, double (&pacc)[ADJ_NPARAM], int pass = -1) {
  using DT = Dual<ADJ_WD>;
  constexpr int NPHI = 9 * N, NIN = NPHI + K + ADJ_NPARAM;
  const int b0 = pass >= 0 ? pass * ADJ_WD : 0, b1 = pass >= 0 ? min(NIN, b0 + ADJ_WD) : NIN;
  double db[N];
  bool any = false;
  if (live) {
#pragma unroll
    for (int a = 0; a < N; a++) {
      db[a] = dphibar[didx(g, a, x, y)];
      any |= db[a] != 0.0;
    }
  }
  double S[N][3][3], M[K][3][3];
  if (live && any) {
    gather<N, K>(c, g, st, x, y, S, M);
    /* a cell with no active phase and no negative phi has delta-phi +0.0 whatever
     * its inputs within the branch (dphi_cell's first return): no derivative */
    bool active = false;
#pragma unroll
    for (int a = 0; a < N; a++) {
      double gxf = (S[a][2][1] - S[a][1][1]), gxb = (S[a][1][1] - S[a][0][1]);
      double gyr = (S[a][1][2] - S[a][1][1]), gyl = (S[a][1][1] - S[a][1][0]);
      active |= (gxf - gxb) != 0.0 || (gyr - gyl) != 0.0 || S[a][1][1] < 0.0;
    }
    any = active;
  }
  if (SORT) return live && any;
  if (live && any) {
    for (int base = b0; base < b1; base += ADJ_WD) {
      DT Sd[N][3][3], md[K], pd[ADJ_NPARAM];
      /* seeding by compile-time input numbers (registers, not local memory) */
#pragma unroll
      for (int a = 0; a < N; a++)
#pragma unroll
        for (int di = 0; di < 3; di++)
#pragma unroll
          for (int dj = 0; dj < 3; dj++) {
            Sd[a][di][dj] = DT(S[a][di][dj]);
#pragma unroll
            for (int w = 0; w < ADJ_WD; w++) Sd[a][di][dj].d[w] = (a * 9 + di * 3 + dj == base + w) ? 1.0 : 0.0;
          }
#pragma unroll
      for (int k = 0; k < K; k++) {
        md[k] = DT(M[k][1][1]);
#pragma unroll
        for (int w = 0; w < ADJ_WD; w++) md[k].d[w] = (NPHI + k == base + w) ? 1.0 : 0.0;
      }
#pragma unroll
      for (int j = 0; j < ADJ_NPARAM; j++) {
        pd[j] = DT(prm.v[j]);
#pragma unroll
        for (int w = 0; w < ADJ_WD; w++) pd[j].d[w] = (NPHI + K + j == base + w) ? 1.0 : 0.0;
      }
      const AK<DT> D = make_ak<DT>(c, pd);
      DT d[N];
      dphi_cell<DT, N, K, A>(D, Sd, md, d);
      for (int w = 0; w < ADJ_WD; w++) {
        const int id = base + w;
        if (id >= NIN) break;
        double gsum = 0.0;
#pragma unroll
        for (int a = 0; a < N; a++) gsum += db[a] * d[a].d[w];
        if (gsum == 0.0) continue;
        if (id < NPHI) {
          const int a = id / 9, r = id % 9;
          const int xs = rmx(x + r / 3 - 1, g, c, 0), ys = rmy(y + r % 3 - 1, g, c, 0);
          atomicAdd(xbar + a * g.plane + (long long)xs * g.pitch + ys, gsum);
        } else if (id < NPHI + K) {
          const int xs = rmx(x, g, c, 1), ys = rmy(y, g, c, 1);
          atomicAdd(xbar + (N + id - NPHI) * g.plane + (long long)xs * g.pitch + ys, gsum);
        } else {
#pragma unroll
          for (int j = 0; j < ADJ_NPARAM; j++)
            if (id - NPHI - K == j) pacc[j] += gsum;
        }
      }
    }
  }
  return false;
}

template <int N, int K, bool A>
__global__ void __launch_bounds__(AB) ka_rev_dphi(const Consts<double> *__restrict__ c, AdjParams prm, Grid g,
                                                  const double *__restrict__ st, const double *__restrict__ dphibar,
                                                  double *__restrict__ xbar, int2 *__restrict__ cells,
                                                  int *__restrict__ count) {
  const int y = blockIdx.x * AB + threadIdx.x - 1, x = (int)blockIdx.y - 1;
  double pacc[ADJ_NPARAM] = {};
  const bool want = rev_dphi_cell<N, K, A, true>(c, prm, g, st, dphibar, xbar, x, y, y <= g.my, pacc);
  push_cell(want, x, y, cells, count);
}

template <int N, int K, bool A>
__global__ void __launch_bounds__(AB) ka_rev_dphi_list(const Consts<double> *__restrict__ c, AdjParams prm, Grid g,
                                                       const double *__restrict__ st,
                                                       const double *__restrict__ dphibar, double *__restrict__ xbar,
                                                       double *__restrict__ pbar, const int2 *__restrict__ cells,
                                                       const int *__restrict__ count) {
  /* one thread per (cell, dual pass) */
  constexpr int NIN = 9 * N + K + ADJ_NPARAM, NPASS = (NIN + ADJ_WD - 1) / ADJ_WD;
  double pacc[ADJ_NPARAM] = {};
  const long long n = (long long)*count * NPASS;
  for (long long i = (long long)blockIdx.x * AB + threadIdx.x; i < n; i += (long long)gridDim.x * AB) {
    const int2 e = cells[i / NPASS];
    rev_dphi_cell<N, K, A, false>(c, prm, g, st, dphibar, xbar, e.x, e.y, true, pacc, (int)(i % NPASS));
  }
  flush_params(pacc, pbar);
}

/* ---- launchers ---------------------------------------------------------- */

template <int N, int K, bool A>
struct AdjKernels {
  static cudaError_t dphi(cudaStream_t s, const void *c, AdjParams p, Grid g, const double *st, double *dp) {
    dim3 grid((g.my + 2 + AB - 1) / AB, g.mx + 2);
    ka_dphi<N, K, A><<<grid, AB, 0, s>>>((const Consts<double> *)c, p, g, st, dp);
    return cudaGetLastError();
  }
  static cudaError_t dphi_sparse(cudaStream_t s, const void *c, AdjParams p, Grid g, const double *st, double *dp,
                                 int2 *cells, int *count) {
    cudaError_t e = cudaMemsetAsync(dp, 0, sizeof(double) * (size_t)N * g.dplane, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(count, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    dim3 grid((g.my + 2 + AB - 1) / AB, g.mx + 2);
    ka_dphi_sort<N, K><<<grid, AB, 0, s>>>((const Consts<double> *)c, g, st, cells, count);
    ka_dphi_list<N, K, A><<<list_grid(), AB, 0, s>>>((const Consts<double> *)c, p, g, st, dp, cells, count);
    return cudaGetLastError();
  }
  static cudaError_t update(cudaStream_t s, const void *c, AdjParams p, Grid g, const double *st, const double *dp,
                            double *next) {
    dim3 grid((g.my + AB - 1) / AB, g.mx);
    ka_update<N, K><<<grid, AB, 0, s>>>((const Consts<double> *)c, p, g, st, dp, next);
    return cudaGetLastError();
  }
  /* the list passes: a persistent grid over the listed cells */
  static int list_grid() {
    /* SM count per device, looked up once (every reverse step asks; a
     * repeated lookup writes the same value) */
    static int nsm_of[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 16 * 148;
    if (!nsm_of[dev]) {
      int nsm = 148;
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
      nsm_of[dev] = nsm;
    }
    return 16 * nsm_of[dev];
  }
  /* DUAL: the listed cells by dual passes, else by the hand-derived reverse */
  template <bool DUAL>
  static cudaError_t rev_update(cudaStream_t s, const void *c, AdjParams p, Grid g, const double *st,
                                const double *dp, const double *ybar, double *xbar, double *dpbar, double *pbar,
                                int2 *cells, int *count) {
    dim3 grid((g.my + AB - 1) / AB, g.mx);
    ka_rev_update<N, K><<<grid, AB, 0, s>>>((const Consts<double> *)c, p, g, st, dp, ybar, xbar, dpbar, cells, count);
    if (DUAL || N != 2 || K != 1)
      ka_rev_update_list<N, K><<<list_grid(), AB, 0, s>>>((const Consts<double> *)c, p, g, st, dp, ybar, xbar,
                                                          dpbar, pbar, cells, count);
    else
      ka_rev_update_hand<<<list_grid(), AB, 0, s>>>((const Consts<double> *)c, p, g, st, dp, ybar, xbar, dpbar, pbar,
                                                    cells, count);
    return cudaGetLastError();
  }
  static cudaError_t rev_dphi(cudaStream_t s, const void *c, AdjParams p, Grid g, const double *st,
                              const double *dpbar, double *xbar, double *pbar, int2 *cells, int *count) {
    dim3 grid((g.my + 2 + AB - 1) / AB, g.mx + 2);
    ka_rev_dphi<N, K, A><<<grid, AB, 0, s>>>((const Consts<double> *)c, p, g, st, dpbar, xbar, cells, count);
    ka_rev_dphi_list<N, K, A><<<list_grid(), AB, 0, s>>>((const Consts<double> *)c, p, g, st, dpbar, xbar, pbar,
                                                         cells, count);
    return cudaGetLastError();
  }
};

}  // namespace gpd

bool gp_adjoint_launch(int N, int K, bool aniso, gpd::AdjLaunch *out) {
  if (N != 2 || K != 1) return false;
  /* the concentration pass by dual passes; GP_ADJOINT_HAND_UPDATE: by the
   * hand-derived reverse (the two cross-check each other; the dual passes,
   * thirty threads per listed cell, hide latency better and are faster) */
  const bool dual = getenv("GP_ADJOINT_HAND_UPDATE") == nullptr;
  if (aniso) {
    out->dphi = gpd::AdjKernels<2, 1, true>::dphi;
    out->dphi_sparse = gpd::AdjKernels<2, 1, true>::dphi_sparse;
    out->update = gpd::AdjKernels<2, 1, true>::update;
    out->rev_update = dual ? gpd::AdjKernels<2, 1, true>::rev_update<true> : gpd::AdjKernels<2, 1, true>::rev_update<false>;
    out->rev_dphi = gpd::AdjKernels<2, 1, true>::rev_dphi;
  } else {
    out->dphi = gpd::AdjKernels<2, 1, false>::dphi;
    out->dphi_sparse = gpd::AdjKernels<2, 1, false>::dphi_sparse;
    out->update = gpd::AdjKernels<2, 1, false>::update;
    out->rev_update = dual ? gpd::AdjKernels<2, 1, false>::rev_update<true> : gpd::AdjKernels<2, 1, false>::rev_update<false>;
    out->rev_dphi = gpd::AdjKernels<2, 1, false>::rev_dphi;
  }
  return true;
}
