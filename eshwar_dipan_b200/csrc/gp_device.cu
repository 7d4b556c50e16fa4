/*
 * gp_device.cu -- libgp: the C ABI (include/gp.h) over the sm_100a kernels.
 * Host orchestration only; the kernels are in gp_fused.cuh (the stepping
 * engine), gp_tiles.cuh (shared tile code and the two-pass kernels of
 * gp_step_noalloc) and gp_smooth.cuh (the smoothing sweeps).
 *
 *  - gp_batch: simulations of different sizes and parameters stepped together
 *    by two kernels per step (bulk tiles, then interface tiles from a device
 *    work list), in FP64 (bit-identical to the reference step) or in the FP32
 *    storage form (gp_batch32.cu); steps are replayed as CUDA graphs of
 *    GP_GRAPH_STEPS steps.
 *  - gp_ctx: one simulation, a batch of one.
 *  - gp_step_noalloc: one FP64 step on caller-owned buffers, two-pass kernels
 *    with constants in __constant__ memory and a fixed scratch array.
 */
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cmath>
#include <climits>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <condition_variable>
#include <functional>
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <string>
#include <thread>
#include <vector>

#include "gp_adjoint_launch.h"
#include "gp_batch_impl.cuh"

static __constant__ gpd::Consts<double> cD;

extern "C" const char *gp_host_thread_error(void);

#define GP_GRAPH_STEPS 100
#define GP_GRAPH_CACHE 16     /* captured step sequences kept per batch */
#define GP_STAGE_BYTES ((size_t)8 << 20)   /* each of a device's two pinned host staging buffers */
#define GP_STAGE_MAX_DEVICES 64

/* ======================================================================= */
/* helpers                                                                 */
/* ======================================================================= */

namespace {

bool pow2(double v) {
  int e;
  double m = frexp(fabs(v), &e);
  return v != 0.0 && m == 0.5;
}

/* Constants of one simulation in the field type.  FP64 divides by dx/dy
 * unless they are powers of two (x*(1/dx) is then the same correctly rounded
 * value); the FP32 form always multiplies. */
template <typename R>
gpd::Consts<R> make_consts(const gp_derived &d) {
  gpd::Consts<R> c;
  memset(&c, 0, sizeof c);
  const bool f64 = sizeof(R) == 8;
  c.dx = (R)d.dx; c.dy = (R)d.dy; c.dt = (R)d.dt; c.eps = (R)d.eps; c.inv_eps = (R)d.inv_eps;
  c.tau = (R)d.tau; c.c16pi2 = (R)d.c16pi2; c.jat_obst = (R)d.jat_obst; c.jat_well = (R)d.jat_well;
  c.well_half = (R)d.well_half;
  c.mul_dx = f64 ? pow2(d.dx) : 1;
  c.mul_dy = f64 ? pow2(d.dy) : 1;
  c.inv_dx = (R)(1.0 / d.dx);
  c.inv_dy = (R)(1.0 / d.dy);
  c.inv_2dy = (R)(1.0 / (2.0 * d.dy));
  c.obstacle = d.obstacle; c.well = d.well; c.aniso = d.aniso; c.inv_mode = d.inv_mode;
  c.rot_identity = d.rot_identity;
  memcpy(c.bc_x, d.bc_x, sizeof c.bc_x);
  memcpy(c.bc_y, d.bc_y, sizeof c.bc_y);
  for (int a = 0; a < GPK_MAXN; a++) {
    for (int b = 0; b < GPK_MAXN; b++) {
      c.gamma[a][b] = (R)d.gamma[a][b]; c.tau_ab[a][b] = (R)d.tau_ab[a][b];
      c.dab16[a][b] = (R)d.dab16[a][b]; c.dab[a][b] = (R)d.dab[a][b];
      for (int e = 0; e < GPK_MAXN; e++) c.gamma_abc[a][b][e] = (R)d.gamma_abc[a][b][e];
      for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) { c.rot[a][b][i][j] = (R)d.rot[a][b][i][j]; c.rinv[a][b][i][j] = (R)d.rinv[a][b][i][j]; }
    }
    for (int i = 0; i < GPK_MAXK; i++) {
      c.E[a][i] = (R)d.E[a][i]; c.twoA[a][i] = (R)d.twoA[a][i]; c.B[a][i] = (R)d.B[a][i]; c.atf[a][i] = (R)d.atf[a][i];
      for (int j = 0; j < GPK_MAXK; j++) {
        c.cmu[a][i][j] = (R)d.cmu[a][i][j]; c.cmu64[a][i][j] = d.cmu[a][i][j];
        c.muc64[a][i][j] = i == j ? d.twoA[a][i] : d.A[a][i][j];
        c.A[a][i][j] = (R)d.A[a][i][j]; c.Dbulk[a][i][j] = (R)d.Dbulk[a][i][j];
        for (int k = 0; k < GPK_MAXK; k++) c.DC[a][i][j][k] = (R)d.DC[a][i][j][k];
      }
    }
    c.C[a] = (R)d.C[a];
  }
  c.tgrad = d.tgrad;
  c.bc_t[0] = d.bc_t[0];
  c.bc_t[1] = d.bc_t[1];
  c.Teq64 = d.Teq;
  for (int a = 0; a < GPK_MAXN; a++) {
    for (int i = 0; i < GPK_MAXK; i++) {
      c.Beq64[a][i] = d.Beq[a][i];
      c.dBbdT64[a][i] = d.dBbdT[a][i];
      c.ceql[a][i] = d.ceql[a][i];
      c.ceqs[a][i] = d.ceqs[a][i];
      c.DCk[a][i] = d.DCk[a][i];
      for (int j = 0; j < GPK_MAXK; j++) c.A64[a][i][j] = d.A[a][i][j];
    }
    c.DTl[a] = d.DTl[a];
    c.DTs[a] = d.DTs[a];
  }
  c.tg_base = d.tg_base; c.tg_dT = d.tg_dT; c.tg_dist = d.tg_dist; c.tg_off = d.tg_off; c.tg_vel = d.tg_vel;
  c.dx64 = d.dx; c.dy64 = d.dy; c.dt64 = d.dt;
  c.shift = d.shift;
  c.shiftj = (int)d.shiftj;
  for (int i = 0; i < GPK_MAXK; i++) c.mu_fill[i] = (R)d.mu_fill[i];
  return c;
}

gpd::Grid make_grid(const gp_derived &d, int pitch_multiple) {
  gpd::Grid g;
  g.mx = (int)d.mx;
  g.my = (int)d.my;
  g.pitch = (int)((d.my + pitch_multiple - 1) / pitch_multiple * pitch_multiple);
  g.plane = (long long)g.pitch * d.mx;
  g.dpitch = (int)((d.my + 2 + 31) / 32 * 32);
  g.dplane = (long long)g.dpitch * (d.mx + 2);
  g.sx0 = 0;
  g.sx1 = (int)d.mx;
  return g;
}

/* Fold per-tile sums of simulation blockIdx.y (tiles [tile0, tile0+ntile))
 * in a fixed order; one CTA per (quantity, simulation). */
__global__ void k_reduce_sums(const double *__restrict__ part, const int *__restrict__ tile0,
                              const int *__restrict__ ntile, int nsum, double *__restrict__ out) {
  __shared__ double r[256];
  const int f = blockIdx.x, s = blockIdx.y, t0 = tile0[s], nt = ntile[s];
  double v = 0.0;
  for (int b = threadIdx.x; b < nt; b += 256) v += part[(long long)(t0 + b) * nsum + f];
  r[threadIdx.x] = v;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) r[threadIdx.x] += r[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[(long long)s * nsum + f] = r[0];
}

double from_ord(long long i) {
  if (i < 0) i ^= 0x7fffffffffffffffLL;
  double v;
  memcpy(&v, &i, 8);
  return v;
}
long long to_ord(double v) {
  long long i;
  memcpy(&i, &v, 8);
  return i < 0 ? i ^ 0x7fffffffffffffffLL : i;
}

/* running extremes start where the reference starts them (serialinfo_xy.h:59-66):
 * phi max 1, min 0; mu max 1, min 1 */
void init_ext(long long *s, int N, int K) {
  for (int a = 0; a < N; a++) { s[a] = to_ord(1.0); s[N + a] = to_ord(0.0); }
  for (int k = 0; k < K; k++) { s[2 * N + k] = to_ord(1.0); s[2 * N + K + k] = to_ord(1.0); }
}

void stats_from(gp_stats *r, const long long *mm, const double *sums, int N, int K, long long steps) {
  memset(r, 0, sizeof *r);
  for (int a = 0; a < N; a++) {
    r->phi_max[a] = from_ord(mm[a]);
    r->phi_min[a] = from_ord(mm[N + a]);
    r->rel_change_phi[a] = sums[a];
    r->phi_sum[a] = sums[N + K + a];
  }
  for (int k = 0; k < K; k++) {
    r->mu_max[k] = from_ord(mm[2 * N + k]);
    r->mu_min[k] = from_ord(mm[2 * N + K + k]);
    r->rel_change_mu[k] = sums[N + k];
    r->comp_sum[k] = sums[2 * N + K + k];
  }
  r->nonfinite = (long long)llround(sums[2 * N + 2 * K]);
  r->steps_done = steps;
}

}  // namespace

/* ======================================================================= */
/* two-pass FP64 kernels of gp_step_noalloc: one CTA per tile, constants   */
/* in __constant__ memory                                                  */
/* ======================================================================= */

namespace gpd {

template <int N, int K, bool A>
__global__ void __launch_bounds__(NT) k_dphi(const double *__restrict__ phi, const double *__restrict__ mu,
                                             double *__restrict__ dphi, Grid g) {
  extern __shared__ __align__(16) unsigned char smraw[];
  dphi_tile<double, N, K, A>(cD, g, phi, mu, dphi, blockIdx.y * TX - 1, blockIdx.x * TY - 1,
                             *reinterpret_cast<DphiSmem<double, N> *>(smraw));
}

template <int N, int K>
__global__ void __launch_bounds__(NT) k_update(const double *__restrict__ phi, const double *__restrict__ mu,
                                               const double *__restrict__ dphi, double *__restrict__ phin,
                                               double *__restrict__ mun, Grid g, StatBufs st) {
  extern __shared__ __align__(16) unsigned char smraw[];
  update_tile<double, N, K>(cD, g, phi, mu, dphi, phin, mun, blockIdx.y * TX, blockIdx.x * TY, st,
                            (long long)blockIdx.y * gridDim.x + blockIdx.x,
                            *reinterpret_cast<UpdSmem<double, N, K> *>(smraw));
}

}  // namespace gpd

namespace {

struct Kern {
  void (*dphi)(const double *, const double *, double *, gpd::Grid);
  void (*upd)(const double *, const double *, const double *, double *, double *, gpd::Grid, gpd::StatBufs);
  size_t smem_dphi, smem_upd;
};

template <int N, int K, bool A>
Kern make() {
  Kern k;
  k.dphi = gpd::k_dphi<N, K, A>;
  k.upd = gpd::k_update<N, K>;
  k.smem_dphi = sizeof(gpd::DphiSmem<double, N>);
  k.smem_upd = sizeof(gpd::UpdSmem<double, N, K>);
  return k;
}

bool pick(int N, int K, bool A, Kern *out) {
#define CASE(n, k)                                       \
  if (N == n && K == k) {                                \
    *out = A ? make<n, k, true>() : make<n, k, false>(); \
    return true;                                         \
  }
  CASE(2, 1) CASE(3, 1) CASE(4, 1) CASE(2, 2) CASE(3, 2) CASE(4, 2)
#undef CASE
  return false;
}

}  // namespace

bool gp_batch_launch_f64(int N, int K, bool aniso, gpd::BatchLaunch *out) {
  return gpd::batch_launch_table<double>(N, K, aniso, out);
}


struct gp_batch;

/* A single simulation is a batch of one. */
struct gp_ctx {
  gp_batch *b;
  char err[256];
  /* background VTK write (gp_vtk_write_async) */
  std::thread *writer;          /* the write in flight, or NULL */
  int wstatus;                  /* its result */
  char werr[256];
  void *snap;                   /* device copy of the state being written (then the frame state) */
  long long wsteps;             /* steps taken when the snapshot was queued */
  cudaStream_t wstream;         /* the writer's copies */
  cudaEvent_t wready;           /* the snapshot is complete */
  double *hphi, *hmu, *htemp;   /* host copies of the snapshot; its temperature field */
};

static int fail(gp_ctx *c, int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  if (c) vsnprintf(c->err, sizeof c->err, fmt, ap);
  else {
    char buf[256];
    vsnprintf(buf, sizeof buf, fmt, ap);
    gp_set_thread_error("%s", buf);
  }
  va_end(ap);
  return code;
}

#define CK(call)                                                                                \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess) return fail(c, GP_ECUDA, "%s: %s", #call, cudaGetErrorString(e_));  \
  } while (0)

/* ======================================================================= */
/* batches                                                                 */
/* ======================================================================= */

/* How a step is launched; every shape gives the same bits (tiles are
 * independent of the warp or CTA that steps them), so shapes can be timed on
 * the live simulation. */
struct LaunchShape {
  bool fused;        /* kf_step (one launch) rather than kf_bulk + kf_general */
  int bch_max, bch_div;
  bool mixed;        /* kf_step: odd CTAs start with bulk tiles, even ones with interface tiles */
};
/* batches that share these tune alike: the first one's choice is kept for
 * the process */
struct ShapeKey {
  int N, K, aniso, elem, tiles_log2;
  bool operator<(const ShapeKey &o) const {
    return std::tie(N, K, aniso, elem, tiles_log2) < std::tie(o.N, o.K, o.aniso, o.elem, o.tiles_log2);
  }
};
static std::map<ShapeKey, LaunchShape> g_shapes;
static std::mutex g_shapes_mutex;

struct gp_batch {
  int nsims, N, K, aniso;
  gp_precision prec;
  size_t elem;
  gpd::BatchLaunch L;
  std::vector<gp_params> params;
  std::vector<gp_derived> derived;
  std::vector<gpd::SimDesc> desc;
  int dev, nsm, grid_b, grid_g, grid_s;   /* grid_s: kf_step (0: bulk and interface kernels apart) */
  bool mul;                     /* every simulation's dx and dy are powers of two (or FP32) */
  bool diag;                    /* off-diagonal D, c_mu, A all zero and no E is -0, in every simulation */
  int mbar_tries;               /* kf_bulk's polls of a box barrier before it reports an error */
  LaunchShape shape;            /* how a step is launched (tuned on the first graph chunks) */
  LaunchShape cand[6];          /* the candidates */
  float cand_ms[6];
  int ncand, tune_next;         /* tuning is over when tune_next == ncand */
  ShapeKey key;
  unsigned tma_extra;           /* 0; a test sets more (GP_TEST_TMA_SHORTFALL) to make the boxes never complete */
  int ntiles;                   /* TX x TY tiles over all simulations */
  cudaStream_t stream;
  gpd::SimDesc *d_desc;
  void *d_consts;
  size_t consts_bytes;
  int *d_tsim, *d_seg0, *d_segn;
  void *state[2];               /* ping-pong: every simulation's N phi then K mu planes */
  gpd::TileFlags *flags[2];     /* per tile and state buffer: one-hot phase of the tile and its edge bands */
  int *glist;                   /* interface tiles of the current step */
  int4 *blist;                  /* bulk tiles of the current step (entries written by kf_classify) */
  int *counters;                /* gpd::CTR_* */
  gpd::TensorMapSlot *tmaps;    /* [nsims][2]: TMA maps of each simulation's mu planes in state[0], state[1] */
  int cur;
  long long *ext;               /* running extremes per simulation [nsims][2(N+K)] */
  bool tgrad;                   /* some simulation is non-isothermal: temperature rows each step */
  bool shift;                   /* some simulation has the moving frame: a check every 100 steps */
  int *spos;                    /* its interface position per simulation */
  double *trows;                /* their temperature rows (SimDesc::off_T) */
  gpd::SimDyn *dyn;             /* per simulation moving-frame state */
  double *dphi_out = nullptr;   /* the adjoint's forward steps: where the interface tiles write delta-phi */
  /* the adjoint's forward steps over its tape (a batch of one): the step reads
   * redir_in (bulk boxes through redir_map) and writes redir_out instead of
   * the ping-pong buffers; the flags still follow the parity.  redir_have
   * stands in for the output buffer's flags in the classification: "unknown"
   * for every tile, since redir_out holds nothing the flags describe (the
   * bulk tiles then write their phi too) */
  const void *redir_in = nullptr;
  void *redir_out = nullptr;
  const gpd::TensorMapSlot *redir_map = nullptr;
  const gpd::TileFlags *redir_have = nullptr;
  double *partials, *sums_sim;
  /* captured step sequences: graphs[(starting parity, steps)], steps <= GP_GRAPH_STEPS */
  std::map<std::pair<int, long>, cudaGraphExec_t> graphs;
  cudaEvent_t ev[4];
  long long steps;
  std::vector<gp_stats> last;
  char err[256];
};

static int bfail(gp_batch *b, int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  char buf[256];
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (b) snprintf(b->err, sizeof b->err, "%s", buf);
  gp_set_thread_error("%s", buf);
  return code;
}

#define BK(call)                                                                                 \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess) return bfail(b, GP_ECUDA, "%s: %s", #call, cudaGetErrorString(e_));  \
  } while (0)

/* One step: bulk tiles (and the interface list), then the interface tiles.
 * ev: optional events around the two kernels. */
static int batch_step_once(gp_batch *b, int want_sums, cudaEvent_t *ev) {
  gpd::StatBufs st = {};
  st.ext = b->ext;
  st.partials = b->partials;
  st.want_sums = want_sums;
  st.round_step = (const unsigned *)(b->counters + gpd::CTR_STEP);
  st.mbar_tries = b->mbar_tries;
  st.tma_extra = b->tma_extra;
  st.dphi_out = b->dphi_out;
  st.bch_max = b->shape.bch_max;
  st.mixed = b->shape.mixed ? 1 : 0;
  st.trows = b->tgrad ? b->trows : nullptr;
  st.bch_div = b->shape.bch_div;
  const int in = b->cur, out = b->cur ^ 1;
  const void *sin = b->redir_in ? b->redir_in : b->state[in];
  void *sout = b->redir_in ? b->redir_out : b->state[out];
  const gpd::TensorMapSlot *tmaps = b->redir_in ? b->redir_map : b->tmaps;
  const int tbuf = b->redir_in ? 0 : in;
  if (ev) BK(cudaEventRecord(ev[0], b->stream));
  if (b->tgrad) BK(b->L.trows(b->nsims, b->stream, b->d_desc, b->d_consts, b->counters, b->dyn, b->trows));
  BK(b->L.classify(b->ntiles, b->stream, b->d_desc, b->d_consts, b->d_tsim, b->flags[in],
                   b->redir_in ? b->redir_have : b->flags[out], b->glist, b->blist, b->counters));
  if (!want_sums && b->grid_s > 0 && b->shape.fused && (!ev || ev[3] == nullptr)) {
    /* one launch for both kinds of tile; ev (with ev[3] null): events after
     * the classification and after the step */
    if (ev) BK(cudaEventRecord(ev[1], b->stream));
    BK(b->L.step(b->grid_s, b->mul, b->diag, b->stream, b->d_desc, b->d_consts, b->d_tsim, b->blist, b->glist,
                 tmaps, tbuf, sin, sout, b->flags[out], b->counters, b->grid_s, st));
    if (ev) BK(cudaEventRecord(ev[2], b->stream));
    b->cur = out;
    b->steps++;
    return GP_OK;
  }
  /* kf_bulk then kf_general; the last CTA of the two resets the lists */
  const int nd = b->grid_b + b->grid_g;
  BK(b->L.bulk(b->grid_b, b->mul, b->diag, b->stream, b->d_desc, b->d_consts, b->d_tsim, b->blist, tmaps, tbuf,
               sin, sout, b->flags[out], b->counters, nd, st));
  if (ev) BK(cudaEventRecord(ev[1], b->stream));
  BK(b->L.general(b->grid_g, b->mul, b->stream, b->d_desc, b->d_consts, b->d_tsim, sin, sout,
                  b->flags[out], b->glist, b->counters, nd, st));
  if (ev) BK(cudaEventRecord(ev[2], b->stream));
  b->cur = out;
  b->steps++;
  return GP_OK;
}

/* Flags of the current buffer from its contents; the other buffer's are
 * unknown (it is rewritten in full by the next step). */
static int batch_reflag(gp_batch *b, bool other_unknown) {
  BK(b->L.flags(b->ntiles, b->stream, b->d_desc, b->d_tsim, b->state[b->cur], b->flags[b->cur]));
  if (other_unknown)
    BK(cudaMemsetAsync(b->flags[b->cur ^ 1], 0xfe, sizeof(gpd::TileFlags) * (size_t)b->ntiles, b->stream));
  return GP_OK;
}

/* The moving-frame check after a step whose number is a multiple of 100
 * (microsim_gp.c:115-123): every simulation's state goes to the other buffer,
 * shifted where its interface passed Shiftj, copied otherwise. */
static int batch_shift(gp_batch *b) {
  BK(cudaMemsetAsync(b->spos, 0, sizeof(int) * (size_t)b->nsims, b->stream));
  BK(b->L.shift_pos(b->ntiles, b->stream, b->d_desc, b->d_consts, b->d_tsim, b->state[b->cur], b->spos));
  BK(b->L.shift_apply(b->ntiles, b->stream, b->d_desc, b->d_consts, b->d_tsim, b->state[b->cur], b->state[b->cur ^ 1],
                      b->spos, b->dyn));
  b->cur ^= 1;
  return batch_reflag(b, true);
}

static int batch_fold_stats(gp_batch *b, gp_stats *out) {
  const int N = b->N, K = b->K, ne = 2 * (N + K), ns = 2 * N + 2 * K + 1;
  k_reduce_sums<<<dim3(ns, b->nsims), 256, 0, b->stream>>>(b->partials, b->d_seg0, b->d_segn, ns, b->sums_sim);
  BK(cudaGetLastError());
  std::vector<long long> mm((size_t)ne * b->nsims);
  std::vector<double> sums((size_t)ns * b->nsims);
  BK(cudaMemcpyAsync(mm.data(), b->ext, mm.size() * 8, cudaMemcpyDeviceToHost, b->stream));
  BK(cudaMemcpyAsync(sums.data(), b->sums_sim, sums.size() * 8, cudaMemcpyDeviceToHost, b->stream));
  std::vector<gpd::SimDyn> dyn(b->nsims);
  BK(cudaMemcpyAsync(dyn.data(), b->dyn, sizeof(gpd::SimDyn) * dyn.size(), cudaMemcpyDeviceToHost, b->stream));
  BK(cudaStreamSynchronize(b->stream));
  for (int s = 0; s < b->nsims; s++) {
    stats_from(&b->last[s], &mm[(size_t)s * ne], &sums[(size_t)s * ns], N, K, b->steps);
    b->last[s].shift_offset = dyn[s].shift_off;
    if (out) out[s] = b->last[s];
  }
  return GP_OK;
}

/* The error flag of the step kernels (a TMA box of kf_bulk that did not
 * arrive within its poll limit): read, clear, report. */
static int batch_check_error(gp_batch *b) {
  int e = 0;
  BK(cudaMemcpyAsync(&e, b->counters + gpd::CTR_ERR, sizeof e, cudaMemcpyDeviceToHost, b->stream));
  BK(cudaStreamSynchronize(b->stream));
  if (e) {
    BK(cudaMemsetAsync(b->counters + gpd::CTR_ERR, 0, sizeof e, b->stream));
    return bfail(b, GP_ETIMEOUT, "kf_bulk: a tile's mu did not arrive within the wait limit; the state is not valid");
  }
  return GP_OK;
}

/* GP_ENONFINITE when the statistics just folded count non-finite interior
 * cells in any simulation (the steps are done and the statistics filled). */
static int batch_check_finite(gp_batch *b) {
  for (int s = 0; s < b->nsims; s++)
    if (b->last[s].nonfinite > 0)
      return bfail(b, GP_ENONFINITE, "simulation %d: %lld interior cells hold a non-finite phi or mu after step %lld", s,
                   b->last[s].nonfinite, b->steps);
  return GP_OK;
}

/* Drop every captured graph (the launch shape they were captured with is no
 * longer the batch's). */
static void batch_drop_graphs(gp_batch *b) {
  for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);
  b->graphs.clear();
}

/* The graph of n steps from the current parity, captured on first use; null
 * when the cache is full (the caller then launches the steps one by one). */
static int batch_graph(gp_batch *b, long n, bool shift_at_end, cudaGraphExec_t *out) {
  *out = nullptr;
  const auto key = std::make_pair(b->cur, n | (shift_at_end ? (1L << 30) : 0L));
  auto it = b->graphs.find(key);
  if (it != b->graphs.end()) {
    *out = it->second;
    return GP_OK;
  }
  if (b->graphs.size() >= GP_GRAPH_CACHE) return GP_OK;
  cudaGraph_t gr;
  BK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  int rc = GP_OK;
  const int cur0 = b->cur;
  for (long i = 0; i < n && rc == GP_OK; i++) rc = batch_step_once(b, 0, nullptr);
  if (rc == GP_OK && shift_at_end) rc = batch_shift(b);
  b->steps -= n; /* captured, not run */
  b->cur = cur0;
  cudaError_t ec = cudaStreamEndCapture(b->stream, &gr);
  if (rc != GP_OK) return rc;
  if (ec != cudaSuccess) return bfail(b, GP_ECUDA, "graph capture: %s", cudaGetErrorString(ec));
  cudaGraphExec_t ge;
  ec = cudaGraphInstantiate(&ge, gr, 0);
  cudaGraphDestroy(gr);
  if (ec != cudaSuccess) return bfail(b, GP_ECUDA, "graph instantiate: %s", cudaGetErrorString(ec));
  b->graphs[key] = ge;
  *out = ge;
  return GP_OK;
}

/* nsteps steps, replayed as CUDA graphs of up to GP_GRAPH_STEPS steps (one
 * graph per starting ping-pong parity and length, captured on first use);
 * when statistics are asked for, the last step runs outside a graph so that
 * it can produce the sums.  While the launch-shape autotuner has candidates
 * left, whole GP_GRAPH_STEPS chunks time them.  With ms_bulk/ms_iface every
 * step runs outside graphs with events around the two kernels. */
static int batch_step_impl(gp_batch *b, long nsteps, gp_stats *stats, double *total_ms, double *ms_bulk,
                           double *ms_iface) {
  const bool split = ms_bulk || ms_iface;
  double tb = 0.0, ti = 0.0;
  if (total_ms) BK(cudaEventRecord(b->ev[3], b->stream));
  long s = 0;
  const long graphed = stats ? nsteps - 1 : nsteps;   /* steps that may run inside graphs */
  while (!split && graphed - s >= 2) {
    long n = std::min<long>(GP_GRAPH_STEPS, graphed - s);
    bool sh = false;
    if (b->shift) {   /* chunks end at the moving frame's checks */
      const long to_check = GP_GRAPH_STEPS - (long)(b->steps % GP_GRAPH_STEPS);
      if (n >= to_check) { n = to_check; sh = true; }
      if (n < 2) break;
    }
    if (b->tune_next < b->ncand && n == GP_GRAPH_STEPS) {
      /* autotuning: one 100-step chunk per candidate shape, each captured
       * afresh and timed with events; then the fastest is kept */
      b->shape = b->cand[b->tune_next];
      cudaGraph_t gr;
      cudaGraphExec_t ge;
      BK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      int rc = GP_OK;
      for (int i = 0; i < GP_GRAPH_STEPS && rc == GP_OK; i++) rc = batch_step_once(b, 0, nullptr);
      b->steps -= GP_GRAPH_STEPS;
      cudaError_t ec = cudaStreamEndCapture(b->stream, &gr);
      if (rc != GP_OK) return rc;
      if (ec != cudaSuccess) return bfail(b, GP_ECUDA, "graph capture: %s", cudaGetErrorString(ec));
      ec = cudaGraphInstantiate(&ge, gr, 0);
      cudaGraphDestroy(gr);
      if (ec != cudaSuccess) return bfail(b, GP_ECUDA, "graph instantiate: %s", cudaGetErrorString(ec));
      BK(cudaEventRecord(b->ev[0], b->stream));
      BK(cudaGraphLaunch(ge, b->stream));
      BK(cudaEventRecord(b->ev[1], b->stream));
      BK(cudaEventSynchronize(b->ev[1]));
      cudaGraphExecDestroy(ge);
      BK(cudaEventElapsedTime(&b->cand_ms[b->tune_next], b->ev[0], b->ev[1]));
      if (++b->tune_next == b->ncand) {
        int best = 0;
        for (int i = 1; i < b->ncand; i++)
          if (b->cand_ms[i] < b->cand_ms[best]) best = i;
        b->shape = b->cand[best];
        batch_drop_graphs(b);   /* captured with a candidate's shape */
        std::lock_guard<std::mutex> lock(g_shapes_mutex);
        g_shapes[b->key] = b->shape;
      }
      b->steps += GP_GRAPH_STEPS;
      s += GP_GRAPH_STEPS;
      continue;
    }
    cudaGraphExec_t ge = nullptr;
    int rc = batch_graph(b, n, sh, &ge);
    if (rc != GP_OK) return rc;
    if (!ge) break;   /* cache full: the rest one by one */
    BK(cudaGraphLaunch(ge, b->stream));
    if ((n & 1) ^ (sh ? 1 : 0)) b->cur ^= 1;
    b->steps += n;
    s += n;
  }
  for (; s < nsteps; s++) {
    int rc = batch_step_once(b, stats != nullptr && s == nsteps - 1, split ? b->ev : nullptr);
    if (rc != GP_OK) return rc;
    if (b->shift && b->steps % GP_GRAPH_STEPS == 0 && (rc = batch_shift(b)) != GP_OK) return rc;
    if (split) {
      float x = 0.f, y = 0.f;
      BK(cudaEventSynchronize(b->ev[2]));
      BK(cudaEventElapsedTime(&x, b->ev[0], b->ev[1]));
      BK(cudaEventElapsedTime(&y, b->ev[1], b->ev[2]));
      tb += x;
      ti += y;
    }
  }
  if (total_ms) {
    float ms = 0.f;
    BK(cudaEventRecord(b->ev[2], b->stream));
    BK(cudaEventSynchronize(b->ev[2]));
    BK(cudaEventElapsedTime(&ms, b->ev[3], b->ev[2]));
    *total_ms = ms;
  }
  if (ms_bulk) *ms_bulk = tb;
  if (ms_iface) *ms_iface = ti;
  int rc = batch_check_error(b);
  if (rc != GP_OK) return rc;
  if (stats && nsteps > 0) {
    if ((rc = batch_fold_stats(b, stats)) != GP_OK) return rc;
    return batch_check_finite(b);
  }
  BK(cudaStreamSynchronize(b->stream));
  if (stats)
    for (int i = 0; i < b->nsims; i++) stats[i] = b->last[i];
  return GP_OK;
}

/* Pinned host staging buffers of gp_set/gp_get, one pair per device. */
struct StagePair {
  void *buf[2];
  cudaEvent_t ev[2];
};
static StagePair g_stage[GP_STAGE_MAX_DEVICES];
static std::mutex g_stage_mutex;

/* A few host threads that stay up for the staging copies: a chunk's copy is
 * split over them and the caller, without a thread start per chunk (a 671 MB
 * transfer is ~80 chunks).  One job at a time: the staging copies run under
 * g_stage_mutex. */
class HostPool {
 public:
  static constexpr int MAXW = 7;   /* workers besides the caller */
  static HostPool &get() {
    static HostPool pool;
    return pool;
  }
  /* run part(i) for i in [0, n) on the workers and the caller; returns when all are done */
  void run(int n, const std::function<void(int)> &part) {
    std::unique_lock<std::mutex> lk(mu_);
    job_ = &part;
    njobs_ = n;
    next_ = 0;
    finished_ = 0;
    gen_++;
    cv_.notify_all();
    while (true) {
      if (next_ >= njobs_) break;
      const int i = next_++;
      lk.unlock();
      part(i);
      lk.lock();
      finished_++;
    }
    done_.wait(lk, [this] { return finished_ == njobs_; });
    job_ = nullptr;
  }
  ~HostPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto &t : th_) t.join();
  }

 private:
  HostPool() {
    const unsigned hc = std::thread::hardware_concurrency();
    const int nw = (int)std::min<unsigned>(MAXW, hc > 1 ? hc - 1 : 0);
    for (int w = 0; w < nw; w++) th_.emplace_back([this] { loop(); });
  }
  void loop() {
    long seen = 0;
    std::unique_lock<std::mutex> lk(mu_);
    while (true) {
      cv_.wait(lk, [&] { return stop_ || (gen_ != seen && job_ && next_ < njobs_); });
      if (stop_) return;
      seen = gen_;
      while (job_ && next_ < njobs_) {
        const int i = next_++;
        const std::function<void(int)> *f = job_;
        lk.unlock();
        (*f)(i);
        lk.lock();
        if (++finished_ == njobs_) done_.notify_all();
      }
    }
  }
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_, done_;
  const std::function<void(int)> *job_ = nullptr;
  int njobs_ = 0, next_ = 0, finished_ = 0;
  long gen_ = 0;
  bool stop_ = false;
};

/* Host-side copy of n bytes (or conversion of n elements) split over the
 * pool when it is large: a single thread moves about 10 GB/s, below what the
 * DMA engines take from pinned memory. */
template <typename F>
static void host_parallel(size_t n, size_t grain, F &&part) {
  const int nt = (int)std::min<size_t>(HostPool::MAXW + 1, std::max<size_t>(1, n / grain));
  if (nt == 1) {
    part((size_t)0, n);
    return;
  }
  const size_t per = (n + nt - 1) / nt;
  const std::function<void(int)> f = [&](int i) {
    const size_t lo = std::min(n, (size_t)i * per), hi = std::min(n, lo + per);
    if (lo < hi) part(lo, hi);
  };
  HostPool::get().run(nt, f);
}

/* nf device planes (rows of my elements of es bytes, dpitch bytes apart;
 * planes plane_bytes apart from base) and nf host arrays of mx*my doubles */
struct StagedPlanes {
  int dev;
  char *base;
  size_t plane_bytes, dpitch, mx, my, es;
  int nf;
};

/* Host arrays -> device planes through the device's pinned staging pair, in
 * chunks of rows: the host copy (FP64) or conversion (FP32) of one chunk
 * overlaps the DMA of the other.  Work is ordered on `stream`; returns when
 * the last DMA is queued. */
static cudaError_t stage_up(const StagedPlanes &sp, double *const *host, cudaStream_t stream) {
  std::lock_guard<std::mutex> lock(g_stage_mutex);
  if (sp.dev < 0 || sp.dev >= GP_STAGE_MAX_DEVICES) return cudaErrorInvalidDevice;
  StagePair &pr = g_stage[sp.dev];
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < 2 && !pr.buf[0 + i]; i++) {
    if ((e = cudaHostAlloc(&pr.buf[i], GP_STAGE_BYTES, cudaHostAllocDefault)) != cudaSuccess) return e;
    if ((e = cudaEventCreateWithFlags(&pr.ev[i], cudaEventDisableTiming)) != cudaSuccess) return e;
  }
  const size_t rows_per = std::max<size_t>(1, GP_STAGE_BYTES / (sp.my * sp.es)), grain = (size_t)1 << 20;
  size_t i = 0;
  for (int f = 0; f < sp.nf; f++)
    for (size_t r0 = 0; r0 < sp.mx; r0 += rows_per, i++) {
      const size_t nr = std::min(rows_per, sp.mx - r0), n = nr * sp.my;
      const int k = (int)(i & 1);
      if (i >= 2 && (e = cudaEventSynchronize(pr.ev[k])) != cudaSuccess) return e;   /* last DMA from it */
      const double *src = host[f] + r0 * sp.my;
      if (sp.es == 8) {
        char *dst = (char *)pr.buf[k];
        host_parallel(n * 8, grain, [&](size_t lo, size_t hi) { memcpy(dst + lo, (const char *)src + lo, hi - lo); });
      } else {
        float *dst = (float *)pr.buf[k];
        host_parallel(n, grain / 4, [&](size_t lo, size_t hi) {
          for (size_t j = lo; j < hi; j++) dst[j] = (float)src[j];
        });
      }
      if ((e = cudaMemcpy2DAsync(sp.base + f * sp.plane_bytes + r0 * sp.dpitch, sp.dpitch, pr.buf[k], sp.my * sp.es,
                                 sp.my * sp.es, nr, cudaMemcpyHostToDevice, stream)) != cudaSuccess)
        return e;
      if ((e = cudaEventRecord(pr.ev[k], stream)) != cudaSuccess) return e;
    }
  /* the staging pair is reused by the next caller: wait for the last DMAs */
  for (int k = 0; k < 2; k++)
    if ((e = cudaEventSynchronize(pr.ev[k])) != cudaSuccess) return e;
  return cudaSuccess;
}

/* Device planes -> host arrays, the DMA of one chunk overlapping the host
 * copy of the previous one. */
static cudaError_t stage_down(const StagedPlanes &sp, double *const *host, cudaStream_t stream) {
  std::lock_guard<std::mutex> lock(g_stage_mutex);
  if (sp.dev < 0 || sp.dev >= GP_STAGE_MAX_DEVICES) return cudaErrorInvalidDevice;
  StagePair &pr = g_stage[sp.dev];
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < 2 && !pr.buf[0 + i]; i++) {
    if ((e = cudaHostAlloc(&pr.buf[i], GP_STAGE_BYTES, cudaHostAllocDefault)) != cudaSuccess) return e;
    if ((e = cudaEventCreateWithFlags(&pr.ev[i], cudaEventDisableTiming)) != cudaSuccess) return e;
  }
  const size_t rows_per = std::max<size_t>(1, GP_STAGE_BYTES / (sp.my * sp.es)), grain = (size_t)1 << 20;
  struct Chunk {
    int f;
    size_t r0, nr;
  };
  std::vector<Chunk> ch;
  for (int f = 0; f < sp.nf; f++)
    for (size_t r = 0; r < sp.mx; r += rows_per) ch.push_back({f, r, std::min(rows_per, sp.mx - r)});
  auto fetch = [&](size_t i) {
    const int k = (int)(i & 1);
    cudaError_t x = cudaMemcpy2DAsync(pr.buf[k], sp.my * sp.es, sp.base + ch[i].f * sp.plane_bytes + ch[i].r0 * sp.dpitch,
                                      sp.dpitch, sp.my * sp.es, ch[i].nr, cudaMemcpyDeviceToHost, stream);
    return x != cudaSuccess ? x : cudaEventRecord(pr.ev[k], stream);
  };
  if (!ch.empty() && (e = fetch(0)) != cudaSuccess) return e;
  for (size_t i = 0; i < ch.size(); i++) {
    const int k = (int)(i & 1);
    /* the other buffer was emptied by the previous iteration */
    if (i + 1 < ch.size() && (e = fetch(i + 1)) != cudaSuccess) return e;
    if ((e = cudaEventSynchronize(pr.ev[k])) != cudaSuccess) return e;
    double *dst = host[ch[i].f] + ch[i].r0 * sp.my;
    const size_t n = ch[i].nr * sp.my;
    if (sp.es == 8) {
      const char *src = (const char *)pr.buf[k];
      host_parallel(n * 8, grain, [&](size_t lo, size_t hi) { memcpy((char *)dst + lo, src + lo, hi - lo); });
    } else {
      const float *src = (const float *)pr.buf[k];
      host_parallel(n, grain / 4, [&](size_t lo, size_t hi) {
        for (size_t j = lo; j < hi; j++) dst[j] = (double)src[j];
      });
    }
  }
  return cudaSuccess;
}

/* host <-> state of one simulation (kind: H2D, D2H, D2D).  Host buffers move
 * through the batch's two pinned staging buffers in chunks of rows: the DMA
 * of one chunk overlaps the host copy (FP64) or conversion (FP32) of the
 * other.  FP32 exchanges host buffers only. */
static int batch_copy(gp_batch *b, int s, const double *phi, const double *mu, double *ophi, double *omu,
                      cudaMemcpyKind kind) {
  const gpd::SimDesc &sd = b->desc[s];
  const int N = b->N, K = b->K;
  const size_t mx = sd.g.mx, my = sd.g.my, es = b->elem, dpitch = (size_t)sd.g.pitch * es;
  char *base = (char *)b->state[b->cur] + (size_t)sd.off_state * es;
  const bool up = phi != nullptr;
  if (kind == cudaMemcpyDeviceToDevice) {
    for (int f = 0; f < N + K; f++) {
      char *plane = base + (size_t)f * sd.g.plane * es;
      if (up) {
        const double *src = f < N ? phi + (size_t)f * mx * my : mu + (size_t)(f - N) * mx * my;
        BK(cudaMemcpy2DAsync(plane, dpitch, src, my * 8, my * 8, mx, kind, b->stream));
      } else {
        double *dst = f < N ? ophi + (size_t)f * mx * my : omu + (size_t)(f - N) * mx * my;
        BK(cudaMemcpy2DAsync(dst, my * 8, plane, dpitch, my * 8, mx, kind, b->stream));
      }
    }
    BK(cudaStreamSynchronize(b->stream));
    return GP_OK;
  }
  double *hp[GP_MAX_PHASES + GP_MAX_COMP];
  for (int f = 0; f < N + K; f++)
    hp[f] = up ? (double *)(f < N ? phi + (size_t)f * mx * my : mu + (size_t)(f - N) * mx * my)
               : (f < N ? ophi + (size_t)f * mx * my : omu + (size_t)(f - N) * mx * my);
  const StagedPlanes sp = {b->dev, base, (size_t)sd.g.plane * es, dpitch, mx, my, es, N + K};
  const cudaError_t e = up ? stage_up(sp, hp, b->stream) : stage_down(sp, hp, b->stream);
  if (e != cudaSuccess) return bfail(b, GP_ECUDA, "state copy: %s", cudaGetErrorString(e));
  BK(cudaStreamSynchronize(b->stream));
  return GP_OK;
}

static_assert(sizeof(CUtensorMap) == sizeof(gpd::TensorMapSlot), "tensor map size");

/* cuTensorMapEncodeTiled through the runtime's driver entry point (no link
 * against libcuda) */
static PFN_cuTensorMapEncodeTiled_v12000 encode_tiled_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

/* The TMA maps of kf_bulk: per simulation and state buffer, the K mu planes
 * as a 3-D tensor {pitch, mx, K} (strides one row, one plane) read in boxes
 * of {BW, SH, K}; coordinates outside the tensor read zeros. */
/* The tensor map of simulation s's K mu planes in a state buffer whose
 * simulation-s planes start at `state` (the bulk tiles' TMA boxes). */
static int encode_mu_map(gp_batch *b, int s, void *state, gpd::TensorMapSlot *out) {
  PFN_cuTensorMapEncodeTiled_v12000 fn = encode_tiled_fn();
  if (!fn) return bfail(b, GP_ECUDA, "cuTensorMapEncodeTiled is not available");
  const bool f64 = b->elem == 8;
  const cuuint32_t bw = f64 ? gpd::BulkGeom<double, 1>::BW : gpd::BulkGeom<float, 1>::BW;
  const gpd::SimDesc &sd = b->desc[s];
  void *base = (char *)state + (size_t)((long long)b->N * sd.g.plane) * b->elem;
  const cuuint64_t dims[3] = {(cuuint64_t)sd.g.pitch, (cuuint64_t)sd.g.mx, (cuuint64_t)b->K};
  const cuuint64_t strides[2] = {(cuuint64_t)sd.g.pitch * b->elem, (cuuint64_t)sd.g.plane * b->elem};
  const cuuint32_t box[3] = {bw, (cuuint32_t)gpd::SH, (cuuint32_t)b->K};
  const cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn((CUtensorMap *)out, f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                  base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return bfail(b, GP_ECUDA, "cuTensorMapEncodeTiled failed (%d) for simulation %d", (int)r, s);
  return GP_OK;
}

static int encode_mu_maps(gp_batch *b, gpd::TensorMapSlot *out) {
  for (int s = 0; s < b->nsims; s++)
    for (int p = 0; p < 2; p++) {
      const int rc = encode_mu_map(b, s, (char *)b->state[p] + (size_t)b->desc[s].off_state * b->elem, &out[2 * s + p]);
      if (rc != GP_OK) return rc;
    }
  return GP_OK;
}

/* Gather (pack) or scatter rows of the current state, one CTA per row. */
template <typename T>
__global__ void k_rows_copy(T *__restrict__ state, long long plane, int pitch, int my, gpd::RowItems it,
                            T *__restrict__ buf, int pack) {
  const int i = blockIdx.x;
  T *r = state + (long long)it.field[i] * plane + (long long)it.row[i] * pitch;
  T *q = buf + (long long)i * my;
  if (pack)
    for (int y = threadIdx.x; y < my; y += blockDim.x) q[y] = r[y];
  else
    for (int y = threadIdx.x; y < my; y += blockDim.x) r[y] = q[y];
}

static int rows_copy(gp_ctx *c, const char *who, int n, const int *fields, const int *rows, void *buf, int pack) {
  if (!c || !fields || !rows || !buf) return fail(c, GP_EINVAL, "%s: NULL argument", who);
  gp_batch *b = c->b;
  const gpd::SimDesc &sd = b->desc[0];
  if (n < 1 || n > gpd::ROW_ITEMS_MAX) return fail(c, GP_EINVAL, "%s: %d rows (1..%d)", who, n, gpd::ROW_ITEMS_MAX);
  gpd::RowItems it;
  for (int i = 0; i < n; i++) {
    if (fields[i] < 0 || fields[i] >= b->N + b->K || rows[i] < 0 || rows[i] >= sd.g.mx)
      return fail(c, GP_EINVAL, "%s: item %d (field %d, row %d) outside the state", who, i, fields[i], rows[i]);
    it.field[i] = fields[i];
    it.row[i] = rows[i];
  }
  c->err[0] = 0;
  CK(cudaSetDevice(b->dev));
  char *base = (char *)b->state[b->cur] + (size_t)sd.off_state * b->elem;
  if (b->elem == 8)
    k_rows_copy<double><<<n, 256, 0, b->stream>>>((double *)base, sd.g.plane, sd.g.pitch, sd.g.my, it, (double *)buf,
                                                   pack);
  else
    k_rows_copy<float><<<n, 256, 0, b->stream>>>((float *)base, sd.g.plane, sd.g.pitch, sd.g.my, it, (float *)buf,
                                                  pack);
  CK(cudaGetLastError());
  if (!pack) {
    const int rc = batch_reflag(b, false);   /* the tiles' phase flags follow the new rows */
    if (rc != GP_OK) return rc;
  }
  return GP_OK;
}

extern "C" {

void gp_batch_destroy(gp_batch *b) {
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  batch_drop_graphs(b);
  for (int p = 0; p < 2; p++) cudaFree(b->state[p]);
  for (int i = 0; i < 4; i++)
    if (b->ev[i]) cudaEventDestroy(b->ev[i]);
  cudaFree(b->flags[0]);   /* flags[1] is part of the same allocation */
  cudaFree(b->glist);
  cudaFree(b->blist);
  cudaFree(b->d_desc);
  cudaFree(b->d_consts);
  cudaFree(b->d_tsim);
  cudaFree(b->d_seg0);
  cudaFree(b->d_segn);
  cudaFree(b->ext);
  cudaFree(b->partials);
  cudaFree(b->sums_sim);
  cudaFree(b->counters);
  cudaFree(b->tmaps);
  cudaFree(b->trows);
  cudaFree(b->dyn);
  cudaFree(b->spos);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

const char *gp_batch_last_error(const gp_batch *b) { return b ? b->err : gp_host_thread_error(); }

int gp_batch_create(gp_batch **out, int nsims, const gp_params *params, const double *const *phi,
                    const double *const *mu, gp_precision prec) {
  gp_batch *b = nullptr;
  if (!out || nsims < 1 || !params || !phi || !mu) return bfail(nullptr, GP_EINVAL, "gp_batch_create: bad argument");
  *out = nullptr;
  if (prec != GP_FP64 && prec != GP_FP32) return bfail(nullptr, GP_EINVAL, "gp_batch_create: precision");
  b = new gp_batch();
  b->nsims = nsims;
  b->prec = prec;
  b->params.assign(params, params + nsims);
  b->derived.resize(nsims);
  b->last.resize(nsims);
  for (int s = 0; s < nsims; s++) {
    char err[256] = "";
    if (gp_host_derive(&params[s], &b->derived[s], err, sizeof err) != GP_OK) {
      int r = bfail(nullptr, GP_EINVAL, "gp_batch_create: simulation %d: %s", s, err);
      delete b;
      return r;
    }
    const gp_derived &d = b->derived[s];
    if (s == 0) { b->N = d.N; b->K = d.K; b->aniso = d.aniso; }
    else if (d.N != b->N || d.K != b->K || d.aniso != b->aniso) {
      delete b;
      return bfail(nullptr, GP_EINVAL, "gp_batch_create: simulation %d differs in NUMPHASES, NUMCOMPONENTS or "
                                       "Function_anisotropy from simulation 0", s);
    }
  }
  bool ok = prec == GP_FP64 ? gp_batch_launch_f64(b->N, b->K, b->aniso != 0, &b->L)
                            : gp_batch_launch_f32(b->N, b->K, b->aniso != 0, &b->L);
  if (!ok) {
    delete b;
    return bfail(nullptr, GP_EINVAL, "gp_batch_create: no kernel for N=%d K=%d", b->N, b->K);
  }
  b->elem = b->L.elem;
  int rc = GP_OK;
  cudaError_t e = cudaGetDevice(&b->dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, b->dev);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  for (int i = 0; i < 4 && e == cudaSuccess; i++) e = cudaEventCreate(&b->ev[i]);
  if (e != cudaSuccess) {
    rc = bfail(b, GP_ECUDA, "gp_batch_create: %s", cudaGetErrorString(e));
    gp_batch_destroy(b);
    return rc;
  }
  /* layout: every simulation's N+K planes back to back, pitch a multiple of 32 */
  const int N = b->N, K = b->K, ne = 2 * (N + K), ns = 2 * N + 2 * K + 1;
  long long off = 0;
  int nt = 0, offT = 0;
  std::vector<int> tsim, seg0, segn;
  std::vector<char> consts;
  const size_t csz = b->elem == 8 ? sizeof(gpd::Consts<double>) : sizeof(gpd::Consts<float>);
  b->consts_bytes = csz;
  consts.resize(csz * nsims);
  for (int s = 0; s < nsims; s++) {
    const gp_derived &d = b->derived[s];
    gpd::SimDesc sd;
    memset(&sd, 0, sizeof sd);
    sd.g = make_grid(d, 32);
    sd.off_state = off;
    sd.tiles_x = (sd.g.my + gpd::TY - 1) / gpd::TY;
    const int tiles_y = (sd.g.mx + gpd::TX - 1) / gpd::TX;
    sd.tile0 = nt;
    sd.off_T = offT;
    offT += 2 * (int)(sd.g.my + 6);
    seg0.push_back(nt);
    segn.push_back(sd.tiles_x * tiles_y);
    for (int t = 0; t < sd.tiles_x * tiles_y; t++) tsim.push_back(s);
    nt += sd.tiles_x * tiles_y;
    off += (long long)(N + K) * sd.g.plane;
    b->desc.push_back(sd);
    if (b->elem == 8) {
      gpd::Consts<double> c = make_consts<double>(d);
      memcpy(&consts[csz * s], &c, csz);
    } else {
      gpd::Consts<float> c = make_consts<float>(d);
      memcpy(&consts[csz * s], &c, csz);
    }
  }
  b->ntiles = nt;
  for (int s = 0; s < nsims; s++) {
    /* kf_bulk packs a tile's row and column into 15 and 16 bits */
    const gpd::SimDesc &sd = b->desc[s];
    if ((sd.g.mx + gpd::TX - 1) / gpd::TX >= (1 << 15) || sd.tiles_x >= (1 << 16)) {
      rc = bfail(b, GP_EINVAL, "gp_batch_create: simulation %d: grid %dx%d has more than 2^15 tile rows or 2^16 tile "
                               "columns", s, sd.g.mx, sd.g.my);
      gp_batch_destroy(b);
      return rc;
    }
  }
  if (nt >= (1 << 28)) {
    rc = bfail(b, GP_EINVAL, "gp_batch_create: %d tiles of %dx%d cells, at most 2^28", nt, gpd::TX, gpd::TY);
    gp_batch_destroy(b);
    return rc;
  }
  b->mul = true;
  for (int s = 0; s < nsims; s++)
    if (b->elem == 8 && !(pow2(b->derived[s].dx) && pow2(b->derived[s].dy))) b->mul = false;
  b->diag = true;
  for (int s = 0; s < nsims; s++) {
    const gp_derived &d = b->derived[s];
    for (int a = 0; a < N; a++)
      for (int k = 0; k < K; k++) {
        if (d.E[a][k] == 0.0 && std::signbit(d.E[a][k])) b->diag = false;   /* E = -0 */
        for (int l = 0; l < K; l++)
          if (k != l && (d.Dbulk[a][k][l] != 0.0 || d.cmu[a][k][l] != 0.0 || d.A[a][k][l] != 0.0)) b->diag = false;
      }
  }
  /* the give-up path of kf_bulk's barrier waits, exercised by a test: the
   * barriers expect more bytes than a box brings, and the polls are few */
  b->mbar_tries = gpd::MBAR_TRIES;
  b->tma_extra = 0;
  if (const char *v = getenv("GP_TEST_TMA_SHORTFALL")) {
    b->tma_extra = (unsigned)std::max(0, std::min(4096, atoi(v)));
    if (b->tma_extra) b->mbar_tries = 256;
  }
  int bpb = 1, bpg = 1;
  e = b->L.prepare(&bpb, &bpg);
  if (e != cudaSuccess) {
    rc = bfail(b, GP_ECUDA, "gp_batch_create: %s", cudaGetErrorString(e));
    gp_batch_destroy(b);
    return rc;
  }
  b->grid_b = std::min(nt, b->nsm * std::max(1, bpb));
  b->grid_g = b->nsm * std::max(1, bpg);
  /* the single-launch step when it keeps the bulk kernel's occupancy */
  {
    const int bps = b->L.step_occupancy();
    b->grid_s = (bps >= bpb && getenv("GP_SPLIT_KERNELS") == nullptr) ? b->nsm * bps : 0;
  }
  /* launch shapes: the first graph chunks of the first batch of its kind time
   * each candidate; later batches of that kind take its choice (GP_NO_TUNING:
   * the first candidate, untimed) */
  {
    int lg = 0;
    while ((1 << lg) < nt) lg++;
    b->key = ShapeKey{N, K, b->aniso, (int)b->elem, lg};
    const LaunchShape fused16 = {true, 16, 2, false}, fused8 = {true, 8, 2, false}, mixed16 = {true, 16, 2, true},
                      mixed8 = {true, 8, 2, true}, two = {false, 16, 2, false};
    b->ncand = 0;
    if (b->grid_s > 0) {
      b->cand[b->ncand++] = fused16;
      b->cand[b->ncand++] = fused8;
      b->cand[b->ncand++] = mixed16;
      b->cand[b->ncand++] = mixed8;
    }
    b->cand[b->ncand++] = two;
    b->shape = b->cand[0];
    b->tune_next = b->ncand;   /* nothing to tune */
    if (getenv("GP_NO_TUNING") == nullptr) {
      std::lock_guard<std::mutex> lock(g_shapes_mutex);
      auto it = g_shapes.find(b->key);
      if (it != g_shapes.end()) b->shape = it->second;
      else if (b->ncand > 1) b->tune_next = 0;
    }
  }
#define BALLOC(ptr, bytes)                                                                        \
  do {                                                                                            \
    if (cudaMalloc((void **)&(ptr), (bytes)) != cudaSuccess) {                                     \
      rc = bfail(b, GP_ENOMEM, "gp_batch_create: cudaMalloc of %zu bytes failed", (size_t)(bytes)); \
      gp_batch_destroy(b);                                                                        \
      return rc;                                                                                  \
    }                                                                                             \
  } while (0)
  BALLOC(b->state[0], (size_t)off * b->elem);
  BALLOC(b->state[1], (size_t)off * b->elem);
  BALLOC(b->flags[0], 2 * sizeof(gpd::TileFlags) * (size_t)nt);
  b->flags[1] = b->flags[0] + nt;
  BALLOC(b->glist, sizeof(int) * (size_t)nt);
  BALLOC(b->blist, sizeof(int4) * (size_t)nt);
  BALLOC(b->d_desc, sizeof(gpd::SimDesc) * nsims);
  BALLOC(b->d_consts, csz * nsims);
  BALLOC(b->d_tsim, sizeof(int) * (size_t)nt);
  BALLOC(b->d_seg0, sizeof(int) * nsims);
  BALLOC(b->d_segn, sizeof(int) * nsims);
  BALLOC(b->ext, sizeof(long long) * (size_t)ne * nsims);
  BALLOC(b->partials, sizeof(double) * (size_t)ns * nt);
  BALLOC(b->sums_sim, sizeof(double) * (size_t)ns * nsims);
  BALLOC(b->counters, gpd::CTR_COUNT * sizeof(int));
  BALLOC(b->tmaps, sizeof(gpd::TensorMapSlot) * 2 * (size_t)nsims);
  b->tgrad = false;
  b->shift = false;
  for (int s = 0; s < nsims; s++) {
    b->tgrad |= b->derived[s].tgrad != 0;
    b->shift |= b->derived[s].shift != 0;
  }
  BALLOC(b->spos, sizeof(int) * (size_t)nsims);
  if (b->shift) b->tune_next = b->ncand;   /* the first chunks end at the frame checks: no tuning */
  BALLOC(b->trows, sizeof(double) * (size_t)std::max(offT, 1));
  BALLOC(b->dyn, sizeof(gpd::SimDyn) * (size_t)nsims);
#undef BALLOC
  std::vector<gpd::TensorMapSlot> tm(2 * (size_t)nsims);
  if (encode_mu_maps(b, tm.data()) != GP_OK) {
    rc = GP_ECUDA;
    gp_batch_destroy(b);
    return rc;
  }
  std::vector<long long> ext((size_t)ne * nsims);
  for (int t = 0; t < nsims; t++) init_ext(&ext[(size_t)t * ne], N, K);
#define BUP(dst, src, bytes)                                                                       \
  do {                                                                                             \
    if (cudaMemcpyAsync((dst), (src), (bytes), cudaMemcpyHostToDevice, b->stream) != cudaSuccess) { \
      rc = bfail(b, GP_ECUDA, "gp_batch_create: upload failed");                                   \
      gp_batch_destroy(b);                                                                         \
      return rc;                                                                                   \
    }                                                                                              \
  } while (0)
  BUP(b->d_desc, b->desc.data(), sizeof(gpd::SimDesc) * nsims);
  BUP(b->d_consts, consts.data(), csz * nsims);
  BUP(b->d_tsim, tsim.data(), sizeof(int) * (size_t)nt);
  BUP(b->d_seg0, seg0.data(), sizeof(int) * nsims);
  BUP(b->d_segn, segn.data(), sizeof(int) * nsims);
  BUP(b->ext, ext.data(), sizeof(long long) * ext.size());
  BUP(b->tmaps, tm.data(), sizeof(gpd::TensorMapSlot) * tm.size());
#undef BUP
  if (cudaMemsetAsync(b->dyn, 0, sizeof(gpd::SimDyn) * (size_t)nsims, b->stream) != cudaSuccess ||
      cudaMemsetAsync(b->counters, 0, gpd::CTR_COUNT * sizeof(int), b->stream) != cudaSuccess) {
    rc = bfail(b, GP_ECUDA, "gp_batch_create: memset failed");
    gp_batch_destroy(b);
    return rc;
  }
  for (int s = 0; s < nsims; s++) {
    if ((rc = batch_copy(b, s, phi[s], mu[s], nullptr, nullptr, cudaMemcpyHostToDevice)) != GP_OK) {
      gp_batch_destroy(b);
      return rc;
    }
  }
  if ((rc = batch_reflag(b, true)) != GP_OK) {
    gp_batch_destroy(b);
    return rc;
  }
  *out = b;
  return GP_OK;
}

int gp_batch_smooth(gp_batch *b, long nsteps) {
  if (!b || nsteps < 0) return bfail(b, GP_EINVAL, "gp_batch_smooth: bad argument");
  const size_t csz = b->consts_bytes;
  /* the sweeps run before the first step: the temperature as copied at t = 0 */
  if (b->tgrad && nsteps > 0)
    BK(b->L.trows(b->nsims, b->stream, b->d_desc, b->d_consts, b->counters, b->dyn, b->trows));
  for (long t = 0; t < nsteps; t++) {
    for (int s = 0; s < b->nsims; s++) {
      const gpd::SimDesc &sd = b->desc[s];
      const char *cs = (const char *)b->d_consts + csz * s;
      const char *st = (const char *)b->state[b->cur] + (size_t)sd.off_state * b->elem;
      char *nx = (char *)b->state[b->cur ^ 1] + (size_t)sd.off_state * b->elem;
      const size_t mu_off = (size_t)b->N * sd.g.plane * b->elem;
      const double *tcc = b->derived[s].tgrad ? b->trows + sd.off_T + (sd.g.my + 6) : nullptr;
      BK(b->L.smooth(b->stream, cs, st, st + mu_off, nx, nx + mu_off, sd.g, tcc));
    }
    b->cur ^= 1;
  }
  if (nsteps > 0) {
    int rc = batch_reflag(b, true);
    if (rc != GP_OK) return rc;
  }
  BK(cudaStreamSynchronize(b->stream));
  return GP_OK;
}

int gp_batch_step(gp_batch *b, long nsteps, gp_stats *stats) {
  if (!b || nsteps < 0) return bfail(b, GP_EINVAL, "gp_batch_step: bad argument");
  return batch_step_impl(b, nsteps, stats, nullptr, nullptr, nullptr);
}

int gp_batch_step_timed(gp_batch *b, long nsteps, gp_stats *stats, double *total_ms) {
  if (!b || nsteps < 0) return bfail(b, GP_EINVAL, "gp_batch_step_timed: bad argument");
  return batch_step_impl(b, nsteps, stats, total_ms, nullptr, nullptr);
}

int gp_batch_get(gp_batch *b, int sim, double *phi, double *mu) {
  if (!b || sim < 0 || sim >= b->nsims || !phi || !mu) return bfail(b, GP_EINVAL, "gp_batch_get: bad argument");
  return batch_copy(b, sim, nullptr, nullptr, phi, mu, cudaMemcpyDeviceToHost);
}

int gp_batch_set(gp_batch *b, int sim, const double *phi, const double *mu) {
  if (!b || sim < 0 || sim >= b->nsims || !phi || !mu) return bfail(b, GP_EINVAL, "gp_batch_set: bad argument");
  int rc = batch_copy(b, sim, phi, mu, nullptr, nullptr, cudaMemcpyHostToDevice);
  if (rc != GP_OK) return rc;
  /* the other buffer still holds what its flags say */
  rc = batch_reflag(b, false);
  if (rc != GP_OK) return rc;
  BK(cudaStreamSynchronize(b->stream));
  return GP_OK;
}

int gp_batch_size(const gp_batch *b) { return b ? b->nsims : 0; }

/* ======================================================================= */
/* single-simulation API: a batch of one                                   */
/* ======================================================================= */

const char *gp_version(void) { return "libgp 0.3 (sm_100a; bulk/interface tile engine, FP64 and FP32)"; }

size_t gp_params_size(void) { return sizeof(gp_params); }

const char *gp_last_error(const gp_ctx *ctx) {
  if (!ctx) return gp_host_thread_error();
  if (ctx->err[0]) return ctx->err;
  return ctx->b ? ctx->b->err : "";
}

void *gp_stream(gp_ctx *ctx) { return ctx && ctx->b ? (void *)ctx->b->stream : nullptr; }

void gp_destroy(gp_ctx *c) {
  if (!c) return;
  gp_vtk_wait(c);
  cudaFree(c->snap);
  if (c->wstream) cudaStreamDestroy(c->wstream);
  if (c->wready) cudaEventDestroy(c->wready);
  free(c->hphi);
  free(c->hmu);
  free(c->htemp);
  gp_batch_destroy(c->b);
  free(c);
}

/* The temperature field [mx][my] of simulation 0 after `steps` steps with the
 * frame state `dd`: the field laid down after the last step (with shift_OFFSET
 * as it was then) and moved with the frame when the frame moved at that step,
 * as kt_rows lays it for the next step's phase-field pass. */
static void temperature_field(const gp_batch *b, long long steps, const gpd::SimDyn &dd, double *T) {
  const gp_derived &d = b->derived[0];
  const size_t mx = (size_t)d.mx, my = (size_t)d.my;
  if (!d.tgrad) {
    for (size_t i = 0; i < mx * my; i++) T[i] = b->params[0].T;
    return;
  }
  gp_host_temperature_column(&d, steps, dd.fresh ? dd.shift_T : dd.shift_off, dd.fresh ? dd.dlast : 0, T);
  for (size_t x = 1; x < mx; x++) memcpy(T + x * my, T, sizeof(double) * my);
}

/* Bytes of the state planes of simulation 0 in a snapshot (16-byte multiple:
 * the frame state follows them). */
static size_t snap_state_bytes(const gp_batch *b) {
  const size_t n = (size_t)(b->N + b->K) * b->desc[0].g.plane * b->elem;
  return (n + 15) & ~(size_t)15;
}

/* The writer thread of gp_vtk_write_async: wait for the snapshot, bring it
 * down through the staging buffers on the writer's own stream (the context's
 * stream keeps stepping), write the file. */
static void vtk_writer(gp_ctx *c, std::string path, int ascii) {
  gp_batch *b = c->b;
  const gpd::SimDesc &sd = b->desc[0];
  const int N = b->N, K = b->K;
  const size_t mx = sd.g.mx, my = sd.g.my, es = b->elem;
  int rc = GP_OK;
  cudaError_t e = cudaSetDevice(b->dev);
  if (e == cudaSuccess) e = cudaEventSynchronize(c->wready);
  if (e == cudaSuccess) {
    double *hp[GP_MAX_PHASES + GP_MAX_COMP];
    for (int f = 0; f < N + K; f++) hp[f] = f < N ? c->hphi + (size_t)f * mx * my : c->hmu + (size_t)(f - N) * mx * my;
    const StagedPlanes sp = {b->dev, (char *)c->snap, (size_t)sd.g.plane * es, (size_t)sd.g.pitch * es, mx, my, es,
                             N + K};
    e = stage_down(sp, hp, c->wstream);
  }
  if (e != cudaSuccess) {
    snprintf(c->werr, sizeof c->werr, "gp_vtk_write_async: %s", cudaGetErrorString(e));
    rc = GP_ECUDA;
  } else if (b->derived[0].tgrad) {
    gpd::SimDyn dd;
    e = cudaMemcpyAsync(&dd, (char *)c->snap + snap_state_bytes(b), sizeof dd, cudaMemcpyDeviceToHost, c->wstream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->wstream);
    if (e != cudaSuccess) {
      snprintf(c->werr, sizeof c->werr, "gp_vtk_write_async: %s", cudaGetErrorString(e));
      rc = GP_ECUDA;
    } else {
      temperature_field(b, c->wsteps, dd, c->htemp);
      if ((rc = gp_vtk_write_temperature(&b->params[0], path.c_str(), c->hphi, c->hmu, c->htemp, ascii)) != GP_OK)
        snprintf(c->werr, sizeof c->werr, "%s", gp_host_thread_error());
    }
  } else if ((rc = gp_vtk_write(&b->params[0], path.c_str(), c->hphi, c->hmu, ascii)) != GP_OK) {
    snprintf(c->werr, sizeof c->werr, "%s", gp_host_thread_error());
  }
  c->wstatus = rc;
}

int gp_vtk_wait(gp_ctx *c) {
  if (!c) return fail(nullptr, GP_EINVAL, "gp_vtk_wait: NULL context");
  if (c->writer) {
    c->writer->join();
    delete c->writer;
    c->writer = nullptr;
  }
  const int rc = c->wstatus;
  c->wstatus = GP_OK;
  if (rc != GP_OK) return fail(c, rc, "%s", c->werr);
  return GP_OK;
}

int gp_vtk_write_async(gp_ctx *c, const char *path, int ascii) {
  if (!c || !path) return fail(c, GP_EINVAL, "gp_vtk_write_async: NULL argument");
  int rc = gp_vtk_wait(c);   /* one write in flight per context */
  if (rc != GP_OK) return rc;
  c->err[0] = 0;
  gp_batch *b = c->b;
  const gpd::SimDesc &sd = b->desc[0];
  const size_t bytes = snap_state_bytes(b);
  if (!c->snap) {
    const size_t cells = (size_t)sd.g.mx * sd.g.my;
    CK(cudaMalloc(&c->snap, bytes + sizeof(gpd::SimDyn)));
    CK(cudaStreamCreateWithFlags(&c->wstream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&c->wready, cudaEventDisableTiming));
    c->hphi = (double *)malloc(sizeof(double) * cells * b->N);
    c->hmu = (double *)malloc(sizeof(double) * cells * b->K);
    c->htemp = (double *)malloc(sizeof(double) * cells);
    if (!c->hphi || !c->hmu || !c->htemp) return fail(c, GP_ENOMEM, "gp_vtk_write_async: out of host memory");
  }
  /* the snapshot is ordered after the steps already queued; later steps
   * write the other state buffer or this one after the copy has read it.  The
   * frame state (which sets the temperature field) travels with it. */
  CK(cudaMemcpyAsync(c->snap, (char *)b->state[b->cur] + (size_t)sd.off_state * b->elem, bytes,
                     cudaMemcpyDeviceToDevice, b->stream));
  CK(cudaMemcpyAsync((char *)c->snap + bytes, b->dyn, sizeof(gpd::SimDyn), cudaMemcpyDeviceToDevice, b->stream));
  c->wsteps = b->steps;
  CK(cudaEventRecord(c->wready, b->stream));
  try {
    c->writer = new std::thread(vtk_writer, c, std::string(path), ascii);
  } catch (...) {
    return fail(c, GP_ENOMEM, "gp_vtk_write_async: cannot start the writer thread");
  }
  return GP_OK;
}

int gp_init(gp_ctx **out, const gp_params *p, const double *phi, const double *mu, gp_precision prec) {
  if (!out || !p || !phi || !mu) return fail(nullptr, GP_EINVAL, "gp_init: NULL argument");
  *out = nullptr;
  if (prec != GP_FP64 && prec != GP_FP32) return fail(nullptr, GP_EINVAL, "gp_init: unknown precision %d", (int)prec);
  gp_ctx *c = (gp_ctx *)calloc(1, sizeof(gp_ctx));
  if (!c) return fail(nullptr, GP_ENOMEM, "gp_init: out of host memory");
  const double *ph[1] = {phi}, *m[1] = {mu};
  int r = gp_batch_create(&c->b, 1, p, ph, m, prec);
  if (r != GP_OK) {
    free(c);
    return r;   /* the message is in the thread's error slot */
  }
  *out = c;
  return GP_OK;
}

int gp_smooth(gp_ctx *c, long nsteps) {
  if (!c || nsteps < 0) return fail(c, GP_EINVAL, "gp_smooth: bad argument");
  c->err[0] = 0;
  return gp_batch_smooth(c->b, nsteps);
}

int gp_step(gp_ctx *c, long nsteps, gp_stats *stats) {
  if (!c || nsteps < 0) return fail(c, GP_EINVAL, "gp_step: bad argument");
  c->err[0] = 0;
  return batch_step_impl(c->b, nsteps, stats, nullptr, nullptr, nullptr);
}

int gp_step_timed(gp_ctx *c, long nsteps, gp_stats *stats, double *total_ms, double *ms_bulk, double *ms_iface) {
  if (!c || nsteps < 0) return fail(c, GP_EINVAL, "gp_step_timed: bad argument");
  c->err[0] = 0;
  return batch_step_impl(c->b, nsteps, stats, total_ms, ms_bulk, ms_iface);
}

int gp_step_kernel_times(gp_ctx *c, long nsteps, gp_kernel_times *t) {
  if (!c || nsteps < 1 || !t) return fail(c, GP_EINVAL, "gp_step_kernel_times: bad argument");
  c->err[0] = 0;
  gp_batch *b = c->b;
  memset(t, 0, sizeof *t);
  const bool fused = b->grid_s > 0 && b->shape.fused;
  cudaEvent_t ev[4] = {b->ev[0], b->ev[1], b->ev[2], fused ? nullptr : b->ev[3]};
  for (long i = 0; i < nsteps; i++) {
    int rc = batch_step_once(b, 0, ev);
    if (rc != GP_OK) return rc;
    float x = 0.f, y = 0.f, z = 0.f;
    BK(cudaEventSynchronize(ev[2]));
    if (fused) {
      BK(cudaEventElapsedTime(&x, ev[0], ev[1]));
      BK(cudaEventElapsedTime(&y, ev[1], ev[2]));
      t->classify_ms += x;
      t->step_ms += y;
    } else {
      /* two-launch form: ev[0] classify+bulk ev[1] general ev[2] */
      BK(cudaEventElapsedTime(&z, ev[0], ev[1]));
      BK(cudaEventElapsedTime(&y, ev[1], ev[2]));
      t->bulk_ms += z;
      t->iface_ms += y;
    }
  }
  t->launches_per_step = fused ? 2 : 3;
  t->fused = fused ? 1 : 0;
  return batch_check_error(b);
}

int gp_get_stats(gp_ctx *c, gp_stats *s) {
  if (!c || !s) return fail(c, GP_EINVAL, "gp_get_stats: bad argument");
  *s = c->b->last[0];
  return GP_OK;
}

int gp_temperature(gp_ctx *c, double *T) {
  if (!c || !T) return fail(c, GP_EINVAL, "gp_temperature: NULL argument");
  gp_batch *b = c->b;
  gpd::SimDyn dd;
  CK(cudaSetDevice(b->dev));
  CK(cudaMemcpyAsync(&dd, b->dyn, sizeof dd, cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  temperature_field(b, b->steps, dd, T);
  return GP_OK;
}

int gp_get(gp_ctx *c, double *phi, double *mu) {
  if (!c || !phi || !mu) return fail(c, GP_EINVAL, "gp_get: NULL argument");
  c->err[0] = 0;
  return gp_batch_get(c->b, 0, phi, mu);
}

int gp_set(gp_ctx *c, const double *phi, const double *mu) {
  if (!c || !phi || !mu) return fail(c, GP_EINVAL, "gp_set: NULL argument");
  c->err[0] = 0;
  return gp_batch_set(c->b, 0, phi, mu);
}

int gp_get_dev(gp_ctx *c, double *phi, double *mu) {
  if (!c || !phi || !mu) return fail(c, GP_EINVAL, "gp_get_dev: NULL argument");
  if (c->b->elem != 8) return fail(c, GP_EUNSUPPORTED, "gp_get_dev: FP32 contexts exchange host buffers only");
  c->err[0] = 0;
  return batch_copy(c->b, 0, nullptr, nullptr, phi, mu, cudaMemcpyDeviceToDevice);
}

int gp_set_dev(gp_ctx *c, const double *phi, const double *mu) {
  if (!c || !phi || !mu) return fail(c, GP_EINVAL, "gp_set_dev: NULL argument");
  if (c->b->elem != 8) return fail(c, GP_EUNSUPPORTED, "gp_set_dev: FP32 contexts exchange host buffers only");
  c->err[0] = 0;
  gp_batch *b = c->b;
  int rc = batch_copy(b, 0, phi, mu, nullptr, nullptr, cudaMemcpyDeviceToDevice);
  if (rc != GP_OK) return rc;
  rc = batch_reflag(b, false);
  if (rc != GP_OK) return rc;
  BK(cudaStreamSynchronize(b->stream));
  return GP_OK;
}

int gp_set_stat_rows(gp_ctx *c, long x0, long x1) {
  if (!c) return fail(nullptr, GP_EINVAL, "gp_set_stat_rows: NULL context");
  gp_batch *b = c->b;
  gpd::SimDesc &sd = b->desc[0];
  if (x0 < 0 || x1 > sd.g.mx || x0 >= x1)
    return fail(c, GP_EINVAL, "gp_set_stat_rows: rows [%ld, %ld) outside [0, %d)", x0, x1, sd.g.mx);
  if (b->shift) return fail(c, GP_EUNSUPPORTED, "gp_set_stat_rows: the moving frame needs the whole grid");
  c->err[0] = 0;
  sd.g.sx0 = (int)x0;
  sd.g.sx1 = (int)x1;
  CK(cudaSetDevice(b->dev));
  CK(cudaMemcpyAsync(b->d_desc, b->desc.data(), sizeof(gpd::SimDesc) * b->desc.size(), cudaMemcpyHostToDevice,
                     b->stream));
  CK(cudaStreamSynchronize(b->stream));
  return GP_OK;
}

int gp_rows_pack(gp_ctx *c, int n, const int *fields, const int *rows, void *dev_buf) {
  return rows_copy(c, "gp_rows_pack", n, fields, rows, dev_buf, 1);
}

int gp_rows_unpack(gp_ctx *c, int n, const int *fields, const int *rows, const void *dev_buf) {
  return rows_copy(c, "gp_rows_unpack", n, fields, rows, const_cast<void *>(dev_buf), 0);
}

}  /* extern "C" */


/* ======================================================================= */
/* adjoint                                                                 */
/* ======================================================================= */

namespace {

/* host planes [nf][mx][my] <-> device planes with the state layout */
int planes_copy(gp_batch *b, double *dst, size_t dpitch, const double *src, size_t spitch, int nf, size_t dplane,
                size_t splane, size_t mx, size_t my, cudaMemcpyKind kind) {
  for (int f = 0; f < nf; f++)
    BK(cudaMemcpy2DAsync(dst + f * dplane, dpitch * 8, src + f * splane, spitch * 8, my * 8, mx, kind, b->stream));
  return GP_OK;
}

/* Whatever enqueue() puts on the batch's stream, captured as one executable
 * CUDA graph (nothing runs): long runs of short launches whose arguments
 * change from one launch to the next get the launch gaps of a graph. */
template <typename F>
static int capture_graph(gp_batch *b, F &&enqueue, cudaGraphExec_t *out) {
  *out = nullptr;
  cudaGraph_t gr = nullptr;
  BK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  const int rc = enqueue();
  const cudaError_t ec = cudaStreamEndCapture(b->stream, &gr);
  if (rc != GP_OK || ec != cudaSuccess) {
    if (gr) cudaGraphDestroy(gr);
    return rc != GP_OK ? rc : bfail(b, GP_ECUDA, "graph capture: %s", cudaGetErrorString(ec));
  }
  const cudaError_t ei = cudaGraphInstantiate(out, gr, 0);
  cudaGraphDestroy(gr);
  if (ei != cudaSuccess) {
    *out = nullptr;
    return bfail(b, GP_ECUDA, "graph instantiate: %s", cudaGetErrorString(ei));
  }
  return GP_OK;
}

/* Launch an executable graph once; *ge is freed when that launch completes
 * and set to NULL. */
static int launch_once(gp_batch *b, cudaGraphExec_t *ge) {
  const cudaError_t e = cudaGraphLaunch(*ge, b->stream);
  cudaGraphExecDestroy(*ge);
  *ge = nullptr;
  if (e != cudaSuccess) return bfail(b, GP_ECUDA, "graph launch: %s", cudaGetErrorString(e));
  return GP_OK;
}

struct AdjBufs {
  double *snap = nullptr, *seg = nullptr, *ybar = nullptr, *xbar = nullptr, *dphi = nullptr, *dphibar = nullptr,
         *pbar = nullptr, *final_state = nullptr;
  double *rblk = nullptr;   /* two reverse blocks: adjoint of a state, adjoint of its delta-phi, list counters */
  double *dtape = nullptr;  /* delta-phi of every step, written by the forward pass (whole-tape mode) */
  gpd::TensorMapSlot *smaps = nullptr;   /* whole-tape mode: the tensor map of each slot's mu planes */
  int2 *cells = nullptr;    /* cells of a reverse pass that take the dual passes */
  int *ncells = nullptr;
  gpd::TileFlags *unknown = nullptr;   /* whole-tape mode: "unknown" flags of every tile (redir_have) */
  cudaGraphExec_t first[2] = {nullptr, nullptr};   /* whole-tape mode: the first graph of each sweep */
  ~AdjBufs() {   /* ybar, xbar and dphibar point into rblk */
    for (cudaGraphExec_t ge : first)
      if (ge) cudaGraphExecDestroy(ge);
    cudaFree(snap); cudaFree(seg); cudaFree(dphi); cudaFree(pbar); cudaFree(final_state); cudaFree(rblk);
    cudaFree(dtape); cudaFree(smaps); cudaFree(cells); cudaFree(ncells); cudaFree(unknown);
  }
};

int adj_check(gp_ctx *c, gpd::AdjLaunch *L) {
  if (!c || !c->b) return fail(c, GP_EINVAL, "gp_adjoint: NULL context");
  gp_batch *b = c->b;
  const gp_derived &d = b->derived[0];
  if (b->elem != 8) return fail(c, GP_EUNSUPPORTED, "gp_adjoint: FP64 contexts only");
  if (d.tgrad || d.shift)
    return fail(c, GP_EUNSUPPORTED, "gp_adjoint: isothermal runs without a moving frame only");
  if (d.N != 2 || d.K != 1 || d.inv_mode != GP_INV_BINARY)
    return fail(c, GP_EUNSUPPORTED, "gp_adjoint: NUMPHASES=2 with one BINARY component only (have N=%d K=%d)", d.N,
                d.K);
  if (!gp_adjoint_launch(d.N, d.K, d.aniso != 0, L)) return fail(c, GP_EUNSUPPORTED, "gp_adjoint: no kernels");
  return GP_OK;
}

/* Fewest forward steps that reverse l steps when the state at their start is
 * kept and s more states can be: with s+1 checkpoints, r the least repetition
 * number with C(s+1+r, r) >= l, the bound r*l - C(s+1+r, r-1) of binomial
 * checkpointing (Griewank, "Achieving logarithmic growth of temporal and
 * spatial complexity in reverse automatic differentiation", 1992). */
long adj_rev_cost(long l, long s) {
  if (l <= 1) return 0;
  if (s <= 0) return l * (l - 1) / 2;
  const long long S1 = s + 1;
  long long r = 0, b = 1;   /* b = C(S1 + r, r) */
  while (b < l) {
    r++;
    b = b * (S1 + r) / r;
  }
  return (long)(r * l - b * r / (S1 + 1));
}

gpd::AdjParams adj_params(const gp_params &p) {
  gpd::AdjParams a;
  a.v[gpd::ADJ_TAU] = p.tau_ab[0][1];
  a.v[gpd::ADJ_DAB] = p.dab[0][1];
  a.v[gpd::ADJ_EPS] = p.epsilon;
  a.v[gpd::ADJ_GAMMA] = p.gamma[0][1];
  return a;
}

}  // namespace

extern "C" {

int gp_adjoint(gp_ctx *c, const gp_adj_req *req, gp_adj_out *out) {
  gpd::AdjLaunch L;
  int rc = adj_check(c, &L);
  if (rc) return rc;
  if (!req || !out || req->nsteps < 1 || (!req->phi_bar && !req->target_phi))
    return fail(c, GP_EINVAL, "gp_adjoint: need nsteps >= 1 and phi_bar or target_phi");
  c->err[0] = 0;
  gp_batch *b = c->b;
  const gp_derived &d = b->derived[0];
  const gpd::SimDesc &sd = b->desc[0];
  const gpd::Grid &g = sd.g;
  const int N = d.N, K = d.K;
  const size_t mx = g.mx, my = g.my, S = (size_t)(N + K) * g.plane, Sd = (size_t)N * g.dplane;
  const long T = req->nsteps;
  const bool dev = req->device != 0;
  const cudaMemcpyKind h2d = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  const cudaMemcpyKind d2h = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  CK(cudaSetDevice(b->dev));

  /* snapshots of the state besides the start state: the caller's number, or
   * one state every checkpoint_every steps, or as many as half the free
   * device memory holds (every state, when they fit: no step is recomputed).
   * With every state kept, the forward pass also keeps each step's delta-phi
   * when that fits as well, and the reverse sweep does not recompute it. */
  long nsnap;
  size_t fre = 0, tot = 0;
  CK(cudaMemGetInfo(&fre, &tot));
  if (req->snapshots > 0) nsnap = req->snapshots;
  else if (req->checkpoint_every > 0) nsnap = (T + req->checkpoint_every - 1) / req->checkpoint_every;
  else nsnap = (long)std::min<size_t>((size_t)T, fre / 2 / (S * 8));
  nsnap = std::max(0L, std::min(nsnap, T - 1));
  const bool dtape = nsnap == T - 1 && (size_t)T * (S + Sd) * 8 <= fre / 2;
  const gpd::AdjParams prm = adj_params(b->params[0]);
  const void *consts = b->d_consts;
  AdjBufs m;
#define AALLOC(ptr, n)                                                                                  \
  do {                                                                                                  \
    if (cudaMalloc((void **)&(ptr), (n) * sizeof(double)) != cudaSuccess)                               \
      return fail(c, GP_ENOMEM, "gp_adjoint: cudaMalloc of %zu bytes failed", (size_t)(n) * sizeof(double)); \
  } while (0)
  /* a reverse block: the adjoint of a state (S), of its delta-phi (Sd) and
   * the two list counters of the reverse passes; a reverse step reads one
   * block and clears and fills the other with one memset */
  const size_t RB = S + Sd + 8;
  AALLOC(m.snap, S * (size_t)(nsnap + 1));   /* slot 0: the start state */
  AALLOC(m.seg, S);                          /* the state before the last step */
  AALLOC(m.rblk, 2 * RB);
  AALLOC(m.dphi, Sd);
  AALLOC(m.pbar, gpd::ADJ_NPARAM);
  AALLOC(m.final_state, S);
  if (dtape) AALLOC(m.dtape, Sd * (size_t)T);
#undef AALLOC
  if (dtape) {
    std::vector<gpd::TensorMapSlot> hm((size_t)T);
    for (long t = 0; t < T; t++)
      if ((rc = encode_mu_map(b, 0, m.snap + S * (size_t)t, &hm[(size_t)t])) != GP_OK) return fail(c, rc, "%s", b->err);
    if (cudaMalloc((void **)&m.smaps, sizeof(gpd::TensorMapSlot) * (size_t)T) != cudaSuccess ||
        cudaMalloc((void **)&m.unknown, sizeof(gpd::TileFlags) * (size_t)b->ntiles) != cudaSuccess)
      return fail(c, GP_ENOMEM, "gp_adjoint: cudaMalloc of the slot maps failed");
    CK(cudaMemcpyAsync(m.smaps, hm.data(), sizeof(gpd::TensorMapSlot) * (size_t)T, cudaMemcpyHostToDevice, b->stream));
    CK(cudaMemsetAsync(m.unknown, 0xfe, sizeof(gpd::TileFlags) * (size_t)b->ntiles, b->stream));
    /* the interface tiles write the delta-phi of their cells and rings; every
     * other cell of every step keeps this +0.0 */
    CK(cudaMemsetAsync(m.dtape, 0, Sd * (size_t)T * 8, b->stream));
    CK(cudaStreamSynchronize(b->stream));
  }
  int rcur = 0;   /* the block holding the adjoint of the state after the step being reversed */
  auto rbar = [&](int k) { return m.rblk + RB * (size_t)k; };
  m.ybar = rbar(0);
  std::vector<char> have_dphi((size_t)T, 0);
  {
    const size_t ncell = (size_t)(g.mx + 2) * (g.my + 2);
    if (cudaMalloc((void **)&m.cells, ncell * sizeof(int2)) != cudaSuccess ||
        cudaMalloc((void **)&m.ncells, sizeof(int)) != cudaSuccess)
      return fail(c, GP_ENOMEM, "gp_adjoint: cudaMalloc of the cell list failed");
  }
  const long long steps0 = b->steps;
  /* the three timing events, destroyed on every return */
  struct Events {
    cudaEvent_t e[3] = {nullptr, nullptr, nullptr};
    ~Events() {
      for (cudaEvent_t x : e)
        if (x) cudaEventDestroy(x);
    }
  } ev;
  for (cudaEvent_t &x : ev.e) CK(cudaEventCreate(&x));
  cudaEvent_t e0 = ev.e[0], e1 = ev.e[1], e2 = ev.e[2];
  out->loss = 0.0;

  /* ---- the steps are reversed by the binomial checkpointing schedule:
   * reversing steps [a, a+l) with the state at a in a slot and s free slots
   * advances m steps from a, keeps that state, reverses [a+m, a+l) with s-1
   * slots and then [a, a+m) with s; m minimises the recomputed steps (the
   * cost is convex in m).  The first chain of advances is the forward pass:
   * when it reaches the last step's start state, one more step gives the
   * final state and the seed of the reverse sweep.  With every state kept
   * (nsnap = T - 1) nothing is recomputed. */
  struct Task {
    long a, l, s;
    int slot;   /* the state a, or the slot to release (l = 0) */
  };
  std::vector<Task> stack;
  std::vector<int> free_slots;
  for (int i = (int)nsnap; i >= 1; i--) free_slots.push_back(i);
  stack.push_back({0, T, nsnap, 0});
  long work_t = 0;    /* the state the engine's buffer holds (-1: none of ours) */
  bool seeded = false;
  auto slot_ptr = [&](int k) { return m.snap + S * (size_t)k; };
  auto advance = [&](long k) -> int {
    for (long i = 0; i < k; i++) {
      const int r = batch_step_once(b, 0, nullptr);
      if (r != GP_OK) return r;
    }
    work_t += k;
    return GP_OK;
  };
  auto load = [&](long a, int slot) -> int {
    if (work_t == a) return GP_OK;
    BK(cudaMemcpyAsync(b->state[b->cur], slot_ptr(slot), S * 8, cudaMemcpyDeviceToDevice, b->stream));
    work_t = a;
    return batch_reflag(b, true);
  };
  /* the seed: dL/d(final state) from the state after the last step */
  auto seed = [&]() -> int {
    const double *fin = m.dtape ? m.final_state : (const double *)b->state[b->cur];
    if (fin != m.final_state) BK(cudaMemcpyAsync(m.final_state, fin, S * 8, cudaMemcpyDeviceToDevice, b->stream));
    BK(cudaEventRecord(e1, b->stream));
    BK(cudaMemsetAsync(m.ybar, 0, S * 8, b->stream));
    int r;
    if (req->phi_bar) {
      if ((r = planes_copy(b, m.ybar, g.pitch, req->phi_bar, my, N, g.plane, mx * my, mx, my, h2d)) != GP_OK)
        return r;
      if (req->mu_bar &&
          (r = planes_copy(b, m.ybar + N * g.plane, g.pitch, req->mu_bar, my, K, g.plane, mx * my, mx, my, h2d)) !=
              GP_OK)
        return r;
    } else {
      std::vector<double> phT((size_t)N * mx * my), tgt;
      if ((r = planes_copy(b, phT.data(), my, fin, g.pitch, N, mx * my, g.plane, mx, my, cudaMemcpyDeviceToHost)) !=
          GP_OK)
        return r;
      const double *target = req->target_phi;
      if (dev) {
        tgt.resize(phT.size());
        BK(cudaMemcpyAsync(tgt.data(), req->target_phi, tgt.size() * 8, cudaMemcpyDeviceToHost, b->stream));
        target = tgt.data();
      }
      BK(cudaStreamSynchronize(b->stream));
      double loss = 0.0;
      for (size_t i = 0; i < phT.size(); i++) {
        phT[i] -= target[i];
        loss += phT[i] * phT[i];
      }
      out->loss = 0.5 * loss;
      if ((r = planes_copy(b, m.ybar, g.pitch, phT.data(), my, N, g.plane, mx * my, mx, my,
                           cudaMemcpyHostToDevice)) != GP_OK)
        return r;
      BK(cudaStreamSynchronize(b->stream));   /* phT is released on return */
    }
    seeded = true;
    return GP_OK;
  };
  /* reverse of the step from state t held at x: ybar (after) -> ybar (before) */
  auto reverse = [&](long t, const double *x) -> int {
    const double *dph = m.dphi;
    if (m.dtape && have_dphi[(size_t)t]) dph = m.dtape + Sd * (size_t)t;
    else BK(L.dphi_sparse(b->stream, consts, prm, g, x, m.dphi, m.cells, m.ncells));
    double *ybar = rbar(rcur), *xbar = rbar(rcur ^ 1), *dphibar = xbar + S;
    int *cnt = (int *)(xbar + S + Sd);
    BK(cudaMemsetAsync(xbar, 0, RB * 8, b->stream));
    BK(L.rev_update(b->stream, consts, prm, g, x, dph, ybar, xbar, dphibar, m.pbar, m.cells, cnt));
    BK(L.rev_dphi(b->stream, consts, prm, g, x, dphibar, xbar, m.pbar, m.cells, cnt + 1));
    rcur ^= 1;
    m.ybar = xbar;
    return GP_OK;
  };
  /* reverse of the step from the state the engine's buffer holds (t); the
   * first such step is the last one (T - 1): the final state comes first */
  auto reverse_work = [&]() -> int {
    int r;
    const long t = work_t;
    if (!seeded) {
      BK(cudaMemcpyAsync(m.seg, b->state[b->cur], S * 8, cudaMemcpyDeviceToDevice, b->stream));
      if ((r = advance(1)) != GP_OK || (r = seed()) != GP_OK) return r;
      work_t = -1;
      return reverse(t, m.seg);
    }
    return reverse(t, (const double *)b->state[b->cur]);
  };
  /* whole tape: step t reads slot t and writes slot t+1 (the last one the
   * final state) directly, its bulk boxes through the slot's tensor map, and
   * leaves its delta-phi on the tape; then every step is reversed from its
   * slot, last first.  Both sweeps go to the GPU as graphs of GP_GRAPH_STEPS
   * steps, each captured once and launched once (the steps' arguments differ
   * from graph to graph): the host captures a graph while the GPU runs the
   * one before it, and the first graph of each sweep before the timed
   * region, as a plain run's graphs are captured before it runs. */
  auto capture_forward = [&](long t0, cudaGraphExec_t *ge) -> int {
    const long t1 = std::min<long>(T, t0 + GP_GRAPH_STEPS);
    return capture_graph(
        b,
        [&]() -> int {
          for (long t = t0; t < t1; t++) {
            b->redir_in = slot_ptr((int)t);
            b->redir_out = t + 1 < T ? slot_ptr((int)t + 1) : m.final_state;
            b->redir_map = m.smaps + t;
            b->redir_have = m.unknown;
            b->dphi_out = m.dtape + Sd * (size_t)t;
            const int r = batch_step_once(b, 0, nullptr);
            b->redir_in = nullptr;
            b->redir_out = nullptr;
            b->redir_map = nullptr;
            b->redir_have = nullptr;
            b->dphi_out = nullptr;
            if (r != GP_OK) return r;
          }
          return GP_OK;
        },
        ge);
  };
  auto capture_reverse = [&](long t1, cudaGraphExec_t *ge) -> int {
    const long t0 = std::max<long>(0, t1 - GP_GRAPH_STEPS);
    return capture_graph(
        b,
        [&]() -> int {
          for (long t = t1 - 1; t >= t0; t--) {
            const int r = reverse(t, slot_ptr((int)t));
            if (r != GP_OK) return r;
          }
          return GP_OK;
        },
        ge);
  };
  int rcur_seed = rcur, rcur_after = rcur;
  double *ybar_seed = m.ybar, *ybar_after = m.ybar;
  const void *start = b->state[b->cur];   /* a capture of steps moves b->cur on */
  if (m.dtape) {
    /* every step's delta-phi is on the tape by the time the reverse sweep reads it */
    std::fill(have_dphi.begin(), have_dphi.end(), 1);
    if ((rc = capture_forward(0, &m.first[0])) != GP_OK || (rc = capture_reverse(T, &m.first[1])) != GP_OK)
      return rc;
    /* the seed goes into the block the first reverse graph reads */
    rcur_after = rcur;
    ybar_after = m.ybar;
    rcur = rcur_seed;
    m.ybar = ybar_seed;
  }
  CK(cudaEventRecord(e0, b->stream));
  CK(cudaMemcpyAsync(m.snap, start, S * 8, cudaMemcpyDeviceToDevice, b->stream));
  CK(cudaMemsetAsync(m.pbar, 0, gpd::ADJ_NPARAM * 8, b->stream));
  if (m.dtape) {
    for (long t0 = 0; t0 < T; t0 += GP_GRAPH_STEPS) {
      if (t0 == 0) rc = launch_once(b, &m.first[0]);
      else {
        cudaGraphExec_t ge;
        if ((rc = capture_forward(t0, &ge)) == GP_OK) rc = launch_once(b, &ge);
      }
      if (rc != GP_OK) return rc;
    }
    if ((rc = seed()) != GP_OK) return rc;
    rcur = rcur_after;
    m.ybar = ybar_after;
    for (long t1 = T; t1 > 0; t1 -= GP_GRAPH_STEPS) {
      if (t1 == T) rc = launch_once(b, &m.first[1]);
      else {
        cudaGraphExec_t ge;
        if ((rc = capture_reverse(t1, &ge)) == GP_OK) rc = launch_once(b, &ge);
      }
      if (rc != GP_OK) return rc;
    }
  }
  while (!m.dtape && !stack.empty()) {
    const Task t = stack.back();
    stack.pop_back();
    if (t.l == 0) {
      free_slots.push_back(t.slot);
      continue;
    }
    if (t.l == 1) {
      /* the state is in its slot; unless this is the last step, which comes
       * straight after the forward pass reached it */
      if (!seeded) {
        if ((rc = load(t.a, t.slot)) != GP_OK || (rc = reverse_work()) != GP_OK) return rc;
      } else if ((rc = reverse(t.a, slot_ptr(t.slot))) != GP_OK)
        return rc;
      continue;
    }
    if (t.s == 0) {
      for (long i = t.l - 1; i >= 0; i--)
        if ((rc = load(t.a, t.slot)) != GP_OK || (rc = advance(i)) != GP_OK || (rc = reverse_work()) != GP_OK)
          return rc;
      continue;
    }
    long lo = 1, hi = t.l - 1;
    auto cost_at = [&](long mm) { return mm + adj_rev_cost(t.l - mm, t.s - 1) + adj_rev_cost(mm, t.s); };
    while (lo < hi) {
      const long mid = (lo + hi) / 2;
      if (cost_at(mid + 1) < cost_at(mid)) lo = mid + 1;
      else hi = mid;
    }
    const long mm = lo;
    const int j = free_slots.back();
    free_slots.pop_back();
    if ((rc = load(t.a, t.slot)) != GP_OK || (rc = advance(mm)) != GP_OK) return rc;
    CK(cudaMemcpyAsync(slot_ptr(j), b->state[b->cur], S * 8, cudaMemcpyDeviceToDevice, b->stream));
    stack.push_back({t.a, mm, t.s, t.slot});
    stack.push_back({0, 0, 0, j});
    stack.push_back({t.a + mm, t.l - mm, t.s - 1, j});
  }
  CK(cudaEventRecord(e2, b->stream));
  if ((rc = batch_check_error(b)) != GP_OK) return rc;

  /* ---- results; the context goes back to the final state */
  double pb[gpd::ADJ_NPARAM];
  CK(cudaMemcpyAsync(pb, m.pbar, sizeof pb, cudaMemcpyDeviceToHost, b->stream));
  if (out->phi0_bar &&
      (rc = planes_copy(b, out->phi0_bar, my, m.ybar, g.pitch, N, mx * my, g.plane, mx, my, d2h)) != GP_OK)
    return rc;
  if (out->mu0_bar &&
      (rc = planes_copy(b, out->mu0_bar, my, m.ybar + N * g.plane, g.pitch, K, mx * my, g.plane, mx, my, d2h)) !=
          GP_OK)
    return rc;
  CK(cudaMemcpyAsync(b->state[b->cur], m.final_state, S * 8, cudaMemcpyDeviceToDevice, b->stream));
  if ((rc = batch_reflag(b, true)) != GP_OK) return rc;
  CK(cudaStreamSynchronize(b->stream));
  b->steps = steps0 + T;
  out->d_tau = pb[gpd::ADJ_TAU];
  out->d_dab = pb[gpd::ADJ_DAB];
  out->d_epsilon = pb[gpd::ADJ_EPS];
  out->d_gamma = pb[gpd::ADJ_GAMMA];
  out->snapshots = nsnap;
  out->recomputed = adj_rev_cost(T, nsnap) - (T - 1);
  float f1 = 0.f, f2 = 0.f;
  CK(cudaEventElapsedTime(&f1, e0, e1));
  CK(cudaEventElapsedTime(&f2, e1, e2));
  out->ms_forward = f1;
  out->ms_reverse = f2;
  return GP_OK;
}

int gp_adjoint_replay(gp_ctx *c, long nsteps, double *max_abs_diff, long long *n_diff) {
  gpd::AdjLaunch L;
  int rc = adj_check(c, &L);
  if (rc) return rc;
  if (nsteps < 0 || !max_abs_diff || !n_diff) return fail(c, GP_EINVAL, "gp_adjoint_replay: bad argument");
  c->err[0] = 0;
  gp_batch *b = c->b;
  const gpd::Grid &g = b->desc[0].g;
  const int N = b->N, K = b->K;
  const size_t S = (size_t)(N + K) * g.plane, Sd = (size_t)N * g.dplane;
  const gpd::AdjParams prm = adj_params(b->params[0]);
  AdjBufs m;
  if (cudaMalloc((void **)&m.seg, 2 * S * 8) != cudaSuccess || cudaMalloc((void **)&m.dphi, Sd * 8) != cudaSuccess)
    return fail(c, GP_ENOMEM, "gp_adjoint_replay: cudaMalloc failed");
  double *a = m.seg, *a2 = m.seg + S;
  CK(cudaMemcpyAsync(a, b->state[b->cur], S * 8, cudaMemcpyDeviceToDevice, b->stream));
  for (long s = 0; s < nsteps; s++) {
    CK(L.dphi(b->stream, b->d_consts, prm, g, a, m.dphi));
    CK(L.update(b->stream, b->d_consts, prm, g, a, m.dphi, a2));
    std::swap(a, a2);
  }
  if ((rc = batch_step_impl(b, nsteps, nullptr, nullptr, nullptr, nullptr)) != GP_OK) return rc;
  std::vector<double> x(S), y(S);
  CK(cudaMemcpyAsync(x.data(), a, S * 8, cudaMemcpyDeviceToHost, b->stream));
  CK(cudaMemcpyAsync(y.data(), b->state[b->cur], S * 8, cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  double mxd = 0.0;
  long long nd = 0;
  for (int f = 0; f < N + K; f++)
    for (int i = 0; i < g.mx; i++)
      for (int j = 0; j < g.my; j++) {
        const size_t o = (size_t)f * g.plane + (size_t)i * g.pitch + j;
        if (memcmp(&x[o], &y[o], 8) != 0) {
          nd++;
          mxd = std::max(mxd, fabs(x[o] - y[o]));
        }
      }
  *max_abs_diff = mxd;
  *n_diff = nd;
  return GP_OK;
}

}  /* extern "C" */

/* ======================================================================= */
/* One time step without any allocation (gp_step_noalloc in gp.h).          */
/*                                                                         */
/* Some callers cannot call cudaMalloc: a host application that hands us   */
/* device buffers from its own pool or arena allocator and forbids any     */
/* other allocation (memory budgets fixed up front, allocator locks it     */
/* must not contend on, or code paths where a failing allocation cannot be */
/* handled).  For them the step's only scratch buffer, delta-phi over the  */
/* interior plus a one-cell ring, lives in this fixed array instead of      */
/* per-context cudaMalloc'd memory.  Every GPU that loads the library holds */
/* these 32 MiB until the process exits.                                    */


#define GP_NOALLOC_SCRATCH_DOUBLES (4u * 1024u * 1024u)   /* 32 MiB */
static __device__ __align__(256) double g_noalloc_scratch[GP_NOALLOC_SCRATCH_DOUBLES];

#define GP_NOALLOC_MAX_DEVICES 64
/* Device address of g_noalloc_scratch per device, looked up on the first call
 * on that device.  In host code the array's name only stands in for the
 * symbol; kernels must be given the address cudaGetSymbolAddress returns. */
static double *g_noalloc_ptr[GP_NOALLOC_MAX_DEVICES];

extern "C" int gp_step_noalloc(const gp_params *p, const double *phi_in, const double *mu_in, double *phi_out,
                               double *mu_out, void *stream) {
  gp_ctx *c = nullptr; /* CK() reports through the thread's error slot */
  if (!p || !phi_in || !mu_in || !phi_out || !mu_out)
    return fail(nullptr, GP_EINVAL, "gp_step_noalloc: NULL argument");
  gp_derived d;
  char err[256] = "";
  if (gp_host_derive(p, &d, err, sizeof err) != GP_OK) return fail(nullptr, GP_EINVAL, "gp_step_noalloc: %s", err);
  if (d.tgrad || d.shift)
    return fail(nullptr, GP_EUNSUPPORTED, "gp_step_noalloc: isothermal runs without a moving frame only");
  Kern k;
  if (!pick(d.N, d.K, d.aniso != 0, &k)) return fail(nullptr, GP_EINVAL, "gp_step_noalloc: no kernel for N=%d K=%d", d.N, d.K);
  gpd::Grid g = make_grid(d, 1); /* caller's planes are contiguous [field][MESH_X][MESH_Y] */
  gpd::Consts<double> cs = make_consts<double>(d);
  /* the scratch holds the delta-phi planes (N of them, interior plus a
   * one-cell ring); k_dphi rewrites all of it before k_update reads it, so
   * what an earlier call left there needs no clearing */
  const size_t need = (size_t)d.N * (size_t)g.dplane;
  if (need > GP_NOALLOC_SCRATCH_DOUBLES)
    return fail(nullptr, GP_EINVAL,
                "gp_step_noalloc: grid %ldx%ld with %d phases needs %zu doubles of scratch, the fixed maximum is %u "
                "(about 1.3 million cells for 3 phases); use gp_init/gp_step for larger grids",
                d.mx, d.my, d.N, need, GP_NOALLOC_SCRATCH_DOUBLES);
  /* the step reads every input cell's neighbours after other cells' outputs
   * are written: an output range may share no byte with an input range or
   * with the other output range */
  {
    const size_t cells = (size_t)d.mx * (size_t)d.my;
    struct Range {
      const char *lo, *hi;
    };
    const Range in[2] = {{(const char *)phi_in, (const char *)(phi_in + (size_t)d.N * cells)},
                         {(const char *)mu_in, (const char *)(mu_in + (size_t)d.K * cells)}};
    const Range out[2] = {{(const char *)phi_out, (const char *)(phi_out + (size_t)d.N * cells)},
                          {(const char *)mu_out, (const char *)(mu_out + (size_t)d.K * cells)}};
    auto overlap = [](const Range &a, const Range &b) { return a.lo < b.hi && b.lo < a.hi; };
    for (int o = 0; o < 2; o++)
      for (int i = 0; i < 2; i++)
        if (overlap(out[o], in[i]))
          return fail(nullptr, GP_EINVAL, "gp_step_noalloc: output %s overlaps input %s", o ? "mu" : "phi",
                      i ? "mu" : "phi");
    if (overlap(out[0], out[1])) return fail(nullptr, GP_EINVAL, "gp_step_noalloc: outputs phi and mu overlap");
  }
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= GP_NOALLOC_MAX_DEVICES) return fail(nullptr, GP_EINVAL, "gp_step_noalloc: device %d", dev);
  if (!g_noalloc_ptr[dev]) {
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr)
      return fail(nullptr, GP_ECUDA, "gp_step_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    g_noalloc_ptr[dev] = (double *)ptr;
  }
  double *scratch = g_noalloc_ptr[dev];
  cudaStream_t s = (cudaStream_t)stream;
  CK(cudaFuncSetAttribute(k.dphi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem_dphi));
  CK(cudaFuncSetAttribute(k.upd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem_upd));
  CK(cudaMemcpyToSymbolAsync(cD, &cs, sizeof(cs), 0, cudaMemcpyHostToDevice, s));
  gpd::StatBufs st = {};
  st.ext = nullptr;      /* no progress record on this path: no extremes */
  st.partials = nullptr; /* and no sums */
  st.want_sums = 0;
  double *dphi = scratch;
  dim3 gd((g.my + 2 + gpd::TY - 1) / gpd::TY, (g.mx + 2 + gpd::TX - 1) / gpd::TX);
  dim3 gu((g.my + gpd::TY - 1) / gpd::TY, (g.mx + gpd::TX - 1) / gpd::TX);
  k.dphi<<<gd, gpd::NT, k.smem_dphi, s>>>(phi_in, mu_in, dphi, g);
  k.upd<<<gu, gpd::NT, k.smem_upd, s>>>(phi_in, mu_in, dphi, phi_out, mu_out, g, st);
  CK(cudaGetLastError());
  return GP_OK;
}
