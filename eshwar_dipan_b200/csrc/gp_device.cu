/*
 * gp_device.cu -- libgp: the C ABI (include/gp.h) over the sm_100a kernels.
 * Host orchestration only; the kernels are in gp_step64.cuh / gp_smooth64.cuh.
 */
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <climits>
#include <cstring>

#include "gp_smooth64.cuh"


extern "C" const char *gp_host_thread_error(void);

struct gp_ctx {
  gp_params p;
  gp_derived d;
  gp_precision prec;
  int dev;
  cudaStream_t stream;
  gpd::Grid g;
  double *phi[2], *mu[2];       /* ping-pong state planes */
  int cur;
  double *dphi;                 /* delta-phi over the interior plus a ring */
  long long *ext;               /* per-block running extremes, ordered integers [ublocks][2(N+K)] */
  long long *ext_red;           /* their fold over blocks [2(N+K)] */
  double *partials;             /* per-block sums of the last stats step */
  double *sums;                 /* reduced sums */
  int ublocks;                  /* blocks of k_update */
  long long steps;
  gp_stats last;
  char err[256];
};

namespace {

int fail(gp_ctx *c, int code, const char *fmt, ...) {
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

#define CK(call)                                                                        \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess) return fail(c, GP_ECUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

bool pow2(double v) {
  int e;
  double m = frexp(fabs(v), &e);
  return v != 0.0 && m == 0.5;
}

/* ---- kernel dispatch over the template parameters -------------------- */

struct Kern {
  void (*dphi)(const double *, const double *, double *, gpd::Grid);
  void (*upd)(const double *, const double *, const double *, double *, double *, gpd::Grid, gpd::StatBufs);
  void (*sdphi)(const double *, double *, gpd::Grid);
  void (*supd)(const double *, const double *, const double *, double *, double *, gpd::Grid);
  size_t smem_dphi, smem_upd;
};

template <int N, int K, bool A>
Kern make() {
  Kern k;
  k.dphi = gpd::k_dphi<N, K, A>;
  k.upd = gpd::k_update<N, K>;
  k.sdphi = gpd::k_sdphi<N, A>;
  k.supd = gpd::k_supdate<N, K>;
  k.smem_dphi = sizeof(gpd::DphiSmem<N>);
  k.smem_upd = sizeof(gpd::UpdSmem<N, K>);
  return k;
}

bool pick(int N, int K, bool A, Kern *out) {
#define CASE(n, k)                                   \
  if (N == n && K == k) {                            \
    *out = A ? make<n, k, true>() : make<n, k, false>(); \
    return true;                                     \
  }
  CASE(2, 1) CASE(3, 1) CASE(4, 1) CASE(2, 2) CASE(3, 2) CASE(4, 2)
#undef CASE
  return false;
}

int setup_kernels(gp_ctx *c, const Kern &k) {
  CK(cudaFuncSetAttribute(k.dphi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem_dphi));
  CK(cudaFuncSetAttribute(k.upd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem_upd));
  return GP_OK;
}

/* Fold the per-block sums (one CTA per quantity) in a fixed order: the result
 * does not depend on scheduling. */
__global__ void k_reduce_partials(const double *__restrict__ part, int nblocks, int nsum, double *__restrict__ out) {
  __shared__ double r[256];
  const int f = blockIdx.x;
  double s = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += 256) s += part[(long long)b * nsum + f];
  r[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) r[threadIdx.x] += r[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[f] = r[0];
}

/* Fold the per-block running extremes: slot f < nmax is a maximum, else a minimum. */
__global__ void k_reduce_ext(const long long *__restrict__ ext, int nblocks, int nslot, int N, int K,
                             long long *__restrict__ out) {
  __shared__ long long r[256];
  const int f = blockIdx.x;
  const bool isMax = f < N || (f >= 2 * N && f < 2 * N + K);
  long long v = isMax ? LLONG_MIN : LLONG_MAX;
  for (int b = threadIdx.x; b < nblocks; b += 256) {
    long long w = ext[(long long)b * nslot + f];
    v = isMax ? (w > v ? w : v) : (w < v ? w : v);
  }
  r[threadIdx.x] = v;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      long long a = r[threadIdx.x], b = r[threadIdx.x + w];
      r[threadIdx.x] = isMax ? (a > b ? a : b) : (a < b ? a : b);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) out[f] = r[0];
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

int upload_state(gp_ctx *c, const double *phi, const double *mu, cudaMemcpyKind kind) {
  const gp_derived &d = c->d;
  for (int a = 0; a < d.N; a++)
    CK(cudaMemcpy2DAsync(c->phi[c->cur] + a * c->g.plane, (size_t)c->g.pitch * 8, phi + (size_t)a * d.mx * d.my,
                         (size_t)d.my * 8, (size_t)d.my * 8, (size_t)d.mx, kind, c->stream));
  for (int k = 0; k < d.K; k++)
    CK(cudaMemcpy2DAsync(c->mu[c->cur] + k * c->g.plane, (size_t)c->g.pitch * 8, mu + (size_t)k * d.mx * d.my,
                         (size_t)d.my * 8, (size_t)d.my * 8, (size_t)d.mx, kind, c->stream));
  return GP_OK;
}

int download_state(gp_ctx *c, double *phi, double *mu, cudaMemcpyKind kind) {
  const gp_derived &d = c->d;
  for (int a = 0; a < d.N; a++)
    CK(cudaMemcpy2DAsync(phi + (size_t)a * d.mx * d.my, (size_t)d.my * 8, c->phi[c->cur] + a * c->g.plane,
                         (size_t)c->g.pitch * 8, (size_t)d.my * 8, (size_t)d.mx, kind, c->stream));
  for (int k = 0; k < d.K; k++)
    CK(cudaMemcpy2DAsync(mu + (size_t)k * d.mx * d.my, (size_t)d.my * 8, c->mu[c->cur] + k * c->g.plane,
                         (size_t)c->g.pitch * 8, (size_t)d.my * 8, (size_t)d.mx, kind, c->stream));
  return GP_OK;
}

/* Running extremes start where the reference starts them (serialinfo_xy.h:59-66):
 * phi max 1, min 0; mu max 1, min 1; every block slot holds them. */
int reset_minmax(gp_ctx *c) {
  const int N = c->d.N, K = c->d.K, ne = 2 * (N + K);
  long long *h = (long long *)malloc(sizeof(long long) * (size_t)ne * c->ublocks);
  if (!h) return fail(c, GP_ENOMEM, "gp_init: out of host memory");
  for (int b = 0; b < c->ublocks; b++) {
    long long *s = h + (size_t)b * ne;
    for (int a = 0; a < N; a++) { s[a] = to_ord(1.0); s[N + a] = to_ord(0.0); }
    for (int k = 0; k < K; k++) { s[2 * N + k] = to_ord(1.0); s[2 * N + K + k] = to_ord(1.0); }
  }
  cudaError_t e = cudaMemcpyAsync(c->ext, h, sizeof(long long) * (size_t)ne * c->ublocks, cudaMemcpyHostToDevice,
                                  c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  free(h);
  if (e != cudaSuccess) return fail(c, GP_ECUDA, "gp_init: %s", cudaGetErrorString(e));
  return GP_OK;
}

}  // namespace

/* ======================================================================= */

/* The constant block is per module and device; a context re-uploads it when
 * another context was used last.  Contexts are not meant to be driven from
 * several host threads at once. */
static const gp_ctx *g_last_ctx = nullptr;

extern "C" {

const char *gp_version(void) { return "libgp 0.1 (sm_100a, FP64 plain step)"; }

size_t gp_params_size(void) { return sizeof(gp_params); }

const char *gp_last_error(const gp_ctx *ctx) { return ctx ? ctx->err : gp_host_thread_error(); }

void *gp_stream(gp_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int gp_init(gp_ctx **out, const gp_params *p, const double *phi, const double *mu, gp_precision prec) {
  gp_ctx *c = nullptr;
  if (!out || !p || !phi || !mu) return fail(nullptr, GP_EINVAL, "gp_init: NULL argument");
  *out = nullptr;
  if (prec != GP_FP64) return fail(nullptr, GP_EUNSUPPORTED, "gp_init: only GP_FP64 is built in this context type");
  c = (gp_ctx *)calloc(1, sizeof(gp_ctx));
  if (!c) return fail(nullptr, GP_ENOMEM, "gp_init: out of host memory");
  c->p = *p;
  c->prec = prec;
  char err[256] = "";
  if (gp_host_derive(p, &c->d, err, sizeof err) != GP_OK) {
    int r = fail(nullptr, GP_EINVAL, "gp_init: %s", err);
    free(c);
    return r;
  }
  Kern k;
  if (!pick(c->d.N, c->d.K, c->d.aniso != 0, &k)) {
    free(c);
    return fail(nullptr, GP_EINVAL, "gp_init: no kernel for N=%d K=%d", c->d.N, c->d.K);
  }
  int rc;
  cudaError_t e = cudaGetDevice(&c->dev);
  if (e != cudaSuccess) {
    free(c);
    return fail(nullptr, GP_ECUDA, "gp_init: no CUDA device: %s", cudaGetErrorString(e));
  }
  e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    free(c);
    return fail(nullptr, GP_ECUDA, "gp_init: %s", cudaGetErrorString(e));
  }
  const gp_derived &d = c->d;
  gpd::Grid &g = c->g;
  g.mx = (int)d.mx;
  g.my = (int)d.my;
  g.pitch = (int)((d.my + 31) / 32 * 32);
  g.plane = (long long)g.pitch * d.mx;
  g.dpitch = (int)((d.my + 2 + 31) / 32 * 32);
  g.dplane = (long long)g.dpitch * (d.mx + 2);
  g.dx_pow2 = pow2(d.dx);
  g.dy_pow2 = pow2(d.dy);
  g.inv_dx = 1.0 / d.dx;
  g.inv_dy = 1.0 / d.dy;
  g.inv_2dy = 1.0 / (2.0 * d.dy);
  const int ublocks = (int)(((d.my + gpd::TY - 1) / gpd::TY) * ((d.mx + gpd::TX - 1) / gpd::TX));
  c->ublocks = ublocks;
  const int nsum = 2 * d.N + 2 * d.K + 1;
#define ALLOC(ptr, bytes)                                                           \
  do {                                                                              \
    if (cudaMalloc((void **)&(ptr), (bytes)) != cudaSuccess) {                       \
      rc = fail(c, GP_ENOMEM, "gp_init: cudaMalloc of %zu bytes failed", (size_t)(bytes)); \
      goto bad;                                                                     \
    }                                                                               \
  } while (0)
  ALLOC(c->phi[0], (size_t)g.plane * d.N * 8);
  ALLOC(c->phi[1], (size_t)g.plane * d.N * 8);
  ALLOC(c->mu[0], (size_t)g.plane * d.K * 8);
  ALLOC(c->mu[1], (size_t)g.plane * d.K * 8);
  ALLOC(c->dphi, (size_t)g.dplane * d.N * 8);
  ALLOC(c->ext, sizeof(long long) * 2 * (d.N + d.K) * (size_t)ublocks);
  ALLOC(c->ext_red, sizeof(long long) * 2 * (d.N + d.K));
  ALLOC(c->partials, sizeof(double) * (size_t)ublocks * nsum);
  ALLOC(c->sums, sizeof(double) * nsum);
#undef ALLOC
  if (cudaDeviceSynchronize() != cudaSuccess ||
      cudaMemcpyToSymbol(cD, &c->d, sizeof(gp_derived)) != cudaSuccess) {
    rc = fail(c, GP_ECUDA, "gp_init: constant upload failed");
    goto bad;
  }
  g_last_ctx = c;
  if ((rc = setup_kernels(c, k)) != GP_OK) goto bad;
  if (cudaMemsetAsync(c->dphi, 0, (size_t)g.dplane * d.N * 8, c->stream) != cudaSuccess) {
    rc = fail(c, GP_ECUDA, "gp_init: memset failed");
    goto bad;
  }
  if ((rc = upload_state(c, phi, mu, cudaMemcpyHostToDevice)) != GP_OK) goto bad;
  if ((rc = reset_minmax(c)) != GP_OK) goto bad;
  *out = c;
  return GP_OK;
bad:
  gp_set_thread_error("%s", c->err);
  gp_destroy(c);
  return rc;
}


static int bind(gp_ctx *c) {
  if (g_last_ctx != c) {
    /* another context's kernels may still read the constant block */
    CK(cudaDeviceSynchronize());
    CK(cudaMemcpyToSymbol(cD, &c->d, sizeof(gp_derived)));
    g_last_ctx = c;
  }
  return GP_OK;
}

int gp_smooth(gp_ctx *c, long nsteps) {
  if (!c || nsteps < 0) return fail(c, GP_EINVAL, "gp_smooth: bad argument");
  Kern k;
  pick(c->d.N, c->d.K, c->d.aniso != 0, &k);
  int rc = bind(c);
  if (rc) return rc;
  const gpd::Grid &g = c->g;
  dim3 grid((g.my + 127) / 128, g.mx);
  for (long s = 0; s < nsteps; s++) {
    k.sdphi<<<grid, 128, 0, c->stream>>>(c->phi[c->cur], c->dphi, g);
    k.supd<<<grid, 128, 0, c->stream>>>(c->phi[c->cur], c->mu[c->cur], c->dphi, c->phi[c->cur ^ 1], c->mu[c->cur ^ 1], g);
    c->cur ^= 1;
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return GP_OK;
}

static int fill_stats(gp_ctx *c, gp_stats *s) {
  const int N = c->d.N, K = c->d.K, nsum = 2 * N + 2 * K + 1;
  long long mm[2 * (GPK_MAXN + GPK_MAXK)];
  double sums[2 * GPK_MAXN + 2 * GPK_MAXK + 1];
  gpd::Grid &g = c->g;
  (void)g;
  k_reduce_partials<<<nsum, 256, 0, c->stream>>>(c->partials, c->ublocks, nsum, c->sums);
  k_reduce_ext<<<2 * (N + K), 256, 0, c->stream>>>(c->ext, c->ublocks, 2 * (N + K), N, K, c->ext_red);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(mm, c->ext_red, sizeof(long long) * 2 * (N + K), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(sums, c->sums, sizeof(double) * nsum, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  gp_stats r;
  memset(&r, 0, sizeof r);
  for (int a = 0; a < N; a++) {
    r.phi_max[a] = from_ord(mm[a]);
    r.phi_min[a] = from_ord(mm[N + a]);
    r.rel_change_phi[a] = sums[a];
    r.phi_sum[a] = sums[N + K + a];
  }
  for (int k = 0; k < K; k++) {
    r.mu_max[k] = from_ord(mm[2 * N + k]);
    r.mu_min[k] = from_ord(mm[2 * N + K + k]);
    r.rel_change_mu[k] = sums[N + k];
    r.comp_sum[k] = sums[2 * N + K + k];
  }
  r.nonfinite = (long long)llround(sums[2 * N + 2 * K]);
  r.steps_done = c->steps;
  c->last = r;
  if (s) *s = r;
  return GP_OK;
}

static int step_impl(gp_ctx *c, long nsteps, gp_stats *stats, double *total_ms, double *ms_phase,
                     double *ms_update);

int gp_step(gp_ctx *c, long nsteps, gp_stats *stats) { return step_impl(c, nsteps, stats, nullptr, nullptr, nullptr); }

int gp_step_timed(gp_ctx *c, long nsteps, gp_stats *stats, double *total_ms, double *ms_phase, double *ms_update) {
  return step_impl(c, nsteps, stats, total_ms, ms_phase, ms_update);
}

static int step_impl(gp_ctx *c, long nsteps, gp_stats *stats, double *total_ms, double *ms_phase,
                     double *ms_update) {
  if (!c || nsteps < 0) return fail(c, GP_EINVAL, "gp_step: bad argument");
  const bool timed = total_ms || ms_phase || ms_update;
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  double t_phase = 0.0, t_update = 0.0;
  Kern k;
  pick(c->d.N, c->d.K, c->d.aniso != 0, &k);
  int rc = bind(c);
  if (rc) return rc;
  const gpd::Grid &g = c->g;
  dim3 gd((g.my + 2 + gpd::TY - 1) / gpd::TY, (g.mx + 2 + gpd::TX - 1) / gpd::TX);
  dim3 gu((g.my + gpd::TY - 1) / gpd::TY, (g.mx + gpd::TX - 1) / gpd::TX);
  if (timed) {
    for (int i = 0; i < 3; i++) CK(cudaEventCreate(&ev[i]));
  }
  cudaEvent_t t_start = nullptr, t_end = nullptr;
  if (total_ms) {
    CK(cudaEventCreate(&t_start));
    CK(cudaEventCreate(&t_end));
    CK(cudaEventRecord(t_start, c->stream));
  }
  for (long s = 0; s < nsteps; s++) {
    gpd::StatBufs st;
    st.ext = c->ext;
    st.partials = c->partials;
    st.want_sums = (stats != nullptr && s == nsteps - 1);
    if (timed) CK(cudaEventRecord(ev[0], c->stream));
    k.dphi<<<gd, gpd::NT, k.smem_dphi, c->stream>>>(c->phi[c->cur], c->mu[c->cur], c->dphi, g);
    if (timed) CK(cudaEventRecord(ev[1], c->stream));
    k.upd<<<gu, gpd::NT, k.smem_upd, c->stream>>>(c->phi[c->cur], c->mu[c->cur], c->dphi, c->phi[c->cur ^ 1],
                                                   c->mu[c->cur ^ 1], g, st);
    if (timed) {
      float a = 0.f, b = 0.f;
      CK(cudaEventRecord(ev[2], c->stream));
      CK(cudaEventSynchronize(ev[2]));
      CK(cudaEventElapsedTime(&a, ev[0], ev[1]));
      CK(cudaEventElapsedTime(&b, ev[1], ev[2]));
      t_phase += a;
      t_update += b;
    }
    c->cur ^= 1;
    c->steps++;
  }
  CK(cudaGetLastError());
  if (total_ms) {
    float tt = 0.f;
    CK(cudaEventRecord(t_end, c->stream));
    CK(cudaEventSynchronize(t_end));
    CK(cudaEventElapsedTime(&tt, t_start, t_end));
    *total_ms = tt;
    cudaEventDestroy(t_start);
    cudaEventDestroy(t_end);
  }
  if (timed) {
    for (int i = 0; i < 3; i++) cudaEventDestroy(ev[i]);
    if (ms_phase) *ms_phase = t_phase;
    if (ms_update) *ms_update = t_update;
  }
  if (stats && nsteps > 0) return fill_stats(c, stats);
  CK(cudaStreamSynchronize(c->stream));
  return GP_OK;
}

int gp_get_stats(gp_ctx *c, gp_stats *s) {
  if (!c || !s) return fail(c, GP_EINVAL, "gp_get_stats: bad argument");
  *s = c->last;
  return GP_OK;
}

int gp_get(gp_ctx *c, double *phi, double *mu) {
  if (!c || !phi || !mu) return fail(c, GP_EINVAL, "gp_get: NULL argument");
  int rc = download_state(c, phi, mu, cudaMemcpyDeviceToHost);
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream));
  return GP_OK;
}

int gp_set(gp_ctx *c, const double *phi, const double *mu) {
  if (!c || !phi || !mu) return fail(c, GP_EINVAL, "gp_set: NULL argument");
  int rc = upload_state(c, phi, mu, cudaMemcpyHostToDevice);
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream));
  return GP_OK;
}

int gp_get_dev(gp_ctx *c, double *phi, double *mu) {
  if (!c || !phi || !mu) return fail(c, GP_EINVAL, "gp_get_dev: NULL argument");
  int rc = download_state(c, phi, mu, cudaMemcpyDeviceToDevice);
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream));
  return GP_OK;
}

int gp_set_dev(gp_ctx *c, const double *phi, const double *mu) {
  if (!c || !phi || !mu) return fail(c, GP_EINVAL, "gp_set_dev: NULL argument");
  int rc = upload_state(c, phi, mu, cudaMemcpyDeviceToDevice);
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream));
  return GP_OK;
}

void gp_destroy(gp_ctx *c) {
  if (!c) return;
  if (c->stream) cudaStreamSynchronize(c->stream);
  cudaFree(c->phi[0]);
  cudaFree(c->phi[1]);
  cudaFree(c->mu[0]);
  cudaFree(c->mu[1]);
  cudaFree(c->dphi);
  cudaFree(c->ext);
  cudaFree(c->ext_red);
  cudaFree(c->partials);
  cudaFree(c->sums);
  if (c->stream) cudaStreamDestroy(c->stream);
  if (g_last_ctx == c) g_last_ctx = nullptr;
  free(c);
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
/* interior plus a one-cell ring, and the running-extreme counters live in */
/* this fixed array instead of per-context cudaMalloc'd memory.  Every GPU */
/* that loads the library holds these 32 MiB until the process exits.      */
/* ======================================================================= */

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
  if (phi_in == phi_out || mu_in == mu_out)
    return fail(nullptr, GP_EINVAL, "gp_step_noalloc: input and output buffers must differ");
  gp_derived d;
  char err[256] = "";
  if (gp_host_derive(p, &d, err, sizeof err) != GP_OK) return fail(nullptr, GP_EINVAL, "gp_step_noalloc: %s", err);
  Kern k;
  if (!pick(d.N, d.K, d.aniso != 0, &k)) return fail(nullptr, GP_EINVAL, "gp_step_noalloc: no kernel for N=%d K=%d", d.N, d.K);
  gpd::Grid g;
  g.mx = (int)d.mx;
  g.my = (int)d.my;
  g.pitch = (int)d.my; /* caller's planes are contiguous [field][MESH_X][MESH_Y] */
  g.plane = (long long)d.mx * d.my;
  g.dpitch = (int)((d.my + 2 + 31) / 32 * 32);
  g.dplane = (long long)g.dpitch * (d.mx + 2);
  g.dx_pow2 = pow2(d.dx);
  g.dy_pow2 = pow2(d.dy);
  g.inv_dx = 1.0 / d.dx;
  g.inv_dy = 1.0 / d.dy;
  g.inv_2dy = 1.0 / (2.0 * d.dy);
  /* scratch layout: [running extremes, 2(N+K) long longs][pad to 256 B][delta-phi, N planes] */
  const size_t head = 32;  /* doubles; holds 2*(4+2) long longs and keeps delta-phi 256-B aligned */
  const size_t need = head + (size_t)d.N * (size_t)g.dplane;
  if (need > GP_NOALLOC_SCRATCH_DOUBLES)
    return fail(nullptr, GP_EINVAL,
                "gp_step_noalloc: grid %ldx%ld with %d phases needs %zu doubles of scratch, the fixed maximum is %u "
                "(about 1.3 million cells for 3 phases); use gp_init/gp_step for larger grids",
                d.mx, d.my, d.N, need, GP_NOALLOC_SCRATCH_DOUBLES);
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
  /* the constant block is shared with the contexts: make them upload theirs again */
  g_last_ctx = nullptr;
  CK(cudaMemcpyToSymbolAsync(cD, &d, sizeof(gp_derived), 0, cudaMemcpyHostToDevice, s));
  /* the previous call's extremes are still in the array: start them from zero */
  CK(cudaMemsetAsync(scratch, 0, head * sizeof(double), s));
  gpd::StatBufs st;
  st.ext = nullptr; /* no progress record on this path */
  st.partials = scratch; /* not written: no sums requested */
  st.want_sums = 0;
  double *dphi = scratch + head;
  dim3 gd((g.my + 2 + gpd::TY - 1) / gpd::TY, (g.mx + 2 + gpd::TX - 1) / gpd::TX);
  dim3 gu((g.my + gpd::TY - 1) / gpd::TY, (g.mx + gpd::TX - 1) / gpd::TX);
  k.dphi<<<gd, gpd::NT, k.smem_dphi, s>>>(phi_in, mu_in, dphi, g);
  k.upd<<<gu, gpd::NT, k.smem_upd, s>>>(phi_in, mu_in, dphi, phi_out, mu_out, g, st);
  CK(cudaGetLastError());
  return GP_OK;
}
