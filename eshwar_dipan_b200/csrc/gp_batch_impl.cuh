/*
 * gp_batch_impl.cuh -- launchers of the batched kernels for one field type.
 * Included by gp_device.cu (FP64, compiled without FMA contraction so that it
 * stays bit-identical to the reference) and gp_batch32.cu (FP32 storage form,
 * compiled with FMA contraction).  Each exposes a BatchLaunch table.
 */
#pragma once
#include <cuda_runtime.h>

#include "gp_fused.cuh"
#include "gp_smooth.cuh"

namespace gpd {

struct BatchLaunch {
  /* occupancy of the bulk and interface kernels (blocks per SM) */
  cudaError_t (*prepare)(int *blocks_per_sm_bulk, int *blocks_per_sm_general);
  /* one step: bulk tiles + interface list, then the interface tiles */
  /* flag_out: the flags of the buffer the step writes (copied into the bulk entries) */
  cudaError_t (*classify)(int ntiles, cudaStream_t s, const SimDesc *sims, const void *consts, const int *tsim,
                          const TileFlags *flag_in, const TileFlags *flag_out, int *glist, int4 *blist, int *ctr);
  /* mul: every simulation's spacings are powers of two (x/dx == x*(1/dx)) */
  /* ndone: the CTAs of this step's kf_bulk and kf_general together */
  /* tmaps: per simulation two tensor maps of its mu planes (state buffer 0
   * and 1); buf: the buffer `state` is; diag: every phase's off-diagonal D,
   * c_mu and A are zero and no E is -0 (the bulk kernel leaves those terms
   * out) */
  cudaError_t (*bulk)(int grid, bool mul, bool diag, cudaStream_t s, const SimDesc *sims, const void *consts, const int *tsim,
                      const int4 *blist, const TensorMapSlot *tmaps, int buf, const void *state, void *next,
                      TileFlags *flag_out, int *ctr, int ndone, StatBufs st);
  /* bulk and interface tiles in one launch (kf_step; not for a sums step) */
  cudaError_t (*step)(int grid, bool mul, bool diag, cudaStream_t s, const SimDesc *sims, const void *consts,
                      const int *tsim, const int4 *blist, const int *glist, const TensorMapSlot *tmaps, int buf,
                      const void *state, void *next, TileFlags *flag_out, int *ctr, int ndone, StatBufs st);
  /* blocks per SM of kf_step */
  int (*step_occupancy)();
  cudaError_t (*general)(int grid, bool mul, cudaStream_t s, const SimDesc *sims, const void *consts, const int *tsim,
                         const void *state, void *next, TileFlags *flag_out, const int *glist, int *ctr, int ndone,
                         StatBufs st);
  cudaError_t (*flags)(int ntiles, cudaStream_t s, const SimDesc *sims, const int *tsim, const void *state,
                       TileFlags *flags);
  /* one smoothing sweep of a simulation (tcc: its temperature rows, or NULL) */
  cudaError_t (*smooth)(cudaStream_t s, const void *consts, const void *phi, const void *mu, void *phin,
                        void *mun, Grid g, const double *tcc);
  /* moving frame: interface position into pos[s] (zeroed by the caller),
   * then the shifted (or copied) state into next */
  cudaError_t (*shift_pos)(int ntiles, cudaStream_t s, const SimDesc *sims, const void *consts, const int *tsim,
                           const void *state, int *pos);
  cudaError_t (*shift_apply)(int ntiles, cudaStream_t s, const SimDesc *sims, const void *consts, const int *tsim,
                             const void *state, void *next, const int *pos, SimDyn *dyn);
  /* the temperature rows of the coming step (non-isothermal simulations) */
  cudaError_t (*trows)(int nsims, cudaStream_t s, const SimDesc *sims, const void *consts, const int *ctr,
                       SimDyn *dyn, double *rows);
  size_t elem;
};

template <typename R, int N, int K, bool A>
struct BatchKernels {
  static constexpr size_t bulk_smem = bulk_smem_bytes<R, K>();
  static constexpr size_t step_smem =
      sizeof(GenSmem<R, N, K>) > bulk_smem ? sizeof(GenSmem<R, N, K>) : bulk_smem;
  template <bool MUL, bool DIAG>
  static cudaError_t step_attr() {
    return cudaFuncSetAttribute(kf_step<R, N, K, A, MUL, DIAG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)step_smem);
  }
  static int step_occupancy() {
    int n = 0;
    if (step_attr<true, false>() != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kf_step<R, N, K, A, true, false>, NT, step_smem) !=
            cudaSuccess)
      return 0;
    return n;
  }
  static cudaError_t step(int grid, bool mul, bool diag, cudaStream_t s, const SimDesc *sims, const void *consts,
                          const int *tsim, const int4 *blist, const int *glist, const TensorMapSlot *tmaps, int buf,
                          const void *state, void *next, TileFlags *flag_out, int *ctr, int ndone, StatBufs st) {
#define GP_STEP(MUL, DIAG)                                                                                      \
  kf_step<R, N, K, A, MUL, DIAG><<<grid, NT, step_smem, s>>>(sims, (const Consts<R> *)consts, tsim, blist, glist,  \
                                                             tmaps, buf, (const R *)state, (R *)next, flag_out, ctr, \
                                                             ndone, st)
    if (diag) {
      if (mul) GP_STEP(true, true);
      else GP_STEP(false, true);
    } else {
      if (mul) GP_STEP(true, false);
      else GP_STEP(false, false);
    }
#undef GP_STEP
    return cudaGetLastError();
  }
  template <bool SUMS, bool MUL, bool DIAG>
  static cudaError_t bulk_attr() {
    return cudaFuncSetAttribute(kf_bulk<R, N, K, SUMS, MUL, DIAG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)bulk_smem);
  }
  static cudaError_t prepare(int *bb, int *bg) {
    cudaError_t e = cudaFuncSetAttribute(kf_general<R, N, K, A, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sizeof(GenSmem<R, N, K>));
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(kf_general<R, N, K, A, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sizeof(GenSmem<R, N, K>));
    if (e == cudaSuccess) e = bulk_attr<false, false, false>();
    if (e == cudaSuccess) e = bulk_attr<false, true, false>();
    if (e == cudaSuccess) e = bulk_attr<false, false, true>();
    if (e == cudaSuccess) e = bulk_attr<false, true, true>();
    if (e == cudaSuccess) e = bulk_attr<true, false, false>();
    if (e == cudaSuccess) e = bulk_attr<true, true, false>();
    if (e == cudaSuccess) e = step_attr<false, false>();
    if (e == cudaSuccess) e = step_attr<true, false>();
    if (e == cudaSuccess) e = step_attr<false, true>();
    if (e == cudaSuccess) e = step_attr<true, true>();
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(bb, kf_bulk<R, N, K, false, true, false>, NT, bulk_smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bg, kf_general<R, N, K, A, true>, NT,
                                                         sizeof(GenSmem<R, N, K>));
  }
  static cudaError_t classify(int ntiles, cudaStream_t s, const SimDesc *sims, const void *consts,
                              const int *tsim, const TileFlags *flag_in, const TileFlags *flag_out, int *glist,
                              int4 *blist, int *ctr) {
    kf_classify<R><<<(ntiles + NTC - 1) / NTC, NTC, 0, s>>>(sims, (const Consts<R> *)consts, tsim, ntiles, flag_in, flag_out, glist,
                                                         blist, ctr);
    return cudaGetLastError();
  }
  static cudaError_t bulk(int grid, bool mul, bool diag, cudaStream_t s, const SimDesc *sims, const void *consts,
                          const int *tsim, const int4 *blist, const TensorMapSlot *tmaps, int buf,
                          const void *state, void *next, TileFlags *flag_out, int *ctr, int ndone, StatBufs st) {
#define GP_BULK(SUMS, MUL, DIAG)                                                                               \
  kf_bulk<R, N, K, SUMS, MUL, DIAG><<<grid, NT, bulk_smem, s>>>(sims, (const Consts<R> *)consts, tsim, blist, tmaps,  \
                                                          buf, (const R *)state, (R *)next, flag_out, ctr, ndone, st)
    /* the sums step (last of a call) takes every term: same results */
    if (st.want_sums) {
      if (mul) GP_BULK(true, true, false);
      else GP_BULK(true, false, false);
    } else if (diag) {
      if (mul) GP_BULK(false, true, true);
      else GP_BULK(false, false, true);
    } else {
      if (mul) GP_BULK(false, true, false);
      else GP_BULK(false, false, false);
    }
#undef GP_BULK
    return cudaGetLastError();
  }
  static cudaError_t general(int grid, bool mul, cudaStream_t s, const SimDesc *sims, const void *consts,
                             const int *tsim, const void *state, void *next, TileFlags *flag_out, const int *glist,
                             int *ctr, int ndone, StatBufs st) {
    if (mul)
      kf_general<R, N, K, A, true><<<grid, NT, sizeof(GenSmem<R, N, K>), s>>>(
          sims, (const Consts<R> *)consts, tsim, (const R *)state, (R *)next, flag_out, glist, ctr, ndone, st);
    else
      kf_general<R, N, K, A, false><<<grid, NT, sizeof(GenSmem<R, N, K>), s>>>(
          sims, (const Consts<R> *)consts, tsim, (const R *)state, (R *)next, flag_out, glist, ctr, ndone, st);
    return cudaGetLastError();
  }
  static cudaError_t flags(int ntiles, cudaStream_t s, const SimDesc *sims, const int *tsim, const void *state,
                           TileFlags *fl) {
    kf_flags<R, N><<<ntiles, NT, 0, s>>>(sims, tsim, (const R *)state, fl);
    return cudaGetLastError();
  }
  static cudaError_t smooth(cudaStream_t s, const void *consts, const void *phi, const void *mu, void *phin,
                            void *mun, Grid g, const double *tcc) {
    dim3 grid((g.my + 127) / 128, g.mx);
    k_smooth<R, N, K, A><<<grid, 128, 0, s>>>((const Consts<R> *)consts, (const R *)phi, (const R *)mu, (R *)phin,
                                              (R *)mun, g, tcc);
    return cudaGetLastError();
  }
  static cudaError_t shift_pos(int ntiles, cudaStream_t s, const SimDesc *sims, const void *consts, const int *tsim,
                               const void *state, int *pos) {
    ks_pos<R, N><<<ntiles, NT, 0, s>>>(sims, (const Consts<R> *)consts, tsim, (const R *)state, pos);
    return cudaGetLastError();
  }
  static cudaError_t shift_apply(int ntiles, cudaStream_t s, const SimDesc *sims, const void *consts,
                                 const int *tsim, const void *state, void *next, const int *pos, SimDyn *dyn) {
    ks_shift<R, N, K><<<ntiles, NT, 0, s>>>(sims, (const Consts<R> *)consts, tsim, (const R *)state, (R *)next, pos,
                                            dyn);
    return cudaGetLastError();
  }
  static cudaError_t trows(int nsims, cudaStream_t s, const SimDesc *sims, const void *consts, const int *ctr,
                           SimDyn *dyn, double *rows) {
    kt_rows<R><<<nsims, 128, 0, s>>>(sims, (const Consts<R> *)consts, ctr, dyn, rows);
    return cudaGetLastError();
  }
  static BatchLaunch table() {
    BatchLaunch t;
    t.prepare = prepare;
    t.classify = classify;
    t.bulk = bulk;
    t.step = step;
    t.step_occupancy = step_occupancy;
    t.general = general;
    t.flags = flags;
    t.smooth = smooth;
    t.trows = trows;
    t.shift_pos = shift_pos;
    t.shift_apply = shift_apply;
    t.elem = sizeof(R);
    return t;
  }
};

template <typename R>
bool batch_launch_table(int N, int K, bool A, BatchLaunch *out) {
#define GP_CASE(n, k)                                                                                   \
  if (N == n && K == k) {                                                                               \
    *out = A ? BatchKernels<R, n, k, true>::table() : BatchKernels<R, n, k, false>::table();            \
    return true;                                                                                        \
  }
  GP_CASE(2, 1) GP_CASE(3, 1) GP_CASE(4, 1) GP_CASE(2, 2) GP_CASE(3, 2) GP_CASE(4, 2)
#undef GP_CASE
  return false;
}

}  // namespace gpd

/* defined in gp_device.cu (FP64) and gp_batch32.cu (FP32) */
bool gp_batch_launch_f64(int N, int K, bool aniso, gpd::BatchLaunch *out);
bool gp_batch_launch_f32(int N, int K, bool aniso, gpd::BatchLaunch *out);
