/*
 * gp_batch_impl.cuh -- launchers of the batched kernels for one field type.
 * Included by gp_device.cu (FP64, compiled without FMA contraction so that it
 * stays bit-identical to the reference) and gp_batch32.cu (FP32 storage form,
 * compiled with FMA contraction).  Each exposes a BatchLaunch table.
 */
#pragma once
#include <cuda_runtime.h>

#include "gp_smooth.cuh"

namespace gpd {

struct BatchLaunch {
  cudaError_t (*prepare)(int *blocks_per_sm_dphi, int *blocks_per_sm_upd);
  cudaError_t (*dphi)(int grid, cudaStream_t s, const SimDesc *sims, const void *consts, const int *tsim,
                      int ntiles, int *counter, const void *state, void *dphi);
  cudaError_t (*update)(int grid, cudaStream_t s, const SimDesc *sims, const void *consts, const int *tsim,
                        int ntiles, int *counter, const void *state, const void *dphi, void *next, StatBufs st);
  cudaError_t (*sdphi)(cudaStream_t s, const void *consts, const void *phi, void *dphi, Grid g);
  cudaError_t (*supd)(cudaStream_t s, const void *consts, const void *phi, const void *mu, const void *dphi,
                      void *phin, void *mun, Grid g);
  size_t elem;
};

template <typename R, int N, int K, bool A>
struct BatchKernels {
  static cudaError_t prepare(int *bd, int *bu) {
    cudaError_t e = cudaFuncSetAttribute(kb_dphi<R, N, K, A>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sizeof(DphiSmem<R, N>));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(kb_update<R, N, K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(UpdSmem<R, N, K>));
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(bd, kb_dphi<R, N, K, A>, NT, sizeof(DphiSmem<R, N>));
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bu, kb_update<R, N, K>, NT, sizeof(UpdSmem<R, N, K>));
  }
  static cudaError_t dphi(int grid, cudaStream_t s, const SimDesc *sims, const void *consts, const int *tsim,
                          int ntiles, int *counter, const void *state, void *dphi) {
    kb_dphi<R, N, K, A><<<grid, NT, sizeof(DphiSmem<R, N>), s>>>(
        sims, (const Consts<R> *)consts, tsim, ntiles, counter, (const R *)state, (R *)dphi);
    return cudaGetLastError();
  }
  static cudaError_t update(int grid, cudaStream_t s, const SimDesc *sims, const void *consts, const int *tsim,
                            int ntiles, int *counter, const void *state, const void *dphi, void *next, StatBufs st) {
    kb_update<R, N, K><<<grid, NT, sizeof(UpdSmem<R, N, K>), s>>>(
        sims, (const Consts<R> *)consts, tsim, ntiles, counter, (const R *)state, (const R *)dphi, (R *)next, st);
    return cudaGetLastError();
  }
  static cudaError_t sdphi(cudaStream_t s, const void *consts, const void *phi, void *dphi, Grid g) {
    dim3 grid((g.my + 127) / 128, g.mx);
    k_sdphi<R, N, A><<<grid, 128, 0, s>>>((const Consts<R> *)consts, (const R *)phi, (R *)dphi, g);
    return cudaGetLastError();
  }
  static cudaError_t supd(cudaStream_t s, const void *consts, const void *phi, const void *mu, const void *dphi,
                          void *phin, void *mun, Grid g) {
    dim3 grid((g.my + 127) / 128, g.mx);
    k_supdate<R, N, K><<<grid, 128, 0, s>>>((const Consts<R> *)consts, (const R *)phi, (const R *)mu,
                                            (const R *)dphi, (R *)phin, (R *)mun, g);
    return cudaGetLastError();
  }
  static BatchLaunch table() {
    BatchLaunch t;
    t.prepare = prepare;
    t.dphi = dphi;
    t.update = update;
    t.sdphi = sdphi;
    t.supd = supd;
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
