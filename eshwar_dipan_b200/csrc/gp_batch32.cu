/*
 * gp_batch32.cu -- the FP32 storage form of the batched step: fields stored
 * and stepped in float (with FMA contraction), the dc/dmu inversion and all
 * reductions in FP64 (see update_tile / block_stats in gp_tiles.cuh).
 */
#include "gp_batch_impl.cuh"

bool gp_batch_launch_f32(int N, int K, bool aniso, gpd::BatchLaunch *out) {
  return gpd::batch_launch_table<float>(N, K, aniso, out);
}
