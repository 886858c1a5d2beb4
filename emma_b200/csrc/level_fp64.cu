// level_fp64.cu -- plain-path instantiation of the level kernel.  Built with
// -fmad=false so that FP64 expressions round exactly as the reference's CPU
// build (gcc, no FMA contraction) does.
#include "level_kernel.cuh"

namespace emma {

using KF64 = BrickSmem<MathF64>;

size_t level_smem_fp64() { return KF64::bytes; }

// Persistent launch of a work list: grid = co-resident CTAs (occupancy x SMs).
cudaError_t launch_level_fp64(const BatchArgs &a, int nsm, cudaStream_t s) {
  static int blocks_per_sm = 0;
  auto k = level_batch_kernel<MathF64>;
  if (blocks_per_sm == 0) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)KF64::bytes);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k, kNT, KF64::bytes);
    if (e != cudaSuccess) return e;
    if (blocks_per_sm < 1) return cudaErrorInvalidConfiguration;
  }
  if (a.nwork == 0) return cudaSuccess;
  int grid = blocks_per_sm * nsm;
  if (grid > a.nwork) grid = a.nwork;
  k<<<grid, kNT, KF64::bytes, s>>>(a);
  return cudaGetLastError();
}

}  // namespace emma
