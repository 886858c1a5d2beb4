// level_f32.cu -- mixed-path instantiation of the level kernel: FP32
// reconstruction, wave speeds and fluxes; FP64 compensated update.
#include "level_kernel.cuh"

namespace emma {

using KF32 = BrickSmem<MathF32>;

size_t level_smem_f32() { return KF32::bytes; }

// Persistent launch of a work list: grid = co-resident CTAs (occupancy x SMs).
cudaError_t launch_level_f32(const BatchArgs &a, int nsm, cudaStream_t s) {
  static int blocks_per_sm = 0;
  auto k = level_batch_kernel<MathF32>;
  if (blocks_per_sm == 0) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)KF32::bytes);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k, kNT, KF32::bytes);
    if (e != cudaSuccess) return e;
    if (blocks_per_sm < 1) return cudaErrorInvalidConfiguration;
  }
  if (a.nwork == 0) return cudaSuccess;
  int grid = blocks_per_sm * nsm;
  if (grid > a.nwork) grid = a.nwork;
  k<<<grid, kNT, KF32::bytes, s>>>(a);
  return cudaGetLastError();
}

}  // namespace emma
