// level_f32.cu -- mixed-path instantiation of the level kernel: FP32
// reconstruction, wave speeds and fluxes; FP64 compensated update.
#include "level_kernel.cuh"

namespace emma {

using KF32 = LevelSmem<MathF32, kTileOcts, kSMax, kHMax, kBMax>;

size_t level_smem_f32() { return KF32::bytes; }

cudaError_t launch_level_f32(const LevelArgs &a, cudaStream_t s) {
  static bool attr = false;
  auto k = level_advance_kernel<MathF32, kTileOcts, kSMax, kHMax, kBMax>;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)KF32::bytes);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  if (a.ntiles == 0) return cudaSuccess;
  k<<<a.ntiles, 8 * kTileOcts, KF32::bytes, s>>>(a);
  return cudaGetLastError();
}

}  // namespace emma
