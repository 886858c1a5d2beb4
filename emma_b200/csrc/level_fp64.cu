// level_fp64.cu -- plain-path instantiation of the level kernel.  Built with
// -fmad=false so that FP64 expressions round exactly as the reference's CPU
// build (gcc, no FMA contraction) does.
#include "level_kernel.cuh"

namespace emma {

using KF64 = LevelSmem<MathF64, kTileOcts, kSMax, kHMax, kBMax>;

size_t level_smem_fp64() { return KF64::bytes; }

cudaError_t launch_level_fp64(const LevelArgs &a, cudaStream_t s) {
  static bool attr = false;
  auto k = level_advance_kernel<MathF64, kTileOcts, kSMax, kHMax, kBMax>;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)KF64::bytes);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  if (a.ntiles == 0) return cudaSuccess;
  k<<<a.ntiles, 8 * kTileOcts, KF64::bytes, s>>>(a);
  return cudaGetLastError();
}

}  // namespace emma
