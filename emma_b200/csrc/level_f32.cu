// level_f32.cu -- mixed-path instantiation of the level kernel: FP32
// reconstruction, wave speeds and fluxes; FP64 compensated update.
#include "level_kernel.cuh"
#include "column_kernel.cuh"
#include "step_kernel.cuh"

namespace emma {

// shapes: bit i = kShapes[i] used by a level of the work list, plus kLaunchGrav
// for the gravity-coupled variant; occupancy (optional) receives the CTAs per SM
// the kernel fits.
cudaError_t launch_level_f32(const BatchArgs &a, unsigned shapes, int nsm, int ctas_per_sm, cudaStream_t s,
                             int *occupancy) {
  return launch_level_any<MathF32>(a, shapes, nsm, ctas_per_sm, s, occupancy);
}

// One fused coarse step of a subcycled tree (step_kernel.cuh).
cudaError_t launch_step_f32(const StepArgs &a, unsigned variant, int groups, int nsm, cudaStream_t s, int *grid,
                            int *threads) {
  return launch_step_any<MathF32>(a, variant, groups, nsm, s, grid, threads);
}

int step_groups_f32(unsigned variant, int groups) { return step_groups_any<MathF32>(variant, groups); }

// Column kernel of a complete periodic level (mixed path), two CTAs per SM; the
// shared-memory or the warp-shuffle x sweep (ColumnArgs::xshfl).
cudaError_t launch_column_f32(const ColumnArgs &a, cudaStream_t s) {
  constexpr int kMaxDev = 64;
  static bool attr_set[kMaxDev] = {false};  // the shared-memory limit is a per-device attribute
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDev) return cudaErrorInvalidDevice;
  if (!attr_set[dev]) {
    e = cudaFuncSetAttribute(column_kernel<2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)col::kSmem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(column_kernel<2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)col::kSmem);
    if (e != cudaSuccess) return e;
    attr_set[dev] = true;
  }
  if (a.nitems <= 0) return cudaSuccess;
  if (a.xshfl)
    column_kernel<2, true><<<a.nitems, col::kColThreads, col::kSmem, s>>>(a);
  else
    column_kernel<2, false><<<a.nitems, col::kColThreads, col::kSmem, s>>>(a);
  return cudaGetLastError();
}

}  // namespace emma
