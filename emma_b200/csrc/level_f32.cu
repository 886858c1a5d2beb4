// level_f32.cu -- mixed-path instantiation of the level kernel: FP32
// reconstruction, wave speeds and fluxes; FP64 compensated update.
#include "level_kernel.cuh"

namespace emma {

// shapes: bit i = kShapes[i] used by a level of the work list, plus kLaunchGrav
// for the gravity-coupled variant; occupancy (optional) receives the CTAs per SM
// the kernel fits.
cudaError_t launch_level_f32(const BatchArgs &a, unsigned shapes, int nsm, int ctas_per_sm, cudaStream_t s,
                             int *occupancy) {
  return launch_level_any<MathF32>(a, shapes, nsm, ctas_per_sm, s, occupancy);
}

}  // namespace emma
