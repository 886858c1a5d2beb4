// level_fp64.cu -- plain-path instantiation of the level kernel.  Built with
// -fmad=false so that FP64 expressions round exactly as the reference's CPU
// build (gcc, no FMA contraction) does.
#include "level_kernel.cuh"

namespace emma {

cudaError_t launch_level_fp64(const BatchArgs &a, unsigned shapes, int nsm, int ctas_per_sm, cudaStream_t s,
                              int *occupancy) {
  return launch_level_any<MathF64>(a, shapes, nsm, ctas_per_sm, s, occupancy);
}

}  // namespace emma
