// level_fp64.cu -- plain-path instantiation of the level kernel.  Built with
// -fmad=false so that FP64 expressions round exactly as the reference's CPU
// build (gcc, no FMA contraction) does.
#include "level_kernel.cuh"
#include "step_kernel.cuh"

namespace emma {

cudaError_t launch_level_fp64(const BatchArgs &a, unsigned shapes, int nsm, int ctas_per_sm, cudaStream_t s,
                              int *occupancy) {
  return launch_level_any<MathF64>(a, shapes, nsm, ctas_per_sm, s, occupancy);
}

int step_groups_fp64(unsigned variant, int groups) { return step_groups_any<MathF64>(variant, groups); }

cudaError_t launch_step_fp64(const StepArgs &a, unsigned variant, int groups, int nsm, cudaStream_t s, int *grid,
                             int *threads) {
  return launch_step_any<MathF64>(a, variant, groups, nsm, s, grid, threads);
}

}  // namespace emma
