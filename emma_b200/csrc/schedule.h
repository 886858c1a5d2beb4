// schedule.h -- device state of the level schedule (see schedule.cu).
#pragma once
#include "plan_types.h"

namespace emma {

struct SchedState {
  double tsim, dt_param, time_max, cfl;
  double adt[kMaxLevels];               // the reference's adt array, index level-1
  double dx[kMaxLevels];                // cell size per level
  unsigned long long smax[kMaxLevels];  // max signal speed per level from the CFL reduction kernel
                                        // (bits of a non-negative double)
  unsigned long long smax_next[kMaxLevels];  // the same, accumulated by the level kernel over the
                                             // state it writes
  int fresh[kMaxLevels];                // smax_next holds the max of the level's current state
  int stale[kMaxLevels];                // !fresh: the state was set from the host (smax is then
                                        // zeroed with it, for the reduction kernel)
  int cfl_gate[kMaxLevels];             // subcycled iteration: active and stale
  int azall[kMaxLevels];                // the level was updated since its state was set: every
                                        // split cell holds the averaged state (sound speed 0)
  double dtacc[kMaxLevels];             // dt accumulated by the current Advance_level(L) call
  double tloc[kMaxLevels];              // its local time
  int is[kMaxLevels];                   // its iteration count
  int active[kMaxLevels];               // gate of the current iteration of level L
  long long updates;                    // cell-updates performed (leaf cells x substeps)
  int lcoarse, lmax, nsub;
  int gate_all;
};

__global__ void k_set_args(LevelArgs *lv, int slot, LevelArgs a);
__global__ void k_bind_level(LevelArgs *lv, int L, int lcoarse, int lmax, double dt);
__global__ void k_swap_level(LevelArgs *lv, int L, const int *gate);
__global__ void k_clear(double *p, long long n, const int *gate);
__global__ void k_batch_begin(SchedState *S, LevelArgs *lv, unsigned *done);
__global__ void k_batch_end(SchedState *S, LevelArgs *lv);
__global__ void k_sub_begin(SchedState *S, int L, int it);
__global__ void k_sub_dt(SchedState *S, int L);
__global__ void k_sub_prelaunch(SchedState *S, LevelArgs *lv, int L, int has_fine);
__global__ void k_sub_end(SchedState *S, LevelArgs *lv, int L);
__global__ void k_sub_final(SchedState *S);

}  // namespace emma
