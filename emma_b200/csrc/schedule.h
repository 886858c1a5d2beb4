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
  unsigned ticket[2];                   // work queue of the level kernel: next item, CTAs done
                                        // (the last CTA of a launch puts both back to 0)
};

// Control block of the fused coarse step (step_kernel.cuh), zeroed before each
// launch: the grid-wide job barrier, the job in progress and the schedule's
// position in Advance_level's recursion.
struct StepCtl {
  unsigned epoch;    // jobs published so far
  unsigned arrived;  // CTAs done with the current job
  unsigned ticket;   // next work item of the current job
  int kind, L, n, shape;  // the current job: kind, level, work items, brick shape
  int pc, pcL;       // schedule position (pc 0: start of the coarse step) and its level
  int pad[7];
};
enum : int { kJobNone = 0, kJobLevel = 1, kJobCfl = 2, kJobDone = 3 };

// Arguments of a fused coarse step.
struct StepArgs {
  LevelArgs *lv;
  SchedState *S;
  StepCtl *ctl;
  unsigned *done;       // scratch for the tiles' completion counts
  unsigned *status;
  long long wait_limit;  // bounded spin of a CTA waiting for the next job
  int lfine;             // finest level with octs
  struct StepJobRecord *jobt;  // optional: kStepJobLog records of the jobs' releases
};
// One released job of a fused coarse step: the device times (ns, %globaltimer) at
// which every CTA had reached the barrier before it and at its release (the
// schedule ran in between), its kind and level.
struct StepJobRecord {
  unsigned long long t_all, t;
  int kind, L;
};
constexpr unsigned kStepJobLog = 256;

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
