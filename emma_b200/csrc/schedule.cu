// schedule.cu -- device side of the level schedule.
//
// The reference drives the level cycle from the host (Advance_level,
// src/advanceamr.c:243-1299): per level substep it computes the CFL time step,
// syncs it with the parent level, recurses into the finer level and calls
// HydroSolver.  Here that bookkeeping runs in single-thread kernels on the
// device, so that a whole coarse step (CFL reductions, dt logic, level kernels,
// buffer swaps) is a fixed sequence of launches that a CUDA graph captures once
// and replays with no host round trip.  A substep that the reference would not
// execute (the subcycle loop ended early) is a launch whose gate flag is 0.
//
// Built with -fmad=false: the dt arithmetic must round as the reference's does.
#include <cuda_runtime.h>
#include <stdint.h>
#include "plan_types.h"
#include "schedule.h"

namespace emma {

// The level's max signal speed: accumulated by the level kernel that wrote the
// current state, or, when the state was set from the host, from the CFL
// reduction kernel.  Both evaluate |v| + sqrt(gamma p / rho) with the same
// IEEE operations, so the dt is the same either way.
__device__ __forceinline__ double smax_of(const SchedState *S, int L) {
  return __longlong_as_double((long long)(S->fresh[L] ? S->smax_next[L] : S->smax[L]));
}

// L_comptstep_hydro's final step (src/advanceamr.c:135): dt = CFL dx / (3 Smax)
__device__ __forceinline__ double cfl_dt(const SchedState *S, int L) {
  double dt = 1e9;
  const double smax = smax_of(S, L);
  const double dxcur = S->dx[L];
  if (smax > 0.) dt = fmin(dxcur * S->cfl / (smax * 3.), dt);
  return dt;
}

// ---------------------------------------------------------------- host-driven
__global__ void k_set_args(LevelArgs *lv, int slot, LevelArgs a) { lv[slot] = a; }

// Bind one level for a sequential launch: dt, current coarser/finer states.
__global__ void k_bind_level(LevelArgs *lv, int L, int lcoarse, int lmax, double dt) {
  LevelArgs &a = lv[L];
  a.dt = dt;
  a.Wc = (L > lcoarse && lv[L - 1].noct > 0) ? lv[L - 1].W : nullptr;
  a.Cc = (L > lcoarse && lv[L - 1].noct > 0) ? lv[L - 1].C : nullptr;
  a.Wf = (L < lmax && lv[L + 1].noct > 0) ? lv[L + 1].W : nullptr;
  a.wait_slot = -1;
}

__global__ void k_swap_level(LevelArgs *lv, int L, const int *gate) {
  if (gate != nullptr && *gate == 0) return;
  double *t = lv[L].W;
  lv[L].W = lv[L].Wn;
  lv[L].Wn = t;
}

__global__ void k_clear(double *p, long long n, const int *gate) {
  if (gate != nullptr && *gate == 0) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = 0.;
}

// ------------------------------------------------------- batched (one dt for all)
// With a single substep per level (nsub == 1) the reference advances every
// level by the same dt: the smallest CFL step over the levels (the coarse dt is
// overwritten by the finer level's, src/advanceamr.c:808-858).  All levels then
// go through one launch, finest first, each level's update waiting for the finer
// level's (corrections, new state for split-cell averaging).
__global__ void k_batch_begin(SchedState *S, LevelArgs *lv, unsigned *done) {
  const int lc = S->lcoarse, lm = S->lmax;
  double *adt = S->adt;
  const double tloc = S->tsim;
  for (int L = lc; L <= lm; L++) {
    if (lv[L].noct == 0) break;
    double dtnew = S->dt_param;
    dtnew = ((S->time_max - tloc) < dtnew ? (S->time_max - tloc) : dtnew);
    const double dthydro = cfl_dt(S, L);
    dtnew = (dthydro < dtnew ? dthydro : dtnew);
    adt[L - 1] = dtnew;
    if (L == lc) adt[L - 2] = adt[L - 1];
    if (adt[L - 2] < adt[L - 1]) adt[L - 1] = adt[L - 2];
    else adt[L - 1] = fmin(adt[L - 1], adt[L - 2] - 0.);
  }
  for (int L = lc; L <= lm; L++) S->smax_next[L] = 0ULL;  // the launch accumulates the new maxima
  int lf = lc;
  while (lf < lm && lv[lf + 1].noct > 0) lf++;
  const double dtf = adt[lf - 1];
  for (int L = lf - 1; L >= lc; L--) {
    adt[L - 1] = dtf;  // dtfine returned by the finer level
    if (L == lc) adt[L - 2] = adt[L - 1];
  }
  for (int L = lc; L <= lf; L++) {
    LevelArgs &a = lv[L];
    a.dt = adt[L - 1];
    a.Wc = (L > lc) ? lv[L - 1].W : nullptr;
    a.Cc = (L > lc) ? lv[L - 1].C : nullptr;
    a.Wf = (L < lf) ? lv[L + 1].Wn : nullptr;  // the finer level's new state
    a.wait_slot = (L < lf) ? L + 1 : -1;
    done[L] = 0;
  }
  S->gate_all = 1;
}

__global__ void k_batch_end(SchedState *S, LevelArgs *lv) {
  const int lc = S->lcoarse, lm = S->lmax;
  for (int L = lc; L <= lm; L++) {
    if (lv[L].noct == 0) break;
    double *t = lv[L].W;
    lv[L].W = lv[L].Wn;
    lv[L].Wn = t;
    lv[L].wait_slot = -1;
    S->updates += lv[L].leaf;
    S->fresh[L] = 1;
    S->stale[L] = 0;
    S->azall[L] = 1;
  }
  S->tsim += S->adt[lc - 1];
}

// ------------------------------------------------ subcycled (Advance_level)
// One loop iteration `it` of Advance_level(L): the gate of this iteration.
__global__ void k_sub_begin(SchedState *S, int L, int it) {
  const int lc = S->lcoarse;
  if (it == 0) {
    S->active[L] = (L == lc) ? 1 : S->active[L - 1];
    S->dtacc[L] = 0.;
    S->is[L] = 0;
    S->tloc[L] = (L == lc) ? S->tsim : S->tloc[L - 1];
  } else {
    S->active[L] = S->active[L] && (S->dtacc[L] < S->adt[L - 2]) && (S->is[L] < S->nsub);
  }
  S->smax[L] = 0ULL;
  S->cfl_gate[L] = S->active[L] && S->stale[L];
}

// dt of the iteration (src/advanceamr.c:708-830)
__global__ void k_sub_dt(SchedState *S, int L) {
  if (!S->active[L]) return;
  const int lc = S->lcoarse;
  double *adt = S->adt;
  const double tloc = S->tloc[L];
  double dtnew = S->dt_param;
  dtnew = ((S->time_max - tloc) < dtnew ? (S->time_max - tloc) : dtnew);
  const double dthydro = cfl_dt(S, L);
  dtnew = (dthydro < dtnew ? dthydro : dtnew);
  adt[L - 1] = dtnew;
  if (L == lc) adt[L - 2] = adt[L - 1];
  if (adt[L - 2] < adt[L - 1]) adt[L - 1] = adt[L - 2];
  else adt[L - 1] = fmin(adt[L - 1], adt[L - 2] - S->dtacc[L]);
}

// after the finer level returned (src/advanceamr.c:843-858), bind the launch
__global__ void k_sub_prelaunch(SchedState *S, LevelArgs *lv, int L, int has_fine) {
  if (!S->active[L]) return;
  const int lc = S->lcoarse, lm = S->lmax;
  if (has_fine) {
    S->adt[L - 1] = S->dtacc[L + 1];
    if (L == lc) S->adt[L - 2] = S->adt[L - 1];
  }
  LevelArgs &a = lv[L];
  a.dt = S->adt[L - 1];
  a.Wc = (L > lc && lv[L - 1].noct > 0) ? lv[L - 1].W : nullptr;
  a.Cc = (L > lc && lv[L - 1].noct > 0) ? lv[L - 1].C : nullptr;
  a.Wf = (L < lm && lv[L + 1].noct > 0) ? lv[L + 1].W : nullptr;
  a.wait_slot = -1;
  S->smax_next[L] = 0ULL;  // the launch accumulates the new maximum
}

// bookkeeping of the iteration (src/advanceamr.c:1278-1281)
__global__ void k_sub_end(SchedState *S, LevelArgs *lv, int L) {
  if (!S->active[L]) return;
  double *t = lv[L].W;
  lv[L].W = lv[L].Wn;
  lv[L].Wn = t;
  S->dtacc[L] += S->adt[L - 1];
  S->tloc[L] += S->adt[L - 1];
  S->is[L]++;
  S->updates += lv[L].leaf;
  S->fresh[L] = 1;
  S->stale[L] = 0;
  S->azall[L] = 1;
}

__global__ void k_sub_final(SchedState *S) { S->tsim += S->adt[S->lcoarse - 1]; }

}  // namespace emma
