// step_kernel.cuh -- one coarse step of a subcycled tree in one launch.
//
// The reference advances the levels from the host (Advance_level,
// src/advanceamr.c:243-1299): per level iteration the CFL step, the dt logic,
// the recursion into the finer level, HydroSolver, the bookkeeping.  The level
// schedule of this library (schedule.cu) runs that logic in single-thread
// kernels between the level launches of a CUDA graph: about seven launches per
// level iteration, half of them gated off.  Here one persistent kernel runs the
// whole recursion: its CTAs process a sequence of jobs (a level iteration's
// tiles, or a CFL reduction of a level whose state was set from the host) with
// a grid-wide barrier between jobs.  CTA 0 leads: once every CTA has reached the
// barrier it runs the schedule up to the next job (the same steps, in the same
// order and with the same IEEE operations, as k_sub_begin / k_sub_dt /
// k_sub_prelaunch / k_sub_end / k_sub_final) and releases the others.  Only
// the leader writes the schedule state and the level slots during the launch.
// Its threads copy both from L2 (the signal-speed maxima the other CTAs
// accumulated with atomics included) into CTA 0's tile region, idle between
// jobs; one thread runs the schedule on that copy and all write it back before
// the release, so the schedule's many dependent reads cost shared-memory
// latency instead of an L2 round trip each.
//
// Tiles of a level job are taken from a ticket queue by tile groups: a CTA holds
// as many groups of kThreads threads as the shared memory of the job's brick
// shape allows (its own region and named barrier each), so each shape runs at
// the occupancy of its own level kernel although every level of the tree goes
// through one kernel.  The corrections a level receives from its finer level
// are cleared by the update that reads them (BatchArgs::zero_c), so no buffer is
// cleared between jobs.
//
// Every wait is bounded: a CTA that waits longer than wait_limit polls for the
// next job sets EMMA_ST_TIMEOUT and leaves; the others then time out too.
#pragma once
#include "level_kernel.cuh"
#include "schedule.h"

namespace emma {

constexpr size_t kStepDynMax = 227 * 1024;  // dynamic shared memory of one CTA
constexpr size_t kStepCtlBytes = 64;        // per-CTA control words after the slot tables
constexpr size_t kStepRegion0 = kTabBytes + kStepCtlBytes;

template <class M, class G, bool DUAL, int NTR>
__host__ __device__ constexpr size_t step_region_bytes() {
  return TileSmem<M, G, DUAL, NTR>::bytes - kTabBytes;
}
template <class M, class G, bool DUAL, int NTR>
__host__ __device__ constexpr int step_groups_fit() {
  const size_t n = (kStepDynMax - kStepRegion0) / step_region_bytes<M, G, DUAL, NTR>();
  return n > 4 ? 4 : (int)n;
}
// Tile groups per CTA: at most as many 4x4x2-brick tiles as fit; a kernel with NG
// groups runs its 2x2x2 jobs on as many of them as their larger regions allow.
// More groups hide more latency, fewer leave each thread more registers (the CTA's
// 64 K registers are shared by NG x kThreads threads).
template <class M, bool DUAL, int NTR>
constexpr int kStepGroups = step_groups_fit<M, GeomA, DUAL, NTR>();
template <class M, bool DUAL, int NTR, int NG>
constexpr int kStepGroupsB = step_groups_fit<M, GeomB, DUAL, NTR>() < NG ? step_groups_fit<M, GeomB, DUAL, NTR>() : NG;
template <class M, bool DUAL, int NTR, int NG>
__host__ __device__ constexpr size_t step_smem_bytes() {
  const size_t a = NG * step_region_bytes<M, GeomA, DUAL, NTR>();
  const size_t b = kStepGroupsB<M, DUAL, NTR, NG> * step_region_bytes<M, GeomB, DUAL, NTR>();
  return kStepRegion0 + (a > b ? a : b);
}

// ------------------------------------------------------------------ schedule
// The dt arithmetic of schedule.cu with explicit IEEE operations (this unit may be
// built with FMA contraction).  S and lv: the leader's shared-memory copy.
using VS = SchedState;
using VLA = LevelArgs;
__device__ __forceinline__ double step_smax(VS *S, int L) {
  return __longlong_as_double((long long)(S->fresh[L] ? S->smax_next[L] : S->smax[L]));
}
// L_comptstep_hydro's final step (src/advanceamr.c:135): dt = CFL dx / (3 Smax)
__device__ __forceinline__ double step_cfl_dt(VS *S, int L) {
  double dt = 1e9;
  const double smax = step_smax(S, L);
  if (smax > 0.) dt = fmin(__ddiv_rn(__dmul_rn(S->dx[L], S->cfl), __dmul_rn(smax, 3.)), dt);
  return dt;
}
// dt of an iteration (src/advanceamr.c:708-830)
__device__ __forceinline__ void step_sub_dt(VS *S, int L) {
  const int lc = S->lcoarse;
  double *adt = S->adt;
  double dtnew = S->dt_param;
  const double rem = __dsub_rn(S->time_max, S->tloc[L]);
  dtnew = (rem < dtnew ? rem : dtnew);
  const double dthydro = step_cfl_dt(S, L);
  dtnew = (dthydro < dtnew ? dthydro : dtnew);
  adt[L - 1] = dtnew;
  if (L == lc) adt[L - 2] = adt[L - 1];
  if (adt[L - 2] < adt[L - 1]) adt[L - 1] = adt[L - 2];
  else adt[L - 1] = fmin(adt[L - 1], __dsub_rn(adt[L - 2], S->dtacc[L]));
}
// after the finer level returned (src/advanceamr.c:843-858): bind the level job
__device__ __forceinline__ void step_prelaunch(VS *S, VLA *lv, int L, bool has_fine) {
  const int lc = S->lcoarse, lm = S->lmax;
  if (has_fine) {
    S->adt[L - 1] = S->dtacc[L + 1];
    if (L == lc) S->adt[L - 2] = S->adt[L - 1];
  }
  VLA &a = lv[L];
  a.dt = S->adt[L - 1];
  a.Wc = (L > lc && lv[L - 1].noct > 0) ? lv[L - 1].W : nullptr;
  a.Cc = (L > lc && lv[L - 1].noct > 0) ? lv[L - 1].C : nullptr;
  a.Wf = (L < lm && lv[L + 1].noct > 0) ? lv[L + 1].W : nullptr;
  a.wait_slot = -1;
  S->smax_next[L] = 0ULL;  // the job accumulates the new maximum
}
// bookkeeping of an iteration (src/advanceamr.c:1278-1281)
__device__ __forceinline__ void step_sub_end(VS *S, VLA *lv, int L) {
  double *t = lv[L].W;
  lv[L].W = lv[L].Wn;
  lv[L].Wn = t;
  S->dtacc[L] = __dadd_rn(S->dtacc[L], S->adt[L - 1]);
  S->tloc[L] = __dadd_rn(S->tloc[L], S->adt[L - 1]);
  S->is[L]++;
  S->updates += lv[L].leaf;
  S->fresh[L] = 1;
  S->stale[L] = 0;
  S->azall[L] = 1;
}

enum : int { kPcStart = 0, kPcEnter, kPcIter, kPcDt, kPcEnd, kPcReturn };

// Runs Advance_level's recursion from the saved position to the next job and
// writes it into the control block (one thread; S and lv: the copy in shared
// memory).
static __device__ __noinline__ void step_schedule(VS *S, VLA *lv, StepCtl *c, int lf) {
  const int lc = S->lcoarse;
  int pc = c->pc, L = c->pcL;
  if (pc == kPcStart) {
    pc = kPcEnter;
    L = lc;
  }
  for (int guard = 0; guard < 64 * kMaxLevels; guard++) {
    if (pc == kPcEnter) {  // Advance_level(L) called
      S->dtacc[L] = 0.;
      S->is[L] = 0;
      S->tloc[L] = (L == lc) ? S->tsim : S->tloc[L - 1];
      S->active[L] = 1;
      pc = kPcIter;
    } else if (pc == kPcIter) {  // top of an iteration: the loop condition, the CFL step
      if (S->is[L] > 0 && !((S->dtacc[L] < S->adt[L - 2]) && (S->is[L] < S->nsub))) {
        S->active[L] = 0;
        pc = kPcReturn;
        continue;
      }
      S->smax[L] = 0ULL;
      pc = kPcDt;
      if (S->stale[L]) {  // the state was set from the host: a CFL reduction first
        c->kind = kJobCfl;
        c->L = L;
        c->n = 0;
        c->shape = 0;
        c->pc = pc;
        c->pcL = L;
        return;
      }
    } else if (pc == kPcDt) {
      step_sub_dt(S, L);
      if (L < lf) {
        L++;
        pc = kPcEnter;
        continue;
      }
      step_prelaunch(S, lv, L, false);
      c->kind = kJobLevel;
      c->L = L;
      c->n = lv[L].ntiles;
      c->shape = lv[L].shape;
      c->pc = kPcEnd;
      c->pcL = L;
      return;
    } else if (pc == kPcEnd) {
      step_sub_end(S, lv, L);
      pc = kPcIter;
    } else {  // kPcReturn: Advance_level(L) returns dtacc[L]
      if (L == lc) {
        S->tsim = __dadd_rn(S->tsim, S->adt[lc - 1]);
        c->kind = kJobDone;
        c->pc = kPcStart;
        c->pcL = 0;
        return;
      }
      L--;
      step_prelaunch(S, lv, L, true);
      c->kind = kJobLevel;
      c->L = L;
      c->n = lv[L].ntiles;
      c->shape = lv[L].shape;
      c->pc = kPcEnd;
      c->pcL = L;
      return;
    }
  }
  c->kind = kJobDone;  // unreachable with a consistent tree: stop rather than spin
}

// ------------------------------------------------------------------ kernel
template <class M, bool DUAL, int NTR, int NG>
__global__ void __launch_bounds__(NG * kThreads, 1) step_kernel(const StepArgs P) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int NGB = kStepGroupsB<M, DUAL, NTR, NG>;
  static_assert(NG >= 1 && NG <= kStepGroups<M, DUAL, NTR> && NGB >= 1, "a tile of each shape fits");
  // the leader's copy of the schedule state and the level slots (8-byte words)
  constexpr int kMirS = (int)(sizeof(SchedState) / 8), kMirL = (int)(kMaxLevels * sizeof(LevelArgs) / 8);
  static_assert(sizeof(SchedState) % 8 == 0 && sizeof(LevelArgs) % 8 == 0 && kStepRegion0 % 16 == 0, "8-byte words");
  static_assert(8 * (kMirS + kMirL) <= step_region_bytes<M, GeomA, DUAL, NTR>() &&
                    8 * (kMirS + kMirL) <= step_region_bytes<M, GeomB, DUAL, NTR>(),
                "the copy fits in one tile region");
  slot_tables<GeomA>(smem);
  slot_tables<GeomB>(smem + kTabOffB);
  unsigned long long *sSmax = reinterpret_cast<unsigned long long *>(smem + kSmaxOff);
  // control words: the job, two tickets per group, the CTA's CFL maximum
  volatile int *sJob = reinterpret_cast<volatile int *>(smem + kTabBytes);          // kind, L, n, shape, abort
  volatile int *sTicket = reinterpret_cast<volatile int *>(smem + kTabBytes + 20);  // [2][4]
  unsigned long long *sCfl = reinterpret_cast<unsigned long long *>(smem + kTabBytes + 56);
  if (threadIdx.x < kMaxLevels) sSmax[threadIdx.x] = 0ULL;
  if (threadIdx.x == 0) *sCfl = 0ULL;
  const int grp = tile_group(), gtid = threadIdx.x % kThreads;
  StepCtl *ctl = P.ctl;
  BatchArgs Bt{};  // what the level tiles read
  Bt.lv = P.lv;
  Bt.done = P.done;
  Bt.status = P.status;
  Bt.wait_limit = P.wait_limit;
  Bt.smax = P.S->smax_next;
  Bt.zero_c = 1;
  unsigned st = 0;
  unsigned seen = 0;  // jobs this CTA has taken
  int kind = kJobNone, L = 0;
  unsigned long long t_all = 0;  // the leader's job log: when every CTA had arrived
  for (;;) {
    // ---- the end of a job (or the start): flush, arrive, wait for the next job
    __syncthreads();
    if (threadIdx.x == 0) {
      if (kind == kJobLevel && sSmax[L] != 0ULL) {
        atomicMax(P.S->smax_next + L, sSmax[L]);
        sSmax[L] = 0ULL;
      }
      if (kind == kJobCfl && *sCfl != 0ULL) {
        atomicMax(P.S->smax + L, *sCfl);
        *sCfl = 0ULL;
      }
      __threadfence();
      atomicAdd(&ctl->arrived, 1u);
    }
    if (blockIdx.x == 0) {
      // the leader: once every CTA is done with the job (thread 0 waits), the
      // schedule to the next on a shared-memory copy of its state (block-uniform)
      if (threadIdx.x == 0) {
        int abort = 0;
        long long it = 0;
        while (*reinterpret_cast<volatile unsigned *>(&ctl->arrived) < gridDim.x) {
          if (++it > P.wait_limit) {
            abort = 1;
            break;
          }
          __nanosleep(32);
        }
        if (!abort) {
          if (P.jobt != nullptr) asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_all));
          __threadfence();
          ctl->arrived = 0u;
        }
        sJob[4] = abort;
      }
      __syncthreads();
      if (!sJob[4]) {
        unsigned long long *mir = reinterpret_cast<unsigned long long *>(smem + kStepRegion0);
        const unsigned long long *gS = reinterpret_cast<const unsigned long long *>(P.S);
        const unsigned long long *gL = reinterpret_cast<const unsigned long long *>(P.lv);
        for (int i = threadIdx.x; i < kMirS + kMirL; i += blockDim.x)
          mir[i] = i < kMirS ? __ldcg(gS + i) : __ldcg(gL + (i - kMirS));
        __syncthreads();
        if (threadIdx.x == 0) step_schedule(reinterpret_cast<VS *>(mir), reinterpret_cast<VLA *>(mir + kMirS), ctl,
                                            P.lfine);
        __syncthreads();
        unsigned long long *wS = reinterpret_cast<unsigned long long *>(P.S);
        unsigned long long *wL = reinterpret_cast<unsigned long long *>(P.lv);
        for (int i = threadIdx.x; i < kMirS + kMirL; i += blockDim.x) {
          if (i < kMirS) wS[i] = mir[i];
          else wL[i - kMirS] = mir[i];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
          // every group starts on two items of its own (below); the queue hands out the rest
          ctl->ticket = 2u * gridDim.x * (ctl->shape == 0 ? NG : NGB);
          if (P.jobt != nullptr && seen < kStepJobLog) {  // device time of the release
            unsigned long long t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            P.jobt[seen].t_all = t_all;
            P.jobt[seen].t = t;
            P.jobt[seen].kind = ctl->kind;
            P.jobt[seen].L = ctl->L;
          }
          __threadfence();  // the copy written back by every thread (ordered by the barrier) first
          atomicExch(&ctl->epoch, seen + 1);
        }
      }
    }
    if (threadIdx.x == 0) {
      int abort = (blockIdx.x == 0) ? sJob[4] : 0;
      long long it = 0;
      while (!abort && *reinterpret_cast<volatile unsigned *>(&ctl->epoch) == seen) {
        if (++it > P.wait_limit) {
          abort = 1;
          break;
        }
        __nanosleep(64);
      }
      __threadfence();
      const volatile StepCtl *vc = ctl;
      sJob[0] = abort ? kJobDone : vc->kind;
      sJob[1] = vc->L;
      sJob[2] = vc->n;
      sJob[3] = vc->shape;
      sJob[4] = abort;
    }
    __syncthreads();
    seen++;
    kind = sJob[0];
    L = sJob[1];
    const int n = sJob[2], shape = sJob[3];
    if (sJob[4]) st |= kStTimeout;
    if (kind == kJobDone) break;
    if (kind == kJobCfl) {
      // L_comptstep_hydro's maximum (src/advanceamr.c:122-128), every thread of the grid
      const LevelArgs *a = P.lv + L;
      const double *W = reinterpret_cast<const double *>(__ldcg(reinterpret_cast<const unsigned long long *>(&a->W)));
      const long long n8 = 8LL * __ldcg(&a->noct);
      double m = 0.;
      for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n8;
           i += (long long)gridDim.x * blockDim.x) {
        const double d = __ldcg(W + i), u = __ldcg(W + n8 + i), v = __ldcg(W + 2 * n8 + i),
                     w = __ldcg(W + 3 * n8 + i), p = __ldcg(W + 4 * n8 + i);
        const double va = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v)), __dmul_rn(w, w)));
        const double aa = __dsqrt_rn(__ddiv_rn(__dmul_rn(5. / 3., p), d));
        m = fmax(m, __dadd_rn(va, aa));  // fmax drops NaN like the reference's FMAX
      }
      for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
      // non-negative doubles order like their bit patterns
      if ((threadIdx.x & 31) == 0 && m > 0.) atomicMax(sCfl, (unsigned long long)__double_as_longlong(m));
      continue;
    }
    // ---- a level job: tiles from the queue, one per group at a time
    const int ngroups = (shape == 0) ? NG : NGB;
    if (grp >= ngroups) continue;
    const size_t rb =
        (shape == 0) ? step_region_bytes<M, GeomA, DUAL, NTR>() : step_region_bytes<M, GeomB, DUAL, NTR>();
    unsigned char *smem_g = smem + kStepRegion0 + grp * rb - kTabBytes;  // TileSmem offsets start at kTabBytes
    int cur = 0, args_slot = -1;
    bool have = false;
    // the group holds the tickets of its tile and of the next and asks for the one
    // after while it works (as the level kernel's queue); its first two items are
    // its own, so no atomic stands between the job's release and its first tile
    volatile int *gT = sTicket + 2 * grp;
    const int nworkers = gridDim.x * ngroups;
    int t = blockIdx.x * ngroups + grp, tn = t + nworkers;
    while (t < n) {
      unsigned tnn = 0u;
      if (gtid == 0) tnn = atomicAdd(&ctl->ticket, 1u);  // read after the tile
      const int next = (tn < n) ? tn : -1;
      if (shape == 0)
        level_tile<M, GeomA, false, DUAL, NTR, true>(Bt, P.lv + L, L, t, next, smem_g, smem, sSmax, st, cur, have,
                                                     args_slot);
      else
        level_tile<M, GeomB, false, DUAL, NTR, true>(Bt, P.lv + L, L, t, next, smem_g, smem + kTabOffB, sSmax, st,
                                                     cur, have, args_slot);
      if (gtid == 0) gT[0] = (int)tnn;  // every thread of the group read gT before the tile's barriers
      tile_sync<true>();
      t = tn;
      tn = gT[0];
    }
  }
  if (st) atomicOr(P.status, st);
}

}  // namespace emma

namespace emma {
namespace {  // internal linkage: each library keeps its own occupancy cache

template <class M, bool DUAL, int NTR, int NG>
cudaError_t launch_step_v(const StepArgs &a, int nsm, cudaStream_t s, int *grid_out, int *threads_out) {
  constexpr int kMaxDev = 64;
  static int occ_dev[kMaxDev] = {0};  // the shared-memory limit is a per-device attribute
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDev) return cudaErrorInvalidDevice;
  int &occ = occ_dev[dev];
  auto k = step_kernel<M, DUAL, NTR, NG>;
  constexpr size_t bytes = step_smem_bytes<M, DUAL, NTR, NG>();
  constexpr int threads = NG * kThreads;
  static_assert(bytes <= kStepDynMax, "the tile regions fit one CTA");
  if (occ == 0) {
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    int o = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k, threads, bytes);
    if (e != cudaSuccess) return e;
    if (o < 1) return cudaErrorInvalidConfiguration;
    occ = o;
  }
  // every CTA co-resident: the job barrier waits for all of them
  const int grid = occ * nsm;
  if (grid_out != nullptr) *grid_out = grid;
  if (threads_out != nullptr) *threads_out = threads;
  k<<<grid, threads, bytes, s>>>(a);
  return cudaGetLastError();
}

template <class M, bool DUAL, int NTR>
cudaError_t launch_step_g(const StepArgs &a, int groups, int nsm, cudaStream_t s, int *grid_out, int *threads_out) {
  constexpr int G = kStepGroups<M, DUAL, NTR>;
  if (groups <= 0 || groups >= G) return launch_step_v<M, DUAL, NTR, G>(a, nsm, s, grid_out, threads_out);
  if constexpr (G > 2) {  // fewer groups, more registers a thread
    if (groups == G - 1) return launch_step_v<M, DUAL, NTR, G - 1>(a, nsm, s, grid_out, threads_out);
  }
  if constexpr (G > 3) {
    if (groups == G - 2) return launch_step_v<M, DUAL, NTR, G - 2>(a, nsm, s, grid_out, threads_out);
  }
  return cudaErrorInvalidValue;
}

// the tile groups a launch with `groups` requested runs with (0: as many as fit), or
// 0 where that count is not built
template <class M>
int step_groups_any(unsigned variant, int groups) {
  int G = 0;
  switch (variant) {
    case 0u: G = kStepGroups<M, false, 0>; break;
    case kLaunchDual: G = kStepGroups<M, true, 0>; break;
    case kLaunchTracer: G = kStepGroups<M, false, 1>; break;
    case kLaunchHelium: G = kStepGroups<M, false, 3>; break;
    default: return 0;
  }
  if (groups <= 0 || groups >= G) return G;
  if (variant == 0u && ((G > 2 && groups == G - 1) || (G > 3 && groups == G - 2))) return groups;
  return 0;
}

// variant: 0, kLaunchDual, kLaunchTracer or kLaunchHelium; groups: tile groups per
// CTA (0: as many as fit; the plain variant also has the two next smaller counts)
template <class M>
cudaError_t launch_step_any(const StepArgs &a, unsigned variant, int groups, int nsm, cudaStream_t s, int *grid_out,
                            int *threads_out) {
  switch (variant) {
    case 0u: return launch_step_g<M, false, 0>(a, groups, nsm, s, grid_out, threads_out);
    case kLaunchDual: return launch_step_v<M, true, 0, kStepGroups<M, true, 0>>(a, nsm, s, grid_out, threads_out);
    case kLaunchTracer: return launch_step_v<M, false, 1, kStepGroups<M, false, 1>>(a, nsm, s, grid_out, threads_out);
    case kLaunchHelium: return launch_step_v<M, false, 3, kStepGroups<M, false, 3>>(a, nsm, s, grid_out, threads_out);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace
}  // namespace emma
