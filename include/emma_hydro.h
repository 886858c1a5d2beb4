/*
 * emma_hydro.h -- C ABI of libemmahydro, a B200 (sm_100a) implementation of
 * EMMA's hydro level advance: oct-neighbour gather, MUSCL-Hancock
 * reconstruction, HLLC fluxes, flux-divergence update and scatter back to the
 * oct tree, for one AMR level or for a whole coarse step of levels.
 *
 * Two ways in:
 *  1. Drop-in entries with the reference's own names and signatures
 *     (src/hydro_utils.h:9-10, src/hydro_utils_gpu.h:1-5).  They read and write
 *     the caller's host oct tree (struct OCT, include/emma_oct.h) on every call,
 *     so they cost PCIe traffic, exactly like the reference's GPU twin.
 *  2. Resident entries (emma_hydro_*): upload the tree once, advance levels or
 *     whole coarse steps on the GPU, download only for I/O.  This is the
 *     performance path.
 *
 * Errors: the reference aborts on invalid states (src/hydro_utils.c:1212,1283,
 * 1298,3135) and ignores CUDA errors.  Here every entry records a bitmask
 * (EMMA_ST_*) readable with emma_hydro_status(); entries returning int return
 * that bitmask of the call (0 = success, negative = argument/setup error).
 * With EMMA_HYDRO_ABORT=1 in the environment the library aborts like the
 * reference instead.
 */
#ifndef EMMA_HYDRO_H
#define EMMA_HYDRO_H

#include <stdint.h>
#include "emma_oct.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define EMMA_ST_NEG_DENSITY 0x01  /* negative density in a face state   (src/hydro_utils.c:1212) */
#define EMMA_ST_NEG_PSTAR   0x02  /* negative star pressure             (src/hydro_utils.c:1283) */
#define EMMA_ST_NAN         0x04  /* NaN in a flux or an updated state  (src/hydro_utils.c:1302,3135) */
#define EMMA_ST_TREE        0x08  /* tree the device path cannot stage (missing neighbour, unsupported slot) */
#define EMMA_ST_CUDA        0x10  /* a CUDA call failed */
#define EMMA_ST_ARG         0x20  /* bad argument (level out of range, NULL pointer, no tree) */
#define EMMA_ST_TIMEOUT     0x40  /* a bounded device wait gave up */

int emma_hydro_status(void);        /* sticky bitmask since the last clear */
void emma_hydro_clear_status(void);
const char *emma_hydro_last_error(void); /* human-readable text of the last error */

/* ------------------------------------------------------------ options */
#define EMMA_PREC_FP64  0  /* plain path: FP64 everywhere, reference operation order */
#define EMMA_PREC_MIXED 1  /* FP32 reconstruction/Riemann/flux, FP64 compensated update */

/* transmissive boundaries (the reference's -DTRANSXM ... -DTRANSZP) */
#define EMMA_TRANS_XM 0x01
#define EMMA_TRANS_XP 0x02
#define EMMA_TRANS_YM 0x04
#define EMMA_TRANS_YP 0x08
#define EMMA_TRANS_ZM 0x10
#define EMMA_TRANS_ZP 0x20

struct EmmaHydroOptions {
  int precision;        /* EMMA_PREC_* */
  int trans_flags;      /* EMMA_TRANS_* */
  double cfl;           /* Courant number of the level time step (reference param.h: 0.85) */
  int tile_octs;        /* octs per brick: 0 = autotuned per level, 32 = 4x4x2, 8 = 2x2x2 */
  int device;           /* CUDA device ordinal */
  int use_graph;        /* coarse steps as a captured CUDA graph with a device-side schedule */
  int gravity;          /* gravity coupling of the reference's -DWGRAV build (resident mode):
                           half-step kick -f dt/2 of the MUSCL face velocities
                           (src/hydro_utils.c:1219-1226) and grav_correction after each
                           level update (src/hydro_utils.c:2388, called at
                           src/advanceamr.c:999); the accelerations f come from
                           emma_hydro_set_level_force.  Not with trans_flags. */
  int dual_energy;      /* the reference's -DDUAL_E build (its production default,
                           init/param_init.mk): the internal energy is tracked with its
                           flux and a p div(u) term, and the pressure comes from it unless
                           E - Ekin is resolved (src/hydro_utils.c:45-49, 2126-2129,
                           3164-3182).  Drop-in and resident modes. */
  int column;           /* mixed precision, resident complete periodic levels without split
                           cells (plain variant): 0 = the autotuner picks the column kernel
                           (16 x 16-cell columns marching through z) or the brick kernel,
                           -1 = brick kernel only, n > 0 = column kernel with n cell planes
                           per work item (even, dividing the level's cells per side) */
  int fused_step;       /* subcycled coarse steps of a resident tree on the CUDA graph: one
                           persistent kernel per coarse step that runs the whole level recursion
                           (plain, dual-energy and tracer trees without gravity or transmissive
                           boundaries, no level on the column kernel), or the level schedule as
                           separate launches.  0 = autotuned at the first graph step (each mode
                           timed over five coarse steps from a snapshot of the state, which is
                           then restored), -1 = separate launches, k > 0 = fused with k tile
                           groups per CTA (as many as fit if k is not built) */
  int column_xshfl;     /* x sweep of the column kernel: the faces inside a 16-cell row solved
                           from the left cell's face state passed up a lane by a warp shuffle
                           (1) or read from shared memory (-1); 0 = the faster of the two at
                           the autotuned depth (shared memory when `column` forces a depth) */
  int column_balanced;  /* work of the column kernel: two CTAs per SM, each an equal run of the
                           level's column-planes (1), or items of `nz` planes handed out by the
                           block scheduler (-1); 0 = the faster of the two (items when `column`
                           forces a depth) */
};
void emma_hydro_default_options(struct EmmaHydroOptions *opt);

/* ------------------------------------------- drop-in entries (reference names) */

/* HydroSolver (src/hydro_utils.h:9, src/hydro_utils.c:3378): advance every
 * level-`level` oct of rank cpu->rank by dtnew.  Writes fieldnew of the level's
 * leaf cells and of their unsplit coarser neighbours (fine->coarse flux
 * correction), then field := fieldnew on leaves and the primitive mean of the
 * children on split cells.  `param`, `stencil` and `stride` are accepted for
 * signature compatibility and not used. */
void HydroSolver(int level, struct RUNPARAMS *param, struct OCT **firstoct, struct CPUINFO *cpu,
                 struct HGRID *stencil, int stride, REAL dtnew);

/* advancehydroGPU (src/hydro_utils_gpu.h:1, src/hydro_utils_gpu.cu:2470): the
 * flux computation + scatter part of HydroSolver; returns the number of octs
 * advanced (0 leaves the caller's final field update out, as in the reference). */
int advancehydroGPU(struct OCT **firstoct, int level, struct CPUINFO *cpu, struct HGRID *stencil,
                    int stride, REAL dxcur, REAL dtnew);

/* clean_new_hydro (src/hydro_utils.h:10, src/hydro_utils.c:3501): fieldnew := field. */
void clean_new_hydro(int level, struct RUNPARAMS *param, struct OCT **firstoct, struct CPUINFO *cpu);

/* Lifecycle entries (src/hydro_utils_gpu.h:2-5, src/hydro_utils_gpu.cu:25-43).
 * create_hydstencil_GPU initialises the library's device context (the
 * reference stores a device stencil in cpu->hyd_stencil; this library keeps its
 * own context and leaves *cpu untouched).  create_pinned_stencil allocates the
 * caller's page-locked HGRID scratch of `stride` entries as the reference does. */
void create_hydstencil_GPU(struct CPUINFO *cpu, int stride);
void destroy_hydstencil_GPU(struct CPUINFO *cpu, int stride);
void create_pinned_stencil(struct HGRID **stencil, int stride);
void destroy_pinned_stencil(struct HGRID **stencil, int stride);

/* ---------------------------------------------------------- resident path */

/* Create the device context (idempotent).  NULL options = defaults. */
int emma_hydro_init(const struct EmmaHydroOptions *opt);
int emma_hydro_set_options(const struct EmmaHydroOptions *opt);
void emma_hydro_shutdown(void);
/* Launch on the caller's CUDA stream (a cudaStream_t; NULL = the library's own
 * stream).  Entries still synchronise the stream where they return host data. */
int emma_hydro_set_stream(void *stream);

/* Mirror levels lcoarse..lmax of the host tree (rank `rank`) onto the GPU:
 * per-level SoA state (d,u,v,w,p of `field`), topology and tile plans.
 * The tree structure must not change until the next upload. */
int emma_hydro_tree_upload(struct OCT **firstoct, int lcoarse, int lmax, int rank);
/* Copy the device state back into `field` and `fieldnew` of the host tree
 * (a and E recomputed as the reference stores them). */
int emma_hydro_tree_download(struct OCT **firstoct);
/* Release the resident tree uploaded from `firstoct` (no-op for another tree):
 * device buffers and the captured coarse step are freed, emma_hydro_is_resident
 * returns 0 afterwards.  emma_hydro_restore_amr calls it, since it overwrites
 * the pool the resident tree mirrors.  No reference counterpart. */
int emma_hydro_tree_release(struct OCT **firstoct);
/* ------------------------------------------ refinement of a resident tree
 * The reference's marking and refinement of one level (called by Advance_level,
 * src/advanceamr.c:348-373 and 1230-1241) on the tree uploaded from `firstoct`,
 * without moving its fields off the GPU.  Periodic trees of the plain variant
 * (EMMA_ST_ARG with transmissive boundaries, gravity, dual energy or the
 * -DWRADHYD library).  The marks of every resident cell live on the device
 * (uploaded from the cells' `marked`).
 *
 * emma_hydro_mark_cells: L_clean_marks + L_mark_cells (src/amr.c:1480, 883):
 * nsmooth rounds of (keep split cells whose children are marked or split; mark
 * the 3x3x3 neighbourhood of marked cells; in the first round only, mark cells
 * whose density exceeds `threshold` -- the criterion of the reference's
 * -DSNTEST build, src/amr.c:1330-1354, which fixes it at 1.1).
 * emma_hydro_check_rule: L_check_rule (src/amr.c:746): marks of octs whose 26
 * neighbours do not all exist become 10.
 * emma_hydro_marks_to_host: the device marks of a level into the cells' `marked`.
 * emma_hydro_refine_cells: L_refine_cells (src/amr.c:286), same signature and
 * return value (the new head of the free-oct chain; NULL and status bits on
 * failure, where the reference aborts): octs of level+1 are destroyed and created
 * in the host tree in the reference's order, from and onto the caller's free
 * chain; their device state is gathered on the device (new cells take the parent
 * cell's state, src/amr.c:512-520) and the resident mirror is re-planned.  The
 * caller still calls setOctList for level+1 as L_refine_cells does internally.
 * `param` supplies lcoarse (NULL: the resident tree's); aexp is unused. */
int emma_hydro_mark_cells(int level, struct RUNPARAMS *param, struct OCT **firstoct, int nsmooth, REAL threshold,
                          struct CPUINFO *cpu);
int emma_hydro_check_rule(int level, struct RUNPARAMS *param, struct OCT **firstoct, struct CPUINFO *cpu);
int emma_hydro_marks_to_host(struct OCT **firstoct, int level);
struct OCT *emma_hydro_refine_cells(int level, struct RUNPARAMS *param, struct OCT **firstoct, struct OCT **lastoct,
                                    struct OCT *freeoct, struct CPUINFO *cpu, struct OCT *limit, REAL aexp);
/* Re-read only the fields (same structure) / write only the fields. */
int emma_hydro_fields_upload(struct OCT **firstoct);

/* Level operations on the resident tree (reference counterparts in brackets). */
int emma_hydro_clean_new(int level);                      /* [clean_new_hydro] */
int emma_hydro_comptstep(int level, double *dt_out);      /* [L_comptstep_hydro, src/advanceamr.c:92] */
int emma_hydro_advance_level(int level, double dt);       /* [HydroSolver] */

/* One coarse step of the hydro-only level schedule (src/advanceamr.c:243-1299):
 * finer levels first, up to `nsub` subcycles, CFL time steps.  `adt` (lmax
 * entries, in/out) is the reference's per-level dt array; tsim is advanced. */
int emma_hydro_advance_coarse_step(double dt_param, double time_max, int nsub,
                                   double *tsim, double *adt);
/* The same, queued on the library's stream without waiting: time and dt stay
 * on the device (start from the last values set or returned).  Read them with
 * emma_hydro_get_time, which synchronises. */
int emma_hydro_advance_coarse_step_async(double dt_param, double time_max, int nsub);
int emma_hydro_get_time(double *tsim, double *adt);
int emma_hydro_set_time(double tsim, const double *adt);

/* 1 if a resident tree was uploaded from this firstoct array (and not freed since). */
int emma_hydro_is_resident(struct OCT **firstoct);

/* Checkpoints in the reference's raw-OCT restart format.  emma_hydro_save_amr
 * writes what save_amr (src/restart.c:12-103, -DWHYDRO2 build) writes: tsim,
 * tinit, nsteps, ndumps, lcoarse, lmax, adt[0..lmax-1], the 7 unit scales
 * (unit_l, unit_v, unit_t, unit_n, unit_mass, unit_d, unit_N), the addresses of
 * firstoct[0], of its cell 0 and `proot`, then each oct of levels 1..lmax in list
 * order as its address and its bytes; for a resident tree of the same firstoct
 * the device state is downloaded into the tree first.  emma_hydro_restore_amr
 * reads such a file back as restore_amr (src/restart.c:108-328) does: into the
 * caller's pool of ngridmax octs starting at firstoct[0] (octs at their snapshot
 * offset, pointers shifted, level-1 parents set to `root`), rebuilding firstoct
 * and lastoct (levelmax entries) and the free-oct chain (*freeoct). */
int emma_hydro_save_amr(const char *filename, struct OCT **firstoct, double tsim, double tinit, int nsteps,
                        int ndumps, int lcoarse, int lmax, const double *adt, const double *units7,
                        const void *proot);
int emma_hydro_restore_amr(const char *filename, struct OCT **firstoct, struct OCT **lastoct, int levelmax,
                           long long ngridmax, struct CELL *root, double *tsim, double *tinit, int *nsteps,
                           int *ndumps, int *lcoarse, int *lmax, double *adt, double *units7,
                           struct OCT **freeoct);

/* Field dump in the reference's ALLOCT format, dumpalloct_serial (src/io.c:1233).
 * One file per field i: <folder>grid_<names[i]>/<names[i]>.<ndumps %05d>.p<rank %05d>
 * (folder ends with '/'; the directory is created), holding int n_cell and seven
 * 4-byte words (the first 4 bytes of the double tsim, then xmin, xmax, ymin, ymax,
 * zmin, zmax of the dumped octs as floats), then one float per dumped cell: the
 * cells without a child (every cell at lmax) of the octs with cpu == rank, levels
 * lcoarse..lmax in list order.  ids are assign_grid_field's (src/io.c:32): 0-2
 * cell corner x,y,z, 3 level, 4 cpu, 12 marked, 13-17 field d,u,v,w,p; the
 * -DWGRAV library also 5 gdata.d, 7 gdata.p, 8 res, 9-11 f.  For a tree resident
 * on the GPU, ids 13-17 come from the device state (compacted to floats on the
 * GPU), the others from the host tree.  Returns 0, EMMA_ST_ARG (bad argument,
 * unknown id, file error), EMMA_ST_TREE (a resident tree whose host tree was
 * refined or coarsened since its upload: upload it again) or EMMA_ST_CUDA. */
int emma_hydro_dump_alloct(const char *folder, struct OCT **firstoct, int lcoarse, int lmax, int rank, int ndumps,
                           double tsim, int nfields, const int *ids, const char *const *names);

/* SoA access for tests and I/O: 5 planes (d,u,v,w,p) of 8*noct doubles each, list order. */
int emma_hydro_level_noct(int level);
int emma_hydro_get_level_state(int level, double *host_out);
int emma_hydro_set_level_state(int level, const double *host_in);
/* Gravity builds: the gravitational acceleration of the level's cells, 3 planes
 * (fx, fy, fz) of 8*noct doubles in list order, from host or device memory
 * (the reference's cell f[3], src/prototypes.h:841); zero after an upload. */
int emma_hydro_set_level_force(int level, const double *host_f);
int emma_hydro_set_level_force_device(int level, const double *dev_f);
/* Leaf cell count of a level (cells advanced per level substep). */
long long emma_hydro_level_leaf_cells(int level);
/* Cell-updates performed since the last reset (leaf cells x level substeps). */
long long emma_hydro_cell_updates(void);
/* Kernels of this library launched since the last reset. */
long long emma_hydro_kernel_launches(void);
/* Bytes of field state copied host->device and device->host by this library
 * since the last reset (drop-in entries, state set/get, tree fields upload and
 * download; not the one-off topology and plan uploads). */
int emma_hydro_transfer_bytes(long long *h2d, long long *d2h);
/* Host-side phases (ms) of the last advancehydroGPU / HydroSolver call:
 * [0] walk and hash of the level lists, [1] mirror build (0 when cached),
 * [2] pack + queue of the uploads, [3] kernel launch, download and unpack,
 * [4] mean wait of a host thread for its downloaded range, [5] fine->coarse
 * corrections, [6] rest of HydroSolver's final update, [7] the whole call. */
int emma_hydro_dropin_profile(double *ms8);
void emma_hydro_reset_counters(void);
/* Average device time (ms) of the level kernel launches since the last reset,
 * measured with CUDA events on the launching stream, and their count. */
int emma_hydro_kernel_timing(double *avg_ms, long long *launches, long long *cells);
/* The same for the single-level launches of one resident level (level -1: the
 * batched launches): total device time (ms), count and cell-updates. */
int emma_hydro_kernel_timing_level(int level, double *total_ms, long long *launches, long long *cells);

/* The coarse step captured on the CUDA graph (no reference counterpart): *fused = 1
 * when it is one persistent kernel running the whole level recursion
 * (EmmaHydroOptions.fused_step), with *ctas CTAs of *groups tile groups each (0
 * otherwise); *kernel_nodes = the kernel launches of one captured coarse step (0
 * before the first graph step). */
int emma_hydro_graph_info(int *fused, int *ctas, int *groups, int *kernel_nodes);
/* The coarse-step mode of the resident tree (no reference counterpart): *groups = 0
 * for the level schedule's separate launches, k > 0 for the fused kernel with k
 * tile groups per CTA, -2 before the first graph step; sweep_ms[5] = the
 * autotuner's device time of the fastest of four coarse steps of the separate
 * launches ([0]) and of the fused kernel with k groups ([k]), 0 where not timed. */
int emma_hydro_step_tuning(int *groups, double *sweep_ms);
/* The jobs of the last fused coarse step (no reference counterpart), after the
 * step has run: kinds (1 a level iteration's tiles, 2 a CFL reduction, 3 the end
 * of the step), levels, the device time in microseconds from the step's first
 * release to each job's release, and the time the schedule took before it (from
 * the last CTA's arrival to the release); up to max records, any pointer may be
 * NULL.  Returns the number of jobs, or a negative status. */
int emma_hydro_fused_job_log(int max, int *kinds, int *levels, double *release_us, double *schedule_us);
/* nsteps coarse steps queued as emma_hydro_advance_coarse_step_async does, with
 * their device time (ms, CUDA events on the library's stream) in *ms (no
 * reference counterpart). */
int emma_hydro_timed_coarse_steps(double dt_param, double time_max, int nsub, int nsteps, double *ms);

/* Column kernel of a resident level (no reference counterpart): *planes = the cell
 * planes per work item its launches use with the current options (0: the brick
 * kernel), sweep_ms[6] = the autotuner's ms per launch with 2, 4, 8, 16, 32, 64
 * planes per item (0 = not tried). */
int emma_hydro_column_tuning(int level, int *planes, double *sweep_ms);
/* The column kernel's x sweep on a resident level (no reference counterpart):
 * *xshfl = 1 when its launches pass the x face states by warp shuffle, 0 when
 * they read them from shared memory; ms[2] = the autotuner's ms per launch of the
 * shared-memory and the shuffle sweep at the chosen depth (0 = not timed). */
int emma_hydro_column_xshfl(int level, int *xshfl, double *ms);
/* The column kernel's work split on a resident level (no reference counterpart):
 * *balanced = 1 when its launches give every CTA (two per SM) an equal run of the
 * level's column-planes, 0 for items of the chosen depth; ms[2] = the autotuner's
 * ms per launch of the two (0 = not timed). */
int emma_hydro_column_balanced(int level, int *balanced, double *ms);
/* Autotuner record of a resident level (emma_hydro_tree_upload tunes every
 * level when options.tile_octs == 0): the chosen brick (32 = 4x4x2 octs, one
 * per tile; 8 = 2x2x2 octs, four per tile), the CTAs per SM of its launches,
 * and the measured ms per launch of every candidate, sweep_ms[4*shape + ctas-1]
 * (shape 0: 4x4x2, 1: 2x2x2; 0 = not tried).  Returns EMMA_ST_ARG if the level
 * was not tuned.  EMMA_HYDRO_AUTOTUNE=0 in the environment skips the timing pass
 * (shape from a tile-count cost model, CTAs at the occupancy limit). */
int emma_hydro_tuning(int level, int *tile_octs, int *ctas_per_sm, double *sweep_ms);

/* Diagnostics of the bounded device-side waits (a batched launch's update phase
 * waits for the finer level's tiles; every wait gives up after a bounded number
 * of polls and reports EMMA_ST_TIMEOUT instead of hanging).  Launches the
 * coarsest resident level once with its update waiting for a completion count
 * that no tile can reach, each wait bounded by `polls` (64 ns each), and returns
 * the status bits of that launch (EMMA_ST_TIMEOUT expected).  The resident state,
 * the sticky status and the completion counters are left as they were. */
int emma_hydro_probe_wait_timeout(long long polls);

/* Planning diagnostics, host only (no GPU needed): per level lcoarse..lmax,
 * stats5[5*(L-lcoarse)+{0..4}] = octs, tiles (4x4x2-oct bricks), max staged
 * octs per tile, staged octs summed over the tiles, leaf cells.  Returns
 * EMMA_ST_* bits of the planning. */
int emma_hydro_plan_stats(struct OCT **firstoct, int lcoarse, int lmax, int trans_flags, long long *stats5);

/* Level time step computed without allocating any memory.  No counterpart in
 * the reference.  For callers that cannot call cudaMalloc: a solver whose
 * device memory all belongs to a host code's pool, or a process that must not
 * allocate after start-up.  `d_state` is a level state ALREADY on the current
 * device, laid out like emma_hydro_get_level_state's (5 planes d,u,v,w,p of
 * `ncells` doubles); *dt_out receives what emma_hydro_comptstep returns for
 * that state at `level` with Courant number `cfl`.  Works on the current
 * device and needs neither emma_hydro_init nor a resident tree.
 * Scratch is a fixed 128 KiB array inside the library, held on every GPU that
 * loads it until exit, so ncells is limited to 33554432 (EMMA_ST_ARG beyond).
 * The first call on each device looks up the array's address (make it before
 * any stream capture).  Calls overlapping on the GPU share the array and race.
 * Runs on `stream` (a cudaStream_t, NULL = legacy default stream) and
 * synchronises it.  Returns EMMA_ST_* bits of this call only (it does not
 * touch emma_hydro_status). */
int emma_hydro_level_dt_noalloc(const double *d_state, long long ncells, int level, double cfl,
                                void *stream, double *dt_out);
/* Drops the device addresses of the fixed scratch that emma_hydro_level_dt_noalloc
 * cached per device.  Call it after a cudaDeviceReset (or any other teardown of a
 * device's primary context) and before the next emma_hydro_level_dt_noalloc call:
 * the reset unloads the library's module, so the cached address is stale.  No
 * counterpart in the reference. */
void emma_hydro_noalloc_forget(void);

/* --------------------------------------------------- host tree utilities */
/* Build an oct tree with the reference's construction order
 * (build_initial_grid src/amr.c:1507, L_refine_cells src/amr.c:286), for
 * callers (tests, benchmarks) that have no EMMA tree.  One tree at a time. */
struct EmmaTree;
struct EmmaTree *emma_tree_create(int lcoarse, int lmax, long long ngridmax);
void emma_tree_destroy(struct EmmaTree *t);
int emma_tree_refine(struct EmmaTree *t, int level, const signed char *mark);
struct OCT **emma_tree_firstoct(struct EmmaTree *t);
int emma_tree_noct(struct EmmaTree *t, int level);
void emma_tree_oct_xyz(struct EmmaTree *t, int level, double *xyz);
void emma_tree_set_field(struct EmmaTree *t, int level, const double *d, const double *u,
                         const double *v, const double *w, const double *p);
void emma_tree_get_field(struct EmmaTree *t, int level, int which, double *out7);
/* Inverse of emma_tree_get_field: writes d,u,v,w,p,a,E (planes of 8*noct) as
 * they are into `field` (which=0) or `fieldnew` (which=1). */
void emma_tree_put_field(struct EmmaTree *t, int level, int which, const double *in7);
/* Owner rank (struct OCT cpu) of every oct of the level, in list order: the
 * octs of other ranks are a multi-rank run's boundary octs. */
void emma_tree_set_cpu(struct EmmaTree *t, int level, const int *cpu);
void emma_tree_topology(struct EmmaTree *t, int level, int *nei, int *parent, int *child, int *lev);

#ifdef __cplusplus
}
#endif
#endif
