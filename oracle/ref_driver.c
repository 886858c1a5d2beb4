/*
 * ref_driver.c -- test harness around the reference's OWN CPU hydro.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is compiled together with the
 * reference's unmodified sources (src/hydro_utils.c, oct.c, amr.c, segment.c,
 * hilbert.c, advanceamr.c for L_comptstep_hydro) into oracle/_ref/*.so by
 * oracle/Makefile.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference arm load it, always as the checker or the timed CPU
 * baseline, never as part of the product path.
 *
 * What it does (all single rank, rank 0):
 *  - builds the initial uniform oct tree with the reference's
 *    build_initial_grid (src/amr.c:1507) and links the free-oct list like
 *    main() does (src/emma.c:763-771);
 *  - refines marked cells with the reference's L_refine_cells (src/amr.c:286)
 *    to build static AMR trees;
 *  - sets primitive fields (computing a and E as the reference's ICs do);
 *  - runs the hydro-only subset of Advance_level (src/advanceamr.c:243-1299:
 *    clean_new_hydro :423, dt selection :708-830, finer-first recursion
 *    :843-858, HydroSolver :989, bookkeeping :1278-1290) with the
 *    reference's clean_new_hydro, L_comptstep_hydro and HydroSolver;
 *  - exports tree topology and fields per level in the `next` list order.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include "prototypes.h"
#include "amr.h"
#include "oct.h"
#include "hydro_utils.h"
#include "segment.h"
#include "restart.h"

/* defined in src/advanceamr.c:92 (compiled through ref_advanceamr_cfl.c) */
REAL L_comptstep_hydro(int level, struct RUNPARAMS *param, struct OCT **firstoct,
                       REAL fa, REAL fa2, struct CPUINFO *cpu, REAL tmax);

static struct OCT *g_grid = NULL;
static struct OCT **g_first = NULL, **g_last = NULL;
static struct CPUINFO g_cpu;
static struct RUNPARAMS g_param;
static struct HGRID *g_stencil = NULL;
static struct CELL g_root;
static REAL *g_adt = NULL;
static int *g_ndt = NULL;
static int g_ngridmax = 0, g_levelmax = 0;
static double g_hydro_seconds = 0.0;   /* wall time inside HydroSolver */
static long long g_cell_updates = 0;   /* leaf cells x level substeps */

/* ---------------------------------------------------------------- utils */
static double now_s(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

static void recount(void) {
  int l;
  for (l = 1; l <= g_levelmax; l++) {
    int n = 0;
    struct OCT *o = g_first[l - 1];
    while (o != NULL) { n++; o = o->next; }
    g_cpu.noct[l - 1] = n;
    g_cpu.locNoct[l - 1] = n;
  }
}

void ref_free(void) {
  int l;
  if (g_grid == NULL) return;
  for (l = 0; l < g_levelmax; l++) free(g_cpu.octList[l]);
  free(g_cpu.octList); free(g_cpu.locNoct); free(g_cpu.noct);
  free(g_cpu.allkmin); free(g_cpu.allkmax); free(g_cpu.bndoct); free(g_cpu.htable);
  free(g_first); free(g_last); free(g_stencil); free(g_adt); free(g_ndt);
  free(g_grid);
  g_grid = NULL;
}

/* Build the uniform tree of levels 1..lcoarse (src/emma.c:459-771 subset). */
int ref_init(int lcoarse, int lmax, int ngridmax, int hstride) {
  int l;
  struct OCT *freeoct, *cur;
  ref_free();
  memset(&g_cpu, 0, sizeof(g_cpu));
  memset(&g_param, 0, sizeof(g_param));
  g_levelmax = lmax;
  g_ngridmax = ngridmax;
  g_param.lcoarse = lcoarse;
  g_param.lmax = lmax;
  g_param.ngridmax = ngridmax;
  g_param.hstride = hstride;
  g_param.nsubcycles = 2;
  g_param.dt = 1e9;
  g_param.time_max = 1e9;
  g_param.tmax = 1e9;
  g_cpu.rank = 0;
  g_cpu.nproc = 1;
  g_cpu.levelcoarse = lcoarse;
  g_grid = (struct OCT *)calloc((size_t)ngridmax, sizeof(struct OCT));
  if (g_grid == NULL) return -1;
  g_first = (struct OCT **)calloc((size_t)lmax, sizeof(struct OCT *));
  g_last = (struct OCT **)calloc((size_t)lmax, sizeof(struct OCT *));
  g_cpu.noct = (int *)calloc((size_t)lmax, sizeof(int));
  g_cpu.locNoct = (int *)calloc((size_t)lmax, sizeof(int));
  g_cpu.octList = (struct OCT ***)calloc((size_t)lmax, sizeof(struct OCT **));
  for (l = 0; l < lmax; l++) g_cpu.octList[l] = (struct OCT **)calloc((size_t)ngridmax, sizeof(struct OCT *));
  g_cpu.allkmin = (int *)calloc(1, sizeof(int));
  g_cpu.allkmax = (int *)calloc(1, sizeof(int));
  g_cpu.nbuff = g_cpu.nbufforg = 1;
  g_cpu.bndoct = (struct OCT **)calloc(1, sizeof(struct OCT *));
  g_cpu.maxhash = 1;
  g_cpu.htable = (struct OCT **)calloc(1, sizeof(struct OCT *));
  load_balance(lcoarse, &g_cpu);
  g_cpu.allkmin[0] = (int)g_cpu.kmin;
  g_cpu.allkmax[0] = (int)g_cpu.kmax;

  g_root = build_initial_grid(g_grid, g_first, g_last, &g_cpu, &g_param);

  /* free-oct chain, src/emma.c:765-771 */
  freeoct = g_last[lcoarse - 1] + 1;
  freeoct->prev = NULL;
  freeoct->next = freeoct + 1;
  for (cur = freeoct + 1; cur < g_grid + ngridmax; cur++) {
    cur->prev = cur - 1;
    cur->next = NULL;
    if (cur != g_grid + ngridmax - 1) cur->next = cur + 1;
  }
  g_cpu.freeoct = freeoct;

  /* single rank: every oct below the root belongs to rank 0 */
  for (l = 2; l <= lmax; l++) {
    struct OCT *o = g_first[l - 1];
    while (o != NULL) { o->cpu = 0; o = o->next; }
  }
  recount();
  for (l = 1; l <= lmax; l++) setOctList(g_first[l - 1], &g_cpu, &g_param, l);

  g_stencil = (struct HGRID *)calloc((size_t)(hstride < 8 ? 8 : hstride), sizeof(struct HGRID));
  g_param.hstride = (hstride < 8 ? 8 : hstride);
  g_adt = (REAL *)malloc(sizeof(REAL) * (size_t)lmax);
  g_ndt = (int *)calloc((size_t)lmax, sizeof(int));
  for (l = 1; l <= lmax; l++) g_adt[l - 1] = g_param.dt;
  g_hydro_seconds = 0.0;
  g_cell_updates = 0;
  return 0;
}

int ref_noct(int level) { return g_cpu.noct[level - 1]; }
int ref_sizeof_oct(void) { return (int)sizeof(struct OCT); }
int ref_sizeof_hgrid(void) { return (int)sizeof(struct HGRID); }
void *ref_grid_base(void) { return (void *)g_grid; }
void *ref_firstoct_array(void) { return (void *)g_first; }

/* Refine the level-`level` cells whose mark is non-zero (mark[oct*8+icell] in
 * list order) with the reference's L_refine_cells.  Cells that are already split
 * keep marked=1 so that the reference does not destroy them (src/amr.c:339). */
int ref_refine(int level, const signed char *mark) {
  int i = 0, icell;
  struct OCT *o = g_first[level - 1];
  struct OCT *limit = g_grid + g_ngridmax;
  while (o != NULL) {
    for (icell = 0; icell < 8; icell++) {
      int m = mark[i * 8 + icell] != 0 || o->cell[icell].child != NULL;
      o->cell[icell].marked = m ? 1. : 0.;
    }
    i++;
    o = o->next;
  }
  g_cpu.freeoct = L_refine_cells(level, &g_param, g_first, g_last, g_cpu.freeoct, &g_cpu, limit, 1.0);
  o = g_first[level];
  while (o != NULL) { o->cpu = 0; o = o->next; }
  for (o = g_first[level - 1]; o != NULL; o = o->next)
    for (icell = 0; icell < 8; icell++) o->cell[icell].marked = 0.;
  recount();
  return g_cpu.noct[level];
}

/* oct lower-left corners, list order */
void ref_oct_xyz(int level, double *xyz) {
  int i = 0;
  struct OCT *o;
  for (o = g_first[level - 1]; o != NULL; o = o->next, i++) {
    xyz[3 * i + 0] = o->x; xyz[3 * i + 1] = o->y; xyz[3 * i + 2] = o->z;
  }
}

/* index of an oct within its level list (linear scan cache rebuilt per call) */
static int *g_idx = NULL;
static void build_index(void) {
  int l;
  free(g_idx);
  g_idx = (int *)malloc(sizeof(int) * (size_t)g_ngridmax);
  memset(g_idx, 0xff, sizeof(int) * (size_t)g_ngridmax);
  for (l = 1; l <= g_levelmax; l++) {
    int i = 0;
    struct OCT *o;
    for (o = g_first[l - 1]; o != NULL; o = o->next) g_idx[o - g_grid] = i++;
  }
}
static int cell_code(struct CELL *c) {
  /* (oct index in its level)*8 + cell index, or -1 */
  struct OCT *o;
  if (c == NULL) return -1;
  o = cell2oct(c);
  if (o < g_grid || o >= g_grid + g_ngridmax) return -2;  /* the root stand-in cell */
  return g_idx[o - g_grid] * 8 + c->idx;
}

/* Topology of one level, list order:
 *   nei[6*i+k]   = cell code (level-1 list) of oct->nei[k]
 *   parent[i]    = cell code (level-1 list) of oct->parent
 *   child[8*i+c] = index (level+1 list) of cell c's child oct, -1 if leaf
 *   lev[i]       = oct->level, cpu[i] = oct->cpu                            */
void ref_topology(int level, int *nei, int *parent, int *child, int *lev) {
  int i = 0, k;
  struct OCT *o;
  build_index();
  for (o = g_first[level - 1]; o != NULL; o = o->next, i++) {
    for (k = 0; k < 6; k++) nei[6 * i + k] = cell_code(o->nei[k]);
    parent[i] = cell_code(o->parent);
    for (k = 0; k < 8; k++) child[8 * i + k] = o->cell[k].child ? g_idx[o->cell[k].child - g_grid] : -1;
    lev[i] = o->level;
  }
}

/* Set field and fieldnew of every cell of a level from primitive arrays
 * (list order, oct*8+icell); a and E computed with the reference's own
 * formulas (getE, src/hydro_utils.c:29; a as in U2W, :64). */
void ref_set_field(int level, const double *d, const double *u, const double *v,
                   const double *w, const double *p) {
  int i = 0, c;
  struct OCT *o;
  for (o = g_first[level - 1]; o != NULL; o = o->next, i++) {
    for (c = 0; c < 8; c++) {
      struct Wtype *W = &o->cell[c].field;
      int k = i * 8 + c;
      W->d = d[k]; W->u = u[k]; W->v = v[k]; W->w = w[k]; W->p = p[k];
      W->a = SQRT(GAMMA * W->p / W->d);
      getE(W);
      memcpy(&o->cell[c].fieldnew, W, sizeof(struct Wtype));
    }
  }
}

#ifdef WGRAV
/* Set the gravitational acceleration f[3] of every cell of a level (list order). */
void ref_set_force(int level, const double *fx, const double *fy, const double *fz) {
  int i = 0, c;
  struct OCT *o;
  for (o = g_first[level - 1]; o != NULL; o = o->next, i++)
    for (c = 0; c < 8; c++) {
      o->cell[c].f[0] = fx[8 * i + c];
      o->cell[c].f[1] = fy[8 * i + c];
      o->cell[c].f[2] = fz[8 * i + c];
    }
}
#endif

#ifdef WRADHYD
/* Set the ionised density dX of field and fieldnew of every cell of a level
 * (list order), and read it back from field (which=0) or fieldnew (which=1). */
void ref_set_tracer(int level, const double *dX) {
  int i = 0, c;
  struct OCT *o;
  for (o = g_first[level - 1]; o != NULL; o = o->next, i++)
    for (c = 0; c < 8; c++) {
      o->cell[c].field.dX = dX[8 * i + c];
      o->cell[c].fieldnew.dX = dX[8 * i + c];
    }
}
void ref_get_tracer(int level, int which, double *out) {
  int i = 0, c;
  struct OCT *o;
  for (o = g_first[level - 1]; o != NULL; o = o->next, i++)
    for (c = 0; c < 8; c++) out[8 * i + c] = which ? o->cell[c].fieldnew.dX : o->cell[c].field.dX;
}
/* Tracer t (0: dX; with -DHELIUM 1: dXHE, 2: dXXHE, the members that follow dX in
 * struct Wtype, src/prototypes.h:620-625) of field and fieldnew. */
#ifdef HELIUM
#define REF_NTR 3
#else
#define REF_NTR 1
#endif
int ref_ntracers(void) { return REF_NTR; }
void ref_set_tracer_n(int level, int t, const double *x) {
  int i = 0, c;
  struct OCT *o;
  if (t < 0 || t >= REF_NTR) return;
  for (o = g_first[level - 1]; o != NULL; o = o->next, i++)
    for (c = 0; c < 8; c++) {
      (&o->cell[c].field.dX)[t] = x[8 * i + c];
      (&o->cell[c].fieldnew.dX)[t] = x[8 * i + c];
    }
}
void ref_get_tracer_n(int level, int t, int which, double *out) {
  int i = 0, c;
  struct OCT *o;
  if (t < 0 || t >= REF_NTR) return;
  for (o = g_first[level - 1]; o != NULL; o = o->next, i++)
    for (c = 0; c < 8; c++) out[8 * i + c] = which ? (&o->cell[c].fieldnew.dX)[t] : (&o->cell[c].field.dX)[t];
}
#endif

/* Checkpoints through the reference's own src/restart.c (save_amr / restore_amr),
 * units from `units7` (unit_l, _v, _t, _n, _mass, _d, _N), no particles. */
void ref_save_amr(const char *filename, double tsim, double tinit, int nsteps, int ndumps, const double *units7) {
  g_param.unit.unit_l = units7[0]; g_param.unit.unit_v = units7[1]; g_param.unit.unit_t = units7[2];
  g_param.unit.unit_n = units7[3]; g_param.unit.unit_mass = units7[4]; g_param.unit.unit_d = units7[5];
  g_param.unit.unit_N = units7[6];
  save_amr((char *)filename, g_first, tsim, tinit, nsteps, ndumps, &g_param, &g_cpu, NULL, g_adt);
}
void ref_restore_amr(const char *filename, double *tsim, double *tinit, int *nsteps, int *ndumps) {
  g_cpu.freeoct = restore_amr((char *)filename, g_first, g_last, tsim, tinit, nsteps, ndumps, &g_param, &g_cpu,
                              NULL, g_adt, &g_root);
  recount();
}
void *ref_lastoct_array(void) { return g_last; }
void *ref_root_cell(void) { return &g_root; }
void *ref_freeoct(void) { return g_cpu.freeoct; }
void ref_set_freeoct(void *f) { g_cpu.freeoct = (struct OCT *)f; recount(); }
int ref_ngridmax(void) { return g_ngridmax; }

/* Export d,u,v,w,p,a,E of field (which=0) or fieldnew (which=1) as 7 planes. */
void ref_get_field(int level, int which, double *out) {
  int n = g_cpu.noct[level - 1] * 8, i = 0, c;
  struct OCT *o;
  for (o = g_first[level - 1]; o != NULL; o = o->next, i++) {
    for (c = 0; c < 8; c++) {
      struct Wtype *W = which ? &o->cell[c].fieldnew : &o->cell[c].field;
      int k = i * 8 + c;
      out[0 * n + k] = W->d; out[1 * n + k] = W->u; out[2 * n + k] = W->v;
      out[3 * n + k] = W->w; out[4 * n + k] = W->p; out[5 * n + k] = W->a;
      out[6 * n + k] = W->E;
    }
  }
}

/* ---------------------------------------------------- single entry points */
void ref_clean_new_hydro(int level) { clean_new_hydro(level, &g_param, g_first, &g_cpu); }
double ref_comptstep_hydro(int level) {
  return L_comptstep_hydro(level, &g_param, g_first, 1.0, 1.0, &g_cpu, 1e9);
}
static long long leaf_cells(int level) {
  long long n = 0;
  int c;
  struct OCT *o;
  for (o = g_first[level - 1]; o != NULL; o = o->next)
    for (c = 0; c < 8; c++) n += (o->cell[c].child == NULL);
  return n;
}
void ref_hydro_solver(int level, double dt) {
  double t0 = now_s();
  HydroSolver(level, &g_param, g_first, &g_cpu, g_stencil, g_param.hstride, dt);
  g_hydro_seconds += now_s() - t0;
  g_cell_updates += leaf_cells(level);
}

/* A bounded sample of one level step on a large level: clean_new_hydro and
 * HydroSolver run unmodified on the first `nsample` octs of the level list.
 * The list is cut after that oct for the duration of the calls (both walk
 * firstoct[level-1] through `next`, src/hydro_utils.c:3322-3366, 3410-3483,
 * 3501-3546) and relinked afterwards; the gather still reads every neighbour
 * through the tree's pointers, so each sampled oct does exactly the work of a
 * whole-level step.  Timed like ref_hydro_solver (HydroSolver only).  The CFL
 * step of the whole level is taken first (L_comptstep_hydro, untimed). */
double ref_hydro_solver_prefix(int level, int nsample) {
  struct OCT *o = g_first[level - 1], *cut;
  int i;
  double t0, dt;
  long long n = 0;
  if (o == NULL || nsample <= 0) return 0.;
  for (i = 1; i < nsample && o->next != NULL; i++) o = o->next;
  cut = o->next;
  dt = L_comptstep_hydro(level, &g_param, g_first, 1.0, 1.0, &g_cpu, 1e9);
  o->next = NULL;
  clean_new_hydro(level, &g_param, g_first, &g_cpu);
  t0 = now_s();
  HydroSolver(level, &g_param, g_first, &g_cpu, g_stencil, g_param.hstride, dt);
  g_hydro_seconds += now_s() - t0;
  n = leaf_cells(level);
  o->next = cut;
  g_cell_updates += n;
  return dt;
}

/* ------------------------------------------------ refinement (one level) */
/* The reference's refinement calls of Advance_level (src/advanceamr.c:348-373,
 * 1230-1241): L_clean_marks, L_mark_cells (the criterion of this build: see
 * ref_amr_sntest.c), L_check_rule and L_refine_cells, which takes new octs from
 * the free-oct chain and returns its new head. */
void ref_clean_marks(int level) { L_clean_marks(level, g_first); }
void ref_mark_cells(int level, int nsmooth, double threshold) {
  L_mark_cells(level, &g_param, g_first, nsmooth, threshold, &g_cpu, NULL, NULL);
}
void ref_check_rule(int level) { L_check_rule(level, &g_param, g_first, &g_cpu); }
void ref_refine_cells(int level) {
  g_cpu.freeoct = L_refine_cells(level, &g_param, g_first, g_last, g_cpu.freeoct, &g_cpu,
                                 g_grid + g_ngridmax, 1.0);
  recount();
}
/* marks of a level's cells in list order */
void ref_get_marks(int level, double *out) {
  int i = 0, c;
  struct OCT *o;
  for (o = g_first[level - 1]; o != NULL; o = o->next, i++)
    for (c = 0; c < 8; c++) out[8 * i + c] = o->cell[c].marked;
}

/* -------------------------------------- hydro-only Advance_level schedule */
static REAL advance_level(int level, REAL tloc) {
  REAL dt = 0., dtnew, dthydro, dtfine;
  int is = 0;
  int nsub = g_param.nsubcycles;
  REAL *adt = g_adt;
  do {
    clean_new_hydro(level, &g_param, g_first, &g_cpu);            /* :423 */
    dtnew = g_param.dt;                                            /* :709 */
    dtnew = ((g_param.time_max - tloc) < dtnew ? (g_param.time_max - tloc) : dtnew);
    dthydro = L_comptstep_hydro(level, &g_param, g_first, 1.0, 1.0, &g_cpu, 1e9);
    dtnew = (dthydro < dtnew ? dthydro : dtnew);                   /* :752 */
    adt[level - 1] = dtnew;                                        /* :808 */
    if (level == g_param.lcoarse) adt[level - 2] = adt[level - 1];
    if (adt[level - 2] < adt[level - 1]) {
      adt[level - 1] = adt[level - 2];
    } else {
      adt[level - 1] = FMIN(adt[level - 1], adt[level - 2] - dt);
    }
    if (level < g_param.lmax) {                                    /* :843 */
      if (g_cpu.noct[level] > 0) {
        dtfine = advance_level(level + 1, tloc);
        adt[level - 1] = dtfine;
        if (level == g_param.lcoarse) adt[level - 2] = adt[level - 1];
      }
    }
    ref_hydro_solver(level, adt[level - 1]);                       /* :989 */
#ifdef WGRAV
    grav_correction(level, &g_param, g_first, &g_cpu, adt[level - 1]); /* :999 */
#endif
    dt += adt[level - 1];                                          /* :1278 */
    tloc += adt[level - 1];
    is++;
    g_ndt[level - 1]++;
  } while ((dt < adt[level - 2]) && (is < nsub));                  /* :1290 */
  return dt;
}

/* Run `nsteps` coarse steps (main loop, src/emma.c:1701-1918); returns tsim.
 * steps_done receives the number of coarse steps taken. */
double ref_run(int nsteps, double dt_param, double time_max, int nsub, double tsim0, int *steps_done) {
  int n, l;
  double tsim = tsim0;
  g_param.dt = dt_param;
  g_param.time_max = time_max;
  g_param.nsubcycles = nsub;
  for (l = 1; l <= g_levelmax; l++) g_adt[l - 1] = g_param.dt;
  for (n = 0; n < nsteps && tsim < time_max; n++) {
    for (l = 1; l <= g_levelmax; l++) g_ndt[l - 1] = 0;
    advance_level(g_param.lcoarse, tsim);
    tsim += g_adt[g_param.lcoarse - 1];
  }
  if (steps_done) *steps_done = n;
  return tsim;
}

/* level dt array after a run (adt[level-1]) */
double ref_adt(int level) { return g_adt[level - 1]; }
int ref_ndt(int level) { return g_ndt[level - 1]; }
double ref_hydro_seconds(void) { return g_hydro_seconds; }
long long ref_cell_updates(void) { return g_cell_updates; }
void ref_reset_counters(void) { g_hydro_seconds = 0.0; g_cell_updates = 0; }

/* Stubs for symbols referenced by advanceamr.c / amr.c but never reached on
 * the hydro-only path driven here (I/O lives in src/io.c, which needs MPI). */
void dumpIO(REAL tsim, struct RUNPARAMS *param, struct CPUINFO *cpu, struct OCT **firstoct, REAL *adt, int pdump) {
  (void)tsim; (void)param; (void)cpu; (void)firstoct; (void)adt; (void)pdump;
  fprintf(stderr, "ref_driver: dumpIO is not part of the oracle\n");
  abort();
}

#ifdef WGRAV
/* -DWGRAV builds leave out src/tools.c, whose multicheck reads a member that
 * exists only with -DPIC; these stand in for the three functions of it that
 * other compiled files reference.  Only myradixsort is reached (the single-rank
 * neighbour list of setup_mpi, src/communication.c:232): ascending order. */
REAL multicheck(struct OCT **firstoct, int *npart, int levelcoarse, int levelmax, int rank, struct CPUINFO *cpu,
                struct RUNPARAMS *param, int label) {
  (void)firstoct; (void)npart; (void)levelcoarse; (void)levelmax; (void)rank; (void)cpu; (void)param; (void)label;
  return 0.;
}
void grid_census(struct RUNPARAMS *param, struct CPUINFO *cpu) { (void)param; (void)cpu; }
void myradixsort(int *a, int n) {
  int i, j;
  for (i = 1; i < n; i++) {
    int x = a[i];
    for (j = i - 1; j >= 0 && a[j] > x; j--) a[j + 1] = a[j];
    a[j + 1] = x;
  }
}
#endif
