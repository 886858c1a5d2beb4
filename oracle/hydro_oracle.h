/*
 * hydro_oracle.h -- CPU restatement of EMMA's hydro level advance.
 *
 * TEST INFRASTRUCTURE ONLY (the checker).  Only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline / reference arm may load liboracle.so.  The
 * product library (libemmahydro.so) never links or calls it.
 *
 * The restatement works in place on an oct tree laid out like the reference's
 * `struct OCT` built with -DWHYDRO2 -DRIEMANN_HLLC -DPRIMITIVE, REAL=double,
 * NVAR=6 (src/prototypes.h:611,825,1028): 1200 bytes per oct.  It is pinned
 * bit-for-bit against the reference compiled from its own sources
 * (oracle/_ref, see oracle/Makefile and tests/test_oracle_pin.py).
 */
#ifndef EMMA_HYDRO_ORACLE_H
#define EMMA_HYDRO_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* boundary / gather variant flags (compile-time -D switches in the reference) */
#define ORC_TRANSXM 0x01   /* -DTRANSXM: transmissive at x=0 */
#define ORC_TRANSXP 0x02   /* -DTRANSXP: transmissive at x=1 */
#define ORC_TRANSYM 0x04
#define ORC_TRANSYP 0x08
#define ORC_TRANSZM 0x10
#define ORC_TRANSZP 0x20
#define ORC_HYDROTEST 0x40 /* -DHYDROTEST gather (src/hydro_utils.c:2464-2845) */
#define ORC_DUAL_E 0x80    /* -DDUAL_E: tracked internal energy (src/hydro_utils.c:45-49, 2126-2129, 3167-3180) */

/* error bits returned by the entry points (the reference aborts instead) */
#define ORC_ERR_NEG_DENSITY 0x01   /* src/hydro_utils.c:1212 */
#define ORC_ERR_NEG_PSTAR   0x02   /* src/hydro_utils.c:1283 */
#define ORC_ERR_SLSR        0x04   /* src/hydro_utils.c:1298 */
#define ORC_ERR_NAN         0x08   /* src/hydro_utils.c:1302, 2006, 3135 */
#define ORC_ERR_TREE        0x10   /* missing neighbour (reference dereferences NULL) */

/* firstoct[level-1] is the first oct of each level's `next` list. */
int orc_hydro_solver(void **firstoct, int level, double dt, int flags);
void orc_clean_new_hydro(void **firstoct, int level);
double orc_comptstep_hydro(void **firstoct, int level, double cfl);
/* Built with -DORC_WGRAV (liboracle_grav.so): the tree carries the -DWGRAV cell
 * layout (192-byte CELL with the force f[3]), the MUSCL face states get the
 * half-step gravity kick and the schedule calls grav_correction after each
 * HydroSolver (src/advanceamr.c:999). */
int orc_grav_correction(void **firstoct, int level, double dt);
/* Gravity build: copy of a default-layout tree (levels 1..lmax, pointers
 * remapped, forces zero) in the -DWGRAV layout; NULL if a pointer leads out of
 * the tree.  orc_grav_first gives its firstoct array. */
void *orc_grav_clone(void **src_firstoct, int lmax);
void **orc_grav_first(void *clone);
void orc_grav_set_force(void *clone, int level, const double *fx, const double *fy, const double *fz);
void orc_grav_get_field(void *clone, int level, int which, double *out);
void orc_grav_free(void *clone);
/* Hydro-only Advance_level schedule; returns tsim after `nsteps` coarse steps.
 * adt has lmax entries (in/out), like the reference's adt array. */
double orc_run(void **firstoct, int lcoarse, int lmax, int nsteps, double dt_param,
               double time_max, int nsub, double cfl, int flags, double tsim0,
               double *adt, int *steps_done, int *err);
long long orc_cell_updates(void);
void orc_reset_counters(void);
int orc_sizeof_oct(void);

/* ALLOCT field dump, dumpalloct_serial (src/io.c:1233): see hydro_oracle.c */
int orc_dump_alloct(const char *folder, void **firstoct, int lcoarse, int lmax, int rank, int ndumps, double tsim,
                    int nfields, const int *ids, const char *const *names);

#ifdef __cplusplus
}
#endif
#endif
