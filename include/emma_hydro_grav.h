/*
 * emma_hydro_grav.h -- entries of libemmahydro_grav.so only: the library built
 * for the reference's -DWGRAV cell layout (compile the caller with
 * -DEMMA_WGRAV so that include/emma_oct.h declares the 192-byte CELL with the
 * force f[3]).  That library also exports everything in emma_hydro.h; its
 * drop-in HydroSolver / advancehydroGPU run the gravity-coupled advance of the
 * reference's -DWGRAV build (force kick of the MUSCL face states, forces of
 * coarser neighbours spread by coarse2fine_forcelin).
 */
#ifndef EMMA_HYDRO_GRAV_H
#define EMMA_HYDRO_GRAV_H

#ifndef EMMA_WGRAV
#error "emma_hydro_grav.h needs -DEMMA_WGRAV (the -DWGRAV cell layout)"
#endif

#include "emma_hydro.h"

#ifdef __cplusplus
extern "C" {
#endif

/* grav_correction (src/hydro_utils.h:7, src/hydro_utils.c:2388-2444, PRIMITIVE):
 * after HydroSolver, every leaf cell of rank cpu->rank gets u += -f dt (and v,
 * w), then E; called by the reference's Advance_level at src/advanceamr.c:999. */
void grav_correction(int level, struct RUNPARAMS *param, struct OCT **firstoct, struct CPUINFO *cpu, REAL dt);

/* Test-tree helper: set f[3] of every cell of a level (list order, 8*noct each). */
void emma_tree_set_force(struct EmmaTree *t, int level, const double *fx, const double *fy, const double *fz);

#ifdef __cplusplus
}
#endif

#endif
