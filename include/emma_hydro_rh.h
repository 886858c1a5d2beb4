/*
 * emma_hydro_rh.h -- entries of libemmahydro_rh.so only: the library built for
 * the reference's -DWRADHYD cell layout without -DHELIUM (compile the caller
 * with -DEMMA_WRADHYD so that include/emma_oct.h declares the 152-byte CELL whose
 * Wtype ends with the ionised density dX).  That library also exports everything
 * in emma_hydro.h; its drop-in HydroSolver / advancehydroGPU advance dX with the
 * gas as the reference's -DWRADHYD hydro does (face values from the centre's
 * ionised fraction, src/hydro_utils.c:1244-1246; HLLC fluxes du dX/d with the star
 * correction; the ceiling 0 <= dX <= d; fine->coarse corrections; split-cell
 * means), and so does its resident mode, where dX is the sixth plane of every
 * level state on the device (emma_hydro_tree_upload / _download move it with the
 * tree; emma_hydro_get/set_level_state still exchange the first five planes).
 * The tracer build has neither dual energy, transmissive boundaries nor gravity
 * (EMMA_ST_ARG).
 */
#ifndef EMMA_HYDRO_RH_H
#define EMMA_HYDRO_RH_H

#ifndef EMMA_WRADHYD
#error "emma_hydro_rh.h needs -DEMMA_WRADHYD (the -DWRADHYD cell layout)"
#endif

#include "emma_hydro.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Test-tree helpers: dX of field and fieldnew of every cell of a level (list order,
 * 8*noct), and dX of field (which=0) or fieldnew (which=1) read back. */
void emma_tree_set_tracer(struct EmmaTree *t, int level, const double *dX);
void emma_tree_get_tracer(struct EmmaTree *t, int level, int which, double *out);
/* dX of field (which=0) or fieldnew (which=1) only. */
void emma_tree_put_tracer(struct EmmaTree *t, int level, int which, const double *dX);

#ifdef __cplusplus
}
#endif

#endif
