/*
 * emma_hydro_he.h -- entries of libemmahydro_he.so only: the library built for
 * the reference's -DWRADHYD -DHELIUM cell layout (compile the caller with
 * -DEMMA_WRADHYD -DEMMA_HELIUM so that include/emma_oct.h declares the 184-byte
 * CELL whose Wtype ends with dX, dXHE, dXXHE).  That library also exports
 * everything in emma_hydro.h; its drop-in and resident entries advance the three
 * tracers with the gas as the reference's -DWRADHYD -DHELIUM hydro does, with the
 * helium mass fraction YHE = 0.24 (src/param.h:47-48): face values from the
 * centre's fractions, dX / (d (1 - YHE)) and dXHE / (d YHE), dXXHE / (d YHE)
 * (src/hydro_utils.c:1244-1252); HLLC fluxes u dT/d with the star correction
 * (:1534-1539 and the y, x sweeps); dX kept in [0, d (1 - YHE)], the helium
 * densities below d YHE (:3197-3203); fine->coarse corrections (:3277-3281);
 * split-cell means (:3446-3460).  In the resident mode the tracers are planes 6-8
 * of every level state on the device.  Like libemmahydro_rh.so it has neither dual
 * energy, transmissive boundaries nor gravity (EMMA_ST_ARG).
 */
#ifndef EMMA_HYDRO_HE_H
#define EMMA_HYDRO_HE_H

#if !defined(EMMA_WRADHYD) || !defined(EMMA_HELIUM)
#error "emma_hydro_he.h needs -DEMMA_WRADHYD -DEMMA_HELIUM (the -DWRADHYD -DHELIUM cell layout)"
#endif

#include "emma_hydro.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Test-tree helpers: tracer t (0: dX, 1: dXHE, 2: dXXHE) of field and fieldnew of
 * every cell of a level (list order, 8*noct); read back from field (which=0) or
 * fieldnew (which=1); written into field or fieldnew only. */
void emma_tree_set_tracer_n(struct EmmaTree *t, int level, int tracer, const double *x);
void emma_tree_get_tracer_n(struct EmmaTree *t, int level, int tracer, int which, double *out);
void emma_tree_put_tracer_n(struct EmmaTree *t, int level, int tracer, int which, const double *x);

#ifdef __cplusplus
}
#endif

#endif
