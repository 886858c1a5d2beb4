/*
 * Compiles the reference's src/amr.c where it lies (it is included, not copied)
 * with -DSNTEST, whose refinement criterion in L_mark_cells is the cell density
 * (src/amr.c:1330-1354: field.d > 1.1).  A pure-hydro build of the reference has no
 * criterion at all (den is only set with WGRAV or TESTCOSMO), so this build is the
 * reference marking of the density criterion the device-side refinement offers.
 * SNTEST adds a member to struct RUNPARAMS after its first hundred bytes; amr.c
 * reads only lcoarse and lmax, whose offsets it does not change.
 * Test infrastructure only, linked into oracle/_ref/libemmaref_mark.so.
 */
#define SNTEST
#include "amr.c"
