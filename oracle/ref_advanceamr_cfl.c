/*
 * Compiles the reference's src/advanceamr.c where it lies (it is included, not
 * copied) with the Courant number set to 0.8 instead of param.h's 0.85
 * (src/param.h:5), because the benchmark configurations are quoted at CFL 0.8.
 * Only L_comptstep_hydro (src/advanceamr.c:92) is called, by ref_driver.c.
 * Test infrastructure only.
 */
#include "prototypes.h"
#undef CFL
#define CFL (0.8)
#include "advanceamr.c"
