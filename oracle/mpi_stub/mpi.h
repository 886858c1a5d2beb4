/*
 * Minimal stand-in for <mpi.h>, used only to compile the reference's CPU hydro
 * sources as a test oracle in a container without MPI.  The reference includes
 * <mpi.h> unconditionally (src/hydro_utils.c:9) but, built without -DWMPI, only
 * calls MPI_Wtime() for its phase timers (src/hydro_utils.c:3394,3485).
 * Test infrastructure: never linked into the product library.
 */
#ifndef EMMA_ORACLE_MPI_STUB_H
#define EMMA_ORACLE_MPI_STUB_H
#include <time.h>
static inline double MPI_Wtime(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}
#endif
