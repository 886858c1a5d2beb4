/*
 * Single-rank stand-in for <mpi.h>, used only to compile the reference's field
 * dump (src/io.c) as a test oracle in a container without MPI.  io.c reads
 * CPUINFO members that exist only with -DWMPI, so it is built with -DWMPI; of
 * MPI it then needs the types CPUINFO names and the three calls of dump_domain
 * (MPI_Allgather, MPI_Barrier) and its timers (MPI_Wtime), here for one rank.
 * Test infrastructure: never linked into the product library.
 */
#ifndef EMMA_ORACLE_MPI_STUB_IO_H
#define EMMA_ORACLE_MPI_STUB_IO_H
#include <string.h>
#include <time.h>
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
#define MPI_COMM_WORLD 0
#define MPI_INT 4
#define MPI_FLOAT 4
#define MPI_DOUBLE 8
static inline int MPI_Allgather(const void *s, int n, MPI_Datatype t, void *r, int rn, MPI_Datatype rt, MPI_Comm c) {
  (void)rn, (void)rt, (void)c;
  memcpy(r, s, (size_t)n * (size_t)t);  /* one rank: its own contribution */
  return 0;
}
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
static inline double MPI_Wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
#endif
