/*
 * Test infrastructure (oracle): drives the reference's own field dump,
 * dumpalloct_serial (src/io.c:1233-1358), on a caller's oct tree, so that the
 * library's emma_hydro_dump_alloct can be compared with it byte for byte.
 * Built with -DWMPI and the single-rank stand-in oracle/mpi_stub_io/mpi.h (io.c
 * reads CPUINFO members that exist only with -DWMPI; struct OCT and struct CELL
 * do not change with it).  Nothing here is part of the product.
 */
#include <stdlib.h>
#include <string.h>
#include "prototypes.h"
#include "io.h"
#include "oct.h"

/* The reference's dump of levels lcoarse..lmax of the tree whose level lists start
 * at firstoct[level-1]: for every field id in ids (names in names), the file
 * <folder>grid_<name>/<name>.<ndumps>.p<rank>.  The octs of `rank` are listed per
 * level by the reference's own setOctList (src/oct.c:250).  folder ends with '/'. */
int ref_dump_alloct(const char *folder, struct OCT **firstoct, int lcoarse, int lmax, int rank, int ndumps,
                    double tsim, int nf, const int *ids, const char **names) {
  struct CPUINFO cpu;
  struct RUNPARAMS param;
  struct OUTPUTPARAM og;
  memset(&cpu, 0, sizeof(cpu));
  memset(&param, 0, sizeof(param));
  memset(&og, 0, sizeof(og));
  cpu.rank = rank;
  cpu.ndumps = &ndumps;
  cpu.locNoct = (int *)calloc((size_t)lmax, sizeof(int));
  cpu.octList = (struct OCT ***)calloc((size_t)lmax, sizeof(struct OCT **));
  for (int level = lcoarse; level <= lmax; level++) {
    int n = 0;
    for (struct OCT *o = firstoct[level - 1]; o != NULL; o = o->next) n++;
    cpu.octList[level - 1] = (struct OCT **)calloc((size_t)(n > 0 ? n : 1), sizeof(struct OCT *));
    setOctList(firstoct[level - 1], &cpu, &param, level);
  }
  param.lcoarse = lcoarse;
  param.lmax = lmax;
  param.out_grid = &og;
  og.n_field_tot = OUTPUTPARAM_n_field_max;
  for (int i = 0; i < nf; i++) {
    if (ids[i] < 0 || ids[i] >= OUTPUTPARAM_n_field_max) return -1;
    og.field_id[ids[i]] = 1;
    og.field_name[ids[i]] = (char *)names[i];
  }
  og.n_field = nf;
  char dir[256];
  strncpy(dir, folder, sizeof(dir) - 1);
  dir[sizeof(dir) - 1] = 0;
  dumpalloct_serial(dir, (REAL)tsim, &param, &cpu);
  for (int level = lcoarse; level <= lmax; level++) free(cpu.octList[level - 1]);
  free(cpu.octList);
  free(cpu.locNoct);
  return 0;
}
