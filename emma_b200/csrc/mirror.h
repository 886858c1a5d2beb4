// mirror.h -- host-side mirror of an EMMA oct tree: per-level oct lists,
// split masks, child links and the tile plans the level kernels execute.
#pragma once
#include <string>
#include <vector>
#include "emma_oct.h"
#include "plan_types.h"

namespace emma {

struct HostLevel {
  int L = 0;
  int noct = 0;                       // mirrored octs: nown of this rank, then ghosts
  int nown = 0;                       // octs with cpu == rank (advanced); octs[nown..noct) are the
                                      // octs of other ranks (staged as neighbours, never advanced)
  long long leaf = 0;                 // leaf cells of this rank's octs
  std::vector<struct OCT *> octs;     // this rank's octs in list order, then the others in list order
  std::vector<uint8_t> split;         // per oct: bit c set if cell c has a child
  std::vector<int32_t> child;         // per cell: index of the child oct at L+1, or -1
  std::vector<TileDesc> tiles;        // brick tiles, in order of their first oct in the list
  std::vector<uint32_t> keys;         // kSlots slot keys per tile
  std::vector<int32_t> inj_cells;     // level L-1 cells that receive fine->coarse corrections
  bool reads_coarse = false;          // some tile stages an injected level L-1 cell
  std::vector<int32_t> interp;        // transmissive or gravity builds: per interpolated level L-1
                                      // cell, the cell and its 6 slope neighbours (7 entries)
  int shape = 0;                      // brick shape of the plan (kShapes)
  std::vector<int32_t> pos;           // per oct: integer position on the level grid (x,y,z)
  std::vector<int32_t> nb6;           // per oct and face -x,+x,-y,+y,-z,+z: the neighbouring oct of
                                      // this level, -1 where there is none (coarser leaf or domain
                                      // edge), -2 across a transmissive boundary
};

struct HostTree {
  int lcoarse = 0, lmax = 0, rank = 0, trans = 0;
  int grav = 0;  // gravity coupling: injected coarser cells carry interpolated forces
  int dual = 0;  // dual energy: split cells next to a leaf are reconstructed too (their faces enter div u)
  int ghosts = 0;  // some level list holds octs of other ranks (a multi-rank run's boundary octs)
  std::vector<HostLevel> lev;  // indexed by level (0..lmax)
};

// Build the mirror of levels lcoarse..lmax and the tile plans of levels
// plan_lo..plan_hi (a plan of level L needs the mirror of L-1 when L-1 >=
// lcoarse).  Returns 0 on success, else an EMMA_ST_* bit with a message in `err`.
// shapes (optional, indexed by level): brick shape of each plan, -1 = the
// cheaper by tile count x tile cost.  grav: gravity-coupled build (every
// injected coarser cell gets an interpolation entry for its force; not
// combined with transmissive boundaries).  dual: dual-energy build (the planner
// checks the kernel's reconstruction rule of that build).
int build_host_tree(struct OCT **firstoct, int lcoarse, int lmax, int rank, int trans, int plan_lo, int plan_hi,
                    HostTree &H, std::string &err, const int *shapes = nullptr, int grav = 0, int dual = 0);

// Re-plan level L of a built tree with brick shape `shape` (the autotuner's
// candidates); validates the new plan.
int replan_level(HostTree &H, int L, int shape, std::string &err);

// Bounds check of every index the level kernels read (run by build_host_tree).
int validate_host_tree(const HostTree &H, int plan_lo, int plan_hi, std::string &err);

}  // namespace emma
