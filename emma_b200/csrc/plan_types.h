// plan_types.h -- data shared by the host planner and the level kernels.
#pragma once
#include <stdint.h>

namespace emma {

// Virtual-oct keys of a tile plan: kind in bits 28..31, index in bits 0..27.
//   kKeyReal        : an oct of this level, index in the level list
//   kKeyInj         : a coarser leaf cell (level L-1, index oct*8+cell) whose
//                     state fills all 8 cells, as the reference's gather injects
//                     it (src/hydro_utils.c:2912-2944)
//   kKeyGhost0 + k  : transmissive ghost across face k of an oct of this level,
//                     filled through the reference's mirror map of face k
//                     (src/hydro_utils.c:2504-2610)
//   kKeyInterp      : a coarser leaf cell interpolated into 8 cells, as the
//                     reference's transmissive build (-DHYDROTEST) gathers it
//                     (coarse2fine_hydro2, src/hydro_utils.c:311); index into
//                     the level's interpolation list
constexpr uint32_t kKeyReal = 0, kKeyInj = 1, kKeyGhost0 = 2, kKeyInterp = 8;
constexpr uint32_t kKeyNone = 0xFFFFFFFFu;
constexpr uint32_t key_make(uint32_t kind, uint32_t idx) { return (kind << 28) | idx; }

// Brick tiles.  A brick is BX x BY x BZ oct positions of a level's grid; a
// tile is NB bricks that hold at least one oct of the level, advanced by one
// CTA of kThreads threads (one per brick cell).  For each brick the kernel
// stages a (BX+2) x (BY+2) x (BZ+2) box of virtual-oct slots (the brick and a
// ring of one oct), so every neighbour a stencil reads sits at a fixed offset.
// Slot s = sx + SX (sy + SY sz); the brick interior is sx in 1..BX etc.; slots
// no stencil reads hold kKeyNone.  Two shapes: 4x4x2 octs x 1 brick (complete
// levels) and 2x2x2 octs (the children of one parent oct) x 4 bricks (sparse
// refined levels); the autotuner picks one per level.
constexpr int kThreads = 256;
struct BrickShape {
  int bx, by, bz, nb;
  constexpr int octs() const { return bx * by * bz; }
  constexpr int slots() const { return (bx + 2) * (by + 2) * (bz + 2); }
  constexpr int tile_slots() const { return nb * slots(); }
};
constexpr int kNumShapes = 2;
// Launch flag beside the shape bits of a level-kernel launch: the gravity-coupled
// variant (levels with accelerations); the plain variant has no gravity code.
constexpr unsigned kLaunchGrav = 4u;
// ... and the dual-energy variant (-DDUAL_E: tracked internal energy, 6 correction planes).
constexpr unsigned kLaunchDual = 8u;
// ... and the tracer variant (-DWRADHYD: the advected ionised density dX; its
// corrections are plane kXPlane of Cc).  Not combined with gravity or dual energy.
constexpr unsigned kLaunchTracer = 16u;
// ... and its -DHELIUM variant: dX and the helium densities dXHE, dXXHE (corrections
// in planes kXPlane .. kXPlane + 2 of Cc).
constexpr unsigned kLaunchHelium = 32u;
constexpr int kXPlane = 5;
constexpr BrickShape kShapes[kNumShapes] = {{4, 4, 2, 1}, {2, 2, 2, 4}};
static_assert(kShapes[0].nb * 8 * kShapes[0].octs() == kThreads, "one thread per brick cell");
static_assert(kShapes[1].nb * 8 * kShapes[1].octs() == kThreads, "one thread per brick cell");
constexpr int kTileOcts = 32;  // octs per tile (mask bits), both shapes

struct TileDesc {
  uint32_t mask;  // bit (nb * octs + ix + BX (iy + BY iz)): brick nb holds an oct at that position
  int noct;       // octs in the tile (popcount of mask)
  int ox, oy, oz; // origin of the first brick in oct coordinates of the level
  int pad[3];
};

// Arguments of one level, resident in device memory (one slot per level).
// Schedule kernels update dt and the state buffers between launches, so a
// captured CUDA graph can run a whole coarse step without the host.
struct LevelArgs {
  int L;
  int noct;
  double *W;          // level state, planes d,u,v,w,p of 8*noct
  double *Wn;         // next state (written by the level kernel)
  double *C;          // conserved corrections received from the finer level
  const double *B;    // optional update base: planes d,u,v,w,p,E of the caller's fieldnew
                      // (drop-in mode); when null the base is W2U(W) + C
  const double *Wc;   // level L-1 state read for injected neighbours, may be null
  double *Cc;         // level L-1 corrections (fine->coarse), may be null
  long long nc8;      // plane stride of Wc/Cc
  const double *Wf;   // level L+1 state for split-cell averaging, may be null
  long long nf8;      // plane stride of Wf
  double *Wv;         // interpolated coarser cells: planes d,u,v,w,p of 8 * nv
  const int *vcell;   // per interpolated cell: the level L-1 cell, then its 6 neighbours
                      // (-x,+x,-y,+y,-z,+z) the slopes are taken from
  long long nv;       // interpolated coarser cells
  const uint8_t *split;  // per oct bitmask of split cells
  const int *child;      // per cell: child oct index at L+1, -1 for a leaf
  const TileDesc *tiles;
  const uint32_t *keys;  // kShapes[shape].tile_slots() keys per tile
  int shape;             // brick shape of the plan (index into kShapes)
  int pad_shape;
  double dt, dx;
  int ntiles;
  int wait_slot;      // level whose tiles must all be updated before this level's
                      // update phase starts (batched launches), -1 for none
  long long leaf;     // leaf cells (cell-updates of one substep)
  // gravity coupling (-DWGRAV), all null/0 without it.  The tracer variant
  // (-DWRADHYD) has neither gravity nor dual energy and reuses their pointer
  // slots (unions): the struct is copied into every CTA's shared memory, whose
  // 4-CTA budget of the FP32 kernel leaves no room for more members.
  union {
    const double *F;  // acceleration of the level's cells: planes fx,fy,fz of 8*noct
    const double *X;  // tracer: dX of the level's field (plane of 8*noct)
  };
  union {
    const double *Fc;  // acceleration of level L-1 (read by the interpolation kernel)
    const double *Xc;  // tracer: dX of level L-1 (injected neighbours)
  };
  double *Fv;         // accelerations of the interpolated coarser cells: planes of 8 * nv
  int gcorr;          // apply grav_correction (src/hydro_utils.c:2388-2444) to the new state
  int wv_inject;      // the interpolation list fills Wv by injection (gravity build), not by
                      // limited-slope interpolation (transmissive build)
  // dual energy: split cells whose stored sound speed is 0 (the reference's
  // averaging leaves a = 0, src/hydro_utils.c:3417-3481, and its predictor reads the
  // stored a, :976-1120): per cell, or every split cell once *azall != 0
  union {
    const uint8_t *az;
    double *Xn;  // tracer: the new dX written by the level kernel
  };
  union {
    const int *azall;
    const double *BX;  // tracer: the update base, the caller's fieldnew.dX (drop-in mode)
  };
};

// A launch of the level kernel: a list of (level slot, tile) work items,
// processed by a persistent grid in list order.
struct BatchArgs {
  LevelArgs *lv;        // device array of level slots
  const int *work;      // (slot << 24) | tile
  int nwork;
  unsigned *done;       // per slot: tiles whose update phase has completed
  const int *gate;      // launch does nothing unless *gate != 0 (null: always run)
  unsigned *status;
  long long wait_limit; // bounded spin on `done` before reporting a timeout
  unsigned long long *smax;  // per slot: max signal speed |v| + c_s of the states written
                             // (bits of a non-negative double, atomicMax), or null
  int zero_c;           // clear each correction once the update has read it
  unsigned *ticket;     // work queue: [0] next item, [1] CTAs finished (reset by the last)
};

// A launch of the column kernel (column_kernel.cuh): one complete periodic level
// without split cells, as columns of 16 x 16 cells marching through `nz` planes.
struct ColumnArgs {
  const LevelArgs *lv;  // the level's device slot: W, Wn, dt, dx are read at launch
  int L;
  const int *octidx;    // oct (list index) at every oct position, ((oz * n + oy) * n + ox)
  int n;                // octs per side
  int nz;               // cell planes per work item (even, divides 2n)
  int ncol;             // columns per side (2n / 16)
  int nitems;           // ncol * ncol * (2n / nz)
  const int *gate;      // launch does nothing unless *gate != 0 (null: always)
  unsigned *status;
  unsigned long long *smax;  // [L]: max signal speed of the new state (bits of a double), or null
  int xshfl;            // x faces inside the column through warp shuffles (column_kernel.cuh XS)
  int balanced;         // nitems CTAs, each an equal run of the level's column-planes (nz unused)
};
constexpr int kColumnWidth = 16;  // cells per column side

constexpr int kWorkSlotShift = 24;
constexpr int kMaxLevels = 32;

}  // namespace emma
