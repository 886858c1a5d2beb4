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
constexpr uint32_t kKeyReal = 0, kKeyInj = 1, kKeyGhost0 = 2;
constexpr uint32_t kKeyNone = 0xFFFFFFFFu;
constexpr uint32_t key_make(uint32_t kind, uint32_t idx) { return (kind << 28) | idx; }

// Brick tiles.  A tile is one brick of 4 x 4 x 2 oct positions of a level's
// grid holding at least one oct of the level (mask: which).  The kernel stages
// a 6 x 6 x 4 box of virtual-oct slots (the brick and a ring of one oct), i.e.
// 12 x 12 x 8 cells, so that every neighbour a stencil reads sits at a fixed
// offset (+-1, +-12, +-144 cells).  Slot s = sx + 6 (sy + 6 sz); the brick
// interior is sx,sy in 1..4, sz in 1..2; slots no stencil reads hold kKeyNone.
constexpr int kBrickX = 4, kBrickY = 4, kBrickZ = 2, kTileOcts = kBrickX * kBrickY * kBrickZ;
constexpr int kSlotX = kBrickX + 2, kSlotY = kBrickY + 2, kSlotZ = kBrickZ + 2;
constexpr int kSlots = kSlotX * kSlotY * kSlotZ;                       // 144
constexpr int kBoxX = 2 * kSlotX, kBoxY = 2 * kSlotY, kBoxZ = 2 * kSlotZ;
constexpr int kBox = kBoxX * kBoxY * kBoxZ;                            // 1152 staged cells
constexpr int kNT = 8 * kTileOcts;                                     // 256 brick cells = threads
constexpr int kHaloCells = 2 * (8 * 4) * 2 + 2 * (8 * 8);              // 256 cells face-adjacent to the brick
constexpr int kFacesX = 9 * 8 * 4, kFacesY = 8 * 9 * 4, kFacesZ = 8 * 8 * 5;
constexpr int kFaces = kFacesX + kFacesY + kFacesZ;                    // 896 faces of the brick cells

struct TileDesc {
  uint32_t mask;  // bit (ix + 4 iy + 16 iz): brick position holds an oct of this level
  int noct;       // octs in the tile (popcount of mask)
  int ox, oy, oz; // brick origin in oct coordinates of the level
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
  const uint8_t *split;  // per oct bitmask of split cells
  const int *child;      // per cell: child oct index at L+1, -1 for a leaf
  const TileDesc *tiles;
  const uint32_t *keys;  // kSlots keys per tile
  double dt, dx;
  int ntiles;
  int wait_slot;      // level whose tiles must all be updated before this level's
                      // update phase starts (batched launches), -1 for none
  long long leaf;     // leaf cells (cell-updates of one substep)
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
};

constexpr int kWorkSlotShift = 24;
constexpr int kMaxLevels = 32;

}  // namespace emma
