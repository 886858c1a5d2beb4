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

// Kernel shape the plans are cut for: octs per tile, staged octs, directional
// halo entries, boundary faces.
constexpr int kTileOcts = 32;
constexpr int kSMax = 136;
constexpr int kHMax = 256;
constexpr int kBMax = 128;

struct TileDesc {
  int oct0;       // first oct of the tile (level list index)
  int noct;       // octs in the tile (<= kTileOcts)
  int S;          // staged virtual octs (tile octs first)
  int H;          // halo entries: (staged cell s*8+c) << 3 | face k of that cell toward the tile
  int B;          // boundary faces: tile cell t*4 + axis whose + face borders a non-tile oct
  int keys_off;   // offset into the keys array
  int graph_off;  // offset into the graph array (S*6 bytes; 255 = not staged)
  int halo_off;   // offset into the halo array
  int bface_off;  // offset into the boundary-face array
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
  const uint32_t *keys;
  const uint8_t *graph;
  const uint16_t *halo;
  const uint16_t *bface;
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
