// level_kernel.cuh -- the hydro level advance on the GPU, one CTA per tile.
//
// A tile is NB bricks of BX x BY x BZ oct positions of one level (one thread
// per brick cell, 256 per CTA) holding at least one oct of the level.  For each
// brick the CTA:
//   P0  stages a (BX+2) x (BY+2) x (BZ+2)-slot box (the brick and a ring of one
//       oct) of "virtual octs": a real oct of the level, a coarser leaf cell
//       injected into 8 cells as the reference's gather does, or a transmissive
//       mirror ghost; only the slots a stencil reads (faces and edges of the
//       tile octs) are filled.  Neighbours are then fixed offsets in the box;
//   P1  MUSCL-Hancock once per needed cell: slopes + predictor of every brick
//       cell that is a leaf of the tile or borders one, and for every ring cell
//       face-adjacent to the brick the one face state it contributes;
//   P2  one HLLC solve per face: three rounds (the -x, -y, -z face of every
//       brick cell), then the + faces on the brick boundary;
//   P3  per leaf of the tile: the six face fluxes summed in the reference's
//       order (-x,+x,-y,+y,-z,+z), conserved update, primitive recovery,
//       floors; split cells get the primitive mean of their children; faces
//       bordering a coarser leaf add the fine->coarse correction (atomics, x 1/8).
// The reference does the same per oct on a 27-oct copy, recomputing each
// cell's reconstruction up to 9 times and each face twice
// (src/hydro_utils.c:1407-2238, 2973-3303).
#pragma once
#include <type_traits>
#include "hydro_math.cuh"
#include "plan_types.h"

namespace emma {

// 4-wide shared-memory groups: one 128-bit access per group for FP32 (float4),
// two for FP64 (double2 pairs).  Element i of arrays of n groups (n a compile-time
// constant at every call site; consecutive arrays of n groups each may follow):
// FP32 stores the 4 values together; FP64 stores (x,y) and (z,w) in two planes of
// n double2 each, so that consecutive threads touch consecutive 16-byte words.
template <class R>
struct Q4;
template <>
struct Q4<float> {
  static __device__ __forceinline__ void st(float *b, int i, int, float x, float y, float z, float w) {
    reinterpret_cast<float4 *>(b)[i] = make_float4(x, y, z, w);
  }
  static __device__ __forceinline__ void ld(const float *b, int i, int, float &x, float &y, float &z, float &w) {
    const float4 v = reinterpret_cast<const float4 *>(b)[i];
    x = v.x;
    y = v.y;
    z = v.z;
    w = v.w;
  }
};
template <>
struct Q4<double> {
  static __device__ __forceinline__ void st(double *b, int i, int n, double x, double y, double z, double w) {
    const int g = i / n, j = i - g * n;
    double2 *p = reinterpret_cast<double2 *>(b) + 2 * n * g;
    p[j] = make_double2(x, y);
    p[n + j] = make_double2(z, w);
  }
  static __device__ __forceinline__ void ld(const double *b, int i, int n, double &x, double &y, double &z,
                                            double &w) {
    const int g = i / n, j = i - g * n;
    const double2 *p = reinterpret_cast<const double2 *>(b) + 2 * n * g;
    const double2 a = p[j];
    const double2 c = p[n + j];
    x = a.x;
    y = a.y;
    z = c.x;
    w = c.y;
  }
};

// mirror maps of the transmissive ghost octs (src/hydro_utils.c:2504-2610)
__constant__ uint8_t c_mirror[6][8] = {
    {0, 0, 2, 2, 4, 4, 6, 6}, {1, 1, 3, 3, 5, 5, 7, 7}, {0, 1, 0, 1, 4, 5, 4, 5},
    {2, 3, 2, 3, 7, 6, 6, 7}, {0, 1, 2, 3, 0, 1, 2, 3}, {4, 5, 6, 7, 4, 5, 6, 7}};

// cell flags of the staged box (kFInterp: the slot reads the interpolated coarse cells)
constexpr uint8_t kFPresent = 1, kFSplit = 2, kFTile = 4, kFInj = 8, kFInterp = 16;
constexpr uint8_t kFAzero = 32;  // dual energy: a split cell whose stored sound speed is 0
__device__ __forceinline__ bool f_ok(uint8_t f) { return (f & (kFPresent | kFSplit)) == kFPresent; }
__device__ __forceinline__ bool f_tileleaf(uint8_t f) {
  return (f & (kFPresent | kFSplit | kFTile)) == (kFPresent | kFTile);
}

// Geometry of a tile of NB bricks of BX x BY x BZ octs.  Brick cell
// t = x + CX (y + CY z) sits at box cell (x+2) + XX ((y+2) + XY (z+2)).  Ring cell
// j (face-adjacent to the brick): -x side (y + CY z), +x side, -y (x + CX z), +y,
// -z (x + CX y), +z.  Face arrays, -d face of brick cell (x,y,z):
// x: x + (CX+1)(y + CY z), y: FX + x + CX (y + (CY+1) z), z: FX + FY + x + CX (y + CY z),
// with coordinate CX, CY or CZ for the + faces on the brick boundary.
template <int BX, int BY, int BZ, int NB>
struct Geom {
  static constexpr int kNB = NB, kOcts = BX * BY * BZ;
  static constexpr int CX = 2 * BX, CY = 2 * BY, CZ = 2 * BZ, kCells = CX * CY * CZ;
  static constexpr int SX = BX + 2, SY = BY + 2, SZ = BZ + 2, kSlots = SX * SY * SZ;
  static constexpr int XX = 2 * SX, XY = 2 * SY, XZ = 2 * SZ, kBox = XX * XY * XZ, XS = XX * XY;
  static constexpr int kPX = CY * CZ, kPY = CX * CZ, kPZ = CX * CY;  // cells of one face layer
  static constexpr int kRing = 2 * (kPX + kPY + kPZ), kPlus = kPX + kPY + kPZ;
  static constexpr int kFX = (CX + 1) * CY * CZ, kFY = CX * (CY + 1) * CZ, kFZ = CX * CY * (CZ + 1);
  static constexpr int kFaces = kFX + kFY + kFZ;
  static_assert(NB * kCells == kThreads, "one thread per brick cell");
  static_assert(NB * kOcts <= 32, "tile mask is 32 bits");

  static __device__ __forceinline__ int box_of(int x, int y, int z) { return (x + 2) + XX * ((y + 2) + XY * (z + 2)); }
  static __device__ __forceinline__ void cell_of(int t, int &x, int &y, int &z) {
    x = t % CX;
    y = (t / CX) % CY;
    z = t / (CX * CY);
  }
  // ring cell j: box cell, its face k toward the brick and the brick cell across it
  static __device__ __forceinline__ void ring_cell(int j, int &b, int &k, int &bin) {
    if (j < 2 * kPX) {
      const int side = j >= kPX, i = j - side * kPX, y = i % CY, z = i / CY;
      b = (side ? CX + 2 : 1) + XX * ((y + 2) + XY * (z + 2));
      k = side ? 0 : 1;
      bin = b + (side ? -1 : 1);
    } else if (j < 2 * (kPX + kPY)) {
      int i = j - 2 * kPX;
      const int side = i >= kPY;
      i -= side * kPY;
      const int x = i % CX, z = i / CX;
      b = (x + 2) + XX * ((side ? CY + 2 : 1) + XY * (z + 2));
      k = side ? 2 : 3;
      bin = b + (side ? -XX : XX);
    } else {
      int i = j - 2 * (kPX + kPY);
      const int side = i >= kPZ;
      i -= side * kPZ;
      const int x = i % CX, y = i / CX;
      b = (x + 2) + XX * ((y + 2) + XY * (side ? CZ + 2 : 1));
      k = side ? 4 : 5;
      bin = b + (side ? -XS : XS);
    }
  }
  // ring cell across the -d (plus = false) or +d face of brick cell (x,y,z) on the brick boundary
  static __device__ __forceinline__ int ring_index(int d, bool plus, int x, int y, int z) {
    if (d == 0) return (plus ? kPX : 0) + y + CY * z;
    if (d == 1) return 2 * kPX + (plus ? kPY : 0) + x + CX * z;
    return 2 * (kPX + kPY) + (plus ? kPZ : 0) + x + CX * y;
  }
  static __device__ __forceinline__ int face_index(int d, int x, int y, int z) {
    if (d == 0) return x + (CX + 1) * (y + CY * z);
    if (d == 1) return kFX + x + CX * (y + (CY + 1) * z);
    return kFX + kFY + x + CX * (y + CY * z);
  }
};
using GeomA = Geom<4, 4, 2, 1>;  // kShapes[0]
using GeomB = Geom<2, 2, 2, 4>;  // kShapes[1]
static_assert(GeomA::kOcts == 32 && GeomB::kOcts == 8, "shapes match kShapes");

// Per-CTA slot tables of both shapes (tile independent), at the start of
// shared memory: box cell of child 0, brick position bit (255 outside the
// brick).
template <class G>
struct SlotTab {
  static constexpr size_t bytes = ((size_t)G::kSlots * 4 + 15) & ~size_t(15);
};
constexpr size_t kTabOffB = SlotTab<GeomA>::bytes;
constexpr size_t kSmaxOff = kTabOffB + SlotTab<GeomB>::bytes;  // u64 [kMaxLevels] per-CTA signal-speed maxima
constexpr size_t kTabBytes = kSmaxOff + 8 * kMaxLevels;

template <class G>
__device__ __forceinline__ void slot_tables(unsigned char *tab) {
  uint16_t *sBase = reinterpret_cast<uint16_t *>(tab);
  uint8_t *sBit = tab + 2 * G::kSlots;
  for (int s = threadIdx.x; s < G::kSlots; s += blockDim.x) {
    const int sz = s / (G::SX * G::SY), sy = (s / G::SX) % G::SY, sx = s % G::SX;
    sBase[s] = (uint16_t)(2 * sx + G::XX * (2 * sy + G::XY * 2 * sz));
    const bool inner = sx >= 1 && sx <= G::SX - 2 && sy >= 1 && sy <= G::SY - 2 && sz >= 1 && sz <= G::SZ - 2;
    sBit[s] = inner ? (uint8_t)((sx - 1) + (G::SX - 2) * ((sy - 1) + (G::SY - 2) * (sz - 1))) : (uint8_t)255;
  }
}

// Tile groups.  A tile is advanced by kThreads threads; a CTA of the fused coarse
// step (step_kernel.cuh) runs several tiles at once, one per group of kThreads
// threads, each group with its own shared-memory region and its own named
// barrier (1 + group; barrier 0 stays the CTA-wide __syncthreads).  In the level
// kernel the CTA is one group and the barrier is __syncthreads.
__device__ __forceinline__ int tile_group() { return (int)(threadIdx.x / kThreads); }
template <bool GRP>
__device__ __forceinline__ void tile_sync() {
  if constexpr (GRP) asm volatile("bar.sync %0, %1;" ::"r"(1 + tile_group()), "n"(kThreads) : "memory");
  else __syncthreads();
}
// Loads of level states.  COH (the fused coarse step, where a state read here was
// written by another CTA earlier in the same launch): through L2 only (ld.global.cg),
// never the non-coherent read-only path, whose cache may still hold the lines of an
// earlier job; measured 2.7% faster than plain L1-allocating loads on the cosmology
// tree and as fast on the Sedov tree, the staged lines being used once per tile.
template <bool COH, class T>
__device__ __forceinline__ T ld_state(const T *p) {
  if constexpr (COH) return __ldcg(p);
  else return __ldg(p);
}

// Shared memory of one tile, after the slot tables.  DUAL: dual-energy builds add
// the internal-energy flux and the normal star velocity of every face.  NTR
// tracers (-DWRADHYD: 1, with -DHELIUM: 3; not with DUAL): the fraction of every
// tracer in every staged cell and the tracer fluxes of every face.
template <class M, class G, bool DUAL = false, int NTR = 0>
struct TileSmem {
  using R = typename M::R;
  static constexpr bool kF64 = sizeof(R) == 8;
  static constexpr int NS = G::kNB * G::kSlots, NBOX = G::kNB * G::kBox, NRING = G::kNB * G::kRing;
  static constexpr int NF = G::kNB * G::kFaces;
  // FP64 with dual energy or tracers: the faces are solved in two rounds (x and y,
  // then z) and each round's fluxes summed into the cells before the next, so that
  // the per-face arrays fit in the staged box; the tracer fractions are kept only
  // for the cells a face reads (the brick cells, then the ring)
  static constexpr bool kR2 = kF64 && (DUAL || NTR > 0);
  static constexpr int NFA = G::kNB * (G::kFX + G::kFY), NFB = G::kNB * G::kFZ;
  static constexpr int NFS = kR2 ? NFA : NF;  // face entries of the flux arrays
  static constexpr int NXC = kThreads + NRING;  // compact tracer cells (kR2)
  // descriptor buffers: the current tile's and the next tile's (prefetched), or one
  // (FP64 single tracer: no prefetch, so that two CTAs fit an SM)
  static constexpr int kDB = (kF64 && NTR == 1) ? 1 : 2;
  static constexpr size_t a16(size_t x) { return (x + 15) & ~size_t(15); }
  static constexpr size_t off_args = kTabBytes;                                // LevelArgs of the tile's level
  // per-slot descriptors
  static constexpr size_t off_key = a16(off_args + sizeof(LevelArgs));         // u32 [kDB][NS]
  static constexpr size_t off_ob = a16(off_key + 4 * kDB * NS);                // i32 [kDB][NS] source offset
  static constexpr size_t off_sf = a16(off_ob + 4 * kDB * NS);                 // u8  [kDB][NS] slot flags
  static constexpr size_t off_spm = a16(off_sf + kDB * NS);                    // u8  [kDB][NS] split mask (cell order)
  static constexpr size_t off_cmk = a16(off_spm + kDB * NS);                   // u8  [kDB][NS] cell map
  static constexpr size_t off_st = a16(off_cmk + kDB * NS);                    // u8  [NBOX] cell flags
  static constexpr size_t off_W = a16(off_st + NBOX);                          // R4  [NBOX] (d,u,v,w)
  static constexpr size_t off_Wp = a16(off_W + sizeof(R) * 4 * NBOX);          // R   [NBOX] p
  // reconstruction of the brick cells: R4 groups [kMG][kThreads] (slopes, predicted
  // state; FP64 also the centre state, so that the box is dead after P1), then the
  // FP64 centre pressure R [kThreads]
  static constexpr int kMG = kF64 ? 6 : 5;
  static constexpr size_t off_M = a16(off_Wp + sizeof(R) * NBOX);
  static constexpr size_t off_Mp = off_M + sizeof(R) * 4 * kMG * kThreads;
  // ring face states: FP32 R4 [2][NRING] (d,u,v,w | p,1/d,a); FP64 R4 [NRING] + R [NRING]
  // (d,u,v,w | p: a and E are recomputed by the consumer)
  static constexpr size_t off_HS = a16(off_Mp + (kF64 ? sizeof(R) * kThreads : 0));
  static constexpr size_t off_end = a16(off_HS + (kF64 ? sizeof(R) * 5 * NRING : sizeof(R) * 4 * 2 * NRING));
  // face fluxes reuse the staged box, dead after reconstruction
  static constexpr size_t off_F = off_W;                                // R4 [NFS]
  static constexpr size_t off_F1 = a16(off_F + sizeof(R) * 4 * NFS);    // R  [NFS]
  static constexpr size_t off_F5 = kR2 ? a16(off_F1 + sizeof(R) * NFS) : off_end;  // R [NFS] (DUAL)
  static constexpr size_t off_S = a16(off_F5 + sizeof(R) * NFS);                   // R [NFS] (DUAL)
  // tracers: fractions R [NTR][NBOX] (kR2: [NTR][NXC], after the ring face states),
  // face fluxes R [NTR][NFS] (kR2: in the box)
  static constexpr size_t off_X = off_end;
  static constexpr size_t off_FX = kR2 ? a16(off_F1 + sizeof(R) * NFS) : a16(off_X + sizeof(R) * NTR * NBOX);
  static constexpr size_t face_end =
      DUAL ? a16(off_S + sizeof(R) * NFS) : (NTR > 0 ? a16(off_FX + sizeof(R) * NTR * NFS) : off_F1 + sizeof(R) * NFS);
  static constexpr size_t bytes = kR2 ? (NTR > 0 ? a16(off_X + sizeof(R) * NTR * NXC) : off_end)
                                      : (DUAL ? face_end : (NTR > 0 ? face_end : off_end));
  static_assert(!(DUAL && NTR > 0), "the tracer variants have no dual energy");
  static_assert(NTR == 0 || NTR == 1 || NTR == 3, "dX alone, or dX and the two helium tracers");
  static_assert(off_F1 + sizeof(R) * NFS <= off_M, "face fluxes must fit in the staged box");
  // FP64 gravity kicks of the brick cells during P2/P3: R [3][kThreads] at the end of
  // the staged box, after the face fluxes
  static constexpr size_t off_K = off_M - sizeof(R) * 3 * kThreads;
  static_assert(!kF64 || off_K >= off_F1 + sizeof(R) * NFS, "FP64 kicks must not overlap the face fluxes");
  static_assert(!kR2 || face_end <= off_K, "two-round face arrays must fit in the staged box before the kicks");
};

// One tile.  Software pipeline over the tiles of a CTA: the level's arguments
// stay in shared memory while consecutive tiles belong to the same level, and
// the next tile's slot descriptors (next_tile >= 0: same level) are loaded
// while this tile is reconstructed and solved, into the other descriptor
// buffer; `cur`/`have` track which buffer holds the current tile's.
// smem: the tile's shared memory, offsets TileSmem (the slot tables at `tab`, the
// per-CTA signal-speed maxima at sSmax, both shared by the CTA's tile groups).
// COH: the fused coarse step (ld_state, group barriers).
template <class M, class G, bool GRAV, bool DUAL, int NTR = 0, bool COH = false>
__device__ __forceinline__ void level_tile(const BatchArgs &Bt, const LevelArgs *gA, const int slot, const int tile,
                                           const int next_tile, unsigned char *smem, const unsigned char *tab,
                                           unsigned long long *sSmax, unsigned &st, int &cur, bool &have,
                                           int &args_slot) {
  using R = typename M::R;
  using SM = TileSmem<M, G, DUAL, NTR>;
  constexpr bool TRACER = NTR > 0;
  using TR = Tracers<(NTR > 0 ? NTR : 1)>;
  constexpr bool F64 = SM::kF64;
  constexpr int NS = SM::NS, NRING = SM::NRING;
  using V = Q4<R>;
  uint32_t *sKey = reinterpret_cast<uint32_t *>(smem + SM::off_key) + cur * NS;
  int *sOb = reinterpret_cast<int *>(smem + SM::off_ob) + cur * NS;
  uint8_t *sSf = smem + SM::off_sf + cur * NS;
  uint8_t *sSpm = smem + SM::off_spm + cur * NS;
  uint8_t *sCmk = smem + SM::off_cmk + cur * NS;
  const int nxt = NS * (1 - 2 * cur);  // offset of the other buffer
  const uint16_t *sBase = reinterpret_cast<const uint16_t *>(tab);
  const uint8_t *sBit = tab + 2 * G::kSlots;
  uint8_t *sSt = smem + SM::off_st;
  R *sW = reinterpret_cast<R *>(smem + SM::off_W);
  R *sWp = reinterpret_cast<R *>(smem + SM::off_Wp);
  R *sM = reinterpret_cast<R *>(smem + SM::off_M);
  R *sMp = reinterpret_cast<R *>(smem + SM::off_Mp);
  R *sHS = reinterpret_cast<R *>(smem + SM::off_HS);
  R *sF = reinterpret_cast<R *>(smem + SM::off_F);
  R *sF1 = reinterpret_cast<R *>(smem + SM::off_F1);
  R *sF5 = reinterpret_cast<R *>(smem + SM::off_F5);
  R *sS = reinterpret_cast<R *>(smem + SM::off_S);
  R *sX = reinterpret_cast<R *>(smem + SM::off_X);    // tracers: dT / (d frac) of the staged cells
  R *sFX = reinterpret_cast<R *>(smem + SM::off_FX);  // tracers: face fluxes
  // cells whose face states are built: leaves; dual-energy builds also split cells,
  // whose faces enter the p div(u) term (src/hydro_utils.c:2126-2129 sum every face)
  auto recon_ok = [](uint8_t f) { return DUAL ? (f & kFPresent) != 0 : f_ok(f); };

  const int tid = threadIdx.x % kThreads;
  // the level's arguments in shared memory, read again only when the level changes
  LevelArgs &A = *reinterpret_cast<LevelArgs *>(smem + SM::off_args);
  static_assert(sizeof(LevelArgs) % 4 == 0, "LevelArgs copied as 32-bit words");
  if (slot != args_slot) {
    if (tid < (int)(sizeof(LevelArgs) / 4)) {
      const uint32_t *src = reinterpret_cast<const uint32_t *>(gA) + tid;
      reinterpret_cast<uint32_t *>(&A)[tid] = *src;
    }
    tile_sync<COH>();
    args_slot = slot;
  }
  const long long N8 = 8LL * A.noct;
  // tracer planes (tracer t at plane offset t times the level's plane stride).
  // Drop-in levels (B set) name them; resident levels keep them as planes 6.. of
  // every state buffer, so that the schedule's buffer swaps carry them
  const bool res_tr = TRACER && A.B == nullptr;
  const double *Xs = res_tr ? A.W + 5 * N8 : A.X;
  const double *Xcs = res_tr ? (A.Wc != nullptr ? A.Wc + 5 * A.nc8 : nullptr) : A.Xc;
  double *Xns = res_tr ? A.Wn + 5 * N8 : A.Xn;
  const int tn = tid / G::kCells, tt = tid - tn * G::kCells;  // brick of the tile, cell of the brick
  int tx, ty, tz;
  G::cell_of(tt, tx, ty, tz);
  const int bo = tn * G::kBox;                 // this brick's box in the tile's boxes
  const int tb = bo + G::box_of(tx, ty, tz);   // this thread's brick cell
  // compact tracer cell of box cell b (two-round FP64 layout): the brick cell's
  // thread, kThreads + its ring cell, or -1 where no face reads it
  auto xc_of = [&](int b) -> int {
    const int nb = b / G::kBox, bl = b - nb * G::kBox;
    const int x = bl % G::XX - 2, y = (bl / G::XX) % G::XY - 2, z = bl / G::XS - 2;
    const bool ix = x >= 0 && x < G::CX, iy = y >= 0 && y < G::CY, iz = z >= 0 && z < G::CZ;
    if (ix && iy && iz) return nb * G::kCells + x + G::CX * (y + G::CY * z);
    if (iy && iz && (x == -1 || x == G::CX)) return kThreads + nb * G::kRing + G::ring_index(0, x == G::CX, x, y, z);
    if (ix && iz && (y == -1 || y == G::CY)) return kThreads + nb * G::kRing + G::ring_index(1, y == G::CY, x, y, z);
    if (ix && iy && (z == -1 || z == G::CZ)) return kThreads + nb * G::kRing + G::ring_index(2, z == G::CZ, x, y, z);
    return -1;
  };

  // ------------------------------------------------------------------ P0
  // per slot: key, source offset, flags, split mask in cell order, cell map
  // (0: cell c of an oct, 1: an injected cell, 2+k: mirror across face k);
  // `raw` is the split byte of a real or ghost slot's oct
  auto build = [&](int i, uint32_t key, uint8_t raw, uint32_t mask, int off) {
    const int nb = i / G::kSlots, s = i - nb * G::kSlots;
    uint8_t sf = 0, spm = 0, cmk = 0;
    int ob = 0;
    if (key != kKeyNone) {
      const uint32_t kind = key >> 28, idx = key & 0x0FFFFFFFu;
      sf = kFPresent;
      if (kind == kKeyReal) {
        ob = 8 * (int)idx;
        spm = raw;
        const uint8_t bit = sBit[s];
        if (bit != 255 && ((mask >> (nb * G::kOcts + bit)) & 1)) sf |= kFTile;
      } else if (kind == kKeyInj) {
        cmk = 1;
        if (A.Wc != nullptr) {
          ob = (int)idx;
          sf |= kFInj;
        } else {
          st |= kStTree;  // plan/launch mismatch: never read through a null level
        }
      } else if (kind == kKeyInterp) {
        if (A.wv_inject) {  // gravity build: the coarse cell injected (its force is interpolated)
          cmk = 1;
          if (A.Wc != nullptr && A.vcell != nullptr) {
            ob = __ldg(A.vcell + 7 * (size_t)idx);
            sf |= kFInj;
          } else {
            st |= kStTree;
          }
        } else if (A.Wv != nullptr) {  // 8 interpolated sub-cells, laid out like an oct
          ob = 8 * (int)idx;
          sf |= kFInj | kFInterp;
        } else {
          st |= kStTree;
          cmk = 1;
        }
      } else {
        const int k0 = (int)(kind - kKeyGhost0);
        ob = 8 * (int)idx;
        cmk = (uint8_t)(2 + k0);
#pragma unroll
        for (int c = 0; c < 8; c++) spm |= (uint8_t)(((raw >> c_mirror[k0][c]) & 1) << c);
      }
    }
    sKey[off + i] = key;
    sOb[off + i] = ob;
    sSf[off + i] = sf;
    sSpm[off + i] = spm;
    sCmk[off + i] = cmk;
  };
  auto split_of = [&](uint32_t key) -> uint8_t {
    const uint32_t kind = key >> 28;
    return (key != kKeyNone && kind != kKeyInj && kind != kKeyInterp) ? A.split[key & 0x0FFFFFFFu] : (uint8_t)0;
  };
  if (!have) {
    const uint32_t mask = A.tiles[tile].mask;
    for (int i = tid; i < NS; i += kThreads) {
      const uint32_t key = A.keys[(size_t)tile * NS + i];
      build(i, key, split_of(key), mask, 0);
    }
    tile_sync<COH>();
  }
  {
    // Thread tid stages the pair q = tid & 3 of x-neighbour children (2q, 2q+1)
    // of slots tid/4 + 64 m, two cells per 16-byte load.  Ghost children come
    // from one pair of the boundary oct too (the mirror maps keep x-pairs).
    const int q = tid & 3, s0 = tid >> 2, c0 = 2 * q;
    const int cb = G::XX * ((q & 1) + G::XY * (q >> 1));
    unsigned mir = 0;  // per ghost face k, 4 bits: source pair, element of child c0, of child c0+1
#pragma unroll
    for (int k = 0; k < 6; k++) {
      const unsigned m0 = c_mirror[k][c0], m1 = c_mirror[k][c0 + 1];
      mir |= ((m0 >> 1) | ((m0 & 1) << 2) | ((m1 & 1) << 3)) << (4 * k);
    }
    const double *W = A.W, *Wc = A.Wc;
    const long long nc8 = A.nc8;
    constexpr int kIter = (4 * NS + kThreads - 1) / kThreads;
#pragma unroll
    for (int m = 0; m < kIter; m++) {
      const int sg = s0 + (kThreads / 4) * m;  // slot of the tile
      if (sg >= NS) break;
      const int nb = sg / G::kSlots, s = sg - nb * G::kSlots;
      const int b0 = nb * G::kBox + sBase[s] + cb;
      const uint8_t sf = sSf[sg];
      if (sf == 0) {
        sSt[b0] = 0;
        sSt[b0 + 1] = 0;
        continue;
      }
      const int cmk = sCmk[sg];
      double x0[5], x1[5];
      double t0[NTR > 0 ? NTR : 1] = {}, t1[NTR > 0 ? NTR : 1] = {};  // tracers of the two cells
      if (cmk == 1) {  // injected coarser cell: one value for both children
        const bool inj = sf & kFInj;
        const double *p = (inj ? Wc : W) + (long long)sOb[sg];
        const long long stride = inj ? nc8 : N8;
#pragma unroll
        for (int v = 0; v < 5; v++) x0[v] = x1[v] = ld_state<COH>(p + v * stride);
        if constexpr (TRACER) {
          const double *px = inj ? Xcs : Xs;
          const long long ts = inj ? nc8 : N8;
          if (px != nullptr) {
#pragma unroll
            for (int t = 0; t < NTR; t++) t0[t] = t1[t] = ld_state<COH>(px + t * ts + (long long)sOb[sg]);
          } else {
            st |= kStTree;
          }
        }
      } else {
        unsigned code = (unsigned)q | (1u << 3);  // pair q, elements 0 and 1
        if (cmk >= 2) code = (mir >> (4 * (cmk - 2))) & 15u;
        const bool itp = sf & kFInterp;
        const double *p = (itp ? A.Wv : W) + (long long)sOb[sg] + 2 * (code & 3);
        const long long stride = itp ? 8 * A.nv : N8;
        const bool e0 = (code >> 2) & 1, e1 = (code >> 3) & 1;
#pragma unroll
        for (int v = 0; v < 5; v++) {
          const double2 x = ld_state<COH>(reinterpret_cast<const double2 *>(p + v * stride));
          x0[v] = e0 ? x.y : x.x;
          x1[v] = e1 ? x.y : x.x;
        }
        if constexpr (TRACER) {
          if (!itp && Xs != nullptr) {
#pragma unroll
            for (int t = 0; t < NTR; t++) {
              const double2 x =
                  ld_state<COH>(reinterpret_cast<const double2 *>(Xs + t * N8 + (long long)sOb[sg] + 2 * (code & 3)));
              t0[t] = e0 ? x.y : x.x;
              t1[t] = e1 ? x.y : x.x;
            }
          } else {
            st |= kStTree;  // no tracer for interpolated coarser cells
          }
        }
      }
      if constexpr (TRACER) {  // X0 = dT / (d frac) (src/hydro_utils.c:1245, 1248-1251)
        if constexpr (SM::kR2) {  // only the cells a face reads
          const int xc0 = xc_of(b0), xc1 = xc_of(b0 + 1);
#pragma unroll
          for (int t = 0; t < NTR; t++) {
            if (xc0 >= 0) sX[t * SM::NXC + xc0] = (R)(t0[t] / (x0[0] * (TR::frac(t))));
            if (xc1 >= 0) sX[t * SM::NXC + xc1] = (R)(t1[t] / (x1[0] * (TR::frac(t))));
          }
        } else {
#pragma unroll
          for (int t = 0; t < NTR; t++) {
            sX[t * SM::NBOX + b0] = (R)(t0[t] / (x0[0] * (TR::frac(t))));
            sX[t * SM::NBOX + b0 + 1] = (R)(t1[t] / (x1[0] * (TR::frac(t))));
          }
        }
      }
      V::st(sW, b0, SM::NBOX, (R)x0[0], (R)x0[1], (R)x0[2], (R)x0[3]);
      V::st(sW, b0 + 1, SM::NBOX, (R)x1[0], (R)x1[1], (R)x1[2], (R)x1[3]);
      sWp[b0] = (R)x0[4];
      sWp[b0 + 1] = (R)x1[4];
      const uint8_t spm = sSpm[sg];
      uint8_t f0 = sf | (((spm >> c0) & 1) ? kFSplit : 0), f1 = sf | (((spm >> (c0 + 1)) & 1) ? kFSplit : 0);
      if constexpr (DUAL) {
        // split cells of the level whose stored sound speed is 0
        if (cmk != 1 && !(sf & kFInterp) && ((f0 | f1) & kFSplit)) {
          const bool all = A.azall != nullptr && ld_state<COH>(A.azall) != 0;
          unsigned code = (unsigned)q | (1u << 3);
          if (cmk >= 2) code = (mir >> (4 * (cmk - 2))) & 15u;
          const long long ib = (long long)sOb[sg] + 2 * (code & 3);
          const bool a0 = all || (A.az != nullptr && A.az[ib + ((code >> 2) & 1)]);
          const bool a1 = all || (A.az != nullptr && A.az[ib + ((code >> 3) & 1)]);
          if ((f0 & kFSplit) && a0) f0 |= kFAzero;
          if ((f1 & kFSplit) && a1) f1 |= kFAzero;
        }
      }
      sSt[b0] = f0;
      sSt[b0 + 1] = f1;
    }
  }
  tile_sync<COH>();
  // the next tile's slot keys and mask (consumed after the reconstruction phase)
  static_assert(NS <= kThreads, "one slot descriptor per thread");
  const bool pre = SM::kDB > 1 && next_tile >= 0 && tid < NS;
  uint32_t nkey = kKeyNone, nmask = 0;
  uint8_t nraw = 0;
  if (pre) {
    nmask = __ldg(&A.tiles[next_tile].mask);
    nkey = __ldg(A.keys + (size_t)next_tile * NS + tid);
  }

  auto q_at = [&](int b, R q[5]) {
    V::ld(sW, b, SM::NBOX, q[0], q[1], q[2], q[3]);
    q[4] = sWp[b];
  };
  // gravity kick -f dt/2 (the reference's expression, in FP64) of box cell b:
  // the force of the level's cell, or the interpolated force of an injected one
  const bool grav = GRAV && A.F != nullptr;
  auto kick_of = [&](int b, R g[3]) {
    const int nb = b / G::kBox, bl = b - nb * G::kBox;
    const int x2 = bl % G::XX, y2 = (bl / G::XX) % G::XY, z2 = bl / G::XS;
    const uint32_t key = sKey[nb * G::kSlots + (x2 >> 1) + G::SX * ((y2 >> 1) + G::SY * (z2 >> 1))];
    const long long off = 8LL * (key & 0x0FFFFFFFu) + ((x2 & 1) | ((y2 & 1) << 1) | ((z2 & 1) << 2));
    const uint32_t kind = key >> 28;
    const double *src = (kind == kKeyReal) ? A.F : ((kind == kKeyInterp) ? A.Fv : nullptr);
    const long long stride = (kind == kKeyReal) ? N8 : 8 * A.nv;
#pragma unroll
    for (int v = 0; v < 3; v++) {
      const double f = (key != kKeyNone && src != nullptr) ? ld_state<COH>(src + v * stride + off) : 0.;
      g[v] = (R)(-f * 0.5 * A.dt);
    }
  };

  // ------------------------------------------------------------------ P1
  // Items < kThreads: brick cell tid (slopes and predictor, when it is a leaf of
  // the tile or borders one); then the ring cells (the one face state each
  // contributes).  One call site each for the reconstruction and the face
  // state, so that a face on a brick boundary, solved by both bricks, rounds
  // the same in both.
#pragma unroll 1
  for (int w = tid; w < kThreads + NRING; w += kThreads) {
    int b = tb, k = 0, r = 0;
    bool need;
    if (w < kThreads) {
      const uint8_t f = sSt[tb];
      need = f_tileleaf(f);
      if (!need && recon_ok(f))
        need = f_tileleaf(sSt[tb - 1]) || f_tileleaf(sSt[tb + 1]) || f_tileleaf(sSt[tb - G::XX]) ||
               f_tileleaf(sSt[tb + G::XX]) || f_tileleaf(sSt[tb - G::XS]) || f_tileleaf(sSt[tb + G::XS]);
      if constexpr (F64) {  // the centre state, for the face states and the update
        R q[5];
        q_at(tb, q);
        V::st(sM, 5 * kThreads + tid, kThreads, q[0], q[1], q[2], q[3]);
        sMp[tid] = q[4];
      }
    } else {
      r = w - kThreads;
      const int nb = r / G::kRing;
      int bin;
      G::ring_cell(r - nb * G::kRing, b, k, bin);
      b += nb * G::kBox;
      bin += nb * G::kBox;
      need = recon_ok(sSt[b]) && f_tileleaf(sSt[bin]);
    }
    if (!need) continue;
    R q0[5], qm[3][5], qp[3][5], D[3][5], Wt[5], X[5];
    q_at(b, q0);
    q_at(b - 1, qm[0]);
    q_at(b + 1, qp[0]);
    q_at(b - G::XX, qm[1]);
    q_at(b + G::XX, qp[1]);
    q_at(b - G::XS, qm[2]);
    q_at(b + G::XS, qp[2]);
    const bool azero = DUAL && (sSt[b] & kFAzero);
    if constexpr (F64) M::muscl(q0, qm, qp, A.dt, A.dx, D, Wt, azero);
    else M::muscl(q0, qm, qp, (R)(A.dt / A.dx * 0.5), D, Wt, azero);
    // X = W0 + Wt (FP32 path) or Wt (FP64 path, which adds W0 in the reference's order)
#pragma unroll
    for (int v = 0; v < 5; v++) X[v] = F64 ? Wt[v] : q0[v] + Wt[v];
    R gk[3] = {(R)0, (R)0, (R)0};
    if (grav) {
      kick_of(b, gk);
      // FP32: the kick joins the predicted state, for the brick and the ring alike
      if constexpr (!F64) {
        X[1] += gk[0];
        X[2] += gk[1];
        X[3] += gk[2];
      }
    }
    if (w < kThreads) {
      // groups: D_x(d,u,v,w), D_y, D_z, X(d,u,v,w), (D_x.p, D_y.p, D_z.p, X.p)
#pragma unroll
      for (int dir = 0; dir < 3; dir++)
        V::st(sM, dir * kThreads + tid, kThreads, D[dir][0], D[dir][1], D[dir][2], D[dir][3]);
      V::st(sM, 3 * kThreads + tid, kThreads, X[0], X[1], X[2], X[3]);
      V::st(sM, 4 * kThreads + tid, kThreads, D[0][4], D[1][4], D[2][4], X[4]);
    } else {
      const int ax = k >> 1;
      R Dax[5], W[7];
#pragma unroll
      for (int v = 0; v < 5; v++) Dax[v] = (ax == 0) ? D[0][v] : ((ax == 1) ? D[1][v] : D[2][v]);
      if constexpr (F64) {
        M::face_ax(q0, Dax, Wt, k, W, st, grav ? gk : nullptr);
        V::st(sHS, r, NRING, W[0], W[1], W[2], W[3]);
        sHS[4 * NRING + r] = W[4];
      } else {
        M::face_px(X, Dax, k, W, st);
        V::st(sHS, r, NRING, W[0], W[1], W[2], W[3]);
        V::st(sHS, NRING + r, NRING, W[4], W[5], W[6], (R)0);
      }
    }
  }
  tile_sync<COH>();
  if (pre) nraw = split_of(nkey);
  // FP64 gravity: the kick of each brick cell once, for its six face states (the
  // box is dead after P1; the kicks sit after the face fluxes)
  R *sK = reinterpret_cast<R *>(smem + SM::off_K);
  if constexpr (F64 && GRAV) {
    if (grav) {
      R gk[3];
      kick_of(tb, gk);
      sK[tid] = gk[0];
      sK[kThreads + tid] = gk[1];
      sK[2 * kThreads + tid] = gk[2];
      tile_sync<COH>();
    }
  }

  // face state k of brick cell t (index into the tile's cells, box cell b)
  auto brick_face = [&](int t, int b, int k, R W[7]) {
    const int ax = k >> 1;
    R Dax[5], X[5], p0, p1, p2;
    V::ld(sM, ax * kThreads + t, kThreads, Dax[0], Dax[1], Dax[2], Dax[3]);
    V::ld(sM, 3 * kThreads + t, kThreads, X[0], X[1], X[2], X[3]);
    V::ld(sM, 4 * kThreads + t, kThreads, p0, p1, p2, X[4]);
    Dax[4] = (ax == 0) ? p0 : ((ax == 1) ? p1 : p2);
    if constexpr (F64) {
      R q0[5];
      V::ld(sM, 5 * kThreads + t, kThreads, q0[0], q0[1], q0[2], q0[3]);
      q0[4] = sMp[t];
      if (grav) {
        const R gk[3] = {sK[t], sK[kThreads + t], sK[2 * kThreads + t]};
        M::face_ax(q0, Dax, X, k, W, st, gk);
      } else {
        M::face_ax(q0, Dax, X, k, W, st);
      }
    } else {
      M::face_px(X, Dax, k, W, st);
    }
  };
  auto ring_face = [&](int r, R W[7]) {
    V::ld(sHS, r, NRING, W[0], W[1], W[2], W[3]);
    if constexpr (F64) {
      W[4] = sHS[4 * NRING + r];
      M::face_finish(W);
    } else {
      R pad;
      V::ld(sHS, NRING + r, NRING, W[4], W[5], W[6], pad);
    }
  };

  // One face e normal to axis d between left (brick cell tL at box cell bL, or
  // ring face jL) and right; the flux is zero across a split cell, and without a
  // leaf of the tile on either side the face is not solved.
  auto solve_face = [&](int d, int e, int tL, int bL, int jL, int tR, int bR, int jR) {
    const uint8_t fL = sSt[bL], fR = sSt[bR];
    R F[5] = {0, 0, 0, 0, 0}, du[2] = {0, 0}, fx[NTR > 0 ? NTR : 1] = {};
    if ((f_tileleaf(fL) || f_tileleaf(fR)) && recon_ok(fL) && recon_ok(fR)) {
      R WL[7], WR[7];
      if (jL >= 0) ring_face(jL, WL);
      else brick_face(tL, bL, 2 * d + 1, WL);
      if (jR >= 0) ring_face(jR, WR);
      else brick_face(tR, bR, 2 * d, WR);
      if constexpr (TRACER) {
        R xs[2 * NTR];
#pragma unroll
        for (int t = 0; t < NTR; t++) {
          if constexpr (SM::kR2) {
            xs[2 * t] = sX[t * SM::NXC + (jL >= 0 ? kThreads + jL : tL)];
            xs[2 * t + 1] = sX[t * SM::NXC + (jR >= 0 ? kThreads + jR : tR)];
          } else {
            xs[2 * t] = sX[t * SM::NBOX + bL];
            xs[2 * t + 1] = sX[t * SM::NBOX + bR];
          }
        }
        M::template hllc<NTR>(WL, WR, d, F, st, nullptr, xs, fx);
      } else {
        M::hllc(WL, WR, d, F, st, DUAL ? du : nullptr);
      }
      if (DUAL && !(f_ok(fL) && f_ok(fR))) {
#pragma unroll
        for (int v = 0; v < 5; v++) F[v] = (R)0;
        du[1] = (R)0;  // the internal-energy flux is cancelled too; u* stays for div(u)
      }
    }
    V::st(sF, e, SM::NFS, F[0], F[1], F[2], F[3]);
    sF1[e] = F[4];
    if constexpr (DUAL) {
      sF5[e] = du[0] * du[1];  // (Us.m_n / Us.d) ebar (src/hydro_utils.c:2128)
      sS[e] = du[0];
    }
    if constexpr (TRACER) {
#pragma unroll
      for (int t = 0; t < NTR; t++) sFX[t * SM::NFS + e] = fx[t];
    }
  };

  // ------------------------------------------------------------------ P2
  // FP32: per axis d (a compile-time constant, so the solver's axis selects fold): the
  // -d face of every brick cell, then the +d faces on the brick boundaries,
  // run by the last warps (z, then y, then x from the top).  One HLLC call site
  // per axis: a face on a brick boundary, solved by both bricks, rounds the same.
  auto solve_axis = [&](auto dc) {
    constexpr int d = decltype(dc)::value;
    constexpr int bs = (d == 0) ? 1 : ((d == 1) ? G::XX : G::XS);
    constexpr int ts = (d == 0) ? 1 : ((d == 1) ? G::CX : G::CX * G::CY);
    constexpr int nplus = G::kNB * ((d == 0) ? G::kPX : ((d == 1) ? G::kPY : G::kPZ));
    constexpr int start = kThreads - G::kNB * G::kPZ - ((d < 2) ? G::kNB * G::kPY : 0) - ((d < 1) ? G::kNB * G::kPX : 0);
    static_assert(start >= 0 && start + nplus <= kThreads, "plus faces fit the CTA");
#pragma unroll 1
    for (int pass = 0; pass < 2; pass++) {
      int e, tL, bL, jL = -1, tR, bR, jR = -1;
      if (pass == 0) {
        const int coord = (d == 0) ? tx : ((d == 1) ? ty : tz);
        e = tn * G::kFaces + G::face_index(d, tx, ty, tz);
        tR = tid;
        bR = tb;
        tL = tid - ts;
        bL = tb - bs;
        if (coord == 0) jL = tn * G::kRing + G::ring_index(d, false, tx, ty, tz);
      } else {
        const int p = tid - start;
        if (p < 0 || p >= nplus) break;
        constexpr int per = nplus / G::kNB;
        const int nb = p / per, j = p - nb * per;
        int x, y, z;
        if (d == 0) {
          x = G::CX - 1; y = j % G::CY; z = j / G::CY;
        } else if (d == 1) {
          x = j % G::CX; y = G::CY - 1; z = j / G::CX;
        } else {
          x = j % G::CX; y = j / G::CX; z = G::CZ - 1;
        }
        tL = nb * G::kCells + x + G::CX * (y + G::CY * z);
        bL = nb * G::kBox + G::box_of(x, y, z);
        tR = tL;
        bR = bL + bs;
        jR = nb * G::kRing + G::ring_index(d, true, x, y, z);
        e = nb * G::kFaces + G::face_index(d, x + (d == 0), y + (d == 1), z + (d == 2));
      }
      solve_face(d, e, tL, bL, jL, tR, bR, jR);
    }
  };
  // Two-round FP64 layout: this cell's sums over the faces of the rounds already
  // solved, in the faces' order -x,+x,-y,+y,-z,+z (the sums of P3 below, split after
  // the y faces), and the fine->coarse corrections of those faces
  double aU[5] = {0., 0., 0., 0., 0.}, aUe = 0., aDivu = 0., aX[NTR > 0 ? NTR : 1] = {};
  auto round_face = [&](int d, int nb, int x, int y, int z) {
    return (d < 2) ? nb * (G::kFX + G::kFY) + G::face_index(d, x, y, z)
                   : nb * G::kFZ + G::face_index(2, x, y, z) - (G::kFX + G::kFY);
  };
  auto face_sums = [&](int k0, int k1) {
    const uint8_t f = sSt[tb];
    if (!(f & kFTile) || (f & kFSplit)) return;
    const double dtsurdx = A.dt / A.dx;
    R q4;
    q4 = sMp[tid];
    const double eold = (double)q4 / (kGam - 1.);
#pragma unroll
    for (int k = k0; k < k1; k++) {
      const int d = k >> 1, up = k & 1;
      const int e = round_face(d, tn, tx + (d == 0 ? up : 0), ty + (d == 1 ? up : 0), tz + (d == 2 ? up : 0));
      const double one = up ? -1. : 1.;
      double F[5];
      {
        R f0, f1, f2, f3;
        V::ld(sF, e, SM::NFS, f0, f1, f2, f3);
        F[0] = (double)f0;
        F[1] = (double)f1;
        F[2] = (double)f2;
        F[3] = (double)f3;
        F[4] = (double)sF1[e];
      }
#pragma unroll
      for (int v = 0; v < 5; v++) aU[v] += F[v] * dtsurdx * one;
      if constexpr (DUAL) {
        aUe += (double)sF5[e] * dtsurdx * one;
        const double dl = (kGam - 1.) * (double)sS[e] * eold;
        aDivu += up ? dl : -dl;
      }
      if constexpr (TRACER) {
#pragma unroll
        for (int t = 0; t < NTR; t++) aX[t] += (double)sFX[t * SM::NFS + e] * dtsurdx * one;
      }
      // fine -> coarse correction into an unsplit coarser neighbour (src/hydro_utils.c:3206-3295)
      const int bs = (d == 0) ? 1 : ((d == 1) ? G::XX : G::XS);
      const int b2 = up ? tb + bs : tb - bs;
      if (!(sSt[b2] & kFInj) || A.Cc == nullptr) continue;
      const int bl = b2 - bo;
      const int x2 = bl % G::XX, y2 = (bl / G::XX) % G::XY, z2 = bl / G::XS;
      const uint32_t ck = sKey[tn * G::kSlots + (x2 >> 1) + G::SX * ((y2 >> 1) + G::SY * (z2 >> 1))];
      const long long cc = ((ck >> 28) == kKeyInterp) ? A.vcell[7 * (ck & 0x0FFFFFFFu)] : (ck & 0x0FFFFFFFu);
      const double cs = up ? 1. : -1.;
#pragma unroll
      for (int v = 0; v < 5; v++) atomicAdd(A.Cc + v * A.nc8 + cc, F[v] * dtsurdx * cs * 0.125);
      if constexpr (DUAL) atomicAdd(A.Cc + 5 * A.nc8 + cc, (double)sF5[e] * dtsurdx * cs * 0.125);
      if constexpr (TRACER) {
#pragma unroll
        for (int t = 0; t < NTR; t++)
          atomicAdd(A.Cc + (kXPlane + t) * A.nc8 + cc, (double)sFX[t * SM::NFS + e] * dtsurdx * cs * 0.125);
      }
    }
  };
  if constexpr (!F64) {
    solve_axis(std::integral_constant<int, 0>{});
    solve_axis(std::integral_constant<int, 1>{});
    solve_axis(std::integral_constant<int, 2>{});
  } else if constexpr (SM::kR2) {
    // FP64 with dual energy or tracers: the x and y faces, their sums, the z faces
    // (the axis at run time, one copy of the solver, as below)
#pragma unroll 1
    for (int round = 0; round < 2; round++) {
      const int nmain = (round == 0 ? 2 : 1) * kThreads;
      const int per = (round == 0) ? (G::kPX + G::kPY) : G::kPZ;
#pragma unroll 1
      for (int w = tid; w < nmain + G::kNB * per; w += kThreads) {
        int d, e, tL, bL, jL = -1, tR, bR, jR = -1;
        if (w < nmain) {
          d = (round == 0) ? w / kThreads : 2;
          const int bs = (d == 0) ? 1 : ((d == 1) ? G::XX : G::XS);
          const int ts = (d == 0) ? 1 : ((d == 1) ? G::CX : G::CX * G::CY);
          const int coord = (d == 0) ? tx : ((d == 1) ? ty : tz);
          e = round_face(d, tn, tx, ty, tz);
          tR = tid;
          bR = tb;
          tL = tid - ts;
          bL = tb - bs;
          if (coord == 0) jL = tn * G::kRing + G::ring_index(d, false, tx, ty, tz);
        } else {
          const int p = w - nmain, nb = p / per;
          int j = p - nb * per, x, y, z;
          if (round == 1) {
            d = 2; x = j % G::CX; y = j / G::CX; z = G::CZ - 1;
          } else if (j < G::kPX) {
            d = 0; x = G::CX - 1; y = j % G::CY; z = j / G::CY;
          } else {
            j -= G::kPX;
            d = 1; x = j % G::CX; y = G::CY - 1; z = j / G::CX;
          }
          const int bs = (d == 0) ? 1 : ((d == 1) ? G::XX : G::XS);
          tL = nb * G::kCells + x + G::CX * (y + G::CY * z);
          bL = nb * G::kBox + G::box_of(x, y, z);
          tR = tL;
          bR = bL + bs;
          jR = nb * G::kRing + G::ring_index(d, true, x, y, z);
          e = round_face(d, nb, x + (d == 0), y + (d == 1), z + (d == 2));
        }
        solve_face(d, e, tL, bL, jL, tR, bR, jR);
      }
      tile_sync<COH>();
      face_sums(round == 0 ? 0 : 4, round == 0 ? 4 : 6);
      if (round == 0) tile_sync<COH>();  // the z faces overwrite the arrays
    }
  } else {
    // FP64: one loop over all faces with the axis at run time (one copy of the
    // FP64 solver; three copies measured slower on trees with strong rarefactions)
    constexpr int kPlusTasks = G::kNB * G::kPlus;
#pragma unroll 1
    for (int w = tid; w < 3 * kThreads + kPlusTasks; w += kThreads) {
      int d, e, tL, bL, jL = -1, tR, bR, jR = -1;
      if (w < 3 * kThreads) {
        d = w / kThreads;
        const int bs = (d == 0) ? 1 : ((d == 1) ? G::XX : G::XS);
        const int ts = (d == 0) ? 1 : ((d == 1) ? G::CX : G::CX * G::CY);
        const int coord = (d == 0) ? tx : ((d == 1) ? ty : tz);
        e = tn * G::kFaces + G::face_index(d, tx, ty, tz);
        tR = tid;
        bR = tb;
        tL = tid - ts;
        bL = tb - bs;
        if (coord == 0) jL = tn * G::kRing + G::ring_index(d, false, tx, ty, tz);
      } else {
        const int p = w - 3 * kThreads, nb = p / G::kPlus;
        int j = p - nb * G::kPlus, x, y, z;
        if (j < G::kPX) {
          d = 0; x = G::CX - 1; y = j % G::CY; z = j / G::CY;
        } else if (j < G::kPX + G::kPY) {
          j -= G::kPX;
          d = 1; x = j % G::CX; y = G::CY - 1; z = j / G::CX;
        } else {
          j -= G::kPX + G::kPY;
          d = 2; x = j % G::CX; y = j / G::CX; z = G::CZ - 1;
        }
        const int bs = (d == 0) ? 1 : ((d == 1) ? G::XX : G::XS);
        tL = nb * G::kCells + x + G::CX * (y + G::CY * z);
        bL = nb * G::kBox + G::box_of(x, y, z);
        tR = tL;
        bR = bL + bs;
        jR = nb * G::kRing + G::ring_index(d, true, x, y, z);
        e = nb * G::kFaces + G::face_index(d, x + (d == 0), y + (d == 1), z + (d == 2));
      }
      solve_face(d, e, tL, bL, jL, tR, bR, jR);
    }
  }
  tile_sync<COH>();

  // ------------------------------------------------------------------ P3
  // In a batched launch the finer level's update (its corrections into C and
  // its new state, averaged into split cells here) must be complete first.
  if (A.wait_slot >= 0) {
    if (tid == 0) {
      const unsigned need = (unsigned)Bt.lv[A.wait_slot].ntiles;
      long long it = 0;
      while (*reinterpret_cast<volatile unsigned *>(Bt.done + A.wait_slot) < need) {
        if (++it > Bt.wait_limit) {
          st |= kStTimeout;
          break;
        }
        __nanosleep(64);
      }
      __threadfence();
    }
    tile_sync<COH>();
  }
  const uint8_t fme = sSt[tb];
  double smx = 0.;  // |v| + c_s of the state this thread writes
  if (fme & kFTile) {
    const int s = tn * G::kSlots + ((tx + 2) >> 1) + G::SX * (((ty + 2) >> 1) + G::SY * ((tz + 2) >> 1));
    const int c = (tx & 1) | ((ty & 1) << 1) | ((tz & 1) << 2);
    const long long gi = 8LL * (sKey[s] & 0x0FFFFFFFu) + c;
    double q[5];  // the FP64 state: staged (plain path) or read again from L2 (mixed path)
    if constexpr (F64) {
      V::ld(sM, 5 * kThreads + tid, kThreads, q[0], q[1], q[2], q[3]);
      q[4] = sMp[tid];
    } else {
#pragma unroll
      for (int v = 0; v < 5; v++) q[v] = ld_state<COH>(A.W + v * N8 + gi);
    }
    double Wout[5];
    double Xout[NTR > 0 ? NTR : 1] = {};  // the new tracers
    if (fme & kFSplit) {
      if constexpr (TRACER) {
        // the children's mean (src/hydro_utils.c:3446-3460) when the finer level is at hand
        const long long ch = (A.Wf != nullptr && res_tr) ? A.child[gi] : -1;
#pragma unroll
        for (int t = 0; t < NTR; t++) {
          Xout[t] = (Xs != nullptr) ? ld_state<COH>(Xs + t * N8 + gi) : 0.;
          if (ch >= 0) {
            double ax = 0.;
            for (int i = 0; i < 8; i++) ax += __ldcg(A.Wf + (5 + t) * A.nf8 + 8 * ch + i) * 0.125;
            Xout[t] = ax;
          }
        }
      }
      // split cell: primitive mean of the 8 children (src/hydro_utils.c:3420-3481);
      // without the finer level (drop-in mode) the caller averages on the host
      double acc[5] = {0., 0., 0., 0., 0.};
      if (A.Wf == nullptr) {
#pragma unroll
        for (int v = 0; v < 5; v++) acc[v] = q[v];
      } else {
        const long long ch = A.child[gi];
        if (ch >= 0) {
          for (int i = 0; i < 8; i++)
#pragma unroll
            for (int v = 0; v < 5; v++) acc[v] += __ldcg(A.Wf + v * A.nf8 + 8 * ch + i) * 0.125;
        } else {
          st |= kStTree;
        }
      }
#pragma unroll
      for (int v = 0; v < 5; v++) Wout[v] = acc[v];
    } else {
      const double dtsurdx = A.dt / A.dx;
      // face e of this cell: -x,+x,-y,+y,-z,+z
      const int eb = tn * G::kFaces;
      const int ex = eb + G::face_index(0, tx, ty, tz), ey = eb + G::face_index(1, tx, ty, tz),
                ez = eb + G::face_index(2, tx, ty, tz);
      auto flux5 = [&](int k, double F[5]) {
        const int e = (k < 2) ? (ex + (k & 1)) : ((k < 4) ? (ey + G::CX * (k & 1)) : (ez + G::CX * G::CY * (k & 1)));
        R f0, f1, f2, f3;
        V::ld(sF, e, SM::NFS, f0, f1, f2, f3);
        F[0] = (double)f0;
        F[1] = (double)f1;
        F[2] = (double)f2;
        F[3] = (double)f3;
        F[4] = (double)sF1[e];
      };
      auto face_of = [&](int k) {
        return (k < 2) ? (ex + (k & 1)) : ((k < 4) ? (ey + G::CX * (k & 1)) : (ez + G::CX * G::CY * (k & 1)));
      };
      // correction plane v of this cell, received from the finer level; with
      // Bt.zero_c the planes read nonzero are cleared after the update (below), so
      // that the level's corrections are zero again when the finer level next runs
      // (the fused coarse step clears no buffer).  The stores wait until every plane
      // is read: a store between the loads would hold the later loads back.
      unsigned cnz = 0u;
      auto take_c = [&](int v) -> double {
        const double c = __ldcg(A.C + v * N8 + gi);
        if (c != 0.) cnz |= 1u << v;
        return c;
      };
      double Ud, Udu, Udv, Udw, UE;
      double Ue = 0.;  // dual energy: the tracked internal energy of the base state
      if (A.B != nullptr) {  // drop-in: W2U of the caller's fieldnew
        const double bd = A.B[gi];
        Ud = bd;
        Udu = bd * A.B[N8 + gi];
        Udv = bd * A.B[2 * N8 + gi];
        Udw = bd * A.B[3 * N8 + gi];
        UE = A.B[5 * N8 + gi];
        if constexpr (DUAL) Ue = A.B[4 * N8 + gi] / (kGam - 1.);
      } else {  // resident: W2U(field) + corrections received from the finer level
        Ud = q[0];
        Udu = q[0] * q[1];
        Udv = q[0] * q[2];
        Udw = q[0] * q[3];
        UE = q[4] / (kGam - 1.) + 0.5 * q[0] * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
        if constexpr (DUAL) {
          Ue = q[4] / (kGam - 1.);
          if (A.C != nullptr) Ue += take_c(5);
        }
      }
      // dual energy (src/hydro_utils.c:2126-2129, 3064, 3167-3177): the internal-energy
      // flux divergence and the p div(u) term, summed over the faces in the
      // reference's order (x-, x+, y-, y+, z-, z+), eold the cell's old eint
      double dUe = 0., divu = 0.;
      if constexpr (DUAL && SM::kR2) {  // summed round by round (face_sums)
        dUe = aUe;
        divu = aDivu;
      } else if constexpr (DUAL) {
        const double eold = q[4] / (kGam - 1.);
        double one = 1.;
#pragma unroll
        for (int k = 0; k < 6; k++) {
          const int e = face_of(k);
          dUe += (double)sF5[e] * dtsurdx * one;
          const double dl = (kGam - 1.) * (double)sS[e] * eold;
          divu += (k & 1) ? dl : -dl;
          one *= -1.;
        }
      }
      if constexpr (F64) {
        // updatefield (src/hydro_utils.c:3050-3082): dU = sum over faces -x,+x,-y,+y,-z,+z
        // of (+-F dt/dx), signs alternating from +
        double dU[5] = {0., 0., 0., 0., 0.};
        if constexpr (SM::kR2) {  // summed round by round (face_sums)
#pragma unroll
          for (int v = 0; v < 5; v++) dU[v] = aU[v];
        } else {
          double one = 1.;
#pragma unroll
          for (int k = 0; k < 6; k++) {
            double F[5];
            flux5(k, F);
#pragma unroll
            for (int v = 0; v < 5; v++) dU[v] += F[v] * dtsurdx * one;
            one *= -1.;
          }
        }
        // scatterstencil central update (src/hydro_utils.c:3129-3188), reference order
        if (A.B == nullptr && A.C != nullptr) {
          Ud += take_c(0);
          Udu += take_c(1);
          Udv += take_c(2);
          Udw += take_c(3);
          UE += take_c(4);
        }
        Ud += dU[0];
        Udu += dU[1];
        Udv += dU[2];
        Udw += dU[3];
        UE += dU[4];
      } else {
        // mixed: FP32 face fluxes, their divergence accumulated in FP64 and added to
        // the FP64 conserved state with Neumaier-compensated summation (base + corrections + dU)
        double dU[5] = {0., 0., 0., 0., 0.};
#pragma unroll
        for (int k = 0; k < 6; k++) {
          double F[5];
          flux5(k, F);
#pragma unroll
          for (int v = 0; v < 5; v++) dU[v] = (k & 1) ? dU[v] - F[v] : dU[v] + F[v];
        }
        double sum[5] = {Ud, Udu, Udv, Udw, UE}, comp[5] = {0., 0., 0., 0., 0.};
        auto add = [&](int v, double x) {
          const double t = sum[v] + x;
          comp[v] += (fabs(sum[v]) >= fabs(x)) ? ((sum[v] - t) + x) : ((x - t) + sum[v]);
          sum[v] = t;
        };
        if (A.B == nullptr && A.C != nullptr) {
#pragma unroll
          for (int v = 0; v < 5; v++) add(v, take_c(v));
        }
#pragma unroll
        for (int v = 0; v < 5; v++) add(v, dU[v] * dtsurdx);
        Ud = sum[0] + comp[0];
        Udu = sum[1] + comp[1];
        Udv = sum[2] + comp[2];
        Udw = sum[3] + comp[3];
        UE = sum[4] + comp[4];
      }
      // U2W (src/hydro_utils.c:35-64), pressure floor, E - Ekin recovery
      const double dl = (Ud == 0. ? 10. : Ud);
      Wout[0] = Ud;
      if constexpr (F64) {
        Wout[1] = Udu / dl;
        Wout[2] = Udv / dl;
        Wout[3] = Udw / dl;
        Wout[4] = (kGam - 1.) * (UE - ((Udu) * (Udu) + (Udv) * (Udv) + (Udw) * (Udw)) / (dl) * 0.5);
      } else {
        const double inv = 1. / dl;  // mixed path: one FP64 division per cell
        Wout[1] = Udu * inv;
        Wout[2] = Udv * inv;
        Wout[3] = Udw * inv;
        Wout[4] = (kGam - 1.) * (UE - (Udu * Udu + Udv * Udv + Udw * Udw) * inv * 0.5);
      }
      if constexpr (DUAL) {
        // the tracked eint, unless E - Ekin is well resolved against div(u); the
        // floor; the pressure from eint (src/hydro_utils.c:3164-3182, 45-46)
        const double ekin = 0.5 * (Udu * Udu + Udv * Udv + Udw * Udw) / Ud;
        double eint = Ue + dUe;
        eint = eint + (-divu * dtsurdx);
        if ((UE - ekin) > 0.5 * (divu * divu)) eint = UE - ekin;
        eint = fmax(eint * (kGam - 1.), kPmin) / (kGam - 1.);
        Wout[4] = eint * (kGam - 1.);
      }
      Wout[4] = fmax(Wout[4], kPmin);
      if (isnan(Wout[1]) || isnan(Wout[4]) || isnan(Wout[0])) st |= kStNan;
      // grav_correction (src/hydro_utils.c:2388-2444, PRIMITIVE): full-step kick of the
      // leaf velocities after the update, before the next step's CFL term
      if (A.gcorr && grav) {
#pragma unroll
        for (int v = 0; v < 3; v++) Wout[1 + v] += (-ld_state<COH>(A.F + v * N8 + gi) * A.dt);
      }
      if constexpr (TRACER) {
        // tracers: the caller's fieldnew (or field + corrections) plus the flux
        // divergence in the faces' order (src/hydro_utils.c:3068-3072, 3158-3162),
        // then dX in [0, d (1 - YHE)] and the helium densities below d YHE
        // (:3197-3203)
#pragma unroll
        for (int t = 0; t < NTR; t++) {
          double Ux = (A.BX != nullptr) ? A.BX[t * N8 + gi] : ((Xs != nullptr) ? ld_state<COH>(Xs + t * N8 + gi) : 0.);
          if (A.BX == nullptr && A.C != nullptr) Ux += take_c(kXPlane + t);
          double dUx = 0., one = 1.;
          if constexpr (SM::kR2) {  // summed round by round (face_sums)
            dUx = aX[t];
          } else {
#pragma unroll
            for (int k = 0; k < 6; k++) {
              dUx += (double)sFX[t * SM::NFS + face_of(k)] * dtsurdx * one;
              one *= -1.;
            }
          }
          double x = Ux + dUx;
          if (t == 0 && x < 0) x = 0.;
          if (x > (Wout[0] * (TR::frac(t)))) x = Wout[0] * (TR::frac(t));
          Xout[t] = x;
        }
      }

      // fine -> coarse correction into unsplit coarser neighbours (src/hydro_utils.c:3206-3295);
      // the two-round layout sent them with its sums
#pragma unroll
      for (int k = 0; k < (SM::kR2 ? 0 : 6); k++) {
        const int bs = (k < 2) ? 1 : ((k < 4) ? G::XX : G::XS);
        const int b2 = (k & 1) ? tb + bs : tb - bs;
        if (!(sSt[b2] & kFInj) || A.Cc == nullptr) continue;
        const int bl = b2 - bo;
        const int x2 = bl % G::XX, y2 = (bl / G::XX) % G::XY, z2 = bl / G::XS;
        const uint32_t ck = sKey[tn * G::kSlots + (x2 >> 1) + G::SX * ((y2 >> 1) + G::SY * (z2 >> 1))];
        const long long cc = ((ck >> 28) == kKeyInterp) ? A.vcell[7 * (ck & 0x0FFFFFFFu)] : (ck & 0x0FFFFFFFu);
        const double one = (k & 1) ? 1. : -1.;
        double F[5];
        flux5(k, F);
#pragma unroll
        for (int v = 0; v < 5; v++) atomicAdd(A.Cc + v * A.nc8 + cc, F[v] * dtsurdx * one * 0.125);
        if constexpr (DUAL) atomicAdd(A.Cc + 5 * A.nc8 + cc, (double)sF5[face_of(k)] * dtsurdx * one * 0.125);
        if constexpr (TRACER) {
#pragma unroll
          for (int t = 0; t < NTR; t++)
            atomicAdd(A.Cc + (kXPlane + t) * A.nc8 + cc, (double)sFX[t * SM::NFS + face_of(k)] * dtsurdx * one * 0.125);
        }
      }
      if (Bt.zero_c)
        for (unsigned m = cnz; m != 0u; m &= m - 1u) A.C[(__ffs(m) - 1) * N8 + gi] = 0.;
    }
#pragma unroll
    for (int v = 0; v < 5; v++) A.Wn[v * N8 + gi] = Wout[v];
    if constexpr (TRACER) {
      if (Xns != nullptr) {
#pragma unroll
        for (int t = 0; t < NTR; t++) Xns[t * N8 + gi] = Xout[t];
      }
    }
    if (Bt.smax != nullptr) {
      // the next time step's CFL term of this cell, as L_comptstep_hydro evaluates it
      // (src/advanceamr.c:122-128): IEEE operations, no contraction
      const double va = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(Wout[1], Wout[1]), __dmul_rn(Wout[2], Wout[2])),
                                             __dmul_rn(Wout[3], Wout[3])));
      const double aa = __dsqrt_rn(__ddiv_rn(__dmul_rn(5. / 3., Wout[4]), Wout[0]));
      smx = fmax(smx, __dadd_rn(va, aa));  // fmax drops NaN like the reference's FMAX
    }
  }
  if (Bt.smax != nullptr) {
    for (int o = 16; o > 0; o >>= 1) smx = fmax(smx, __shfl_xor_sync(0xffffffffu, smx, o));
    if ((tid & 31) == 0 && smx > 0.)
      atomicMax(sSmax + slot, (unsigned long long)__double_as_longlong(smx));
  }
  if (pre) build(tid, nkey, nraw, nmask, nxt);
  tile_sync<COH>();
  if (tid == 0) {
    __threadfence();
    atomicAdd(Bt.done + slot, 1u);
  }
  have = SM::kDB > 1 && next_tile >= 0;
  if (have) cur ^= 1;
}

// Bytes of dynamic shared memory of a kernel handling the shapes in `shapes`
// (bit i: kShapes[i]).
template <class M, bool DUAL = false, int NTR = 0>
constexpr size_t level_smem_bytes(unsigned shapes) {
  const size_t a = (shapes & 1u) ? TileSmem<M, GeomA, DUAL, NTR>::bytes : 0,
               b = (shapes & 2u) ? TileSmem<M, GeomB, DUAL, NTR>::bytes : 0;
  return a > b ? a : b;
}

// Persistent launch over a work list of (level slot, tile) items.  All CTAs are
// co-resident (grid <= occupancy x SMs) and take items in list order, so a
// tile waiting for a finer level (listed first) never blocks the CTAs that
// still have to finish that level.  SHAPES: the brick shapes the levels of the
// launch use (bit i: kShapes[i]); each level's plan names its own.
// Occupancy targets: the FP32 kernel with 4x4x2 bricks only fits 4 CTAs per SM
// (64 registers, 55 KB of shared memory); with 2x2x2 bricks shared memory
// allows 2; the FP64 kernel 2 with 4x4x2 bricks (128 registers, 110 KB; its
// dual-energy and single-tracer variants too, through their two-round layout), 1
// with 2x2x2 bricks.
template <class M, unsigned SHAPES, bool DUAL = false, int NTR = 0>
constexpr int kMinBlocks = (sizeof(typename M::R) == 8) ? ((SHAPES == 1u && NTR <= 1) ? 2 : 1)
                                                         : (SHAPES == 1u ? (NTR == 3 ? 2 : ((DUAL || NTR > 0) ? 3 : 4))
                                                                         : (NTR == 3 ? 1 : 2));
// 228 KB of shared memory per SM, 1 KB reserved per CTA
static_assert(4 * (TileSmem<MathF32, GeomA>::bytes + 1024) <= 228 * 1024, "4 FP32 4x4x2 CTAs per SM");
static_assert(2 * (TileSmem<MathF32, GeomB>::bytes + 1024) <= 228 * 1024, "2 FP32 2x2x2 CTAs per SM");
static_assert(2 * (TileSmem<MathF64, GeomA>::bytes + 1024) <= 228 * 1024, "2 FP64 4x4x2 CTAs per SM");
static_assert(2 * (TileSmem<MathF64, GeomA, true>::bytes + 1024) <= 228 * 1024, "2 dual-energy FP64 4x4x2 CTAs");
static_assert(2 * (TileSmem<MathF64, GeomA, false, 1>::bytes + 1024) <= 228 * 1024, "2 tracer FP64 4x4x2 CTAs");
static_assert(3 * (TileSmem<MathF32, GeomA, true>::bytes + 1024) <= 228 * 1024, "3 dual-energy FP32 4x4x2 CTAs");
static_assert(2 * (TileSmem<MathF32, GeomB, true>::bytes + 1024) <= 228 * 1024, "2 dual-energy FP32 2x2x2 CTAs");
static_assert(TileSmem<MathF64, GeomB, true>::bytes + 1024 <= 227 * 1024, "a dual-energy FP64 2x2x2 CTA");
static_assert(3 * (TileSmem<MathF32, GeomA, false, 1>::bytes + 1024) <= 228 * 1024, "3 tracer FP32 4x4x2 CTAs");
static_assert(2 * (TileSmem<MathF32, GeomB, false, 1>::bytes + 1024) <= 228 * 1024, "2 tracer FP32 2x2x2 CTAs");
static_assert(TileSmem<MathF64, GeomB, false, 1>::bytes + 1024 <= 227 * 1024, "a tracer FP64 2x2x2 CTA");
static_assert(2 * (TileSmem<MathF32, GeomA, false, 3>::bytes + 1024) <= 228 * 1024, "2 helium FP32 4x4x2 CTAs");
static_assert(TileSmem<MathF32, GeomB, false, 3>::bytes + 1024 <= 227 * 1024, "a helium FP32 2x2x2 CTA");
static_assert(TileSmem<MathF64, GeomA, false, 3>::bytes + 1024 <= 227 * 1024, "a helium FP64 4x4x2 CTA");
static_assert(TileSmem<MathF64, GeomB, false, 3>::bytes + 1024 <= 227 * 1024, "a helium FP64 2x2x2 CTA");

template <class M, unsigned SHAPES, bool GRAV, bool DUAL, int NTR = 0>
__global__ void __launch_bounds__(kThreads, (kMinBlocks<M, SHAPES, DUAL, NTR>))
    level_batch_kernel(const BatchArgs Bt) {
  extern __shared__ __align__(16) unsigned char smem[];
  if (Bt.gate != nullptr && *Bt.gate == 0) return;
  if constexpr ((SHAPES & 1u) != 0) slot_tables<GeomA>(smem);
  if constexpr ((SHAPES & 2u) != 0) slot_tables<GeomB>(smem + kTabOffB);
  unsigned long long *sSmax = reinterpret_cast<unsigned long long *>(smem + kSmaxOff);
  if (threadIdx.x < kMaxLevels) sSmax[threadIdx.x] = 0ULL;
  __syncthreads();
  unsigned st = 0;
  int cur = 0, args_slot = -1;
  bool have = false;
  constexpr int kTileMask = (1 << kWorkSlotShift) - 1;
  // Work queue: items are taken in list order, one ticket per item.  A CTA holds
  // the ticket of its tile and of the next one (whose descriptors it prefetches
  // if it is on the same level) and asks for the one after while it works, so
  // the atomic's latency hides behind the tile.  Slot 0 of the per-CTA maxima (no
  // level 0) passes tickets on.  Tickets rise along the list, finest level
  // first: a tile waiting for a finer level holds no finer item.
  volatile int *sTicket = reinterpret_cast<volatile int *>(sSmax);
  if (threadIdx.x == 0) {
    sTicket[0] = (int)atomicAdd(Bt.ticket, 1u);
    sTicket[1] = (int)atomicAdd(Bt.ticket, 1u);
  }
  __syncthreads();
  int w = sTicket[0], wn = sTicket[1];
  while (w < Bt.nwork) {
    unsigned wnn = 0u;
    if (threadIdx.x == 0) wnn = atomicAdd(Bt.ticket, 1u);  // read after the tile
    const int item = Bt.work[w];
    const int slot = item >> kWorkSlotShift, tile = item & kTileMask;
    int next_tile = -1;
    if (wn < Bt.nwork) {
      const int itn = Bt.work[wn];
      if ((itn >> kWorkSlotShift) == slot) next_tile = itn & kTileMask;
    }
    const LevelArgs *gA = Bt.lv + slot;
    if constexpr (SHAPES == 1u) {
      level_tile<M, GeomA, GRAV, DUAL, NTR>(Bt, gA, slot, tile, next_tile, smem, smem, sSmax, st, cur, have,
                                               args_slot);
    } else if constexpr (SHAPES == 2u) {
      level_tile<M, GeomB, GRAV, DUAL, NTR>(Bt, gA, slot, tile, next_tile, smem, smem + kTabOffB, sSmax, st, cur,
                                               have, args_slot);
    } else {
      if (gA->shape == 0)
        level_tile<M, GeomA, GRAV, DUAL, NTR>(Bt, gA, slot, tile, next_tile, smem, smem, sSmax, st, cur, have,
                                                 args_slot);
      else
        level_tile<M, GeomB, GRAV, DUAL, NTR>(Bt, gA, slot, tile, next_tile, smem, smem + kTabOffB, sSmax, st,
                                                 cur, have, args_slot);
    }
    if (threadIdx.x == 0) sTicket[0] = (int)wnn;  // every thread read sTicket before the tile's barriers
    __syncthreads();
    w = wn;
    wn = sTicket[0];
  }
  // non-negative doubles order like their bit patterns
  if (Bt.smax != nullptr && threadIdx.x > 0 && threadIdx.x < kMaxLevels && sSmax[threadIdx.x] != 0ULL)
    atomicMax(Bt.smax + threadIdx.x, sSmax[threadIdx.x]);
  if (st) atomicOr(Bt.status, st);
  // the last CTA to finish puts the queue back for the next launch
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(Bt.ticket + 1, 1u) == gridDim.x - 1) {
      Bt.ticket[0] = 0u;
      Bt.ticket[1] = 0u;
      __threadfence();
    }
  }
}

}  // namespace emma

namespace emma {
// The launchers have internal linkage: their occupancy cache is a static local,
// and a template's static local would otherwise be one object for every library
// of the process that holds the same instantiation (libemmahydro.so and
// libemmahydro_grav.so share these object files), so the second library would
// skip setting its own kernel's shared-memory limit.
namespace {

// Launch of a work list on a persistent grid of ctas_per_sm CTAs per SM (0 or
// above the occupancy limit: the limit), so that every CTA is co-resident.
template <class M, unsigned SHAPES, bool GRAV, bool DUAL, int NTR = 0>
cudaError_t launch_level_shapes(const BatchArgs &a, int nsm, int ctas_per_sm, cudaStream_t s, int *occupancy) {
  // per device: the shared-memory limit is a per-device function attribute, and the
  // co-residency of the persistent grid rests on that device's own occupancy
  constexpr int kMaxDev = 64;
  static int occ_dev[kMaxDev] = {0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDev) return cudaErrorInvalidDevice;
  int &occ = occ_dev[dev];
  auto k = level_batch_kernel<M, SHAPES, GRAV, DUAL, NTR>;
  constexpr size_t bytes = level_smem_bytes<M, DUAL, NTR>(SHAPES);
  if (occ == 0) {
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    int o = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k, kThreads, bytes);
    if (e != cudaSuccess) return e;
    if (o < 1) return cudaErrorInvalidConfiguration;
    occ = o;
  }
  if (occupancy != nullptr) *occupancy = occ;
  if (a.nwork == 0) return cudaSuccess;
  const int per = (ctas_per_sm > 0 && ctas_per_sm < occ) ? ctas_per_sm : occ;
  int grid = per * nsm;
  if (grid > a.nwork) grid = a.nwork;
  k<<<grid, kThreads, bytes, s>>>(a);
  return cudaGetLastError();
}

template <class M>
cudaError_t launch_level_any(const BatchArgs &a, unsigned shapes, int nsm, int ctas_per_sm, cudaStream_t s,
                             int *occupancy) {
  constexpr unsigned G = kLaunchGrav, D = kLaunchDual, T = kLaunchTracer, H = kLaunchHelium;
  switch (shapes) {
    case 1u | T: return launch_level_shapes<M, 1u, false, false, 1>(a, nsm, ctas_per_sm, s, occupancy);
    case 2u | T: return launch_level_shapes<M, 2u, false, false, 1>(a, nsm, ctas_per_sm, s, occupancy);
    case 3u | T: return launch_level_shapes<M, 3u, false, false, 1>(a, nsm, ctas_per_sm, s, occupancy);
    case 1u | H: return launch_level_shapes<M, 1u, false, false, 3>(a, nsm, ctas_per_sm, s, occupancy);
    case 2u | H: return launch_level_shapes<M, 2u, false, false, 3>(a, nsm, ctas_per_sm, s, occupancy);
    case 3u | H: return launch_level_shapes<M, 3u, false, false, 3>(a, nsm, ctas_per_sm, s, occupancy);
    case 1u: return launch_level_shapes<M, 1u, false, false>(a, nsm, ctas_per_sm, s, occupancy);
    case 2u: return launch_level_shapes<M, 2u, false, false>(a, nsm, ctas_per_sm, s, occupancy);
    case 3u: return launch_level_shapes<M, 3u, false, false>(a, nsm, ctas_per_sm, s, occupancy);
    case 1u | G: return launch_level_shapes<M, 1u, true, false>(a, nsm, ctas_per_sm, s, occupancy);
    case 2u | G: return launch_level_shapes<M, 2u, true, false>(a, nsm, ctas_per_sm, s, occupancy);
    case 3u | G: return launch_level_shapes<M, 3u, true, false>(a, nsm, ctas_per_sm, s, occupancy);
    case 1u | D: return launch_level_shapes<M, 1u, false, true>(a, nsm, ctas_per_sm, s, occupancy);
    case 2u | D: return launch_level_shapes<M, 2u, false, true>(a, nsm, ctas_per_sm, s, occupancy);
    case 3u | D: return launch_level_shapes<M, 3u, false, true>(a, nsm, ctas_per_sm, s, occupancy);
    case 1u | G | D: return launch_level_shapes<M, 1u, true, true>(a, nsm, ctas_per_sm, s, occupancy);
    case 2u | G | D: return launch_level_shapes<M, 2u, true, true>(a, nsm, ctas_per_sm, s, occupancy);
    case 3u | G | D: return launch_level_shapes<M, 3u, true, true>(a, nsm, ctas_per_sm, s, occupancy);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace
}  // namespace emma
