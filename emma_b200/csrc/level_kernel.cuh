// level_kernel.cuh -- the hydro level advance on the GPU, one CTA per tile.
//
// A tile is a brick of 4x4x2 oct positions of one level (8x8x4 cells, one
// thread per cell) holding at least one oct of the level.  Each CTA:
//   P0  stages a 6x6x4-slot box (the brick and a ring of one oct) of "virtual
//       octs": a real oct of the level, a coarser leaf cell injected into 8
//       cells as the reference's gather does, or a transmissive mirror ghost;
//       only the slots a stencil reads (faces and edges of the tile octs) are
//       filled.  Neighbours are then fixed offsets in the 12x12x8-cell box;
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
#include "hydro_math.cuh"
#include "plan_types.h"

namespace emma {

// 4-wide shared-memory groups: one 128-bit access per group for FP32 (float4),
// two for FP64 (double2 pairs).
template <class R>
struct Q4;
template <>
struct Q4<float> {
  static __device__ __forceinline__ void st(float *b, int i, float x, float y, float z, float w) {
    reinterpret_cast<float4 *>(b)[i] = make_float4(x, y, z, w);
  }
  static __device__ __forceinline__ void ld(const float *b, int i, float &x, float &y, float &z, float &w) {
    const float4 v = reinterpret_cast<const float4 *>(b)[i];
    x = v.x;
    y = v.y;
    z = v.z;
    w = v.w;
  }
};
template <>
struct Q4<double> {
  static __device__ __forceinline__ void st(double *b, int i, double x, double y, double z, double w) {
    reinterpret_cast<double2 *>(b)[2 * i] = make_double2(x, y);
    reinterpret_cast<double2 *>(b)[2 * i + 1] = make_double2(z, w);
  }
  static __device__ __forceinline__ void ld(const double *b, int i, double &x, double &y, double &z, double &w) {
    const double2 a = reinterpret_cast<const double2 *>(b)[2 * i];
    const double2 c = reinterpret_cast<const double2 *>(b)[2 * i + 1];
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

// cell flags of the staged box
constexpr uint8_t kFPresent = 1, kFSplit = 2, kFTile = 4, kFInj = 8;
__device__ __forceinline__ bool f_ok(uint8_t f) { return (f & (kFPresent | kFSplit)) == kFPresent; }
__device__ __forceinline__ bool f_tileleaf(uint8_t f) {
  return (f & (kFPresent | kFSplit | kFTile)) == (kFPresent | kFTile);
}

// Shared memory of one brick.  Brick cell t = x + 8 (y + 8 z) sits at box cell
// (x+2) + 12 ((y+2) + 12 (z+2)).  Ring cell j (face-adjacent to the brick):
// j < 32 -x side (y + 8 z), 32.. +x side, 64.. -y (x + 8 z), 96.. +y,
// 128.. -z (x + 8 y), 192.. +z.  Face arrays, -d face of brick cell (x,y,z):
// x: x + 9 (y + 8 z), y: 288 + x + 8 (y + 9 z), z: 576 + x + 8 (y + 8 z),
// with coordinate 8 (x, y) or 4 (z) for the + faces on the brick boundary.
template <class M>
struct BrickSmem {
  using R = typename M::R;
  static constexpr bool kF64 = sizeof(R) == 8;
  static constexpr size_t a16(size_t x) { return (x + 15) & ~size_t(15); }
  static constexpr size_t off_args = 0;                                          // LevelArgs of the tile's level
  static constexpr size_t off_key = a16(off_args + sizeof(LevelArgs));           // u32 [kSlots]
  static constexpr size_t off_ob = a16(off_key + 4 * kSlots);                    // i32 [kSlots] source offset
  static constexpr size_t off_sf = a16(off_ob + 4 * kSlots);                     // u8  [kSlots] slot flags
  static constexpr size_t off_spm = a16(off_sf + kSlots);                        // u8  [kSlots] split mask (cell order)
  static constexpr size_t off_cmk = a16(off_spm + kSlots);                       // u8  [kSlots] cell map
  static constexpr size_t off_sbase = a16(off_cmk + kSlots);                     // u16 [kSlots] box cell of child 0
  static constexpr size_t off_sbit = a16(off_sbase + 2 * kSlots);                // u8  [kSlots] brick position or 255
  static constexpr size_t off_tbase = a16(off_sbit + kSlots);                    // u8  [kSlots] brick cell of child 0
  static constexpr size_t off_st = a16(off_tbase + kSlots);                      // u8  [kBox] cell flags
  static constexpr size_t off_W = a16(off_st + kBox);                            // R4  [kBox] (d,u,v,w)
  static constexpr size_t off_Wp = a16(off_W + sizeof(R) * 4 * kBox);            // R   [kBox] p
  static constexpr size_t off_M = a16(off_Wp + sizeof(R) * kBox);                // R4  [5][kNT] slopes, predictor
  static constexpr size_t off_HS = a16(off_M + sizeof(R) * 4 * 5 * kNT);         // R4  [2][kHaloCells] ring faces
  static constexpr size_t off_Q = a16(off_HS + sizeof(R) * 4 * 2 * kHaloCells);  // f64 [5][kNT] (FP32 path)
  static constexpr size_t q_bytes = kF64 ? 0 : sizeof(double) * 5 * kNT;
  // face fluxes: the FP32 path reuses the staged box, dead after reconstruction
  static constexpr size_t off_F = kF64 ? a16(off_Q + q_bytes) : off_W;  // R4 [kFaces]
  static constexpr size_t off_F1 = a16(off_F + sizeof(R) * 4 * kFaces);  // R  [kFaces]
  static constexpr size_t bytes = kF64 ? a16(off_F1 + sizeof(R) * kFaces) : a16(off_Q + q_bytes);
  static_assert(kF64 || off_F1 + sizeof(R) * kFaces <= off_M, "FP32 face fluxes must fit in the staged box");
};

__device__ __forceinline__ int box_of(int x, int y, int z) { return (x + 2) + kBoxX * ((y + 2) + kBoxY * (z + 2)); }

// ring cell j: box cell, its face k toward the brick and the brick cell across it
__device__ __forceinline__ void ring_cell(int j, int &b, int &k, int &bin) {
  if (j < 64) {
    const int side = j >> 5, y = j & 7, z = (j >> 3) & 3;
    b = (side ? 10 : 1) + kBoxX * ((y + 2) + kBoxY * (z + 2));
    k = side ? 0 : 1;
    bin = b + (side ? -1 : 1);
  } else if (j < 128) {
    const int i = j - 64, side = i >> 5, x = i & 7, z = (i >> 3) & 3;
    b = (x + 2) + kBoxX * ((side ? 10 : 1) + kBoxY * (z + 2));
    k = side ? 2 : 3;
    bin = b + (side ? -kBoxX : kBoxX);
  } else {
    const int i = j - 128, side = i >> 6, x = i & 7, y = (i >> 3) & 7;
    b = (x + 2) + kBoxX * ((y + 2) + kBoxY * (side ? 6 : 1));
    k = side ? 4 : 5;
    bin = b + (side ? -kBoxX * kBoxY : kBoxX * kBoxY);
  }
}

// Per-CTA slot tables (tile independent): box cell of child 0, brick position
// bit (255 outside the brick), brick cell of child 0.
template <class M>
__device__ __forceinline__ void slot_tables(unsigned char *smem) {
  using SM = BrickSmem<M>;
  uint16_t *sBase = reinterpret_cast<uint16_t *>(smem + SM::off_sbase);
  uint8_t *sBit = smem + SM::off_sbit;
  uint8_t *sTb = smem + SM::off_tbase;
  for (int s = threadIdx.x; s < kSlots; s += blockDim.x) {
    const int sz = s / (kSlotX * kSlotY), sy = (s / kSlotX) % kSlotY, sx = s % kSlotX;
    sBase[s] = (uint16_t)(2 * sx + kBoxX * (2 * sy + kBoxY * 2 * sz));
    const bool inner = sx >= 1 && sx <= kBrickX && sy >= 1 && sy <= kBrickY && sz >= 1 && sz <= kBrickZ;
    sBit[s] = inner ? (uint8_t)((sx - 1) + kBrickX * ((sy - 1) + kBrickY * (sz - 1))) : (uint8_t)255;
    sTb[s] = inner ? (uint8_t)(2 * (sx - 1) + 8 * (2 * (sy - 1) + 8 * 2 * (sz - 1))) : (uint8_t)0;
  }
}

template <class M>
__device__ __forceinline__ void level_tile(const BatchArgs &Bt, const LevelArgs *gA, const int slot, const int tile,
                                           unsigned char *smem, unsigned &st) {
  using R = typename M::R;
  using SM = BrickSmem<M>;
  constexpr bool F64 = SM::kF64;
  using V = Q4<R>;
  uint32_t *sKey = reinterpret_cast<uint32_t *>(smem + SM::off_key);
  int *sOb = reinterpret_cast<int *>(smem + SM::off_ob);
  uint8_t *sSf = smem + SM::off_sf;
  uint8_t *sSpm = smem + SM::off_spm;
  uint8_t *sCmk = smem + SM::off_cmk;
  const uint16_t *sBase = reinterpret_cast<const uint16_t *>(smem + SM::off_sbase);
  const uint8_t *sBit = smem + SM::off_sbit;
  const uint8_t *sTb = smem + SM::off_tbase;
  uint8_t *sSt = smem + SM::off_st;
  R *sW = reinterpret_cast<R *>(smem + SM::off_W);
  R *sWp = reinterpret_cast<R *>(smem + SM::off_Wp);
  R *sM = reinterpret_cast<R *>(smem + SM::off_M);
  R *sHS = reinterpret_cast<R *>(smem + SM::off_HS);
  double *sQ = reinterpret_cast<double *>(smem + SM::off_Q);
  R *sF = reinterpret_cast<R *>(smem + SM::off_F);
  R *sF1 = reinterpret_cast<R *>(smem + SM::off_F1);

  const int tid = threadIdx.x;
  // the level's arguments, read once per tile into shared memory
  LevelArgs &A = *reinterpret_cast<LevelArgs *>(smem + SM::off_args);
  static_assert(sizeof(LevelArgs) % 4 == 0, "LevelArgs copied as 32-bit words");
  if (tid < (int)(sizeof(LevelArgs) / 4))
    reinterpret_cast<uint32_t *>(&A)[tid] = reinterpret_cast<const uint32_t *>(gA)[tid];
  __syncthreads();
  const long long N8 = 8LL * A.noct;
  const int tx = tid & 7, ty = (tid >> 3) & 7, tz = tid >> 6;
  const int tb = box_of(tx, ty, tz);

  // ------------------------------------------------------------------ P0
  // per slot: key, source offset, flags, split mask in cell order, cell map
  // (0: cell c of an oct, 1: an injected cell, 2+k: mirror across face k)
  if (tid < kSlots) {
    const uint32_t mask = A.tiles[tile].mask;
    const uint32_t key = A.keys[(size_t)tile * kSlots + tid];
    uint8_t sf = 0, spm = 0, cmk = 0;
    int ob = 0;
    if (key != kKeyNone) {
      const uint32_t kind = key >> 28, idx = key & 0x0FFFFFFFu;
      sf = kFPresent;
      if (kind == kKeyReal) {
        ob = 8 * (int)idx;
        spm = A.split[idx];
        const uint8_t bit = sBit[tid];
        if (bit != 255 && ((mask >> bit) & 1)) sf |= kFTile;
      } else if (kind == kKeyInj) {
        cmk = 1;
        if (A.Wc != nullptr) {
          ob = (int)idx;
          sf |= kFInj;
        } else {
          st |= kStTree;  // plan/launch mismatch: never read through a null level
        }
      } else {
        const int k0 = (int)(kind - kKeyGhost0);
        ob = 8 * (int)idx;
        cmk = (uint8_t)(2 + k0);
        const uint8_t raw = A.split[idx];
#pragma unroll
        for (int c = 0; c < 8; c++) spm |= (uint8_t)(((raw >> c_mirror[k0][c]) & 1) << c);
      }
    }
    sKey[tid] = key;
    sOb[tid] = ob;
    sSf[tid] = sf;
    sSpm[tid] = spm;
    sCmk[tid] = cmk;
  }
  __syncthreads();
  {
    // Thread tid stages the pair q = tid & 3 of x-neighbour children (2q, 2q+1)
    // of slots tid/4 + 64 m, two cells per 16-byte load.  Ghost children come
    // from one pair of the boundary oct too (the mirror maps keep x-pairs).
    const int q = tid & 3, s0 = tid >> 2, c0 = 2 * q;
    const int cb = kBoxX * ((q & 1) + kBoxY * (q >> 1));
    const int ct = 8 * ((q & 1) + 8 * (q >> 1));
    unsigned mir = 0;  // per ghost face k, 4 bits: source pair, element of child c0, of child c0+1
#pragma unroll
    for (int k = 0; k < 6; k++) {
      const unsigned m0 = c_mirror[k][c0], m1 = c_mirror[k][c0 + 1];
      mir |= ((m0 >> 1) | ((m0 & 1) << 2) | ((m1 & 1) << 3)) << (4 * k);
    }
    const double *W = A.W, *Wc = A.Wc;
    const long long nc8 = A.nc8;
#pragma unroll
    for (int m = 0; m < 3; m++) {
      if (m == 2 && tid >= kBox / 2 - 2 * kNT) break;
      const int s = s0 + 64 * m;
      const int b0 = sBase[s] + cb;
      const uint8_t sf = sSf[s];
      if (sf == 0) {
        sSt[b0] = 0;
        sSt[b0 + 1] = 0;
        continue;
      }
      const int cmk = sCmk[s];
      double x0[5], x1[5];
      if (cmk == 1) {  // injected coarser cell: one value for both children
        const bool inj = sf & kFInj;
        const double *p = (inj ? Wc : W) + (long long)sOb[s];
        const long long stride = inj ? nc8 : N8;
#pragma unroll
        for (int v = 0; v < 5; v++) x0[v] = x1[v] = __ldg(p + v * stride);
      } else {
        unsigned code = (unsigned)q | (1u << 3);  // pair q, elements 0 and 1
        if (cmk >= 2) code = (mir >> (4 * (cmk - 2))) & 15u;
        const double *p = W + (long long)sOb[s] + 2 * (code & 3);
        const bool e0 = (code >> 2) & 1, e1 = (code >> 3) & 1;
#pragma unroll
        for (int v = 0; v < 5; v++) {
          const double2 x = __ldg(reinterpret_cast<const double2 *>(p + v * N8));
          x0[v] = e0 ? x.y : x.x;
          x1[v] = e1 ? x.y : x.x;
        }
      }
      V::st(sW, b0, (R)x0[0], (R)x0[1], (R)x0[2], (R)x0[3]);
      V::st(sW, b0 + 1, (R)x1[0], (R)x1[1], (R)x1[2], (R)x1[3]);
      sWp[b0] = (R)x0[4];
      sWp[b0 + 1] = (R)x1[4];
      const uint8_t spm = sSpm[s];
      const uint8_t f0 = sf | (((spm >> c0) & 1) ? kFSplit : 0), f1 = sf | (((spm >> (c0 + 1)) & 1) ? kFSplit : 0);
      sSt[b0] = f0;
      sSt[b0 + 1] = f1;
      if constexpr (!F64) {
        if (sf & kFTile) {
          const int t = sTb[s] + ct;
#pragma unroll
          for (int v = 0; v < 5; v++) {
            sQ[v * kNT + t] = x0[v];
            sQ[v * kNT + t + 1] = x1[v];
          }
        }
      }
    }
  }
  __syncthreads();

  auto q_at = [&](int b, R q[5]) {
    V::ld(sW, b, q[0], q[1], q[2], q[3]);
    q[4] = sWp[b];
  };

  // ------------------------------------------------------------------ P1
  // Pass 0: brick cell tid (slopes and predictor, when it is a leaf of the tile
  // or borders one); pass 1: ring cell tid (the one face state it contributes).
  // One call site each for the reconstruction and the face state, so that a
  // face on a brick boundary, solved by both bricks, rounds the same in both.
#pragma unroll 1
  for (int pass = 0; pass < 2; pass++) {
    int b = tb, k = 0, bin = tb;
    bool need;
    if (pass == 0) {
      const uint8_t f = sSt[tb];
      need = f_tileleaf(f);
      if (!need && f_ok(f))
        need = f_tileleaf(sSt[tb - 1]) || f_tileleaf(sSt[tb + 1]) || f_tileleaf(sSt[tb - kBoxX]) ||
               f_tileleaf(sSt[tb + kBoxX]) || f_tileleaf(sSt[tb - kBoxX * kBoxY]) ||
               f_tileleaf(sSt[tb + kBoxX * kBoxY]);
    } else {
      ring_cell(tid, b, k, bin);
      need = f_ok(sSt[b]) && f_tileleaf(sSt[bin]);
    }
    if (!need) continue;
    R q0[5], qm[3][5], qp[3][5], D[3][5], Wt[5], X[5];
    q_at(b, q0);
    q_at(b - 1, qm[0]);
    q_at(b + 1, qp[0]);
    q_at(b - kBoxX, qm[1]);
    q_at(b + kBoxX, qp[1]);
    q_at(b - kBoxX * kBoxY, qm[2]);
    q_at(b + kBoxX * kBoxY, qp[2]);
    if constexpr (F64) M::muscl(q0, qm, qp, A.dt, A.dx, D, Wt);
    else M::muscl(q0, qm, qp, (R)(A.dt / A.dx * 0.5), D, Wt);
    // X = W0 + Wt (FP32 path) or Wt (FP64 path, which adds W0 in the reference's order)
#pragma unroll
    for (int v = 0; v < 5; v++) X[v] = F64 ? Wt[v] : q0[v] + Wt[v];
    if (pass == 0) {
      // groups: D_x(d,u,v,w), D_y, D_z, X(d,u,v,w), (D_x.p, D_y.p, D_z.p, X.p)
#pragma unroll
      for (int dir = 0; dir < 3; dir++) V::st(sM, dir * kNT + tid, D[dir][0], D[dir][1], D[dir][2], D[dir][3]);
      V::st(sM, 3 * kNT + tid, X[0], X[1], X[2], X[3]);
      V::st(sM, 4 * kNT + tid, D[0][4], D[1][4], D[2][4], X[4]);
    } else {
      const int ax = k >> 1;
      R Dax[5], W[7];
#pragma unroll
      for (int v = 0; v < 5; v++) Dax[v] = (ax == 0) ? D[0][v] : ((ax == 1) ? D[1][v] : D[2][v]);
      if constexpr (F64) M::face_ax(q0, Dax, Wt, k, W, st);
      else M::face_px(X, Dax, k, W, st);
      V::st(sHS, tid, W[0], W[1], W[2], W[3]);
      V::st(sHS, kHaloCells + tid, W[4], W[5], W[6], (R)0);
    }
  }
  __syncthreads();

  // face state k of brick cell t (box cell b) from its slopes and predictor
  auto brick_face = [&](int t, int b, int k, R W[7]) {
    const int ax = k >> 1;
    R Dax[5], X[5], p0, p1, p2;
    V::ld(sM, ax * kNT + t, Dax[0], Dax[1], Dax[2], Dax[3]);
    V::ld(sM, 3 * kNT + t, X[0], X[1], X[2], X[3]);
    V::ld(sM, 4 * kNT + t, p0, p1, p2, X[4]);
    Dax[4] = (ax == 0) ? p0 : ((ax == 1) ? p1 : p2);
    if constexpr (F64) {
      R q0[5];
      q_at(b, q0);
      M::face_ax(q0, Dax, X, k, W, st);
    } else {
      M::face_px(X, Dax, k, W, st);
    }
  };
  auto ring_face = [&](int j, R W[7]) {
    R pad;
    V::ld(sHS, j, W[0], W[1], W[2], W[3]);
    V::ld(sHS, kHaloCells + j, W[4], W[5], W[6], pad);
  };

  // ------------------------------------------------------------------ P2
  // Rounds 0..2: the -d face of every brick cell; round 3 (threads < 128): the
  // + faces on the brick boundary.  One HLLC call site for all rounds.
#pragma unroll 1
  for (int r = 0; r < 4; r++) {
    if (r == 3 && tid >= 128) break;
    int d, e, tL, bL, jL = -1, tR, bR, jR = -1;
    if (r < 3) {
      d = r;
      const int bs = (d == 0) ? 1 : ((d == 1) ? kBoxX : kBoxX * kBoxY);
      const int ts = (d == 0) ? 1 : ((d == 1) ? 8 : 64);
      const int coord = (d == 0) ? tx : ((d == 1) ? ty : tz);
      e = (d == 0) ? (tx + 9 * (ty + 8 * tz)) : ((d == 1) ? (kFacesX + tx + 8 * (ty + 9 * tz)) : (kFacesX + kFacesY + tid));
      tR = tid;
      bR = tb;
      tL = tid - ts;
      bL = tb - bs;
      if (coord == 0) jL = (d == 0) ? (ty + 8 * tz) : ((d == 1) ? (64 + tx + 8 * tz) : (128 + tx + 8 * ty));
    } else {
      int x, y, z;
      if (tid < 32) {
        d = 0; x = 7; y = tid & 7; z = tid >> 3; jR = 32 + tid; e = 8 + 9 * (y + 8 * z);
      } else if (tid < 64) {
        d = 1; x = tid & 7; y = 7; z = (tid - 32) >> 3; jR = 96 + (tid - 32); e = kFacesX + x + 8 * (8 + 9 * z);
      } else {
        d = 2; x = tid & 7; y = (tid - 64) >> 3; z = 3; jR = 192 + (tid - 64);
        e = kFacesX + kFacesY + x + 8 * (y + 32);
      }
      const int bs = (d == 0) ? 1 : ((d == 1) ? kBoxX : kBoxX * kBoxY);
      tL = x + 8 * (y + 8 * z);
      bL = box_of(x, y, z);
      tR = tL;
      bR = bL + bs;
    }
    const uint8_t fL = sSt[bL], fR = sSt[bR];
    R F[5] = {0, 0, 0, 0, 0};
    if ((f_tileleaf(fL) || f_tileleaf(fR)) && f_ok(fL) && f_ok(fR)) {
      R WL[7], WR[7];
      if (jL >= 0) ring_face(jL, WL);
      else brick_face(tL, bL, 2 * d + 1, WL);
      if (jR >= 0) ring_face(jR, WR);
      else brick_face(tR, bR, 2 * d, WR);
      M::hllc(WL, WR, d, F, st);
    }
    V::st(sF, e, F[0], F[1], F[2], F[3]);
    sF1[e] = F[4];
  }
  __syncthreads();

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
    __syncthreads();
  }
  const uint8_t fme = sSt[tb];
  if (fme & kFTile) {
    const int s = ((tx + 2) >> 1) + kSlotX * (((ty + 2) >> 1) + kSlotY * ((tz + 2) >> 1));
    const int c = (tx & 1) | ((ty & 1) << 1) | ((tz & 1) << 2);
    const long long gi = 8LL * (sKey[s] & 0x0FFFFFFFu) + c;
    double q[5];
    if constexpr (F64) {
      V::ld(sW, tb, q[0], q[1], q[2], q[3]);
      q[4] = sWp[tb];
    } else {
#pragma unroll
      for (int v = 0; v < 5; v++) q[v] = sQ[v * kNT + tid];
    }
    double Wout[5];
    if (fme & kFSplit) {
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
      const int ex = tx + 9 * (ty + 8 * tz), ey = kFacesX + tx + 8 * (ty + 9 * tz), ez = kFacesX + kFacesY + tid;
      auto flux5 = [&](int k, double F[5]) {
        const int e = (k < 2) ? (ex + (k & 1)) : ((k < 4) ? (ey + 8 * (k & 1)) : (ez + 64 * (k & 1)));
        R f0, f1, f2, f3;
        V::ld(sF, e, f0, f1, f2, f3);
        F[0] = (double)f0;
        F[1] = (double)f1;
        F[2] = (double)f2;
        F[3] = (double)f3;
        F[4] = (double)sF1[e];
      };
      double Ud, Udu, Udv, Udw, UE;
      if (A.B != nullptr) {  // drop-in: W2U of the caller's fieldnew
        const double bd = A.B[gi];
        Ud = bd;
        Udu = bd * A.B[N8 + gi];
        Udv = bd * A.B[2 * N8 + gi];
        Udw = bd * A.B[3 * N8 + gi];
        UE = A.B[5 * N8 + gi];
      } else {  // resident: W2U(field) + corrections received from the finer level
        Ud = q[0];
        Udu = q[0] * q[1];
        Udv = q[0] * q[2];
        Udw = q[0] * q[3];
        UE = q[4] / (kGam - 1.) + 0.5 * q[0] * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
      }
      if constexpr (F64) {
        // updatefield (src/hydro_utils.c:3050-3082): dU = sum over faces -x,+x,-y,+y,-z,+z
        // of (+-F dt/dx), signs alternating from +
        double dU[5] = {0., 0., 0., 0., 0.};
        double one = 1.;
#pragma unroll
        for (int k = 0; k < 6; k++) {
          double F[5];
          flux5(k, F);
#pragma unroll
          for (int v = 0; v < 5; v++) dU[v] += F[v] * dtsurdx * one;
          one *= -1.;
        }
        // scatterstencil central update (src/hydro_utils.c:3129-3188), reference order
        if (A.B == nullptr && A.C != nullptr) {
          Ud += __ldcg(A.C + gi);
          Udu += __ldcg(A.C + N8 + gi);
          Udv += __ldcg(A.C + 2 * N8 + gi);
          Udw += __ldcg(A.C + 3 * N8 + gi);
          UE += __ldcg(A.C + 4 * N8 + gi);
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
          for (int v = 0; v < 5; v++) add(v, __ldcg(A.C + v * N8 + gi));
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
      Wout[4] = fmax(Wout[4], kPmin);
      if (isnan(Wout[1]) || isnan(Wout[4]) || isnan(Wout[0])) st |= kStNan;

      // fine -> coarse correction into unsplit coarser neighbours (src/hydro_utils.c:3206-3295)
#pragma unroll
      for (int k = 0; k < 6; k++) {
        const int bs = (k < 2) ? 1 : ((k < 4) ? kBoxX : kBoxX * kBoxY);
        const int b2 = (k & 1) ? tb + bs : tb - bs;
        if (!(sSt[b2] & kFInj) || A.Cc == nullptr) continue;
        const int x2 = b2 % kBoxX, y2 = (b2 / kBoxX) % kBoxY, z2 = b2 / (kBoxX * kBoxY);
        const long long cc = sKey[(x2 >> 1) + kSlotX * ((y2 >> 1) + kSlotY * (z2 >> 1))] & 0x0FFFFFFFu;
        const double one = (k & 1) ? 1. : -1.;
        double F[5];
        flux5(k, F);
#pragma unroll
        for (int v = 0; v < 5; v++) atomicAdd(A.Cc + v * A.nc8 + cc, F[v] * dtsurdx * one * 0.125);
      }
    }
#pragma unroll
    for (int v = 0; v < 5; v++) A.Wn[v * N8 + gi] = Wout[v];
  }
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    atomicAdd(Bt.done + slot, 1u);
  }
}

// Persistent launch over a work list of (level slot, tile) items.  All CTAs are
// co-resident (grid <= occupancy x SMs) and take items in list order, so a
// tile waiting for a finer level (listed first) never blocks the CTAs that
// still have to finish that level.
template <class M>
__global__ void __launch_bounds__(kNT, (sizeof(typename M::R) == 8) ? 1 : 3) level_batch_kernel(const BatchArgs Bt) {
  extern __shared__ __align__(16) unsigned char smem[];
  if (Bt.gate != nullptr && *Bt.gate == 0) return;
  slot_tables<M>(smem);
  __syncthreads();
  unsigned st = 0;
  for (int w = blockIdx.x; w < Bt.nwork; w += gridDim.x) {
    const int item = Bt.work[w];
    const int slot = item >> kWorkSlotShift, tile = item & ((1 << kWorkSlotShift) - 1);
    level_tile<M>(Bt, Bt.lv + slot, slot, tile, smem, st);
    __syncthreads();
  }
  if (st) atomicOr(Bt.status, st);
}

}  // namespace emma
