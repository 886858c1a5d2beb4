// level_kernel.cuh -- the hydro level advance on the GPU, one CTA per tile.
//
// A tile is a run of up to T consecutive octs of one level (list order, which
// is spatially clustered: Morton order on complete levels).  Each CTA:
//   P0  stages into shared memory every oct the tile's MUSCL stencils touch:
//       the tile octs, their 6 face and 12 edge neighbours at the same level
//       ("virtual octs": a real oct, a coarser leaf cell injected into 8 cells
//       as the reference's gather does, or a transmissive mirror ghost), with
//       the neighbour graph between staged octs (precomputed per tile);
//   P1  MUSCL-Hancock once per needed cell: slopes + predictor of every tile
//       cell (kept in shared memory), and for every halo entry (a cell outside
//       the tile face-adjacent to it) the one face state it contributes;
//   P2  one HLLC solve per face, as an axis-major task list spread evenly over
//       the CTA: task (axis d, tile cell t) is the -d face of t; then the +d
//       faces on the tile's + boundary;
//   P3  per tile cell: the six face fluxes summed in the reference's order
//       (-x,+x,-y,+y,-z,+z), conserved update, primitive recovery, floors;
//       split cells get the primitive mean of their children; faces bordering
//       a coarser leaf add the fine->coarse correction (atomics, x 1/8).
// The reference does the same per oct on a 27-oct copy, recomputing each
// cell's reconstruction up to 9 times and each face twice
// (src/hydro_utils.c:1407-2238, 2973-3303).
#pragma once
#include "hydro_math.cuh"
#include "plan_types.h"

namespace emma {

__device__ __forceinline__ bool nei_inside(int c, int k) {
  const int bit = 1 << (k >> 1);
  return (k & 1) ? !(c & bit) : (c & bit);
}

// mirror maps of the transmissive ghost octs (src/hydro_utils.c:2504-2610)
__constant__ uint8_t c_mirror[6][8] = {
    {0, 0, 2, 2, 4, 4, 6, 6}, {1, 1, 3, 3, 5, 5, 7, 7}, {0, 1, 0, 1, 4, 5, 4, 5},
    {2, 3, 2, 3, 7, 6, 6, 7}, {0, 1, 2, 3, 0, 1, 2, 3}, {4, 5, 6, 7, 4, 5, 6, 7}};

template <class M, int T, int SMAX, int HMAX, int BMAX>
struct LevelSmem {
  using R = typename M::R;
  static constexpr int NT = 8 * T;  // tile cells = threads
  static constexpr size_t a16(size_t x) { return (x + 15) & ~size_t(15); }
  static constexpr size_t off_W = 0;                                       // R [5][SMAX*8] staged states
  static constexpr size_t off_M = a16(off_W + sizeof(R) * 5 * SMAX * 8);   // R [20][NT] slopes + predictor
  static constexpr size_t off_HS = a16(off_M + sizeof(R) * 20 * NT);       // R [7][HMAX] halo face states
  static constexpr size_t off_F = a16(off_HS + sizeof(R) * 7 * HMAX);      // R [5][3*NT] -d face fluxes
  static constexpr size_t off_FB = a16(off_F + sizeof(R) * 5 * 3 * NT);    // R [5][BMAX] boundary + faces
  static constexpr size_t off_key = a16(off_FB + sizeof(R) * 5 * BMAX);    // u32 [SMAX]
  static constexpr size_t off_G = a16(off_key + sizeof(uint32_t) * SMAX);  // u8 [SMAX*6]
  static constexpr size_t off_hmap = a16(off_G + 6 * SMAX);               // u16 [SMAX*8] first halo entry
  static constexpr size_t off_halo = a16(off_hmap + 2 * SMAX * 8);        // u16 [HMAX] halo entries
  static constexpr size_t off_bface = a16(off_halo + 2 * HMAX);           // u16 [BMAX] boundary faces
  static constexpr size_t off_bmap = a16(off_bface + 2 * BMAX);           // u16 [3*NT] (cell,axis) -> face
  static constexpr size_t off_sp = a16(off_bmap + 2 * 3 * NT);            // u8 [SMAX*8] split flags
  static constexpr size_t bytes = a16(off_sp + SMAX * 8);
};

template <class M, int T, int SMAX, int HMAX, int BMAX>
__device__ __forceinline__ void level_tile(const BatchArgs &Bt, const LevelArgs &A, const int slot, const int tile,
                                           unsigned char *smem, unsigned &st) {
  using R = typename M::R;
  using SM = LevelSmem<M, T, SMAX, HMAX, BMAX>;
  constexpr int NT = SM::NT;
  R *sW = reinterpret_cast<R *>(smem + SM::off_W);
  R *sM = reinterpret_cast<R *>(smem + SM::off_M);
  R *sHS = reinterpret_cast<R *>(smem + SM::off_HS);
  R *sF = reinterpret_cast<R *>(smem + SM::off_F);
  R *sFB = reinterpret_cast<R *>(smem + SM::off_FB);
  uint32_t *sKey = reinterpret_cast<uint32_t *>(smem + SM::off_key);
  uint8_t *sG = smem + SM::off_G;
  uint16_t *sHmap = reinterpret_cast<uint16_t *>(smem + SM::off_hmap);
  uint16_t *sHalo = reinterpret_cast<uint16_t *>(smem + SM::off_halo);
  uint16_t *sBface = reinterpret_cast<uint16_t *>(smem + SM::off_bface);
  uint16_t *sBmap = reinterpret_cast<uint16_t *>(smem + SM::off_bmap);
  uint8_t *sSp = smem + SM::off_sp;

  const int tid = threadIdx.x;
  const TileDesc td = A.tiles[tile];
  const int n = td.noct, S = td.S, H = td.H, B = td.B;
  const int n8 = 8 * n;
  const long long N8 = 8LL * A.noct;
  if (S > SMAX || H > HMAX || B > BMAX || n > T || n < 1) {  // plan cut for another kernel shape
    st |= kStTree;
    if (tid == 0) atomicAdd(Bt.done + slot, 1u);  // keep batched waits bounded
    return;
  }

  // ------------------------------------------------------------------ P0
  for (int i = tid; i < S; i += NT) sKey[i] = A.keys[td.keys_off + i];
  for (int i = tid; i < S * 6; i += NT) sG[i] = A.graph[td.graph_off + i];
  for (int i = tid; i < S * 8; i += NT) sHmap[i] = 0xFFFF;
  for (int i = tid; i < H; i += NT) sHalo[i] = A.halo[td.halo_off + i];
  for (int i = tid; i < B; i += NT) sBface[i] = A.bface[td.bface_off + i];
  __syncthreads();
  for (int h = tid; h < H; h += NT) {
    const int cell = sHalo[h] >> 3;
    if (h == 0 || (sHalo[h - 1] >> 3) != cell) sHmap[cell] = (uint16_t)h;
  }
  for (int b = tid; b < B; b += NT) {
    const int e = sBface[b];
    sBmap[(e >> 2) * 3 + (e & 3)] = (uint16_t)b;
  }
#pragma unroll 4
  for (int i = tid; i < S * 8; i += NT) {
    const int s = i >> 3, c = i & 7;
    const uint32_t key = sKey[s];
    const uint32_t kind = key >> 28, idx = key & 0x0FFFFFFFu;
    const double *src = A.W;
    long long stride = N8, off;
    uint8_t sp = 0;
    if (kind == kKeyReal) {
      off = 8LL * idx + c;
      sp = (A.split[idx] >> c) & 1;
    } else if (kind == kKeyInj) {
      src = A.Wc;
      stride = A.nc8;
      off = idx;
      if (src == nullptr) {  // plan/launch mismatch: never read through a null level
        st |= kStTree;
        src = A.W;
        stride = N8;
        off = 0;
      }
    } else {
      const int mc = c_mirror[kind - kKeyGhost0][c];
      off = 8LL * idx + mc;
      sp = (A.split[idx] >> mc) & 1;
    }
    const double v0 = __ldg(src + off), v1 = __ldg(src + stride + off), v2 = __ldg(src + 2 * stride + off);
    const double v3 = __ldg(src + 3 * stride + off), v4 = __ldg(src + 4 * stride + off);
    sW[0 * SMAX * 8 + i] = (R)v0;
    sW[1 * SMAX * 8 + i] = (R)v1;
    sW[2 * SMAX * 8 + i] = (R)v2;
    sW[3 * SMAX * 8 + i] = (R)v3;
    sW[4 * SMAX * 8 + i] = (R)v4;
    sSp[i] = sp;
  }
  __syncthreads();

  // staged-cell neighbour across face k (same oct or via the graph); -1 if absent
  auto nb = [&](int s, int c, int k, int &c2) -> int {
    c2 = c ^ (1 << (k >> 1));
    if (nei_inside(c, k)) return s;
    const int g = sG[s * 6 + k];
    return g == 255 ? -1 : g;
  };
  auto q_of = [&](int s, int c, R q[5]) {
#pragma unroll
    for (int v = 0; v < 5; v++) q[v] = sW[v * SMAX * 8 + s * 8 + c];
  };
  auto muscl_of = [&](int s, int c, R D[3][5], R Wt[5]) {
    R q0[5], qm[3][5], qp[3][5];
    q_of(s, c, q0);
#pragma unroll
    for (int dir = 0; dir < 3; dir++) {
      int c2;
      int s2 = nb(s, c, 2 * dir, c2);
      if (s2 < 0) { st |= kStTree; s2 = s; c2 = c; }
      q_of(s2, c2, qm[dir]);
      s2 = nb(s, c, 2 * dir + 1, c2);
      if (s2 < 0) { st |= kStTree; s2 = s; c2 = c; }
      q_of(s2, c2, qp[dir]);
    }
    if constexpr (sizeof(R) == 8) M::muscl(q0, qm, qp, A.dt, A.dx, D, Wt);
    else M::muscl(q0, qm, qp, (R)(A.dt / A.dx * 0.5), D, Wt);
  };

  // ------------------------------------------------------------------ P1
  for (int j = tid; j < n8 + H; j += NT) {
    int s, c, k = -1;
    if (j < n8) {
      s = j >> 3;
      c = j & 7;
    } else {
      const int e = sHalo[j - n8];
      s = e >> 6;
      c = (e >> 3) & 7;
      k = e & 7;
    }
    if (sSp[s * 8 + c]) continue;  // split cells carry no flux: no reconstruction
    R D[3][5], Wt[5];
    muscl_of(s, c, D, Wt);
    if (k < 0) {
#pragma unroll
      for (int dir = 0; dir < 3; dir++)
#pragma unroll
        for (int v = 0; v < 5; v++) sM[(dir * 5 + v) * NT + j] = D[dir][v];
#pragma unroll
      for (int v = 0; v < 5; v++) sM[(15 + v) * NT + j] = Wt[v];
    } else {
      R q0[5], Dax[5], W[7];
      q_of(s, c, q0);
      const int ax = k >> 1;
#pragma unroll
      for (int v = 0; v < 5; v++) Dax[v] = (ax == 0) ? D[0][v] : ((ax == 1) ? D[1][v] : D[2][v]);
      M::face_ax(q0, Dax, Wt, k, W, st);
      const int h = j - n8;
#pragma unroll
      for (int v = 0; v < 7; v++) sHS[v * HMAX + h] = W[v];
    }
  }
  __syncthreads();

  // face state k of tile cell t from its slopes and predictor
  auto tile_face = [&](int t, int k, R W[7]) {
    R q0[5], Dax[5], Wt[5];
    q_of(t >> 3, t & 7, q0);
    const int ax = k >> 1;
#pragma unroll
    for (int v = 0; v < 5; v++) {
      Dax[v] = sM[(ax * 5 + v) * NT + t];
      Wt[v] = sM[(15 + v) * NT + t];
    }
    M::face_ax(q0, Dax, Wt, k, W, st);
  };
  // stored face state k of halo cell `cell` (s*8+c); false if absent
  auto halo_face = [&](int cell, int k, R W[7]) -> bool {
    int h = sHmap[cell];
    if (h == 0xFFFF) return false;
    while (h < H && (sHalo[h] >> 3) == cell && (sHalo[h] & 7) != k) h++;
    if (h >= H || (sHalo[h] >> 3) != cell) return false;
#pragma unroll
    for (int v = 0; v < 7; v++) W[v] = sHS[v * HMAX + h];
    return true;
  };

  // ------------------------------------------------------------------ P2
  for (int f = tid; f < 3 * n8 + B; f += NT) {
    int t, d;
    bool plus;
    if (f < 3 * n8) {
      d = f / n8;
      t = f - d * n8;
      plus = false;
    } else {
      const int e = sBface[f - 3 * n8];
      t = e >> 2;
      d = e & 3;
      plus = true;
    }
    const int o = t >> 3, c = t & 7;
    const int k = 2 * d + (plus ? 1 : 0);
    R F[5] = {0, 0, 0, 0, 0};
    int c2;
    const int s2 = nb(o, c, k, c2);
    if (s2 < 0) {
      st |= kStTree;
    } else if (!sSp[t] && !sSp[s2 * 8 + c2]) {
      R Wa[7], Wb[7];  // a: this cell's state at the face, b: the neighbour's
      tile_face(t, k, Wa);
      bool ok = true;
      if (s2 < n) tile_face(s2 * 8 + c2, k ^ 1, Wb);
      else ok = halo_face(s2 * 8 + c2, k ^ 1, Wb);
      if (!ok) {
        st |= kStTree;
      } else if (plus) {
        M::hllc(Wa, Wb, d, F, st);
      } else {
        M::hllc(Wb, Wa, d, F, st);
      }
    }
    if (plus) {
      const int b = f - 3 * n8;
#pragma unroll
      for (int v = 0; v < 5; v++) sFB[v * BMAX + b] = F[v];
    } else {
#pragma unroll
      for (int v = 0; v < 5; v++) sF[v * 3 * NT + d * NT + t] = F[v];
    }
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
  if (tid < n8) {
    const int o = tid >> 3, c = tid & 7;
    const long long gi = 8LL * (td.oct0 + o) + c;
    double q[5];
#pragma unroll
    for (int v = 0; v < 5; v++) q[v] = A.W[v * N8 + gi];
    double Wout[5];
    if (sSp[tid]) {
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
      // flux of face k (0:-x 1:+x ...) of this cell, from the face tasks of P2
      auto flux = [&](int k, int v) -> double {
        const int d = k >> 1;
        if (!(k & 1)) return (double)sF[v * 3 * NT + d * NT + tid];
        int c2;
        const int s2 = nb(o, c, k, c2);
        if (s2 >= 0 && s2 < n) return (double)sF[v * 3 * NT + d * NT + s2 * 8 + c2];
        return (double)sFB[v * BMAX + sBmap[tid * 3 + d]];
      };
      // updatefield (src/hydro_utils.c:3050-3082): dU = sum over faces -x,+x,-y,+y,-z,+z
      // of (+-F dt/dx), signs alternating from +
      double dU[5] = {0., 0., 0., 0., 0.};
      double one = 1.;
#pragma unroll
      for (int k = 0; k < 6; k++) {
#pragma unroll
        for (int v = 0; v < 5; v++) dU[v] += flux(k, v) * dtsurdx * one;
        one *= -1.;
      }
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
      if constexpr (sizeof(R) == 8) {
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
        // mixed: FP32 face fluxes summed in FP64, added to the FP64 conserved state
        // with Neumaier-compensated summation (base + corrections + dU)
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
        for (int v = 0; v < 5; v++) add(v, dU[v]);
        Ud = sum[0] + comp[0];
        Udu = sum[1] + comp[1];
        Udv = sum[2] + comp[2];
        Udw = sum[3] + comp[3];
        UE = sum[4] + comp[4];
      }
      // U2W (src/hydro_utils.c:35-64), pressure floor, E - Ekin recovery
      const double dl = (Ud == 0. ? 10. : Ud);
      Wout[0] = Ud;
      Wout[1] = Udu / dl;
      Wout[2] = Udv / dl;
      Wout[3] = Udw / dl;
      Wout[4] = (kGam - 1.) * (UE - ((Udu) * (Udu) + (Udv) * (Udv) + (Udw) * (Udw)) / (dl) * 0.5);
      Wout[4] = fmax(Wout[4], kPmin);
      if (isnan(Wout[1]) || isnan(Wout[4]) || isnan(Wout[0])) st |= kStNan;

      // fine -> coarse correction into unsplit coarser neighbours (src/hydro_utils.c:3206-3295)
#pragma unroll
      for (int k = 0; k < 6; k++) {
        if (nei_inside(c, k)) continue;
        const int g = sG[o * 6 + k];
        if (g == 255) continue;
        const uint32_t key = sKey[g];
        if ((key >> 28) != kKeyInj) continue;
        const long long cc = key & 0x0FFFFFFFu;
        const double one = (k & 1) ? 1. : -1.;
#pragma unroll
        for (int v = 0; v < 5; v++) atomicAdd(A.Cc + v * A.nc8 + cc, flux(k, v) * dtsurdx * one * 0.125);
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
template <class M, int T, int SMAX, int HMAX, int BMAX>
__global__ void __launch_bounds__(8 * T, (sizeof(typename M::R) == 8) ? 1 : 3)
    level_batch_kernel(const BatchArgs Bt) {
  extern __shared__ __align__(16) unsigned char smem[];
  if (Bt.gate != nullptr && *Bt.gate == 0) return;
  unsigned st = 0;
  for (int w = blockIdx.x; w < Bt.nwork; w += gridDim.x) {
    const int item = Bt.work[w];
    const int slot = item >> kWorkSlotShift, tile = item & ((1 << kWorkSlotShift) - 1);
    level_tile<M, T, SMAX, HMAX, BMAX>(Bt, Bt.lv[slot], slot, tile, smem, st);
    __syncthreads();
  }
  if (st) atomicOr(Bt.status, st);
}

}  // namespace emma
