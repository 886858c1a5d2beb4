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

template <class M, int T, int SMAX, int HMAX, int BMAX>
struct LevelSmem {
  using R = typename M::R;
  static constexpr int NT = 8 * T;  // tile cells = threads
  static constexpr size_t a16(size_t x) { return (x + 15) & ~size_t(15); }
  static constexpr size_t off_W = 0;                                        // R4 [SMAX*8] (d,u,v,w)
  static constexpr size_t off_Wp = a16(off_W + sizeof(R) * 4 * SMAX * 8);   // R  [SMAX*8] p
  static constexpr size_t off_M = a16(off_Wp + sizeof(R) * SMAX * 8);       // R4 [5][NT] slopes + predictor
  static constexpr size_t off_HS = a16(off_M + sizeof(R) * 4 * 5 * NT);     // R4 [2][HMAX] halo face states
  static constexpr size_t off_F = a16(off_HS + sizeof(R) * 4 * 2 * HMAX);   // R4 [3*NT] + R [3*NT] -d face fluxes
  static constexpr size_t off_F4 = a16(off_F + sizeof(R) * 4 * 3 * NT);
  static constexpr size_t off_FB = a16(off_F4 + sizeof(R) * 3 * NT);        // R4 [BMAX] + R [BMAX] boundary faces
  static constexpr size_t off_FB4 = a16(off_FB + sizeof(R) * 4 * BMAX);
  static constexpr size_t off_key = a16(off_FB4 + sizeof(R) * BMAX);       // u32 [SMAX]
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
  using V = Q4<R>;
  R *sW = reinterpret_cast<R *>(smem + SM::off_W);
  R *sWp = reinterpret_cast<R *>(smem + SM::off_Wp);
  R *sM = reinterpret_cast<R *>(smem + SM::off_M);
  R *sHS = reinterpret_cast<R *>(smem + SM::off_HS);
  R *sF = reinterpret_cast<R *>(smem + SM::off_F);
  R *sF4 = reinterpret_cast<R *>(smem + SM::off_F4);
  R *sFB = reinterpret_cast<R *>(smem + SM::off_FB);
  R *sFB4 = reinterpret_cast<R *>(smem + SM::off_FB4);
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
    V::st(sW, i, (R)v0, (R)v1, (R)v2, (R)v3);
    sWp[i] = (R)v4;
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
    V::ld(sW, s * 8 + c, q[0], q[1], q[2], q[3]);
    q[4] = sWp[s * 8 + c];
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
      // groups: D_x(d,u,v,w), D_y(..), D_z(..), Wt(d,u,v,w), (D_x.p, D_y.p, D_z.p, Wt.p)
#pragma unroll
      for (int dir = 0; dir < 3; dir++) V::st(sM, dir * NT + j, D[dir][0], D[dir][1], D[dir][2], D[dir][3]);
      V::st(sM, 3 * NT + j, Wt[0], Wt[1], Wt[2], Wt[3]);
      V::st(sM, 4 * NT + j, D[0][4], D[1][4], D[2][4], Wt[4]);
    } else {
      R q0[5], Dax[5], W[7];
      q_of(s, c, q0);
      const int ax = k >> 1;
#pragma unroll
      for (int v = 0; v < 5; v++) Dax[v] = (ax == 0) ? D[0][v] : ((ax == 1) ? D[1][v] : D[2][v]);
      M::face_ax(q0, Dax, Wt, k, W, st);
      const int h = j - n8;
      V::st(sHS, h, W[0], W[1], W[2], W[3]);
      V::st(sHS, HMAX + h, W[4], W[5], W[6], (R)0);
    }
  }
  __syncthreads();

  // face state k of tile cell t from its slopes and predictor
  auto tile_face = [&](int t, int k, R W[7]) {
    R q0[5], Dax[5], Wt[5];
    q_of(t >> 3, t & 7, q0);
    const int ax = k >> 1;
    R p0, p1, p2;
    V::ld(sM, ax * NT + t, Dax[0], Dax[1], Dax[2], Dax[3]);
    V::ld(sM, 3 * NT + t, Wt[0], Wt[1], Wt[2], Wt[3]);
    V::ld(sM, 4 * NT + t, p0, p1, p2, Wt[4]);
    Dax[4] = (ax == 0) ? p0 : ((ax == 1) ? p1 : p2);
    M::face_ax(q0, Dax, Wt, k, W, st);
  };
  // stored face state k of halo cell `cell` (s*8+c); false if absent
  auto halo_face = [&](int cell, int k, R W[7]) -> bool {
    int h = sHmap[cell];
    if (h == 0xFFFF) return false;
    while (h < H && (sHalo[h] >> 3) == cell && (sHalo[h] & 7) != k) h++;
    if (h >= H || (sHalo[h] >> 3) != cell) return false;
    R pad;
    V::ld(sHS, h, W[0], W[1], W[2], W[3]);
    V::ld(sHS, HMAX + h, W[4], W[5], W[6], pad);
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
      V::st(sFB, b, F[0], F[1], F[2], F[3]);
      sFB4[b] = F[4];
    } else {
      V::st(sF, d * NT + t, F[0], F[1], F[2], F[3]);
      sF4[d * NT + t] = F[4];
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
      auto flux_slot = [&](int k, const R *&b4, const R *&b1, int &idx) {
        const int d = k >> 1;
        b4 = sF;
        b1 = sF4;
        idx = d * NT + tid;
        if (!(k & 1)) return;
        int c2;
        const int s2 = nb(o, c, k, c2);
        if (s2 >= 0 && s2 < n) {
          idx = d * NT + s2 * 8 + c2;
        } else {
          b4 = sFB;
          b1 = sFB4;
          idx = sBmap[tid * 3 + d];
        }
      };
      auto flux5 = [&](int k, double F[5]) {
        const R *b4, *b1;
        int idx;
        flux_slot(k, b4, b1, idx);
        R f0, f1, f2, f3;
        V::ld(b4, idx, f0, f1, f2, f3);
        F[0] = (double)f0;
        F[1] = (double)f1;
        F[2] = (double)f2;
        F[3] = (double)f3;
        F[4] = (double)b1[idx];
      };
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
      if constexpr (sizeof(R) == 8) {
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
        if (nei_inside(c, k)) continue;
        const int g = sG[o * 6 + k];
        if (g == 255) continue;
        const uint32_t key = sKey[g];
        if ((key >> 28) != kKeyInj) continue;
        const long long cc = key & 0x0FFFFFFFu;
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
