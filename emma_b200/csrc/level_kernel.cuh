// level_kernel.cuh -- the hydro level advance on the GPU, one CTA per tile.
//
// A tile is a run of up to T consecutive octs of one level (list order, which
// is spatially clustered: Morton order on complete levels).  Each CTA:
//   P0  stages into shared memory every oct the tile's MUSCL stencils touch:
//       the tile octs, their 6 face and 12 edge neighbours at the same level
//       ("virtual octs": a real oct, a coarser leaf cell injected into 8 cells
//       as the reference's gather does, or a transmissive mirror ghost), with
//       the neighbour graph between staged octs (precomputed per tile);
//   P1  computes MUSCL-Hancock slopes and predictor once per needed cell: the
//       tile cells plus the halo cells face-adjacent to them;
//   P2  solves each face once (HLLC); a face is owned by the tile cell on its +
//       side, faces on the tile's + boundary by the cell on their - side;
//   P3  sums the six face fluxes in the reference's order (-x,+x,-y,+y,-z,+z),
//       updates the conserved state, recovers primitives, applies the floors,
//       restricts split cells from the finer level and adds the fine->coarse
//       corrections of faces that border a coarser leaf (atomics, x 1/8).
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

template <class M, int T, int SMAX, int HMAX>
struct LevelSmem {
  using R = typename M::R;
  static constexpr int NM = 8 * T + HMAX;  // MUSCL scratch entries
  static constexpr size_t off_W = 0;                                        // R [5][SMAX*8]
  static constexpr size_t off_M = off_W + sizeof(R) * 5 * SMAX * 8;         // R [20][NM]
  static constexpr size_t off_F = off_M + sizeof(R) * 20 * NM;              // R [15][8T]
  static constexpr size_t off_key = off_F + sizeof(R) * 15 * 8 * T;         // u32 [SMAX]
  static constexpr size_t off_G = off_key + sizeof(uint32_t) * SMAX;        // u8 [SMAX*6]
  static constexpr size_t off_H = (off_G + 6 * SMAX + 15) & ~size_t(15);    // u16 [SMAX*8]
  static constexpr size_t off_S = off_H + sizeof(uint16_t) * SMAX * 8;      // u8 [SMAX*8]
  static constexpr size_t bytes = (off_S + SMAX * 8 + 15) & ~size_t(15);
};

template <class M, int T, int SMAX, int HMAX>
__global__ void __launch_bounds__(8 * T, (sizeof(typename M::R) == 8) ? 1 : 2)
    level_advance_kernel(const LevelArgs A) {
  using R = typename M::R;
  using SM = LevelSmem<M, T, SMAX, HMAX>;
  constexpr int NM = SM::NM;
  extern __shared__ __align__(16) unsigned char smem[];
  R *sW = reinterpret_cast<R *>(smem + SM::off_W);
  R *sM = reinterpret_cast<R *>(smem + SM::off_M);
  R *sF = reinterpret_cast<R *>(smem + SM::off_F);
  uint32_t *sKey = reinterpret_cast<uint32_t *>(smem + SM::off_key);
  uint8_t *sG = smem + SM::off_G;
  uint16_t *sH = reinterpret_cast<uint16_t *>(smem + SM::off_H);
  uint8_t *sSp = smem + SM::off_S;

  const int tid = threadIdx.x;
  const TileDesc td = A.tiles[blockIdx.x];
  const int n = td.noct, S = td.S, H = td.H;
  const long long n8 = 8LL * A.noct;
  unsigned st = 0;
  if (S > SMAX || H > HMAX || n > T) {  // plan built for another kernel shape
    if (tid == 0) atomicOr(A.status, kStTree);
    return;
  }

  // ------------------------------------------------------------------ P0
  for (int i = tid; i < S; i += 8 * T) sKey[i] = A.keys[td.keys_off + i];
  for (int i = tid; i < S * 6; i += 8 * T) sG[i] = A.graph[td.graph_off + i];
  for (int i = tid; i < S * 8; i += 8 * T) sH[i] = 0xFFFF;
  __syncthreads();
  for (int i = tid; i < H; i += 8 * T) sH[A.halo[td.halo_off + i]] = (uint16_t)(8 * T + i);
  for (int i = tid; i < S * 8; i += 8 * T) {
    const int s = i >> 3, c = i & 7;
    const uint32_t key = sKey[s];
    const uint32_t kind = key >> 28, idx = key & 0x0FFFFFFFu;
    const double *src;
    long long stride, off;
    uint8_t sp = 0;
    if (kind == kKeyReal) {
      src = A.W; stride = n8; off = 8LL * idx + c;
      sp = (A.split[idx] >> c) & 1;
    } else if (kind == kKeyInj) {
      src = A.Wc; stride = A.nc8; off = idx;
      if (src == nullptr) {  // plan/launch mismatch: never read through a null level
        st |= kStTree;
        src = A.W; stride = n8; off = 0;
      }
    } else {
      const int mc = c_mirror[kind - kKeyGhost0][c];
      src = A.W; stride = n8; off = 8LL * idx + mc;
      sp = (A.split[idx] >> mc) & 1;
    }
#pragma unroll
    for (int v = 0; v < 5; v++) sW[v * SMAX * 8 + i] = (R)__ldg(src + v * stride + off);
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
  auto mi_of = [&](int s, int c) -> int { return (s < n) ? (s * 8 + c) : (int)sH[s * 8 + c]; };

  // ------------------------------------------------------------------ P1
  const R dt = (R)A.dt, dx = (R)A.dx;
  for (int j = tid; j < 8 * T + H; j += 8 * T) {
    int s, c;
    if (j < 8 * T) {
      if (j >= 8 * n) continue;
      s = j >> 3; c = j & 7;
    } else {
      const int e = A.halo[td.halo_off + (j - 8 * T)];
      s = e >> 3; c = e & 7;
    }
    if (sSp[s * 8 + c]) continue;  // split cells have no flux: no reconstruction needed
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
    R D[3][5], Wt[5];
    if constexpr (sizeof(R) == 8) M::muscl(q0, qm, qp, dt, dx, D, Wt);
    else M::muscl(q0, qm, qp, (R)(A.dt / A.dx * 0.5), D, Wt);
#pragma unroll
    for (int dir = 0; dir < 3; dir++)
#pragma unroll
      for (int v = 0; v < 5; v++) sM[(dir * 5 + v) * NM + j] = D[dir][v];
#pragma unroll
    for (int v = 0; v < 5; v++) sM[(15 + v) * NM + j] = Wt[v];
  }
  __syncthreads();

  auto face_of = [&](int s, int c, int mi, int k, R W[7]) {
    R q0[5], D[3][5], Wt[5];
    q_of(s, c, q0);
#pragma unroll
    for (int dir = 0; dir < 3; dir++)
#pragma unroll
      for (int v = 0; v < 5; v++) D[dir][v] = sM[(dir * 5 + v) * NM + mi];
#pragma unroll
    for (int v = 0; v < 5; v++) Wt[v] = sM[(15 + v) * NM + mi];
    M::face(q0, D, Wt, k, W, st);
  };

  // ------------------------------------------------------------------ P2
  R Fp[3][5];
  bool own_plus[3] = {false, false, false};
  const bool active = tid < 8 * n;
  const int o = tid >> 3, c = tid & 7;
  const bool my_split = active ? (sSp[tid] != 0) : true;
  if (active) {
#pragma unroll
    for (int d = 0; d < 3; d++) {
      // minus face: left = -d neighbour's +d state, right = own -d state
      R F[5] = {0, 0, 0, 0, 0};
      int c2;
      int s2 = nb(o, c, 2 * d, c2);
      if (!my_split) {
        if (s2 < 0) {
          st |= kStTree;
        } else if (!sSp[s2 * 8 + c2]) {
          const int mi = mi_of(s2, c2);
          if (mi == 0xFFFF) {
            st |= kStTree;
          } else {
            R WL[7], WR[7];
            face_of(s2, c2, mi, 2 * d + 1, WL);
            face_of(o, c, tid, 2 * d, WR);
            M::hllc(WL, WR, d, F, st);
          }
        }
      }
#pragma unroll
      for (int v = 0; v < 5; v++) sF[(d * 5 + v) * 8 * T + tid] = F[v];
      // plus face on the tile boundary
#pragma unroll
      for (int v = 0; v < 5; v++) Fp[d][v] = 0;
      s2 = nb(o, c, 2 * d + 1, c2);
      if (s2 < 0 || s2 >= n) {
        own_plus[d] = true;
        if (!my_split) {
          if (s2 < 0) {
            st |= kStTree;
          } else if (!sSp[s2 * 8 + c2]) {
            const int mi = mi_of(s2, c2);
            if (mi == 0xFFFF) {
              st |= kStTree;
            } else {
              R WL[7], WR[7];
              face_of(o, c, tid, 2 * d + 1, WL);
              face_of(s2, c2, mi, 2 * d, WR);
              M::hllc(WL, WR, d, Fp[d], st);
            }
          }
        }
      }
    }
  }
  __syncthreads();

  // ------------------------------------------------------------------ P3
  if (active) {
    const long long gi = 8LL * (td.oct0 + o) + c;
    double Wout[5];
    if (my_split) {
      // split cell: primitive mean of the 8 children (src/hydro_utils.c:3420-3481);
      // without the finer level (drop-in mode) the caller averages on the host
      const long long ch = A.child[gi];
      double acc[5] = {0., 0., 0., 0., 0.};
      if (A.Wf == nullptr) {
#pragma unroll
        for (int v = 0; v < 5; v++) acc[v] = A.W[v * n8 + gi];
      } else if (ch >= 0) {
        for (int i = 0; i < 8; i++)
#pragma unroll
          for (int v = 0; v < 5; v++) acc[v] += A.Wf[v * A.nf8 + 8 * ch + i] * 0.125;
      } else {
        st |= kStTree;
      }
#pragma unroll
      for (int v = 0; v < 5; v++) Wout[v] = acc[v];
    } else {
      const double dtsurdx = A.dt / A.dx;
      // fluxes of the six faces in the reference's order
      double Fd[6][5];
#pragma unroll
      for (int d = 0; d < 3; d++) {
#pragma unroll
        for (int v = 0; v < 5; v++) Fd[2 * d][v] = (double)sF[(d * 5 + v) * 8 * T + tid];
        if (own_plus[d]) {
#pragma unroll
          for (int v = 0; v < 5; v++) Fd[2 * d + 1][v] = (double)Fp[d][v];
        } else {
          int c2;
          const int s2 = nb(o, c, 2 * d + 1, c2);
          const int t2 = s2 * 8 + c2;
#pragma unroll
          for (int v = 0; v < 5; v++) Fd[2 * d + 1][v] = (double)sF[(d * 5 + v) * 8 * T + t2];
        }
      }
      double q[5];
#pragma unroll
      for (int v = 0; v < 5; v++) q[v] = A.W[v * n8 + gi];
      double corr[5];
#pragma unroll
      for (int v = 0; v < 5; v++) corr[v] = (A.C != nullptr && A.B == nullptr) ? A.C[v * n8 + gi] : 0.;
      double Ud, Udu, Udv, Udw, UE;
      if constexpr (sizeof(R) == 8) {
        // updatefield (src/hydro_utils.c:3050-3082): dU = sum (+-F dt/dx), alternating signs
        double dU[5] = {0., 0., 0., 0., 0.};
        double one = 1.;
#pragma unroll
        for (int f = 0; f < 6; f++) {
#pragma unroll
          for (int v = 0; v < 5; v++) dU[v] += Fd[f][v] * dtsurdx * one;
          one *= -1.;
        }
        // scatterstencil central update (src/hydro_utils.c:3129-3188): W2U + dU
        if (A.B != nullptr) {
          const double bd = A.B[gi];
          Ud = bd;
          Udu = bd * A.B[n8 + gi];
          Udv = bd * A.B[2 * n8 + gi];
          Udw = bd * A.B[3 * n8 + gi];
          UE = A.B[5 * n8 + gi];
        } else {
          const double E0 = q[4] / (kGam - 1.) + 0.5 * q[0] * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
          Ud = q[0] + corr[0];
          Udu = q[0] * q[1] + corr[1];
          Udv = q[0] * q[2] + corr[2];
          Udw = q[0] * q[3] + corr[3];
          UE = E0 + corr[4];
        }
        Ud += dU[0];
        Udu += dU[1];
        Udv += dU[2];
        Udw += dU[3];
        UE += dU[4];
      } else {
        // mixed: FP32 fluxes, FP64 Neumaier-compensated accumulation of
        // W2U(state) + corrections + sum(+-F dt/dx)
        double s[5];
        if (A.B != nullptr) {
          const double bd = A.B[gi];
          s[0] = bd; s[1] = bd * A.B[n8 + gi]; s[2] = bd * A.B[2 * n8 + gi]; s[3] = bd * A.B[3 * n8 + gi];
          s[4] = A.B[5 * n8 + gi];
        } else {
          s[0] = q[0]; s[1] = q[0] * q[1]; s[2] = q[0] * q[2]; s[3] = q[0] * q[3];
          s[4] = q[4] / (kGam - 1.) + 0.5 * q[0] * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
        }
        double comp[5] = {0., 0., 0., 0., 0.};
        auto add = [&](int v, double x) {
          const double t = s[v] + x;
          comp[v] += (fabs(s[v]) >= fabs(x)) ? ((s[v] - t) + x) : ((x - t) + s[v]);
          s[v] = t;
        };
#pragma unroll
        for (int v = 0; v < 5; v++) add(v, corr[v]);
#pragma unroll
        for (int f = 0; f < 6; f++)
#pragma unroll
          for (int v = 0; v < 5; v++) add(v, (f & 1) ? -(Fd[f][v] * dtsurdx) : (Fd[f][v] * dtsurdx));
        Ud = s[0] + comp[0];
        Udu = s[1] + comp[1];
        Udv = s[2] + comp[2];
        Udw = s[3] + comp[3];
        UE = s[4] + comp[4];
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
        for (int v = 0; v < 5; v++) atomicAdd(A.Cc + v * A.nc8 + cc, Fd[k][v] * dtsurdx * one * 0.125);
      }
    }
#pragma unroll
    for (int v = 0; v < 5; v++) A.Wn[v * n8 + gi] = Wout[v];
  }
  if (st) atomicOr(A.status, st);
}

}  // namespace emma
