// column_kernel.cuh -- the hydro level advance of a complete periodic level
// without split cells (a uniform box, the base level of a tree refined nowhere),
// marching through z.
//
// A work item is a column of 16 x 16 cells in x,y and `nz` cell planes in z.
// The CTA walks its planes bottom to top.  Per plane it converts the staged
// plane (the column and a halo of two cells) from the FP64 state to FP32 once,
// reconstructs every cell of the column and of its one-cell ring once (MUSCL-
// Hancock slopes and predictor, stored as the predicted state X and the three
// limited slopes), solves every face once (the -x, -y and -z face of each
// column cell, the +x and +y faces on the column's boundary from the ring), and
// updates the column cells in FP64.  The brick kernel (level_kernel.cuh)
// stages a 4.5x larger box per cell, reconstructs each advanced cell twice and
// solves 3.5 faces per cell; here it is 1.56x, 1.25 and 3.125 (the z halo is
// two planes per item).
//
// Software pipeline over planes, two barriers per plane.  Step s:
//   A  convert plane s+3 into the FP32 planes P (3 slots);
//      solve the faces of plane s+1 from the reconstructions R (2 slots) into
//      the fluxes FL (2 slots);
//   B  update plane s from FL; reconstruct plane s+2 from P into R.
// Threads (320): 256 own a column cell (x,y in 0..15), 64 the ring cells
// (x = -1, 16 with y in 0..15; y = -1, 16 with x in 0..15).  Each converts its
// own cell; the ring threads also convert the outer halo (x = -2, 17; y = -2, 17)
// and four column threads the ring's corner columns (+-1 diagonal).  Every face
// is solved at one call site per axis, so a face on the boundary of two columns
// (or of two z chunks) gets the same bits in both.
//
// XS (warp-shuffle x sweep): a warp holds two 16-cell x rows of the column, so
// the left neighbour of a column cell is the next lane down.  Each column thread
// computes both x face states of its own cell and passes the +x one up a lane
// (__shfl_up_sync) instead of reading the left cell's reconstruction from shared
// memory; the faces inside the column are solved there.  The column's two x
// boundary faces are solved by the x = -1 and x = 16 ring threads at the one
// call site of the shared-memory sweep, so a face shared by two columns still
// gets the same bits in both.  The autotuner times both sweeps.
//
// Work: a CTA runs either one item (column, nz planes) or, with
// ColumnArgs::balanced, an equal share of all the level's column-planes (two
// CTAs per SM, no partial last wave), cut into segments where it crosses into
// the next column.  Each segment stages and reconstructs its own z halo; as no
// face or cell depends on where a segment starts, both give the same bits.
//
// The reference does the same per oct on a 27-oct copy
// (src/hydro_utils.c:1407-2238, 2973-3303), recomputing each cell's
// reconstruction up to 9 times and each face twice.
#pragma once
#include <type_traits>
#include "hydro_math.cuh"
#include "plan_types.h"

namespace emma {

namespace col {
constexpr int TX = kColumnWidth, TY = kColumnWidth;
constexpr int kInt = TX * TY;       // column cells per plane
constexpr int kRec = kInt + 64;     // reconstructed cells per plane (column + ring)
constexpr int kColThreads = kRec;   // one thread per reconstructed cell
constexpr int PW = TX + 4;          // staged plane: x, y in -2 .. 17
constexpr int kP = PW * (TY + 4);
constexpr int kFl = kInt + 16;      // flux entries per axis: column cells, then the ring's boundary faces

// shared memory (bytes)
constexpr size_t kOffP4 = 0;                               // float4 [3][kP] (d,u,v,w)
constexpr size_t kOffPp = kOffP4 + 16 * 3 * kP;            // float  [3][kP] p
constexpr size_t kOffR = kOffPp + 4 * 3 * kP;              // float4 [2][5][kRec]
constexpr size_t kOffF4 = kOffR + 16 * 2 * 5 * kRec;       // float4 [2][3][kFl]
constexpr size_t kOffF1 = kOffF4 + 16 * 2 * 3 * kFl;       // float  [2][3][kFl]
constexpr size_t kSmem = kOffF1 + 4 * 2 * 3 * kFl;
static_assert(2 * (kSmem + 1024) <= 228 * 1024, "two CTAs per SM");

// ring cell r (0..63): x = -1 (r < 16), x = 16, y = -1, y = 16
__device__ __forceinline__ void ring_xy(int r, int &x, int &y) {
  const int side = r >> 4, i = r & 15;
  if (side < 2) {
    x = side ? TX : -1;
    y = i;
  } else {
    x = i;
    y = (side == 3) ? TY : -1;
  }
}
// outer halo column h (0..63): x = -2, 17 (y in 0..15), y = -2, 17 (x in 0..15)
__device__ __forceinline__ void halo_xy(int h, int &x, int &y) {
  const int side = h >> 4, i = h & 15;
  if (side < 2) {
    x = side ? TX + 1 : -2;
    y = i;
  } else {
    x = i;
    y = (side == 3) ? TY + 1 : -2;
  }
}
__device__ __forceinline__ int pidx(int x, int y) { return (y + 2) * PW + (x + 2); }
constexpr int kCornerT0 = kInt - 4;  // column threads that also convert a ring corner column
}  // namespace col

// The mixed path's column kernel: FP32 reconstruction and fluxes, FP64 update;
// XS: x faces inside the column through warp shuffles.
template <int MINB, bool XS>
__global__ void __launch_bounds__(col::kColThreads, MINB) column_kernel(const ColumnArgs a) {
  using namespace col;
  using M = MathF32;
  extern __shared__ __align__(16) unsigned char smem[];
  if (a.gate != nullptr && *a.gate == 0) return;
  const int item = blockIdx.x;
  if (item >= a.nitems) return;
  float4 *P4 = reinterpret_cast<float4 *>(smem + kOffP4);
  float *Pp = reinterpret_cast<float *>(smem + kOffPp);
  float4 *Rg = reinterpret_cast<float4 *>(smem + kOffR);
  float4 *F4 = reinterpret_cast<float4 *>(smem + kOffF4);
  float *F1 = reinterpret_cast<float *>(smem + kOffF1);

  const LevelArgs &A = *a.lv;
  const double *__restrict__ W = A.W;
  double *__restrict__ Wn = A.Wn;
  const long long N8 = 8LL * A.noct;
  const double dtsurdx = A.dt / A.dx;
  const float dtdx_half = (float)(A.dt / A.dx * 0.5);
  const int n = a.n, cmask = 2 * n - 1;
  const long long nn = (long long)n * n;
  const int *__restrict__ octidx = a.octidx;

  const int tid = threadIdx.x;
  const bool interior = tid < kInt;
  unsigned st = 0;
  double wmax = 0.;  // exact max signal speed of the cells this warp wrote (warp-uniform)

  int x0 = 0, y0 = 0;  // the column of the current segment (first cell in x, y)

  // this thread's cell (column or ring) and the second column it converts (ring
  // threads: an outer halo column; four column threads: a ring corner column)
  int rx, ry, hx = 0, hy = 0;
  if (interior) {
    rx = tid & 15;
    ry = tid >> 4;
  } else {
    ring_xy(tid - kInt, rx, ry);
  }
  const bool conv2 = !interior || tid >= kCornerT0;
  if (!interior) {
    halo_xy(tid - kInt, hx, hy);
  } else if (tid >= kCornerT0) {
    const int k = tid - kCornerT0;
    hx = (k & 1) ? TX : -1;
    hy = (k & 2) ? TY : -1;
  }
  const int rp = pidx(rx, ry), hp = pidx(hx, hy);
  // plane-independent parts of the global cell index (periodic in x, y)
  auto xy_part = [&](int x, int y, int &oxy, int &cxy) {
    const int xg = (x0 + x) & cmask, yg = (y0 + y) & cmask;
    oxy = (yg >> 1) * n + (xg >> 1);
    cxy = (xg & 1) | ((yg & 1) << 1);
  };
  int oxy1 = 0, cxy1 = 0, oxy2 = 0, cxy2 = 0;  // set per segment
  auto gidx = [&](int oxy, int cxy, int z) -> long long {
    const int zg = z & cmask;
    const int o = __ldg(octidx + (zg >> 1) * nn + oxy);
    return 8LL * o + (cxy | ((zg & 1) << 2));
  };
  auto load5 = [&](long long gi, double q[5]) {
#pragma unroll
    for (int v = 0; v < 5; v++) q[v] = __ldg(W + v * N8 + gi);
  };
  auto pstore = [&](int slot, int p, const double q[5]) {
    P4[slot * kP + p] = make_float4((float)q[0], (float)q[1], (float)q[2], (float)q[3]);
    Pp[slot * kP + p] = (float)q[4];
  };
  auto pload = [&](int slot, int p, float q[5]) {
    const float4 v = P4[slot * kP + p];
    q[0] = v.x;
    q[1] = v.y;
    q[2] = v.z;
    q[3] = v.w;
    q[4] = Pp[slot * kP + p];
  };
  // reconstruction of this thread's cell at the plane in P slot s0 (s_m below, s_p
  // above) into R buffer Rw: groups (X.d X.u X.v X.w) (X.p Dx.d Dx.u Dx.v)
  // (Dx.w Dx.p Dy.d Dy.u) (Dy.v Dy.w Dy.p Dz.d) (Dz.u Dz.v Dz.w Dz.p)
  auto reconstruct = [&](int s0, int sm, int sp, float4 *Rw) {
    float q0[5], qm[3][5], qp[3][5], D[3][5], Wt[5];
    pload(s0, rp, q0);
    pload(s0, rp - 1, qm[0]);
    pload(s0, rp + 1, qp[0]);
    pload(s0, rp - PW, qm[1]);
    pload(s0, rp + PW, qp[1]);
    pload(sm, rp, qm[2]);
    pload(sp, rp, qp[2]);
    M::muscl(q0, qm, qp, dtdx_half, D, Wt);
    float X[5];
#pragma unroll
    for (int v = 0; v < 5; v++) X[v] = q0[v] + Wt[v];
    Rw[tid] = make_float4(X[0], X[1], X[2], X[3]);
    Rw[kRec + tid] = make_float4(X[4], D[0][0], D[0][1], D[0][2]);
    Rw[2 * kRec + tid] = make_float4(D[0][3], D[0][4], D[1][0], D[1][1]);
    Rw[3 * kRec + tid] = make_float4(D[1][2], D[1][3], D[1][4], D[2][0]);
    Rw[4 * kRec + tid] = make_float4(D[2][1], D[2][2], D[2][3], D[2][4]);
  };
  // predicted state X and the slope along axis d of reconstructed cell r in R buffer R
  auto rload = [&](const float4 *R, int r, auto dc, float X[5], float Dd[5]) {
    constexpr int d = decltype(dc)::value;
    const float4 g0 = R[r], g1 = R[kRec + r];
    X[0] = g0.x;
    X[1] = g0.y;
    X[2] = g0.z;
    X[3] = g0.w;
    X[4] = g1.x;
    if constexpr (d == 0) {
      const float4 g2 = R[2 * kRec + r];
      Dd[0] = g1.y;
      Dd[1] = g1.z;
      Dd[2] = g1.w;
      Dd[3] = g2.x;
      Dd[4] = g2.y;
    } else if constexpr (d == 1) {
      const float4 g2 = R[2 * kRec + r], g3 = R[3 * kRec + r];
      Dd[0] = g2.z;
      Dd[1] = g2.w;
      Dd[2] = g3.x;
      Dd[3] = g3.y;
      Dd[4] = g3.z;
    } else {
      const float4 g3 = R[3 * kRec + r], g4 = R[4 * kRec + r];
      Dd[0] = g3.w;
      Dd[1] = g4.x;
      Dd[2] = g4.y;
      Dd[3] = g4.z;
      Dd[4] = g4.w;
    }
  };
  // one face normal to axis d: left cell rl in RL, right cell rr in RR, flux to entry f
  auto solve = [&](auto dc, const float4 *RL, int rl, const float4 *RR, int rr, int f) {
    constexpr int d = decltype(dc)::value;
    float X[5], Dd[5], WL[7], WR[7], F[5];
    rload(RL, rl, dc, X, Dd);
    M::face_px(X, Dd, 2 * d + 1, WL, st);
    rload(RR, rr, dc, X, Dd);
    M::face_px(X, Dd, 2 * d, WR, st);
    M::hllc(WL, WR, d, F, st);
    F4[f] = make_float4(F[0], F[1], F[2], F[3]);
    F1[f] = F[4];
  };
  // the x and y faces each thread solves: column cells their -x and -y faces, the
  // +x ring the column's +x boundary faces, the +y ring its +y boundary faces.
  // XS: column cells solve their -x face with the shuffle sweep, except those at
  // x = 0, whose -x face the -x ring solves at the shared-memory call site.
  const int ring = tid - kInt;
  const bool solve_x = XS ? (ring >= 0 && ring < 32) : (interior || (ring >= 16 && ring < 32));
  const bool solve_y = interior || ring >= 48;
  // the x face of a solve_x thread: left and right cell, flux entry
  int lx, rxc, ex;
  if (interior) {
    lx = (rx == 0) ? kInt + ry : tid - 1;
    rxc = tid;
    ex = tid;
  } else if (XS && ring < 16) {  // the column's -x boundary face: the ring cell | column cell (0, y)
    lx = tid;
    rxc = ry * TX;
    ex = ry * TX;
  } else {  // the column's +x boundary face: column cell (15, y) | the ring cell
    lx = ry * TX + TX - 1;
    rxc = tid;
    ex = kInt + ry;
  }
  const int ly = interior ? ((ry == 0) ? kInt + 32 + rx : tid - TX) : ((TY - 1) * TX + rx);
  const int ey = interior ? tid : kInt + rx;
  // XS: the -x faces inside the column; every column thread takes part in the
  // shuffle (column warps are whole), those at x = 0 drop their result
  auto solve_x_shfl = [&](const float4 *R, int fb) {
    float X[5], Dd[5], Wp[7], WL[7], WR[7], F[5];
    rload(R, tid, std::integral_constant<int, 0>{}, X, Dd);
    M::face_px(X, Dd, 1, Wp, st);  // toward +x: the right neighbour's left state
    M::face_px(X, Dd, 0, WR, st);
#pragma unroll
    for (int k = 0; k < 7; k++) WL[k] = __shfl_up_sync(0xffffffffu, Wp[k], 1);
    unsigned sx = 0;
    M::hllc(WL, WR, 0, F, sx);
    if (rx != 0) {
      st |= sx;
      F4[fb + tid] = make_float4(F[0], F[1], F[2], F[3]);
      F1[fb + tid] = F[4];
    }
  };
  // the +x and +y fluxes of a column cell
  const int px = (rx == TX - 1) ? kInt + ry : tid + 1, py = (ry == TY - 1) ? kInt + rx : tid + TX;

  // P slots of planes z-1, z, z+1 rotate through 0..2 (plane z in slot z mod 3)
  auto mod3 = [](int z) { return ((z % 3) + 3) % 3; };
  // One segment: planes [z0, z1) of the column (cx, cy), the two planes below and
  // one above it staged and reconstructed as its halo.  The result of a face or
  // cell does not depend on where a segment starts or ends.
  auto segment = [&](int cx, int cy, int z0, int z1) {
    x0 = cx * TX;
    y0 = cy * TY;
    xy_part(rx, ry, oxy1, cxy1);
    xy_part(hx, hy, oxy2, cxy2);
    // prologue: the two planes below the first reconstructed one
    {
      double q[5];
      for (int z = z0 - 2; z < z0; z++) {
        load5(gidx(oxy1, cxy1, z), q);
        pstore(mod3(z), rp, q);
        if (conv2) {
          load5(gidx(oxy2, cxy2, z), q);
          pstore(mod3(z), hp, q);
        }
      }
    }
    __syncthreads();

    int sc = mod3(z0);  // P slot of the plane converted in this step (s + 3)
    for (int s = z0 - 3; s < z1; s++) {
      // ---------------------------------------------------------------- A
      // loads of plane s+3 first; they land while the faces of plane s+1 are solved
      const bool conv = s + 3 <= z1 + 1;
      double q1[5], q2[5];
      if (conv) {
        load5(gidx(oxy1, cxy1, s + 3), q1);
        if (conv2) load5(gidx(oxy2, cxy2, s + 3), q2);
      }
      const int zs = s + 1;  // plane whose faces are solved
      if (zs >= z0 && zs <= z1) {
        const float4 *Rc = Rg + (zs & 1) * 5 * kRec, *Rb = Rg + ((zs - 1) & 1) * 5 * kRec;
        const int fb = (zs & 1) * 3 * kFl;
        if (zs < z1) {  // the plane above the column only closes its top face
          if constexpr (XS)
            if (interior) solve_x_shfl(Rc, fb);
          if (solve_x) solve(std::integral_constant<int, 0>{}, Rc, lx, Rc, rxc, fb + ex);
          if (solve_y) solve(std::integral_constant<int, 1>{}, Rc, ly, Rc, tid, fb + kFl + ey);
        }
        if (interior) solve(std::integral_constant<int, 2>{}, Rb, tid, Rc, tid, fb + 2 * kFl + tid);
      }
      if (conv) {
        pstore(sc, rp, q1);
        if (conv2) pstore(sc, hp, q2);
      }
      __syncthreads();
      // ---------------------------------------------------------------- B
      // the FP64 state of plane s is loaded first (from L2: the plane was staged three
      // steps ago) and lands while plane s+2 is reconstructed
      const bool upd = s >= z0 && interior;
      long long gi = 0;
      double q[5];
      if (upd) {
        gi = gidx(oxy1, cxy1, s);
        load5(gi, q);
      }
      const int zr = s + 2;  // plane reconstructed
      if (zr >= z0 - 1 && zr <= z1) {
        const int s0 = mod3(zr);
        reconstruct(s0, s0 == 0 ? 2 : s0 - 1, s0 == 2 ? 0 : s0 + 1, Rg + (zr & 1) * 5 * kRec);
      }
      if (upd) {
        // fluxes of the six faces, -x,+x,-y,+y,-z,+z, summed in FP64 with the signs of
        // updatefield (src/hydro_utils.c:3050-3082)
        const int fs = (s & 1) * 3 * kFl, fn = ((s + 1) & 1) * 3 * kFl;
        const int ef[6] = {fs + tid, fs + px, fs + kFl + tid, fs + kFl + py, fs + 2 * kFl + tid, fn + 2 * kFl + tid};
        double dU[5] = {0., 0., 0., 0., 0.};
  #pragma unroll
        for (int k = 0; k < 6; k++) {
          const float4 f = F4[ef[k]];
          const float f4 = F1[ef[k]];
          const double F[5] = {(double)f.x, (double)f.y, (double)f.z, (double)f.w, (double)f4};
  #pragma unroll
          for (int v = 0; v < 5; v++) dU[v] = (k & 1) ? dU[v] - F[v] : dU[v] + F[v];
        }
        // conserved state W2U(W) + dU dt/dx (src/hydro_utils.c:3129-3188).  The mixed
        // path's compensated sum of the base state and the flux divergence (the brick
        // kernel's, which also adds the corrections of a finer level) returns the
        // rounded sum when there are only these two terms, as on a level without split
        // cells: the compensation term is below half an ulp of the rounded sum.
        const double Ud = q[0] + dU[0] * dtsurdx;
        const double Udu = q[0] * q[1] + dU[1] * dtsurdx;
        const double Udv = q[0] * q[2] + dU[2] * dtsurdx;
        const double Udw = q[0] * q[3] + dU[3] * dtsurdx;
        const double UE = (q[4] / (kGam - 1.) + 0.5 * q[0] * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3])) + dU[4] * dtsurdx;
        // U2W (src/hydro_utils.c:35-64), pressure floor
        const double dl = (Ud == 0. ? 10. : Ud);
        const double inv = 1. / dl;
        double Wout[5];
        Wout[0] = Ud;
        Wout[1] = Udu * inv;
        Wout[2] = Udv * inv;
        Wout[3] = Udw * inv;
        Wout[4] = fmax((kGam - 1.) * (UE - (Udu * Udu + Udv * Udv + Udw * Udw) * inv * 0.5), kPmin);
        if (isnan(Wout[1]) || isnan(Wout[4]) || isnan(Wout[0])) st |= kStNan;
  #pragma unroll
        for (int v = 0; v < 5; v++) Wn[v * N8 + gi] = Wout[v];
        if (a.smax != nullptr) {
          // the next CFL step's |v| + c_s (src/advanceamr.c:122-128), exact in FP64 for
          // every cell that may raise this warp's maximum: an FP32 estimate (relative
          // error below 2e-6) screens the others out, whole warps at a time
          const float u = (float)Wout[1], v = (float)Wout[2], w = (float)Wout[3];
          const float s32 = sqrtf(u * u + v * v + w * w) + sqrtf(5.f / 3.f * (float)Wout[4] / (float)Wout[0]);
          const bool cand = !(s32 < (float)wmax * (1.f - 1e-5f));
          if (__any_sync(0xffffffffu, cand)) {
            double ex = 0.;
            if (cand) {
              const double va = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(Wout[1], Wout[1]), __dmul_rn(Wout[2], Wout[2])),
                                                     __dmul_rn(Wout[3], Wout[3])));
              const double aa = __dsqrt_rn(__ddiv_rn(__dmul_rn(5. / 3., Wout[4]), Wout[0]));
              ex = fmax(0., __dadd_rn(va, aa));  // fmax drops NaN like the reference's FMAX
            }
            for (int o = 16; o > 0; o >>= 1) ex = fmax(ex, __shfl_xor_sync(0xffffffffu, ex, o));
            wmax = fmax(wmax, ex);
          }
        }
      }
      __syncthreads();
      sc = (sc == 2) ? 0 : sc + 1;
    }
  };
  // this CTA's range of the level's column-planes (columns in order, each bottom
  // to top): an item (one column, nz planes), or an equal share of all of them cut
  // into segments where it crosses into the next column
  const int per_col = 2 * n;
  int p0, p1;
  if (a.balanced) {
    const long long total = (long long)a.ncol * a.ncol * per_col;
    p0 = (int)(total * blockIdx.x / gridDim.x);
    p1 = (int)(total * (blockIdx.x + 1) / gridDim.x);
  } else {
    const int cz = item / (a.ncol * a.ncol), col = item % (a.ncol * a.ncol);
    p0 = col * per_col + cz * a.nz;
    p1 = p0 + a.nz;
  }
  for (int pos = p0; pos < p1;) {
    const int col = pos / per_col, z = pos - col * per_col;
    const int zend = (p1 - pos < per_col - z) ? z + (p1 - pos) : per_col;
    segment(col % a.ncol, col / a.ncol, z, zend);
    pos += zend - z;
  }
  if (a.smax != nullptr && interior && (tid & 31) == 0 && wmax > 0.)
    atomicMax(a.smax + a.L, (unsigned long long)__double_as_longlong(wmax));
  if (st) atomicOr(a.status, st);
}

}  // namespace emma
