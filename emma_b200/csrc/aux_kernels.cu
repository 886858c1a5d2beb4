// aux_kernels.cu -- level time step (CFL) reduction.  Built with -fmad=false:
// the per-cell signal speed must round as L_comptstep_hydro's does
// (src/advanceamr.c:122-128), so that the level dt is bit-identical.
#include <cuda_runtime.h>
#include <stdint.h>
#include "plan_types.h"

namespace emma {

__global__ void cfl_smax_kernel(const LevelArgs *lv, int slot, const int *gate, unsigned long long *out) {
  if (gate != nullptr && *gate == 0) return;
  const double *__restrict__ W = lv[slot].W;
  const long long n8 = 8LL * lv[slot].noct;
  double m = 0.;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n8; i += (long long)gridDim.x * blockDim.x) {
    const double d = W[i], u = W[n8 + i], v = W[2 * n8 + i], w = W[3 * n8 + i], p = W[4 * n8 + i];
    const double va = sqrt(u * u + v * v + w * w);
    const double aa = sqrt((5. / 3.) * p / d);
    const double s = va + aa;
    m = fmax(m, s);  // fmax drops NaN like the reference's FMAX
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ double sm[32];
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = (threadIdx.x < (blockDim.x >> 5)) ? sm[threadIdx.x] : 0.;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    // non-negative doubles order like their bit patterns
    if (threadIdx.x == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
  }
}

cudaError_t launch_cfl(const LevelArgs *lv, int slot, long long n8, const int *gate, unsigned long long *out, int nsm,
                       cudaStream_t s) {
  long long blocks = (n8 + 255) / 256;
  long long cap = 4LL * nsm;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  cfl_smax_kernel<<<(unsigned)blocks, 256, 0, s>>>(lv, slot, gate, out);
  return cudaGetLastError();
}

}  // namespace emma

namespace emma {

// coarse2fine_hydro2 (src/hydro_utils.c:311-420) for the transmissive build's
// gather: each listed level L-1 cell is interpolated into 8 sub-cells with
// minmod-limited slopes from its listed neighbours, W = W0 + ox Dx + oy Dy + oz Dz
// with o = -0.25 or +0.25, evaluated in that order (built with -fmad=false).
__device__ __forceinline__ double minmod_w(double m, double p) {
  if (p > 0) return fmax(fmax(0., fmin(m, p)), fmin(m, p));
  return fmin(fmin(0., fmax(m, p)), fmax(m, p));
}

__global__ void interp_coarse_kernel(const LevelArgs *lv, int slot, const int *gate) {
  if (gate != nullptr && *gate == 0) return;
  const LevelArgs &A = lv[slot];
  const double *Wc = A.Wc;
  if (Wc == nullptr || A.Wv == nullptr) return;
  const long long nc8 = A.nc8, nv = A.nv, nv8 = 8 * A.nv;
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < nv; j += (long long)gridDim.x * blockDim.x) {
    const int *vc = A.vcell + 7 * j;
    double q0[5], D[3][5];
#pragma unroll
    for (int v = 0; v < 5; v++) q0[v] = Wc[v * nc8 + vc[0]];
#pragma unroll
    for (int dir = 0; dir < 3; dir++) {
      const int cm = vc[1 + 2 * dir], cp = vc[2 + 2 * dir];
#pragma unroll
      for (int v = 0; v < 5; v++) D[dir][v] = minmod_w(q0[v] - Wc[v * nc8 + cm], Wc[v * nc8 + cp] - q0[v]);
    }
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const double ox = (c & 1) ? 0.25 : -0.25, oy = ((c >> 1) & 1) ? 0.25 : -0.25, oz = (c >> 2) ? 0.25 : -0.25;
#pragma unroll
      for (int v = 0; v < 5; v++) A.Wv[v * nv8 + 8 * j + c] = q0[v] + ox * D[0][v] + oy * D[1][v] + oz * D[2][v];
    }
  }
}

// Gravity builds: the force of each listed coarse cell spread over its 8
// sub-cells by coarse2fine_forcelin (src/poisson_utils.c:315-425): unlimited
// one-sided differences, f = f0 + Dx ox + Dy oy + Dz oz with D = f0 - f(-nei)
// for a sub-cell on the - side of an axis and f(+nei) - f0 on the + side,
// o = -1/4 or +1/4 (built with -fmad=false).  One thread per sub-cell.
__global__ void force_interp_kernel(const LevelArgs *lv, int slot, const int *gate) {
  if (gate != nullptr && *gate == 0) return;
  const LevelArgs &A = lv[slot];
  if (A.Fc == nullptr || A.Fv == nullptr) return;
  const long long nc8 = A.nc8, nv8 = 8 * A.nv;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv8; i += (long long)gridDim.x * blockDim.x) {
    const long long j = i >> 3;
    const int c = (int)(i & 7), ix = c & 1, iy = (c >> 1) & 1, iz = c >> 2;
    const int *vc = A.vcell + 7 * j;
    const int c0 = vc[0], nx = vc[1 + ix], ny = vc[3 + iy], nz = vc[5 + iz];
#pragma unroll
    for (int v = 0; v < 3; v++) {
      const double *F = A.Fc + v * nc8;
      const double f0 = F[c0];
      const double dx = ix ? F[nx] - f0 : f0 - F[nx];
      const double dy = iy ? F[ny] - f0 : f0 - F[ny];
      const double dz = iz ? F[nz] - f0 : f0 - F[nz];
      A.Fv[v * nv8 + i] = f0 + dx * (-0.25 + ix * 0.5) + dy * (-0.25 + iy * 0.5) + dz * (-0.25 + iz * 0.5);
    }
  }
}

// grav: the level belongs to a gravity build (forces interpolated, states injected),
// else a transmissive build (states interpolated)
cudaError_t launch_interp(const LevelArgs *lv, int slot, long long nv, const int *gate, int nsm, cudaStream_t s,
                          bool grav) {
  if (nv <= 0) return cudaSuccess;
  if (grav) {
    long long blocks = (8 * nv + 255) / 256;
    if (blocks > 8LL * nsm) blocks = 8LL * nsm;
    force_interp_kernel<<<(unsigned)blocks, 256, 0, s>>>(lv, slot, gate);
    return cudaGetLastError();
  }
  long long blocks = (nv + 127) / 128;
  if (blocks > 4LL * nsm) blocks = 4LL * nsm;
  interp_coarse_kernel<<<(unsigned)blocks, 128, 0, s>>>(lv, slot, gate);
  return cudaGetLastError();
}

}  // namespace emma

namespace emma {

// Drop-in base state: fieldnew = field (planes d,u,v,w,p,E of the uploaded
// block) except for the listed cells {cell, d, u, v, w, p, E, 0}.
__global__ void dropin_base_copy(const double *wb, double *base, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    base[i] = wb[i];
}
__global__ void dropin_base_scatter(double *base, long long n8, const double *exc, long long nexc, int np, int rec) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < nexc; j += (long long)gridDim.x * blockDim.x) {
    const double *e = exc + (long long)rec * j;
    const long long k = (long long)e[0];
    if (k < 0 || k >= n8) continue;
    for (int v = 0; v < np; v++) base[v * n8 + k] = e[1 + v];
  }
}

cudaError_t launch_dropin_base(const double *wb, double *base, long long n8, const double *exc, long long nexc, int nsm,
                               cudaStream_t s, int np, int rec) {
  if (np < 6 || np > 9 || rec < np + 1) return cudaErrorInvalidValue;  // a record: the cell, then np values
  const long long n = np * n8;
  long long blocks = (n + 255) / 256;
  if (blocks > 8LL * nsm) blocks = 8LL * nsm;
  if (n > 0) dropin_base_copy<<<(unsigned)blocks, 256, 0, s>>>(wb, base, n);
  if (nexc > 0) {
    long long b2 = (nexc + 255) / 256;
    if (b2 > 8LL * nsm) b2 = 8LL * nsm;
    dropin_base_scatter<<<(unsigned)b2, 256, 0, s>>>(base, n8, exc, nexc, np, rec);
  }
  return cudaGetLastError();
}

}  // namespace emma
