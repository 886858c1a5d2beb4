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
