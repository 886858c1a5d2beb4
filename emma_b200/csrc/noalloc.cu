// noalloc.cu -- level time step of a device-resident level state, computed
// without allocating any memory.
//
// Some callers cannot call cudaMalloc at all: a solver embedded in another
// code's memory pool (every byte on the device owned by that pool), a process
// that must not allocate after start-up, or a stream in the middle of work that
// an allocation would serialise.  emma_hydro_level_dt_noalloc serves them: the
// caller passes the level state already on the device and receives dt; the
// reduction's scratch is a fixed array inside this library.
//
// Scratch: g_dt_scratch, a file-scope __device__ array of kMaxBlocks + 1
// 64-bit slots (128 KiB + 8 B) that every GPU which loads the library holds
// until the process exits.  Slot b < kMaxBlocks receives the maximum signal
// speed of block b, slot kMaxBlocks the maximum over the blocks.  Every slot a
// call reads is written earlier in the same call, so nothing has to start at
// zero; the array keeps the last call's values.  Calls whose kernels overlap on
// the GPU (different streams, or several host threads) share the array and
// race: serialise them on one stream.
//
// Host code only ever uses the array's device address, obtained once per device
// with cudaGetSymbolAddress on the first call made while that device is
// current; that first call must therefore not be made during a stream capture.
// The address is cached for the life of the device's primary context: after a
// cudaDeviceReset (which unloads this library's module) call
// emma_hydro_noalloc_forget() before the next call, so that the address is
// looked up again in the new context.  The per-device cache slots are atomic, so
// host threads may make first calls concurrently.
//
// Built with -fmad=false: the signal speed rounds exactly as the reference's
// L_comptstep_hydro (src/advanceamr.c:122-135) and emma_hydro_comptstep do.
#include <cuda_runtime.h>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include "emma_hydro.h"

namespace {

constexpr int kThreads = 256;
constexpr int kCellsPerThread = 8;
constexpr int kMaxBlocks = 16384;
constexpr long long kCellsPerBlock = (long long)kThreads * kCellsPerThread;
constexpr long long kMaxCells = kMaxBlocks * kCellsPerBlock;  // 33,554,432 cells (a 256^3 level is 16,777,216)
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned long long g_dt_scratch[kMaxBlocks + 1];

std::atomic<unsigned long long *> g_scratch_addr[kMaxDevices];  // zero-initialised (static storage)

__device__ __forceinline__ double block_max(double m) {
  __shared__ double part[kThreads / 32];
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = m;
  __syncthreads();
  m = (threadIdx.x < kThreads / 32) ? part[threadIdx.x] : 0.;
  if (threadIdx.x < 32)
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  return m;
}

// per block: max over its cells of |v| + sqrt(gamma p / rho); W = 5 planes of n8 cells
__global__ void __launch_bounds__(kThreads) dt_partial_kernel(const double *__restrict__ W, long long n8,
                                                              unsigned long long *scratch) {
  double m = 0.;
  const long long base = blockIdx.x * kCellsPerBlock;
#pragma unroll
  for (int j = 0; j < kCellsPerThread; j++) {
    const long long i = base + (long long)j * kThreads + threadIdx.x;
    if (i < n8) {
      const double d = W[i], u = W[n8 + i], v = W[2 * n8 + i], w = W[3 * n8 + i], p = W[4 * n8 + i];
      const double va = sqrt(u * u + v * v + w * w);
      const double aa = sqrt((5. / 3.) * p / d);
      m = fmax(m, va + aa);  // fmax drops NaN like the reference's FMAX
    }
  }
  m = block_max(m);
  if (threadIdx.x == 0) scratch[blockIdx.x] = (unsigned long long)__double_as_longlong(m);
}

// one block: max over the partials -> scratch[kMaxBlocks]
__global__ void __launch_bounds__(kThreads) dt_final_kernel(unsigned long long *scratch, int nblocks) {
  double m = 0.;
  for (int b = threadIdx.x; b < nblocks; b += kThreads) m = fmax(m, __longlong_as_double((long long)scratch[b]));
  m = block_max(m);
  if (threadIdx.x == 0) scratch[kMaxBlocks] = (unsigned long long)__double_as_longlong(m);
}

}  // namespace

extern "C" int emma_hydro_level_dt_noalloc(const double *d_state, long long ncells, int level, double cfl,
                                           void *stream, double *dt_out) {
  if (d_state == nullptr || dt_out == nullptr || ncells < 0 || level < 1 || level > 40) {
    std::fputs("emma_hydro_level_dt_noalloc: null pointer, negative size or level out of range\n", stderr);
    return EMMA_ST_ARG;
  }
  if (ncells > kMaxCells) {
    std::fputs("emma_hydro_level_dt_noalloc: more than 33554432 cells, beyond the fixed scratch of this entry\n",
               stderr);
    return EMMA_ST_ARG;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return EMMA_ST_CUDA;
  unsigned long long *scratch = g_scratch_addr[dev].load(std::memory_order_acquire);
  if (scratch == nullptr) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_dt_scratch) != cudaSuccess || p == nullptr) return EMMA_ST_CUDA;
    scratch = static_cast<unsigned long long *>(p);
    g_scratch_addr[dev].store(scratch, std::memory_order_release);
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double smax = 0.;
  if (ncells > 0) {
    const int nblocks = (int)((ncells + kCellsPerBlock - 1) / kCellsPerBlock);
    dt_partial_kernel<<<nblocks, kThreads, 0, s>>>(d_state, ncells, scratch);
    dt_final_kernel<<<1, kThreads, 0, s>>>(scratch, nblocks);
    if (cudaGetLastError() != cudaSuccess) return EMMA_ST_CUDA;
    unsigned long long bits = 0;
    if (cudaMemcpyAsync(&bits, scratch + kMaxBlocks, sizeof(bits), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return EMMA_ST_CUDA;
    std::memcpy(&smax, &bits, sizeof(smax));
  }
  // L_comptstep_hydro's final step (src/advanceamr.c:135)
  double dt = 1e9;
  const double dxcur = std::pow(0.5, level);
  if (smax > 0.) dt = std::fmin(dxcur * cfl / (smax * 3.), dt);
  *dt_out = dt;
  return 0;
}

extern "C" void emma_hydro_noalloc_forget(void) {
  for (int d = 0; d < kMaxDevices; d++) g_scratch_addr[d].store(nullptr, std::memory_order_release);
}
