// Gauss-law residual over caller-owned FP32 field planes, without allocating.
//
// For callers that cannot allocate device memory themselves -- code that runs
// as a plugin inside a host application which owns every device allocation
// (a pre-reserved memory pool, an allocator that plugins must not bypass) --
// this entry point takes its inputs and its output as caller-provided device
// pointers and keeps its only scratch, the per-block partial sums of a
// two-pass reduction, in the file-scope device array below. That array
// exists once per GPU that loads the library and lives until the process
// exits. Its size caps the input: at most kMaxBlocks blocks of kThreads
// threads, each thread covering up to kCellsPerThread cells.
//
// Host code must not pass `g_noalloc_partials` itself to a kernel: in host code
// that name is a host-side stand-in, not a device address. Every call looks the
// device address up with cudaGetSymbolAddress in the calling thread's current
// context and passes that to the kernels, so a context the host application
// created itself, or one re-created after cudaDeviceReset, gets its own
// address. The first call in a context also loads the library's device code
// into it (a one-time set-up); make that first call before any stream capture.
//
// Every call reuses the same array and leaves its partial sums there. Each
// call overwrites every partial slot it later reads, so nothing has to be
// cleared between calls, but two calls whose kernels overlap on the GPU (for
// example on two streams at once) race on the array and must be ordered by the
// caller.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>

#include "../../include/plasma_b200.h"

namespace {

constexpr int kThreads = 256;
constexpr int kCellsPerThread = 64;
constexpr int kMaxBlocks = 2048;
constexpr int kFinalThreads = 256;

// [kMaxBlocks][4]: sum r^2, sum (rho/e0)^2, max |r|, cells of each block
__device__ __align__(256) double g_noalloc_partials[kMaxBlocks * 4];

struct Planes {
  const float *ex, *ey, *ez, *ni, *ne;
};

__global__ void __launch_bounds__(kThreads) gauss_partials_kernel(Planes p, int nx, int ny, int nz,
                                                                  double inv24dx, double q_e0,
                                                                  double* partials) {
  const int gy = ny + 4, gz = nz + 4, sx = gy * gz, sy = gz;
  const long long ncells = (long long)nx * ny * nz;
  double s2 = 0.0, r2 = 0.0, mx = 0.0, cnt = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < ncells;
       t += (long long)gridDim.x * blockDim.x) {
    const int m = 2 + (int)(t % nz), l = 2 + (int)((t / nz) % ny), k = 2 + (int)(t / ((long long)nz * ny));
    const long long n = (long long)k * sx + (long long)l * sy + m;
    const double dvx = 27.0 * ((double)p.ex[n + sx] - (double)p.ex[n]) - ((double)p.ex[n + 2 * sx] - (double)p.ex[n - sx]);
    const double dvy = 27.0 * ((double)p.ey[n + sy] - (double)p.ey[n]) - ((double)p.ey[n + 2 * sy] - (double)p.ey[n - sy]);
    const double dvz = 27.0 * ((double)p.ez[n + 1] - (double)p.ez[n]) - ((double)p.ez[n + 2] - (double)p.ez[n - 1]);
    const double rho = q_e0 * ((double)p.ni[n] - (double)p.ne[n]);
    const double r = (dvx + dvy + dvz) * inv24dx - rho;
    s2 += r * r;
    r2 += rho * rho;
    mx = fmax(mx, fabs(r));
    cnt += 1.0;
  }
  __shared__ double sm[4][kThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    s2 += __shfl_down_sync(0xffffffffu, s2, o);
    r2 += __shfl_down_sync(0xffffffffu, r2, o);
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    cnt += __shfl_down_sync(0xffffffffu, cnt, o);
  }
  if (lane == 0) {
    sm[0][wid] = s2; sm[1][wid] = r2; sm[2][wid] = mx; sm[3][wid] = cnt;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0, c = 0.0, d = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) {
      a += sm[0][w]; b += sm[1][w]; c = fmax(c, sm[2][w]); d += sm[3][w];
    }
    double* o = partials + 4 * blockIdx.x;
    o[0] = a; o[1] = b; o[2] = c; o[3] = d;
  }
}

// The block partials summed by one block: thread t takes partials t,
// t + kFinalThreads, ... in turn, then the threads' sums are combined in a
// fixed tree, so that repeated calls on the same input give the same bits.
__global__ void __launch_bounds__(kFinalThreads) gauss_final_kernel(const double* partials, int nblocks,
                                                                    double* out4) {
  double a = 0.0, b = 0.0, c = 0.0, d = 0.0;
  for (int q = threadIdx.x; q < nblocks; q += kFinalThreads) {
    a += partials[4 * q]; b += partials[4 * q + 1]; c = fmax(c, partials[4 * q + 2]); d += partials[4 * q + 3];
  }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
    c = fmax(c, __shfl_down_sync(0xffffffffu, c, o));
    d += __shfl_down_sync(0xffffffffu, d, o);
  }
  __shared__ double sm[4][kFinalThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    sm[0][wid] = a; sm[1][wid] = b; sm[2][wid] = c; sm[3][wid] = d;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    a = b = c = d = 0.0;
    for (int w = 0; w < kFinalThreads / 32; ++w) {
      a += sm[0][w]; b += sm[1][w]; c = fmax(c, sm[2][w]); d += sm[3][w];
    }
    out4[0] = a; out4[1] = b; out4[2] = c; out4[3] = d;
  }
}

// Device address of the scratch array in the current context.
int partials_address(double** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
  if (e != cudaSuccess) {
    fprintf(stderr, "plasma_b200: cudaGetSymbolAddress: %s\n", cudaGetErrorString(e));
    return PIC_ERR_CUDA;
  }
  *out = static_cast<double*>(p);
  return PIC_OK;
}

}  // namespace

extern "C" int pic_gauss_residual_noalloc(const float* ex, const float* ey, const float* ez,
                                          const float* ni, const float* ne, int nx, int ny, int nz,
                                          double dx, double q, double e0, void* stream, double* out4) {
  if (!ex || !ey || !ez || !ni || !ne || !out4 || nx < 1 || ny < 1 || nz < 1 || !std::isfinite(dx) ||
      !(dx > 0) || !std::isfinite(q) || !std::isfinite(e0) || e0 == 0)
    return PIC_ERR_ARG;
  const long long ncells = (long long)nx * ny * nz;
  const long long per_block = (long long)kThreads * kCellsPerThread;
  const long long nblocks = (ncells + per_block - 1) / per_block;
  if (nblocks > kMaxBlocks) {
    fprintf(stderr,
            "plasma_b200: pic_gauss_residual_noalloc: %lld cells exceed the %lld-cell maximum of its "
            "static scratch\n",
            ncells, (long long)kMaxBlocks * per_block);
    return PIC_ERR_TOO_LARGE;
  }
  double* partials = nullptr;
  const int rc = partials_address(&partials);
  if (rc != PIC_OK) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Planes p{ex, ey, ez, ni, ne};
  gauss_partials_kernel<<<(unsigned)nblocks, kThreads, 0, s>>>(p, nx, ny, nz, 1.0 / (24.0 * dx), q / e0, partials);
  if (cudaGetLastError() != cudaSuccess) return PIC_ERR_CUDA;
  gauss_final_kernel<<<1, kFinalThreads, 0, s>>>(partials, (int)nblocks, out4);
  if (cudaGetLastError() != cudaSuccess) return PIC_ERR_CUDA;
  return PIC_OK;
}
