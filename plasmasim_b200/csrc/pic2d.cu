// Batched 2D particle-in-cell runs of PIC2D/2d_pic278_mpi.c (the x-z sail
// model) at MPI size 1: many independent runs of uneven grid sizes advanced
// together, every phase of the step one batched kernel over all runs, the
// step replayed from CUDA graphs.
//
// Per run the step is fdtd's loop body (:627-1015): renew_grid; add_ion5 /
// add_electron5 every add_interval steps (:645-653, :3311-3566); renew_b4
// (:1391-1417) + sr_grid; the push loop (cal_track_c4 :1520-1560 with the
// bilinear gathers :1948-2016, the ballistic margins :682-686, the J deposit
// :2018-2145); sr_current (:1073-1144) and external_current_perp (:2238-2268);
// renew_b4 + sr_grid; the drift loop with the density deposit (:762-828) and
// sr_density (:1146-1209); renew_e4 (:1419-1449) + sr_grid; renew_phi
// (:2589-2771) + sr_grid; the x exchange and the removal (:861-960).
// thrust_F (:2304-2387) on request.
//
// Layout: runs are concatenated. Fields: per run 18 planes of (nx+4)(nz+4)
// nodes, z fastest. Particles: per species one pool, run r owning slots
// [poff_r, poff_r + cap_r): cell (i << 16 | k), the in-cell offsets along x
// and z, and vx vy vz, in the tiled layout of Layout2 (one lane column of 32
// slot-wide rows per cell), which the cell sort rebuilds every sort_interval
// steps and after each refill. Work lists map persistent blocks onto (run,
// chunk) or (run, tile) items so that one launch covers every run whatever
// its size.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/plasma_b200.h"
#include "common.cuh"
#include "particles.cuh"

using namespace pb;

namespace p2 {

enum Plane {
  P_EX, P_EY, P_EZ, P_BX, P_BY, P_BZ, P_B0X, P_B0Y, P_B0Z,
  P_JIX, P_JIY, P_JIZ, P_JEX, P_JEY, P_JEZ, P_NI, P_NE, P_PHI, P_COUNT
};
static_assert(P_EY == P_EX + 1 && P_BZ == P_EX + 5 && P_JEX == P_JIX + 3 && P_NE == P_NI + 1,
              "the push indexes E, B, J and n planes by offset");

constexpr int kChunk = 2048;     // particle slots per work item

constexpr int kCellShift = 16;   // cell = (i << 16) | k

__host__ __device__ __forceinline__ int pack2(int i, int k) { return (i << kCellShift) | k; }
__host__ __device__ __forceinline__ void unpack2(int c, int& i, int& k) {
  i = c >> kCellShift;
  k = c & ((1 << kCellShift) - 1);
}

// Constant description of one run on the device.
template <typename real>
struct Run {
  int nx, nz, gx, gz, nodes;
  int np;                 // particles per cell per axis (Np); Np*Np per cell
  long long foff;         // first node of the run's field block (18 planes)
  long long poff;         // first slot in each species pool
  long long cap;          // slots per species
  int a1, a2, a3;         // Absorb_grid (fields), Absorb_grid2 (particles), Absorb_grid3 (phi)
  double dx, dt, q, e0, mu0, c;
  double sigma_a;
  double coil_i;
  double vdrift, sig[2];  // drift and thermal spread per species
  double nw;              // N0i = N0e = Nall / Np / Np
  double T[2];            // 0.5 q dt / m, m < 0 for electrons
  double ex_add, ey_add;  // V IMF_y, -V IMF_x
  unsigned long long seed_p, seed_v;
  int add_interval;
  int sz_dst;             // offset of the run's sine tables (Nx then Nz)
  long long roff;         // offset of the run's Poisson buffers (nx * nz)
  // tiled layout: group (i, b) holds cells (i, 2 + 32 b + lane); the run's
  // groups are [gbase, gbase + ngroups), nx rows of nzb = ceil(nz / 32)
  int nzb, gbase, ngroups;
};

struct Pools {
  int* cell[2];
  void* o[2][2];  // [species][axis x, z]
  void* v[2][3];
};

template <typename real>
struct PView {
  int* cell;
  real* ox;
  real* oz;
  real* vx;
  real* vy;
  real* vz;
};

template <typename real>
__device__ __forceinline__ PView<real> pview(const Pools& P, int s) {
  PView<real> v;
  v.cell = P.cell[s];
  v.ox = (real*)P.o[s][0];
  v.oz = (real*)P.o[s][1];
  v.vx = (real*)P.v[s][0];
  v.vy = (real*)P.v[s][1];
  v.vz = (real*)P.v[s][2];
  return v;
}

// Mutable per-run device state.
struct State {
  int count[2];
  int live[2];
  unsigned long long ctr_p, ctr_v;  // random-stream draw counters
  double thrust[3];                 // Fx, Fz, My of the last pic2d_thrust
};

// ------------------------------------------------------------ helpers
__device__ __forceinline__ double ramp2(int idx, int n, int absorb) {
  if (idx - 4 <= 2 * absorb) return (2 * absorb - (idx - 4)) / 4.;
  if (idx - 4 >= 2 * n - 2 * absorb) return ((idx - 4) - (2 * n - 2 * absorb)) / 4.;
  return 0.;
}

// init_grid's damping profile (:252-276) on the doubled grid; zero, without
// the powers, away from the damping layers (most nodes). The 4th and 12th
// powers are taken as products: x and z are quarters of small integers, so
// x^4 is exact and x^12 within a rounding of pow's value, and the field
// updates, which evaluate this at every damping-layer node of every step,
// spend a few multiplies where pow spent a library call per term.
__device__ __forceinline__ double sigma2(double a, int kk, int mm, int nx, int nz, int absorb) {
  const double x = ramp2(kk, nx, absorb), z = ramp2(mm, nz, absorb);
  if (x == 0. && z == 0.) return 0.;
  const double x2 = x * x, z2 = z * z, x4 = x2 * x2, z4 = z2 * z2;
  return a * (0.1 * sqrt(x4 + z4) + 0.01 * sqrt(x4 * x4 * x4 + z4 * z4 * z4));
}

template <typename real>
__device__ __forceinline__ real* plane(real* F, const Run<real>& R, int p) {
  return F + R.foff + (long long)p * R.nodes;
}

// Work item lists: run index and a first row/slot per item.
struct Item {
  int run;
  int first;
};

// ------------------------------------------------------------ grid
// Rows of one item of the field updates: a block of 256 threads takes
// kFieldRows rows of a run, so that a thread updates several nodes per item.
constexpr int kFieldRows = 4;

// The nodes (k, m) of one item, k0 <= k < k0 + kFieldRows (and < nx + 2), 2 <=
// m < nz + 2, flattened over the block's threads and walked without a
// division per node.
struct NodeWalk {
  int k, m, dk, dm;
  __device__ NodeWalk(int k0, int nz, int first, int stride)
      : k(k0 + first / nz), m(2 + first % nz), dk(stride / nz), dm(stride % nz) {}
  __device__ void next(int nz) {
    k += dk;
    m += dm;
    if (m >= nz + 2) {
      m -= nz;
      ++k;
    }
  }
};

// Whether cells 2 idx and 2 idx + 1 of the doubled grid lie outside the
// damping layers of an axis of n cells (ramp2 zero for both).
__device__ __forceinline__ bool undamped(int idx, int n, int absorb) {
  return 2 * idx - 4 > 2 * absorb && 2 * idx + 1 - 4 < 2 * n - 2 * absorb;
}

// The 4th-order difference (27 (f[0] - f[-1]) - (f[1] - f[-2])) / 24 / dx with
// the run's 1 / (24 dx), in the field's precision; d is the stride.
template <typename real>
__device__ __forceinline__ real d4(const real* f, int n, int d, real inv24dx) {
  return ((real)27 * (f[n] - f[n - d]) - (f[n + d] - f[n - 2 * d])) * inv24dx;
}

// renew_b4 (:1391-1417) on the interior of every run; item = (run, first row
// k0) for rows k0 .. k0 + kFieldRows - 1, in the field's precision. Away from
// the damping layers s = 0, where the two factors are exactly 1 and dt / 2
// and are taken without their divisions.
template <typename real>
__global__ void __launch_bounds__(256) renew_b4_kernel(real* F, const Run<real>* __restrict__ runs,
                                                       const Item* __restrict__ items, int nitems) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const Run<real>& R = runs[items[it].run];
    const int k0 = items[it].first;
    const int nx = R.nx, nz = R.nz, G = R.gz, a1 = R.a1;
    const double sa = R.sigma_a;
    const real inv24dx = (real)(1. / (24. * R.dx));
    const real* ex = plane(F, R, P_EX);
    const real* ey = plane(F, R, P_EY);
    const real* ez = plane(F, R, P_EZ);
    real* bx = plane(F, R, P_BX);
    real* by = plane(F, R, P_BY);
    real* bz = plane(F, R, P_BZ);
    const real* b0x = plane(F, R, P_B0X);
    const real* b0y = plane(F, R, P_B0Y);
    const real* b0z = plane(F, R, P_B0Z);
    const double t = 1. / R.e0 * R.dt * 0.5 * 0.5;
    const real hdt = (real)(0.5 * R.dt);
    // (1 - s t) / (1 + s t) and dt / 2 / (1 + s t)
    auto ca = [&](double s) { return s == 0. ? (real)1 : (real)((1. - s * t) / (1. + s * t)); };
    auto cb = [&](double s) { return s == 0. ? hdt : (real)(0.5 * R.dt / (1. + s * t)); };
    const int kend = min(k0 + kFieldRows, nx + 2);
    for (NodeWalk w(k0, nz, threadIdx.x, blockDim.x); w.k < kend; w.next(nz)) {
      const int k = w.k, m = w.m;
      const int n = k * G + m;
      const real dex = d4(ex, n, 1, inv24dx), dez = d4(ez, n, G, inv24dx);
      const real deyx = d4(ey, n, 1, inv24dx), deyz = d4(ey, n, G, inv24dx);
      if (undamped(k, nx, a1) && undamped(m, nz, a1)) {  // s = 0 for all three
        bx[n] = b0x[n] + (bx[n] - b0x[n]) + hdt * deyx;
        by[n] = b0y[n] + (by[n] - b0y[n]) - hdt * (dex - dez);
        bz[n] = b0z[n] + (bz[n] - b0z[n]) - hdt * deyz;
        continue;
      }
      double s = sigma2(sa, 2 * k + 1, 2 * m, nx, nz, a1);
      bx[n] = b0x[n] + ca(s) * (bx[n] - b0x[n]) + cb(s) * deyx;
      s = sigma2(sa, 2 * k, 2 * m, nx, nz, a1);
      by[n] = b0y[n] + ca(s) * (by[n] - b0y[n]) - cb(s) * (dex - dez);
      s = sigma2(sa, 2 * k, 2 * m + 1, nx, nz, a1);
      bz[n] = b0z[n] + ca(s) * (bz[n] - b0z[n]) - cb(s) * deyz;
    }
  }
}

// renew_e4 (:1419-1449); items and precision as renew_b4_kernel's; s = 0 as
// there. dB = B - B0 on both sides of each difference.
template <typename real>
__global__ void __launch_bounds__(256) renew_e4_kernel(real* F, const Run<real>* __restrict__ runs,
                                                       const Item* __restrict__ items, int nitems) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const Run<real>& R = runs[items[it].run];
    const int k0 = items[it].first;
    const int nx = R.nx, nz = R.nz, G = R.gz, a1 = R.a1;
    const double sa = R.sigma_a, mu0 = R.mu0;
    const real inv24dx = (real)(1. / (24. * R.dx));
    const real rmu0 = (real)mu0;
    real* ex = plane(F, R, P_EX);
    real* ey = plane(F, R, P_EY);
    real* ez = plane(F, R, P_EZ);
    const real* bx = plane(F, R, P_BX);
    const real* by = plane(F, R, P_BY);
    const real* bz = plane(F, R, P_BZ);
    const real* b0x = plane(F, R, P_B0X);
    const real* b0y = plane(F, R, P_B0Y);
    const real* b0z = plane(F, R, P_B0Z);
    const real* jix = plane(F, R, P_JIX);
    const real* jiy = plane(F, R, P_JIY);
    const real* jiz = plane(F, R, P_JIZ);
    const real* jex = plane(F, R, P_JEX);
    const real* jey = plane(F, R, P_JEY);
    const real* jez = plane(F, R, P_JEZ);
    const double cc = R.c * R.c * R.dt;
    const real rcc = (real)cc;
    // the 4th-order difference of B - B0 at the half-shifted nodes n + d/2
    auto db4 = [&](const real* b, const real* b0, int n, int d) {
      auto v = [&](int o) { return b[n + o] - b0[n + o]; };
      return ((real)27 * (v(d) - v(0)) - (v(2 * d) - v(-d))) * inv24dx;
    };
    // h = mu0 s cc / 2: (1 - h) / (1 + h) and cc / (1 + h)
    auto ca = [&](double s) {
      const double h = 0.5 * mu0 * s * cc;
      return s == 0. ? (real)1 : (real)((1. - h) / (1. + h));
    };
    auto cb = [&](double s) { return s == 0. ? rcc : (real)(cc / (1. + 0.5 * mu0 * s * cc)); };
    const int kend = min(k0 + kFieldRows, nx + 2);
    for (NodeWalk w(k0, nz, threadIdx.x, blockDim.x); w.k < kend; w.next(nz)) {
      const int k = w.k, m = w.m;
      const int n = k * G + m;
      const real tx = -db4(by, b0y, n, 1) - rmu0 * (jix[n] - jex[n]);
      const real tz = db4(by, b0y, n, G) - rmu0 * (jiz[n] - jez[n]);
      const real ty = db4(bx, b0x, n, 1) - db4(bz, b0z, n, G) - rmu0 * (jiy[n] - jey[n]);
      if (undamped(k, nx, a1) && undamped(m, nz, a1)) {  // s = 0 for all three
        ex[n] = ex[n] + rcc * tx;
        ez[n] = ez[n] + rcc * tz;
        ey[n] = ey[n] + rcc * ty;
        continue;
      }
      double s = sigma2(sa, 2 * k, 2 * m + 1, nx, nz, a1);
      ex[n] = ca(s) * ex[n] + cb(s) * tx;
      s = sigma2(sa, 2 * k + 1, 2 * m, nx, nz, a1);
      ez[n] = ca(s) * ez[n] + cb(s) * tz;
      s = sigma2(sa, 2 * k + 1, 2 * m + 1, nx, nz, a1);
      ey[n] = ca(s) * ey[n] + cb(s) * ty;
    }
  }
}

// sr_grid at size 1 (:1021-1071): columns 0,1 <- N, N+1 and N+2, N+3 <- 2, 3
// of every plane (the whole Grid record); one block per run.
template <typename real>
__global__ void sr_grid_kernel(real* F, const Run<real>* __restrict__ runs, int nruns) {
  for (int r = blockIdx.x; r < nruns; r += gridDim.x) {
    const Run<real> R = runs[r];
    const int G = R.gz, N = R.nx;
    for (int q = threadIdx.x; q < P_COUNT * G; q += blockDim.x) {
      real* a = plane(F, R, q / G);
      const int m = q % G;
      const real v0 = a[N * G + m], v1 = a[(N + 1) * G + m], v2 = a[2 * G + m], v3 = a[3 * G + m];
      a[m] = v0;
      a[G + m] = v1;
      a[(N + 2) * G + m] = v2;
      a[(N + 3) * G + m] = v3;
    }
  }
}

// sr_current / sr_density at size 1 (:1073-1209): column 2 += column N+2,
// column N+1 += column 1, for planes [p0, p0 + np).
template <typename real>
__global__ void fold_kernel(real* F, const Run<real>* __restrict__ runs, int nruns, int p0, int np) {
  for (int r = blockIdx.x; r < nruns; r += gridDim.x) {
    const Run<real> R = runs[r];
    const int G = R.gz, N = R.nx;
    for (int q = threadIdx.x; q < np * G; q += blockDim.x) {
      real* a = plane(F, R, p0 + q / G);
      const int m = q % G;
      a[2 * G + m] += a[(N + 2) * G + m];
      a[(N + 1) * G + m] += a[G + m];
    }
  }
}

// external_current_perp (:2238-2268) at rank p/2 = 0: the coil's two line
// currents, ramped up over the first 10000 steps.
template <typename real>
__global__ void coil_kernel(real* F, const Run<real>* __restrict__ runs, int nruns, const int* __restrict__ step) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nruns) return;
  const Run<real> R = runs[r];
  const int c = *step;
  const double Pi = 3.14159265358979323846;
  const double w = Pi / 10000.;
  real* jiy = plane(F, R, P_JIY);
  const int G = R.gz;
  const int lo = 3 * G + (R.nz + 4) / 2 - 3, hi = 3 * G + (R.nz + 4) / 2 + 2;
  if (c < 10000) {
    jiy[lo] = (real)(-R.coil_i / R.dx / R.dx * (1. + cos(w * c - Pi)) / 2.);
    jiy[hi] = (real)(R.coil_i / R.dx / R.dx * (1. + cos(w * c - Pi)) / 2.);
  } else {
    jiy[lo] = (real)(-R.coil_i / R.dx / R.dx);
    jiy[hi] = (real)(R.coil_i / R.dx / R.dx);
  }
}

// renew_grid (:1348-1389): J, n and phi of every run to zero (the last nine
// planes of each run's block); one block per run.
template <typename real>
__global__ void zero_sources_kernel(real* F, const Run<real>* __restrict__ runs, int nruns) {
  for (int r = blockIdx.x; r < nruns; r += gridDim.x) {
    const Run<real> R = runs[r];
    real* base = F + R.foff + (long long)P_JIX * R.nodes;
    const long long n = (long long)(P_COUNT - P_JIX) * R.nodes;
    for (long long q = threadIdx.x; q < n; q += blockDim.x) base[q] = (real)0;
  }
}

__global__ void step_advance_kernel(int* step) { *step += 1; }

// ------------------------------------------------------------ particles
// Bilinear weights of one axis in cell units (shape_func_*3, :1948-2016):
// node-aligned base i with (1 - f, f); half-shifted base (int)(x - 0.5).
template <typename real>
struct Ax2 {
  int a, b;
  real a0, a1, b0, b1;
};

template <typename real>
__device__ __forceinline__ Ax2<real> ax2(int i, real f) {
  Ax2<real> w;
  w.a = i;
  w.a1 = f;
  w.a0 = (real)1 - f;
  const bool up = f >= (real)0.5 || i == 0;
  w.b = up ? i : i - 1;
  w.b1 = up ? f - (real)0.5 : f + (real)0.5;
  w.b0 = (real)1 - w.b1;
  return w;
}

template <typename real>
__device__ __forceinline__ real bil(const real* P, int G, int i, int k, real x0, real x1, real z0, real z1) {
  return (P[i * G + k] * (x0 * z0) + P[(i + 1) * G + k] * (x1 * z0)) +
         (P[i * G + k + 1] * (x0 * z1) + P[(i + 1) * G + k + 1] * (x1 * z1));
}

// E and B at a particle from a window of one plane per component (ex ey ez
// bx by bz, WN nodes each, z rows of WZ nodes; window coordinates of the
// stencil bases): bil's arithmetic in FP64. In FP32 the two x nodes of each
// stencil row travel as one packed pair through two-wide multiplies and FMAs
// (0.2 ms per step off the 256-run batch against bil's scalar form).
template <typename real>
struct EB2 {
  real ex, ey, ez, bx, by, bz;
};
template <int WZ, int WN>
__device__ __forceinline__ EB2<double> gather_win2(const double* fw, int xa, int xb, int za, int zb,
                                                   const Ax2<double>& X, const Ax2<double>& Z) {
  EB2<double> r;
  r.ex = bil(fw + 0 * WN, WZ, xa, zb, X.a0, X.a1, Z.b0, Z.b1);
  r.ey = bil(fw + 1 * WN, WZ, xb, zb, X.b0, X.b1, Z.b0, Z.b1);
  r.ez = bil(fw + 2 * WN, WZ, xb, za, X.b0, X.b1, Z.a0, Z.a1);
  r.bx = bil(fw + 3 * WN, WZ, xb, za, X.b0, X.b1, Z.a0, Z.a1);
  r.by = bil(fw + 4 * WN, WZ, xa, za, X.a0, X.a1, Z.a0, Z.a1);
  r.bz = bil(fw + 5 * WN, WZ, xa, zb, X.a0, X.a1, Z.b0, Z.b1);
  return r;
}
template <int WZ>
__device__ __forceinline__ float bil_pair(const float* P, int i, int k, float x0, float x1, float2 Z0, float2 Z1) {
  const float2 n0 = make_float2(P[i * WZ + k], P[(i + 1) * WZ + k]);
  const float2 n1 = make_float2(P[i * WZ + k + 1], P[(i + 1) * WZ + k + 1]);
  const float2 cz = __ffma2_rn(n1, Z1, __fmul2_rn(n0, Z0));
  return cz.x * x0 + cz.y * x1;
}
template <int WZ, int WN>
__device__ __forceinline__ EB2<float> gather_win2(const float* fw, int xa, int xb, int za, int zb,
                                                  const Ax2<float>& X, const Ax2<float>& Z) {
  const float2 za0 = make_float2(Z.a0, Z.a0), za1 = make_float2(Z.a1, Z.a1);
  const float2 zb0 = make_float2(Z.b0, Z.b0), zb1 = make_float2(Z.b1, Z.b1);
  EB2<float> r;
  r.ex = bil_pair<WZ>(fw + 0 * WN, xa, zb, X.a0, X.a1, zb0, zb1);
  r.ey = bil_pair<WZ>(fw + 1 * WN, xb, zb, X.b0, X.b1, zb0, zb1);
  r.ez = bil_pair<WZ>(fw + 2 * WN, xb, za, X.b0, X.b1, za0, za1);
  r.bx = bil_pair<WZ>(fw + 3 * WN, xb, za, X.b0, X.b1, za0, za1);
  r.by = bil_pair<WZ>(fw + 4 * WN, xa, za, X.a0, X.a1, za0, za1);
  r.bz = bil_pair<WZ>(fw + 5 * WN, xa, zb, X.a0, X.a1, zb0, zb1);
  return r;
}

template <typename real>
__device__ __forceinline__ void dep4(real* P, int G, int i, int k, real v, real x0, real x1, real z0, real z1) {
  atomicAdd(P + i * G + k, v * (x0 * z0));
  atomicAdd(P + (i + 1) * G + k, v * (x1 * z0));
  atomicAdd(P + i * G + k + 1, v * (x0 * z1));
  atomicAdd(P + (i + 1) * G + k + 1, v * (x1 * z1));
}

// cal_track_c4 (:1520-1560) on (vx, vy, vz) with T = q dt / 2m; FP32
// divides with __fdividef.
template <typename real>
__device__ __forceinline__ void rotate_c4(real T, real ex, real ey, real ez, real bx, real by, real bz, real& vx,
                                          real& vy, real& vz) {
  const real den = (real)1 + T * T * (bx * bx + by * by + bz * bz);
  real S;
  if constexpr (sizeof(real) == 4) S = __fdividef(2.f * T, den);
  else S = (real)2 * T / den;
  const real ux = vx + ex * T, uy = vy + ey * T, uz = vz + ez * T;
  const real uox = ux + T * (uy * bz - uz * by);
  const real uoy = uy + T * (uz * bx - ux * bz);
  const real uoz = uz + T * (ux * by - uy * bx);
  vx = ux + S * (uoy * bz - uoz * by) + ex * T;
  vy = uy + S * (uoz * bx - uox * bz) + ey * T;
  vz = uz + S * (uox * by - uoy * bx) + ez * T;
}

// The particle layout the cell sort builds, per run and species: group
// (i, b) holds the particles of cells (i, 2 + 32 b + l), l = 0 .. 31 the lane,
// in gmax rows of 32 slots, slot = poff + goff[G] - goff[gbase] + 32 row + l.
// After the sort every particle sits in its lane's home cell; between sorts a
// particle keeps its slot wherever it moves. Empty slots hold cell -1.
struct Layout2 {
  const int* goff[2];  // per group: exclusive scan of 32 gmax over all groups (+ the total)
  const int* gmax[2];  // per group: rows
};

// Rows of particles each warp of push2d_tiled_kernel fetches ahead with
// cp.async (1: loads at the point of use)
#ifndef PB_RING2D
#define PB_RING2D 3
#endif

__device__ __forceinline__ void cp_async_ca(void* smem, const void* gmem, int bytes) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  if (bytes == 4)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" :: "r"(sa), "l"(gmem) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" :: "r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit2() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait2() { asm volatile("cp.async.wait_group %0;" :: "n"(N) : "memory"); }

// Sums of one lane's home cell (hi, hk) over the nodes its particles deposit
// on: jx on x nodes hi, hi+1 and z nodes hk-1 .. hk+1 (node-aligned x,
// half-shifted z); jy and n on x and z nodes hi-1 .. hi+1, hk-1 .. hk+1; jz on
// x nodes hi-1 .. hi+1 and z nodes hk, hk+1.
template <typename real>
struct Home2 {
  real jx_[2][3], jy_[3][3], jz_[3][2], n_[3][3];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        jy_[a][c] = n_[a][c] = (real)0;
        if (a < 2) jx_[a][c] = (real)0;
        if (c < 2) jz_[a][c] = (real)0;
      }
  }
  // J of one particle with charge weight q, x-aligned weights (xa0, xa1),
  // z-aligned (za0, za1) and half-shifted weights xb, zb over the 3 nodes
  __device__ __forceinline__ void add_j(real q, real vx, real vy, real vz, real xa0, real xa1, real za0, real za1,
                                        const real (&xb)[3], const real (&zb)[3]) {
    const real px0 = q * vx * xa0, px1 = q * vx * xa1;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      jx_[0][c] += px0 * zb[c];
      jx_[1][c] += px1 * zb[c];
    }
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const real py = q * vy * xb[b], pz = q * vz * xb[b];
#pragma unroll
      for (int c = 0; c < 3; ++c) jy_[b][c] += py * zb[c];
      jz_[b][0] += pz * za0;
      jz_[b][1] += pz * za1;
    }
  }
  __device__ __forceinline__ void add_n(real w, const real (&xb)[3], const real (&zb)[3]) {
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const real pn = w * xb[b];
#pragma unroll
      for (int c = 0; c < 3; ++c) n_[b][c] += pn * zb[c];
    }
  }
  __device__ __forceinline__ real jx(int a, int c) const { return jx_[a][c]; }
  __device__ __forceinline__ real jy(int b, int c) const { return jy_[b][c]; }
  __device__ __forceinline__ real jz(int b, int c) const { return jz_[b][c]; }
  __device__ __forceinline__ real n(int b, int c) const { return n_[b][c]; }
};

// FP32: pairs of sums updated with the two-wide multiplies and FMAs of sm_100
// (jx over its two x nodes, jz over its two z nodes, jy and n over the first
// two x nodes beside a scalar third).
template <>
struct Home2<float> {
  float2 jx_[3], jy01_[3], jz_[3], n01_[3];  // jx_[c] = (a 0, a 1); jy01_[c] = (b 0, b 1); jz_[b] = (c 0, c 1)
  float jy2_[3], n2_[3];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      jx_[c] = jy01_[c] = jz_[c] = n01_[c] = make_float2(0.f, 0.f);
      jy2_[c] = n2_[c] = 0.f;
    }
  }
  __device__ __forceinline__ void add_j(float q, float vx, float vy, float vz, float xa0, float xa1, float za0,
                                        float za1, const float (&xb)[3], const float (&zb)[3]) {
    const float qx = q * vx, qy = q * vy, qz = q * vz;
    const float2 px = __fmul2_rn(make_float2(qx, qx), make_float2(xa0, xa1));
    const float2 py = __fmul2_rn(make_float2(qy, qy), make_float2(xb[0], xb[1]));
    const float py2 = qy * xb[2];
    const float2 za = make_float2(za0, za1);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float2 zc = make_float2(zb[c], zb[c]);
      jx_[c] = __ffma2_rn(px, zc, jx_[c]);
      jy01_[c] = __ffma2_rn(py, zc, jy01_[c]);
      jy2_[c] = fmaf(py2, zb[c], jy2_[c]);
      const float pz = qz * xb[c];
      jz_[c] = __ffma2_rn(make_float2(pz, pz), za, jz_[c]);
    }
  }
  __device__ __forceinline__ void add_n(float w, const float (&xb)[3], const float (&zb)[3]) {
    const float2 pn = __fmul2_rn(make_float2(w, w), make_float2(xb[0], xb[1]));
    const float pn2 = w * xb[2];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      n01_[c] = __ffma2_rn(pn, make_float2(zb[c], zb[c]), n01_[c]);
      n2_[c] = fmaf(pn2, zb[c], n2_[c]);
    }
  }
  __device__ __forceinline__ float jx(int a, int c) const { return a ? jx_[c].y : jx_[c].x; }
  __device__ __forceinline__ float jy(int b, int c) const { return b == 2 ? jy2_[c] : b ? jy01_[c].y : jy01_[c].x; }
  __device__ __forceinline__ float jz(int b, int c) const { return c ? jz_[b].y : jz_[b].x; }
  __device__ __forceinline__ float n(int b, int c) const { return b == 2 ? n2_[c] : b ? n01_[c].y : n01_[c].x; }
};

// The half-shifted weights (b0, b1) of a particle of home cell h over the
// three nodes h-1 .. h+1 (its base is h-1 or h).
template <typename real>
__device__ __forceinline__ void spread3(const Ax2<real>& A, int h, real (&w)[3]) {
  const bool lo = A.b < h;
  w[0] = lo ? A.b0 : (real)0;
  w[1] = lo ? A.b1 : A.b0;
  w[2] = lo ? (real)0 : A.b1;
}
// FP32: the same three weights straight from the offset f of a particle in
// its home cell (an interior cell, so never cell 0): with g = f - 1/2 they are
// (max(-g, 0), 1 - |g|, max(g, 0)), equal to spread3's to within a rounding.
template <typename real>
__device__ __forceinline__ void home_w3(int i, real f, int h, real (&w)[3]) {
  if constexpr (sizeof(real) == 4) {
    const float g = f - 0.5f;
    w[0] = fmaxf(-g, 0.f);
    w[1] = 1.f - fabsf(g);
    w[2] = fmaxf(g, 0.f);
  } else {
    spread3(ax2(i, f), h, w);
  }
}

// The particle part of one step for every run and species (the push loop,
// the drift loop and the x exchange + removal in one pass) over the tiled
// layout. item = (run * 2 + species, tile): a tile is TX x 32 cells (TX rows
// of groups), one warp per group. The block stages the tile's E and B over a
// window of two nodes around it in shared memory; a particle whose stencil
// leaves the window (it moved more than a cell since the sort) gathers from
// the planes. J (at x^{n+1/2}) and n (at x^{n+1}) of a particle in its lane's
// home cell are summed in the lane's registers (Home2) and added to the planes
// once per group; a particle elsewhere adds its terms to the planes directly.
// 512 resident threads per SM in FP32 (128 registers: the 30 home sums and
// the particle in flight fit without spills), 256 in FP64.
template <typename real, int TX>
__global__ void __launch_bounds__(TX * 32, (sizeof(real) == 4 ? 512 : 256) / (TX * 32))
    push2d_tiled_kernel(Pools pools, real* F, const Run<real>* __restrict__ runs, Layout2 L,
                        const Item* __restrict__ items, int nitems, unsigned long long* err) {
  constexpr int WX = TX + 4, WZ = 36, WN = WX * WZ;
  // static shared memory: two stages in FP64 and with eight-row tiles
  constexpr int kSt = (sizeof(real) == 4 && TX < 8) || PB_RING2D < 2 ? PB_RING2D : 2;
  __shared__ real fw[6 * WN];  // ex ey ez bx by bz
  // per warp and stage: the row's five reals and cells, lane-contiguous
  __shared__ real ring_r[TX][kSt][5][32];
  __shared__ int ring_c[TX][kSt][32];
  // FP32: per warp, queues of the J (7 words: cell, offsets, q n v, a pad for
  // the banks) and n (3 words: cell, offsets) deposits of particles off their
  // lane's home cell, made 32 at a time by the whole warp with global
  // reductions. (A shared deposit window per tile taking these and the home
  // sums by FP32 shared atomics, added to the planes once per tile, measured
  // 0.5 ms per step slower, although these reductions cost the step about 2.4
  // ms.)
  constexpr bool kQueue = sizeof(real) == 4;
  constexpr int kQ = 64;
  __shared__ float jq_s[kQueue ? TX : 1][kQueue ? kQ : 1][7];
  __shared__ float nq_s[kQueue ? TX : 1][kQueue ? kQ : 1][3];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned pushed = 0;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int rs = items[it].run;
    const int r = rs >> 1, s = rs & 1;
    // the run's constants as scalars (a copy of the whole Run, indexed by the
    // species, would live in local memory)
    const Run<real>& RR = runs[r];
    struct {
      int nx, nz, gx, gz, nzb, gbase, a2;
      long long nodes, poff, foff;
    } R{RR.nx, RR.nz, RR.gx, RR.gz, RR.nzb, RR.gbase, RR.a2, RR.nodes, RR.poff, RR.foff};
    const double Ts = s == 0 ? RR.T[0] : RR.T[1];
    const int tile = items[it].first;
    const int i0 = 2 + (tile / R.nzb) * TX, k0 = 2 + 32 * (tile % R.nzb);
    const int wx0 = i0 - 2, wz0 = k0 - 2;  // window origin (node)
    const int G = R.gz;
    real* const F0 = F + R.foff;
    // planes of this species' J (p = 0..2) and n (p = 3)
    auto pj = [&](int p) { return F0 + (long long)(p < 3 ? P_JIX + 3 * s + p : P_NI + s) * R.nodes; };
    __syncthreads();  // the last item's gathers are done
    for (int q = threadIdx.x; q < 6 * WN; q += blockDim.x) {
      const int p = q / WN, a = (q / WZ) % WX, c = q % WZ;
      const int gi = wx0 + a, gk = wz0 + c;
      fw[q] = gi < R.gx && gk < G ? F0[(long long)(P_EX + p) * R.nodes + gi * G + gk] : (real)0;
    }
    __syncthreads();
    const int hi = i0 + warp, hk = k0 + lane;  // this lane's home cell
    if (hi < R.nx + 2) {  // warp-uniform
      const PView<real> P = pview<real>(pools, s);
      const int Gi = R.gbase + (hi - 2) * R.nzb + (tile % R.nzb);
      const long long base = R.poff + L.goff[s][Gi] - L.goff[s][R.gbase] + lane;
      const long long end = R.poff + RR.cap;  // rows of a layout that overflowed the run were not written
      const int m = L.gmax[s][Gi];
      const real T = (real)Ts;
      const real hdt = (real)(0.5 * RR.dt / RR.dx);
      const real qn = (real)(RR.q * RR.nw);
      const real nw = (real)RR.nw;
      const real ex_add = (real)RR.ex_add, ey_add = (real)RR.ey_add;
      const int hz = R.nz + 4 - R.a2, hx = R.nx + 4 - R.a2;
      Home2<real> h;
      h.zero();
      // each lane copies and reads only its own slots, so the per-thread
      // cp.async groups need no warp barrier
      auto fetch = [&](int row) {
        const long long t = base + 32LL * row;
        if (kSt > 1 && row < m && t < end) {
          const int st = row % kSt;
          cp_async_ca(&ring_c[warp][st][lane], P.cell + t, 4);
          cp_async_ca(&ring_r[warp][st][0][lane], P.ox + t, sizeof(real));
          cp_async_ca(&ring_r[warp][st][1][lane], P.oz + t, sizeof(real));
          cp_async_ca(&ring_r[warp][st][2][lane], P.vx + t, sizeof(real));
          cp_async_ca(&ring_r[warp][st][3][lane], P.vy + t, sizeof(real));
          cp_async_ca(&ring_r[warp][st][4][lane], P.vz + t, sizeof(real));
        }
        if (kSt > 1) cp_async_commit2();
      };
#pragma unroll
      for (int q = 0; q < kSt - 1; ++q) fetch(q);
      int njq = 0, nnq = 0;  // queue lengths (warp-uniform)
      auto dep_j = [&](int q) {
        const float* e = jq_s[kQueue ? warp : 0][q];
        int qi, qk;
        unpack2(__float_as_int(e[0]), qi, qk);
        const Ax2<real> X = ax2(qi, (real)e[1]), Z = ax2(qk, (real)e[2]);
        dep4(pj(0), G, X.a, Z.b, (real)e[3], X.a0, X.a1, Z.b0, Z.b1);
        dep4(pj(1), G, X.b, Z.b, (real)e[4], X.b0, X.b1, Z.b0, Z.b1);
        dep4(pj(2), G, X.b, Z.a, (real)e[5], X.b0, X.b1, Z.a0, Z.a1);
      };
      auto dep_n = [&](int q) {
        const float* e = nq_s[kQueue ? warp : 0][q];
        int qi, qk;
        unpack2(__float_as_int(e[0]), qi, qk);
        const Ax2<real> X = ax2(qi, (real)e[1]), Z = ax2(qk, (real)e[2]);
        dep4(pj(3), G, X.b, Z.b, nw, X.b0, X.b1, Z.b0, Z.b1);
      };
      for (int row = 0; row < m; ++row) {
        fetch(row + kSt - 1);
        const long long t = base + 32LL * row;
        int c;
        real fx, fz, vx, vy, vz;
        if (kSt > 1) {
          cp_async_wait2<kSt - 1>();
          const int st = row % kSt;
          c = ring_c[warp][st][lane];
          fx = ring_r[warp][st][0][lane];
          fz = ring_r[warp][st][1][lane];
          vx = ring_r[warp][st][2][lane];
          vy = ring_r[warp][st][3][lane];
          vz = ring_r[warp][st][4][lane];
        } else {
          c = t < end ? P.cell[t] : -1;
          if (c >= 0) {
            fx = P.ox[t]; fz = P.oz[t];
            vx = P.vx[t]; vy = P.vy[t]; vz = P.vz[t];
          }
        }
        if (t >= end) c = -1;  // rows of a layout that overflowed the run were not written
        bool qj = false, qnn = false;  // J / n of this particle go to the warp's queues
        int jc = 0, ncell = 0;
        real jfx = 0, jfz = 0;
        if (c >= 0) {
          ++pushed;
          int i, k;
          unpack2(c, i, k);
          // ballistic margins (:682-686): z < A2, z > Nz+4-A2, x < A2, x > Nx+4-A2 (cells)
          const bool bal = k < R.a2 || i < R.a2 || k > hz || (k == hz && fz > (real)0) || i > hx ||
                           (i == hx && fx > (real)0);
          if (!bal) {
            if (i < 1 || k < 1 || i > R.gx - 2 || k > R.gz - 2) {
              atomicAdd(err + ERR_DEPOSIT_OOB, 1ull);
            } else {
              const Ax2<real> X = ax2(i, fx), Z = ax2(k, fz);
              // ex, bz: x aligned, z shifted; ez, bx: x shifted, z aligned; ey: both shifted; by: both aligned
              real ex, ey, ez, bx, by, bz;
              if (i - 1 >= wx0 && i + 1 < wx0 + WX && k - 1 >= wz0 && k + 1 < wz0 + WZ) {
                const EB2<real> e = gather_win2<WZ, WN>(fw, X.a - wx0, X.b - wx0, Z.a - wz0, Z.b - wz0, X, Z);
                ex = e.ex; ey = e.ey; ez = e.ez; bx = e.bx; by = e.by; bz = e.bz;
              } else {
                ex = bil(F0 + (long long)P_EX * R.nodes, G, X.a, Z.b, X.a0, X.a1, Z.b0, Z.b1);
                ey = bil(F0 + (long long)P_EY * R.nodes, G, X.b, Z.b, X.b0, X.b1, Z.b0, Z.b1);
                ez = bil(F0 + (long long)P_EZ * R.nodes, G, X.b, Z.a, X.b0, X.b1, Z.a0, Z.a1);
                bx = bil(F0 + (long long)P_BX * R.nodes, G, X.b, Z.a, X.b0, X.b1, Z.a0, Z.a1);
                by = bil(F0 + (long long)P_BY * R.nodes, G, X.a, Z.a, X.a0, X.a1, Z.a0, Z.a1);
                bz = bil(F0 + (long long)P_BZ * R.nodes, G, X.a, Z.b, X.a0, X.a1, Z.b0, Z.b1);
              }
              rotate_c4(T, ex + ex_add, ey + ey_add, ez, bx, by, bz, vx, vy, vz);
            }
          }
          advance(i, fx, vx * hdt);
          advance(k, fz, vz * hdt);
          // J deposit at x^{n+1/2} for dx <= x < (Nx+3) dx, 2 dx <= z < (Nz+2) dx
          if (i == hi && k == hk) {
            real xb[3], zb[3];
            home_w3(i, fx, hi, xb);
            home_w3(k, fz, hk, zb);
            h.add_j(qn, vx, vy, vz, (real)1 - fx, fx, (real)1 - fz, fz, xb, zb);
          } else if (i >= 1 && i < R.nx + 3 && k >= 2 && k < R.nz + 2) {
            if constexpr (kQueue) {
              qj = true;
              jc = pack2(i, k);
              jfx = fx;
              jfz = fz;
            } else {
              const Ax2<real> X = ax2(i, fx), Z = ax2(k, fz);
              dep4(pj(0), G, X.a, Z.b, qn * vx, X.a0, X.a1, Z.b0, Z.b1);
              dep4(pj(1), G, X.b, Z.b, qn * vy, X.b0, X.b1, Z.b0, Z.b1);
              dep4(pj(2), G, X.b, Z.a, qn * vz, X.b0, X.b1, Z.a0, Z.a1);
            }
          }
          advance(i, fx, vx * hdt);
          advance(k, fz, vz * hdt);
          // n at x^{n+1}, same range
          if (i == hi && k == hk) {
            real xb[3], zb[3];
            home_w3(i, fx, hi, xb);
            home_w3(k, fz, hk, zb);
            h.add_n(nw, xb, zb);
          } else if (i >= 1 && i < R.nx + 3 && k >= 2 && k < R.nz + 2) {
            if constexpr (kQueue) {
              qnn = true;
              ncell = pack2(i, k);
            } else {
              const Ax2<real> X = ax2(i, fx), Z = ax2(k, fz);
              dep4(pj(3), G, X.b, Z.b, nw, X.b0, X.b1, Z.b0, Z.b1);
            }
          }
          // x exchange at size 1: forward crossers wrap, backward ones are dropped; then removal
          if (i == R.nx + 2 && k >= 2 && k < R.nz + 2) i -= R.nx;
          const bool keep = i >= 2 && i < R.nx + 2 && k >= 2 && k < R.nz + 2;
          P.cell[t] = keep ? pack2(i, k) : -1;
          P.ox[t] = fx; P.oz[t] = fz;
          P.vx[t] = vx; P.vy[t] = vy; P.vz[t] = vz;
        }
        if constexpr (kQueue) {
          // warp-uniform: the row's queued lanes take consecutive entries, and
          // a full warp's worth is deposited by all 32 lanes at once
          const unsigned below = (1u << lane) - 1u;
          const unsigned mj = __ballot_sync(0xffffffffu, qj), mn = __ballot_sync(0xffffffffu, qnn);
          if (qj) {
            float* e = jq_s[warp][njq + __popc(mj & below)];
            e[0] = __int_as_float(jc);
            e[1] = (float)jfx; e[2] = (float)jfz;
            e[3] = (float)(qn * vx); e[4] = (float)(qn * vy); e[5] = (float)(qn * vz);
          }
          if (qnn) {
            float* e = nq_s[warp][nnq + __popc(mn & below)];
            e[0] = __int_as_float(ncell);
            e[1] = (float)fx; e[2] = (float)fz;
          }
          njq += __popc(mj);
          nnq += __popc(mn);
          if (njq >= 32 || nnq >= 32) {
            __syncwarp();
            if (njq >= 32) {
              dep_j(njq - 32 + lane);
              njq -= 32;
            }
            if (nnq >= 32) {
              dep_n(nnq - 32 + lane);
              nnq -= 32;
            }
            __syncwarp();
          }
        }
      }
      if constexpr (kQueue) {
        __syncwarp();
        if (lane < njq) dep_j(lane);
        if (lane < nnq) dep_n(lane);
      }
      if (kSt > 1) cp_async_wait2<0>();  // the next item refills the ring
      // the home sums into the planes (home cells are interior, so every
      // node lies in the array); untouched nodes are skipped
      if (hk < R.nz + 2) {
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int cc = 0; cc < 3; ++cc) {
            const int node = (hi - 1 + a) * G + (hk - 1 + cc);
            if (a < 2 && h.jx(a, cc) != (real)0) atomicAdd(pj(0) + node + G, h.jx(a, cc));
            if (h.jy(a, cc) != (real)0) atomicAdd(pj(1) + node, h.jy(a, cc));
            if (cc < 2 && h.jz(a, cc) != (real)0) atomicAdd(pj(2) + node + 1, h.jz(a, cc));
            if (h.n(a, cc) != (real)0) atomicAdd(pj(3) + node, h.n(a, cc));
          }
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) pushed += __shfl_down_sync(0xffffffffu, pushed, o);
  if (lane == 0 && pushed) atomicAdd(err + CNT_PUSHED, (unsigned long long)pushed);
}

// Density deposit of every particle (fdtd's set-up, :583-607).
template <typename real>
__global__ void density2d_kernel(Pools pools, real* F, const Run<real>* __restrict__ runs, const State* __restrict__ st,
                                 const Item* __restrict__ items, int nitems, int chunk) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int rs = items[it].run;
    const int r = rs >> 1, s = rs & 1;
    const Run<real> R = runs[r];
    const int n = st[r].count[s];
    const int first = items[it].first;
    if (first >= n) continue;
    const int last = min(first + chunk, n);
    const PView<real> P = pview<real>(pools, s);
    real* dn = plane(F, R, s == 0 ? P_NI : P_NE);
    for (int q = first + threadIdx.x; q < last; q += blockDim.x) {
      const long long t = R.poff + q;
      const int c = P.cell[t];
      if (c < 0) continue;
      int i, k;
      unpack2(c, i, k);
      if (i >= 1 && i < R.nx + 3 && k >= 2 && k < R.nz + 2) {
        const Ax2<real> X = ax2(i, P.ox[t]), Z = ax2(k, P.oz[t]);
        dep4(dn, R.gz, X.b, Z.b, (real)R.nw, X.b0, X.b1, Z.b0, Z.b1);
      }
    }
  }
}

// ------------------------------------------------------------ sources
// A source block: `count` particles uniform in [x0, x1) x [z0, z1) (absolute
// units), drifting Maxwellian, drawing x, z from the position stream and vx,
// vz (two normals, vy = 0) from the velocity stream, in order.
struct Slab2 {
  double x0, x1, z0, z1;
  long long count;
};

struct SourceSet {
  Slab2 slab[4];
  int nslab;
  long long total;
};

// Particles of species s for every run: slab blocks of run r appended after
// the run's current count; the stream counters advance by 2 and 4 draws per
// particle. item = (run, first particle index of the source set).
template <typename real>
__global__ void source2d_kernel(Pools pools, const Run<real>* __restrict__ runs, State* st, const SourceSet* __restrict__ sets,
                                const Item* __restrict__ items, int nitems, int chunk, int s, unsigned long long* err) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int r = items[it].run;
    const Run<real> R = runs[r];
    const SourceSet S = sets[r];
    const long long first = items[it].first;
    const long long last = min(first + (long long)chunk, S.total);
    const PView<real> P = pview<real>(pools, s);
    const int base = st[r].count[s];
    const unsigned long long bp = st[r].ctr_p, bv = st[r].ctr_v;
    for (long long j = first + threadIdx.x; j < last; j += blockDim.x) {
      if (base + j >= R.cap) {
        atomicAdd(err + ERR_CELL_RANGE, 1ull);
        continue;
      }
      long long rem = j;
      int q = 0;
      while (q < S.nslab - 1 && rem >= S.slab[q].count) rem -= S.slab[q].count, ++q;
      const Slab2& sl = S.slab[q];
      const double x = flat_rn(sl.x0, sl.x1, uniform53(R.seed_p, bp + 2 * j));
      const double z = flat_rn(sl.z0, sl.z1, uniform53(R.seed_p, bp + 2 * j + 1));
      const double vx = R.sig[s] * gauss_bm(R.seed_v, bv + 4 * j);
      const double vz = R.vdrift + R.sig[s] * gauss_bm(R.seed_v, bv + 4 * j + 2);
      const long long t = R.poff + base + j;
      int i, k;
      real fx, fz;
      split_coord(x / R.dx, i, fx);
      split_coord(z / R.dx, k, fz);
      P.cell[t] = pack2(i, k);
      P.ox[t] = fx;
      P.oz[t] = fz;
      P.vx[t] = (real)vx;
      P.vy[t] = (real)0;
      P.vz[t] = (real)vz;
    }
  }
}

// After a source launch: counts and stream counters of every run advance.
template <typename real>
__global__ void source2d_commit_kernel(const Run<real>* __restrict__ runs, State* st, const SourceSet* __restrict__ sets,
                                       int nruns, int s) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nruns) return;
  const long long total = sets[r].total;
  const long long n = min((long long)st[r].count[s] + total, runs[r].cap);
  st[r].count[s] = (int)n;
  st[r].ctr_p += 2ull * total;
  st[r].ctr_v += 4ull * total;
}

// add_ion5 / add_electron5's removal (:3317-3332) at size 1: z < 3 dx,
// z > (Nz+1) dx, x < 3 dx, x > (Nx+1) dx.
template <typename real>
__global__ void delete5_kernel(Pools pools, const Run<real>* __restrict__ runs, const State* __restrict__ st,
                               const Item* __restrict__ items, int nitems, int chunk) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int rs = items[it].run;
    const int r = rs >> 1, s = rs & 1;
    const Run<real> R = runs[r];
    const int n = st[r].count[s];
    const int first = items[it].first;
    if (first >= n) continue;
    const int last = min(first + chunk, n);
    const PView<real> P = pview<real>(pools, s);
    for (int q = first + threadIdx.x; q < last; q += blockDim.x) {
      const long long t = R.poff + q;
      const int c = P.cell[t];
      if (c < 0) continue;
      int i, k;
      unpack2(c, i, k);
      const real fx = P.ox[t], fz = P.oz[t];
      const bool del = k < 3 || k > R.nz + 1 || (k == R.nz + 1 && fz > (real)0) || i < 3 || i > R.nx + 1 ||
                       (i == R.nx + 1 && fx > (real)0);
      if (del) P.cell[t] = -1;
    }
  }
}

// ------------------------------------------------------------ renew_phi
// rho of renew_phi (:2608-2638, the rank-0 branch at size 1): the Gauss-law
// residual on grid rows [Absorb_grid3, Nx+2) x columns [Absorb_grid3,
// Nz+4-Absorb_grid3), zero elsewhere; buffer [nx][nz].
template <typename real>
__global__ void phi_rho_kernel(real* F, const Run<real>* __restrict__ runs, const Item* __restrict__ items, int nitems,
                               real* rho) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const Run<real> R = runs[items[it].run];
    const int kk = items[it].first;  // rho row 0..nx-1 (grid row kk + 2)
    const int k = kk + 2;
    const int G = R.gz;
    const real* ex = plane(F, R, P_EX);
    const real* ez = plane(F, R, P_EZ);
    const real* ni = plane(F, R, P_NI);
    const real* ne = plane(F, R, P_NE);
    real* out = rho + R.roff + (long long)kk * R.nz;
    for (int mm = threadIdx.x; mm < R.nz; mm += blockDim.x) {
      const int m = mm + 2;
      double v = 0.0;
      if (k >= R.a3 && k < R.nx + 2 && m >= R.a3 && m < R.nz + 4 - R.a3) {
        const int n = k * G + m;
        v = -(-R.q * ((double)ni[n] - (double)ne[n]) / R.e0 + ((double)ex[n + G] - (double)ex[n]) / R.dx +
              ((double)ez[n + 1] - (double)ez[n]) / R.dx);
      }
      out[mm] = (real)v;
    }
  }
}

// Batched small GEMM C = alpha * op(A B) over every run (row-major, the run's
// sizes): 64x64 output tiles, 256 threads of 4x4 outputs each (4 consecutive
// rows by 4 consecutive columns, read from the staged tiles as 4-wide vector
// loads), K staged through shared memory 32 at a time, both tiles k-major. mode selects the operands of the four
// sine transforms:
//  0: C[nx][nz] = A[nx][nz] * S_nz        (transform along z)
//  1: C[nx][nz] = S_nx * A[nx][nz], then / eigenvalue  (along x, solve)
//  2: C[nx][nz] = (2/nx) S_nx * A          (inverse along x)
//  3: C[nx][nz] = (2/nz) A * S_nz          (inverse along z)
// S_n[i][j] = sin(pi i j / n); its row and column 0 vanish, so the transforms
// skip the first element as the reference's sinft does (y[1] = 0, :2902).
constexpr int kGemmTile = 64;
__device__ __forceinline__ void ld4(const float* p, float (&v)[4]) {
  const float4 q = *reinterpret_cast<const float4*>(p);
  v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void ld4(const double* p, double (&v)[4]) {
  const double2 q0 = reinterpret_cast<const double2*>(p)[0], q1 = reinterpret_cast<const double2*>(p)[1];
  v[0] = q0.x; v[1] = q0.y; v[2] = q1.x; v[3] = q1.y;
}
template <typename real>
__global__ void __launch_bounds__(256) dst_gemm_kernel(const Run<real>* __restrict__ runs, const Item* __restrict__ items,
                                                       int nitems, const real* __restrict__ A, real* C,
                                                       const real* __restrict__ sines, int mode) {
  constexpr int T = kGemmTile, KT = 32;
  __shared__ __align__(16) real As[KT][T + 4];  // [k][row of C]
  __shared__ __align__(16) real Bs[KT][T + 4];  // [k][col of C]
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;  // 16 x 16; outputs (4 ty + u, 4 tx + v)
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const Run<real>& R = runs[items[it].run];
    const int nx = R.nx, nz = R.nz;
    const int tiles_n = (nz + T - 1) / T;
    const int ti = items[it].first / tiles_n, tj = items[it].first % tiles_n;
    const real* a = A + R.roff;
    real* cmat = C + R.roff;
    const real* Sx = sines + R.sz_dst;
    const real* Sz = sines + R.sz_dst + (long long)nx * nx;
    const bool left = mode == 1 || mode == 2;  // S * A (K = nx) or A * S (K = nz)
    const int K = left ? nx : nz;
    real acc[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[u][v] = 0;
    for (int k0 = 0; k0 < K; k0 += KT) {
      __syncthreads();  // the last tile's reads are done
      // left operand tile [T rows of C][KT of K], right operand tile [KT of K][T cols of C]
      for (int q = threadIdx.x; q < T * KT; q += blockDim.x) {
        // left: a warp takes 4 rows x 8 consecutive k (coalesced reads; its
        // transposed stores fall on 32 different banks)
        const int ch = q >> 5, l = q & 31;
        const int r = 4 * (ch % (T / 4)) + (l >> 3), kc = 8 * (ch / (T / 4)) + (l & 7);
        const int row = ti * T + r, kk = k0 + kc;
        real lv = 0;
        if (left) {
          if (row < nx && kk < nx) lv = Sx[(long long)row * nx + kk];
        } else {
          if (row < nx && kk < nz) lv = a[(long long)row * nz + kk];
        }
        As[kc][r] = lv;
        const int kr = q / T, cc = q % T;  // right: row k0 + kr, column cc
        const int krow = k0 + kr, col = tj * T + cc;
        real rv = 0;
        if (left) {
          if (krow < nx && col < nz) rv = a[(long long)krow * nz + col];
        } else {
          if (krow < nz && col < nz) rv = Sz[(long long)krow * nz + col];
        }
        Bs[kr][cc] = rv;
      }
      __syncthreads();
#pragma unroll 8
      for (int kk = 0; kk < KT; ++kk) {
        real av[4], bv[4];
        ld4(&As[kk][4 * ty], av);
        ld4(&Bs[kk][4 * tx], bv);
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int v = 0; v < 4; ++v) acc[u][v] += av[u] * bv[v];
      }
    }
    const double Pi = 3.14159265358979323846;
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int row = ti * T + 4 * ty + u, col = tj * T + 4 * tx + v;
        if (row >= nx || col >= nz) continue;
        real w = acc[u][v];
        if (mode == 1) {
          // renew_phi's eigenvalue (:2680-2690): row = x wave number, col = z wave number
          const double sz = sin(Pi * (double)col / (double)nz / 2.), sx = sin(Pi * (double)row / (double)nx / 2.);
          const double Aev = -(sz * sz + sx * sx) / ((R.dx / 2.) * (R.dx / 2.));
          w = Aev == 0. ? (real)0 : (real)((double)w / Aev);
        } else if (mode == 2) {
          w = (real)(2. * (double)w / nx);
        } else if (mode == 3) {
          w = (real)(2. * (double)w / nz);
        }
        cmat[(long long)row * nz + col] = w;
      }
  }
}

// renew_phi's correction (:2749-2768): ex += d(phi)/dx (periodic at size 1:
// the left neighbour of row 0 is row Nx-1), ez += d(phi)/dz (zero below
// column 0), phi stored.
template <typename real>
__global__ void phi_apply_kernel(real* F, const Run<real>* __restrict__ runs, const Item* __restrict__ items, int nitems,
                                 const real* __restrict__ rho) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const Run<real> R = runs[items[it].run];
    const int kk = items[it].first;
    const int G = R.gz;
    real* ex = plane(F, R, P_EX);
    real* ez = plane(F, R, P_EZ);
    real* phi = plane(F, R, P_PHI);
    const real* row = rho + R.roff + (long long)kk * R.nz;
    const real* left = rho + R.roff + (long long)(kk == 0 ? R.nx - 1 : kk - 1) * R.nz;
    for (int mm = threadIdx.x; mm < R.nz; mm += blockDim.x) {
      const int n = (kk + 2) * G + mm + 2;
      const double v = row[mm];
      ex[n] = (real)((double)ex[n] + (v - (double)left[mm]) / R.dx);
      phi[n] = (real)v;
      ez[n] = (real)((double)ez[n] + (v - (mm == 0 ? 0.0 : (double)row[mm - 1])) / R.dx);
    }
  }
}

// ------------------------------------------------------------ thrust_F
// thrust_F (:2304-2387) per run, FP64. Where the reference's test
// (x != xf0 && z != zf0) fails it keeps the previous node's terms: for the row
// x == xf0 those of the last node of the row before, elsewhere those of the
// node before in z. One block per run.
__device__ __forceinline__ void coil_terms(double jy, double x, double z, double x0, double z0, double K, double& fx,
                                           double& fz) {
  const double Pi = 3.14159265358979323846;
  const double d = 2. * Pi * ((x - x0) * (x - x0) + (z - z0) * (z - z0));
  fx = K * jy * (x - x0) / d;
  fz = K * jy * (z - z0) / d;
}

template <typename real>
__global__ void thrust2d_kernel(const real* __restrict__ F, const Run<real>* __restrict__ runs, int nruns, State* st) {
  __shared__ double red[3][32];
  for (int r = blockIdx.x; r < nruns; r += gridDim.x) {
    const Run<real> R = runs[r];
    const real* jiy = plane((real*)F, R, P_JIY);
    const real* jey = plane((real*)F, R, P_JEY);
    const int G = R.gz;
    const double dx = R.dx;
    const double xf0 = 1.5 * dx, zf0 = -2.5 * dx, xb0 = 1.5 * dx, zb0 = 2.5 * dx;
    const double K = R.mu0 * R.coil_i * dx * dx;
    auto xs = [&](int k) { return ((double)(k - 2) + 0.5) * dx - dx * 1 * R.nx / 2.; };
    auto zs = [&](int m) { return (double)(m - 2) * dx - (double)(R.nz / 2) * dx + 0.5 * dx; };
    auto terms = [&](int k, int m, double& fx0, double& fz0, double& fx1, double& fz1) {
      const double x = xs(k), z = zs(m);
      const double jy = (double)jiy[k * G + m] - (double)jey[k * G + m];
      coil_terms(jy, x, z, xf0, zf0, -K, fx0, fz0);
      coil_terms(jy, x, z, xb0, zb0, K, fx1, fz1);
    };
    double s[3] = {0, 0, 0};
    const int tot = R.nx * R.nz;
    for (int q = threadIdx.x; q < tot; q += blockDim.x) {
      const int k = 2 + q / R.nz, m = 2 + q % R.nz;
      double fx0, fz0, fx1, fz1, a, b;
      terms(k, m, fx0, fz0, fx1, fz1);
      const double x = xs(k), z = zs(m);
      if (!(x != xf0 && z != zf0)) {
        if (x == xf0) terms(k - 1, R.nz + 1, fx0, fz0, a, b);
        else terms(k, m - 1, fx0, fz0, a, b);
      }
      if (!(x != xb0 && z != zb0)) {
        if (x == xb0) terms(k - 1, R.nz + 1, a, b, fx1, fz1);
        else terms(k, m - 1, a, b, fx1, fz1);
      }
      s[0] += fx0 + fx1;
      s[1] += fz0 + fz1;
      s[2] += (-(zf0 + 0.5 * dx) * fx0 + xf0 * fz0) + (-(zb0 + 0.5 * dx) * fx1 + xb0 * fz1);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int q = 0; q < 3; ++q) {
      double v = s[q];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) red[q][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
      double v = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[threadIdx.x][w];
      st[r].thrust[threadIdx.x] = v;
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------ exports
template <typename real>
__global__ void grid2d_export_kernel(const real* F, Run<real> R, double* rec) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= R.nodes) return;
  // the reference's Grid record order (:104-112)
  const int map[18] = {P_B0X, P_B0Y, P_B0Z, P_BX, P_BY, P_BZ, P_EX, P_EY, P_EZ,
                       P_JIX, P_JIY, P_JIZ, P_JEX, P_JEY, P_JEZ, P_NI, P_NE, P_PHI};
  for (int q = 0; q < 18; ++q) rec[18LL * n + q] = (double)F[R.foff + (long long)map[q] * R.nodes + n];
}

template <typename real>
__global__ void parts2d_export_kernel(Pools pools, Run<real> R, int s, int n, const int* __restrict__ pos, double* rows) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const PView<real> P = pview<real>(pools, s);
  const long long t = R.poff + q;
  const int c = P.cell[t];
  if (c < 0) return;
  int i, k;
  unpack2(c, i, k);
  double* r = rows + 6LL * pos[q];
  r[0] = ((double)i + (double)P.ox[t]) * R.dx;
  r[1] = ((double)k + (double)P.oz[t]) * R.dx;
  r[2] = (double)P.vx[t];
  r[3] = (double)P.vy[t];
  r[4] = (double)P.vz[t];
  r[5] = R.nw;
}

__global__ void flag_kernel(const int* __restrict__ cell, long long off, int n, int* flags) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) flags[q] = cell[off + q] >= 0 ? 1 : 0;
}

}  // namespace p2

// ================================================================ host
using namespace p2;

struct pic2d_batch {
  int prec = 32;
  int device = 0;
  size_t rsize = 4;
  int nruns = 0;
  std::vector<pic2d_config> cfg;
  cudaStream_t stream = nullptr;
  void* runs_dev = nullptr;       // Run<real>[nruns]
  std::vector<char> runs_host;    // same, host copy (bytes)
  State* st = nullptr;            // device State[nruns]
  void* field = nullptr;
  long long field_nodes = 0;
  Pools pool[2]{};                // double-buffered particle pools
  int cur = 0;
  long long pool_slots = 0;
  void* sines = nullptr;
  void* rho = nullptr;
  void* rho2 = nullptr;
  long long rho_len = 0;
  // work lists
  Item* row_items = nullptr;   int n_row = 0;    // (run, first of kFieldRows interior rows)
  Item* rho_items = nullptr;   int n_rhorow = 0; // (run, rho row 0..nx-1)
  Item* part_items = nullptr;  int n_part = 0;   // (run*2+s, first slot) over [0, cap)
  Item* tile_items = nullptr;  int n_tile = 0;   // (run, 64x64 tile of nx x nz)
  Item* src_items[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [init/add][species]
  int n_src[2][2] = {{0, 0}, {0, 0}};
  SourceSet* sets[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  int* perm = nullptr;   // cell sort: the source slot of every destination slot (pool_slots)
  int* scan_tmp = nullptr;
  size_t scan_len = 0;
  int* ccnt = nullptr;   // cell sort: particles per cell and cursors (rho_len each)
  int* ccur = nullptr;
  int* gfree = nullptr;  // cell sort: per group and lane, its first free slot number (32 ngroups)
  int* gover = nullptr;  // cell sort: per group, the particles placed in other lanes' free slots
  int* hcnt = nullptr;   // cell sort: per cell, the particles that stayed in it (rho_len)
  // tiled layout (Layout2): groups of every run, their run, rows and offsets
  int ngroups = 0;
  int* grun = nullptr;
  int* gsz = nullptr;                   // ngroups + 1 (the last stays 0)
  // the layout of each pool, per species: goff (ngroups + 1) and gmax
  int* goff[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  int* gmax[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  bool laid = false;                    // the current pool holds a layout (a sort has run since init)
  Item* ptile_items = nullptr; int n_ptile = 0;  // (run*2+s, tile) of the push
  int tile_x = 4;                       // group rows per push tile (tuned)
  int* step_dev = nullptr;
  unsigned long long* err = nullptr;
  int c_add = 0;
  long long step = 0;
  bool ready = false;
  // launch configuration (tuned)
  int push_block = 256;
  int push_blocks = 148 * 8;
  // graphs
  bool use_graph = true;
  // one graph per kind of step (plain, sort, refill) and starting pool; a
  // sort or refill step ends on the other pool (graph_cur)
  cudaGraphExec_t graph[3][2] = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};
  long long graph_launches[3][2] = {{0, 0}, {0, 0}, {0, 0}};  // kernels in each graph
  int graph_cur[3][2] = {{0, 0}, {0, 0}, {0, 0}};
  long long launches = 0;
};

namespace {

#define CK2(x)                                                                   \
  do {                                                                           \
    cudaError_t e_ = (x);                                                        \
    if (e_ != cudaSuccess) {                                                     \
      fprintf(stderr, "plasma_b200 (2d): %s: %s\n", #x, cudaGetErrorString(e_)); \
      return PIC_ERR_CUDA;                                                       \
    }                                                                            \
  } while (0)
#define CKL2()                \
  do {                        \
    ++b->launches;            \
    CK2(cudaGetLastError());  \
  } while (0)
#define CKR2(x)                  \
  do {                           \
    int r_ = (x);                \
    if (r_ != PIC_OK) return r_; \
  } while (0)


int persistent(long long items, int per_sm = 8) {
  long long b = std::min<long long>(items, 148LL * per_sm);
  return (int)std::max<long long>(b, 1);
}

template <typename real>
const Run<real>* runs_of(pic2d_batch* b) { return (const Run<real>*)b->runs_dev; }
template <typename real>
Run<real>* runs_host(pic2d_batch* b) { return (Run<real>*)b->runs_host.data(); }

// The source sets of every run: the initial load (init_particle :389-525) or
// the refill of add_ion5 / add_electron5 (:3311-3566) at size 1.
template <typename real>
void make_sets(pic2d_batch* b, int which, std::vector<SourceSet>& sets) {
  sets.assign(b->nruns, SourceSet{});
  for (int r = 0; r < b->nruns; ++r) {
    const pic2d_config& k = b->cfg[r];
    const double dx = k.dx;
    const long long Np = k.np, Nx = k.nx, Nz = k.nz;
    SourceSet& S = sets[r];
    if (which == 0) {
      // N * Step_p / THREAD_N + 1 particles uniform over the interior
      S.slab[0] = {2. * dx, 2. * dx + Nx * dx, 2. * dx, 2. * dx + Nz * dx, Np * Nx * Np * Nz + 1};
      S.nslab = 1;
    } else {
      S.slab[0] = {2 * dx, (Nx + 2) * dx, 2 * dx, 3 * dx, Np * Nx * Np};
      S.slab[1] = {2 * dx, (Nx + 2) * dx, (Nz + 1) * dx, (Nz + 2) * dx, Np * Nx * Np};
      S.slab[2] = {2 * dx, 3 * dx, 3 * dx, (Nz + 1) * dx, (Np * Nz - 2) * Np};
      S.slab[3] = {(Nx + 1) * dx, (Nx + 2) * dx, 3 * dx, (Nz + 1) * dx, (Np * Nz - 2) * Np};
      S.nslab = 4;
    }
    S.total = 0;
    for (int q = 0; q < S.nslab; ++q) S.total += S.slab[q].count;
  }
}

template <typename real>
int run_sources(pic2d_batch* b, int which) {
  for (int s = 0; s < 2; ++s) {
    if (b->n_src[which][s] > 0) {
      source2d_kernel<real><<<persistent(b->n_src[which][s]), 256, 0, b->stream>>>(
          b->pool[b->cur], runs_of<real>(b), b->st, b->sets[which][s], b->src_items[which][s], b->n_src[which][s], kChunk, s,
          b->err);
      CKL2();
    }
    source2d_commit_kernel<real><<<(b->nruns + 127) / 128, 128, 0, b->stream>>>(runs_of<real>(b), b->st, b->sets[which][s],
                                                                                b->nruns, s);
    CKL2();
  }
  return PIC_OK;
}

int scan_excl(pic2d_batch* b, const int* in, int* out, long long n, int* tmp, size_t tmp_len) {
  const long long tiles = (n + kScanTile - 1) / kScanTile;
  if ((size_t)tiles + 1 > tmp_len) return PIC_ERR_STATE;
  scan_tile_kernel<<<(unsigned)tiles, kScanThreads, 0, b->stream>>>(in, out, tmp, n);
  CKL2();
  if (tiles > 1) {
    CKR2(scan_excl(b, tmp, tmp, tiles, tmp + tiles + 1, tmp_len - (size_t)tiles - 1));
    scan_add_kernel<<<(unsigned)tiles, 256, 0, b->stream>>>(out, tmp, n);
    CKL2();
  }
  return PIC_OK;
}

// ---------------------------------------------------------- cell sort
// The reference draws its particles uniformly over each source slab, so their
// order in the lists says nothing about where they are. A counting sort of
// every run's particles by cell into the tiled layout of the other pool
// (Layout2; empty and deleted slots dropped) puts the particles of one cell in
// one lane's column, so that push2d_tiled_kernel's warps read whole rows and
// their lanes deposit on different nodes. Keys index the run's interior cells
// from R.roff (the nx * nz layout of its Poisson buffer).
__device__ __forceinline__ int warp_add_count(int* counter, int key, bool active) {
  const int lane = threadIdx.x & 31;
  const unsigned peers = __match_any_sync(0xffffffffu, active ? key : -1 - lane);
  const int leader = __ffs(peers) - 1;
  int old = 0;
  if (active && lane == leader) old = atomicAdd(counter + key, __popc(peers));
  old = __shfl_sync(0xffffffffu, old, leader);
  return old + __popc(peers & ((1u << lane) - 1u));
}

template <typename real>
__device__ __forceinline__ int sort_key(const Run<real>& R, int c) {
  if (c < 0) return -1;
  int i, k;
  unpack2(c, i, k);
  i -= 2;
  k -= 2;
  if (i < 0 || k < 0 || i >= R.nx || k >= R.nz) return -1;
  return (int)R.roff + i * R.nz + k;
}

// Particles per cell of species s (every lane of a block walks its chunk in rows).
template <typename real>
__global__ void cellcount2d_kernel(Pools pools, const Run<real>* __restrict__ runs, const State* __restrict__ st,
                                   const Item* __restrict__ items, int nitems, int chunk, int s, int* cnt) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int rs = items[it].run;
    if ((rs & 1) != s) continue;
    const Run<real> R = runs[rs >> 1];
    const int n = st[rs >> 1].count[s];
    const int first = items[it].first;
    const int last = min(first + chunk, n);
    const int* cell = pools.cell[s];
    for (int qb = first; qb < last; qb += blockDim.x) {  // block-uniform
      const int q = qb + threadIdx.x;
      const int key = q < last ? sort_key(R, cell[R.poff + q]) : -1;
      warp_add_count(cnt, key < 0 ? 0 : key, key >= 0);
    }
  }
}

// Rows of every group (one warp per group): the mean count of its cells,
// rounded up (at most its fullest cell's count); gsz = 32 rows, scanned into
// the groups' offsets. A row runs as long as its fullest lane's column, so
// rows sized for the fullest cell of 32 left 30-40 % of the lanes idle at
// 16-64 particles per cell (the whole 2D step took 19.9 ms against 17.8). The
// particles of a cell past the group's rows take the free slots of the
// group's other lanes (rows past their own cells' counts), so every particle
// stays in its group and its tile's field window; they deposit as particles
// off their lane's home cell do. gfree holds each lane's first free slot
// number (an exclusive scan of the lanes' free rows). The rows cover the mean
// of all 32 lanes, so the free slots hold every such particle. (Rows of the
// mean plus half or one standard deviation of a Poisson count measured 18.4
// and 18.9 ms.)
template <typename real>
__global__ void group_rows2d_kernel(const Run<real>* __restrict__ runs, const int* __restrict__ grun, int ngroups,
                                    const int* __restrict__ cnt, int* gmax, int* gsz, int* gfree) {
  const int G = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (G >= ngroups) return;  // warp-uniform
  const Run<real> R = runs[grun[G]];
  const int q = G - R.gbase;
  const int i = q / R.nzb, k = (q % R.nzb) * 32 + lane;
  const int c = k < R.nz ? cnt[R.roff + i * R.nz + k] : 0;
  int m = c, sum = c, nv = k < R.nz;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    sum += __shfl_xor_sync(0xffffffffu, sum, o);
    nv += __shfl_xor_sync(0xffffffffu, nv, o);
  }
  const int rows = min(m, (sum + max(nv, 1) - 1) / max(nv, 1));
  // free rows of this lane, scanned over the warp
  const int fr = max(rows - c, 0);
  int pre = fr;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, pre, o);
    if (lane >= o) pre += v;
  }
  gfree[32LL * G + lane] = pre - fr;
  if (lane == 0) {
    gmax[G] = rows;
    gsz[G] = 32 * rows;
  }
}

// The destination of the particle of rank `rank` in cell `key`, relative to
// the run's first slot: row `rank` of the cell's lane column in the new
// layout, or, past its group's rows, the next free slot of the group (gover
// counts them; the free slots are numbered lane by lane, gfree). -1 for a
// particle past the run's capacity, which is lost (ERR_STORE_FULL).
template <typename real>
__device__ __forceinline__ long long dest_slot(const Run<real>& R, const int* __restrict__ goff,
                                               const int* __restrict__ gmax, const int* __restrict__ gfree,
                                               const int* __restrict__ cnt, int* gover, int key, int rank,
                                               unsigned long long* err) {
  const int rk = key - (int)R.roff;
  const int i = rk / R.nz, k = rk % R.nz;
  const int Gk = R.gbase + i * R.nzb + (k >> 5);
  const int rows = gmax[Gk];
  const long long base = goff[R.gbase];
  long long rel;
  if (rank < rows) {
    rel = goff[Gk] - base + 32LL * rank + (k & 31);
  } else {
    // the j-th free slot of the group: the last lane whose first free slot
    // number is <= j, at the row after its own cell's particles
    const int j = atomicAdd(gover + Gk, 1);
    const int* f = gfree + 32LL * Gk;
    int l = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1)
      if (f[l + step] <= j) l += step;
    const int kl = (k & ~31) + l;
    const int cl = kl < R.nz ? min(cnt[R.roff + i * R.nz + kl], rows) : 0;
    const int row = cl + (j - f[l]);
    if (row >= rows) {  // the group's free slots are spent (cannot happen: the rows cover the mean)
      atomicAdd(err + ERR_STORE_FULL, 1ull);
      return -1;
    }
    rel = goff[Gk] - base + 32LL * row + l;
  }
  if (rel >= R.cap) {
    atomicAdd(err + ERR_STORE_FULL, 1ull);
    return -1;
  }
  return rel;
}

// Each particle's destination (dest_slot), ranked by per-cell cursors over
// every slot of the pool (the first sort after init). perm[destination] = the
// particle's slot; layout_gather2d_kernel then moves the particles destination
// by destination, so that the stores of its six arrays are whole rows (stores
// of single particles to scattered rows cost the sort about eight times the
// bytes it moves).
template <typename real>
__global__ void cellscatter2d_kernel(Pools src, int* perm, const Run<real>* __restrict__ runs,
                                     const State* __restrict__ st, const Item* __restrict__ items, int nitems,
                                     int chunk, int s, const int* __restrict__ goff, const int* __restrict__ gmax,
                                     const int* __restrict__ gfree, const int* __restrict__ cnt, int* cursor,
                                     int* gover, unsigned long long* err) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int rs = items[it].run;
    if ((rs & 1) != s) continue;
    const Run<real> R = runs[rs >> 1];
    const int n = st[rs >> 1].count[s];
    const int first = items[it].first;
    const int last = min(first + chunk, n);
    const int* cell = src.cell[s];
    for (int qb = first; qb < last; qb += blockDim.x) {  // block-uniform
      const int q = qb + threadIdx.x;
      const long long t = R.poff + q;
      const int c = q < last ? cell[t] : -1;
      const int key = q < last ? sort_key(R, c) : -1;
      const int rank = warp_add_count(cursor, key < 0 ? 0 : key, key >= 0);
      if (key < 0) continue;
      const long long rel = dest_slot(R, goff, gmax, gfree, cnt, gover, key, rank, err);
      if (rel >= 0) perm[R.poff + rel] = (int)t;
    }
  }
}

// The move of the sort, destination by destination over every run's new
// layout: perm[d] is the slot of the particle that goes to slot d, or -1 for
// an empty slot.
template <typename real>
__global__ void layout_gather2d_kernel(Pools src, Pools dst, const Run<real>* __restrict__ runs,
                                       const Item* __restrict__ items, int nitems, int chunk, int s,
                                       const int* __restrict__ goff, const int* __restrict__ perm) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int rs = items[it].run;
    if ((rs & 1) != s) continue;
    const Run<real>& R = runs[rs >> 1];
    const long long lay = min((long long)goff[R.gbase + R.ngroups] - goff[R.gbase], R.cap);
    const int first = items[it].first, last = (int)min((long long)first + chunk, lay);
    const PView<real> A = pview<real>(src, s), B = pview<real>(dst, s);
    for (int q = first + threadIdx.x; q < last; q += blockDim.x) {
      const long long d = R.poff + q;
      const int t = perm[d];
      if (t < 0) {
        B.cell[d] = -1;
        continue;
      }
      B.cell[d] = A.cell[t];
      B.ox[d] = A.ox[t]; B.oz[d] = A.oz[t];
      B.vx[d] = A.vx[t]; B.vy[d] = A.vy[t]; B.vz[d] = A.vz[t];
    }
  }
}

// The empty slots of every group (rows past its lane's count) to -1 in `cell`
// (the sort's destination map).
template <typename real>
__global__ void pad2d_kernel(int* cell, const Run<real>* __restrict__ runs, const int* __restrict__ grun, int ngroups,
                             const int* __restrict__ goff, const int* __restrict__ gmax, const int* __restrict__ cnt) {
  const int G = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (G >= ngroups) return;
  const Run<real> R = runs[grun[G]];
  const int q = G - R.gbase;
  const int i = q / R.nzb, k = (q % R.nzb) * 32 + lane;
  const int have = k < R.nz ? cnt[R.roff + i * R.nz + k] : 0;
  const long long rel0 = (long long)goff[G] - goff[R.gbase] + lane;
  for (int row = have; row < gmax[G]; ++row) {
    const long long rel = rel0 + 32LL * row;
    if (rel < R.cap) cell[R.poff + rel] = -1;
  }
}

// Slots in use of every run after the sort: the end of its last group.
template <typename real>
__global__ void layout_count2d_kernel(const Run<real>* __restrict__ runs, State* st, int nruns, int s,
                                      const int* __restrict__ goff) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nruns) return;
  const Run<real> R = runs[r];
  st[r].count[s] = (int)min((long long)goff[R.gbase + R.ngroups] - goff[R.gbase], R.cap);
}

// The sort of a pool that holds a layout (every sort after the first): one
// warp per group of the old layout, lane l walking its column. The particles
// still in the lane's home cell (stayers) are counted in a register and added
// once, hcnt[cell] = their number; a particle that moved adds itself to its
// new cell. layout_perm_kernel then gives the stayers ranks in their old row
// order from the same per-lane counter, so that the gather of the move reads
// each new row from nearby old rows; the others take ranks after their new
// cell's stayers from its cursor.
template <typename real>
__global__ void layout_count_kernel(Pools pools, const Run<real>* __restrict__ runs, const int* __restrict__ grun,
                                    int ngroups, const int* __restrict__ goff, const int* __restrict__ gmax, int s,
                                    int* cnt, int* hcnt) {
  const int G = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (G >= ngroups) return;  // warp-uniform
  const Run<real>& R = runs[grun[G]];
  const int q = G - R.gbase;
  const int i = q / R.nzb, k = (q % R.nzb) * 32 + lane;
  const bool valid = k < R.nz;
  const int home = valid ? (int)R.roff + i * R.nz + k : -1;
  const long long base = R.poff + goff[G] - goff[R.gbase] + lane, end = R.poff + R.cap;
  const int* cell = pools.cell[s];
  int stay = 0;
  for (int row = 0; row < gmax[G]; ++row) {
    const long long t = base + 32LL * row;
    if (t >= end) break;
    const int key = sort_key(R, cell[t]);
    if (key < 0) continue;
    if (key == home) ++stay;
    else atomicAdd(cnt + key, 1);
  }
  if (valid) {
    hcnt[home] = stay;
    if (stay) atomicAdd(cnt + home, stay);
  }
}

// The destinations of the old layout's particles (see layout_count_kernel),
// four rows in flight per lane.
template <typename real>
__global__ void layout_perm_kernel(Pools pools, const Run<real>* __restrict__ runs, const int* __restrict__ grun,
                                   int ngroups, const int* __restrict__ goff_old, const int* __restrict__ gmax_old,
                                   const int* __restrict__ goff, const int* __restrict__ gmax,
                                   const int* __restrict__ gfree, const int* __restrict__ cnt,
                                   const int* __restrict__ hcnt, int* cursor, int* gover, int s, int* perm,
                                   unsigned long long* err) {
  const int G = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (G >= ngroups) return;  // warp-uniform
  const Run<real>& R = runs[grun[G]];
  const int q = G - R.gbase;
  const int i = q / R.nzb, k = (q % R.nzb) * 32 + lane;
  const int home = k < R.nz ? (int)R.roff + i * R.nz + k : -1;
  const long long base = R.poff + goff_old[G] - goff_old[R.gbase] + lane, end = R.poff + R.cap;
  const int* cell = pools.cell[s];
  constexpr int U = 4;
  const int m = gmax_old[G];
  int stay = 0;
  for (int r0 = 0; r0 < m; r0 += U) {
    int key[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const long long t = base + 32LL * (r0 + u);
      key[u] = r0 + u < m && t < end ? sort_key(R, cell[t]) : -1;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (key[u] < 0) continue;
      const int rank = key[u] == home ? stay++ : hcnt[key[u]] + atomicAdd(cursor + key[u], 1);
      const long long rel = dest_slot(R, goff, gmax, gfree, cnt, gover, key[u], rank, err);
      if (rel >= 0) perm[R.poff + rel] = (int)(base + 32LL * (r0 + u));
    }
  }
}

// The destinations of the slots after the old layout (a refill appended
// there): ranks after their cells' stayers.
template <typename real>
__global__ void tail_perm_kernel(Pools pools, const Run<real>* __restrict__ runs, const State* __restrict__ st,
                                 const Item* __restrict__ items, int nitems, int chunk, int s,
                                 const int* __restrict__ goff_old, const int* __restrict__ goff,
                                 const int* __restrict__ gmax, const int* __restrict__ gfree,
                                 const int* __restrict__ cnt, const int* __restrict__ hcnt, int* cursor, int* gover,
                                 int* perm, unsigned long long* err) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int rs = items[it].run;
    if ((rs & 1) != s) continue;
    const Run<real>& R = runs[rs >> 1];
    const int lay = goff_old[R.gbase + R.ngroups] - goff_old[R.gbase];
    const int first = max(items[it].first, lay), last = min(items[it].first + chunk, st[rs >> 1].count[s]);
    for (int q = first + threadIdx.x; q < last; q += blockDim.x) {
      const long long t = R.poff + q;
      const int key = sort_key(R, pools.cell[s][t]);
      if (key < 0) continue;
      const long long rel =
          dest_slot(R, goff, gmax, gfree, cnt, gover, key, hcnt[key] + atomicAdd(cursor + key, 1), err);
      if (rel >= 0) perm[R.poff + rel] = (int)t;
    }
  }
}

// Pass 1 for the slots after the old layout (a refill appended there).
template <typename real>
__global__ void tail_count_kernel(Pools pools, const Run<real>* __restrict__ runs, const State* __restrict__ st,
                                  const Item* __restrict__ items, int nitems, int chunk, int s,
                                  const int* __restrict__ goff, int* cnt) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int rs = items[it].run;
    if ((rs & 1) != s) continue;
    const Run<real>& R = runs[rs >> 1];
    const int lay = goff[R.gbase + R.ngroups] - goff[R.gbase];  // the old layout's end
    const int first = max(items[it].first, lay), last = min(items[it].first + chunk, st[rs >> 1].count[s]);
    for (int q = first + threadIdx.x; q < last; q += blockDim.x) {
      const int key = sort_key(R, pools.cell[s][R.poff + q]);
      if (key >= 0) atomicAdd(cnt + key, 1);
    }
  }
}

// Every run's particles by cell into the tiled layout of the other pool: the
// counts over every slot (the first sort after init) or by the layout-aware
// passes above, then the ranks by per-cell cursors.
template <typename real>
int cellsort(pic2d_batch* b) {
  const int nb = 1 - b->cur;
  const long long nc = b->rho_len;
  const Run<real>* R = runs_of<real>(b);
  const int gblocks = (int)((32LL * b->ngroups + 255) / 256);
  for (int s = 0; s < 2; ++s) {
    int* goff_old = b->goff[b->cur][s];
    int* gmax_old = b->gmax[b->cur][s];
    int* goff = b->goff[nb][s];
    int* gmax = b->gmax[nb][s];
    CK2(cudaMemsetAsync(b->ccnt, 0, sizeof(int) * (size_t)nc, b->stream));
    CK2(cudaMemsetAsync(b->ccur, 0, sizeof(int) * (size_t)nc, b->stream));
    if (b->laid) {
      layout_count_kernel<real><<<gblocks, 256, 0, b->stream>>>(b->pool[b->cur], R, b->grun, b->ngroups, goff_old,
                                                                gmax_old, s, b->ccnt, b->hcnt);
      CKL2();
      tail_count_kernel<real><<<persistent(b->n_part), 256, 0, b->stream>>>(b->pool[b->cur], R, b->st, b->part_items,
                                                                             b->n_part, kChunk, s, goff_old, b->ccnt);
      CKL2();
    } else {
      cellcount2d_kernel<real><<<persistent(b->n_part), 256, 0, b->stream>>>(b->pool[b->cur], R, b->st,
                                                                              b->part_items, b->n_part, kChunk, s,
                                                                              b->ccnt);
      CKL2();
    }
    group_rows2d_kernel<real><<<gblocks, 256, 0, b->stream>>>(R, b->grun, b->ngroups, b->ccnt, gmax, b->gsz,
                                                               b->gfree);
    CKL2();
    CKR2(scan_excl(b, b->gsz, goff, b->ngroups + 1, b->scan_tmp, b->scan_len));
    // the destinations: the empty slots first (perm -1), since the scatter then
    // fills some of them with other cells' particles; then the move
    int* perm = b->perm;
    pad2d_kernel<real><<<gblocks, 256, 0, b->stream>>>(perm, R, b->grun, b->ngroups, goff, gmax, b->ccnt);
    CKL2();
    CK2(cudaMemsetAsync(b->gover, 0, sizeof(int) * (size_t)std::max(b->ngroups, 1), b->stream));
    if (b->laid) {
      layout_perm_kernel<real><<<gblocks, 256, 0, b->stream>>>(b->pool[b->cur], R, b->grun, b->ngroups, goff_old,
                                                               gmax_old, goff, gmax, b->gfree, b->ccnt, b->hcnt,
                                                               b->ccur, b->gover, s, perm, b->err);
      CKL2();
      tail_perm_kernel<real><<<persistent(b->n_part), 256, 0, b->stream>>>(
          b->pool[b->cur], R, b->st, b->part_items, b->n_part, kChunk, s, goff_old, goff, gmax, b->gfree, b->ccnt,
          b->hcnt, b->ccur, b->gover, perm, b->err);
      CKL2();
    } else {
      cellscatter2d_kernel<real><<<persistent(b->n_part), 256, 0, b->stream>>>(
          b->pool[b->cur], perm, R, b->st, b->part_items, b->n_part, kChunk, s, goff, gmax, b->gfree, b->ccnt,
          b->ccur, b->gover, b->err);
      CKL2();
    }
    layout_gather2d_kernel<real><<<persistent(b->n_part), 256, 0, b->stream>>>(
        b->pool[b->cur], b->pool[nb], R, b->part_items, b->n_part, kChunk, s, goff, perm);
    CKL2();
    layout_count2d_kernel<real><<<(b->nruns + 127) / 128, 128, 0, b->stream>>>(R, b->st, b->nruns, s, goff);
    CKL2();
  }
  b->cur = nb;
  b->laid = true;
  return PIC_OK;
}

template <typename real>
int sr_grid(pic2d_batch* b) {
  sr_grid_kernel<real><<<persistent(b->nruns), 256, 0, b->stream>>>((real*)b->field, runs_of<real>(b), b->nruns);
  CKL2();
  return PIC_OK;
}

template <typename real>
int renew_phi(pic2d_batch* b) {
  real* rho = (real*)b->rho;
  real* tmp = (real*)b->rho2;
  const Run<real>* R = runs_of<real>(b);
  phi_rho_kernel<real><<<persistent(b->n_rhorow), 128, 0, b->stream>>>((real*)b->field, R, b->rho_items, b->n_rhorow, rho);
  CKL2();
  const real* S = (const real*)b->sines;
  dst_gemm_kernel<real><<<persistent(b->n_tile), 256, 0, b->stream>>>(R, b->tile_items, b->n_tile, rho, tmp, S, 0);
  CKL2();
  dst_gemm_kernel<real><<<persistent(b->n_tile), 256, 0, b->stream>>>(R, b->tile_items, b->n_tile, tmp, rho, S, 1);
  CKL2();
  dst_gemm_kernel<real><<<persistent(b->n_tile), 256, 0, b->stream>>>(R, b->tile_items, b->n_tile, rho, tmp, S, 2);
  CKL2();
  dst_gemm_kernel<real><<<persistent(b->n_tile), 256, 0, b->stream>>>(R, b->tile_items, b->n_tile, tmp, rho, S, 3);
  CKL2();
  phi_apply_kernel<real><<<persistent(b->n_rhorow), 128, 0, b->stream>>>((real*)b->field, R, b->rho_items, b->n_rhorow, rho);
  CKL2();
  return PIC_OK;
}

template <typename real>
int push(pic2d_batch* b) {
  const Run<real>* R = runs_of<real>(b);
  real* F = (real*)b->field;
  Layout2 L{{b->goff[b->cur][0], b->goff[b->cur][1]}, {b->gmax[b->cur][0], b->gmax[b->cur][1]}};
  const Pools P = b->pool[b->cur];
  switch (b->tile_x) {
    case 1:
      push2d_tiled_kernel<real, 1><<<b->push_blocks, 32, 0, b->stream>>>(P, F, R, L, b->ptile_items, b->n_ptile, b->err);
      break;
    case 2:
      push2d_tiled_kernel<real, 2><<<b->push_blocks, 64, 0, b->stream>>>(P, F, R, L, b->ptile_items, b->n_ptile, b->err);
      break;
    case 8:
      push2d_tiled_kernel<real, 8><<<b->push_blocks, 256, 0, b->stream>>>(P, F, R, L, b->ptile_items, b->n_ptile, b->err);
      break;
    default:
      push2d_tiled_kernel<real, 4><<<b->push_blocks, 128, 0, b->stream>>>(P, F, R, L, b->ptile_items, b->n_ptile, b->err);
  }
  CKL2();
  return PIC_OK;
}

// The push's work list for tiles of tx group rows: per run and species, the
// tiles in row-major order (consecutive items share the run's fields in L2).
int set_tiles(pic2d_batch* b, int tx) {
  std::vector<Item> v;
  for (int r = 0; r < b->nruns; ++r) {
    const int nx = b->cfg[r].nx, nzb = (b->cfg[r].nz + 31) / 32, tn = (nx + tx - 1) / tx;
    for (int s = 0; s < 2; ++s)
      for (int t = 0; t < tn * nzb; ++t) v.push_back({2 * r + s, t});
  }
  cudaFree(b->ptile_items);
  b->ptile_items = nullptr;
  b->n_ptile = (int)v.size();
  CK2(cudaMalloc(&b->ptile_items, sizeof(Item) * std::max<size_t>(v.size(), 1)));
  CK2(cudaMemcpy(b->ptile_items, v.data(), sizeof(Item) * v.size(), cudaMemcpyHostToDevice));
  b->tile_x = tx;
  return PIC_OK;
}

// Zero J, n and phi of every run (renew_grid, :1348-1389).
template <typename real>
int renew_grid(pic2d_batch* b) {
  zero_sources_kernel<real><<<persistent(b->nruns), 256, 0, b->stream>>>((real*)b->field, runs_of<real>(b), b->nruns);
  CKL2();
  return PIC_OK;
}

// One loop body for every run (fdtd :627-1015).
template <typename real>
int step_body(pic2d_batch* b, bool refill, bool sort = false) {
  const Run<real>* R = runs_of<real>(b);
  real* F = (real*)b->field;
  CKR2(renew_grid<real>(b));
  if (refill) {
    delete5_kernel<real><<<persistent(b->n_part), 256, 0, b->stream>>>(b->pool[b->cur], R, b->st, b->part_items,
                                                                        b->n_part, kChunk);
    CKL2();
    CKR2(run_sources<real>(b, 1));  // appended after the layout
    CKR2(cellsort<real>(b));        // everything into a new layout, the deleted slots dropped
  } else if (sort) {
    CKR2(cellsort<real>(b));
  }
  renew_b4_kernel<real><<<persistent(b->n_row), 256, 0, b->stream>>>(F, R, b->row_items, b->n_row);
  CKL2();
  CKR2(sr_grid<real>(b));
  CKR2(push<real>(b));
  fold_kernel<real><<<persistent(b->nruns), 256, 0, b->stream>>>(F, R, b->nruns, P_JIX, 6);
  CKL2();
  fold_kernel<real><<<persistent(b->nruns), 256, 0, b->stream>>>(F, R, b->nruns, P_NI, 2);
  CKL2();
  coil_kernel<real><<<(b->nruns + 127) / 128, 128, 0, b->stream>>>(F, R, b->nruns, b->step_dev);
  CKL2();
  renew_b4_kernel<real><<<persistent(b->n_row), 256, 0, b->stream>>>(F, R, b->row_items, b->n_row);
  CKL2();
  CKR2(sr_grid<real>(b));
  renew_e4_kernel<real><<<persistent(b->n_row), 256, 0, b->stream>>>(F, R, b->row_items, b->n_row);
  CKL2();
  CKR2(sr_grid<real>(b));
  CKR2(renew_phi<real>(b));
  CKR2(sr_grid<real>(b));
  step_advance_kernel<<<1, 1, 0, b->stream>>>(b->step_dev);
  CKL2();
  return PIC_OK;
}

void drop_graphs(pic2d_batch* b) {
  for (auto& row : b->graph)
    for (auto& g : row)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
}

// nsteps loop bodies, each replayed from a CUDA graph captured on first use:
// one graph per kind of step -- plain, with the cell sort (every
// sort_interval steps), with the refill (every add_interval steps) -- and per
// pool the step starts on, since the sort moves the particles to the other
// pool. The launches of a step depend on nothing else the host holds (counts,
// stream counters and the step number live on the device), so at most six
// graphs cover a run.
template <typename real>
int run_steps(pic2d_batch* b, int nsteps) {
  for (int i = 0; i < nsteps; ++i) {
    const bool refill = b->c_add > b->cfg[0].add_interval - 1;
    const int si = b->cfg[0].sort_interval;
    const bool sort = !refill && si > 0 && b->step > 0 && b->step % si == 0;
    if (!b->use_graph) {
      CKR2(step_body<real>(b, refill, sort));
    } else {
      const int kind = refill ? 2 : sort ? 1 : 0, cur = b->cur;
      if (!b->graph[kind][cur]) {
        CK2(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        const long long l0 = b->launches;
        const int rc = step_body<real>(b, refill, sort);
        cudaGraph_t graph = nullptr;
        const cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
        b->graph_launches[kind][cur] = b->launches - l0;
        b->launches = l0;
        b->graph_cur[kind][cur] = b->cur;
        b->cur = cur;
        if (rc != PIC_OK) {
          if (graph) cudaGraphDestroy(graph);
          return rc;
        }
        CK2(e);
        const cudaError_t ei = cudaGraphInstantiate(&b->graph[kind][cur], graph, 0);
        cudaGraphDestroy(graph);
        CK2(ei);
      }
      CK2(cudaGraphLaunch(b->graph[kind][cur], b->stream));
      b->launches += b->graph_launches[kind][cur];
      b->cur = b->graph_cur[kind][cur];
    }
    if (refill) b->c_add = 0;
    b->c_add++;
    b->step++;
  }
  return PIC_OK;
}

template <typename real>
int do_init(pic2d_batch* b) {
  real* F = (real*)b->field;
  const Run<real>* R = runs_of<real>(b);
  const Run<real>* H = runs_host<real>(b);
  // init_grid (:224-387): fields zero apart from B0 = B = IMF (the dipole terms
  // are zeroed in the reference, :368, :385), so the whole block is cleared
  CK2(cudaMemsetAsync(F, 0, sizeof(real) * (size_t)b->field_nodes, b->stream));
  for (int r = 0; r < b->nruns; ++r) {
    const pic2d_config& k = b->cfg[r];
    // b0y = by = IMF_y everywhere; bx, bz, b0x, b0z = IMF_x / IMF_z on the interior
    std::vector<real> h((size_t)H[r].nodes);
    std::fill(h.begin(), h.end(), (real)k.imf_y);
    CK2(cudaMemcpyAsync(F + H[r].foff + (long long)P_BY * H[r].nodes, h.data(), sizeof(real) * h.size(),
                        cudaMemcpyHostToDevice, b->stream));
    CK2(cudaMemcpyAsync(F + H[r].foff + (long long)P_B0Y * H[r].nodes, h.data(), sizeof(real) * h.size(),
                        cudaMemcpyHostToDevice, b->stream));
    for (int comp = 0; comp < 2; ++comp) {
      const double imf = comp == 0 ? k.imf_x : k.imf_z;
      if (imf == 0.0) continue;
      std::fill(h.begin(), h.end(), (real)0);
      for (int kk = 2; kk < k.nx + 2; ++kk)
        for (int m = 2; m < k.nz + 2; ++m) h[(size_t)kk * (k.nz + 4) + m] = (real)imf;
      const int pa = comp == 0 ? P_BX : P_BZ, pb0 = comp == 0 ? P_B0X : P_B0Z;
      CK2(cudaMemcpyAsync(F + H[r].foff + (long long)pa * H[r].nodes, h.data(), sizeof(real) * h.size(),
                          cudaMemcpyHostToDevice, b->stream));
      CK2(cudaMemcpyAsync(F + H[r].foff + (long long)pb0 * H[r].nodes, h.data(), sizeof(real) * h.size(),
                          cudaMemcpyHostToDevice, b->stream));
    }
    CK2(cudaStreamSynchronize(b->stream));
  }
  // particles (init_particle :389-525)
  CK2(cudaMemsetAsync(b->st, 0, sizeof(State) * b->nruns, b->stream));
  for (int p = 0; p < 2; ++p) CK2(cudaMemsetAsync(b->pool[p].cell[0], 0xff, sizeof(int) * b->pool_slots, b->stream));
  for (int p = 0; p < 2; ++p) CK2(cudaMemsetAsync(b->pool[p].cell[1], 0xff, sizeof(int) * b->pool_slots, b->stream));
  b->laid = false;  // the first sort goes from slot order
  CKR2(run_sources<real>(b, 0));
  CKR2(cellsort<real>(b));  // the particles by cell (only their order changes)
  // fdtd's set-up (:583-625)
  CKR2(renew_grid<real>(b));
  density2d_kernel<real><<<persistent(b->n_part), 256, 0, b->stream>>>(b->pool[b->cur], F, R, b->st, b->part_items,
                                                                        b->n_part, kChunk);
  CKL2();
  fold_kernel<real><<<persistent(b->nruns), 256, 0, b->stream>>>(F, R, b->nruns, P_NI, 2);
  CKL2();
  CKR2(sr_grid<real>(b));
  CK2(cudaMemsetAsync(b->step_dev, 0, sizeof(int), b->stream));
  CKR2(renew_phi<real>(b));
  CKR2(sr_grid<real>(b));
  CK2(cudaStreamSynchronize(b->stream));
  b->c_add = 0;
  b->step = 0;
  b->ready = true;
  drop_graphs(b);
  return PIC_OK;
}

template <typename real>
int do_create(pic2d_batch* b) {
  const int n = b->nruns;
  b->runs_host.assign(sizeof(Run<real>) * n, 0);
  Run<real>* H = runs_host<real>(b);
  long long foff = 0, poff = 0, roff = 0;
  int ngroups = 0;
  std::vector<int> sine_sizes;
  std::vector<std::pair<int, long long>> sine_off;  // size -> offset
  std::vector<double> sines;
  auto sine_table = [&](int m) -> long long {
    for (auto& p : sine_off)
      if (p.first == m) return p.second;
    const long long o = (long long)sines.size();
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < m; ++j) sines.push_back(std::sin(3.14159265358979323846 * (double)i * (double)j / (double)m));
    sine_off.push_back({m, o});
    return o;
  };
  for (int r = 0; r < n; ++r) {
    const pic2d_config& k = b->cfg[r];
    Run<real>& R = H[r];
    R.nx = k.nx; R.nz = k.nz; R.gx = k.nx + 4; R.gz = k.nz + 4; R.nodes = R.gx * R.gz;
    R.np = k.np;
    R.foff = foff;
    foff += (long long)P_COUNT * R.nodes;
    foff = (foff + 63) & ~63LL;
    const long long refill = 2LL * k.np * k.nx * k.np + 2LL * (k.np * (long long)k.nz - 2) * k.np;
    R.nzb = (k.nz + 31) / 32;
    R.ngroups = k.nx * R.nzb;
    R.gbase = ngroups;
    ngroups += R.ngroups;
    // the tiled layout takes 32 slots per group row, as many rows as the
    // group's fullest cell: with m = Np^2 particles per cell on average (about
    // Poisson-distributed), room for 1.25 m + 4 sqrt(m) + 4 in every lane,
    // then a refill appended before the next sort
    const double m = (double)k.np * k.np;
    const long long layout = 32LL * R.ngroups * (long long)std::ceil(1.25 * m + 4 * std::sqrt(m) + 4);
    R.cap = k.capacity > 0 ? k.capacity : layout + 2 * refill + 4096;
    R.cap = (R.cap + kChunk - 1) / kChunk * kChunk;
    R.poff = poff;
    poff += R.cap;
    R.a1 = k.absorb_grid; R.a2 = k.absorb_grid2; R.a3 = k.absorb_grid3;
    R.dx = k.dx; R.dt = k.dt; R.q = k.q; R.e0 = k.e0; R.mu0 = k.mu0; R.c = k.c;
    R.sigma_a = k.sigma_a;
    R.coil_i = k.coil_i;
    R.vdrift = k.v_drift;
    R.sig[0] = std::sqrt(k.kb * k.ti / k.mi);
    R.sig[1] = std::sqrt(k.kb * k.te / k.me);
    R.nw = k.n_all / k.np / k.np;
    R.T[0] = 0.5 * k.q * k.dt / k.mi;
    R.T[1] = 0.5 * k.q * k.dt / -k.me;
    R.ex_add = k.v_drift * k.imf_y;
    R.ey_add = -k.v_drift * k.imf_x;
    R.seed_p = k.seed_p;
    R.seed_v = k.seed_v;
    R.add_interval = k.add_interval;
    R.sz_dst = 0;
    R.roff = roff;
    roff += (long long)k.nx * k.nz;
    const long long sx = sine_table(k.nx);
    const long long sz = sine_table(k.nz);
    // the kernel expects S_nx then S_nz back to back: store a pair when they are not
    if (sz != sx + (long long)k.nx * k.nx) {
      const long long o = (long long)sines.size();
      for (long long q = 0; q < (long long)k.nx * k.nx; ++q) sines.push_back(sines[sx + q]);
      for (long long q = 0; q < (long long)k.nz * k.nz; ++q) sines.push_back(sines[sz + q]);
      R.sz_dst = (int)o;
    } else {
      R.sz_dst = (int)sx;
    }
  }
  b->field_nodes = foff;
  b->pool_slots = poff;
  b->rho_len = roff;
  b->ngroups = ngroups;
  if (poff >= (1LL << 31) - kChunk) return PIC_ERR_CAPACITY;  // slot offsets are 32-bit
  {
    std::vector<int> grun(ngroups);
    for (int r = 0; r < n; ++r)
      for (int q = 0; q < H[r].ngroups; ++q) grun[H[r].gbase + q] = r;
    CK2(cudaMalloc(&b->grun, sizeof(int) * std::max(ngroups, 1)));
    CK2(cudaMemcpy(b->grun, grun.data(), sizeof(int) * ngroups, cudaMemcpyHostToDevice));
    CK2(cudaMalloc(&b->gsz, sizeof(int) * (ngroups + 1)));
    CK2(cudaMemset(b->gsz, 0, sizeof(int) * (ngroups + 1)));
    for (int p = 0; p < 2; ++p)
      for (int s = 0; s < 2; ++s) {
        CK2(cudaMalloc(&b->goff[p][s], sizeof(int) * (ngroups + 1)));
        CK2(cudaMemset(b->goff[p][s], 0, sizeof(int) * (ngroups + 1)));
        CK2(cudaMalloc(&b->gmax[p][s], sizeof(int) * std::max(ngroups, 1)));
        CK2(cudaMemset(b->gmax[p][s], 0, sizeof(int) * std::max(ngroups, 1)));
      }
  }
  CK2(cudaMalloc(&b->runs_dev, sizeof(Run<real>) * n));
  CK2(cudaMemcpy(b->runs_dev, H, sizeof(Run<real>) * n, cudaMemcpyHostToDevice));
  CK2(cudaMalloc(&b->st, sizeof(State) * n));
  CK2(cudaMemset(b->st, 0, sizeof(State) * n));
  CK2(cudaMalloc(&b->field, sizeof(real) * (size_t)foff));
  for (int p = 0; p < 2; ++p)
    for (int s = 0; s < 2; ++s) {
      CK2(cudaMalloc(&b->pool[p].cell[s], sizeof(int) * (size_t)poff));
      for (int a = 0; a < 2; ++a) CK2(cudaMalloc(&b->pool[p].o[s][a], sizeof(real) * (size_t)poff));
      for (int a = 0; a < 3; ++a) CK2(cudaMalloc(&b->pool[p].v[s][a], sizeof(real) * (size_t)poff));
    }
  std::vector<real> sr(sines.begin(), sines.end());
  CK2(cudaMalloc(&b->sines, sizeof(real) * std::max<size_t>(sr.size(), 1)));
  CK2(cudaMemcpy(b->sines, sr.data(), sizeof(real) * sr.size(), cudaMemcpyHostToDevice));
  CK2(cudaMalloc(&b->rho, sizeof(real) * (size_t)roff));
  CK2(cudaMalloc(&b->rho2, sizeof(real) * (size_t)roff));
  // work lists
  std::vector<Item> rows, rhos, parts, tiles;
  for (int r = 0; r < n; ++r) {
    for (int k = 2; k < H[r].nx + 2; k += kFieldRows) rows.push_back({r, k});
    for (int k = 0; k < H[r].nx; ++k) rhos.push_back({r, k});
    for (int s = 0; s < 2; ++s)
      for (long long q = 0; q < H[r].cap; q += kChunk) parts.push_back({2 * r + s, (int)q});
    const int tn = (H[r].nz + kGemmTile - 1) / kGemmTile, tm = (H[r].nx + kGemmTile - 1) / kGemmTile;
    for (int t = 0; t < tn * tm; ++t) tiles.push_back({r, t});
  }
  auto upload = [&](const std::vector<Item>& v, Item** dst, int* cnt) -> int {
    *cnt = (int)v.size();
    CK2(cudaMalloc(dst, sizeof(Item) * std::max<size_t>(v.size(), 1)));
    CK2(cudaMemcpy(*dst, v.data(), sizeof(Item) * v.size(), cudaMemcpyHostToDevice));
    return PIC_OK;
  };
  CKR2(upload(rows, &b->row_items, &b->n_row));
  CKR2(upload(rhos, &b->rho_items, &b->n_rhorow));
  CKR2(upload(parts, &b->part_items, &b->n_part));
  CKR2(upload(tiles, &b->tile_items, &b->n_tile));
  for (int which = 0; which < 2; ++which) {
    std::vector<SourceSet> sets;
    make_sets<real>(b, which, sets);
    for (int s = 0; s < 2; ++s) {
      CK2(cudaMalloc(&b->sets[which][s], sizeof(SourceSet) * n));
      CK2(cudaMemcpy(b->sets[which][s], sets.data(), sizeof(SourceSet) * n, cudaMemcpyHostToDevice));
      std::vector<Item> it;
      for (int r = 0; r < n; ++r)
        for (long long q = 0; q < sets[r].total; q += kChunk) it.push_back({r, (int)q});
      CKR2(upload(it, &b->src_items[which][s], &b->n_src[which][s]));
    }
  }
  CK2(cudaMalloc(&b->perm, sizeof(int) * (size_t)poff));
  b->scan_len = (size_t)(2 * ((poff + kScanTile - 1) / kScanTile) + 64);
  CK2(cudaMalloc(&b->scan_tmp, sizeof(int) * b->scan_len));
  CK2(cudaMalloc(&b->ccnt, sizeof(int) * (size_t)std::max(b->rho_len, 1LL)));
  CK2(cudaMalloc(&b->ccur, sizeof(int) * (size_t)std::max(b->rho_len, 1LL)));
  CK2(cudaMalloc(&b->gfree, sizeof(int) * 32 * (size_t)std::max(b->ngroups, 1)));
  CK2(cudaMalloc(&b->gover, sizeof(int) * (size_t)std::max(b->ngroups, 1)));
  CK2(cudaMalloc(&b->hcnt, sizeof(int) * (size_t)std::max(b->rho_len, 1LL)));
  CK2(cudaMalloc(&b->step_dev, sizeof(int)));
  CK2(cudaMemset(b->step_dev, 0, sizeof(int)));
  CK2(cudaMalloc(&b->err, sizeof(unsigned long long) * ERR_COUNT));
  CK2(cudaMemset(b->err, 0, sizeof(unsigned long long) * ERR_COUNT));
  CKR2(set_tiles(b, 4));
  b->push_blocks = persistent(b->n_ptile, 8);
  return PIC_OK;
}

void free_batch(pic2d_batch* b) {
  drop_graphs(b);
  cudaFree(b->runs_dev); cudaFree(b->st); cudaFree(b->field);
  for (int p = 0; p < 2; ++p)
    for (int s = 0; s < 2; ++s) {
      cudaFree(b->pool[p].cell[s]);
      for (int a = 0; a < 2; ++a) cudaFree(b->pool[p].o[s][a]);
      for (int a = 0; a < 3; ++a) cudaFree(b->pool[p].v[s][a]);
    }
  cudaFree(b->sines); cudaFree(b->rho); cudaFree(b->rho2);
  cudaFree(b->row_items); cudaFree(b->rho_items); cudaFree(b->part_items); cudaFree(b->tile_items);
  for (int w = 0; w < 2; ++w)
    for (int s = 0; s < 2; ++s) { cudaFree(b->src_items[w][s]); cudaFree(b->sets[w][s]); }
  cudaFree(b->perm); cudaFree(b->scan_tmp); cudaFree(b->step_dev); cudaFree(b->err);
  cudaFree(b->ccnt); cudaFree(b->ccur); cudaFree(b->gfree); cudaFree(b->gover); cudaFree(b->hcnt);
  cudaFree(b->grun); cudaFree(b->gsz); cudaFree(b->ptile_items);
  for (int p = 0; p < 2; ++p)
    for (int s = 0; s < 2; ++s) { cudaFree(b->goff[p][s]); cudaFree(b->gmax[p][s]); }
  if (b->stream) cudaStreamDestroy(b->stream);
}

#define DISPATCH2(b, call) ((b)->prec == 64 ? call<double> : call<float>)

int valid(const pic2d_config& k) {
  if (k.nx < 8 || k.nz < 8 || k.np < 1 || k.nx + 4 >= (1 << kCellShift) || k.nz + 4 >= (1 << kCellShift)) return 0;
  if (k.dx <= 0 || k.dt <= 0 || k.mi <= 0 || k.me <= 0 || k.e0 <= 0 || k.c <= 0) return 0;
  if (k.absorb_grid3 < 2 || k.add_interval < 1) return 0;
  return 1;
}

template <typename real>
int do_get_particles(pic2d_batch* b, int run, int s, double* rows, long long cap, long long* n_out) {
  const Run<real>& R = runs_host<real>(b)[run];
  State S;
  CK2(cudaMemcpyAsync(&S, b->st + run, sizeof(State), cudaMemcpyDeviceToHost, b->stream));
  CK2(cudaStreamSynchronize(b->stream));
  const int n = S.count[s];
  if (n == 0) {
    *n_out = 0;
    return PIC_OK;
  }
  int* flags = nullptr;
  int* pos = nullptr;
  int* tmp = nullptr;
  const size_t tl = (size_t)(2 * ((n + kScanTile - 1) / kScanTile) + 64);
  CK2(cudaMalloc(&flags, sizeof(int) * n));
  CK2(cudaMalloc(&pos, sizeof(int) * n));
  CK2(cudaMalloc(&tmp, sizeof(int) * tl));
  flag_kernel<<<(n + 255) / 256, 256, 0, b->stream>>>(b->pool[b->cur].cell[s], R.poff, n, flags);
  int rc = scan_excl(b, flags, pos, n, tmp, tl);
  int lp = 0, lf = 0;
  double* dev = nullptr;
  if (rc == PIC_OK) {
    cudaMemcpyAsync(&lp, pos + n - 1, sizeof(int), cudaMemcpyDeviceToHost, b->stream);
    cudaMemcpyAsync(&lf, flags + n - 1, sizeof(int), cudaMemcpyDeviceToHost, b->stream);
    cudaStreamSynchronize(b->stream);
    const long long live = (long long)lp + lf;
    *n_out = live;
    if (rows && cap > 0 && live > 0) {
      cudaMalloc(&dev, sizeof(double) * 6 * (size_t)live);
      parts2d_export_kernel<real><<<(n + 255) / 256, 256, 0, b->stream>>>(b->pool[b->cur], R, s, n, pos, dev);
      cudaMemcpyAsync(rows, dev, sizeof(double) * 6 * (size_t)std::min(live, cap), cudaMemcpyDeviceToHost, b->stream);
      cudaStreamSynchronize(b->stream);
    }
  }
  cudaFree(dev); cudaFree(flags); cudaFree(pos); cudaFree(tmp);
  CK2(cudaGetLastError());
  return rc;
}

template <typename real>
int do_get_grid(pic2d_batch* b, int run, double* rec) {
  const Run<real>& R = runs_host<real>(b)[run];
  double* dev = nullptr;
  CK2(cudaMalloc(&dev, sizeof(double) * 18 * (size_t)R.nodes));
  grid2d_export_kernel<real><<<(R.nodes + 255) / 256, 256, 0, b->stream>>>((const real*)b->field, R, dev);
  cudaError_t e = cudaMemcpyAsync(rec, dev, sizeof(double) * 18 * (size_t)R.nodes, cudaMemcpyDeviceToHost, b->stream);
  cudaStreamSynchronize(b->stream);
  cudaFree(dev);
  CK2(e);
  CK2(cudaGetLastError());
  return PIC_OK;
}

template <typename real>
int do_thrust(pic2d_batch* b, double* out) {
  thrust2d_kernel<real><<<persistent(b->nruns), 256, 0, b->stream>>>((const real*)b->field, runs_of<real>(b), b->nruns,
                                                                       b->st);
  CKL2();
  std::vector<State> S(b->nruns);
  CK2(cudaMemcpyAsync(S.data(), b->st, sizeof(State) * b->nruns, cudaMemcpyDeviceToHost, b->stream));
  CK2(cudaStreamSynchronize(b->stream));
  for (int r = 0; r < b->nruns; ++r)
    for (int q = 0; q < 3; ++q) out[3 * r + q] = S[r].thrust[q];
  return PIC_OK;
}

// Online tuning: the next steps of the run itself try each push tile shape
// (1, 2, 4 or 8 group rows of 32 cells, one warp per row) with 8 or 16
// resident blocks' worth of persistent blocks per SM, timing whole loop
// bodies, and the fastest is kept; the steps taken are ordinary steps of the
// run.
template <typename real>
int do_autotune(pic2d_batch* b, int* choice) {
  const int shapes[4] = {1, 2, 4, 8};
  const int per_sm[2] = {8, 16};
  float best = 1e30f;
  int bt = b->tile_x, bs = b->push_blocks;
  cudaEvent_t e0, e1;
  CK2(cudaEventCreate(&e0));
  CK2(cudaEventCreate(&e1));
  int rc = PIC_OK;
  for (int i = 0; i < 4 && rc == PIC_OK; ++i)
    for (int j = 0; j < 2 && rc == PIC_OK; ++j) {
      rc = set_tiles(b, shapes[i]);
      if (rc != PIC_OK) break;
      b->push_blocks = persistent(b->n_ptile, per_sm[j]);
      const bool g = b->use_graph;
      b->use_graph = false;
      cudaEventRecord(e0, b->stream);
      rc = run_steps<real>(b, 2);
      cudaEventRecord(e1, b->stream);
      b->use_graph = g;
      if (cudaEventSynchronize(e1) != cudaSuccess) rc = PIC_ERR_CUDA;
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rc == PIC_OK && ms < best) {
        best = ms;
        bt = shapes[i];
        bs = b->push_blocks;
      }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc == PIC_OK) rc = set_tiles(b, bt);
  b->push_blocks = bs;
  drop_graphs(b);
  if (choice) {
    choice[0] = bt;
    choice[1] = bs;
  }
  return rc;
}

}  // namespace

// ================================================================ C ABI
extern "C" {

int pic2d_config_normalized(pic2d_config* k, int nx, int nz, int np) {
  if (!k) return PIC_ERR_ARG;
  std::memset(k, 0, sizeof(*k));
  k->nx = nx; k->nz = nz; k->np = np;
  k->dx = 1.0; k->dt = 0.5 * 6.0 / (7.0 * std::sqrt(2.0));
  k->q = 1.0; k->mi = 100.0; k->me = 1.0; k->mu0 = 1.0; k->e0 = 1.0; k->kb = 1.0; k->c = 1.0;
  k->v_drift = 0.1; k->n_all = 0.01; k->ti = 0.0025; k->te = 0.0025; k->coil_i = 12.0;
  k->absorb_grid = 32; k->absorb_grid2 = 16; k->absorb_grid3 = 32;
  k->sigma_a = 1e-6;
  k->add_interval = 250;
  k->sort_interval = 12;  // the fastest of 8-24 over whole sort cycles of the 256-run batch
  k->seed_p = 0; k->seed_v = 50;
  return PIC_OK;
}

int pic2d_create(const pic2d_config* cfgs, int nruns, int precision, int device, pic2d_batch** out) {
  if (!cfgs || !out || nruns < 1 || (precision != 32 && precision != 64)) return PIC_ERR_ARG;
  for (int r = 0; r < nruns; ++r) {
    if (!valid(cfgs[r])) return PIC_ERR_ARG;
    if (cfgs[r].add_interval != cfgs[0].add_interval) return PIC_ERR_ARG;  // runs step together
    if (cfgs[r].sort_interval != cfgs[0].sort_interval || cfgs[r].sort_interval < 0) return PIC_ERR_ARG;
  }
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return PIC_ERR_CUDA;
  pic2d_batch* b = new (std::nothrow) pic2d_batch();
  if (!b) return PIC_ERR_ARG;
  b->prec = precision;
  b->device = device;
  b->rsize = precision == 64 ? 8 : 4;
  b->nruns = nruns;
  b->cfg.assign(cfgs, cfgs + nruns);
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete b;
    return PIC_ERR_CUDA;
  }
  const int rc = DISPATCH2(b, do_create)(b);
  if (rc != PIC_OK) {
    free_batch(b);
    delete b;
    return rc;
  }
  *out = b;
  return PIC_OK;
}

int pic2d_destroy(pic2d_batch* b) {
  if (!b) return PIC_ERR_ARG;
  cudaSetDevice(b->device);
  cudaStreamSynchronize(b->stream);
  free_batch(b);
  delete b;
  return PIC_OK;
}

int pic2d_init(pic2d_batch* b) {
  if (!b) return PIC_ERR_ARG;
  if (cudaSetDevice(b->device) != cudaSuccess) return PIC_ERR_CUDA;
  return DISPATCH2(b, do_init)(b);
}

int pic2d_step(pic2d_batch* b, int nsteps) {
  if (!b || nsteps < 0) return PIC_ERR_ARG;
  if (!b->ready) return PIC_ERR_STATE;
  if (cudaSetDevice(b->device) != cudaSuccess) return PIC_ERR_CUDA;
  return DISPATCH2(b, run_steps)(b, nsteps);
}

int pic2d_thrust(pic2d_batch* b, double* out3) {
  if (!b || !out3) return PIC_ERR_ARG;
  if (!b->ready) return PIC_ERR_STATE;
  return DISPATCH2(b, do_thrust)(b, out3);
}

int pic2d_particle_count(pic2d_batch* b, int run, int species, long long* n) {
  if (!b || !n || run < 0 || run >= b->nruns || species < 0 || species > 1) return PIC_ERR_ARG;
  return (b->prec == 64 ? do_get_particles<double> : do_get_particles<float>)(b, run, species, nullptr, 0, n);
}

int pic2d_get_particles(pic2d_batch* b, int run, int species, double* rows6, long long cap, long long* n) {
  if (!b || !n || run < 0 || run >= b->nruns || species < 0 || species > 1) return PIC_ERR_ARG;
  return (b->prec == 64 ? do_get_particles<double> : do_get_particles<float>)(b, run, species, rows6, cap, n);
}

int pic2d_get_grid(pic2d_batch* b, int run, double* records) {
  if (!b || !records || run < 0 || run >= b->nruns) return PIC_ERR_ARG;
  return (b->prec == 64 ? do_get_grid<double> : do_get_grid<float>)(b, run, records);
}

int pic2d_set_push_shape(pic2d_batch* b, int tile_rows, int blocks) {
  if (!b || (tile_rows != 1 && tile_rows != 2 && tile_rows != 4 && tile_rows != 8) || blocks < 1) return PIC_ERR_ARG;
  CKR2(set_tiles(b, tile_rows));
  b->push_blocks = blocks;
  drop_graphs(b);
  return PIC_OK;
}

int pic2d_autotune(pic2d_batch* b, int* choice2) {
  if (!b) return PIC_ERR_ARG;
  if (!b->ready) return PIC_ERR_STATE;
  return DISPATCH2(b, do_autotune)(b, choice2);
}

int pic2d_set_graph(pic2d_batch* b, int enable) {
  if (!b) return PIC_ERR_ARG;
  b->use_graph = enable != 0;
  drop_graphs(b);
  return PIC_OK;
}

int pic2d_status(pic2d_batch* b, long long* counters8) {
  if (!b || !counters8) return PIC_ERR_ARG;
  // read on the batch's stream, after the work queued before this call (the
  // stream does not synchronise with the legacy default stream)
  unsigned long long h[ERR_COUNT];
  if (cudaMemcpyAsync(h, b->err, sizeof(h), cudaMemcpyDeviceToHost, b->stream) != cudaSuccess ||
      cudaStreamSynchronize(b->stream) != cudaSuccess)
    return PIC_ERR_CUDA;
  for (int q = 0; q < 8; ++q) counters8[q] = (long long)h[q];
  counters8[4] = b->step;
  counters8[5] = b->launches;
  return (h[0] | h[1] | h[2] | h[ERR_STORE_FULL]) ? PIC_ERR_DEVICE : PIC_OK;
}

int pic2d_get_stream(pic2d_batch* b, void** stream) {
  if (!b || !stream) return PIC_ERR_ARG;
  *stream = (void*)b->stream;
  return PIC_OK;
}

}  // extern "C"
