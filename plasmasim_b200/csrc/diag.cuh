// FP64 diagnostics: the thrust and energy sums of thrust_f / thrust_fave and
// the Gauss-law residual. Particle and field values are read in the step's
// precision; every product and sum is formed in double.
#pragma once

#include "common.cuh"
#include "particles.cuh"

namespace pb {

template <int N>
__device__ __forceinline__ void block_reduce_add(double (&v)[N], double* out, const int* idx,
                                                 const double* scale) {
  __shared__ double sm[N][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < N; ++q) {
    double x = v[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sm[q][wid] = x;
  }
  __syncthreads();
  if (wid == 0) {
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int q = 0; q < N; ++q) {
      double x = lane < nw ? sm[q][lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (lane == 0 && idx[q] >= 0) atomicAdd(out + idx[q], x * scale[q]);
    }
  }
}

struct ThrustParams {
  double xlo, xhi, ylo, yhi, zlo, zhi;  // open box (0.2 N dx, 0.8 N dx) per axis (:4986-4988)
  double ox, oy;                        // myrank_x Grid_Nx dx, myrank_y Grid_Ny dx (:4984-4985)
  double dx;
  int idx[10];      // output slot per partial sum (F0..F2, F[o..o+5], E[oe])
  double scale[10];
};

// Particle part of thrust_f (:4984-5101) for one species with flag > 0:
// sums over particles inside the central box of (E + v x B), E, v x B and v^2.
template <typename real>
__global__ void __launch_bounds__(256) thrust_particles_kernel(Parts<real> P, const int* __restrict__ count,
                                                               Fields<real> F, Geom g, ThrustParams tp,
                                                               double* acc) {
  double s[10];
#pragma unroll
  for (int q = 0; q < 10; ++q) s[q] = 0.0;
  const int n = *count;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int c = P.cell[t];
    if (c < 0) continue;
    int i, j, k;
    unpack_cell(c, i, j, k);
    const real fx = P.o[0][t], fy = P.o[1][t], fz = P.o[2][t];
    const double x = ((double)i + (double)fx) * tp.dx;
    const double y = ((double)j + (double)fy) * tp.dx;
    const double z = ((double)k + (double)fz) * tp.dx;
    if (!(tp.ox + x < tp.xhi && tp.ox + x > tp.xlo && tp.oy + y < tp.yhi && tp.oy + y > tp.ylo && z < tp.zhi &&
          z > tp.zlo))
      continue;
    if (!stencil_ok(g, i, j, k)) continue;
    const Axis<real> X = axis_weights(i, fx), Y = axis_weights(j, fy), Z = axis_weights(k, fz);
    const Gathered<real> e = gather6(F, g, X, Y, Z);
    const double ex = e.ex, ey = e.ey, ez = e.ez, bx = e.bx, by = e.by, bz = e.bz;
    const double vx = P.v[0][t], vy = P.v[1][t], vz = P.v[2][t];
    const double lx = vy * bz - vz * by, ly = vz * bx - vx * bz, lz = vx * by - vy * bx;
    s[0] += ex + lx; s[1] += ey + ly; s[2] += ez + lz;
    s[3] += ex; s[4] += ey; s[5] += ez;
    s[6] += lx; s[7] += ly; s[8] += lz;
    s[9] += vx * vx + vy * vy + vz * vz;
  }
  block_reduce_add<10>(s, acc, tp.idx, tp.scale);
}

struct CellBox {
  double lo[3], hi[3];   // open box on k-2, l-2, m-2 (:4965-4967)
  int ox, oy;            // myrank_x Grid_Nx, myrank_y Grid_Ny (:4971-4972)
  double e0, inv_mu0;
};

// Field part of thrust_f (:4963-4973): E[0] = sum e0 |E|^2 / 2, E[1] = sum |B|^2 / (2 mu0)
// over interior nodes of the central box (no volume factor, as in the reference).
template <typename real>
__global__ void __launch_bounds__(256) field_energy_kernel(Fields<real> F, Geom g, CellBox b, double* acc) {
  double s[2] = {0.0, 0.0};
  const int nint = g.nx * g.ny * g.nz;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nint; t += gridDim.x * blockDim.x) {
    const int m = t % g.nz, l = (t / g.nz) % g.ny, k = t / (g.nz * g.ny);
    const int kg = b.ox + k, lg = b.oy + l;
    if (!(kg < b.hi[0] && kg > b.lo[0] && lg < b.hi[1] && lg > b.lo[1] && m < b.hi[2] && m > b.lo[2])) continue;
    const int n = (k + 2) * g.sx + (l + 2) * g.gz + (m + 2);
    const double ex = F.f[F_EX][n], ey = F.f[F_EY][n], ez = F.f[F_EZ][n];
    const double bx = F.f[F_BX][n], by = F.f[F_BY][n], bz = F.f[F_BZ][n];
    s[0] += ex * ex + ey * ey + ez * ez;
    s[1] += bx * bx + by * by + bz * bz;
  }
  const int idx[2] = {27, 28};
  const double scale[2] = {0.5 * b.e0, 0.5 * b.inv_mu0};
  block_reduce_add<2>(s, acc, idx, scale);
}

// Gauss-law residual r = div4(E) - q (ni - ne)/e0 at cell centres; acc gets
// [sum r^2, sum (rho/e0)^2, max |r| (as ordered bits), cells].
template <typename real>
__global__ void __launch_bounds__(256) gauss_kernel(Fields<real> F, Geom g, double inv24dx, double q_e0,
                                                    double* acc, unsigned long long* maxbits) {
  double s[3] = {0.0, 0.0, 0.0};
  double mx = 0.0;
  const int nint = g.nx * g.ny * g.nz;
  const int sx = g.sx, sy = g.gz;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nint; t += gridDim.x * blockDim.x) {
    const int m = 2 + t % g.nz, l = 2 + (t / g.nz) % g.ny, k = 2 + t / (g.nz * g.ny);
    const int n = k * sx + l * sy + m;
    const real* ex = F.f[F_EX];
    const real* ey = F.f[F_EY];
    const real* ez = F.f[F_EZ];
    const double dvx = 27.0 * ((double)ex[n + sx] - (double)ex[n]) - ((double)ex[n + 2 * sx] - (double)ex[n - sx]);
    const double dvy = 27.0 * ((double)ey[n + sy] - (double)ey[n]) - ((double)ey[n + 2 * sy] - (double)ey[n - sy]);
    const double dvz = 27.0 * ((double)ez[n + 1] - (double)ez[n]) - ((double)ez[n + 2] - (double)ez[n - 1]);
    const double div = (dvx + dvy + dvz) * inv24dx;
    const double rho = q_e0 * ((double)F.f[F_NI][n] - (double)F.f[F_NE][n]);
    const double r = div - rho;
    s[0] += r * r;
    s[1] += rho * rho;
    s[2] += 1.0;
    mx = fmax(mx, fabs(r));
  }
  const int idx[3] = {0, 1, 3};
  const double scale[3] = {1.0, 1.0, 1.0};
  block_reduce_add<3>(s, acc, idx, scale);
  // max: non-negative doubles order like their bit patterns
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) atomicMax(maxbits, (unsigned long long)__double_as_longlong(mx));
}

// Fave += F / 500 (thrust_fave :5265-5267).
__global__ void fave_accumulate_kernel(const double* __restrict__ acc, double* fave, double scale) {
  const int q = threadIdx.x;
  if (q < 27) fave[q] += acc[q] * scale;
}

}  // namespace pb
