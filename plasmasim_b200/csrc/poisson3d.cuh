// Poisson divergence cleaning of the 3D step: renew_phi3 (PIC/3d_pic458_domain.c
// :8315-8665), sr_phi (:1389-1574) and sr_e at MPI size 1, the block that fdtd
// runs after renew_e4_2 when the reference is built with its PHI blocks
// (:901-907, and once after the first add_*_flat, :676-681).
//
// The reference solves lap(phi) = rho for the Gauss-law residual rho with
// three sine transforms (its sinft, :8182-8210), a division by the eigenvalues
// of the 3-point Laplacian and three inverse transforms. Here each transform
// is a GEMM against the n x n sine matrix S[k][j] = sin(pi j k / n), whose row
// and column 0 vanish (sinft sets data[1] = 0, so the first element of every
// line never enters): the z transform multiplies the (x*y) x z matrix from the
// right, the y transform multiplies every x slab from the left, the x
// transform the x x (y*z) matrix from the left. S is symmetric, so one table
// serves both sides. The transforms run in the engine's precision; the
// residual and the eigenvalue division in FP64.
#pragma once

#include "common.cuh"
#include "fields.cuh"

namespace pb {

// rho of renew_phi3 (:8338-8355) on the interior, [x][y][z], z fastest:
// -( -q (ni - ne)/e0 + div4 E ) on cells with A3 < x < Nx - A3, the same in y,
// and A3 <= z < Nz - A3 (A3 = Absorb_grid3); zero elsewhere.
template <typename real>
__global__ void phi3_rho_kernel(Fields<real> F, Geom g, double d24, double q, double e0, int a3, real* rho) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int kz = (int)(t % g.nz), ky = (int)((t / g.nz) % g.ny), kx = (int)(t / ((long long)g.nz * g.ny));
    double v = 0.0;
    if (kx > a3 && kx < g.nx - a3 && ky > a3 && ky < g.ny - a3 && kz >= a3 && kz < g.nz - a3) {
      const long long sx = g.sx, sy = g.gz;
      const long long c = (kx + 2) * sx + (ky + 2) * sy + (kz + 2);
      const real* ex = F.f[F_EX];
      const real* ey = F.f[F_EY];
      const real* ez = F.f[F_EZ];
      // one left-to-right sum, as the reference writes it
      const double div = -(double)ex[c + 2 * sx] + 27. * (double)ex[c + sx] - 27. * (double)ex[c] + (double)ex[c - sx] -
                         (double)ey[c + 2 * sy] + 27. * (double)ey[c + sy] - 27. * (double)ey[c] + (double)ey[c - sy] -
                         (double)ez[c + 2] + 27. * (double)ez[c + 1] - 27. * (double)ez[c] + (double)ez[c - 1];
      v = -(-q * ((double)F.f[F_NI][c] - (double)F.f[F_NE][c]) / e0 + div / d24);
    }
    rho[t] = (real)v;
  }
}

// Batched GEMM C[b] = mul * L[b] R[b] / div with row-major operands:
// L(m, k) = L[b*lb + m*lm + k], R(k, n) = R[b*rb + k*rk + n], C(m, n) = C[b*cb + m*cm + n].
// `solve` divides each element by the Laplacian eigenvalue of wave numbers
// (kx, ky, kz) = (m, n / nz, n % nz) (:8502-8511: zero where it vanishes).
template <typename real>
struct DstGemm {
  const real* L;
  long long lb;
  long long lm;
  const real* R;
  long long rb;
  long long rk;
  real* C;
  long long cb;
  long long cm;
  int M, N, K, B;
  double mul, div;     // C = mul * (L R) / div: 1, 1 forward; 2, n inverse (:8086-8180)
  int solve;
  const double* sin2;  // sin^2(pi k / 2n): x (nx), then y (ny), then z (nz)
  int nx, ny, nz;
  double h2;           // (dx/2)^2
};

constexpr int kDstTile = 64, kDstK = 16;

template <typename real>
__global__ void __launch_bounds__(256) dst3_gemm_kernel(DstGemm<real> a) {
  __shared__ real Ls[kDstK][kDstTile + 1];
  __shared__ real Rs[kDstK][kDstTile + 1];
  const int tiles_m = (a.M + kDstTile - 1) / kDstTile, tiles_n = (a.N + kDstTile - 1) / kDstTile;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  for (long long blk = blockIdx.x; blk < (long long)tiles_m * tiles_n * a.B; blk += gridDim.x) {
    const int b = (int)(blk / ((long long)tiles_m * tiles_n));
    const int r = (int)(blk % ((long long)tiles_m * tiles_n));
    const int m0 = (r / tiles_n) * kDstTile, n0 = (r % tiles_n) * kDstTile;
    const real* L = a.L + b * a.lb;
    const real* R = a.R + b * a.rb;
    real acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = (real)0;
    for (int k0 = 0; k0 < a.K; k0 += kDstK) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int e = threadIdx.x + 256 * q;
        const int lmi = e / kDstK, lki = e % kDstK;  // L tile: 64 rows x 16 k
        const int gm = m0 + lmi, gk = k0 + lki;
        Ls[lki][lmi] = (gm < a.M && gk < a.K) ? L[gm * a.lm + gk] : (real)0;
        const int rki = e / kDstTile, rni = e % kDstTile;  // R tile: 16 k x 64 cols
        const int gk2 = k0 + rki, gn = n0 + rni;
        Rs[rki][rni] = (gk2 < a.K && gn < a.N) ? R[gk2 * a.rk + gn] : (real)0;
      }
      __syncthreads();
#pragma unroll
      for (int kk = 0; kk < kDstK; ++kk) {
        real lv[4], rv[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) lv[i] = Ls[kk][ty + 16 * i];
#pragma unroll
        for (int j = 0; j < 4; ++j) rv[j] = Rs[kk][tx + 16 * j];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] += lv[i] * rv[j];
      }
      __syncthreads();
    }
    real* C = a.C + b * a.cb;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int gm = m0 + ty + 16 * i;
      if (gm >= a.M) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int gn = n0 + tx + 16 * j;
        if (gn >= a.N) continue;
        double v = a.mul * (double)acc[i][j] / a.div;
        if (a.solve) {
          const int kx = gm, ky = gn / a.nz, kz = gn % a.nz;
          const double ev = -(a.sin2[a.nx + ky] + a.sin2[a.nx + a.ny + kz] + a.sin2[kx]) / a.h2;
          v = ev == 0. ? 0. : v / ev;
        }
        C[gm * a.cm + gn] = (real)v;
      }
    }
  }
}

// phi on the interior (:8655-8661).
template <typename real>
__global__ void phi3_store_kernel(Fields<real> F, Geom g, const real* __restrict__ phi) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int kz = (int)(t % g.nz), ky = (int)((t / g.nz) % g.ny), kx = (int)(t / ((long long)g.nz * g.ny));
    F.f[F_PHI][(kx + 2) * (long long)g.sx + (ky + 2) * (long long)g.gz + (kz + 2)] = phi[t];
  }
}

// sr_phi's correction of E on the interior (:1563-1572): E += the backward
// (27, -1)/24 gradient of phi, which includes phi's ghost planes.
template <typename real>
__global__ void phi3_grad_kernel(Fields<real> F, Geom g, double d24) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int kz = (int)(t % g.nz), ky = (int)((t / g.nz) % g.ny), kx = (int)(t / ((long long)g.nz * g.ny));
    const long long sx = g.sx, sy = g.gz;
    const long long c = (kx + 2) * sx + (ky + 2) * sy + (kz + 2);
    const real* p = F.f[F_PHI];
    const double p0 = p[c];
    F.f[F_EX][c] = (real)((double)F.f[F_EX][c] +
                          (-(double)p[c + sx] + 27. * p0 - 27. * (double)p[c - sx] + (double)p[c - 2 * sx]) / d24);
    F.f[F_EY][c] = (real)((double)F.f[F_EY][c] +
                          (-(double)p[c + sy] + 27. * p0 - 27. * (double)p[c - sy] + (double)p[c - 2 * sy]) / d24);
    F.f[F_EZ][c] = (real)((double)F.f[F_EZ][c] +
                          (-(double)p[c + 1] + 27. * p0 - 27. * (double)p[c - 1] + (double)p[c - 2]) / d24);
  }
}

}  // namespace pb
