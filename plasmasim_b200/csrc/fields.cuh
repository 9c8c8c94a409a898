// Field kernels: dipole B0 and damping profile (init_grid), the damped
// 4th-order B and E updates (renew_b4_2 / renew_e4_2) and the size-1 periodic
// ghost copies and folds (sr_b / sr_e / sr_current2).
//
// Each update is one thread per interior node, k (z) fastest so that a warp
// reads and writes 32 consecutive nodes of every plane it touches; the +-1/+-2
// neighbours along i and j come from L1/L2. HBM bound: per node a B half-step
// moves 12 words (E3 read, DB3 read, B0 3 read, DB3 + B3 written... see below)
// and an E step 15 words.
#pragma once

#include "common.cuh"

namespace pb {

// Damping ramp on the doubled sub-grid (init_grid, PIC/3d_pic458_domain.c:339-365);
// sigma = a (0.1 sqrt(x^4+y^4+z^4) + 0.01 sqrt(x^12+y^12+z^12)) (:366-367).
__device__ __forceinline__ double sigma_of(double a, double x, double y, double z) {
  if (x == 0.0 && y == 0.0 && z == 0.0) return 0.0;
  const double x2 = x * x, y2 = y * y, z2 = z * z;
  const double x4 = x2 * x2, y4 = y2 * y2, z4 = z2 * z2;
  return a * (0.1 * sqrt(x4 + y4 + z4) + 0.01 * sqrt(x4 * x4 * x4 + y4 * y4 * y4 + z4 * z4 * z4));
}

struct Ramps {
  const double* rx;  // 2*gx values
  const double* ry;
  const double* rz;
  double a;
};

// external_current7 (:4579-4634) at rank (0,0): analytic point dipole of
// moment I*pi*R^2 along (0, sin alpha, cos alpha), centred on node
// ((nx+4)/2, (ny+4)/2, (nz+4)/2), each component on its own stagger.
struct DipoleParams {
  double mu0, I, R, alpha, dx, cutoff, imfx, imfy, imfz;
};

template <typename real>
__global__ void init_fields_kernel(Fields<real> F, Geom g, DipoleParams d) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= g.nodes) return;
  const int k = n / g.sx, l = (n / g.gz) % g.gy, m = n % g.gz;
  const double Pi = 3.14159265358979323846;
  // k + myrank_x Grid_Nx - (PROCESS_Nx Grid_Nx + 4)/2 (:4588-4589)
  const int cx = (g.gnx + 4) / 2 - g.ox, cy = (g.gny + 4) / 2 - g.oy, cz = (g.nz + 4) / 2;
  double x = (double)(k - cx) * d.dx, y = (double)(l - cy) * d.dx, z = (double)(m - cz) * d.dx;
  double r = sqrt(x * x + y * y + z * z);
  double b0x = d.imfx, b0y = d.imfy, b0z = d.imfz;
  if (r < d.cutoff * d.dx) {
    const double mom = d.mu0 * d.I * Pi * d.R * d.R;
    const double sa = sin(d.alpha), ca = cos(d.alpha);
    x = ((double)(k - cx) + 0.5) * d.dx; y = (double)(l - cy) * d.dx; z = (double)(m - cz) * d.dx;
    r = sqrt(x * x + y * y + z * z);
    b0x = mom * (3. * x * y * sa + 3. * x * z * ca) / (4. * Pi * pow(r, 5.0)) + d.imfx;
    x = (double)(k - cx) * d.dx; y = ((double)(l - cy) + 0.5) * d.dx; z = (double)(m - cz) * d.dx;
    r = sqrt(x * x + y * y + z * z);
    b0y = mom * (3. * y * y * sa + 3. * y * z * ca - r * r * sa) / (4. * Pi * pow(r, 5.0)) + d.imfy;
    x = (double)(k - cx) * d.dx; y = (double)(l - cy) * d.dx; z = ((double)(m - cz) + 0.5) * d.dx;
    r = sqrt(x * x + y * y + z * z);
    b0z = mom * (3. * y * z * sa + 3. * z * z * ca - r * r * ca) / (4. * Pi * pow(r, 5.0)) + d.imfz;
  }
  F.f[F_B0X][n] = (real)b0x; F.f[F_B0Y][n] = (real)b0y; F.f[F_B0Z][n] = (real)b0z;
  F.f[F_BX][n] = (real)b0x; F.f[F_BY][n] = (real)b0y; F.f[F_BZ][n] = (real)b0z;
  F.f[F_DBX][n] = (real)0; F.f[F_DBY][n] = (real)0; F.f[F_DBZ][n] = (real)0;
  F.f[F_EX][n] = (real)0; F.f[F_EY][n] = (real)0; F.f[F_EZ][n] = (real)0;
#pragma unroll
  for (int q = F_JIX; q <= F_NE; ++q) F.f[q][n] = (real)0;
  F.f[F_PHI][n] = (real)0;  // :325
}

struct BParams {
  double temp;   // dt / (4 e0)           (renew_b4_2 :2583)
  double dth;    // dt / 2
  double inv24dx;
};

struct EParams {
  double temp;   // c^2 dt                (renew_e4_2 :2616)
  double mu0;
  double inv24dx;
};

// Damping coefficients of renew_b4_2 at sigma s: ca = (1 - s t)/(1 + s t),
// cb = (dt/2)/(1 + s t); s = 0 gives exactly (1, dt/2) without the divisions.
__device__ __forceinline__ void b_coeffs(double s, const BParams& p, double& ca, double& cb) {
  if (s == 0.0) { ca = 1.0; cb = p.dth; return; }
  ca = (1. - s * p.temp) / (1. + s * p.temp);
  cb = p.dth / (1. + s * p.temp);
}

// Damping coefficients of renew_e4_2 at sigma s: with h = mu0 s t / 2,
// ca = (1 - h)/(1 + h), cb = t/(1 + h); s = 0 gives exactly (1, t).
__device__ __forceinline__ void e_coeffs(double s, const EParams& p, double& ca, double& cb) {
  if (s == 0.0) { ca = 1.0; cb = p.temp; return; }
  const double h = 0.5 * p.mu0 * s * p.temp;
  ca = (1. - h) / (1. + h);
  cb = p.temp / (1. + h);
}

// renew_b4_2 (:2580-2611) on the induced field: DB <- ca DB - cb curl4(E),
// B = B0 + DB, with ca = (1 - s t)/(1 + s t), cb = (dt/2)/(1 + s t).
template <typename real>
__global__ void __launch_bounds__(256) renew_b_kernel(Fields<real> F, Geom g, Ramps rp, BParams p) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int nint = g.nx * g.ny * g.nz;
  if (t >= nint) return;
  const int m = 2 + t % g.nz, l = 2 + (t / g.nz) % g.ny, k = 2 + t / (g.nz * g.ny);
  const int n = k * g.sx + l * g.gz + m;
  const int sy = g.gz, sx = g.sx;
  const real* __restrict__ ex = F.f[F_EX];
  const real* __restrict__ ey = F.f[F_EY];
  const real* __restrict__ ez = F.f[F_EZ];
  const real c24 = (real)p.inv24dx;
  // x component at (k+1/2, l, m): sigma[2k+1][2l][2m]
  {
    const double s = sigma_of(rp.a, rp.rx[2 * k + 1], rp.ry[2 * l], rp.rz[2 * m]);
    double ca, cb;
    b_coeffs(s, p, ca, cb);
    const real curl = ((real)27 * (ez[n] - ez[n - sy] - ey[n] + ey[n - 1]) -
                       (ez[n + sy] - ez[n - 2 * sy] - ey[n + 1] + ey[n - 2])) * c24;
    const real db = (real)ca * F.f[F_DBX][n] - (real)cb * curl;
    F.f[F_DBX][n] = db;
    F.f[F_BX][n] = F.f[F_B0X][n] + db;
  }
  {
    const double s = sigma_of(rp.a, rp.rx[2 * k], rp.ry[2 * l + 1], rp.rz[2 * m]);
    double ca, cb;
    b_coeffs(s, p, ca, cb);
    const real curl = ((real)27 * (ex[n] - ex[n - 1] - ez[n] + ez[n - sx]) -
                       (ex[n + 1] - ex[n - 2] - ez[n + sx] + ez[n - 2 * sx])) * c24;
    const real db = (real)ca * F.f[F_DBY][n] - (real)cb * curl;
    F.f[F_DBY][n] = db;
    F.f[F_BY][n] = F.f[F_B0Y][n] + db;
  }
  {
    const double s = sigma_of(rp.a, rp.rx[2 * k], rp.ry[2 * l], rp.rz[2 * m + 1]);
    double ca, cb;
    b_coeffs(s, p, ca, cb);
    const real curl = ((real)27 * (ey[n] - ey[n - sx] - ex[n] + ex[n - sy]) -
                       (ey[n + sx] - ey[n - 2 * sx] - ex[n + sy] + ex[n - 2 * sy])) * c24;
    const real db = (real)ca * F.f[F_DBZ][n] - (real)cb * curl;
    F.f[F_DBZ][n] = db;
    F.f[F_BZ][n] = F.f[F_B0Z][n] + db;
  }
}

// renew_e4_2 (:2613-2652): E <- ca E + cb (curl4(DB) - mu0 (J_i - J_e)),
// ca = (1 - mu0 s t/2)/(1 + mu0 s t/2), cb = t/(1 + mu0 s t/2), t = c^2 dt.
template <typename real>
__global__ void __launch_bounds__(256) renew_e_kernel(Fields<real> F, Geom g, Ramps rp, EParams p) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int nint = g.nx * g.ny * g.nz;
  if (t >= nint) return;
  const int m = 2 + t % g.nz, l = 2 + (t / g.nz) % g.ny, k = 2 + t / (g.nz * g.ny);
  const int n = k * g.sx + l * g.gz + m;
  const int sy = g.gz, sx = g.sx;
  const real* __restrict__ bx = F.f[F_DBX];
  const real* __restrict__ by = F.f[F_DBY];
  const real* __restrict__ bz = F.f[F_DBZ];
  const real c24 = (real)p.inv24dx;
  const real mu0 = (real)p.mu0;
  {
    const double s = sigma_of(rp.a, rp.rx[2 * k], rp.ry[2 * l + 1], rp.rz[2 * m + 1]);
    double ca, cb;
    e_coeffs(s, p, ca, cb);
    const real curl = ((real)27 * ((bz[n + sy] - bz[n]) - (by[n + 1] - by[n])) -
                       ((bz[n + 2 * sy] - bz[n - sy]) - (by[n + 2] - by[n - 1]))) * c24;
    F.f[F_EX][n] = (real)ca * F.f[F_EX][n] + (real)cb * (curl - mu0 * (F.f[F_JIX][n] - F.f[F_JEX][n]));
  }
  {
    const double s = sigma_of(rp.a, rp.rx[2 * k + 1], rp.ry[2 * l], rp.rz[2 * m + 1]);
    double ca, cb;
    e_coeffs(s, p, ca, cb);
    const real curl = ((real)27 * ((bx[n + 1] - bx[n]) - (bz[n + sx] - bz[n])) -
                       ((bx[n + 2] - bx[n - 1]) - (bz[n + 2 * sx] - bz[n - sx]))) * c24;
    F.f[F_EY][n] = (real)ca * F.f[F_EY][n] + (real)cb * (curl - mu0 * (F.f[F_JIY][n] - F.f[F_JEY][n]));
  }
  {
    const double s = sigma_of(rp.a, rp.rx[2 * k + 1], rp.ry[2 * l + 1], rp.rz[2 * m]);
    double ca, cb;
    e_coeffs(s, p, ca, cb);
    const real curl = ((real)27 * ((by[n + sx] - by[n]) - (bx[n + sy] - bx[n])) -
                       ((by[n + 2 * sx] - by[n - sx]) - (bx[n + 2 * sy] - bx[n - sy]))) * c24;
    F.f[F_EZ][n] = (real)ca * F.f[F_EZ][n] + (real)cb * (curl - mu0 * (F.f[F_JIZ][n] - F.f[F_JEZ][n]));
  }
}

// Up to 8 planes processed by one ghost kernel.
template <typename real>
struct PlaneSet {
  real* p[8];
  int count;
};

// One thread per (plane, ghost layer, in-layer node): the ghost layers are
// thin (two on each side), so the parallelism comes from the planes and the
// layers as well as the nodes. Sources (interior layers 2, 3, N, N+1) and
// targets (ghost layers 0, 1, N+2, N+3) are disjoint for N >= 2, so the
// threads are independent.
__device__ __forceinline__ void ghost_pair(int r, int N, int& dst, int& src) {
  // r: 0, 1 -> ghosts 0, 1 <- N, N+1; 2, 3 -> ghosts N+2, N+3 <- 2, 3
  dst = r < 2 ? r : N + r;
  src = r < 2 ? N + r : r;
}

// Offset of node e of layer `layer` of an x pass (a whole k plane) or of a y
// pass (row l of every k plane, ghosts included).
__device__ __forceinline__ long long layer_node(const Geom& g, int axis, int layer, int e) {
  if (axis == 0) return (long long)layer * g.sx + e;
  return (long long)(e / g.gz) * g.sx + (long long)layer * g.gz + e % g.gz;
}

// sr_b / sr_e at size 1: x pass (:1016-1101) then y pass (:1103-1190);
// ghosts 0,1 <- N, N+1 and N+2, N+3 <- 2, 3.
template <typename real>
__global__ void wrap_kernel(PlaneSet<real> s, Geom g, int axis) {
  const int per = axis == 0 ? g.gy * g.gz : g.gx * g.gz;
  const int N = axis == 0 ? g.nx : g.ny;
  const long long total = (long long)s.count * 4 * per;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(t / (4LL * per)), r = (int)((t / per) % 4), e = (int)(t % per);
    int dst, src;
    ghost_pair(r, N, dst, src);
    real* a = s.p[q];
    a[layer_node(g, axis, dst, e)] = a[layer_node(g, axis, src, e)];
  }
}

// sr_b at size 1 on the total field (:1016-1190): the ghost planes of B get the
// periodic images of B, while B0 keeps its own (non-periodic) dipole values, so
// the induced field there is B_image - B0_ghost, which the E update then sees.
template <typename real>
__global__ void wrap_b_kernel(Fields<real> F, Geom g, int axis) {
  const int per = axis == 0 ? g.gy * g.gz : g.gx * g.gz;
  const int N = axis == 0 ? g.nx : g.ny;
  const long long total = 3LL * 4 * per;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(t / (4LL * per)), r = (int)((t / per) % 4), e = (int)(t % per);
    int dst, src;
    ghost_pair(r, N, dst, src);
    const long long d = layer_node(g, axis, dst, e);
    const real v = F.f[F_BX + q][layer_node(g, axis, src, e)];
    F.f[F_BX + q][d] = v;
    F.f[F_DBX + q][d] = v - F.f[F_B0X + q][d];
  }
}

// sr_current2 at size 1: x pass (:1815-1935), then y pass over every k
// including the x ghosts (:1937-2036); layers 2,3 += N+2, N+3 and
// N, N+1 += 0, 1 (the sources are ghosts, the targets interior).
template <typename real>
__global__ void fold_kernel(PlaneSet<real> s, Geom g, int axis) {
  const int per = axis == 0 ? g.gy * g.gz : g.gx * g.gz;
  const int N = axis == 0 ? g.nx : g.ny;
  const long long total = (long long)s.count * 4 * per;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(t / (4LL * per)), r = (int)((t / per) % 4), e = (int)(t % per);
    int ghost, target;
    ghost_pair(r, N, ghost, target);  // the wrap's targets are the fold's sources
    real* a = s.p[q];
    a[layer_node(g, axis, target, e)] += a[layer_node(g, axis, ghost, e)];
  }
}

}  // namespace pb
