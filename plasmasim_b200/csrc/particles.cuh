// Particle kernels: push with field gather, current and density deposits,
// boundary removal/wrap, initial load and boundary injection, cell sort.
#pragma once

#include "common.cuh"

namespace pb {

// ------------------------------------------------------------------ shapes
// Per-axis linear weights of shape_func_v2 (PIC/3d_pic458_domain.c:3104-3139)
// in cell units for a coordinate (i, f), x = (i + f) dx:
//  node-aligned components: base i,  weights (1 - f, f)
//  half-shifted components: base (int)(x/dx - 0.5), i.e. i - 1 for f < 1/2
//  (i itself for f >= 1/2, and for i == 0 where the cast truncates toward 0),
//  weights (1 - p, p) with p = x/dx - (base + 1/2).
template <typename real>
struct Axis {
  int a, b;          // node-aligned and half-shifted base index
  real a0, a1, b0, b1;
};

template <typename real>
__device__ __forceinline__ Axis<real> axis_weights(int i, real f) {
  Axis<real> w;
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
__device__ __forceinline__ real ldg(const real* p) { return __ldg(p); }

// Trilinear interpolation of one plane from the 2x2x2 nodes at base n.
template <typename real>
__device__ __forceinline__ real trilerp(const real* __restrict__ F, int n, int sx, int sy,
                                        real x0, real x1, real y0, real y1, real z0, real z1) {
  const real c00 = ldg(F + n) * z0 + ldg(F + n + 1) * z1;
  const real c01 = ldg(F + n + sy) * z0 + ldg(F + n + sy + 1) * z1;
  const real c10 = ldg(F + n + sx) * z0 + ldg(F + n + sx + 1) * z1;
  const real c11 = ldg(F + n + sx + sy) * z0 + ldg(F + n + sx + sy + 1) * z1;
  return (c00 * y0 + c01 * y1) * x0 + (c10 * y0 + c11 * y1) * x1;
}

// Area-weighted scatter of v onto the 2x2x2 nodes at base n.
template <typename real>
__device__ __forceinline__ void scatter8(real* F, int n, int sx, int sy, real v,
                                         real x0, real x1, real y0, real y1, real z0, real z1) {
  const real a0 = v * x0, a1 = v * x1;
  const real a00 = a0 * y0, a01 = a0 * y1, a10 = a1 * y0, a11 = a1 * y1;
  atomicAdd(F + n, a00 * z0);
  atomicAdd(F + n + 1, a00 * z1);
  atomicAdd(F + n + sy, a01 * z0);
  atomicAdd(F + n + sy + 1, a01 * z1);
  atomicAdd(F + n + sx, a10 * z0);
  atomicAdd(F + n + sx + 1, a10 * z1);
  atomicAdd(F + n + sx + sy, a11 * z0);
  atomicAdd(F + n + sx + sy + 1, a11 * z1);
}

template <typename real>
struct Gathered {
  real ex, ey, ez, bx, by, bz;
};

// shape_func_v2 (:3017-3326): E and B at (i,f), each on its own stagger.
template <typename real>
__device__ __forceinline__ Gathered<real> gather6(const Fields<real>& F, const Geom& g,
                                                  const Axis<real>& X, const Axis<real>& Y,
                                                  const Axis<real>& Z) {
  const int sx = g.sx, sy = g.gz;
  Gathered<real> r;
  // ex (k, l+1/2, m+1/2): x aligned, y and z shifted
  r.ex = trilerp(F.f[F_EX], X.a * sx + Y.b * sy + Z.b, sx, sy, X.a0, X.a1, Y.b0, Y.b1, Z.b0, Z.b1);
  // ey (k+1/2, l, m+1/2)
  r.ey = trilerp(F.f[F_EY], X.b * sx + Y.a * sy + Z.b, sx, sy, X.b0, X.b1, Y.a0, Y.a1, Z.b0, Z.b1);
  // ez (k+1/2, l+1/2, m)
  r.ez = trilerp(F.f[F_EZ], X.b * sx + Y.b * sy + Z.a, sx, sy, X.b0, X.b1, Y.b0, Y.b1, Z.a0, Z.a1);
  // bx (k+1/2, l, m)
  r.bx = trilerp(F.f[F_BX], X.b * sx + Y.a * sy + Z.a, sx, sy, X.b0, X.b1, Y.a0, Y.a1, Z.a0, Z.a1);
  // by (k, l+1/2, m)
  r.by = trilerp(F.f[F_BY], X.a * sx + Y.b * sy + Z.a, sx, sy, X.a0, X.a1, Y.b0, Y.b1, Z.a0, Z.a1);
  // bz (k, l, m+1/2)
  r.bz = trilerp(F.f[F_BZ], X.a * sx + Y.a * sy + Z.b, sx, sy, X.a0, X.a1, Y.a0, Y.a1, Z.b0, Z.b1);
  return r;
}

// Particle t's records, read with vector loads.
template <typename real>
struct Rec {
  int cell;
  real o[3];
  real v[3];
};
__device__ __forceinline__ Rec<float> load_records(const Parts<float>& P, long long t) {
  const float4 a = reinterpret_cast<const float4*>(P.ra)[t];
  const float4 b = reinterpret_cast<const float4*>(P.rb)[t];
  return Rec<float>{__float_as_int(a.x), {a.y, a.z, a.w}, {b.x, b.y, b.z}};
}
__device__ __forceinline__ Rec<double> load_records(const Parts<double>& P, long long t) {
  const double2* a = reinterpret_cast<const double2*>(P.ra + 4 * t);
  const double2* b = reinterpret_cast<const double2*>(P.rb + 4 * t);
  const double2 a0 = a[0], a1 = a[1], b0 = b[0], b1 = b[1];
  return Rec<double>{__double2loint(a0.x), {a0.y, a1.x, a1.y}, {b0.x, b0.y, b1.x}};
}

// Particle t's records, written with vector stores.
__device__ __forceinline__ void store_records(const Parts<float>& P, long long t, int c, float fx, float fy,
                                              float fz, float vx, float vy, float vz) {
  reinterpret_cast<float4*>(P.ra)[t] = make_float4(__int_as_float(c), fx, fy, fz);
  reinterpret_cast<float4*>(P.rb)[t] = make_float4(vx, vy, vz, 0.f);
}
__device__ __forceinline__ void store_records(const Parts<double>& P, long long t, int c, double fx, double fy,
                                              double fz, double vx, double vy, double vz) {
  double2* a = reinterpret_cast<double2*>(P.ra + 4 * t);
  double2* b = reinterpret_cast<double2*>(P.rb + 4 * t);
  a[0] = make_double2(__hiloint2double(0, c), fx);
  a[1] = make_double2(fy, fz);
  b[0] = make_double2(vx, vy);
  b[1] = make_double2(vz, 0.0);
}
// Particle s of S to slot d of D with cell index c: two vector copies.
__device__ __forceinline__ void copy_record(const Parts<float>& S, long long s, const Parts<float>& D, long long d,
                                            int c) {
  float4 a = reinterpret_cast<const float4*>(S.ra)[s];
  a.x = __int_as_float(c);
  reinterpret_cast<float4*>(D.ra)[d] = a;
  reinterpret_cast<float4*>(D.rb)[d] = reinterpret_cast<const float4*>(S.rb)[s];
}
__device__ __forceinline__ void copy_record(const Parts<double>& S, long long s, const Parts<double>& D,
                                            long long d, int c) {
  const double2* a = reinterpret_cast<const double2*>(S.ra + 4 * s);
  const double2* b = reinterpret_cast<const double2*>(S.rb + 4 * s);
  double2 a0 = a[0];
  const double2 a1 = a[1], b0 = b[0], b1 = b[1];
  a0.x = __hiloint2double(0, c);
  double2* da = reinterpret_cast<double2*>(D.ra + 4 * d);
  double2* db = reinterpret_cast<double2*>(D.rb + 4 * d);
  da[0] = a0;
  da[1] = a1;
  db[0] = b0;
  db[1] = b1;
}

// sr_particle's packets between ranks: one record per particle, in the
// sending rank's cell indices (the receiver shifts them, :2374-2380).
template <typename real>
struct MigRec {
  int cell;
  int pad;
  real o[3];
  real v[3];
};

// Where the push writes the particles that leave a rank's x-y interior in a
// decomposed run; count is null for a single domain.
template <typename real>
struct Outbox {
  int* count;
  int cap;
  MigRec<real>* rec;
};

template <typename real>
struct PushConst {
  real T;               // 0.5 q dt / m, m < 0 for electrons (cal_track4 :2812)
  real C, C2;           // C, C*C
  real hdt;             // 0.5 dt / dx: cells moved per unit velocity in half a step
  real qn;              // q n: current per unit velocity and unit weight
  real nw;              // n: density per unit weight
  real ex_add, ey_add;  // V*IMF_y, -V*IMF_x (:2817-2818)
  // ballistic region of fdtd (:642-647) in this rank's cell indices:
  // Absorb_grid2 - offset below, N_global + 4 - Absorb_grid2 - offset above
  int bal_lx, bal_ly, bal_lz;
  int bal_hx, bal_hy, bal_hz;
  int bal_interior;            // the ballistic region reaches an interior cell of this rank
  int pjx, pjy, pjz, pn;       // deposit planes of this species
  Outbox<real> out;            // decomposed runs: particles leaving the rank's x-y interior
};

// cal_track4 (:2804-2870) velocity update; returns the new velocity in v.
template <typename real>
__device__ __forceinline__ void boris4(const PushConst<real>& pc, Gathered<real> e, real& vx,
                                       real& vy, real& vz) {
  const real T = pc.T, C = pc.C;
  e.ex += pc.ex_add;
  e.ey += pc.ey_add;
  real g1 = C / sqrt(pc.C2 - vx * vx - vy * vy - vz * vz);
  if (isnan(g1)) g1 = (real)0;
  real ux = g1 * vx, uy = g1 * vy, uz = g1 * vz;
  real g2 = C / sqrt(pc.C2 + ux * ux + uy * uy + uz * uz);
  const real bux = g2 * e.bx, buy = g2 * e.by, buz = g2 * e.bz;
  const real S = (real)2 * T / ((real)1 + T * T * (bux * bux + buy * buy + buz * buz));
  ux += e.ex * T;
  uy += e.ey * T;
  uz += e.ez * T;
  const real uox = ux + T * (uy * buz - uz * buy);
  const real uoy = uy + T * (uz * bux - ux * buz);
  const real uoz = uz + T * (ux * buy - uy * bux);
  real upx = ux + S * (uoy * buz - uoz * buy);
  real upy = uy + S * (uoz * bux - uox * buz);
  real upz = uz + S * (uox * buy - uoy * bux);
  upx += e.ex * T;
  upy += e.ey * T;
  upz += e.ez * T;
  g2 = C / sqrt(pc.C2 + upx * upx + upy * upy + upz * upz);
  vx = g2 * upx;
  vy = g2 * upy;
  vz = g2 * upz;
}

// True when the particle lies outside the Absorb_grid2 box (fdtd :733-735):
// x < ax0 or x > ax1 on any axis.
template <typename real>
__device__ __forceinline__ bool ballistic(const PushConst<real>& pc, int i, int j, int k, real fx,
                                          real fy, real fz) {
  return i < pc.bal_lx || j < pc.bal_ly || k < pc.bal_lz ||
         i > pc.bal_hx || (i == pc.bal_hx && fx > (real)0) ||
         j > pc.bal_hy || (j == pc.bal_hy && fy > (real)0) ||
         k > pc.bal_hz || (k == pc.bal_hz && fz > (real)0);
}

// The 2x2x2 stencil of (i, j, k) lies in the padded array; the reference's
// deposit condition 0 <= x < (N+4) dx (:747-749) also admits i = N+3, whose
// stencil leaves the array, and such deposits are counted instead of made.
__device__ __forceinline__ bool stencil_ok(const Geom& g, int i, int j, int k) {
  return i >= 0 && j >= 0 && k >= 0 && i <= g.gx - 2 && j <= g.gy - 2 && k <= g.gz - 2;
}
__device__ __forceinline__ bool in_array(const Geom& g, int i, int j, int k) {
  return i >= 0 && j >= 0 && k >= 0 && i < g.gx && j < g.gy && k < g.gz;
}

// shape_func_*0_j_2 (:3397-3553) at (i,f) with velocity v.
template <typename real>
__device__ __forceinline__ void deposit_j(const Fields<real>& F, const Geom& g,
                                          const PushConst<real>& pc, const Axis<real>& X,
                                          const Axis<real>& Y, const Axis<real>& Z, real vx,
                                          real vy, real vz) {
  const int sx = g.sx, sy = g.gz;
  scatter8(F.f[pc.pjx], X.a * sx + Y.b * sy + Z.b, sx, sy, pc.qn * vx, X.a0, X.a1, Y.b0, Y.b1, Z.b0, Z.b1);
  scatter8(F.f[pc.pjy], X.b * sx + Y.a * sy + Z.b, sx, sy, pc.qn * vy, X.b0, X.b1, Y.a0, Y.a1, Z.b0, Z.b1);
  scatter8(F.f[pc.pjz], X.b * sx + Y.b * sy + Z.a, sx, sy, pc.qn * vz, X.b0, X.b1, Y.b0, Y.b1, Z.a0, Z.a1);
}

// shape_func_*0_n_2 (:3333-3395): cell-centred density.
template <typename real>
__device__ __forceinline__ void deposit_n(const Fields<real>& F, const Geom& g,
                                          const PushConst<real>& pc, const Axis<real>& X,
                                          const Axis<real>& Y, const Axis<real>& Z) {
  const int sx = g.sx, sy = g.gz;
  scatter8(F.f[pc.pn], X.b * sx + Y.b * sy + Z.b, sx, sy, pc.nw, X.b0, X.b1, Y.b0, Y.b1, Z.b0, Z.b1);
}

__device__ __forceinline__ void count_err(unsigned long long* err, int id) {
  atomicAdd(err + id, 1ull);
}

// Repacks (i,j,k) or marks the slot empty when the cell is not representable.
__device__ __forceinline__ int repack(int i, int j, int k, unsigned long long* err) {
  if (i < 0 || j < 0 || k < 0 || i >= kMaxDim || j >= kMaxDim || k >= kMaxDim) {
    count_err(err, ERR_CELL_RANGE);
    return -1;
  }
  return pack_cell(i, j, k);
}

// sr_particle at size 1 (:2058-2250): returns false when the particle is
// removed; wraps x (then y) crossers by -N cells.
__device__ __forceinline__ bool boundary(const Geom& g, int& i, int& j, int k) {
  if (k < 2 || k >= g.nz + 2) return false;  // z outside [2dx, (Nz+2)dx)
  if (i < 2) return false;                    // backward x packet dropped on rank 0
  if (i >= g.nx + 2) i -= g.nx;               // forward x packet sent to itself
  if (j < 2) return false;
  if (j >= g.ny + 2) j -= g.ny;
  return true;
}

// The slot's cell after sr_particle. A single domain applies `boundary`. A
// decomposed run keeps particles inside the rank's x-y interior, deletes
// those outside z (:2067-2104), and writes the rest to the outbox as packets
// for the exchange between ranks, leaving the slot empty.
template <typename real>
__device__ __forceinline__ int settle(const Geom& g, const Outbox<real>& ob, int i, int j, int k, real fx, real fy,
                                      real fz, real vx, real vy, real vz, unsigned long long* err) {
  if (!ob.count) return boundary(g, i, j, k) ? repack(i, j, k, err) : -1;
  if (k < 2 || k >= g.nz + 2) return -1;
  if (i >= 2 && i < g.nx + 2 && j >= 2 && j < g.ny + 2) return repack(i, j, k, err);
  const int c = repack(i, j, k, err);
  if (c < 0) return -1;
  const int q = atomicAdd(ob.count, 1);
  if (q < ob.cap) {
    MigRec<real> r;
    r.cell = c;
    r.pad = 0;
    r.o[0] = fx; r.o[1] = fy; r.o[2] = fz;
    r.v[0] = vx; r.v[1] = vy; r.v[2] = vz;
    ob.rec[q] = r;
  } else {
    count_err(err, ERR_MIGRATION);
  }
  return -1;
}

enum PushMode { PUSH_J = 0, PUSH_FUSED = 1 };

// The particle part of one fdtd iteration for one species.
//  PUSH_J:     :731-812 only (push, J deposit at x^{n+1/2}).
//  PUSH_FUSED: :731-812, then :818-867 (drift to x^{n+1}, density deposit) and
//              sr_particle, in one pass over the particle arrays. Neither the
//              drift, the density deposit nor the removal reads a field, so the
//              second B half-step that the reference runs between them changes
//              nothing they compute.
template <typename real, int MODE>
__global__ void __launch_bounds__(256) push_kernel(Parts<real> P, int first, const int* __restrict__ count,
                                                   Fields<real> F, Geom g, PushConst<real> pc,
                                                   unsigned long long* err) {
  const int n = *count;
  unsigned pushed = 0;
  for (int t = first + blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const Rec<real> r = load_records(P, t);
    if (r.cell < 0) continue;
    ++pushed;
    int i, j, k;
    unpack_cell(r.cell, i, j, k);
    real fx = r.o[0], fy = r.o[1], fz = r.o[2];
    real vx = r.v[0], vy = r.v[1], vz = r.v[2];
    bool bal = ballistic(pc, i, j, k, fx, fy, fz);
    if (!bal && !stencil_ok(g, i, j, k)) {
      count_err(err, ERR_DEPOSIT_OOB);
      bal = true;
    }
    if (!bal) {
      const Axis<real> X = axis_weights(i, fx), Y = axis_weights(j, fy), Z = axis_weights(k, fz);
      boris4(pc, gather6(F, g, X, Y, Z), vx, vy, vz);
      if (!(isfinite(vx) && isfinite(vy) && isfinite(vz))) count_err(err, ERR_NONFINITE);
    }
    advance(i, fx, vx * pc.hdt);
    advance(j, fy, vy * pc.hdt);
    advance(k, fz, vz * pc.hdt);
    if (in_array(g, i, j, k)) {
      if (stencil_ok(g, i, j, k)) {
        const Axis<real> X = axis_weights(i, fx), Y = axis_weights(j, fy), Z = axis_weights(k, fz);
        deposit_j(F, g, pc, X, Y, Z, vx, vy, vz);
      } else {
        count_err(err, ERR_DEPOSIT_OOB);
      }
    }
    int cell;
    if (MODE == PUSH_FUSED) {
      advance(i, fx, vx * pc.hdt);
      advance(j, fy, vy * pc.hdt);
      advance(k, fz, vz * pc.hdt);
      if (in_array(g, i, j, k)) {
        if (stencil_ok(g, i, j, k)) {
          const Axis<real> X = axis_weights(i, fx), Y = axis_weights(j, fy), Z = axis_weights(k, fz);
          deposit_n(F, g, pc, X, Y, Z);
        } else {
          count_err(err, ERR_DEPOSIT_OOB);
        }
      }
      cell = settle(g, pc.out, i, j, k, fx, fy, fz, vx, vy, vz, err);
    } else {
      cell = repack(i, j, k, err);
    }
    store_records(P, t, cell, fx, fy, fz, vx, vy, vz);
  }
  // particle pushes of this warp, one atomic per warp
  for (int o = 16; o > 0; o >>= 1) pushed += __shfl_down_sync(0xffffffffu, pushed, o);
  if ((threadIdx.x & 31) == 0 && pushed) atomicAdd(err + CNT_PUSHED, (unsigned long long)pushed);
}

// Drift to x^{n+1} and density deposit (fdtd :818-867).
template <typename real>
__global__ void __launch_bounds__(256) drift_n_kernel(Parts<real> P, const int* __restrict__ count,
                                                      Fields<real> F, Geom g, PushConst<real> pc,
                                                      unsigned long long* err) {
  const int n = *count;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int c = P.cell[t];
    if (c < 0) continue;
    int i, j, k;
    unpack_cell(c, i, j, k);
    real fx = P.o[0][t], fy = P.o[1][t], fz = P.o[2][t];
    const real vx = P.v[0][t], vy = P.v[1][t], vz = P.v[2][t];
    advance(i, fx, vx * pc.hdt);
    advance(j, fy, vy * pc.hdt);
    advance(k, fz, vz * pc.hdt);
    if (in_array(g, i, j, k)) {
      if (stencil_ok(g, i, j, k)) {
        const Axis<real> X = axis_weights(i, fx), Y = axis_weights(j, fy), Z = axis_weights(k, fz);
        deposit_n(F, g, pc, X, Y, Z);
      } else {
        count_err(err, ERR_DEPOSIT_OOB);
      }
    }
    P.cell[t] = repack(i, j, k, err);
    P.o[0][t] = fx; P.o[1][t] = fy; P.o[2][t] = fz;
  }
}

// sr_particle at size 1 on its own.
template <typename real>
__global__ void sr_particle_kernel(Parts<real> P, const int* __restrict__ count, Geom g, Outbox<real> ob,
                                   unsigned long long* err) {
  const int n = *count;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int c = P.cell[t];
    if (c < 0) continue;
    int i, j, k;
    unpack_cell(c, i, j, k);
    P.cell[t] = settle(g, ob, i, j, k, P.o[0][t], P.o[1][t], P.o[2][t], P.v[0][t], P.v[1][t], P.v[2][t], err);
  }
}

// Shell deletion of add_*_flat (:6015-6031): x < 4dx on the rank of the
// global low x face, x > Nx dx on the rank of the high face, the same in y;
// z < 4dx or z > Nz dx everywhere (at size 1 the one rank holds every face).
// Whether the particle in slot t (cell c) lies in such a shell.
template <typename real>
__device__ __forceinline__ bool in_refill_shell(const Parts<real>& P, const Geom& g, int c, long long t) {
  int i, j, k;
  unpack_cell(c, i, j, k);
  const bool xl = g.xlo && i < 4, yl = g.ylo && j < 4;
  const bool xh = g.xhi && (i > g.nx || (i == g.nx && P.o[0][t] > (real)0));
  const bool yh = g.yhi && (j > g.ny || (j == g.ny && P.o[1][t] > (real)0));
  const bool zs = k < 4 || k > g.nz || (k == g.nz && P.o[2][t] > (real)0);
  return xl || yl || xh || yh || zs;
}

template <typename real>
__global__ void delete_shell_kernel(Parts<real> P, int first, const int* __restrict__ count, Geom g) {
  const int n = *count;
  for (int t = first + blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int c = P.cell[t];
    if (c >= 0 && in_refill_shell(P, g, c, t)) P.cell[t] = -1;
  }
}

// --------------------------------------------------------------- sources
// A refill slab of add_*_flat: cells [k0, k0+nk) x [l0, l0+nl) x [m0, m0+nm),
// k outermost, Np particles per cell (the loop nest of :6047-6071).
struct Slab {
  int k0, nk, l0, nl, m0, nm;
  long long first;  // index of the slab's first particle in the call's sequence
};

struct SourceParams {
  int nslab;
  Slab slab[5];
  int np;
  long long total;        // particles generated by this call
  double dx;
  double lsig;            // sqrt(sigma0^2): Cholesky factor of the covariance (:7943-7953)
  double vdrift;          // mu[2] = V
  uint64_t seed_p, seed_v;
  long long base_p, base_v;  // first draw index on each stream
  int dst;                // first slot written
  const int* dst_dev;     // when set, the first slot is *dst_dev (a count known only on the device)
  int cap;                // when set, slots from cap on are not written (counted as ERR_STORE_FULL)
  int init_form;          // 1: cell bounds as init_particle_flat writes them, 2dx + k dx (:475)
};

// Positions: three gsl_ran_flat draws (x, y, z) on the position stream;
// velocities: ran_multivar_gaussian = three Box-Muller normals (two draws
// each) on the velocity stream, scaled by the Cholesky factor, plus mu.
// Particle t of the call's sequence, in absolute cell cc, written to slot dst.
template <typename real>
__device__ __forceinline__ void make_particle(const Parts<real>& P, const SourceParams& sp, long long t,
                                              const int (&cc)[3], int dst, unsigned long long* err) {
  const double dx = sp.dx;
  const uint64_t dp = (uint64_t)(sp.base_p + 3 * t);
  double lo[3], hi[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (sp.init_form) {  // 2.*dx + k*dx with k counted from the first interior cell
      lo[a] = __dadd_rn(__dmul_rn(2.0, dx), __dmul_rn((double)(cc[a] - 2), dx));
      hi[a] = __dadd_rn(__dmul_rn(2.0, dx), __dmul_rn((double)(cc[a] - 1), dx));
    } else {             // (k+2)*dx as add_*_flat writes it (:6049)
      lo[a] = __dmul_rn((double)cc[a], dx);
      hi[a] = __dmul_rn((double)(cc[a] + 1), dx);
    }
  }
  double up[3], uv[6];  // the particle's 3 position and 6 velocity draws
  uniform53_run<3>(sp.seed_p, dp, up);
  const double x = flat_rn(lo[0], hi[0], up[0]);
  const double y = flat_rn(lo[1], hi[1], up[1]);
  const double z = flat_rn(lo[2], hi[2], up[2]);
  const uint64_t dv = (uint64_t)(sp.base_v + 6 * t);
  uniform53_run<6>(sp.seed_v, dv, uv);
  real vx, vy, vz;
  if (sizeof(real) == 8) {  // the host's arithmetic, rounded step by step
    const double g0 = gauss_bm_u(uv[0], uv[1]), g1 = gauss_bm_u(uv[2], uv[3]), g2 = gauss_bm_u(uv[4], uv[5]);
    vx = (real)__dadd_rn(__dmul_rn(sp.lsig, g0), 0.0);
    vy = (real)__dadd_rn(__dmul_rn(sp.lsig, g1), 0.0);
    vz = (real)__dadd_rn(__dmul_rn(sp.lsig, g2), sp.vdrift);
  } else {  // the same draws through FP32 log/cos: the FP32 state's own precision
    const float ls = (float)sp.lsig;
    vx = (real)(ls * gauss_bm_f32_u(uv[0], uv[1]));
    vy = (real)(ls * gauss_bm_f32_u(uv[2], uv[3]));
    vz = (real)(ls * gauss_bm_f32_u(uv[4], uv[5]) + (float)sp.vdrift);
  }
  int ci, cj, ck;
  real fx, fy, fz;
  split_coord<real>(x / dx, ci, fx);
  split_coord<real>(y / dx, cj, fy);
  split_coord<real>(z / dx, ck, fz);
  P.cell[dst] = repack(ci, cj, ck, err);
  P.o[0][dst] = fx; P.o[1][dst] = fy; P.o[2][dst] = fz;
  P.v[0][dst] = vx; P.v[1][dst] = vy; P.v[2][dst] = vz;
}

// Sequence number of the particles of absolute cell (i, j, k) in slab sl (the
// first of its np), or -1 when the slab does not cover the cell.
__device__ __forceinline__ long long slab_first(const Slab& sl, int np, int i, int j, int k) {
  const int a = i - sl.k0, b = j - sl.l0, c = k - sl.m0;
  if (a < 0 || b < 0 || c < 0 || a >= sl.nk || b >= sl.nl || c >= sl.nm) return -1;
  return sl.first + ((long long)((long long)a * sl.nl + b) * sl.nm + c) * np;
}

// Particles the slabs put into absolute cell (i, j, k).
__device__ __forceinline__ int slab_need(const SourceParams& sp, int i, int j, int k) {
  int n = 0;
  for (int s = 0; s < sp.nslab; ++s)
    if (slab_first(sp.slab[s], sp.np, i, j, k) >= 0) n += sp.np;
  return n;
}

// The call's particles, one thread each, into slots [dst, dst + total).
template <typename real>
__global__ void source_kernel(Parts<real> P, SourceParams sp, unsigned long long* err) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= sp.total) return;
  int s = 0;
  while (s + 1 < sp.nslab && t >= sp.slab[s + 1].first) ++s;
  const Slab& sl = sp.slab[s];
  long long r = t - sl.first;
  r /= sp.np;
  const int m = (int)(r % sl.nm);
  r /= sl.nm;
  const int l = (int)(r % sl.nl);
  const int k = (int)(r / sl.nl);
  const int cc[3] = {k + sl.k0, l + sl.l0, m + sl.m0};
  const long long d = (long long)(sp.dst_dev ? *sp.dst_dev : sp.dst) + t;
  if (sp.cap && d >= sp.cap) {
    count_err(err, ERR_STORE_FULL);
    return;
  }
  make_particle(P, sp, t, cc, (int)d, err);
}

// ------------------------------------------------------------------- sort
// sorting (:7475-7590): counting sort by interior cell, (i, j, k) order with k
// fastest; particles outside the interior are dropped as the reference does.
__device__ __forceinline__ int interior_key(const Geom& g, int c) {
  if (c < 0) return -1;
  int i, j, k;
  unpack_cell(c, i, j, k);
  i -= 2; j -= 2; k -= 2;
  if (i < 0 || j < 0 || k < 0 || i >= g.nx || j >= g.ny || k >= g.nz) return -1;
  return (i * g.ny + j) * g.nz + k;
}

// Adds one to counter[key] per lane, one atomic per distinct key in the warp;
// returns the lane's rank among lanes with the same key plus the prior value.
__device__ __forceinline__ int warp_aggregated_inc(int* counter, int key, bool active) {
  const unsigned mask = __ballot_sync(0xffffffffu, active);
  int base = 0;
  if (active) {
    const unsigned peers = __match_any_sync(mask, key);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    const int rank = __popc(peers & ((1u << lane) - 1u));
    int old = 0;
    if (lane == leader) old = atomicAdd(counter + key, __popc(peers));
    old = __shfl_sync(peers, old, leader);
    base = old + rank;
  }
  return base;
}

// ------------------------------------------------------- scan (exclusive)
// Block-wise exclusive scan of in[0..n) (4 items per thread, 1024 threads),
// block totals to sums[]; a second level scans the totals.
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

static __global__ void __launch_bounds__(kScanThreads) scan_tile_kernel(const int* __restrict__ in, int* out,
                                                                 int* sums, long long n) {
  __shared__ int warp_tot[32];
  const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
  int v[kScanItems];
  int s = 0;
#pragma unroll
  for (int q = 0; q < kScanItems; ++q) {
    v[q] = (base + q < n) ? in[base + q] : 0;
    s += v[q];
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int incl = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_tot[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    int w = warp_tot[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    warp_tot[lane] = w;
  }
  __syncthreads();
  int run = incl - s + (wid > 0 ? warp_tot[wid - 1] : 0);
#pragma unroll
  for (int q = 0; q < kScanItems; ++q) {
    if (base + q < n) out[base + q] = run;
    run += v[q];
  }
  if (threadIdx.x == kScanThreads - 1) sums[blockIdx.x] = run;
}

static __global__ void scan_add_kernel(int* out, const int* __restrict__ add, long long n) {
  const long long base = (long long)blockIdx.x * kScanTile;
  const int a = add[blockIdx.x];
  for (int q = threadIdx.x; q < kScanTile; q += blockDim.x) {
    if (base + q < n) out[base + q] += a;
  }
}

// -------------------------------------------------------- import / export
// Device-side compaction of live slots for export: flags -> scan -> rows.
template <typename real>
__global__ void live_flag_kernel(Parts<real> P, int n, int* flag) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) flag[t] = P.cell[t] >= 0 ? 1 : 0;
}

template <typename real>
__global__ void export_rows_kernel(Parts<real> P, int n, const int* __restrict__ pos, double dx,
                                   double weight, double* rows) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int c = P.cell[t];
  if (c < 0) return;
  int i, j, k;
  unpack_cell(c, i, j, k);
  double* r = rows + 7 * (long long)pos[t];
  r[0] = ((double)i + (double)P.o[0][t]) * dx;
  r[1] = ((double)j + (double)P.o[1][t]) * dx;
  r[2] = ((double)k + (double)P.o[2][t]) * dx;
  r[3] = (double)P.v[0][t];
  r[4] = (double)P.v[1][t];
  r[5] = (double)P.v[2][t];
  r[6] = weight;
}

// Rows that pic_set_particles refuses: a weight other than the species' n
// (:83-84) or a flag other than 1 (the only value the reference assigns,
// :510); counted, so that the caller can reject the import before it
// changes the store.
static __global__ void import_check_kernel(const double* __restrict__ rows, long long n, double w, double tol,
                                           const int* __restrict__ flag, unsigned long long* bad) {
  unsigned long long nb = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    nb += (fabs(rows[7 * i + 6] - w) > tol || (flag && flag[i] != 1)) ? 1 : 0;
  for (int o = 16; o > 0; o >>= 1) nb += __shfl_down_sync(0xffffffffu, nb, o);
  if ((threadIdx.x & 31) == 0 && nb) atomicAdd(bad, nb);
}

template <typename real>
__global__ void import_rows_kernel(Parts<real> P, int n, const double* __restrict__ rows,
                                   double dx, unsigned long long* err) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double* r = rows + 7 * (long long)t;
  int i, j, k;
  real fx, fy, fz;
  split_coord<real>(r[0] / dx, i, fx);
  split_coord<real>(r[1] / dx, j, fy);
  split_coord<real>(r[2] / dx, k, fz);
  P.cell[t] = repack(i, j, k, err);
  P.o[0][t] = fx; P.o[1][t] = fy; P.o[2][t] = fz;
  P.v[0][t] = (real)r[3]; P.v[1][t] = (real)r[4]; P.v[2][t] = (real)r[5];
}

}  // namespace pb
