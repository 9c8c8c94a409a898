// Discrete adjoint of the time step (push + gather, J deposit, drift,
// sr_particle, the 4th-order B and E updates with their ghost copies and
// folds) for the gradient of the impulse delivered to the dipole with respect
// to the coil current I (the dipole moment is mu0 I pi R^2) and the solar-wind
// drift V. No reference counterpart: the reference has no derivatives.
//
// Objective: J = sum over steps of dt * F, F = -sum_p s_p q n dx^3 (v x B0(x))_z
// over the particles alive after sr_particle (s_p = +1 ions, -1 electrons),
// with B0 gathered by the shape functions of B: the reaction to the Lorentz
// force of the dipole's own field on the plasma.
//
// Conventions: positions are in cell units (xi = x / dx); lambda arrays hold
// dJ/d(state). Every adjoint kernel is the transpose of the forward kernel
// named in its comment, written in gather form where the forward is a stencil.
#pragma once

#include "common.cuh"
#include "diag.cuh"
#include "fields.cuh"
#include "particles.cuh"

namespace pb {

// Value and gradient (per cell along x, y, z) of the trilinear interpolant of
// plane F on the 2x2x2 nodes at base n.
template <typename real>
struct VG {
  real v, gx, gy, gz;
};

template <typename real>
__device__ __forceinline__ VG<real> trilerp_vg(const real* __restrict__ F, int n, int sx, int sy, real x0,
                                               real x1, real y0, real y1, real z0, real z1) {
  const real f000 = F[n], f001 = F[n + 1], f010 = F[n + sy], f011 = F[n + sy + 1];
  const real f100 = F[n + sx], f101 = F[n + sx + 1], f110 = F[n + sx + sy], f111 = F[n + sx + sy + 1];
  const real c00 = f000 * z0 + f001 * z1, c01 = f010 * z0 + f011 * z1;
  const real c10 = f100 * z0 + f101 * z1, c11 = f110 * z0 + f111 * z1;
  const real e0 = c00 * y0 + c01 * y1, e1 = c10 * y0 + c11 * y1;
  VG<real> r;
  r.v = e0 * x0 + e1 * x1;
  r.gx = e1 - e0;
  r.gy = (c01 - c00) * x0 + (c11 - c10) * x1;
  r.gz = ((f001 - f000) * y0 + (f011 - f010) * y1) * x0 + ((f101 - f100) * y0 + (f111 - f110) * y1) * x1;
  return r;
}

// Bases and weights of the six staggers (the order of Gathered: ex ey ez bx by bz).
template <typename real>
struct Stagger {
  int n;
  real x0, x1, y0, y1, z0, z1;
};

template <typename real>
__device__ __forceinline__ Stagger<real> stagger(const Geom& g, const Axis<real>& X, const Axis<real>& Y,
                                                 const Axis<real>& Z, int q) {
  const bool hx = q == 1 || q == 2 || q == 3;  // half-shifted along x: ey ez bx
  const bool hy = q == 0 || q == 2 || q == 4;  // along y: ex ez by
  const bool hz = q == 0 || q == 1 || q == 5;  // along z: ex ey bz
  Stagger<real> s;
  s.n = (hx ? X.b : X.a) * g.sx + (hy ? Y.b : Y.a) * g.gz + (hz ? Z.b : Z.a);
  s.x0 = hx ? X.b0 : X.a0; s.x1 = hx ? X.b1 : X.a1;
  s.y0 = hy ? Y.b0 : Y.a0; s.y1 = hy ? Y.b1 : Y.a1;
  s.z0 = hz ? Z.b0 : Z.a0; s.z1 = hz ? Z.b1 : Z.a1;
  return s;
}

struct AdjConst {
  double K;       // s q n dx^3 of the species (s = +1 ions, -1 electrons)
  double dt;
  double inv_I;   // 1 / I (0 when I == 0)
  double imf[3];
  double jsign;   // +1 ions, -1 electrons: the E update takes J_i - J_e
};

// ------------------------------------------------------------ forward
// The forward of the adjoint run must replay bit for bit when a segment is
// recomputed, so its current deposit sums in 64-bit fixed point (integer
// atomics do not depend on the order of the particles): each term
// v_q W / c is scaled by 2^40, which leaves 23 bits of headroom for the
// number of particles per node; jconvert_kernel turns the sums into
// J = q n c (sum / 2^40). The warp-aggregated scatter below keeps this: it
// converts deterministic per-group sums.
constexpr double kJFixed = 1099511627776.0;  // 2^40

// ------------------------------------------------------------ warp-aggregated scatters
// Slots keep the order of the initial load and of each refill, which is cell
// order, so the lanes of a warp mostly share a few stencil bases. Lanes with
// the same base (found with match.any) sum their eight terms first and the
// group's first lane issues the atomics. `key` is the base node, or -1 for a
// lane that adds nothing. Every lane of the warp calls these together.

constexpr unsigned kFullWarp = 0xffffffffu;

// Sums w over each group of lanes (grp: this lane's group) by pointer jumping
// along the group's lanes: after step s a lane holds the sum of 2^s members
// from itself on, so the group's first lane has the total after
// ceil(log2(largest group)) steps of nine shuffles.
template <typename T>
__device__ __forceinline__ void group_sum8(T (&w)[8], unsigned grp) {
  const int lane = threadIdx.x & 31;
  int nxt = __ffs(grp & ~((2u << lane) - 1u)) - 1;  // the group's next lane above this one
  const int m = __popc(grp);
  const int steps = (int)__reduce_max_sync(kFullWarp, m > 1 ? 32u - (unsigned)__clz(m - 1) : 0u);
  for (int it = 0; it < steps; ++it) {
    const int src = nxt < 0 ? lane : nxt;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const T u = __shfl_sync(kFullWarp, w[q], src);
      if (nxt >= 0) w[q] += u;
    }
    const int nn = __shfl_sync(kFullWarp, nxt, src);
    nxt = nxt < 0 ? -1 : nn;
  }
}

// Fixed-point J: each group's terms are summed in the engine's precision by
// group_sum8, whose order of additions depends only on which slots share the
// warp and the base, and the first lane adds the sums as 64-bit integers.
// A replayed segment has the same slots in the same warps, so it adds the
// same integers, and integer atomics do not depend on their order.
template <typename real>
__device__ __forceinline__ void scatter8_fixed_agg(unsigned long long* F, int key, int sx, int sy, real v, real x0,
                                                   real x1, real y0, real y1, real z0, real z1) {
  const unsigned grp = __match_any_sync(kFullWarp, key);
  const real a0 = v * x0, a1 = v * x1;
  const real a00 = a0 * y0, a01 = a0 * y1, a10 = a1 * y0, a11 = a1 * y1;
  real w[8] = {a00 * z0, a00 * z1, a01 * z0, a01 * z1, a10 * z0, a10 * z1, a11 * z0, a11 * z1};
  group_sum8(w, grp);
  if (key >= 0 && (int)(threadIdx.x & 31) == __ffs(grp) - 1) {
    const int o[8] = {0, 1, sy, sy + 1, sx, sx + 1, sx + sy, sx + sy + 1};
#pragma unroll
    for (int q = 0; q < 8; ++q) atomicAdd(F + key + o[q], (unsigned long long)__double2ll_rn((double)w[q]));
  }
}

// Floating-point terms: one atomic per group and node.
template <typename real>
__device__ __forceinline__ void scatter8_agg(real* F, int key, int sx, int sy, real v, real x0, real x1, real y0,
                                             real y1, real z0, real z1) {
  const unsigned grp = __match_any_sync(kFullWarp, key);
  const real a0 = v * x0, a1 = v * x1;
  const real a00 = a0 * y0, a01 = a0 * y1, a10 = a1 * y0, a11 = a1 * y1;
  real w[8] = {a00 * z0, a00 * z1, a01 * z0, a01 * z1, a10 * z0, a10 * z1, a11 * z0, a11 * z1};
  group_sum8(w, grp);
  if (key >= 0 && (int)(threadIdx.x & 31) == __ffs(grp) - 1) {
    const int o[8] = {0, 1, sy, sy + 1, sx, sx + 1, sx + sy, sx + sy + 1};
#pragma unroll
    for (int q = 0; q < 8; ++q) atomicAdd(F + key + o[q], w[q]);
  }
}

// push_kernel<real, PUSH_FUSED> with the J deposit into fixed-point planes
// J64[3] (v scaled by 2^40 / c).
template <typename real>
__global__ void __launch_bounds__(256, sizeof(real) == 4 ? 4 : 2) push_fixed_kernel(Parts<real> P, const int* count, Fields<real> F, Geom g,
                                                         PushConst<real> pc, unsigned long long* J64x,
                                                         unsigned long long* J64y, unsigned long long* J64z,
                                                         real vscale, int with_n, AdjConst a, double* obj,
                                                         unsigned long long* err) {
  const int n = *count;
  unsigned pushed = 0;
  double fobj = 0.0;
  const int sx = g.sx, sy = g.gz;
  const int lane = threadIdx.x & 31;
  // warp-uniform trip count: the J deposit is aggregated across the warp
  for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += gridDim.x * blockDim.x) {
    const int t = base + lane;
    Rec<real> r{};
    r.cell = -1;
    if (t < n) r = load_records(P, t);
    const bool live = r.cell >= 0;
    int i = 0, j = 0, k = 0;
    real fx = r.o[0], fy = r.o[1], fz = r.o[2];
    real vx = r.v[0], vy = r.v[1], vz = r.v[2];
    bool dep = false;
    Axis<real> X{}, Y{}, Z{};
    if (live) {
      ++pushed;
      unpack_cell(r.cell, i, j, k);
      bool bal = ballistic(pc, i, j, k, fx, fy, fz);
      if (!bal && !stencil_ok(g, i, j, k)) {
        count_err(err, ERR_DEPOSIT_OOB);
        bal = true;
      }
      if (!bal) {
        const Axis<real> X0 = axis_weights(i, fx), Y0 = axis_weights(j, fy), Z0 = axis_weights(k, fz);
        boris4(pc, gather6(F, g, X0, Y0, Z0), vx, vy, vz);
        if (!(isfinite(vx) && isfinite(vy) && isfinite(vz))) count_err(err, ERR_NONFINITE);
      }
      advance(i, fx, vx * pc.hdt);
      advance(j, fy, vy * pc.hdt);
      advance(k, fz, vz * pc.hdt);
      if (in_array(g, i, j, k)) {
        if (stencil_ok(g, i, j, k)) {
          dep = true;
          X = axis_weights(i, fx); Y = axis_weights(j, fy); Z = axis_weights(k, fz);
        } else {
          count_err(err, ERR_DEPOSIT_OOB);
        }
      }
    }
    scatter8_fixed_agg(J64x, dep ? X.a * sx + Y.b * sy + Z.b : -1, sx, sy, dep ? vx * vscale : (real)0, X.a0, X.a1,
                       Y.b0, Y.b1, Z.b0, Z.b1);
    scatter8_fixed_agg(J64y, dep ? X.b * sx + Y.a * sy + Z.b : -1, sx, sy, dep ? vy * vscale : (real)0, X.b0, X.b1,
                       Y.a0, Y.a1, Z.b0, Z.b1);
    scatter8_fixed_agg(J64z, dep ? X.b * sx + Y.b * sy + Z.a : -1, sx, sy, dep ? vz * vscale : (real)0, X.b0, X.b1,
                       Y.b0, Y.b1, Z.a0, Z.a1);
    bool depn = false;
    if (live) {
      advance(i, fx, vx * pc.hdt);
      advance(j, fy, vy * pc.hdt);
      advance(k, fz, vz * pc.hdt);
      if (in_array(g, i, j, k)) {
        if (stencil_ok(g, i, j, k)) {
          depn = true;
          X = axis_weights(i, fx); Y = axis_weights(j, fy); Z = axis_weights(k, fz);
        } else {
          count_err(err, ERR_DEPOSIT_OOB);
        }
      }
    }
    // the density deposit (deposit_n), aggregated like J; only where the caller asks for n
    if (with_n)
      scatter8_agg(F.f[pc.pn], depn ? X.b * sx + Y.b * sy + Z.b : -1, sx, sy, depn ? pc.nw : (real)0, X.b0, X.b1,
                   Y.b0, Y.b1, Z.b0, Z.b1);
    if (live) {
      const int cell = boundary(g, i, j, k) ? repack(i, j, k, err) : -1;
      store_records(P, t, cell, fx, fy, fz, vx, vy, vz);
      // F of this particle after the step (times K dt in the block sum) when obj is given: the objective
      if (obj && cell >= 0 && stencil_ok(g, i, j, k)) {
        const Axis<real> X2 = axis_weights(i, fx), Y2 = axis_weights(j, fy), Z2 = axis_weights(k, fz);
        const Stagger<real> bxs = stagger(g, X2, Y2, Z2, 3), bys = stagger(g, X2, Y2, Z2, 4);
        const double b0x = trilerp(F.f[F_B0X], bxs.n, sx, sy, bxs.x0, bxs.x1, bxs.y0, bxs.y1, bxs.z0, bxs.z1);
        const double b0y = trilerp(F.f[F_B0Y], bys.n, sx, sy, bys.x0, bys.x1, bys.y0, bys.y1, bys.z0, bys.z1);
        fobj -= (double)vx * b0y - (double)vy * b0x;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) pushed += __shfl_down_sync(0xffffffffu, pushed, o);
  if ((threadIdx.x & 31) == 0 && pushed) atomicAdd(err + CNT_PUSHED, (unsigned long long)pushed);
  if (obj) {
    double sv[1] = {fobj};
    const int idx[1] = {0};
    const double scale[1] = {a.K * a.dt};
    block_reduce_add<1>(sv, obj, idx, scale);
  }
}

// J planes of one species from the fixed-point sums.
template <typename real>
__global__ void jconvert_kernel(const unsigned long long* __restrict__ J64, int nodes, real* jx, real* jy, real* jz,
                                double scale) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= nodes) return;
  jx[n] = (real)((double)(long long)J64[n] * scale);
  jy[n] = (real)((double)(long long)J64[nodes + n] * scale);
  jz[n] = (real)((double)(long long)J64[2 * nodes + n] * scale);
}


// Reverse of boris4 (cal_track4, :2804-2870): recomputes the forward from
// (v, E, B) and maps the adjoint of the new velocity av to the adjoints of
// v (returned in av), of the gathered E (ae) and of the gathered B (ab).
template <typename real>
__device__ __forceinline__ void boris4_adjoint(const PushConst<real>& pc, const Gathered<real>& G,
                                               real vx, real vy, real vz, real (&av)[3], real (&ae)[3],
                                               real (&ab)[3]) {
  const real T = pc.T, C = pc.C;
  const real ex = G.ex + pc.ex_add, ey = G.ey + pc.ey_add, ez = G.ez;
  const real bx = G.bx, by = G.by, bz = G.bz;
  const real s1 = pc.C2 - vx * vx - vy * vy - vz * vz;
  real g1 = C / sqrt(s1);
  const bool nan1 = isnan(g1);
  if (nan1) g1 = (real)0;
  const real ux0 = g1 * vx, uy0 = g1 * vy, uz0 = g1 * vz;
  const real s2 = pc.C2 + ux0 * ux0 + uy0 * uy0 + uz0 * uz0;
  const real g2 = C / sqrt(s2);
  const real bux = g2 * bx, buy = g2 * by, buz = g2 * bz;
  const real D = (real)1 + T * T * (bux * bux + buy * buy + buz * buz);
  const real S = (real)2 * T / D;
  const real ux = ux0 + ex * T, uy = uy0 + ey * T, uz = uz0 + ez * T;
  const real uox = ux + T * (uy * buz - uz * buy);
  const real uoy = uy + T * (uz * bux - ux * buz);
  const real uoz = uz + T * (ux * buy - uy * bux);
  const real cx = uoy * buz - uoz * buy, cy = uoz * bux - uox * buz, cz = uox * buy - uoy * bux;
  const real qx = ux + S * cx + ex * T, qy = uy + S * cy + ey * T, qz = uz + S * cz + ez * T;
  const real s3 = pc.C2 + qx * qx + qy * qy + qz * qz;
  const real g3 = C / sqrt(s3);
  // reverse
  const real a_g3 = av[0] * qx + av[1] * qy + av[2] * qz;
  const real a_s3 = a_g3 * ((real)-0.5 * g3 / s3);
  const real aqx = av[0] * g3 + (real)2 * qx * a_s3;
  const real aqy = av[1] * g3 + (real)2 * qy * a_s3;
  const real aqz = av[2] * g3 + (real)2 * qz * a_s3;
  real aex = aqx * T, aey = aqy * T, aez = aqz * T;
  real aux = aqx, auy = aqy, auz = aqz;
  const real aS = aqx * cx + aqy * cy + aqz * cz;
  const real acx = S * aqx, acy = S * aqy, acz = S * aqz;
  real auox = -acy * buz + acz * buy;
  real auoy = acx * buz - acz * bux;
  real auoz = -acx * buy + acy * bux;
  real abux = acy * uoz - acz * uoy;
  real abuy = -acx * uoz + acz * uox;
  real abuz = acx * uoy - acy * uox;
  // uo = u + T (u x bu)
  aux += auox; auy += auoy; auz += auoz;
  auy += T * auox * buz; abuz += T * auox * uy; auz -= T * auox * buy; abuy -= T * auox * uz;
  auz += T * auoy * bux; abux += T * auoy * uz; aux -= T * auoy * buz; abuz -= T * auoy * ux;
  aux += T * auoz * buy; abuy += T * auoz * ux; auy -= T * auoz * bux; abux -= T * auoz * uy;
  // u = u0 + E T
  aex += aux * T; aey += auy * T; aez += auz * T;
  // S = 2T / D, D = 1 + T^2 |bu|^2
  const real aD = -aS * S / D;
  abux += aD * T * T * (real)2 * bux;
  abuy += aD * T * T * (real)2 * buy;
  abuz += aD * T * T * (real)2 * buz;
  // bu = g2 B
  const real a_g2 = abux * bx + abuy * by + abuz * bz;
  ab[0] = abux * g2; ab[1] = abuy * g2; ab[2] = abuz * g2;
  const real a_s2 = a_g2 * ((real)-0.5 * g2 / s2);
  const real aux0 = aux + (real)2 * ux0 * a_s2;
  const real auy0 = auy + (real)2 * uy0 * a_s2;
  const real auz0 = auz + (real)2 * uz0 * a_s2;
  // u0 = g1 v, g1 = C / sqrt(C^2 - |v|^2)
  av[0] = g1 * aux0; av[1] = g1 * auy0; av[2] = g1 * auz0;
  if (!nan1) {
    const real a_g1 = aux0 * vx + auy0 * vy + auz0 * vz;
    const real a_s1 = a_g1 * ((real)-0.5 * g1 / s1);
    av[0] -= (real)2 * vx * a_s1;
    av[1] -= (real)2 * vy * a_s1;
    av[2] -= (real)2 * vz * a_s1;
  }
  ae[0] = aex; ae[1] = aey; ae[2] = aez;
}

template <typename real>
struct AdjPart {
  real* lx[3];          // dJ/dxi of each slot (in: after the step; out: before it)
  real* lv[3];          // dJ/dv
  const real* lj[3];    // dJ/dJ_ion of the three current planes (after the fold's transpose)
  real* le[3];          // dJ/dE at the step start (accumulated)
  real* ldb[3];         // this step's particle terms of dJ/dDB (three zeroed planes; ldb_merge_kernel adds
                        // them to dJ/dDB after the first B half-step)
};

// Reverse of push_kernel<real, PUSH_FUSED> for one species, plus the
// objective term of the particle after the step. P holds the particles as the
// push found them; F the fields it gathered (E at the step start, B after the
// first half-step) and B0. acc[1] += dJ/dI, acc[2] += dJ/dV.
template <typename real>
__global__ void __launch_bounds__(256, sizeof(real) == 4 ? 3 : 2) push_adjoint_kernel(Parts<real> P, int n, Fields<real> F, Geom g,
                                                           PushConst<real> pc, AdjPart<real> A, AdjConst a,
                                                           double* acc) {
  double s[2] = {0.0, 0.0};
  const int sx = g.sx, sy = g.gz;
  const real js = (real)a.jsign;
  const int lane = threadIdx.x & 31;
  // warp-uniform trip count: the field adjoints' scatter is aggregated across the warp
  for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += gridDim.x * blockDim.x) {
    const int t = base + lane;
    Rec<real> r{};
    r.cell = -1;
    if (t < n) r = load_records(P, t);
    const bool live = r.cell >= 0;
    if (t < n && !live) {
#pragma unroll
      for (int q = 0; q < 3; ++q) { A.lx[q][t] = (real)0; A.lv[q][t] = (real)0; }
    }
    bool bal = true;
    Axis<real> X0{}, Y0{}, Z0{};
    const int src[6] = {F_EX, F_EY, F_EZ, F_BX, F_BY, F_BZ};
    real fg[6][3] = {};  // gradients of the six interpolants at xi0, kept from the recompute's gather
    real ax[3] = {0, 0, 0};
    real af[6] = {0, 0, 0, 0, 0, 0};  // adjoints of the gathered E and B
    if (live) {
      int i0, j0, k0;
      unpack_cell(r.cell, i0, j0, k0);
      const real f0x = r.o[0], f0y = r.o[1], f0z = r.o[2];
      const real v0x = r.v[0], v0y = r.v[1], v0z = r.v[2];
      // ---- forward recompute
      bal = ballistic(pc, i0, j0, k0, f0x, f0y, f0z);
      if (!bal && !stencil_ok(g, i0, j0, k0)) bal = true;
      Gathered<real> G{};
      real vx = v0x, vy = v0y, vz = v0z;
      if (!bal) {
        X0 = axis_weights(i0, f0x); Y0 = axis_weights(j0, f0y); Z0 = axis_weights(k0, f0z);
        // gather6 with the gradients: the same interpolants, read once for the recompute and the reverse
        real gv[6];
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          const Stagger<real> st = stagger(g, X0, Y0, Z0, q);
          const VG<real> f = trilerp_vg(F.f[src[q]], st.n, sx, sy, st.x0, st.x1, st.y0, st.y1, st.z0, st.z1);
          gv[q] = f.v;
          fg[q][0] = f.gx; fg[q][1] = f.gy; fg[q][2] = f.gz;
        }
        G = Gathered<real>{gv[0], gv[1], gv[2], gv[3], gv[4], gv[5]};
        boris4(pc, G, vx, vy, vz);
      }
      int ih = i0, jh = j0, kh = k0;
      real fhx = f0x, fhy = f0y, fhz = f0z;
      advance(ih, fhx, vx * pc.hdt);
      advance(jh, fhy, vy * pc.hdt);
      advance(kh, fhz, vz * pc.hdt);
      const bool dep = in_array(g, ih, jh, kh) && stencil_ok(g, ih, jh, kh);
      int i1 = ih, j1 = jh, k1 = kh;
      real f1x = fhx, f1y = fhy, f1z = fhz;
      advance(i1, f1x, vx * pc.hdt);
      advance(j1, f1y, vy * pc.hdt);
      advance(k1, f1z, vz * pc.hdt);
      const bool alive = boundary(g, i1, j1, k1);
      // ---- reverse
      real av[3] = {0, 0, 0};
      if (alive) {
#pragma unroll
        for (int q = 0; q < 3; ++q) { ax[q] = A.lx[q][t]; av[q] = A.lv[q][t]; }
        if (stencil_ok(g, i1, j1, k1)) {
          // objective: F_p = -K (vx B0y - vy B0x) at the new (wrapped) position, times dt
          const Axis<real> X = axis_weights(i1, f1x), Y = axis_weights(j1, f1y), Z = axis_weights(k1, f1z);
          const Stagger<real> bxs = stagger(g, X, Y, Z, 3), bys = stagger(g, X, Y, Z, 4);
          const VG<real> b0x = trilerp_vg(F.f[F_B0X], bxs.n, sx, sy, bxs.x0, bxs.x1, bxs.y0, bxs.y1, bxs.z0, bxs.z1);
          const VG<real> b0y = trilerp_vg(F.f[F_B0Y], bys.n, sx, sy, bys.x0, bys.x1, bys.y0, bys.y1, bys.z0, bys.z1);
          const real w = (real)(-a.K * a.dt);
          av[0] += w * b0y.v;
          av[1] -= w * b0x.v;
          ax[0] += w * (vx * b0y.gx - vy * b0x.gx);
          ax[1] += w * (vx * b0y.gy - vy * b0x.gy);
          ax[2] += w * (vx * b0y.gz - vy * b0x.gz);
          s[0] += (double)w * ((double)vx * ((double)b0y.v - a.imf[1]) - (double)vy * ((double)b0x.v - a.imf[0])) * a.inv_I;
        }
      }
      // drift: xi1 = xih + hdt v
#pragma unroll
      for (int q = 0; q < 3; ++q) av[q] += pc.hdt * ax[q];
      // J deposit at xih: J_q += qn v_q W_q(xih)
      if (dep) {
        const Axis<real> X = axis_weights(ih, fhx), Y = axis_weights(jh, fhy), Z = axis_weights(kh, fhz);
        const real vq[3] = {vx, vy, vz};
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const Stagger<real> st = stagger(g, X, Y, Z, q);
          const VG<real> l = trilerp_vg(A.lj[q], st.n, sx, sy, st.x0, st.x1, st.y0, st.y1, st.z0, st.z1);
          const real k = js * pc.qn;
          av[q] += k * l.v;
          ax[0] += k * vq[q] * l.gx;
          ax[1] += k * vq[q] * l.gy;
          ax[2] += k * vq[q] * l.gz;
        }
      }
      // xih = xi0 + hdt v
#pragma unroll
      for (int q = 0; q < 3; ++q) av[q] += pc.hdt * ax[q];
      if (!bal) {
        real ae[3], ab[3];
        boris4_adjoint(pc, G, v0x, v0y, v0z, av, ae, ab);
        s[1] += (double)ae[0] * a.imf[1] - (double)ae[1] * a.imf[0];  // E += (V IMF_y, -V IMF_x, 0)
        af[0] = ae[0]; af[1] = ae[1]; af[2] = ae[2];
        af[3] = ab[0]; af[4] = ab[1]; af[5] = ab[2];
      }
#pragma unroll
      for (int q = 0; q < 3; ++q) A.lv[q][t] = av[q];
    }
    // gather at xi0: scatter the field adjoints, add the interpolants' gradients
    const bool gat = live && !bal;
    real* const dst[6] = {A.le[0], A.le[1], A.le[2], A.ldb[0], A.ldb[1], A.ldb[2]};
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      Stagger<real> st{};
      if (gat) {
        st = stagger(g, X0, Y0, Z0, q);
        ax[0] += af[q] * fg[q][0];
        ax[1] += af[q] * fg[q][1];
        ax[2] += af[q] * fg[q][2];
      }
      scatter8_agg(dst[q], gat ? st.n : -1, sx, sy, gat ? af[q] : (real)0, st.x0, st.x1, st.y0, st.y1, st.z0,
                   st.z1);
    }
    if (live) {
#pragma unroll
      for (int q = 0; q < 3; ++q) A.lx[q][t] = ax[q];
    }
  }
  const int idx[2] = {1, 2};
  const double scale[2] = {1.0, 1.0};
  block_reduce_add<2>(s, acc, idx, scale);
}

// acc[2] += sum of dJ/dvz over slots [first, n): particles created with
// vz = V + thermal (by the initial load or a refill).
template <typename real>
__global__ void __launch_bounds__(256) drift_grad_kernel(Parts<real> P, const real* __restrict__ lvz,
                                                         int first, int n, double* acc) {
  double s[1] = {0.0};
  for (int t = first + blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
    if (P.cell[t] >= 0) s[0] += (double)lvz[t];
  const int idx[1] = {2};
  const double scale[1] = {1.0};
  block_reduce_add<1>(s, acc, idx, scale);
}

// Reverse of the stable compaction before a refill: the adjoint of old slot
// t is that of its new slot, or zero when it was removed.
template <typename real>
__global__ void uncompact_adjoint_kernel(const int* __restrict__ map, int n_old, AdjPart<real> from,
                                         AdjPart<real> to) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_old) return;
  const int m = map[t];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    to.lx[q][t] = m >= 0 ? from.lx[q][m] : (real)0;
    to.lv[q][t] = m >= 0 ? from.lv[q][m] : (real)0;
  }
}

// ---------------------------------------------------------------- fields
// Value of plane W at (i, j, k), zero outside the array.
template <typename real>
__device__ __forceinline__ real wat(const real* W, const Geom& g, int i, int j, int k) {
  return (i >= 0 && j >= 0 && k >= 0 && i < g.gx && j < g.gy && k < g.gz) ? W[i * g.sx + j * g.gz + k] : (real)0;
}

// Transposes of the two 4th-order differences, in gather form at node (i,j,k)
// along axis d (0 x, 1 y, 2 z):
//   forward  D+(a)[n] = 27 (a[n+s] - a[n]) - (a[n+2s] - a[n-s])   (renew_e4_2)
//   backward D-(a)[n] = 27 (a[n] - a[n-s]) - (a[n+s] - a[n-2s])   (renew_b4_2)
template <typename real>
__device__ __forceinline__ real dplus_t(const real* W, const Geom& g, int i, int j, int k, int d) {
  const int di = d == 0, dj = d == 1, dk = d == 2;
  return (real)27 * (wat(W, g, i - di, j - dj, k - dk) - wat(W, g, i, j, k)) -
         wat(W, g, i - 2 * di, j - 2 * dj, k - 2 * dk) + wat(W, g, i + di, j + dj, k + dk);
}
template <typename real>
__device__ __forceinline__ real dminus_t(const real* W, const Geom& g, int i, int j, int k, int d) {
  const int di = d == 0, dj = d == 1, dk = d == 2;
  return (real)27 * (wat(W, g, i, j, k) - wat(W, g, i + di, j + dj, k + dk)) -
         wat(W, g, i - di, j - dj, k - dk) + wat(W, g, i + 2 * di, j + 2 * dj, k + 2 * dk);
}

template <typename real>
struct AdjField {
  real* le[3];
  real* ldb[3];
  real* lj[3];
  real* w[3];   // scratch planes (zero outside the interior)
};

// The particles' dJ/dDB terms T of one reverse step into lDB, T zeroed for
// the next step, and acc[1] += sum over nodes of T (B0 - IMF) / I: B = B0 +
// DB, and the dipole part of B0 is proportional to I. Summing T (B0 - IMF) per
// node equals summing each particle's term with B0 interpolated at the
// particle, because the interpolation weights of a particle are the weights
// of its scatter and add up to one.
template <typename real>
__global__ void __launch_bounds__(256) ldb_merge_kernel(Fields<real> F, AdjPart<real> T, AdjField<real> A, int nodes,
                                                        AdjConst a, double* acc) {
  double s[1] = {0.0};
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < nodes; n += gridDim.x * blockDim.x) {
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const real t = T.ldb[q][n];
      if (t == (real)0) continue;
      A.ldb[q][n] += t;
      T.ldb[q][n] = (real)0;
      s[0] += (double)t * ((double)F.f[F_B0X + q][n] - a.imf[q]);
    }
  }
  const int idx[1] = {1};
  const double scale[1] = {a.inv_I};
  block_reduce_add<1>(s, acc, idx, scale);
}

// Reverse of renew_e_kernel, part 1 (pointwise on interior nodes):
// W = cb c24 lE, lJ_ion = -cb mu0 lE, lE = ca lE.
template <typename real>
__global__ void __launch_bounds__(256) renew_e_adjoint_point(AdjField<real> A, Geom g, Ramps rp, EParams p) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int nint = g.nx * g.ny * g.nz;
  if (t >= nint) return;
  const int m = 2 + t % g.nz, l = 2 + (t / g.nz) % g.ny, k = 2 + t / (g.nz * g.ny);
  const int n = k * g.sx + l * g.gz + m;
  const double sg[3] = {sigma_of(rp.a, rp.rx[2 * k], rp.ry[2 * l + 1], rp.rz[2 * m + 1]),
                        sigma_of(rp.a, rp.rx[2 * k + 1], rp.ry[2 * l], rp.rz[2 * m + 1]),
                        sigma_of(rp.a, rp.rx[2 * k + 1], rp.ry[2 * l + 1], rp.rz[2 * m])};
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const double h = 0.5 * p.mu0 * sg[q] * p.temp;
    const real ca = (real)((1. - h) / (1. + h)), cb = (real)(p.temp / (1. + h));
    const real le = A.le[q][n];
    A.w[q][n] = cb * (real)p.inv24dx * le;
    A.lj[q][n] = -cb * (real)p.mu0 * le;
    A.le[q][n] = ca * le;
  }
}

// Part 2: lDB += (curl of renew_e)^T W, every node.
template <typename real>
__global__ void __launch_bounds__(256) renew_e_adjoint_curl(AdjField<real> A, Geom g) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= g.nodes) return;
  const int i = n / g.sx, j = (n / g.gz) % g.gy, k = n % g.gz;
  // Ex += W (D+_y Bz - D+_z By), Ey += W (D+_z Bx - D+_x Bz), Ez += W (D+_x By - D+_y Bx)
  A.ldb[0][n] += dplus_t(A.w[1], g, i, j, k, 2) - dplus_t(A.w[2], g, i, j, k, 1);
  A.ldb[1][n] += dplus_t(A.w[2], g, i, j, k, 0) - dplus_t(A.w[0], g, i, j, k, 2);
  A.ldb[2][n] += dplus_t(A.w[0], g, i, j, k, 1) - dplus_t(A.w[1], g, i, j, k, 0);
}

// Reverse of renew_b_kernel, part 1 (pointwise): W = cb c24 lDB, lDB = ca lDB.
template <typename real>
__global__ void __launch_bounds__(256) renew_b_adjoint_point(AdjField<real> A, Geom g, Ramps rp, BParams p) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int nint = g.nx * g.ny * g.nz;
  if (t >= nint) return;
  const int m = 2 + t % g.nz, l = 2 + (t / g.nz) % g.ny, k = 2 + t / (g.nz * g.ny);
  const int n = k * g.sx + l * g.gz + m;
  const double sg[3] = {sigma_of(rp.a, rp.rx[2 * k + 1], rp.ry[2 * l], rp.rz[2 * m]),
                        sigma_of(rp.a, rp.rx[2 * k], rp.ry[2 * l + 1], rp.rz[2 * m]),
                        sigma_of(rp.a, rp.rx[2 * k], rp.ry[2 * l], rp.rz[2 * m + 1])};
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const real ca = (real)((1. - sg[q] * p.temp) / (1. + sg[q] * p.temp));
    const real cb = (real)(p.dth / (1. + sg[q] * p.temp));
    const real l = A.ldb[q][n];
    A.w[q][n] = cb * (real)p.inv24dx * l;
    A.ldb[q][n] = ca * l;
  }
}

// Part 2: lE -= (curl of renew_b)^T W, every node.
template <typename real>
__global__ void __launch_bounds__(256) renew_b_adjoint_curl(AdjField<real> A, Geom g) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= g.nodes) return;
  const int i = n / g.sx, j = (n / g.gz) % g.gy, k = n % g.gz;
  // DBx -= W (D-_y Ez - D-_z Ey), DBy -= W (D-_z Ex - D-_x Ez), DBz -= W (D-_x Ey - D-_y Ex)
  A.le[0][n] += -dminus_t(A.w[1], g, i, j, k, 2) + dminus_t(A.w[2], g, i, j, k, 1);
  A.le[1][n] += -dminus_t(A.w[2], g, i, j, k, 0) + dminus_t(A.w[0], g, i, j, k, 2);
  A.le[2][n] += -dminus_t(A.w[0], g, i, j, k, 1) + dminus_t(A.w[1], g, i, j, k, 0);
}

// Reverse of wrap_kernel (ghost copies): the adjoint of a
// ghost goes to its source and the ghost's own adjoint is cleared.
template <typename real>
__global__ void wrap_x_adjoint(PlaneSet<real> s, Geom g) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.gy * g.gz) return;
  const int N = g.nx, sx = g.sx;
  for (int q = 0; q < s.count; ++q) {
    real* a = s.p[q];
    a[N * sx + t] += a[t];
    a[(N + 1) * sx + t] += a[sx + t];
    a[2 * sx + t] += a[(N + 2) * sx + t];
    a[3 * sx + t] += a[(N + 3) * sx + t];
    a[t] = a[sx + t] = a[(N + 2) * sx + t] = a[(N + 3) * sx + t] = (real)0;
  }
}

template <typename real>
__global__ void wrap_y_adjoint(PlaneSet<real> s, Geom g) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.gx * g.gz) return;
  const int k = t / g.gz, m = t % g.gz;
  const int N = g.ny, sy = g.gz;
  const int b = k * g.sx + m;
  for (int q = 0; q < s.count; ++q) {
    real* a = s.p[q];
    a[b + N * sy] += a[b];
    a[b + (N + 1) * sy] += a[b + sy];
    a[b + 2 * sy] += a[b + (N + 2) * sy];
    a[b + 3 * sy] += a[b + (N + 3) * sy];
    a[b] = a[b + sy] = a[b + (N + 2) * sy] = a[b + (N + 3) * sy] = (real)0;
  }
}

// Reverse of wrap_b_kernel on the induced field:
// DB[dst] = DB[src] + B0[src] - B0[dst], so besides the copy's transpose the
// ghost adjoints add lDB[dst] (B0[src] - B0[dst]) / I to dJ/dI (acc[1]).
template <typename real>
__global__ void __launch_bounds__(256) wrap_b_adjoint(Fields<real> F, AdjField<real> A, Geom g, int axis,
                                                      double inv_I, double* acc) {
  double s[1] = {0.0};
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int lim = axis == 0 ? g.gy * g.gz : g.gx * g.gz;
  if (t < lim) {
    int dst[4], src[4];
    if (axis == 0) {
      const int N = g.nx, sx = g.sx;
      const int d[4] = {t, sx + t, (N + 2) * sx + t, (N + 3) * sx + t};
      const int r[4] = {N * sx + t, (N + 1) * sx + t, 2 * sx + t, 3 * sx + t};
      for (int q = 0; q < 4; ++q) { dst[q] = d[q]; src[q] = r[q]; }
    } else {
      const int k = t / g.gz, m = t % g.gz;
      const int N = g.ny, sy = g.gz, b = k * g.sx + m;
      const int d[4] = {b, b + sy, b + (N + 2) * sy, b + (N + 3) * sy};
      const int r[4] = {b + N * sy, b + (N + 1) * sy, b + 2 * sy, b + 3 * sy};
      for (int q = 0; q < 4; ++q) { dst[q] = d[q]; src[q] = r[q]; }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      real* l = A.ldb[c];
      const real* b0 = F.f[F_B0X + c];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const real ld = l[dst[q]];
        s[0] += (double)ld * ((double)b0[src[q]] - (double)b0[dst[q]]) * inv_I;
        l[src[q]] += ld;
        l[dst[q]] = (real)0;
      }
    }
  }
  const int idx[1] = {1};
  const double scale[1] = {1.0};
  block_reduce_add<1>(s, acc, idx, scale);
}

// Reverse of fold_kernel: the ghosts' adjoints take those
// of the interior planes they were added to.
template <typename real>
__global__ void fold_x_adjoint(PlaneSet<real> s, Geom g) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.gy * g.gz) return;
  const int N = g.nx, sx = g.sx;
  for (int q = 0; q < s.count; ++q) {
    real* a = s.p[q];
    a[(N + 2) * sx + t] += a[2 * sx + t];
    a[(N + 3) * sx + t] += a[3 * sx + t];
    a[t] += a[N * sx + t];
    a[sx + t] += a[(N + 1) * sx + t];
  }
}

template <typename real>
__global__ void fold_y_adjoint(PlaneSet<real> s, Geom g) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.gx * g.gz) return;
  const int k = t / g.gz, m = t % g.gz;
  const int N = g.ny, sy = g.gz, b = k * g.sx + m;
  for (int q = 0; q < s.count; ++q) {
    real* a = s.p[q];
    a[b + (N + 2) * sy] += a[b + 2 * sy];
    a[b + (N + 3) * sy] += a[b + 3 * sy];
    a[b] += a[b + N * sy];
    a[b + sy] += a[b + (N + 1) * sy];
  }
}

// Stable compaction with its slot map (the adjoint run's refill): map[t] is
// the new slot of live slot t, -1 for an empty one. pos = exclusive scan of
// the live flags.
// Sort keys of the refill's compaction: the linear node index of a live
// slot's cell ((i gy + j) gz + k, below the node count), `dead` for an empty
// slot; the values are the slot indices. The keys span few bits, so the radix
// sort makes few passes.
template <typename real>
__global__ void cell_key_kernel(Parts<real> P, int n, Geom g, int dead, int* key, int* slot) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int c = P.cell[t];
  int v = dead;
  if (c >= 0) {
    int i, j, k;
    unpack_cell(c, i, j, k);
    v = (i * g.gy + j) * g.gz + k;
  }
  key[t] = v;
  slot[t] = t;
}

// The compaction's stable sort on those keys is a counting sort: count the
// slots of every key (the dead key counted in bucket `nodes`, after every
// node), scan the counts, scatter each slot to its key's run, then order each
// run by slot. The scatter's order within a run depends on the atomics; the
// last pass makes it the slot order, so a replayed segment gets the same
// result, which is the stable sort's. The dead run keeps the scatter's order:
// none of its slots is copied, and every one of them maps to -1.
__device__ __forceinline__ int key_bucket(int k, int dead, int nodes) { return k == dead ? nodes : k; }

__global__ void key_count_kernel(const int* __restrict__ key, int n, int dead, int nodes, int* cnt) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const bool in = t < n;
  warp_aggregated_inc(cnt, in ? key_bucket(key[t], dead, nodes) : 0, in);
}

// pos[b] holds the start of run b on entry and its end on return.
__global__ void key_scatter_kernel(const int* __restrict__ key, int n, int dead, int nodes, int* pos, int* okey,
                                   int* oslot) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const bool in = t < n;
  const int k = in ? key[t] : 0;
  const int p = warp_aggregated_inc(pos, in ? key_bucket(k, dead, nodes) : 0, in);
  if (in) {
    okey[p] = k;
    oslot[p] = t;
  }
}

// Each live entry's place in its run is the number of entries of the run with
// a lower slot (slots are distinct); `end` is the scatter's pos.
__global__ void key_rank_kernel(const int* __restrict__ skey, const int* __restrict__ sslot, int n, int dead,
                                const int* __restrict__ cnt, const int* __restrict__ end, int* okey, int* oslot) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int k = skey[p], v = sslot[p];
  int dst = p;
  if (k != dead) {
    const int e = end[k], s0 = e - cnt[k];
    int r = 0;
    for (int q = s0; q < e; ++q) r += sslot[q] < v;
    dst = s0 + r;
  }
  okey[dst] = k;
  oslot[dst] = v;
}

// Slot j of Q takes the particle of sorted position j; map[old slot] = j, or
// -1 for an empty slot; *count = the live particles (the first dead key).
template <typename real>
__global__ void cell_gather_kernel(Parts<real> P, int n, int dead, const int* __restrict__ key,
                                   const int* __restrict__ slot, Parts<real> Q, int* map, int* count) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int k = key[j], old = slot[j];
  const bool live = k != dead;
  if (live) copy_record(P, old, Q, j, P.cell[old]);
  if (map) map[old] = live ? j : -1;
  if (live && (j == n - 1 || key[j + 1] == dead)) *count = j + 1;
  if (j == 0 && !live) *count = 0;
}

__global__ void add_count_kernel(int* count, int add) { *count += add; }


}  // namespace pb
