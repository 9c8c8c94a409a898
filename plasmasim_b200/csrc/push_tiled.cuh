// The fused particle kernel over the tiled layout of tiled.cuh.
#pragma once

#include "common.cuh"
#include "particles.cuh"
#include "tiled.cuh"

namespace pb {

constexpr int kStages = 3;   // particle rows in flight per warp


// A box of cells: first cell (ci0, cj0, ck0) and extents; the push uses the
// domain's interior cells [2, n + 2) of each axis.
struct InteriorBox {
  int ci0, cj0, ck0;
  unsigned ex, ey, ez;
  __device__ __forceinline__ bool has(int i, int j, int k) const {
    return (unsigned)(i - ci0) < ex && (unsigned)(j - cj0) < ey && (unsigned)(k - ck0) < ez;
  }
};

// Shared-memory plan of one CTA (8 warps): the J/n window, per warp a ring of
// kStages particle rows fetched ahead with cp.async (records A and B of each
// slot) and, in FP32, the tile's E and B over the same window (the gather
// reads them there; FP64 gathers from global memory, its window would not
// leave room for two CTAs per SM).
template <typename real>
struct PushSmem {
  static constexpr int WX = kTileX + 4, WY = kTileY + 4, WZ = kWinZ, WN = WX * WY * WZ;
  static constexpr int kWarps = kTileX * kTileY;
  static constexpr bool kFieldWin = sizeof(real) == 4;
  static constexpr size_t win_bytes = 4 * WN * sizeof(real);
  static constexpr size_t prec_off = (win_bytes + 15) & ~(size_t)15;  // records A, B of each slot: 8 reals
  static constexpr size_t fwin_off = prec_off + (size_t)kWarps * kStages * kLanes * 8 * sizeof(real);
  // FP32: per warp a queue of kQ off-home J deposits, 7 words each (cell,
  // offsets, velocities), made 32 at a time by the whole warp (1.7 % off the
  // step against each particle depositing where it is found); FP64 has no
  // room for it beside two CTAs per SM
  static constexpr bool kJQueue = sizeof(real) == 4;
  static constexpr int kQ = 2 * kLanes;
  static constexpr size_t jq_off = fwin_off + (kFieldWin ? (size_t)6 * WN * sizeof(float) : 0);
  static constexpr size_t bytes = jq_off + (kJQueue ? (size_t)kWarps * kQ * 7 * sizeof(float) : 0);
};

// Trilinear interpolation from a window plane with compile-time strides (the
// 2x2x2 nodes at window index n), the two x planes as one packed pair.
template <int WY, int WZ>
__device__ __forceinline__ float trilerp_win(const float* __restrict__ w, int n, float x0, float x1, float2 Y0,
                                             float2 Y1, float2 Z0, float2 Z1) {
  constexpr int P = WY * WZ;  // next x plane
  const float2 n00 = make_float2(w[n], w[n + P]), n01 = make_float2(w[n + 1], w[n + P + 1]);
  const float2 n10 = make_float2(w[n + WZ], w[n + P + WZ]), n11 = make_float2(w[n + WZ + 1], w[n + P + WZ + 1]);
  const float2 cy0 = __ffma2_rn(n01, Z1, __fmul2_rn(n00, Z0));
  const float2 cy1 = __ffma2_rn(n11, Z1, __fmul2_rn(n10, Z0));
  const float2 cx = __ffma2_rn(cy1, Y1, __fmul2_rn(cy0, Y0));
  return cx.x * x0 + cx.y * x1;
}

// gather6 from a window of one plane per component (ex ey ez bx by bz, WN
// nodes each, origin (wx0, wy0, wz0)); the caller checks that the stencil lies inside.
template <int WY, int WZ, int WN>
__device__ __forceinline__ Gathered<float> gather6_win(const float* __restrict__ fw, int wx0, int wy0, int wz0,
                                                       const Axis<float>& X, const Axis<float>& Y,
                                                       const Axis<float>& Z) {
  const int ax = X.a - wx0, bx = X.b - wx0, ay = Y.a - wy0, by = Y.b - wy0, az = Z.a - wz0, bz = Z.b - wz0;
  const float2 ya0 = make_float2(Y.a0, Y.a0), ya1 = make_float2(Y.a1, Y.a1);
  const float2 yb0 = make_float2(Y.b0, Y.b0), yb1 = make_float2(Y.b1, Y.b1);
  const float2 za0 = make_float2(Z.a0, Z.a0), za1 = make_float2(Z.a1, Z.a1);
  const float2 zb0 = make_float2(Z.b0, Z.b0), zb1 = make_float2(Z.b1, Z.b1);
  Gathered<float> r;
  r.ex = trilerp_win<WY, WZ>(fw, (ax * WY + by) * WZ + bz, X.a0, X.a1, yb0, yb1, zb0, zb1);
  r.ey = trilerp_win<WY, WZ>(fw + WN, (bx * WY + ay) * WZ + bz, X.b0, X.b1, ya0, ya1, zb0, zb1);
  r.ez = trilerp_win<WY, WZ>(fw + 2 * WN, (bx * WY + by) * WZ + az, X.b0, X.b1, yb0, yb1, za0, za1);
  r.bx = trilerp_win<WY, WZ>(fw + 3 * WN, (bx * WY + ay) * WZ + az, X.b0, X.b1, ya0, ya1, za0, za1);
  r.by = trilerp_win<WY, WZ>(fw + 4 * WN, (ax * WY + by) * WZ + az, X.a0, X.a1, yb0, yb1, za0, za1);
  r.bz = trilerp_win<WY, WZ>(fw + 5 * WN, (ax * WY + ay) * WZ + bz, X.a0, X.a1, ya0, ya1, zb0, zb1);
  return r;
}

// The window's planes from F_EX .. F_BZ (16-byte loads where the row pitch
// allows), zero outside the array.
template <int WX, int WY, int WZ, bool VEC>
__device__ __forceinline__ void fill_win(float* __restrict__ fw, const Fields<float>& F, const Geom& g, int wx0,
                                         int wy0, int wz0) {
  constexpr int NZ4 = WZ / 4, WN = WX * WY * WZ;
  for (int q4 = threadIdx.x; q4 < 6 * WX * WY * NZ4; q4 += blockDim.x) {
    const int p = q4 / (WX * WY * NZ4), r = q4 % (WX * WY * NZ4);
    const int a = r / (WY * NZ4), b = (r / NZ4) % WY, c4 = r % NZ4;
    const int ga = wx0 + a, gb = wy0 + b, gc = wz0 + 4 * c4;
    float v[4] = {0.f, 0.f, 0.f, 0.f};
    if (ga < g.gx && gb < g.gy) {
      const float* src = F.f[p] + (long long)ga * g.sx + gb * g.gz + gc;
      if (VEC && gc + 3 < g.gz) {
        const float4 f4 = __ldg(reinterpret_cast<const float4*>(src));
        v[0] = f4.x; v[1] = f4.y; v[2] = f4.z; v[3] = f4.w;
      } else {
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (gc + e < g.gz) v[e] = __ldg(src + e);
      }
    }
    *reinterpret_cast<float4*>(fw + p * WN + (a * WY + b) * WZ + 4 * c4) = make_float4(v[0], v[1], v[2], v[3]);
  }
}

// The current of the particles that are in a lane's home cell, summed in
// registers over the 2x3x3 / 3x2x3 / 3x3x2 nodes such a particle can touch:
// x(a, b, c) is the jx sum at node (h-1+a+1, h-1+b, h-1+c) of the window flush
// below, and so on for y and z.
template <typename real>
struct HomeJ {
  real jx[2][3][3], jy[3][2][3], jz[3][3][2];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (a < 2) jx[a][b][c] = (real)0;
          if (b < 2) jy[a][b][c] = (real)0;
          if (c < 2) jz[a][b][c] = (real)0;
        }
  }
  __device__ __forceinline__ void add(real qx, real qy, real qz, const Axis<real>& X, const Axis<real>& Y,
                                      const Axis<real>& Z, const W3<real>& bx, const W3<real>& by,
                                      const W3<real>& bz) {
    const real ax[2] = {X.a0, X.a1}, ay[2] = {Y.a0, Y.a1}, az[2] = {Z.a0, Z.a1};
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const real yz = by.w[b] * bz.w[c];
        jx[0][b][c] += (qx * ax[0]) * yz;
        jx[1][b][c] += (qx * ax[1]) * yz;
      }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const real xz = bx.w[a] * bz.w[c];
        jy[a][0][c] += (qy * ay[0]) * xz;
        jy[a][1][c] += (qy * ay[1]) * xz;
      }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const real xy = bx.w[a] * by.w[b];
        jz[a][b][0] += (qz * az[0]) * xy;
        jz[a][b][1] += (qz * az[1]) * xy;
      }
  }
  __device__ __forceinline__ real x(int a, int b, int c) const { return jx[a][b][c]; }
  __device__ __forceinline__ real y(int a, int b, int c) const { return jy[a][b][c]; }
  __device__ __forceinline__ real z(int a, int b, int c) const { return jz[a][b][c]; }
};

// FP32: the two nodes of each component's unshifted axis as one packed pair,
// updated with the two-wide multiplies and FMAs of sm_100.
template <>
struct HomeJ<float> {
  float2 jx[3][3], jy[3][3], jz[3][3];  // jx[b][c] = (a = 0, a = 1); jy[a][c] = (b = 0, 1); jz[a][b] = (c = 0, 1)
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) jx[a][b] = jy[a][b] = jz[a][b] = make_float2(0.f, 0.f);
  }
  __device__ __forceinline__ void add(float qx, float qy, float qz, const Axis<float>& X, const Axis<float>& Y,
                                      const Axis<float>& Z, const W3<float>& bx, const W3<float>& by,
                                      const W3<float>& bz) {
    const float2 qxa = make_float2(qx * X.a0, qx * X.a1);
    const float2 qya = make_float2(qy * Y.a0, qy * Y.a1);
    const float2 qza = make_float2(qz * Z.a0, qz * Z.a1);
    float2 dx[3], dy[3], dz[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      dx[q] = make_float2(bx.w[q], bx.w[q]);
      dy[q] = make_float2(by.w[q], by.w[q]);
      dz[q] = make_float2(bz.w[q], bz.w[q]);
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const float2 tx = __fmul2_rn(qxa, dy[q]);  // jx: b = q
      const float2 ty = __fmul2_rn(qya, dx[q]);  // jy: a = q
      const float2 tz = __fmul2_rn(qza, dx[q]);  // jz: a = q
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        jx[q][r] = __ffma2_rn(tx, dz[r], jx[q][r]);  // c = r
        jy[q][r] = __ffma2_rn(ty, dz[r], jy[q][r]);  // c = r
        jz[q][r] = __ffma2_rn(tz, dy[r], jz[q][r]);  // b = r
      }
    }
  }
  __device__ __forceinline__ float x(int a, int b, int c) const { return a ? jx[b][c].y : jx[b][c].x; }
  __device__ __forceinline__ float y(int a, int b, int c) const { return b ? jy[a][c].y : jy[a][c].x; }
  __device__ __forceinline__ float z(int a, int b, int c) const { return c ? jz[a][b].y : jz[a][b].x; }
};

__device__ __forceinline__ void cp_async_16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(s), "l"(gmem) : "memory");
}

// Records A and B of particle t into 4 reals of shared memory each (16-byte copies).
template <typename real>
__device__ __forceinline__ void fetch_records(real* dst_a, real* dst_b, const Parts<real>& P, long long t) {
  constexpr int kPieces = 4 * (int)sizeof(real) / 16;  // 16-byte pieces per record
  const char* a = reinterpret_cast<const char*>(P.ra + 4 * t);
  const char* b = reinterpret_cast<const char*>(P.rb + 4 * t);
#pragma unroll
  for (int q = 0; q < kPieces; ++q) {
    cp_async_16(reinterpret_cast<char*>(dst_a) + 16 * q, a + 16 * q);
    cp_async_16(reinterpret_cast<char*>(dst_b) + 16 * q, b + 16 * q);
  }
}

// Four reals of one record from shared memory, as vector loads.
__device__ __forceinline__ void read_record(const float* p, float (&r)[4]) {
  const float4 v = *reinterpret_cast<const float4*>(p);
  r[0] = v.x; r[1] = v.y; r[2] = v.z; r[3] = v.w;
}
__device__ __forceinline__ void read_record(const double* p, double (&r)[4]) {
  const double2 v0 = reinterpret_cast<const double2*>(p)[0], v1 = reinterpret_cast<const double2*>(p)[1];
  r[0] = v0.x; r[1] = v0.y; r[2] = v1.x; r[3] = v1.y;
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" :: "n"(N) : "memory"); }

// The fused particle part of one step (push, J deposit at x^{n+1/2}, drift,
// n deposit at x^{n+1}, sr_particle) for one species over the tiled layout;
// the same arithmetic as push_kernel<real, PUSH_FUSED> apart from the FP32
// square roots and divisions and, in FP32, the fixed-point sums of the density
// window. One CTA per tile, one warp per group.
//
// J of a particle in its lane's home cell at x^{n+1/2} is summed in registers;
// the others add theirs to global memory with reductions (a shared J window
// taking every particle's 24 weights by FP32 shared atomics, which frees the
// registers for 3 CTAs per SM, measured 1.7x slower). The density goes to the window with shared
// reductions (every active lane at once): integer ones on fixed-point sums in
// FP32, FP64 atomics in FP64.
// FP64 at one CTA per SM: 254 registers and no spills, against 528 bytes of
// spill stores per thread at two CTAs per SM (128 registers); measured 30.6 ->
// 27.2 ms per step for the FP64 push at 128^3 cells x 64 particles/cell/species.
#ifndef PB_PUSH64_MIN_BLOCKS
#define PB_PUSH64_MIN_BLOCKS 1
#endif
template <typename real, bool VEC_FLUSH>
__global__ void __launch_bounds__(kTileX * kTileY * 32, sizeof(real) == 4 ? 2 : PB_PUSH64_MIN_BLOCKS)
push_tiled_kernel(Parts<real> P, TileArgs ta, Fields<real> F, Geom g, PushConst<real> pc, unsigned long long* err) {
  using S = PushSmem<real>;
  constexpr int WY = S::WY, WZ = S::WZ, WN = S::WN, WX = S::WX;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  real* win = reinterpret_cast<real*>(smem_raw);  // [4][WN]: jx, jy, jz, n
  const int tile = blockIdx.x;
  const TileGeom& t = ta.t;
  const int tz = tile % t.ntz, ty = (tile / t.ntz) % t.nty, tx = tile / (t.ntz * t.nty);
  // window origin: two nodes below the tile's first interior cell (2 + tx*TX)
  const int wx0 = tx * kTileX, wy0 = ty * kTileY, wz0 = tz * kLanes;
  for (int q = threadIdx.x; q < 4 * WN; q += blockDim.x) win[q] = (real)0;
  // FP32: E and B over the window, one plane per component
  float* fw = reinterpret_cast<float*>(smem_raw + S::fwin_off);
  // the interior cells: a particle in one needs none of the array bounds,
  // ballistic or sr_particle checks (below), wherever it sits relative to the
  // tile (testing the tile's own cells instead sent every particle that had
  // crossed into a neighbouring tile down those paths)
  const InteriorBox tb{2, 2, 2, (unsigned)g.nx, (unsigned)g.ny, (unsigned)g.nz};
  if constexpr (S::kFieldWin) fill_win<WX, WY, WZ, VEC_FLUSH>(fw, F, g, wx0, wy0, wz0);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int G = tile * (kTileX * kTileY) + warp;
  const int base = ta.goff[G], jmax = ta.gmax[G];
  // home cell of this lane
  const int hi = wx0 + 2 + warp / kTileY, hj = wy0 + 2 + warp % kTileY, hk = wz0 + 2 + lane;
  const int hcell = pack_cell(hi, hj, hk);
  real* wn = win + 3 * WN;
  // FP32: the density window holds fixed-point sums (scatter8_win_fixed) at a
  // scale that no node of this tile can overflow
  constexpr bool kFixedN = sizeof(real) == 4;
  float nscale = 0.f;
  if (kFixedN) {
    int slots = 0;
#pragma unroll
    for (int w = 0; w < kTileX * kTileY; ++w) slots += ta.gmax[tile * (kTileX * kTileY) + w];
    // below 2^23 as well, where scatter8_win_fixed's rounding by an added 2^23 is exact
    nscale = fminf(4294967295.f / (float)(slots * kLanes + 1), 8388607.f);
  }
  HomeJ<real> acc;
  acc.zero();
  // the warp's queue of J deposits off the home cells: entries [0, nq), 7
  // words each (7 is odd, so the lanes' entries fall on different banks).
  // They go to the planes with global reductions (into the shared J window by
  // FP32 shared atomics, where the stencil allowed, measured 0.7 ms per step
  // slower; z-adjacent pairs as 16-byte vector reductions, 0.2 ms slower)
  float* jq = reinterpret_cast<float*>(smem_raw + S::jq_off) + warp * S::kQ * 7;
  int nq = 0;
  auto deposit_queued = [&](int q) {
    const float* e = jq + q * 7;
    int qi, qj, qk;
    unpack_cell(__float_as_int(e[0]), qi, qj, qk);
    const Axis<real> X = axis_weights(qi, (real)e[1]), Y = axis_weights(qj, (real)e[2]), Z = axis_weights(qk, (real)e[3]);
    deposit_j(F, g, pc, X, Y, Z, (real)e[4], (real)e[5], (real)e[6]);
  };
  // ring of particle rows fetched ahead; each lane copies and reads only its
  // own slots, so the per-thread cp.async groups need no warp barrier. A
  // stage holds the row's 32 records A, then its 32 records B, so that the
  // lanes' 16-byte reads of one record fall on consecutive banks.
  real* prec = reinterpret_cast<real*>(smem_raw + S::prec_off) + warp * kStages * kLanes * 8;
  auto fetch = [&](int row) {
    if (row < jmax) {
      real* stage = prec + (row % kStages) * kLanes * 8;
      fetch_records(stage + lane * 4, stage + (kLanes + lane) * 4, P, base + row * kLanes + lane);
    }
    cp_async_commit();
  };
#pragma unroll
  for (int s = 0; s < kStages - 1; ++s) fetch(s);
  unsigned pushed = 0;
  for (int jj = 0; jj < jmax; ++jj) {
    fetch(jj + kStages - 1);
    cp_async_wait<kStages - 1>();
    const int t = base + jj * kLanes + lane;
    const int st = jj % kStages;
    real ra[4], rb[4];
    read_record(prec + st * kLanes * 8 + lane * 4, ra);
    read_record(prec + st * kLanes * 8 + (kLanes + lane) * 4, rb);
    int c;
    if constexpr (sizeof(real) == 4) c = __float_as_int((float)ra[0]);
    else c = __double2loint((double)ra[0]);
    const bool act = c >= 0;
    int i = 0, j = 0, k = 0;
    real fx = 0, fy = 0, fz = 0, vx = 0, vy = 0, vz = 0;
    bool enq = false;  // J at x^{n+1/2} goes to the warp's queue
    int chalf = 0;     // the packed cell at x^{n+1/2}
    if (act) {
      ++pushed;
      unpack_cell(c, i, j, k);
      fx = ra[1]; fy = ra[2]; fz = ra[3];
      vx = rb[0]; vy = rb[1]; vz = rb[2];
      // a particle in an interior cell has its stencils in the array, and it
      // is ballistic only when the Absorb_grid2 layer reaches interior cells
      const bool inside = tb.has(i, j, k);
      bool bal = (pc.bal_interior || !inside) && ballistic(pc, i, j, k, fx, fy, fz);
      if (!bal && !inside && !stencil_ok(g, i, j, k)) {
        count_err(err, ERR_DEPOSIT_OOB);
        bal = true;
      }
      if (!bal) {
        const Axis<real> X = axis_weights(i, fx), Y = axis_weights(j, fy), Z = axis_weights(k, fz);
        if constexpr (S::kFieldWin) {
          // the window covers the stencils of particles within two halo nodes of the tile
          const bool in_win = i - 1 >= wx0 && i + 1 < wx0 + WX && j - 1 >= wy0 && j + 1 < wy0 + WY &&
                              k - 1 >= wz0 && k + 1 < wz0 + WZ;
          if (in_win)
            boris4_fast(pc, gather6_win<WY, WZ, WN>(fw, wx0, wy0, wz0, X, Y, Z), vx, vy, vz);
          else
            boris4_fast(pc, gather6(F, g, X, Y, Z), vx, vy, vz);
        } else {
          boris4_fast(pc, gather6(F, g, X, Y, Z), vx, vy, vz);
        }
        // one test for the three: |v| < c, so the sum of finite components is finite
        if (!isfinite(vx + vy + vz)) count_err(err, ERR_NONFINITE);
      }
      advance(i, fx, vx * pc.hdt);
      advance(j, fy, vy * pc.hdt);
      advance(k, fz, vz * pc.hdt);
      // J at x^{n+1/2}
      // compared packed: a half step moves an index at most a cell past the
      // padded array, where a -1 packs negative and a kMaxDim sets a bit that
      // only an index 0 or 1 next to it could match, and home cells have indices >= 2
      chalf = pack_cell(i, j, k);
      if (chalf == hcell) {
        const Axis<real> X = axis_weights(i, fx), Y = axis_weights(j, fy), Z = axis_weights(k, fz);
        const W3<real> bx = home3(X, hi), by = home3(Y, hj), bz = home3(Z, hk);
        acc.add(pc.qn * vx, pc.qn * vy, pc.qn * vz, X, Y, Z, bx, by, bz);
      } else if (in_array(g, i, j, k)) {
        if (stencil_ok(g, i, j, k)) {
          if constexpr (S::kJQueue) {
            enq = true;
          } else {
            const Axis<real> X = axis_weights(i, fx), Y = axis_weights(j, fy), Z = axis_weights(k, fz);
            deposit_j(F, g, pc, X, Y, Z, vx, vy, vz);
          }
        } else {
          count_err(err, ERR_DEPOSIT_OOB);
        }
      }
    }
    if constexpr (S::kJQueue) {
      // warp-uniform: the row's queued lanes take consecutive entries; a full
      // warp's worth is deposited by all 32 lanes at once
      const unsigned em = __ballot_sync(0xffffffffu, enq);
      if (em) {
        if (enq) {
          float* e = jq + (nq + __popc(em & ((1u << lane) - 1u))) * 7;
          e[0] = __int_as_float(chalf);
          e[1] = (float)fx; e[2] = (float)fy; e[3] = (float)fz;
          e[4] = (float)vx; e[5] = (float)vy; e[6] = (float)vz;
        }
        nq += __popc(em);
        if (nq >= kLanes) {
          __syncwarp();
          deposit_queued(nq - kLanes + lane);
          nq -= kLanes;
          __syncwarp();
        }
      }
    }
    if (act) {
      advance(i, fx, vx * pc.hdt);
      advance(j, fy, vy * pc.hdt);
      advance(k, fz, vz * pc.hdt);
      // n at x^{n+1}
      const bool inside1 = tb.has(i, j, k);
      if (inside1 || in_array(g, i, j, k)) {
        if (inside1 || stencil_ok(g, i, j, k)) {
          const Axis<real> X = axis_weights(i, fx), Y = axis_weights(j, fy), Z = axis_weights(k, fz);
          if constexpr (kFixedN)
            scatter8_win_fixed(reinterpret_cast<unsigned*>(wn), wx0, wy0, wz0, F.f[pc.pn], g, X.b, Y.b, Z.b,
                               pc.nw, nscale, X.b0, X.b1, Y.b0, Y.b1, Z.b0, Z.b1);
          else
            scatter8_win(wn, wx0, wy0, wz0, F.f[pc.pn], g, X.b, Y.b, Z.b, pc.nw, X.b0, X.b1, Y.b0, Y.b1, Z.b0, Z.b1);
        } else {
          count_err(err, ERR_DEPOSIT_OOB);
        }
      }
      // sr_particle keeps a particle of an interior cell where it is
      const int cnew = inside1 ? pack_cell(i, j, k) : settle(g, pc.out, i, j, k, fx, fy, fz, vx, vy, vz, err);
      store_records(P, t, cnew, fx, fy, fz, vx, vy, vz);
    }
  }
  if constexpr (S::kJQueue) {
    __syncwarp();
    if (lane < nq) deposit_queued(lane);
  }
  for (int o = 16; o > 0; o >>= 1) pushed += __shfl_down_sync(0xffffffffu, pushed, o);
  if (lane == 0 && pushed) atomicAdd(err + CNT_PUSHED, (unsigned long long)pushed);
  // the lane's home-cell sums into the window (nodes h-1 .. h+1 around it)
  if (jmax > 0) {
    const int la = hi - 1 - wx0, lb = hj - 1 - wy0, lc = hk - 1 - wz0;  // window index of node h-1
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
          const int s = ((la + a) * WY + (lb + b)) * WZ + (lc + cc);
          if (a < 2) atomicAdd(win + s + WY * WZ, acc.x(a, b, cc));       // x nodes h, h+1
          if (b < 2) atomicAdd(win + WN + s + WZ, acc.y(a, b, cc));       // y nodes h, h+1
          if (cc < 2) atomicAdd(win + 2 * WN + s + 1, acc.z(a, b, cc));   // z nodes h, h+1
        }
  }
  __syncthreads();
  // flush the window: one reduction per 4 consecutive z nodes
  const int planes[4] = {pc.pjx, pc.pjy, pc.pjz, pc.pn};
  constexpr int NZ4 = WZ / 4;
  for (int q4 = threadIdx.x; q4 < 4 * WX * WY * NZ4; q4 += blockDim.x) {
    const int q = q4 / (WX * WY * NZ4);
    const int r = q4 % (WX * WY * NZ4);
    const int a = r / (WY * NZ4), b = (r / NZ4) % WY, c4 = r % NZ4;
    const int ga = wx0 + a, gb = wy0 + b, gc = wz0 + 4 * c4;
    if (ga >= g.gx || gb >= g.gy || gc >= g.gz) continue;
    const real* src = win + q * WN + (a * WY + b) * WZ + 4 * c4;
    real v0 = src[0], v1 = src[1], v2 = src[2], v3 = src[3];
    if (kFixedN && q == 3) {  // fixed-point density sums back to weights
      const unsigned* u = reinterpret_cast<const unsigned*>(src);
      const real back = pc.nw / (real)nscale;
      v0 = (real)u[0] * back; v1 = (real)u[1] * back; v2 = (real)u[2] * back; v3 = (real)u[3] * back;
    }
    if (v0 == (real)0 && v1 == (real)0 && v2 == (real)0 && v3 == (real)0) continue;
    real* dst = F.f[planes[q]] + ga * g.sx + gb * g.gz + gc;
    if (VEC_FLUSH) {
      red_add_v4(reinterpret_cast<float*>(dst), (float)v0, (float)v1, (float)v2, (float)v3);
    } else {
      const real v[4] = {v0, v1, v2, v3};
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (gc + e < g.gz && v[e] != (real)0) atomicAdd(dst + e, v[e]);
    }
  }
}


}  // namespace pb
