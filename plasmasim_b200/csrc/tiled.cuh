// Tiled particle layout and the fused push kernel that uses it.
//
// Layout. The interior cells are cut into tiles of TX x TY x 32 cells (x, y,
// z). Each (x, y) column of a tile -- 32 consecutive z cells -- is a "group"
// handled by one warp, lane L owning cell z0 + L. A sort writes the particles
// of a group interleaved: particle r of the cell in lane L goes to slot
// goff[G] + 32 r + L, every lane's column padded with empty slots (cell = -1)
// up to the group's largest cell count gmax[G]. A warp then reads 32
// consecutive slots per step of its loop (one coalesced 128-byte line per
// array) and its 32 lanes work on 32 different cells, so their shared-memory
// deposits rarely hit the same address.
//
// Deposit. Each CTA accumulates J and n of its species in a shared-memory
// window of (TX+4) x (TY+4) x 36 nodes around its tile (the stencil of a
// particle that has moved up to one cell from its tile since the sort), then
// adds the window to the global planes with one vector reduction per 4 nodes.
// Deposits whose stencil leaves the window (particles wrapped through the
// periodic boundary, or moved farther since the sort) go straight to global
// memory with atomics.
#pragma once

#include "common.cuh"
#include "particles.cuh"

namespace pb {

constexpr int kTileX = 2;
constexpr int kTileY = 4;
constexpr int kLanes = 32;
constexpr int kWinZ = kLanes + 4;

struct TileGeom {
  int ntx, nty, ntz;  // tiles per axis
  int ngroups;        // ntx * nty * ntz * kTileX * kTileY
};

struct TileArgs {
  TileGeom t;
  const int* goff;  // first slot of each group
  const int* gmax;  // slots per lane of each group
};

// Group and lane of an interior cell (absolute indices), -1 outside the interior.
__device__ __forceinline__ int group_of(const Geom& g, const TileGeom& t, int i, int j, int k,
                                        int& lane) {
  i -= 2; j -= 2; k -= 2;
  if (i < 0 || j < 0 || k < 0 || i >= g.nx || j >= g.ny || k >= g.nz) return -1;
  const int tx = i / kTileX, wx = i % kTileX, ty = j / kTileY, wy = j % kTileY;
  const int tz = k >> 5;
  lane = k & 31;
  const int tile = (tx * t.nty + ty) * t.ntz + tz;
  return tile * (kTileX * kTileY) + wx * kTileY + wy;
}

// One warp per group: gmax = largest cell count of its 32 lanes.
__global__ void group_size_kernel(Geom g, TileGeom t, const int* __restrict__ cnt, int* gmax,
                                  int* gcap) {
  const int G = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (G >= t.ngroups) return;
  const int tile = G / (kTileX * kTileY), w = G % (kTileX * kTileY);
  const int tz = tile % t.ntz, ty = (tile / t.ntz) % t.nty, tx = tile / (t.ntz * t.nty);
  const int i = tx * kTileX + w / kTileY, j = ty * kTileY + w % kTileY, k = tz * kLanes + lane;
  int c = 0;
  if (i < g.nx && j < g.ny && k < g.nz) c = cnt[(i * g.ny + j) * g.nz + k];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c = max(c, __shfl_xor_sync(0xffffffffu, c, o));
  if (lane == 0) {
    gmax[G] = c;
    gcap[G] = c * kLanes;
  }
}

// Marks the padding slots of every lane column empty.
__global__ void group_pad_kernel(Geom g, TileGeom t, const int* __restrict__ cnt,
                                 const int* __restrict__ goff, const int* __restrict__ gmax, int* cell) {
  const int G = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (G >= t.ngroups) return;
  const int tile = G / (kTileX * kTileY), w = G % (kTileX * kTileY);
  const int tz = tile % t.ntz, ty = (tile / t.ntz) % t.nty, tx = tile / (t.ntz * t.nty);
  const int i = tx * kTileX + w / kTileY, j = ty * kTileY + w % kTileY, k = tz * kLanes + lane;
  int c = 0;
  if (i < g.nx && j < g.ny && k < g.nz) c = cnt[(i * g.ny + j) * g.nz + k];
  const int m = gmax[G], base = goff[G];
  for (int r = c; r < m; ++r) cell[base + r * kLanes + lane] = -1;
}

template <typename real>
__global__ void tiled_scatter_kernel(Parts<real> P, const int* __restrict__ count, Geom g, TileGeom t,
                                     const int* __restrict__ goff, int* cursor, Parts<real> Q) {
  const int n = *count;
  const int stride = gridDim.x * blockDim.x;
  const int n_round = (n + 31) & ~31;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n_round; s += stride) {
    int key = -1, G = -1, lane = 0;
    int c = -1;
    if (s < n) {
      c = P.cell[s];
      key = interior_key(g, c);
      if (key >= 0) {
        int i, j, k;
        unpack_cell(c, i, j, k);
        G = group_of(g, t, i, j, k, lane);
      }
    }
    const int r = warp_aggregated_inc(cursor, key < 0 ? 0 : key, key >= 0);
    if (key >= 0) {
      const int d = goff[G] + r * kLanes + lane;
      Q.cell[d] = c;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        Q.o[a][d] = P.o[a][s];
        Q.v[a][d] = P.v[a][s];
      }
    }
  }
}

__global__ void tiled_total_kernel(const int* goff, const int* gcap, int ngroups, int* count_dev) {
  *count_dev = goff[ngroups - 1] + gcap[ngroups - 1];
}

// ------------------------------------------------------------ the push
__device__ __forceinline__ void red_add_v4(float* p, float a, float b, float c, float d) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};"
               :: "l"(p), "f"(a), "f"(b), "f"(c), "f"(d) : "memory");
}

// Window deposit of the 2x2x2 stencil at global base node (a, b, c); falls
// back to global atomics when the stencil leaves the window.
template <typename real>
__device__ __forceinline__ void scatter8_win(real* win, int wx0, int wy0, int wz0, real* gplane,
                                             const Geom& g, int a, int b, int c, real v, real x0,
                                             real x1, real y0, real y1, real z0, real z1) {
  constexpr int WY = kTileY + 4, WZ = kWinZ, WX = kTileX + 4;
  const int la = a - wx0, lb = b - wy0, lc = c - wz0;
  if (la >= 0 && la <= WX - 2 && lb >= 0 && lb <= WY - 2 && lc >= 0 && lc <= WZ - 2) {
    const int s = (la * WY + lb) * WZ + lc;
    const real a0 = v * x0, a1 = v * x1;
    const real a00 = a0 * y0, a01 = a0 * y1, a10 = a1 * y0, a11 = a1 * y1;
    atomicAdd(win + s, a00 * z0);
    atomicAdd(win + s + 1, a00 * z1);
    atomicAdd(win + s + WZ, a01 * z0);
    atomicAdd(win + s + WZ + 1, a01 * z1);
    atomicAdd(win + s + WY * WZ, a10 * z0);
    atomicAdd(win + s + WY * WZ + 1, a10 * z1);
    atomicAdd(win + s + WY * WZ + WZ, a11 * z0);
    atomicAdd(win + s + WY * WZ + WZ + 1, a11 * z1);
  } else {
    scatter8(gplane, a * g.sx + b * g.gz + c, g.sx, g.gz, v, x0, x1, y0, y1, z0, z1);
  }
}

// The fused particle part of one step (push, J deposit at x^{n+1/2}, drift,
// n deposit at x^{n+1}, sr_particle) for one species over the tiled layout;
// same arithmetic as push_kernel<real, PUSH_FUSED>. One CTA per tile.
template <typename real, bool VEC_FLUSH>
__global__ void __launch_bounds__(kTileX * kTileY * 32)
push_tiled_kernel(Parts<real> P, TileArgs ta, Fields<real> F, Geom g, PushConst<real> pc,
                  unsigned long long* err) {
  constexpr int WX = kTileX + 4, WY = kTileY + 4, WZ = kWinZ, WN = WX * WY * WZ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  real* win = reinterpret_cast<real*>(smem_raw);  // [4][WN]: jx, jy, jz, n
  const int tile = blockIdx.x;
  const TileGeom& t = ta.t;
  const int tz = tile % t.ntz, ty = (tile / t.ntz) % t.nty, tx = tile / (t.ntz * t.nty);
  // window origin: two nodes below the tile's first interior cell (2 + tx*TX)
  const int wx0 = tx * kTileX, wy0 = ty * kTileY, wz0 = tz * kLanes;
  for (int q = threadIdx.x; q < 4 * WN; q += blockDim.x) win[q] = (real)0;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int G = tile * (kTileX * kTileY) + warp;
  const int base = ta.goff[G], jmax = ta.gmax[G];
  real* wjx = win;
  real* wjy = win + WN;
  real* wjz = win + 2 * WN;
  real* wn = win + 3 * WN;
  unsigned pushed = 0;
  for (int jj = 0; jj < jmax; ++jj) {
    const int t = base + jj * kLanes + lane;
    const int c = P.cell[t];
    if (c < 0) continue;
    ++pushed;
    int i, j, k;
    unpack_cell(c, i, j, k);
    real fx = P.o[0][t], fy = P.o[1][t], fz = P.o[2][t];
    real vx = P.v[0][t], vy = P.v[1][t], vz = P.v[2][t];
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
        scatter8_win(wjx, wx0, wy0, wz0, F.f[pc.pjx], g, X.a, Y.b, Z.b, pc.qn * vx, X.a0, X.a1, Y.b0, Y.b1, Z.b0, Z.b1);
        scatter8_win(wjy, wx0, wy0, wz0, F.f[pc.pjy], g, X.b, Y.a, Z.b, pc.qn * vy, X.b0, X.b1, Y.a0, Y.a1, Z.b0, Z.b1);
        scatter8_win(wjz, wx0, wy0, wz0, F.f[pc.pjz], g, X.b, Y.b, Z.a, pc.qn * vz, X.b0, X.b1, Y.b0, Y.b1, Z.a0, Z.a1);
      } else {
        count_err(err, ERR_DEPOSIT_OOB);
      }
    }
    advance(i, fx, vx * pc.hdt);
    advance(j, fy, vy * pc.hdt);
    advance(k, fz, vz * pc.hdt);
    if (in_array(g, i, j, k)) {
      if (stencil_ok(g, i, j, k)) {
        const Axis<real> X = axis_weights(i, fx), Y = axis_weights(j, fy), Z = axis_weights(k, fz);
        scatter8_win(wn, wx0, wy0, wz0, F.f[pc.pn], g, X.b, Y.b, Z.b, pc.nw, X.b0, X.b1, Y.b0, Y.b1, Z.b0, Z.b1);
      } else {
        count_err(err, ERR_DEPOSIT_OOB);
      }
    }
    P.cell[t] = boundary(g, i, j, k) ? repack(i, j, k, err) : -1;
    P.o[0][t] = fx; P.o[1][t] = fy; P.o[2][t] = fz;
    P.v[0][t] = vx; P.v[1][t] = vy; P.v[2][t] = vz;
  }
  for (int o = 16; o > 0; o >>= 1) pushed += __shfl_down_sync(0xffffffffu, pushed, o);
  if (lane == 0 && pushed) atomicAdd(err + CNT_PUSHED, (unsigned long long)pushed);
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
    const real v0 = src[0], v1 = src[1], v2 = src[2], v3 = src[3];
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
