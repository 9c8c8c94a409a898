// Tiled particle layout and its incremental sort (the push kernel that uses
// the layout is in push_tiled.cuh).
//
// Layout. The interior cells are cut into tiles of TX x TY x 32 cells (x, y,
// z). Each (x, y) column of a tile -- 32 consecutive z cells -- is a "group"
// handled by one warp, lane L owning cell z0 + L (its "home" cell). A sort
// writes the particles of a group interleaved: particle r of the cell in lane
// L goes to slot goff[G] + 32 r + L, every lane's column padded with empty
// slots (cell = -1) up to the group's largest cell count gmax[G]. A warp then
// reads 32 consecutive slots per step of its loop (one coalesced 128-byte line
// per array) and its 32 lanes work on 32 different cells.
//
// Deposit. A lane accumulates the current of the particles that are in its
// home cell in registers (the 2x3x3 / 3x2x3 / 3x3x2 nodes such a particle can
// touch) and adds them to a shared-memory window of (TX+4) x (TY+4) x 36 nodes
// once, after its last particle. The current of particles that have left
// their home cell since the sort, and every density deposit, go to the window
// with shared atomics, or, when the stencil leaves the window (periodic wrap,
// long moves), to global memory with atomics. The window is added to the
// global planes with one vector reduction per 4 nodes.
//
// Sort. Between sorts most particles stay in their cell. The sort keeps the
// order of those "stayers" within their lane column (a warp walks its columns
// row by row, so stayers are written in order without atomics, into nearly
// the same 128-byte lines they came from) and places the others -- movers,
// and particles appended by a refill -- after the stayers of their new cell
// with per-cell atomic cursors.
#pragma once

#include "common.cuh"
#include "particles.cuh"

namespace pb {

// Layout slack of a full sort: rows added to a group beyond its fullest lane,
// count / kSlackDiv + kSlackRows (a slack of count / 32 measured no faster).
constexpr int kSlackDiv = 16;
constexpr int kSlackRows = 2;

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

// Interior cell key of group G's lane, or -1 when the lane has no cell.
__device__ __forceinline__ int home_key(const Geom& g, const TileGeom& t, int G, int lane) {
  const int tile = G / (kTileX * kTileY), w = G % (kTileX * kTileY);
  const int tz = tile % t.ntz, ty = (tile / t.ntz) % t.nty, tx = tile / (t.ntz * t.nty);
  const int i = tx * kTileX + w / kTileY, j = ty * kTileY + w % kTileY, k = tz * kLanes + lane;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return -1;
  return (i * g.ny + j) * g.nz + k;
}

// Group and lane of an interior cell key.
__device__ __forceinline__ int group_of_key(const Geom& g, const TileGeom& t, int key, int& lane) {
  const int k = key % g.nz, j = (key / g.nz) % g.ny, i = key / (g.nz * g.ny);
  return group_of(g, t, i + 2, j + 2, k + 2, lane);
}

// --------------------------------------------------------------- sort
// Counting: stayers per home cell (no atomics) over the tiled slots, movers
// and appended particles per destination cell (atomics).
template <typename real>
__global__ void tiled_count_kernel(Parts<real> P, Geom g, TileGeom t, const int* __restrict__ goff,
                                   const int* __restrict__ gmax, int* stay, int* moved) {
  const int G = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (G >= t.ngroups) return;
  const int home = home_key(g, t, G, lane);
  const int base = goff[G], m = gmax[G];
  int nstay = 0;
  constexpr int U = 8;  // rows whose loads are in flight together
  for (int r0 = 0; r0 < m; r0 += U) {
    int cell[U];
#pragma unroll
    for (int u = 0; u < U; ++u) cell[u] = r0 + u < m ? P.cell[base + (r0 + u) * kLanes + lane] : -1;
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int key = interior_key(g, cell[u]);
      if (key < 0) continue;
      if (key == home) ++nstay;
      else atomicAdd(moved + key, 1);
    }
  }
  if (home >= 0) stay[home] = nstay;
}

template <typename real>
__global__ void append_count_kernel(Parts<real> P, int first, const int* __restrict__ count, Geom g,
                                    int* moved) {
  const int n = *count;
  for (int s = first + blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const int key = interior_key(g, P.cell[s]);
    if (key >= 0) atomicAdd(moved + key, 1);
  }
}

// Absolute indices of group G's lane cell; false when the lane has no cell.
__device__ __forceinline__ bool home_cell(const Geom& g, const TileGeom& t, int G, int lane, int& i,
                                          int& j, int& k) {
  const int tile = G / (kTileX * kTileY), w = G % (kTileX * kTileY);
  const int tz = tile % t.ntz, ty = (tile / t.ntz) % t.nty, tx = tile / (t.ntz * t.nty);
  i = tx * kTileX + w / kTileY;
  j = ty * kTileY + w % kTileY;
  k = tz * kLanes + lane;
  const bool ok = i < g.nx && j < g.ny && k < g.nz;
  i += 2; j += 2; k += 2;
  return ok;
}

// Rows a lane column keeps for the boundary refill of its cell: the refill's
// particle count plus an eighth and four, so that the refill fits into the
// column's empty slots without moving other particles.
__device__ __forceinline__ int refill_reserve(const SourceParams& sp, const Geom& g, const TileGeom& t,
                                              int G, int lane) {
  int i, j, k;
  if (!home_cell(g, t, G, lane, i, j, k)) return 0;
  const int need = slab_need(sp, i, j, k);
  return need > 0 ? need + need / 8 + 4 : 0;
}

// One warp per group: gmax = largest (stayers + movers) count of its 32
// lanes, or a lane's refill reserve when that is larger, plus a sixteenth and
// two rows of slack: the fullest columns then take the next re-layouts'
// arrivals in holes instead of spilling them to the slot-order tail.
__global__ void group_size_kernel(Geom g, TileGeom t, const int* __restrict__ stay,
                                  const int* __restrict__ moved, SourceParams refill, int* gmax,
                                  int* gcap) {
  const int G = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (G >= t.ngroups) return;
  const int home = home_key(g, t, G, lane);
  int c = home >= 0 ? stay[home] + moved[home] : 0;
  c = max(c, refill_reserve(refill, g, t, G, lane));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c = max(c, __shfl_xor_sync(0xffffffffu, c, o));
  if (c > 0) c += c / kSlackDiv + kSlackRows;
  if (lane == 0) {
    gmax[G] = c;
    gcap[G] = c * kLanes;
  }
}

// Marks the padding slots of every lane column empty.
template <typename CellArray>
__global__ void group_pad_kernel(Geom g, TileGeom t, const int* __restrict__ stay,
                                 const int* __restrict__ moved, const int* __restrict__ goff,
                                 const int* __restrict__ gmax, CellArray cell) {
  const int G = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (G >= t.ngroups) return;
  const int home = home_key(g, t, G, lane);
  const int c = home >= 0 ? stay[home] + moved[home] : 0;
  const int m = gmax[G], base = goff[G];
  for (int r = c; r < m; ++r) cell[base + r * kLanes + lane] = -1;
}

template <typename real>
__device__ __forceinline__ void copy_particle(const Parts<real>& P, int s, const Parts<real>& Q, int d,
                                              int c) {
  copy_record(P, s, Q, d, c);
}

// Scatter over the tiled slots: a stayer keeps its place in its column order;
// a mover goes after the stayers of its new cell.
template <typename real>
__global__ void tiled_scatter_kernel(Parts<real> P, Geom g, TileGeom t, const int* __restrict__ goff_old,
                                     const int* __restrict__ gmax_old, const int* __restrict__ goff_new,
                                     const int* __restrict__ stay, int* cursor, Parts<real> Q) {
  const int G = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (G >= t.ngroups) return;
  const int home = home_key(g, t, G, lane);
  const int base = goff_old[G], m = gmax_old[G], nbase = goff_new[G];
  int rnew = 0;
  constexpr int U = 4;  // rows whose loads are in flight together
  for (int r0 = 0; r0 < m; r0 += U) {
    int cell[U];
    real o[U][3], v[U][3];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int s = base + (r0 + u) * kLanes + lane;
      const bool in = r0 + u < m;
      cell[u] = in ? P.cell[s] : -1;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        o[u][a] = in ? P.o[a][s] : (real)0;
        v[u][a] = in ? P.v[a][s] : (real)0;
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int key = interior_key(g, cell[u]);
      if (key < 0) continue;
      int d;
      if (key == home) {
        d = nbase + rnew * kLanes + lane;
        ++rnew;
      } else {
        int l2;
        const int G2 = group_of_key(g, t, key, l2);
        const int rank = stay[key] + atomicAdd(cursor + key, 1);
        d = goff_new[G2] + rank * kLanes + l2;
      }
      Q.cell[d] = cell[u];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        Q.o[a][d] = o[u][a];
        Q.v[a][d] = v[u][a];
      }
    }
  }
}

template <typename real>
__global__ void append_scatter_kernel(Parts<real> P, int first, const int* __restrict__ count, Geom g,
                                      TileGeom t, const int* __restrict__ goff_new,
                                      const int* __restrict__ stay, int* cursor, Parts<real> Q) {
  const int n = *count;
  for (int s = first + blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const int c = P.cell[s];
    const int key = interior_key(g, c);
    if (key < 0) continue;
    int l2;
    const int G2 = group_of_key(g, t, key, l2);
    const int rank = stay[key] + atomicAdd(cursor + key, 1);
    copy_particle(P, s, Q, goff_new[G2] + rank * kLanes + l2, c);
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

// Density deposit into a fixed-point window: the 2x2x2 area weights (each in
// [0, 1], summing to 1) scaled by `scale` and rounded, added with integer
// shared-memory reductions, which need no compare-and-swap loop and give a sum
// that does not depend on the order of the particles. The caller picks `scale`
// so that no node can overflow: a node collects at most one unit of weight from
// each particle of the tile, so scale = (2^32 - 1) / (slots + 1) is safe; it is
// also kept below 2^23 for the rounding below. With 64 particles per cell this
// resolves 2^-17.7 of a particle's weight, as fine as an FP32 sum of the same
// node. The stencil falls back to FP32 global
// atomics (weight v) when it leaves the window.
__device__ __forceinline__ void red_shared_u32(const unsigned* p, unsigned v) {
  asm volatile("red.shared.add.u32 [%0], %1;" :: "r"((unsigned)__cvta_generic_to_shared(p)), "r"(v) : "memory");
}

__device__ __forceinline__ void scatter8_win_fixed(unsigned* win, int wx0, int wy0, int wz0, float* gplane,
                                                   const Geom& g, int a, int b, int c, float v, float scale,
                                                   float x0, float x1, float y0, float y1, float z0, float z1) {
  constexpr int WY = kTileY + 4, WZ = kWinZ, WX = kTileX + 4;
  const int la = a - wx0, lb = b - wy0, lc = c - wz0;
  if (la >= 0 && la <= WX - 2 && lb >= 0 && lb <= WY - 2 && lc >= 0 && lc <= WZ - 2) {
    const unsigned* s = win + (la * WY + lb) * WZ + lc;
    // the eight node weights (each in [0, scale], scale < 2^23) rounded to
    // integers by adding 2^23 in the FMA: the sum's low mantissa bits are then
    // the rounded weight, with no float-to-integer conversion; the two x
    // planes travel as one packed pair
    constexpr float kM = 8388608.f;                 // 2^23
    constexpr unsigned kMBits = 0x4B000000u;        // its bit pattern
    const float2 M = make_float2(kM, kM);
    const float2 ax = __fmul2_rn(make_float2(x0, x1), make_float2(scale, scale));
    const float2 ay0 = __fmul2_rn(ax, make_float2(y0, y0));  // (a00, a10)
    const float2 ay1 = __fmul2_rn(ax, make_float2(y1, y1));  // (a01, a11)
    const float2 Z0 = make_float2(z0, z0), Z1 = make_float2(z1, z1);
    const float2 t00 = __ffma2_rn(ay0, Z0, M), t01 = __ffma2_rn(ay0, Z1, M);
    const float2 t10 = __ffma2_rn(ay1, Z0, M), t11 = __ffma2_rn(ay1, Z1, M);
    red_shared_u32(s, __float_as_uint(t00.x) - kMBits);
    red_shared_u32(s + 1, __float_as_uint(t01.x) - kMBits);
    red_shared_u32(s + WZ, __float_as_uint(t10.x) - kMBits);
    red_shared_u32(s + WZ + 1, __float_as_uint(t11.x) - kMBits);
    red_shared_u32(s + WY * WZ, __float_as_uint(t00.y) - kMBits);
    red_shared_u32(s + WY * WZ + 1, __float_as_uint(t01.y) - kMBits);
    red_shared_u32(s + WY * WZ + WZ, __float_as_uint(t10.y) - kMBits);
    red_shared_u32(s + WY * WZ + WZ + 1, __float_as_uint(t11.y) - kMBits);
  } else {
    scatter8(gplane, a * g.sx + b * g.gz + c, g.sx, g.gz, v, x0, x1, y0, y1, z0, z1);
  }
}

// Half-shifted weights of a particle in its home cell h as a 3-vector over the
// nodes h-1, h, h+1 (its base is h-1 for an offset below 1/2, h otherwise).
template <typename real>
struct W3 {
  real w[3];
};
template <typename real>
__device__ __forceinline__ W3<real> home3(const Axis<real>& A, int h) {
  W3<real> r;
  const bool up = A.b == h;
  r.w[0] = up ? (real)0 : A.b0;
  r.w[1] = up ? A.b0 : A.b1;
  r.w[2] = up ? A.b1 : (real)0;
  return r;
}
// FP32: the same three weights straight from the offset f = A.a1 of a
// particle in its home cell (an interior cell, so never cell 0): with
// g = f - 1/2 they are (max(-g, 0), 1 - |g|, max(g, 0)), equal to the form
// above to within a rounding, in four instructions instead of the base
// choice and three selects.
__device__ __forceinline__ W3<float> home3(const Axis<float>& A, int) {
  const float g = A.a1 - 0.5f;
  W3<float> r;
  r.w[0] = fmaxf(-g, 0.f);
  r.w[1] = 1.f - fabsf(g);
  r.w[2] = fmaxf(g, 0.f);
  return r;
}

// cal_track4's square roots and divisions: exact in FP64, rsqrt/fast
// reciprocal in FP32 (relative error ~1e-7, below the FP32 path's tolerance).
__device__ __forceinline__ float c_over_sqrt(float c, float x) { return c * rsqrtf(x); }
__device__ __forceinline__ double c_over_sqrt(double c, double x) { return c / sqrt(x); }
__device__ __forceinline__ float quot(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double quot(double a, double b) { return a / b; }

template <typename real>
__device__ __forceinline__ void boris4_fast(const PushConst<real>& pc, Gathered<real> e, real& vx,
                                            real& vy, real& vz) {
  const real T = pc.T, C = pc.C;
  e.ex += pc.ex_add;
  e.ey += pc.ey_add;
  real g1 = c_over_sqrt(C, pc.C2 - vx * vx - vy * vy - vz * vz);
  if (isnan(g1)) g1 = (real)0;
  real ux = g1 * vx, uy = g1 * vy, uz = g1 * vz;
  real g2 = c_over_sqrt(C, pc.C2 + ux * ux + uy * uy + uz * uz);
  const real bux = g2 * e.bx, buy = g2 * e.by, buz = g2 * e.bz;
  const real S = quot((real)2 * T, (real)1 + T * T * (bux * bux + buy * buy + buz * buz));
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
  g2 = c_over_sqrt(C, pc.C2 + upx * upx + upy * upy + upz * upz);
  vx = g2 * upx;
  vy = g2 * upy;
  vz = g2 * upz;
}


}  // namespace pb
