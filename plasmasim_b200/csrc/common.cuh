// Shared device-side definitions for the B200 PIC step.
//
// Grid layout in HBM: one plane per field component over the padded
// (nx+4)*(ny+4)*(nz+4) node array, node index (i*gy + j)*gz + k with k (the
// reference's z, its solar-wind axis) fastest, as grid[k][l][m] of
// PIC/3d_pic458_domain.c:147. Planes are padded to 256-byte boundaries.
//
// Particle layout: structure of arrays per species,
//   cell : int32, (i << 20) | (j << 10) | k, the containing cell of the padded
//          grid (i = floor(x/dx)), -1 for an empty slot
//   ox, oy, oz : in-cell offsets in [0, 1) (x = (i + ox) dx)
//   vx, vy, vz : velocities in the caller's units
// 28 bytes per particle in FP32, 52 in FP64.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace pb {

constexpr int kCellBits = 10;
constexpr int kCellMask = (1 << kCellBits) - 1;
constexpr int kMaxDim = 1 << kCellBits;  // padded extent limit per axis

__host__ __device__ __forceinline__ int pack_cell(int i, int j, int k) {
  return (i << (2 * kCellBits)) | (j << kCellBits) | k;
}
__host__ __device__ __forceinline__ void unpack_cell(int c, int& i, int& j, int& k) {
  i = c >> (2 * kCellBits);
  j = (c >> kCellBits) & kCellMask;
  k = c & kCellMask;
}

struct Geom {
  int nx, ny, nz;   // interior cells
  int gx, gy, gz;   // padded extents (n + 4)
  int sx;           // node stride of i (gy * gz)
  int nodes;        // gx * gy * gz
  // the x-y decomposition (PROCESS_Nx x PROCESS_Ny, :100-101): this rank's
  // first global cell (myrank_x Grid_Nx, myrank_y Grid_Ny), the global
  // interior, and whether the rank holds the global low / high face of x, y
  int ox, oy;
  int gnx, gny;
  int xlo, xhi, ylo, yhi;
};

// Field components stored as planes. B is the total field used by the gather,
// DB = B - B0 the induced part the curl updates work on.
enum FieldId {
  F_EX, F_EY, F_EZ, F_BX, F_BY, F_BZ, F_DBX, F_DBY, F_DBZ, F_B0X, F_B0Y, F_B0Z,
  F_JIX, F_JIY, F_JIZ, F_JEX, F_JEY, F_JEZ, F_NI, F_NE, F_PHI, F_COUNT
};

template <typename real>
struct Fields {
  real* f[F_COUNT];
};

// Element t of an array whose elements lie S values of T apart.
template <typename T, int S>
struct Strided {
  T* p;
  __host__ __device__ __forceinline__ T& operator[](long long t) const { return p[t * S]; }
};

template <typename real>
struct Parts {
  // two 4-value records per particle: A = (cell, ox, oy, oz), the cell index
  // in A's first 4 bytes, and B = (vx, vy, vz, unused); 16 bytes each in FP32,
  // 32 in FP64, so that a particle moves with two vector copies
  static constexpr int kCellStride = 4 * (int)sizeof(real) / (int)sizeof(int);
  real* ra;
  real* rb;
  Strided<int, kCellStride> cell;  // cell[t], o[a][t], v[a][t]: one quantity of particle t
  Strided<real, 4> o[3];
  Strided<real, 4> v[3];
};

template <typename real>
__host__ __device__ __forceinline__ Parts<real> make_parts(real* ra, real* rb) {
  Parts<real> P;
  P.ra = ra;
  P.rb = rb;
  P.cell.p = reinterpret_cast<int*>(ra);
  for (int a = 0; a < 3; ++a) {
    P.o[a].p = ra + 1 + a;
    P.v[a].p = rb + a;
  }
  return P;
}

// Bytes of the records of `cap` particles (A array, then B array).
__host__ __device__ __forceinline__ size_t parts_record_bytes(long long cap, size_t rsize) {
  return (((size_t)cap * 4 * rsize + 255) & ~(size_t)255);
}

// Device error counters (see pic_status).
enum ErrId {
  ERR_DEPOSIT_OOB = 0, ERR_CELL_RANGE = 1, ERR_NONFINITE = 2,
  ERR_FIRST_INFO = 3, CNT_PUSHED = 3,  // slots from here on count work, not errors
  ERR_MIGRATION = 4,  // sr_particle packets lost to a full exchange buffer (an error)
  ERR_FIELD_WAIT = 5,  // staged field tiles whose tensor loads did not arrive in time (an error)
  ERR_STORE_FULL = 6,  // refilled particles lost to a full particle store (an error)
  ERR_COUNT = 8
};

// ---------------------------------------------------------------- Philox
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): the random streams that
// replace the reference's gsl_rng objects. Draw d of the stream keyed by seed
// uses block d/2 and the word pair d&1; a draw is a 53-bit uniform in [0, 1).
__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
    c[1] = (uint32_t)p1;
    c[3] = (uint32_t)p0;
    c[0] = n0;
    c[2] = n2;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

__host__ __device__ __forceinline__ double uniform53(uint64_t seed, uint64_t d) {
  uint32_t c[4] = {(uint32_t)(d >> 1), (uint32_t)(d >> 33), 0u, 0u};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const uint32_t a = (d & 1) ? c[2] : c[0];
  const uint32_t b = (d & 1) ? c[3] : c[1];
  const uint64_t m = ((uint64_t)a << 21) | (uint64_t)(b >> 11);
  return (double)m * (1.0 / 9007199254740992.0);
}

// The uniform53 values of draws d .. d + N - 1 of a stream with each Philox
// block computed once: draw d is the 53 bits of words (0, 1) of block d >> 1
// for even d and of words (2, 3) for odd d, so N consecutive draws need
// N / 2 + 1 blocks at most instead of N. `odd` is d's parity; callers whose
// d has the same parity in every thread of a launch keep the blocks uniform.
__host__ __device__ __forceinline__ double u53_words(uint32_t a, uint32_t b) {
  const uint64_t m = ((uint64_t)a << 21) | (uint64_t)(b >> 11);
  return (double)m * (1.0 / 9007199254740992.0);
}
template <int N>
__host__ __device__ __forceinline__ void uniform53_run(uint64_t seed, uint64_t d, double (&u)[N]) {
  constexpr int kBlocks = N / 2 + 1;
  uint32_t c[kBlocks][4];
#pragma unroll
  for (int q = 0; q < kBlocks; ++q) {
    const uint64_t blk = (d >> 1) + (uint64_t)q;
    c[q][0] = (uint32_t)blk;
    c[q][1] = (uint32_t)(blk >> 32);
    c[q][2] = 0u;
    c[q][3] = 0u;
    if (q < (N + (int)(d & 1) + 1) / 2) philox4x32_10(c[q], (uint32_t)seed, (uint32_t)(seed >> 32));
  }
  const int odd = (int)(d & 1);
#pragma unroll
  for (int q = 0; q < N; ++q) {
    const int w = q + odd;  // word pair of draw d + q, counted from block d >> 1
    u[q] = (w & 1) ? u53_words(c[w >> 1][2], c[w >> 1][3]) : u53_words(c[w >> 1][0], c[w >> 1][1]);
  }
}

#ifdef __CUDACC__
// a*(1-u) + b*u rounded step by step (no contraction), as the host computes it.
__device__ __forceinline__ double flat_rn(double a, double b, double u) {
  return __dadd_rn(__dmul_rn(a, __dadd_rn(1.0, -u)), __dmul_rn(b, u));
}

// Box-Muller from two uniforms v1, v2 (draws d and d+1 of a stream):
// sqrt(-2 ln(1-v1)) cos(2 pi v2).
__device__ __forceinline__ double gauss_bm_u(double v1, double v2) {
  const double u1 = __dadd_rn(1.0, -v1);
  const double r = sqrt(__dmul_rn(-2.0, log(u1)));
  const double ang = __dmul_rn(__dmul_rn(2.0, 3.14159265358979323846), v2);
  return __dmul_rn(r, cos(ang));
}
__device__ __forceinline__ double gauss_bm(uint64_t seed, uint64_t d) {
  return gauss_bm_u(uniform53(seed, d), uniform53(seed, d + 1));
}

// The same normal deviate from FP32 log/cos (for particles stored in FP32).
__device__ __forceinline__ float gauss_bm_f32_u(double v1, double v2) {
  const float u1 = (float)__dadd_rn(1.0, -v1);
  const float u2 = (float)v2;
  return sqrtf(-2.0f * logf(u1)) * cosf(6.28318530717958647692f * u2);
}

// Splits an absolute coordinate in cells into (cell, offset in [0,1)).
template <typename real>
__device__ __forceinline__ void split_coord(double xc, int& i, real& f) {
  double fi = floor(xc);
  i = (int)fi;
  f = (real)(xc - fi);
  if (f >= (real)1) {
    f = (real)0;
    i += 1;
  }
}

// Whether t lies outside [0, 1) as one unsigned compare of its bits: every
// value of [+0, 1) has a pattern below that of 1, every negative one a pattern
// above, and so do -0 (which the slow path below turns into +0) and NaN
// (which it leaves NaN).
__device__ __forceinline__ bool off_unit(float t) { return __float_as_uint(t) >= 0x3f800000u; }
__device__ __forceinline__ bool off_unit(double t) {
  return (unsigned long long)__double_as_longlong(t) >= 0x3ff0000000000000ull;
}

// Adds a displacement d (in cells) to (i, f) keeping f in [0, 1).
template <typename real>
__device__ __forceinline__ void advance(int& i, real& f, real d) {
  real t = f + d;
  if (off_unit(t)) {
    const real fl = floor(t);
    i += (int)fl;
    t -= fl;
    if (t >= (real)1) {  // t - floor(t) rounded up to 1 for a tiny negative t
      t = (real)0;
      i += 1;
    }
  }
  f = t;
}
#endif

}  // namespace pb
