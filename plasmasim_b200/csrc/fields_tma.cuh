// renew_b4_2 / renew_e4_2 (PIC/3d_pic458_domain.c:2580-2652) with the curl's
// operands staged in shared memory by the Tensor Memory Accelerator.
//
// A CTA updates a tile of TX x TY x 32 interior nodes (x, y, z). One thread
// issues three 3D tensor loads, one per operand plane of the curl (E for the
// B half-step, DB for the E step), that complete on one mbarrier. Plane q
// (0: x, 1: y, 2: z) enters the curl only through differences along the two
// other axes, so its box carries three halo nodes on those axes and none on
// axis q. Every thread then takes two z-adjacent nodes per item and reads the
// 4th-order stencil from shared memory with two-wide loads; the pointwise
// terms (DB, B0 and B, or E and J) move between HBM and registers with
// two-wide loads and stores, coalesced along z. The arithmetic of every node
// is that of renew_b_kernel / renew_e_kernel, term for term.
//
// TMA rules kept here: every box starts in z at the tile's first interior
// node minus two, 2 + 32 j - 2 = 32 j elements, a multiple of 16 bytes, and
// spans 36 elements, a multiple of 16 bytes; the plane's row pitch (gz
// elements) must be a multiple of 16 bytes, which the host checks before it
// chooses these kernels. Boxes that reach past the array read zeros, which
// only nodes outside the interior would use.
//
// The pointwise loads of a thread's first item are issued before it waits on
// the mbarrier, so that they overlap the tensor loads. The wait is bounded: a
// thread whose planes do not arrive within the limit counts ERR_FIELD_WAIT,
// waits once more (bounded) for the copies in flight and leaves its nodes
// unchanged.
#pragma once

#include <cuda.h>

#include "common.cuh"
#include "fields.cuh"

namespace pb {

constexpr int kStZ = 32;     // interior z nodes per tile
constexpr int kStBoxZ = 36;  // staged z extent, from two nodes below the tile
constexpr int kStThreads = 256;

__host__ __device__ constexpr size_t align128(size_t b) { return (b + 127) & ~(size_t)127; }

// Box extents of the three staged planes and the tile's shared-memory layout:
// plane 0, plane 1, plane 2 (each from a 128-byte boundary), the mbarrier.
template <typename real, int TX, int TY>
struct StencilTile {
  static constexpr int EX0 = TX, EY0 = TY + 3;      // x operand: halo in y (and z)
  static constexpr int EX1 = TX + 3, EY1 = TY;      // y operand: halo in x (and z)
  static constexpr int EX2 = TX + 3, EY2 = TY + 3;  // z operand: halo in x and y
  static constexpr size_t P0 = (size_t)EX0 * EY0 * kStBoxZ * sizeof(real);
  static constexpr size_t P1 = (size_t)EX1 * EY1 * kStBoxZ * sizeof(real);
  static constexpr size_t P2 = (size_t)EX2 * EY2 * kStBoxZ * sizeof(real);
  static constexpr size_t OFF1 = align128(P0), OFF2 = OFF1 + align128(P1), BAR = OFF2 + align128(P2);
  static constexpr size_t bytes = BAR + 16;
  static constexpr unsigned tx_bytes = (unsigned)(P0 + P1 + P2);
  static constexpr int items = TX * TY * (kStZ / 2);  // node pairs per tile
};

template <typename real> struct Two;
template <> struct Two<float> { using T = float2; };
template <> struct Two<double> { using T = double2; };

template <typename real>
__device__ __forceinline__ typename Two<real>::T ld2(const real* p, long long i) {
  return *reinterpret_cast<const typename Two<real>::T*>(p + i);
}
template <typename real>
__device__ __forceinline__ void st2(real* p, long long i, real a, real b) {
  typename Two<real>::T v;
  v.x = a;
  v.y = b;
  *reinterpret_cast<typename Two<real>::T*>(p + i) = v;
}

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// A 3D tile load into this CTA's own shared memory (no multicast).
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int z, int y, int x,
                                            unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      :: "r"(smem_addr(dst)), "l"(reinterpret_cast<unsigned long long>(map)), "r"(z), "r"(y), "r"(x),
         "r"(smem_addr(bar))
      : "memory");
}

// Waits for phase `parity` of the mbarrier; false after the iteration limit.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
  const unsigned a = smem_addr(bar);
  for (int it = 0; it < (1 << 20); ++it) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done) : "r"(a), "r"(parity) : "memory");
    if (done) return true;
  }
  return false;
}

// Issues the loads of the three planes of the tile at (k0, l0, m0); each box
// starts `lo` nodes below the tile on its halo axes and two below it in z.
template <typename real, int TX, int TY>
__device__ __forceinline__ void stage_issue(unsigned char* sm, const CUtensorMap* m0p, const CUtensorMap* m1p,
                                            const CUtensorMap* m2p, int k0, int l0, int m0, int lo) {
  using T = StencilTile<real, TX, TY>;
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(sm + T::BAR);
  if (threadIdx.x == 0) mbar_init(bar, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_expect_tx(bar, T::tx_bytes);
    tma_load_3d(sm, m0p, m0 - 2, l0 - lo, k0, bar);
    tma_load_3d(sm + T::OFF1, m1p, m0 - 2, l0, k0 - lo, bar);
    tma_load_3d(sm + T::OFF2, m2p, m0 - 2, l0 - lo, k0 - lo, bar);
  }
}

// Waits for the staged planes; false (after counting ERR_FIELD_WAIT and a
// second bounded wait for the copies in flight, before the CTA's shared
// memory is released) if they did not arrive. Every thread of the CTA calls it.
template <typename real, int TX, int TY>
__device__ __forceinline__ bool stage_wait(unsigned char* sm, unsigned long long* err) {
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(sm + StencilTile<real, TX, TY>::BAR);
  if (mbar_wait(bar, 0)) return true;
  count_err(err, ERR_FIELD_WAIT);
  mbar_wait(bar, 0);
  return false;
}

template <int TX, int TY>
__device__ __forceinline__ void tile_origin(int tiles_y, int tiles_z, int& k0, int& l0, int& m0) {
  const int tile = blockIdx.x;
  const int tz = tile % tiles_z, ty = (tile / tiles_z) % tiles_y, tx = tile / (tiles_z * tiles_y);
  k0 = 2 + tx * TX;
  l0 = 2 + ty * TY;
  m0 = 2 + tz * kStZ;
}

template <typename real, int TX, int TY>
__global__ void __launch_bounds__(kStThreads, sizeof(real) == 4 ? 3 : 2)
    renew_b_tma_kernel(const __grid_constant__ CUtensorMap tex, const __grid_constant__ CUtensorMap tey,
                       const __grid_constant__ CUtensorMap tez, Fields<real> F, Geom g, Ramps rp, BParams p,
                       int tiles_y, int tiles_z, unsigned long long* err) {
  using T = StencilTile<real, TX, TY>;
  extern __shared__ __align__(128) unsigned char fsm[];
  int k0, l0, m0;
  tile_origin<TX, TY>(tiles_y, tiles_z, k0, l0, m0);
  stage_issue<real, TX, TY>(fsm, &tex, &tey, &tez, k0, l0, m0, 2);
  static_assert(T::items >= kStThreads, "every thread must take an item, and so wait for the staged planes");
  bool waited = false;
  const real* ex = reinterpret_cast<const real*>(fsm);
  const real* ey = reinterpret_cast<const real*>(fsm + T::OFF1);
  const real* ez = reinterpret_cast<const real*>(fsm + T::OFF2);
  constexpr int SY = kStBoxZ, SX1 = T::EY1 * kStBoxZ, SX2 = T::EY2 * kStBoxZ;
  const real c24 = (real)p.inv24dx;
#pragma unroll 1
  for (int i = threadIdx.x; i < T::items; i += kStThreads) {
    const int z = 2 * (i % (kStZ / 2)), b = (i / (kStZ / 2)) % TY, a = i / (kStZ / 2 * TY);
    const int k = k0 + a, l = l0 + b, m = m0 + z;
    const bool in = k < g.nx + 2 && l < g.ny + 2 && m < g.nz + 2;
    const long long n = in ? (long long)k * g.sx + (long long)l * g.gz + m : 0;
    // the pointwise operands first: their loads overlap the tensor loads
    typename Two<real>::T dbv[3], b0v[3];
    if (in) {
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        dbv[q] = ld2(F.f[F_DBX + q], n);
        b0v[q] = ld2(F.f[F_B0X + q], n);
      }
    }
    if (!waited) {
      if (!stage_wait<real, TX, TY>(fsm, err)) return;
      waited = true;
    }
    if (!in) continue;
    const int s0 = (a * T::EY0 + b + 2) * kStBoxZ + z + 2;        // ex
    const int s1 = ((a + 2) * T::EY1 + b) * kStBoxZ + z + 2;      // ey
    const int s2 = ((a + 2) * T::EY2 + b + 2) * kStBoxZ + z + 2;  // ez
    // z runs of ex and ey: entry 2 + d holds offset d (-2..3) from node m
    real xz[6], yz[6];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const auto u = ld2(ex, s0 - 2 + 2 * d);
      const auto v = ld2(ey, s1 - 2 + 2 * d);
      xz[2 * d] = u.x; xz[2 * d + 1] = u.y;
      yz[2 * d] = v.x; yz[2 * d + 1] = v.y;
    }
    const double2 rzl = *reinterpret_cast<const double2*>(rp.rz + 2 * m);      // rz[2m], rz[2m+1]
    const double2 rzh = *reinterpret_cast<const double2*>(rp.rz + 2 * m + 2);  // rz[2m+2], rz[2m+3]
    const double rz0[2] = {rzl.x, rzh.x}, rz1[2] = {rzl.y, rzh.y};
    // x component at (k+1/2, l, m): ez along y, ey along z
    {
      const auto q0 = ld2(ez, s2 - 2 * SY), q1 = ld2(ez, s2 - SY), q2 = ld2(ez, s2), q3 = ld2(ez, s2 + SY);
      const real m2[2] = {q0.x, q0.y}, m1[2] = {q1.x, q1.y}, c0[2] = {q2.x, q2.y}, p1[2] = {q3.x, q3.y};
      const real dbo[2] = {dbv[0].x, dbv[0].y}, b0[2] = {b0v[0].x, b0v[0].y};
      real db[2];
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        double ca, cb;
        b_coeffs(sigma_of(rp.a, rp.rx[2 * k + 1], rp.ry[2 * l], rz0[j]), p, ca, cb);
        const real curl = ((real)27 * (c0[j] - m1[j] - yz[2 + j] + yz[1 + j]) -
                           (p1[j] - m2[j] - yz[3 + j] + yz[j])) * c24;
        db[j] = (real)ca * dbo[j] - (real)cb * curl;
      }
      st2(F.f[F_DBX], n, db[0], db[1]);
      st2(F.f[F_BX], n, b0[0] + db[0], b0[1] + db[1]);
    }
    // y component at (k, l+1/2, m): ex along z, ez along x
    {
      const auto q0 = ld2(ez, s2 - 2 * SX2), q1 = ld2(ez, s2 - SX2), q2 = ld2(ez, s2), q3 = ld2(ez, s2 + SX2);
      const real m2[2] = {q0.x, q0.y}, m1[2] = {q1.x, q1.y}, c0[2] = {q2.x, q2.y}, p1[2] = {q3.x, q3.y};
      const real dbo[2] = {dbv[1].x, dbv[1].y}, b0[2] = {b0v[1].x, b0v[1].y};
      real db[2];
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        double ca, cb;
        b_coeffs(sigma_of(rp.a, rp.rx[2 * k], rp.ry[2 * l + 1], rz0[j]), p, ca, cb);
        const real curl = ((real)27 * (xz[2 + j] - xz[1 + j] - c0[j] + m1[j]) -
                           (xz[3 + j] - xz[j] - p1[j] + m2[j])) * c24;
        db[j] = (real)ca * dbo[j] - (real)cb * curl;
      }
      st2(F.f[F_DBY], n, db[0], db[1]);
      st2(F.f[F_BY], n, b0[0] + db[0], b0[1] + db[1]);
    }
    // z component at (k, l, m+1/2): ey along x, ex along y
    {
      const auto q0 = ld2(ey, s1 - 2 * SX1), q1 = ld2(ey, s1 - SX1), q2 = ld2(ey, s1), q3 = ld2(ey, s1 + SX1);
      const auto r0 = ld2(ex, s0 - 2 * SY), r1 = ld2(ex, s0 - SY), r2 = ld2(ex, s0), r3 = ld2(ex, s0 + SY);
      const real ym2[2] = {q0.x, q0.y}, ym1[2] = {q1.x, q1.y}, y0[2] = {q2.x, q2.y}, yp1[2] = {q3.x, q3.y};
      const real xm2[2] = {r0.x, r0.y}, xm1[2] = {r1.x, r1.y}, x0[2] = {r2.x, r2.y}, xp1[2] = {r3.x, r3.y};
      const real dbo[2] = {dbv[2].x, dbv[2].y}, b0[2] = {b0v[2].x, b0v[2].y};
      real db[2];
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        double ca, cb;
        b_coeffs(sigma_of(rp.a, rp.rx[2 * k], rp.ry[2 * l], rz1[j]), p, ca, cb);
        const real curl = ((real)27 * (y0[j] - ym1[j] - x0[j] + xm1[j]) -
                           (yp1[j] - ym2[j] - xp1[j] + xm2[j])) * c24;
        db[j] = (real)ca * dbo[j] - (real)cb * curl;
      }
      st2(F.f[F_DBZ], n, db[0], db[1]);
      st2(F.f[F_BZ], n, b0[0] + db[0], b0[1] + db[1]);
    }
  }
}

template <typename real, int TX, int TY>
__global__ void __launch_bounds__(kStThreads, sizeof(real) == 4 ? 3 : 2)
    renew_e_tma_kernel(const __grid_constant__ CUtensorMap tbx, const __grid_constant__ CUtensorMap tby,
                       const __grid_constant__ CUtensorMap tbz, Fields<real> F, Geom g, Ramps rp, EParams p,
                       int tiles_y, int tiles_z, unsigned long long* err) {
  using T = StencilTile<real, TX, TY>;
  extern __shared__ __align__(128) unsigned char fsm[];
  int k0, l0, m0;
  tile_origin<TX, TY>(tiles_y, tiles_z, k0, l0, m0);
  stage_issue<real, TX, TY>(fsm, &tbx, &tby, &tbz, k0, l0, m0, 1);
  static_assert(T::items >= kStThreads, "every thread must take an item, and so wait for the staged planes");
  bool waited = false;
  const real* bx = reinterpret_cast<const real*>(fsm);
  const real* by = reinterpret_cast<const real*>(fsm + T::OFF1);
  const real* bz = reinterpret_cast<const real*>(fsm + T::OFF2);
  constexpr int SY = kStBoxZ, SX1 = T::EY1 * kStBoxZ, SX2 = T::EY2 * kStBoxZ;
  const real c24 = (real)p.inv24dx;
  const real mu0 = (real)p.mu0;
#pragma unroll 1
  for (int i = threadIdx.x; i < T::items; i += kStThreads) {
    const int z = 2 * (i % (kStZ / 2)), b = (i / (kStZ / 2)) % TY, a = i / (kStZ / 2 * TY);
    const int k = k0 + a, l = l0 + b, m = m0 + z;
    const bool in = k < g.nx + 2 && l < g.ny + 2 && m < g.nz + 2;
    const long long n = in ? (long long)k * g.sx + (long long)l * g.gz + m : 0;
    // the pointwise operands first: their loads overlap the tensor loads
    typename Two<real>::T ev[3], jiv[3], jev[3];
    if (in) {
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        ev[q] = ld2(F.f[F_EX + q], n);
        jiv[q] = ld2(F.f[F_JIX + q], n);
        jev[q] = ld2(F.f[F_JEX + q], n);
      }
    }
    if (!waited) {
      if (!stage_wait<real, TX, TY>(fsm, err)) return;
      waited = true;
    }
    if (!in) continue;
    const int s0 = (a * T::EY0 + b + 1) * kStBoxZ + z + 2;        // bx
    const int s1 = ((a + 1) * T::EY1 + b) * kStBoxZ + z + 2;      // by
    const int s2 = ((a + 1) * T::EY2 + b + 1) * kStBoxZ + z + 2;  // bz
    // z runs of bx and by: entry 2 + d holds offset d (-2..3) from node m
    real xz[6], yz[6];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const auto u = ld2(bx, s0 - 2 + 2 * d);
      const auto v = ld2(by, s1 - 2 + 2 * d);
      xz[2 * d] = u.x; xz[2 * d + 1] = u.y;
      yz[2 * d] = v.x; yz[2 * d + 1] = v.y;
    }
    const double2 rzl = *reinterpret_cast<const double2*>(rp.rz + 2 * m);
    const double2 rzh = *reinterpret_cast<const double2*>(rp.rz + 2 * m + 2);
    const double rz0[2] = {rzl.x, rzh.x}, rz1[2] = {rzl.y, rzh.y};
    // x component at (k, l+1/2, m+1/2): bz along y, by along z
    {
      const auto q0 = ld2(bz, s2 - SY), q1 = ld2(bz, s2), q2 = ld2(bz, s2 + SY), q3 = ld2(bz, s2 + 2 * SY);
      const real m1[2] = {q0.x, q0.y}, c0[2] = {q1.x, q1.y}, p1[2] = {q2.x, q2.y}, p2[2] = {q3.x, q3.y};
      const real eo[2] = {ev[0].x, ev[0].y}, ji[2] = {jiv[0].x, jiv[0].y}, je[2] = {jev[0].x, jev[0].y};
      real en[2];
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        double ca, cb;
        e_coeffs(sigma_of(rp.a, rp.rx[2 * k], rp.ry[2 * l + 1], rz1[j]), p, ca, cb);
        const real curl = ((real)27 * ((p1[j] - c0[j]) - (yz[3 + j] - yz[2 + j])) -
                           ((p2[j] - m1[j]) - (yz[4 + j] - yz[1 + j]))) * c24;
        en[j] = (real)ca * eo[j] + (real)cb * (curl - mu0 * (ji[j] - je[j]));
      }
      st2(F.f[F_EX], n, en[0], en[1]);
    }
    // y component at (k+1/2, l, m+1/2): bx along z, bz along x
    {
      const auto q0 = ld2(bz, s2 - SX2), q1 = ld2(bz, s2), q2 = ld2(bz, s2 + SX2), q3 = ld2(bz, s2 + 2 * SX2);
      const real m1[2] = {q0.x, q0.y}, c0[2] = {q1.x, q1.y}, p1[2] = {q2.x, q2.y}, p2[2] = {q3.x, q3.y};
      const real eo[2] = {ev[1].x, ev[1].y}, ji[2] = {jiv[1].x, jiv[1].y}, je[2] = {jev[1].x, jev[1].y};
      real en[2];
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        double ca, cb;
        e_coeffs(sigma_of(rp.a, rp.rx[2 * k + 1], rp.ry[2 * l], rz1[j]), p, ca, cb);
        const real curl = ((real)27 * ((xz[3 + j] - xz[2 + j]) - (p1[j] - c0[j])) -
                           ((xz[4 + j] - xz[1 + j]) - (p2[j] - m1[j]))) * c24;
        en[j] = (real)ca * eo[j] + (real)cb * (curl - mu0 * (ji[j] - je[j]));
      }
      st2(F.f[F_EY], n, en[0], en[1]);
    }
    // z component at (k+1/2, l+1/2, m): by along x, bx along y
    {
      const auto q0 = ld2(by, s1 - SX1), q1 = ld2(by, s1), q2 = ld2(by, s1 + SX1), q3 = ld2(by, s1 + 2 * SX1);
      const auto r0 = ld2(bx, s0 - SY), r1 = ld2(bx, s0), r2 = ld2(bx, s0 + SY), r3 = ld2(bx, s0 + 2 * SY);
      const real ym1[2] = {q0.x, q0.y}, y0[2] = {q1.x, q1.y}, yp1[2] = {q2.x, q2.y}, yp2[2] = {q3.x, q3.y};
      const real xm1[2] = {r0.x, r0.y}, x0[2] = {r1.x, r1.y}, xp1[2] = {r2.x, r2.y}, xp2[2] = {r3.x, r3.y};
      const real eo[2] = {ev[2].x, ev[2].y}, ji[2] = {jiv[2].x, jiv[2].y}, je[2] = {jev[2].x, jev[2].y};
      real en[2];
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        double ca, cb;
        e_coeffs(sigma_of(rp.a, rp.rx[2 * k + 1], rp.ry[2 * l + 1], rz0[j]), p, ca, cb);
        const real curl = ((real)27 * ((yp1[j] - y0[j]) - (xp1[j] - x0[j])) -
                           ((yp2[j] - ym1[j]) - (xp2[j] - xm1[j]))) * c24;
        en[j] = (real)ca * eo[j] + (real)cb * (curl - mu0 * (ji[j] - je[j]));
      }
      st2(F.f[F_EZ], n, en[0], en[1]);
    }
  }
}

}  // namespace pb
