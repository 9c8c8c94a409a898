// Exchanges between the ranks of a decomposed run: the ghost planes of
// sr_b / sr_e / sr_current2 (PIC/3d_pic458_domain.c:1001-2039) and the
// particle packets of sr_particle (:2041-2555). The host side (api.cu)
// sequences them through the context's transport; these kernels pack the
// planes and packets into contiguous buffers and unpack what arrives.
#pragma once

#include "common.cuh"
#include "fields.cuh"
#include "particles.cuh"

namespace pb {

// Node of layer `layer` (a plane of constant k for axis 0, a row of constant l
// over every k for axis 1) and in-layer index e.
__device__ __forceinline__ long long halo_node(const Geom& g, int axis, int layer, int e) {
  if (axis == 0) return (long long)layer * g.sx + e;
  const int k = e / g.gz, m = e % g.gz;
  return (long long)k * g.sx + (long long)layer * g.gz + m;
}

__host__ __device__ __forceinline__ int halo_layer_nodes(const Geom& g, int axis) {
  return axis == 0 ? g.gy * g.gz : g.gx * g.gz;
}

// Layers l0, l0 + 1 of every plane of s into buf, plane-major.
template <typename real>
__global__ void halo_pack_kernel(PlaneSet<real> s, Geom g, int axis, int l0, real* __restrict__ buf) {
  const int per = halo_layer_nodes(g, axis);
  const long long total = (long long)s.count * 2 * per;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(t / (2LL * per));
    const int r = (int)((t / per) % 2);
    const int e = (int)(t % per);
    buf[t] = s.p[q][halo_node(g, axis, l0 + r, e)];
  }
}

enum HaloMode {
  HALO_COPY = 0,    // ghost = received (sr_e, sr_phi)
  HALO_ADD = 1,     // interior += received (sr_current2)
  HALO_BTOTAL = 2,  // B = received total field, DB = B - own B0 (sr_b's total-field exchange)
};

// buf into layers l0, l0 + 1. For HALO_BTOTAL, s = {BX, BY, BZ} and aux =
// {DBX, DBY, DBZ, B0X, B0Y, B0Z}.
template <typename real>
__global__ void halo_unpack_kernel(PlaneSet<real> s, PlaneSet<real> aux, Geom g, int axis, int l0,
                                   const real* __restrict__ buf, int mode) {
  const int per = halo_layer_nodes(g, axis);
  const long long total = (long long)s.count * 2 * per;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(t / (2LL * per));
    const int r = (int)((t / per) % 2);
    const int e = (int)(t % per);
    const long long n = halo_node(g, axis, l0 + r, e);
    const real v = buf[t];
    if (mode == HALO_ADD) {
      s.p[q][n] += v;
    } else {
      s.p[q][n] = v;
      if (mode == HALO_BTOTAL) aux.p[q][n] = v - aux.p[3 + q][n];
    }
  }
}

// ------------------------------------------------------------ particles
// Splits list `in` (n = *in_count) along axis a (0: x, 1: y) into forward
// packets (index >= N + 2), backward packets (index < 2) and the rest, which
// is appended to `stay`. A packet the rank drops (sr_particle zeroes the
// backward counts on rank 0 and the forward ones on the last rank, :2137-2146)
// is not copied anywhere.
template <typename real>
__global__ void mig_split_kernel(const MigRec<real>* __restrict__ in, const int* __restrict__ in_count, Geom g,
                                 int axis, int drop_bak, int drop_fwd, MigRec<real>* fwd, int* fwd_count,
                                 MigRec<real>* bak, int* bak_count, MigRec<real>* stay, int* stay_count, int cap,
                                 unsigned long long* err) {
  const int n = *in_count;
  const int N = axis == 0 ? g.nx : g.ny;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const MigRec<real> r = in[t];
    int i, j, k;
    unpack_cell(r.cell, i, j, k);
    const int x = axis == 0 ? i : j;
    MigRec<real>* dst;
    int* cnt;
    if (x >= N + 2) {
      if (drop_fwd) continue;
      dst = fwd;
      cnt = fwd_count;
    } else if (x < 2) {
      if (drop_bak) continue;
      dst = bak;
      cnt = bak_count;
    } else {
      dst = stay;
      cnt = stay_count;
    }
    const int q = atomicAdd(cnt, 1);
    if (q < cap) dst[q] = r;
    else count_err(err, ERR_MIGRATION);
  }
}

// Received packets: shift the cell index along `axis` by `shift` cells and
// append to `out`.
template <typename real>
__global__ void mig_receive_kernel(const MigRec<real>* __restrict__ in, int n, int axis, int shift,
                                   MigRec<real>* out, int* out_count, int cap, unsigned long long* err) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    MigRec<real> r = in[t];
    int i, j, k;
    unpack_cell(r.cell, i, j, k);
    if (axis == 0) i += shift;
    else j += shift;
    r.cell = repack(i, j, k, err);
    if (r.cell < 0) continue;
    const int q = atomicAdd(out_count, 1);
    if (q < cap) out[q] = r;
    else count_err(err, ERR_MIGRATION);
  }
}

// The settled packets into slots [first, first + n) of the particle store.
template <typename real>
__global__ void mig_append_kernel(const MigRec<real>* __restrict__ in, int n, Parts<real> P, int first) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const MigRec<real> r = in[t];
    const int d = first + t;
    P.cell[d] = r.cell;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      P.o[a][d] = r.o[a];
      P.v[a][d] = r.v[a];
    }
  }
}

}  // namespace pb
