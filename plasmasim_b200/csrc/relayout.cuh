// In-place re-layout of the tiled particle layout (tiled.cuh).
//
// Between two sorts most particles stay in their home cell. A re-layout
// leaves those where they are and moves only the rest:
//  1. classify (one warp per group): a particle whose cell is no longer its
//     lane's home cell is copied to the append region after `count` and its
//     slot becomes a hole (cell = -1); each lane lists the rows of its holes,
//     in row order, in a scratch array laid out like the slots themselves.
//     A warp takes append slots 64 at a time from the shared counter and
//     marks the slots of its last block it does not use empty, so the counter
//     sees one atomic per 64 movers instead of one per row;
//  2. place (movers and refilled particles, all appended after `count`): the
//     particles are bucketed by their new cell -- a rank per particle from a
//     per-cell counter, an exclusive scan of the arrivals that find a hole,
//     the particle's index written to its bucket slot -- and then one warp
//     per group fills each lane's holes, in row order, from its cell's
//     bucket. A particle ranked past its cell's holes is copied, compacted,
//     into the spare buffer instead. Every pass streams its input, so its
//     scattered accesses are independent of one another;
//  3. the particles without a hole are copied back right after the layout,
//     where the slot-order push handles them until a later re-layout finds
//     them a hole (or a full sort, when they become too many).
// Particles outside the interior are dropped, as the reference's sort drops
// them.
#pragma once

#include "common.cuh"
#include "particles.cuh"
#include "tiled.cuh"

namespace pb {

constexpr int kAppendBlock = 64;

template <typename real>
__device__ __forceinline__ void copy_slot(const Parts<real>& S, int s, const Parts<real>& D, int d, int c) {
  copy_record(S, s, D, d, c);
}

// With `shell` set (the re-layout after a refill), a particle of the layout
// that lies in a refill shell is deleted here, as add_*_flat's removal
// (:6015-6031) would have: one pass over the layout for both.
template <typename real>
__global__ void classify_kernel(Parts<real> P, Geom g, TileGeom t, const int* __restrict__ goff,
                                const int* __restrict__ gmax, int cap, int* holes, int* nholes,
                                int* append_at, int* nonhome, int shell) {
  constexpr int U = 4;  // rows whose loads are in flight together (8 measured no faster)
  const int G = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (G >= t.ngroups) return;  // warp-uniform
  const unsigned below = (1u << lane) - 1u;
  const int home = home_key(g, t, G, lane);
  const int base = goff[G], m = gmax[G];
  int nh = 0;
  int blk = 0, used = kAppendBlock;  // current block of append slots (warp-uniform)
  for (int r0 = 0; r0 < m; r0 += U) {
    int c[U], d[U];
    bool moved[U];
#pragma unroll
    for (int u = 0; u < U; ++u) c[u] = r0 + u < m ? P.cell[base + (r0 + u) * kLanes + lane] : -1;
    if (shell) {
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const long long tu = base + (r0 + u) * kLanes + lane;
        if (c[u] >= 0 && in_refill_shell(P, g, c[u], tu)) {
          P.cell[tu] = -1;
          c[u] = -1;
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int r = r0 + u;
      const int key = interior_key(g, c[u]);
      const bool leaves = c[u] >= 0 && key != home;
      const bool mover = leaves && key >= 0;
      const unsigned mm = __ballot_sync(0xffffffffu, mover);
      const int nm = __popc(mm);
      if (nm > kAppendBlock - used) {  // close the block, take a new one
        for (int q = used + lane; q < kAppendBlock; q += kLanes)
          if (blk + q < cap) P.cell[blk + q] = -1;
        int nb = 0;
        if (lane == 0) nb = atomicAdd(append_at, kAppendBlock);
        blk = __shfl_sync(0xffffffffu, nb, 0);
        used = 0;
      }
      d[u] = blk + used + __popc(mm & below);
      used += nm;
      // a mover that finds the append region full stays where it is
      moved[u] = mover && d[u] < cap;
      if (mover && !moved[u]) *nonhome = 1;
      const bool hole = c[u] < 0 || (leaves && (moved[u] || !mover));
      if (hole && c[u] >= 0 && !moved[u]) P.cell[base + r * kLanes + lane] = -1;
      if (hole && r < m) {
        holes[base + nh * kLanes + lane] = r;
        ++nh;
      }
    }
    // the movers of the U rows: their record loads issued together, then the copies
    Rec<real> rec[U];
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (moved[u]) rec[u] = load_records(P, base + (r0 + u) * kLanes + lane);
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (moved[u]) {
        const Rec<real>& q = rec[u];
        store_records(P, d[u], c[u], q.o[0], q.o[1], q.o[2], q.v[0], q.v[1], q.v[2]);
        P.cell[base + (r0 + u) * kLanes + lane] = -1;
      }
  }
  for (int q = used + lane; q < kAppendBlock; q += kLanes)
    if (blk + q < cap && used < kAppendBlock) P.cell[blk + q] = -1;
  if (home >= 0) nholes[home] = nh;
}

__global__ void clamp_count_kernel(const int* append_at, int cap, int* count_dev) {
  *count_dev = min(*append_at, cap);
}

// Placement, pass 1: the particle's rank among the appended particles of its
// new cell (from the per-cell counter `cursor`); -1 for an empty slot or a
// particle outside the interior (dropped).
template <typename real>
__global__ void __launch_bounds__(256) place_count_kernel(Parts<real> P, int first, const int* __restrict__ count,
                                                          Geom g, int* cursor, int* rank) {
  const int span = *count - first;
  const int lane = threadIdx.x & 31;
  const int stride = gridDim.x * blockDim.x;
  for (int w0 = (blockIdx.x * blockDim.x + threadIdx.x) & ~31; w0 < span; w0 += stride) {  // warp-uniform
    const int q = w0 + lane;
    const int key = q < span ? interior_key(g, P.cell[first + q]) : -1;
    const int r = warp_aggregated_inc(cursor, key < 0 ? 0 : key, key >= 0);
    if (q < span) rank[q] = key < 0 ? -1 : r;
  }
}

// Pass 2, per interior cell: the arrivals that find a hole, min(arrivals, holes)
// (exclusive-scanned afterwards into each cell's bucket offset).
__global__ void place_fit_kernel(const int* __restrict__ arrivals, const int* __restrict__ nholes, int* fit,
                                 long long ncells) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncells;
       c += (long long)gridDim.x * blockDim.x)
    fit[c] = min(arrivals[c], nholes[c]);
}

// Pass 3: a particle ranked below its cell's holes writes its index to its
// bucket slot; the others are copied, compacted, into the spare buffer Q.
template <typename real>
__global__ void __launch_bounds__(256) place_bucket_kernel(Parts<real> P, int first, const int* __restrict__ count,
                                                           Geom g, const int* __restrict__ nholes,
                                                           const int* __restrict__ off, const int* __restrict__ rank,
                                                           int* bucket, int* nspill, Parts<real> Q) {
  const int span = *count - first;
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  const int stride = gridDim.x * blockDim.x;
  for (int w0 = (blockIdx.x * blockDim.x + threadIdx.x) & ~31; w0 < span; w0 += stride) {  // warp-uniform
    const int q = w0 + lane;
    const int c = q < span ? P.cell[first + q] : -1;
    const int key = interior_key(g, c);
    const int r = q < span ? rank[q] : -1;
    const bool fits = key >= 0 && r < nholes[key];
    const bool spill = key >= 0 && !fits;
    if (fits) bucket[off[key] + r] = q;
    const unsigned ms = __ballot_sync(0xffffffffu, spill);
    int sb = 0;
    if (lane == 0 && ms) sb = atomicAdd(nspill, __popc(ms));
    sb = __shfl_sync(0xffffffffu, sb, 0);
    if (spill) copy_record(P, first + q, Q, sb + __popc(ms & below), c);
  }
}

// Pass 4, one warp per group: lane l copies the k-th particle of its home
// cell's bucket into the slot of its k-th hole. U holes per lane are in
// flight at once; their slots lie in the lane's own column.
template <typename real>
__global__ void place_fill_kernel(Parts<real> P, int first, Geom g, TileGeom t, const int* __restrict__ goff,
                                  const int* __restrict__ holes, const int* __restrict__ arrivals,
                                  const int* __restrict__ nholes, const int* __restrict__ off,
                                  const int* __restrict__ bucket) {
  constexpr int U = 4;  // holes per lane in flight together
  const int G = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (G >= t.ngroups) return;  // warp-uniform
  const int home = home_key(g, t, G, lane);
  const int n = home >= 0 ? min(arrivals[home], nholes[home]) : 0;
  const int o = home >= 0 ? off[home] : 0;
  const int base = goff[G];
  int nmax = n;
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) nmax = max(nmax, __shfl_xor_sync(0xffffffffu, nmax, s));
  for (int k0 = 0; k0 < nmax; k0 += U) {
    int src[U], dst[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = k0 + u;
      src[u] = k < n ? first + bucket[o + k] : -1;
      dst[u] = k < n ? base + holes[base + k * kLanes + lane] * kLanes + lane : -1;
    }
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (src[u] >= 0) copy_record(P, src[u], P, dst[u], P.cell[src[u]]);
  }
}

// The particles without a hole back to slots [first, first + n).
template <typename real>
__global__ void unspill_kernel(Parts<real> Q, const int* __restrict__ nspill, Parts<real> P, int first) {
  const int n = *nspill;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
    copy_slot(Q, q, P, first + q, Q.cell[q]);
}

}  // namespace pb
