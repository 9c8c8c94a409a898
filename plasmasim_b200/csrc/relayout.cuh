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
//  2. place (one thread per appended slot: movers and refilled particles):
//     the particle takes the next hole of its new cell's column; a particle
//     that finds no hole is copied, compacted, into the spare buffer;
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

template <typename real>
__global__ void classify_kernel(Parts<real> P, Geom g, TileGeom t, const int* __restrict__ goff,
                                const int* __restrict__ gmax, int cap, int* holes, int* nholes,
                                int* append_at) {
  constexpr int U = 4;  // rows whose loads are in flight together
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
      const bool hole = c[u] < 0 || (leaves && (moved[u] || !mover));
      if (hole && c[u] >= 0 && !moved[u]) P.cell[base + r * kLanes + lane] = -1;
      if (hole && r < m) {
        holes[base + nh * kLanes + lane] = r;
        ++nh;
      }
    }
    // the movers of the U rows: their loads issued together, then the copies
    real o[U][3], v[U][3];
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (moved[u]) {
        const int s = base + (r0 + u) * kLanes + lane;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          o[u][a] = P.o[a][s];
          v[u][a] = P.v[a][s];
        }
      }
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (moved[u]) {
        P.cell[d[u]] = c[u];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          P.o[a][d[u]] = o[u][a];
          P.v[a][d[u]] = v[u][a];
        }
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

// Placement: each appended particle takes the next hole of its cell's column;
// the rest go, compacted, to the spare buffer Q. Two streaming passes, each
// with one kind of scattered access, so that many of them are in flight at
// once (one kernel doing the whole chain -- cell, cursor atomic, hole lookup,
// record copy -- per particle ran at 8 % issue).
// Pass 1: the particle's rank among the appended particles of its new cell,
// or, when its column has no hole left, -2 - (its index in the spare buffer
// Q); -1 for an empty slot or a particle outside the interior (dropped).
template <typename real>
__global__ void __launch_bounds__(256) place_rank_kernel(Parts<real> P, int first, const int* __restrict__ count,
                                                         Geom g, const int* __restrict__ nholes, int* cursor,
                                                         int* nspill, int* rank) {
  const int span = *count - first;
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  const int stride = gridDim.x * blockDim.x;
  for (int w0 = (blockIdx.x * blockDim.x + threadIdx.x) & ~31; w0 < span; w0 += stride) {  // warp-uniform
    const int q = w0 + lane;
    const int key = q < span ? interior_key(g, P.cell[first + q]) : -1;
    const int r = warp_aggregated_inc(cursor, key < 0 ? 0 : key, key >= 0);
    const bool spill = key >= 0 && r >= nholes[key];
    const unsigned ms = __ballot_sync(0xffffffffu, spill);
    int sb = 0;
    if (lane == 0 && ms) sb = atomicAdd(nspill, __popc(ms));
    sb = __shfl_sync(0xffffffffu, sb, 0);
    if (q < span) rank[q] = key < 0 ? -1 : (spill ? -2 - (sb + __popc(ms & below)) : r);
  }
}

// Pass 2: each appended particle to its hole (or to Q). Its old slot is left
// as it is: the count after the re-layout ends at first + (spilled
// particles), and unspill_kernel rewrites exactly those slots, so no later
// pass reads the others before a refill or the next re-layout writes them.
template <typename real>
__global__ void __launch_bounds__(256) place_move_kernel(Parts<real> P, int first, const int* __restrict__ count,
                                                         Geom g, TileGeom t, const int* __restrict__ goff,
                                                         const int* __restrict__ holes, const int* __restrict__ rank,
                                                         Parts<real> Q) {
  const int span = *count - first;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < span; q += gridDim.x * blockDim.x) {
    const int s = first + q;
    const int r = rank[q];
    if (r != -1) {
      const int c = P.cell[s];
      if (r >= 0) {
        int l2;
        const int G = group_of_key(g, t, interior_key(g, c), l2);
        const int gb = goff[G];
        copy_record(P, s, P, gb + holes[gb + r * kLanes + l2] * kLanes + l2, c);
      } else {
        copy_record(P, s, Q, -2 - r, c);
      }
    }
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
