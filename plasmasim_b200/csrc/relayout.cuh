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
  D.cell[d] = c;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    D.o[a][d] = S.o[a][s];
    D.v[a][d] = S.v[a][s];
  }
}

template <typename real>
__global__ void classify_kernel(Parts<real> P, Geom g, TileGeom t, const int* __restrict__ goff,
                                const int* __restrict__ gmax, int cap, int* holes, int* nholes,
                                int* append_at) {
  const int G = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (G >= t.ngroups) return;  // warp-uniform
  const unsigned below = (1u << lane) - 1u;
  const int home = home_key(g, t, G, lane);
  const int base = goff[G], m = gmax[G];
  int nh = 0;
  int blk = 0, used = kAppendBlock;  // current block of append slots (warp-uniform)
  for (int r = 0; r < m; ++r) {
    const int s = base + r * kLanes + lane;
    const int c = P.cell[s];
    const int key = interior_key(g, c);
    const bool leaves = c >= 0 && key != home;
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
    const int d = blk + used + __popc(mm & below);
    used += nm;
    // a mover that finds the append region full stays where it is
    const bool moved = mover && d < cap;
    if (moved) copy_slot(P, s, P, d, c);
    const bool hole = c < 0 || (leaves && (moved || !mover));
    if (hole && c >= 0) P.cell[s] = -1;
    if (hole) {
      holes[base + nh * kLanes + lane] = r;
      ++nh;
    }
  }
  for (int q = used + lane; q < kAppendBlock; q += kLanes)
    if (blk + q < cap && used < kAppendBlock) P.cell[blk + q] = -1;
  if (home >= 0) nholes[home] = nh;
}

__global__ void clamp_count_kernel(const int* append_at, int cap, int* count_dev) {
  *count_dev = min(*append_at, cap);
}

// Each appended particle takes the next hole of its cell's column; the rest
// go, compacted, to the spare buffer Q.
template <typename real>
__global__ void place_kernel(Parts<real> P, int first, const int* __restrict__ count, Geom g, TileGeom t,
                             const int* __restrict__ goff, const int* __restrict__ holes,
                             const int* __restrict__ nholes, int* cursor, Parts<real> Q, int* nspill) {
  const int n = *count;
  const int stride = gridDim.x * blockDim.x;
  const int span = n - first;
  const int span_round = (span + 31) & ~31;
  const int lane = threadIdx.x & 31;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < span_round; q += stride) {
    const int s = first + q;
    int c = -1, key = -1;
    if (q < span) {
      c = P.cell[s];
      key = interior_key(g, c);
    }
    const int rank = warp_aggregated_inc(cursor, key < 0 ? 0 : key, key >= 0);
    const bool spill = key >= 0 && rank >= nholes[key];
    const unsigned ms = __ballot_sync(0xffffffffu, spill);
    int sb = 0;
    if (lane == 0 && ms) sb = atomicAdd(nspill, __popc(ms));
    sb = __shfl_sync(0xffffffffu, sb, 0);
    if (q >= span) continue;
    if (key < 0) {
      P.cell[s] = -1;  // empty slot, or outside the interior: dropped
    } else if (spill) {
      copy_slot(P, s, Q, sb + __popc(ms & ((1u << lane) - 1u)), c);
      P.cell[s] = -1;
    } else {
      int l2;
      const int G = group_of_key(g, t, key, l2);
      const int d = goff[G] + holes[goff[G] + rank * kLanes + l2] * kLanes + l2;
      copy_slot(P, s, P, d, c);
      P.cell[s] = -1;
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
