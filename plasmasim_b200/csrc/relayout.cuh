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

// Each appended particle takes the next hole of its cell's column; the rest
// go, compacted, to the spare buffer Q. A warp takes U rows of 32 appended
// slots at a time and issues their loads, cursor atomics and hole lookups
// together, so that the chain of dependent memory accesses of one particle
// overlaps those of the others.
template <typename real>
__global__ void place_kernel(Parts<real> P, int first, const int* __restrict__ count, Geom g, TileGeom t,
                             const int* __restrict__ goff, const int* __restrict__ holes,
                             const int* __restrict__ nholes, int* cursor, Parts<real> Q, int* nspill) {
  constexpr int U = 4;
  const int n = *count;
  const int span = n - first;
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int w0 = warp * (U * kLanes); w0 < span; w0 += nwarps * (U * kLanes)) {  // warp-uniform
    int s[U], c[U], key[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int q = w0 + u * kLanes + lane;
      s[u] = first + q;
      c[u] = q < span ? P.cell[s[u]] : -1;
    }
    real o[U][3], v[U][3];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      key[u] = interior_key(g, c[u]);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        o[u][a] = key[u] >= 0 ? P.o[a][s[u]] : (real)0;
        v[u][a] = key[u] >= 0 ? P.v[a][s[u]] : (real)0;
      }
    }
    // per slot: holes of the destination cell and its column's first slot
    int nh[U], gb[U], l2[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      nh[u] = 0;
      gb[u] = 0;
      l2[u] = 0;
      if (key[u] >= 0) {
        nh[u] = nholes[key[u]];
        gb[u] = goff[group_of_key(g, t, key[u], l2[u])];
      }
    }
    // warp-aggregated cursor increments: one atomic per distinct key and row
    unsigned peers[U];
    int old[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      peers[u] = __match_any_sync(0xffffffffu, key[u] >= 0 ? key[u] : -1 - lane);
      old[u] = 0;
      if (key[u] >= 0 && lane == __ffs(peers[u]) - 1) old[u] = atomicAdd(cursor + key[u], __popc(peers[u]));
    }
    int rank[U], sb[U];
    unsigned ms[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      rank[u] = __shfl_sync(0xffffffffu, old[u], __ffs(peers[u]) - 1) + __popc(peers[u] & below);
      const bool spill = key[u] >= 0 && rank[u] >= nh[u];
      ms[u] = __ballot_sync(0xffffffffu, spill);
      sb[u] = 0;
      if (lane == 0 && ms[u]) sb[u] = atomicAdd(nspill, __popc(ms[u]));
    }
    int hrow[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      sb[u] = __shfl_sync(0xffffffffu, sb[u], 0);
      const bool spill = (ms[u] >> lane) & 1u;
      hrow[u] = (key[u] >= 0 && !spill) ? holes[gb[u] + rank[u] * kLanes + l2[u]] : 0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (w0 + u * kLanes + lane >= span) continue;
      if (key[u] >= 0) {
        const bool spill = (ms[u] >> lane) & 1u;
        const Parts<real>& D = spill ? Q : P;
        const int d = spill ? sb[u] + __popc(ms[u] & below) : gb[u] + hrow[u] * kLanes + l2[u];
        D.cell[d] = c[u];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          D.o[a][d] = o[u][a];
          D.v[a][d] = v[u][a];
        }
      }
      P.cell[s[u]] = -1;  // empty slot, outside the interior (dropped), or moved
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
