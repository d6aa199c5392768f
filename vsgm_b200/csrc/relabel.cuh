// Degree-ordered relabelling of a resident graph on the device (sm_100a).
//
// New id = rank of (degree, old id), ascending - the permutation the host
// relabelling (graph.cpp: degree_relabel) computes.  Two stable LSD radix sorts of
// (key, value) pairs do all the work:
//   1. (degree, id) pairs by degree: the ids in new order;
//   2. the edges, emitted row by row in new-source order as (new destination, new
//      source), by destination: every destination's sources come out in the order
//      they were emitted, ascending - which, the graph being undirected, are the
//      sorted rows of the relabelled graph.
// The radix sort is one histogram pass and one stable scatter pass per 8-bit digit
// over tiles of 4096 pairs; within a tile, ranks among equal digits come from
// warp match masks and per-warp digit counters in shared memory, so equal keys
// keep their input order.
#pragma once

#include <cstdint>

#include "kernels.cuh"

namespace vsgm {
namespace dev {

constexpr int kRadixThreads = 256;
constexpr int kRadixItems = 16;
constexpr int kRadixTile = kRadixThreads * kRadixItems;
constexpr int kRadixWarps = kRadixThreads / 32;

// hist[digit * n_tiles + tile] = pairs of the tile whose digit is `digit`
__global__ void __launch_bounds__(kRadixThreads) k_radix_hist(const uint32_t* __restrict__ keys, uint64_t n, int shift, uint32_t* __restrict__ hist,
                                                              uint64_t n_tiles) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const uint64_t base = (uint64_t)blockIdx.x * kRadixTile;
#pragma unroll 4
  for (int k = 0; k < kRadixItems; k++) {
    const uint64_t i = base + (uint64_t)k * kRadixThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[(__ldg(keys + i) >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[(uint64_t)threadIdx.x * n_tiles + blockIdx.x] = h[threadIdx.x];
}

// stable scatter of one tile: off[digit * n_tiles + tile] is where the tile's first
// pair with that digit goes (exclusive scan of hist)
__global__ void __launch_bounds__(kRadixThreads) k_radix_scatter(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals, uint64_t n, int shift,
                                                                 const uint64_t* __restrict__ off, uint64_t n_tiles, uint32_t* __restrict__ keys_out,
                                                                 uint32_t* __restrict__ vals_out) {
  __shared__ uint64_t at[256];                // next position of each digit
  __shared__ uint32_t wcnt[kRadixWarps][256];  // per warp: count, then exclusive prefix, of each digit
  __shared__ uint32_t round_total[256];
  const unsigned t = threadIdx.x, lane = lane_id(), wid = t / 32;
  at[t] = off[(uint64_t)t * n_tiles + blockIdx.x];
#pragma unroll
  for (int w = 0; w < kRadixWarps; w++) wcnt[w][t] = 0;
  __syncthreads();
  const uint64_t base = (uint64_t)blockIdx.x * kRadixTile;
  const unsigned below = (1u << lane) - 1;
  for (int k = 0; k < kRadixItems; k++) {
    const uint64_t i = base + (uint64_t)k * kRadixThreads + t;
    const bool valid = i < n;
    uint32_t key = 0, val = 0, dg = 256u;  // 256: no digit (past the end)
    if (valid) {
      key = __ldg(keys + i);
      val = __ldg(vals + i);
      dg = (key >> shift) & 255u;
    }
    const unsigned peers = __match_any_sync(kFull, dg);
    const unsigned rank = __popc(peers & below);
    if (valid && rank == 0) wcnt[wid][dg] = __popc(peers);
    __syncthreads();
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kRadixWarps; w++) {
      const uint32_t c = wcnt[w][t];
      wcnt[w][t] = run;
      run += c;
    }
    round_total[t] = run;
    __syncthreads();
    if (valid) {
      const uint64_t pos = at[dg] + wcnt[wid][dg] + rank;
      keys_out[pos] = key;
      vals_out[pos] = val;
    }
    __syncthreads();
    at[t] += round_total[t];
#pragma unroll
    for (int w = 0; w < kRadixWarps; w++) wcnt[w][t] = 0;
    __syncthreads();
  }
}

// keys[v] = degree, vals[v] = v; *dmax = the largest degree
__global__ void k_degree_pairs(const uint64_t* __restrict__ rp, uint64_t V, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals,
                               unsigned long long* __restrict__ dmax) {
  unsigned long long m = 0;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t d = rp[v + 1] - rp[v];
    keys[v] = (uint32_t)d;
    vals[v] = (uint32_t)v;
    if (d > m) m = d;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long y = __shfl_down_sync(kFull, m, o);
    if (y > m) m = y;
  }
  if (lane_id() == 0 && m) atomicMax(dmax, m);
}

// order[r] = old id of new id r: new_of_old, and the new row lengths
__global__ void k_invert_order(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ order, uint64_t V, uint32_t* __restrict__ new_of_old,
                               uint64_t* __restrict__ new_len) {
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < V; r += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t u = order[r];
    new_of_old[u] = (uint32_t)r;
    new_len[r] = rp[u + 1] - rp[u];
  }
}

// one warp per new source s: its edges as (new destination, s) at nrp[s] ...
__global__ void k_emit_edges(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, const uint32_t* __restrict__ order,
                             const uint32_t* __restrict__ new_of_old, const uint64_t* __restrict__ nrp, uint64_t V, uint32_t* __restrict__ keys,
                             uint32_t* __restrict__ vals) {
  const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / kWarp;
  const unsigned lane = lane_id();
  for (uint64_t s = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; s < V; s += warps) {
    const uint32_t u = order[s];
    const uint64_t a = rp[u], n = rp[u + 1] - a, o = nrp[s];
    for (uint64_t k = lane; k < n; k += kWarp) {
      keys[o + k] = new_of_old[__ldg(ci + a + k)];
      vals[o + k] = (uint32_t)s;
    }
  }
}

// ids[i] = map[ids[i]]
__global__ void k_map_ids(uint32_t* __restrict__ ids, uint64_t n, const uint32_t* __restrict__ map) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) ids[i] = map[ids[i]];
}

}  // namespace dev
}  // namespace vsgm
