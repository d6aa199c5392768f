// k-clique counting by bitmaps of each root's out-neighbourhood (sm_100a).
//
// A clique plan (complete pattern whose order conditions rank every vertex, the
// root the smallest: Clique(k) with the partial order v0 < v1 < ... of
// src/query/clique.h, src/query/partial_order.h) counts at root v0 the k-cliques
// whose smallest vertex is v0.  All of them lie in O = N(v0) above v0, the root's
// out-neighbourhood (d = |O|).  Instead of interpreting the plan's levels - for
// every edge (v0, v1) an intersection staged in shared memory, then one searched
// intersection per child v2 (src/executor/ops/compute.h, materialize.h,
// compute_count.h) - the operator builds O's induced adjacency once, as d bit rows
// in shared memory (row i holds bit j > i iff O[j] is a neighbour of O[i]), and
// counts on the rows:
//   k = 3: sum_i popc(row_i)                                  (edges of O)
//   k = 4: sum_i sum_{j in row_i} popc(row_i & row_j)          (triangles of O)
// With ids ascending with degree, d stays small (on R-MAT scale 22 at most 1,036,
// 91% of the roots at most 32), so a row is one word for most roots and at most 32
// words here.  Roots are split by d: one warp per root with one-word rows (d <= 32),
// one warp per root with rows of up to 8 words (d <= 256), one 16-warp block per root
// with rows of up to 32 words (d <= 1024); larger neighbourhoods go back to the
// level-wise plan.  Exact: every bit is a membership test of the plan's own lists.
#pragma once

#include <cstdint>

#include "kernels.cuh"

namespace vsgm {
namespace dev {

constexpr uint32_t kCliqueSmall = 32;     // out-degree of the one-word tier
constexpr uint32_t kCliqueMid = 256;      // out-degree of the warp tier
constexpr uint32_t kCliqueLarge = 1024;   // out-degree of the block tier
constexpr uint32_t kCliqueMidStride = 9;  // words per row (odd: rows read by different lanes fall in different banks)
constexpr uint32_t kCliqueLargeStride = 33;
constexpr int kCliqueMidWarps = 8;
constexpr int kCliqueLargeWarps = 16;
// dynamic shared memory: per warp O[256] + rows[256][9] + list[256]; per block O[1024] + rows[1024][33] + list[16][1024]
constexpr size_t kCliqueMidWarpWords = kCliqueMid + kCliqueMid * kCliqueMidStride + kCliqueMid;
constexpr size_t kCliqueMidSmem = kCliqueMidWarps * kCliqueMidWarpWords * sizeof(uint32_t);
constexpr size_t kCliqueLargeSmem = (kCliqueLarge + (size_t)kCliqueLarge * kCliqueLargeStride) * sizeof(uint32_t) +
                                    (size_t)kCliqueLargeWarps * kCliqueLarge * sizeof(uint16_t);

struct CliqueTiers {
  uint32_t* root[4];          // small / mid / large / beyond the block tier
  unsigned long long* count;  // [4]
};

// Split roots by out-degree d = |N(v) above v| (up[v] = offset of the first
// neighbour above v) into d <= lim0 / lim1 / lim2 / wider; roots with d < min_d
// are dropped (they hold no clique, or no triangle).
// Warp-aggregated appends: one atomic per tier per warp step.
__global__ void k_clique_split(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ up, const uint32_t* __restrict__ roots, uint64_t n,
                               uint32_t min_d, uint32_t lim0, uint32_t lim1, uint32_t lim2, CliqueTiers t) {
  const unsigned lane = lane_id();
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {
    // base is the warp's first index: every lane of a warp runs the same iterations
    const uint64_t i = base + lane;
    int tier = -1;
    uint32_t v = 0;
    if (i < n) {
      v = __ldg(roots + i);
      const uint64_t d = __ldg(rp + v + 1) - __ldg(rp + v) - __ldg(up + v);
      if (d >= min_d) tier = d <= lim0 ? 0 : d <= lim1 ? 1 : d <= lim2 ? 2 : 3;
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const unsigned m = __ballot_sync(kFull, tier == k);
      if (!m) continue;
      unsigned long long at = 0;
      if (lane == (unsigned)(__ffs(m) - 1)) at = atomicAdd(t.count + k, (unsigned long long)__popc(m));
      at = __shfl_sync(kFull, at, __ffs(m) - 1);
      if (tier == k) t.root[k][at + __popc(m & ((1u << lane) - 1))] = v;
    }
  }
}

// Visits the pairs (i, j), j > i, with O[j] a neighbour of O[i]: on_match(j, pos)
// with pos the position of O[j] in the adjacency array (inside O[i]'s row).  Only
// N(O[i]) above O[i] can hold such O[j].  Walks that part (coalesced, up to O's
// largest value) probing O in shared memory, unless it is much longer than the
// rest of O, which is then probed in N(O[i]) instead.  Lanes call on_match
// independently.  Returns the algorithmic bytes of the row (row offsets, and the
// shorter of the two lists).
template <typename OnMatch>
__device__ __forceinline__ uint32_t out_row_matches(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, const uint32_t* __restrict__ up,
                                                    const uint32_t* O, uint32_t d, uint32_t i, OnMatch&& on_match) {
  const unsigned lane = lane_id();
  const uint32_t rest = d - i - 1;
  if (rest == 0) return 0;
  const uint32_t v = O[i];
  const uint64_t z = __ldg(rp + v + 1);
  const uint64_t s = __ldg(rp + v) + __ldg(up + v);
  if (s >= z) return 16;
  const uint64_t len = z - s;
  if (len > 8ull * rest) {
    for (uint32_t j = i + 1 + lane; j < d; j += kWarp) {
      const uint32_t x = O[j];
      const uint64_t q = lower_bound(ci, s, z, x);
      if (q < z && __ldg(ci + q) == x) on_match(j, q);
    }
    return 16 + 4 * rest;
  }
  const uint32_t omax = O[d - 1];
  uint32_t lo = i + 1;  // this lane's values increase from chunk to chunk
  uint64_t walked = 0;
  for (uint64_t base = s; base < z; base += kWarp) {
    const uint64_t k = base + lane;
    const uint32_t x = k < z ? __ldg(ci + k) : 0xffffffffu;
    if (x <= omax) {
      const uint32_t j = smem_lower_bound(O, lo, d, x);
      lo = j;
      if (j < d && O[j] == x) on_match(j, k);
    }
    walked += kWarp;
    if (__any_sync(kFull, x >= omax)) break;
  }
  return 16 + 4 * (uint32_t)(walked < len ? walked : len);
}

// Row i of O's induced adjacency: bit j (j > i) of row[] set iff O[j] is in N(O[i]).
__device__ __forceinline__ uint32_t clique_build_row(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, const uint32_t* __restrict__ up,
                                                     const uint32_t* O, uint32_t d, uint32_t i, uint32_t* row) {
  return out_row_matches(rp, ci, up, O, d, i, [&](uint32_t j, uint64_t) { atomicOr(row + (j >> 5), 1u << (j & 31)); });
}

// sum over the set bits j of row i of popc(row_i & row_j), rows of `stride` words
// holding W words each; the bits of row i are listed in L first so that every lane
// takes one j.  All lanes return the same value only after the caller's reduction.
__device__ __forceinline__ unsigned long long clique_count_row(const uint32_t* R, uint32_t stride, uint32_t W, uint32_t i, uint32_t* L16or32,
                                                               bool list16) {
  const unsigned lane = lane_id();
  const uint32_t* ri = R + (size_t)i * stride;
  uint32_t n = 0;
  for (uint32_t w = (i + 1) >> 5; w < W; w++) {
    const uint32_t m = ri[w];
    if ((m >> lane) & 1u) {
      const uint32_t at = n + __popc(m & ((1u << lane) - 1));
      if (list16)
        ((uint16_t*)L16or32)[at] = (uint16_t)(w * 32 + lane);
      else
        L16or32[at] = w * 32 + lane;
    }
    n += __popc(m);
  }
  __syncwarp();
  unsigned long long acc = 0;
  for (uint32_t t = lane; t < n; t += kWarp) {
    const uint32_t j = list16 ? (uint32_t)((const uint16_t*)L16or32)[t] : L16or32[t];
    const uint32_t* rj = R + (size_t)j * stride;
    uint32_t c = 0;
    for (uint32_t w = j >> 5; w < W; w++) c += __popc(ri[w] & rj[w]);
    acc += c;
  }
  __syncwarp();
  return acc;
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long x) {
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(kFull, x, o);
  return x;
}

// d <= 32: a warp per root; lane i holds O[i] and (after the build) row i.
template <int K>
__global__ void __launch_bounds__(256) k_clique_small(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, const uint32_t* __restrict__ up,
                                                      const uint32_t* __restrict__ roots, uint64_t n, unsigned long long* __restrict__ total,
                                                      unsigned long long* __restrict__ bytes) {
  __shared__ uint32_t sO[8][kCliqueSmall];
  __shared__ uint32_t sR[8][kCliqueSmall];
  const unsigned lane = lane_id(), wid = threadIdx.x / kWarp;
  uint32_t* O = sO[wid];
  uint32_t* R = sR[wid];
  unsigned long long acc = 0, acc_bytes = 0;
  const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / kWarp;
  for (uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; r < n; r += warps) {
    const uint32_t v0 = __ldg(roots + r);
    const uint64_t a = __ldg(rp + v0) + __ldg(up + v0);
    const uint32_t d = (uint32_t)(__ldg(rp + v0 + 1) - a);
    O[lane] = lane < d ? __ldg(ci + a + lane) : 0xffffffffu;
    R[lane] = 0;
    __syncwarp();
    uint32_t b = 16 + 4 * d;
    for (uint32_t i = 0; i + 1 < d; i++) b += clique_build_row(rp, ci, up, O, d, i, R + i);  // one word per row
    __syncwarp();
    const uint32_t ri = lane < d ? R[lane] : 0u;
    if (K == 3) {
      acc += __popc(ri);
    } else {
      uint32_t m = ri;
      while (m) {
        const int j = __ffs(m) - 1;
        m &= m - 1;
        acc += __popc(ri & R[j]);
      }
    }
    if (bytes && lane == 0) acc_bytes += b;
    __syncwarp();
  }
  acc = warp_sum(acc);
  if (bytes) acc_bytes = warp_sum(acc_bytes);
  if (lane == 0) {
    if (acc) atomicAdd(total, acc);
    if (bytes && acc_bytes) atomicAdd(bytes, acc_bytes);
  }
}

// d <= 256: a warp per root, rows of up to 8 words; roots popped from *head.
template <int K>
__global__ void __launch_bounds__(256, 2) k_clique_mid(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, const uint32_t* __restrict__ up,
                                                       const uint32_t* __restrict__ roots, uint64_t n, unsigned long long* __restrict__ head,
                                                       unsigned long long* __restrict__ total, unsigned long long* __restrict__ bytes) {
  extern __shared__ uint32_t smem[];
  const unsigned lane = lane_id(), wid = threadIdx.x / kWarp;
  uint32_t* O = smem + (size_t)wid * kCliqueMidWarpWords;
  uint32_t* R = O + kCliqueMid;
  uint32_t* L = R + kCliqueMid * kCliqueMidStride;
  unsigned long long acc = 0, acc_bytes = 0;
  while (true) {
    unsigned long long r = 0;
    if (lane == 0) r = atomicAdd(head, 1ull);
    r = __shfl_sync(kFull, r, 0);
    if (r >= n) break;
    const uint32_t v0 = __ldg(roots + r);
    const uint64_t a = __ldg(rp + v0) + __ldg(up + v0);
    const uint32_t d = (uint32_t)(__ldg(rp + v0 + 1) - a);
    const uint32_t W = (d + 31) / 32;
    for (uint32_t t = lane; t < d; t += kWarp) O[t] = __ldg(ci + a + t);
    for (uint32_t t = lane; t < d * kCliqueMidStride; t += kWarp) R[t] = 0;
    __syncwarp();
    uint32_t b = 16 + 4 * d;
    for (uint32_t i = 0; i + 1 < d; i++) b += clique_build_row(rp, ci, up, O, d, i, R + i * kCliqueMidStride);
    __syncwarp();
    if (K == 3) {
      for (uint32_t t = lane; t < d * kCliqueMidStride; t += kWarp) acc += __popc(R[t]);
    } else {
      for (uint32_t i = 0; i + 2 < d; i++) acc += clique_count_row(R, kCliqueMidStride, W, i, L, false);
    }
    if (bytes && lane == 0) acc_bytes += b;
    __syncwarp();
  }
  acc = warp_sum(acc);
  if (bytes) acc_bytes = warp_sum(acc_bytes);
  if (lane == 0) {
    if (acc) atomicAdd(total, acc);
    if (bytes && acc_bytes) atomicAdd(bytes, acc_bytes);
  }
}

// d <= 1024: a block of 16 warps per root, rows of up to 32 words; warps take rows
// round-robin in both phases.
template <int K>
__global__ void __launch_bounds__(kCliqueLargeWarps * kWarp, 1)
    k_clique_large(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, const uint32_t* __restrict__ up, const uint32_t* __restrict__ roots,
                   uint64_t n, unsigned long long* __restrict__ head, unsigned long long* __restrict__ total, unsigned long long* __restrict__ bytes) {
  extern __shared__ uint32_t smem[];
  __shared__ unsigned long long s_root;
  __shared__ unsigned long long s_sum[kCliqueLargeWarps][2];
  const unsigned lane = lane_id(), wid = threadIdx.x / kWarp;
  uint32_t* O = smem;
  uint32_t* R = O + kCliqueLarge;
  uint16_t* L = (uint16_t*)(R + (size_t)kCliqueLarge * kCliqueLargeStride) + (size_t)wid * kCliqueLarge;
  unsigned long long acc = 0, acc_bytes = 0;
  while (true) {
    if (threadIdx.x == 0) s_root = atomicAdd(head, 1ull);
    __syncthreads();
    const unsigned long long r = s_root;
    if (r >= n) break;
    const uint32_t v0 = __ldg(roots + r);
    const uint64_t a = __ldg(rp + v0) + __ldg(up + v0);
    const uint32_t d = (uint32_t)(__ldg(rp + v0 + 1) - a);
    const uint32_t W = (d + 31) / 32;
    for (uint32_t t = threadIdx.x; t < d; t += blockDim.x) O[t] = __ldg(ci + a + t);
    for (uint32_t t = threadIdx.x; t < d * kCliqueLargeStride; t += blockDim.x) R[t] = 0;
    __syncthreads();
    uint32_t b = wid == 0 ? 16 + 4 * d : 0;
    for (uint32_t i = wid; i + 1 < d; i += kCliqueLargeWarps) b += clique_build_row(rp, ci, up, O, d, i, R + i * kCliqueLargeStride);
    __syncthreads();
    if (K == 3) {
      for (uint32_t t = threadIdx.x; t < d * kCliqueLargeStride; t += blockDim.x) acc += __popc(R[t]);
    } else {
      for (uint32_t i = wid; i + 2 < d; i += kCliqueLargeWarps) acc += clique_count_row(R, kCliqueLargeStride, W, i, (uint32_t*)L, true);
    }
    if (bytes && lane == 0) acc_bytes += b;
    __syncthreads();  // the next root overwrites O and the rows
  }
  acc = warp_sum(acc);
  if (bytes) acc_bytes = warp_sum(acc_bytes);
  if (lane == 0) {
    s_sum[wid][0] = acc;
    s_sum[wid][1] = acc_bytes;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0, tb = 0;
    for (int w = 0; w < kCliqueLargeWarps; w++) {
      t += s_sum[w][0];
      tb += s_sum[w][1];
    }
    if (t) atomicAdd(total, t);
    if (bytes && tb) atomicAdd(bytes, tb);
  }
}

// ---------------------------------------------------------------------------
// Triangles per edge, for the diamond plan (pm_pipeline -p 2: two triangles on a
// shared edge, src/query/pattern.h).  t[k], for the adjacency slot k of an edge
// (u, v) with u < v (k inside u's row), receives the number of triangles on that
// edge that have their smallest vertex among the roots given: each triangle
// a < b < c is found once, at root a, as the pair (i, j) of row i of O = N(a) above
// a (b = O[i], c = O[j]).  The edge (b, c) gets +1 at its slot, found by the walk;
// the edges (a, b) and (a, c) collect per-member counts in shared memory (row
// count of b plus column count of c) and are added once per root.
// ---------------------------------------------------------------------------
constexpr uint32_t kTriSmall = 32;    // warp per root, O and counts in static shared memory
constexpr uint32_t kTriMid = 1024;    // warp per root, 8 KB of shared memory per warp (measured: a 256 cut with the block tier above it took -p 2 from 134 to 152 ms)
constexpr uint32_t kTriLarge = 16384; // block per root, 128 KB of shared memory
constexpr size_t kTriMidSmem = 8ull * 2 * kTriMid * sizeof(uint32_t);
constexpr size_t kTriLargeSmem = 2ull * kTriLarge * sizeof(uint32_t);

// the triangles of one root a whose O (d members) and counters cnt[d] (zeroed) are
// in shared memory; warps take rows wid, wid + nwarps, ...  Counter updates are
// shared-memory atomics because other warps add column counts concurrently.
// is_src (byte per vertex): the sources whose out-edges are summed.  A root that is
// not one of them only feeds the edges (O[i], O[j]) with O[i] a source, so its other
// rows are skipped (with the sources spread over several GPUs, each does its share).
__device__ __forceinline__ uint32_t edge_tri_rows(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, const uint32_t* __restrict__ up,
                                                  const uint8_t* __restrict__ is_src, bool root_is_src, const uint32_t* O, uint32_t* cnt, uint32_t d,
                                                  uint32_t wid, uint32_t nwarps, uint32_t* __restrict__ t) {
  const unsigned lane = lane_id();
  uint32_t b = 0;
  for (uint32_t i = wid; i + 1 < d; i += nwarps) {
    if (!root_is_src && !is_src[O[i]]) continue;
    uint32_t c = 0;
    b += out_row_matches(rp, ci, up, O, d, i, [&](uint32_t j, uint64_t pos) {
      atomicAdd(t + pos, 1u);
      atomicAdd(cnt + j, 1u);
      c++;
    });
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(kFull, c, o);
    if (lane == 0 && c) atomicAdd(cnt + i, c);
  }
  return b;
}

// d <= DMAX: a warp per root (roots popped from *head)
template <uint32_t DMAX>
__global__ void __launch_bounds__(256) k_edge_tri_warp(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, const uint32_t* __restrict__ up,
                                                       const uint8_t* __restrict__ is_src, const uint32_t* __restrict__ roots, uint64_t n,
                                                       unsigned long long* __restrict__ head, uint32_t* __restrict__ t,
                                                       unsigned long long* __restrict__ bytes) {
  extern __shared__ uint32_t smem[];
  const unsigned lane = lane_id(), wid = threadIdx.x / kWarp;
  uint32_t* O = smem + (size_t)wid * 2 * DMAX;
  uint32_t* cnt = O + DMAX;
  unsigned long long acc_bytes = 0;
  while (true) {
    unsigned long long r = 0;
    if (lane == 0) r = atomicAdd(head, 1ull);
    r = __shfl_sync(kFull, r, 0);
    if (r >= n) break;
    const uint32_t a = __ldg(roots + r);
    const uint64_t base = __ldg(rp + a) + __ldg(up + a);
    const uint32_t d = (uint32_t)(__ldg(rp + a + 1) - base);
    for (uint32_t k = lane; k < d; k += kWarp) {
      O[k] = __ldg(ci + base + k);
      cnt[k] = 0;
    }
    __syncwarp();
    const bool a_src = is_src[a] != 0;
    const uint32_t b = edge_tri_rows(rp, ci, up, is_src, a_src, O, cnt, d, 0, 1, t);
    __syncwarp();
    if (a_src)
      for (uint32_t k = lane; k < d; k += kWarp)
        if (cnt[k]) atomicAdd(t + base + k, cnt[k]);
    if (bytes && lane == 0) acc_bytes += 16 + 4ull * d + b;
    __syncwarp();
  }
  acc_bytes = warp_sum(acc_bytes);
  if (bytes && lane == 0 && acc_bytes) atomicAdd(bytes, acc_bytes);
}

// d <= kTriLarge: a block per root
__global__ void __launch_bounds__(512, 1) k_edge_tri_block(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, const uint32_t* __restrict__ up,
                                                           const uint8_t* __restrict__ is_src, const uint32_t* __restrict__ roots, uint64_t n,
                                                           unsigned long long* __restrict__ head, uint32_t* __restrict__ t,
                                                           unsigned long long* __restrict__ bytes) {
  extern __shared__ uint32_t smem[];
  __shared__ unsigned long long s_root;
  const unsigned lane = lane_id(), wid = threadIdx.x / kWarp, nwarps = blockDim.x / kWarp;
  uint32_t* O = smem;
  uint32_t* cnt = O + kTriLarge;
  unsigned long long acc_bytes = 0;
  while (true) {
    if (threadIdx.x == 0) s_root = atomicAdd(head, 1ull);
    __syncthreads();
    const unsigned long long r = s_root;
    if (r >= n) break;
    const uint32_t a = __ldg(roots + r);
    const uint64_t base = __ldg(rp + a) + __ldg(up + a);
    const uint32_t d = (uint32_t)(__ldg(rp + a + 1) - base);
    for (uint32_t k = threadIdx.x; k < d; k += blockDim.x) {
      O[k] = __ldg(ci + base + k);
      cnt[k] = 0;
    }
    __syncthreads();
    const bool a_src = is_src[a] != 0;
    const uint32_t b = edge_tri_rows(rp, ci, up, is_src, a_src, O, cnt, d, wid, nwarps, t);
    __syncthreads();
    if (a_src)
      for (uint32_t k = threadIdx.x; k < d; k += blockDim.x)
        if (cnt[k]) atomicAdd(t + base + k, cnt[k]);
    if (bytes && lane == 0) acc_bytes += b + (wid == 0 ? 16 + 4ull * d : 0);
    __syncthreads();  // the next root overwrites O and the counters
  }
  acc_bytes = warp_sum(acc_bytes);
  if (bytes && lane == 0 && acc_bytes) atomicAdd(bytes, acc_bytes);
}

// roots whose triangles can lie on an out-edge of a source s: s itself and its
// neighbours below it (a triangle on (s, v), s < v, has its smallest vertex at s
// or at a common neighbour below s)
__global__ void k_tri_mark_roots(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, const uint32_t* __restrict__ up,
                                 const uint32_t* __restrict__ src, uint64_t n, uint8_t* __restrict__ flags, uint8_t* __restrict__ is_src) {
  const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / kWarp;
  const unsigned lane = lane_id();
  for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; i < n; i += warps) {
    const uint32_t s = __ldg(src + i);
    if (lane == 0) {
      set_flag(flags, s);
      set_flag(is_src, s);
    }
    const uint64_t a = __ldg(rp + s), z = a + __ldg(up + s);
    for (uint64_t k = a + lane; k < z; k += kWarp) set_flag(flags, __ldg(ci + k));
  }
}

__global__ void k_flags_to_list(const uint8_t* __restrict__ flags, uint64_t V, uint32_t* __restrict__ out, unsigned long long* __restrict__ count) {
  const unsigned lane = lane_id();
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < V; base += stride) {
    const uint64_t v = base + lane;
    const bool on = v < V && flags[v];
    const unsigned m = __ballot_sync(kFull, on);
    if (!m) continue;
    unsigned long long at = 0;
    if (lane == (unsigned)(__ffs(m) - 1)) at = atomicAdd(count, (unsigned long long)__popc(m));
    at = __shfl_sync(kFull, at, __ffs(m) - 1);
    if (on) out[at + __popc(m & ((1u << lane) - 1))] = (uint32_t)v;
  }
}

// per source a: sum over its edges (a, b), b > a, of the pairs of the t(a, b)
// common neighbours (mode 1: C(t, 2), the two wings ordered; mode 2: t (t - 1))
__global__ void k_diamond_sum(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ up, const uint32_t* __restrict__ src, uint64_t n,
                              const uint32_t* __restrict__ t, int mode, unsigned long long* __restrict__ total, unsigned long long* __restrict__ bytes) {
  const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / kWarp;
  const unsigned lane = lane_id();
  unsigned long long acc = 0, acc_bytes = 0;
  for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; i < n; i += warps) {
    const uint32_t s = __ldg(src + i);
    const uint64_t z = __ldg(rp + s + 1), a = __ldg(rp + s) + __ldg(up + s);
    for (uint64_t k = a + lane; k < z; k += kWarp) {
      const unsigned long long c = __ldg(t + k);
      acc += mode == 1 ? c * (c ? c - 1 : 0) / 2 : c * (c ? c - 1 : 0);
    }
    if (lane == 0) acc_bytes += 16 + 4 * (z - a);
  }
  acc = warp_sum(acc);
  if (bytes) acc_bytes = warp_sum(acc_bytes);
  if (lane == 0) {
    if (acc) atomicAdd(total, acc);
    if (bytes && acc_bytes) atomicAdd(bytes, acc_bytes);
  }
}

}  // namespace dev
}  // namespace vsgm
