// The view-producing tools on the device: the feature graph (features -h 1),
// cosine k-means over adjacency rows (kmeans -init 1) and next-fit view-bin
// packing (view_packing -s 1).  Each gives exactly the reference tool's output:
//
//   - features: every row gets its own vertex inserted in sorted position
//     (src/tools/features.cc:177-201 appends it and re-sorts the row);
//   - k-means: the reference sums doubles in a fixed order (a centroid entry over
//     the cluster's vertices in increasing id, a similarity over the row in
//     increasing column, a squared norm over the entries in increasing index).
//     Floating-point sums are order-dependent, so every sum here runs in that
//     same order with explicitly rounded multiplies and adds (no fused
//     multiply-add); the parallelism is across vertices and clusters, never
//     inside one sum.  A centroid entry is gathered over the feature's own row
//     (the graph is undirected, so the vertices whose rows hold feature f are
//     exactly the row of f, already in increasing id);
//   - packing: the reference grows one bin at a time, source by source, each
//     source adding its (hop-1)-ball's rows not yet in the bin
//     (src/tools/view_bin.h:22-138).  Here a whole chunk of consecutive sources
//     is labelled at once: every vertex gets the first chunk position whose ball
//     reaches it (a min-label propagation over hop-1 rounds), each vertex's row
//     size is credited to that position, and a prefix sum over the chunk finds
//     the first source that no longer fits - the same bin boundary the
//     sequential walk finds.  Sources after that boundary are relabelled against
//     the new bin.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <numeric>
#include <string>
#include <utility>
#include <vector>

#include "graph.hpp"
#include "vsgm.h"

namespace {

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;
__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

struct ToolError {
  int code;
  std::string msg;
};

#define TK(x)                                                                                                                   \
  do {                                                                                                                          \
    cudaError_t e_ = (x);                                                                                                       \
    if (e_ != cudaSuccess)                                                                                                      \
      throw ToolError{VSGM_ECUDA, std::string("CUDA error ") + cudaGetErrorString(e_) + " at partition.cu:" + std::to_string(__LINE__) + \
                                      " in " #x};                                                                               \
  } while (0)

// device buffers of one tool call, freed when the call returns
struct DevBufs {
  std::vector<void*> ptrs;
  template <typename T>
  T* take(uint64_t n) {
    void* p = nullptr;
    TK(cudaMalloc(&p, std::max<uint64_t>(n, 1) * sizeof(T)));
    ptrs.push_back(p);
    return (T*)p;
  }
  ~DevBufs() {
    for (void* p : ptrs) cudaFree(p);
  }
};

struct Stream {
  cudaStream_t s = nullptr;
  Stream() { TK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
  ~Stream() {
    if (s) cudaStreamDestroy(s);
  }
};

template <typename F>
int tool_call(int device, F&& body) {
  try {
    TK(cudaSetDevice(device));
    body();
    return VSGM_OK;
  } catch (const ToolError& t) {
    vsgm::set_host_error(t.msg);
    return t.code;
  } catch (const std::bad_alloc&) {
    vsgm::set_host_error("host memory exhausted");
    return VSGM_ENOMEM;
  } catch (const std::exception& x) {
    vsgm::set_host_error(x.what());
    return VSGM_EINVAL;
  }
}

unsigned grid_for(uint64_t items, unsigned per_block) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint64_t want = (items + per_block - 1) / per_block;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)sms * 16));
}

// ---------------------------------------------------------------------------
// features -h 1
// ---------------------------------------------------------------------------
// warp per row v: the row copied with v inserted after every entry <= v
__global__ void k_self_loops(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, uint64_t V, uint64_t* __restrict__ out_rp,
                             uint32_t* __restrict__ out_ci) {
  const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / kWarp;
  const unsigned lane = lane_id();
  for (uint64_t v = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; v < V; v += warps) {
    const uint64_t a = rp[v], z = rp[v + 1], o = a + v;  // v rows before this one gained one entry each
    if (lane == 0) {
      out_rp[v] = o;
      if (v + 1 == V) out_rp[V] = z + V;
    }
    uint64_t below = 0;  // entries <= v seen in earlier strides
    for (uint64_t base = a; base < z; base += kWarp) {
      const uint64_t j = base + lane;
      const bool in = j < z;
      const uint32_t x = in ? ci[j] : 0xffffffffu;
      const bool le = in && x <= (uint32_t)v;
      const unsigned m = __ballot_sync(kFull, le);
      if (in) out_ci[o + (j - a) + (le ? 0 : 1)] = x;
      below += __popc(m);
    }
    if (lane == 0) out_ci[o + below] = (uint32_t)v;
  }
}

// ---------------------------------------------------------------------------
// cosine k-means (src/tools/kmeans.cc:54-247, 386-505; similarity and centroid
// update in src/tools/kmeans_utils.h:40-160).  Centroids are dense over the F = V features,
// stored feature-major (cen[f * K + k]) so that the K entries one row entry needs
// sit in one or two sectors.
// ---------------------------------------------------------------------------
constexpr int kMaxClusterWords = 4;  // clusters k = lane + 32 j, j < 4: K <= 128

// weight of every entry of v's row: sqrt(1 / deg(v)), as the reference computes it
__global__ void k_row_weights(const uint64_t* __restrict__ rp, uint64_t V, double* __restrict__ w) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x)
    w[v] = sqrt(1.0 / (double)(rp[v + 1] - rp[v]));
}

// entries (v, f) whose reverse (f, v) is missing: the gather below needs an
// undirected graph
__global__ void k_asymmetric(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, uint64_t V, unsigned long long* __restrict__ bad) {
  const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / kWarp;
  const unsigned lane = lane_id();
  unsigned long long n = 0;
  for (uint64_t v = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; v < V; v += warps) {
    for (uint64_t j = rp[v] + lane; j < rp[v + 1]; j += kWarp) {
      const uint32_t f = ci[j];
      if (f >= V) {
        n++;
        continue;
      }
      uint64_t lo = rp[f], hi = rp[f + 1];
      while (lo < hi) {
        const uint64_t mid = (lo + hi) / 2;
        if (ci[mid] < (uint32_t)v)
          lo = mid + 1;
        else
          hi = mid;
      }
      if (lo == rp[f + 1] || ci[lo] != (uint32_t)v) n++;
    }
  }
  if (n) atomicAdd(bad, n);
}

// RandomInit (kmeans.cc:125-141): thread p of T starts at cluster starts[p] and
// hands its vertices p, p + T, ... consecutive clusters
__global__ void k_random_init(uint64_t V, const int32_t* __restrict__ starts, int T, int K, int32_t* __restrict__ assign) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x)
    assign[v] = (int32_t)(((uint64_t)starts[v % T] + v / T) % (uint64_t)K);
}

__global__ void k_cluster_sizes(const int32_t* __restrict__ assign, uint64_t V, unsigned long long* __restrict__ sizes) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x)
    atomicAdd(sizes + assign[v], 1ull);
}

// UpdateAllCentroids (kmeans.cc:171-196): entry f of centroid k is the sum of
// w[v] over the members v of cluster k whose row holds f, in increasing v, then
// divided by the cluster's size.  Warp per feature f walks N(f) (= the vertices
// whose rows hold f) in order; lane k % 32 owns cluster k's running sum.
__global__ void k_centroids(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, uint64_t F, const int32_t* __restrict__ assign,
                            const double* __restrict__ w, const unsigned long long* __restrict__ sizes, int K, double* __restrict__ cen) {
  const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / kWarp;
  const unsigned lane = lane_id();
  for (uint64_t f = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; f < F; f += warps) {
    double acc[kMaxClusterWords] = {0.0, 0.0, 0.0, 0.0};
    const uint64_t a = rp[f], z = rp[f + 1];
    for (uint64_t base = a; base < z; base += kWarp) {
      const uint64_t j = base + lane;
      int32_t c = -1;
      double x = 0.0;
      if (j < z) {
        const uint32_t v = ci[j];
        c = assign[v];
        x = w[v];
      }
      const int n = (int)(z - base < (uint64_t)kWarp ? z - base : (uint64_t)kWarp);
      for (int t = 0; t < n; t++) {
        const int ct = __shfl_sync(kFull, c, t);
        const double xt = __shfl_sync(kFull, x, t);
        if ((unsigned)(ct & 31) == lane) {
#pragma unroll
          for (int q = 0; q < kMaxClusterWords; q++)
            if (q == (ct >> 5)) acc[q] = __dadd_rn(acc[q], xt);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < kMaxClusterWords; q++) {
      const int k = (int)lane + 32 * q;
      if (k < K) {
        const unsigned long long sz = sizes[k];
        cen[f * K + k] = sz ? __ddiv_rn(acc[q], (double)(int)sz) : acc[q];
      }
    }
  }
}

// DenseVector::update_sqr_sum (kmeans_utils.h:43-48): warp per cluster, the
// squares summed in increasing feature order (the multiplies are independent,
// the adds form one chain, as in the reference)
__global__ void k_sqr_sums(const double* __restrict__ cen, uint64_t F, int K, double* __restrict__ sqr) {
  const int k = (int)(((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp);
  if (k >= K) return;
  const unsigned lane = lane_id();
  double s = 0.0;
  double next = lane < F ? cen[(uint64_t)lane * K + k] : 0.0;
  for (uint64_t base = 0; base < F; base += kWarp) {
    const double cur = next;
    const uint64_t j = base + kWarp + lane;
    next = j < F ? cen[j * K + k] : 0.0;  // the next batch is in flight while this one is summed
    const double sq = __dmul_rn(cur, cur);
    const int n = (int)(F - base < (uint64_t)kWarp ? F - base : (uint64_t)kWarp);
    for (int t = 0; t < n; t++) s = __dadd_rn(s, __shfl_sync(kFull, sq, t));
  }
  if (lane == 0) sqr[k] = s;
}

// UpdateAssignment (kmeans.cc:198-211) with CosineSimilarity (kmeans_utils.h:142-151):
// warp per vertex v; lane k % 32 sums cen[f][k] * w[v] over v's row in order, the
// similarity is that sum over sqrt(|c_k|^2), and the first strictly largest wins
__global__ void k_assign(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, uint64_t V, const double* __restrict__ w,
                         const double* __restrict__ cen, const double* __restrict__ sqr, int K, int32_t* __restrict__ assign) {
  const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / kWarp;
  const unsigned lane = lane_id();
  for (uint64_t v = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; v < V; v += warps) {
    const double wv = w[v];
    double s[kMaxClusterWords] = {0.0, 0.0, 0.0, 0.0};
    const uint64_t a = rp[v], z = rp[v + 1];
    for (uint64_t base = a; base < z; base += kWarp) {
      const uint64_t j = base + lane;
      const uint32_t col = j < z ? ci[j] : 0u;
      const int n = (int)(z - base < (uint64_t)kWarp ? z - base : (uint64_t)kWarp);
#pragma unroll
      for (int q = 0; q < kMaxClusterWords; q++) {
        const int k = (int)lane + 32 * q;
        if (32 * q >= K) break;
        int t = 0;
        for (; t + 4 <= n; t += 4) {  // four loads in flight, then the four adds in order
          double c4[4];
#pragma unroll
          for (int u = 0; u < 4; u++) {
            const uint32_t f = __shfl_sync(kFull, col, t + u);
            c4[u] = k < K ? cen[(uint64_t)f * K + k] : 0.0;
          }
#pragma unroll
          for (int u = 0; u < 4; u++) s[q] = __dadd_rn(s[q], __dmul_rn(c4[u], wv));
        }
        for (; t < n; t++) {
          const uint32_t f = __shfl_sync(kFull, col, t);
          const double c = k < K ? cen[(uint64_t)f * K + k] : 0.0;
          s[q] = __dadd_rn(s[q], __dmul_rn(c, wv));
        }
      }
    }
    int best = 0;
    double best_sim = 0.0;
#pragma unroll
    for (int q = 0; q < kMaxClusterWords; q++) {
      if (32 * q >= K) break;
      const int k = (int)lane + 32 * q;
      const double sim = k < K ? __ddiv_rn(s[q], __dsqrt_rn(sqr[k])) : 0.0;
      for (int t = 0; t < 32 && 32 * q + t < K; t++) {
        const double st = __shfl_sync(kFull, sim, t);
        const int kt = 32 * q + t;
        if (kt == 0)
          best_sim = st;
        else if (st > best_sim) {
          best = kt;
          best_sim = st;
        }
      }
    }
    if (lane == 0) assign[v] = best;
  }
}

// non-zero entries of centroids c < n (the -rc reordering, kmeans.cc:452-471)
__global__ void k_nonzeros(const double* __restrict__ cen, uint64_t F, int K, int n, unsigned long long* __restrict__ out) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < F * (uint64_t)n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t f = i / n;
    const int c = (int)(i % n);
    if (cen[f * K + c] != 0.0) atomicAdd(out + c, 1ull);
  }
}

// ---------------------------------------------------------------------------
// next-fit view-bin packing (src/tools/view_bin.h:22-138 with a pool of one bin,
// src/tools/view_packing.cc:141-246).  A label is (tag << 32) | chunk position:
// every pass has a smaller tag than the passes before it, so atomicMin both
// replaces a stale label and keeps the smallest position of the current pass,
// and no label array is ever cleared.  A vertex is touched first in a pass when
// the label it replaced carried a larger tag; the first toucher lists it.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool first_touch(unsigned long long old, uint32_t tag) { return (uint32_t)(old >> 32) > tag; }
__device__ __forceinline__ bool current(unsigned long long l, uint32_t tag) { return (uint32_t)(l >> 32) == tag; }

// round 0: each source of the chunk is at distance 0 from its own position
__global__ void k_pack_sources(const uint32_t* __restrict__ order, uint64_t L, uint32_t tag, unsigned long long* __restrict__ lab1,
                               uint32_t* __restrict__ T1, unsigned long long* __restrict__ nT1) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < L; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t s = order[i];
    const unsigned long long old = atomicMin(lab1 + s, ((unsigned long long)tag << 32) | i);
    if (first_touch(old, tag)) T1[atomicAdd(nT1, 1ull)] = s;
  }
}

// round 1: warp per source, its neighbours take the source's position
__global__ void k_pack_round1(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, const uint32_t* __restrict__ order, uint64_t L,
                              uint32_t tag, unsigned long long* __restrict__ lab1, uint32_t* __restrict__ T1, unsigned long long* __restrict__ nT1) {
  const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / kWarp;
  const unsigned lane = lane_id();
  for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; i < L; i += warps) {
    const uint32_t s = order[i];
    const unsigned long long key = ((unsigned long long)tag << 32) | i;
    for (uint64_t j = rp[s] + lane; j < rp[s + 1]; j += kWarp) {
      const uint32_t m = ci[j];
      const unsigned long long old = atomicMin(lab1 + m, key);
      if (first_touch(old, tag)) T1[atomicAdd(nT1, 1ull)] = m;
    }
  }
}

// round 2 (hop 3): warp per vertex x within distance 1 of a chunk source; its
// neighbours take x's label into lab2 (lab1 is only read here, so a label moves
// one step per round).  x within distance 1 of a source already in the bin is
// skipped: its neighbours are all in the bin (the reference skips visited
// vertices the same way, view_bin.h:44-48).
__global__ void k_pack_round2(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, const uint32_t* __restrict__ T1,
                              const unsigned long long* __restrict__ nT1, uint32_t tag, const unsigned long long* __restrict__ lab1,
                              unsigned long long* __restrict__ lab2, const uint32_t* __restrict__ visited, uint32_t stamp,
                              uint32_t* __restrict__ T2, unsigned long long* __restrict__ nT2) {
  const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / kWarp;
  const unsigned lane = lane_id();
  const uint64_t n = *nT1;
  for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; i < n; i += warps) {
    const uint32_t x = T1[i];
    if (visited[x] == stamp) continue;
    const unsigned long long lx = lab1[x];
    for (uint64_t j = rp[x] + lane; j < rp[x + 1]; j += kWarp) {
      const uint32_t m = ci[j];
      const unsigned long long old = atomicMin(lab2 + m, lx);
      if (first_touch(old, tag)) T2[atomicAdd(nT2, 1ull)] = m;
    }
  }
}

// final label of a touched vertex: the smaller current label of the two rounds
__device__ __forceinline__ unsigned long long final_label(const unsigned long long* lab1, const unsigned long long* lab2, uint32_t m, uint32_t tag,
                                                          bool* in_T1) {
  const unsigned long long l1 = lab1[m], l2 = lab2[m];
  *in_T1 = current(l1, tag);
  if (!*in_T1) return l2;
  return current(l2, tag) ? min(l1, l2) : l1;
}

// each touched vertex not yet in the bin adds its row size to the position
// that reaches it first; lists T1 then T2 (a vertex in both counts via T1)
__global__ void k_pack_contrib(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ T1, const unsigned long long* __restrict__ nT1,
                               const uint32_t* __restrict__ T2, const unsigned long long* __restrict__ nT2, uint32_t tag,
                               const unsigned long long* __restrict__ lab1, const unsigned long long* __restrict__ lab2,
                               const uint32_t* __restrict__ added, uint32_t stamp, unsigned long long* __restrict__ contrib) {
  const uint64_t n1 = *nT1, n = n1 + *nT2;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t m = i < n1 ? T1[i] : T2[i - n1];
    bool in_T1;
    const unsigned long long l = final_label(lab1, lab2, m, tag, &in_T1);
    if (i >= n1 && in_T1) continue;
    if (added[m] == stamp) continue;
    const unsigned long long d = rp[m + 1] - rp[m];
    if (d) atomicAdd(contrib + (uint32_t)l, d);
  }
}

// first chunk position whose source no longer fits: run + prefix[i + 1] > cap
__global__ void k_pack_close(const uint64_t* __restrict__ prefix, uint64_t L, unsigned long long run, unsigned long long cap,
                             unsigned long long* __restrict__ out) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < L; i += (uint64_t)gridDim.x * blockDim.x)
    if (run + prefix[i + 1] > cap) atomicMin(out, (unsigned long long)i);
}

// out[1] = size the sources before the boundary add
__global__ void k_pack_take(const uint64_t* __restrict__ prefix, uint64_t L, unsigned long long* __restrict__ out) {
  if (blockIdx.x == 0 && threadIdx.x == 0) out[1] = prefix[min((unsigned long long)L, out[0])];
}

// the sources before position c join the bin: what they reach is added, what
// lies within distance 1 of them is visited
__global__ void k_pack_commit(const uint32_t* __restrict__ T1, const unsigned long long* __restrict__ nT1, const uint32_t* __restrict__ T2,
                              const unsigned long long* __restrict__ nT2, uint32_t tag, const unsigned long long* __restrict__ lab1,
                              const unsigned long long* __restrict__ lab2, uint64_t c, uint32_t stamp, uint32_t* __restrict__ added,
                              uint32_t* __restrict__ visited) {
  const uint64_t n1 = *nT1, n = n1 + *nT2;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t m = i < n1 ? T1[i] : T2[i - n1];
    bool in_T1;
    const unsigned long long l = final_label(lab1, lab2, m, tag, &in_T1);
    if (i >= n1 && in_T1) continue;
    if ((uint32_t)l < c) added[m] = stamp;
    if (in_T1 && (uint32_t)lab1[m] < c) visited[m] = stamp;
  }
}

__global__ void k_set_u64(unsigned long long* p, unsigned long long v) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *p = v;
}

}  // namespace

namespace {

// exclusive scan of a chunk's n <= 2^20 contributions into out[0..n] (out[n] =
// total): per-tile sums, one block scanning the <= 512 tile sums, then each
// tile scanned from its offset
constexpr int kScanTile = 2048, kScanThreads = 512;

__device__ uint64_t block_exclusive_u64(uint64_t v, uint64_t* total) {
  __shared__ uint64_t ws[kScanThreads / kWarp];
  const unsigned lane = lane_id(), wid = threadIdx.x / kWarp;
  uint64_t x = v;
  for (int o = 1; o < kWarp; o <<= 1) {
    const uint64_t y = __shfl_up_sync(kFull, x, o);
    if (lane >= (unsigned)o) x += y;
  }
  if (lane == kWarp - 1) ws[wid] = x;
  __syncthreads();
  if (wid == 0) {
    uint64_t t = lane < kScanThreads / kWarp ? ws[lane] : 0;
    for (int o = 1; o < kWarp; o <<= 1) {
      const uint64_t y = __shfl_up_sync(kFull, t, o);
      if (lane >= (unsigned)o) t += y;
    }
    if (lane < kScanThreads / kWarp) ws[lane] = t;
  }
  __syncthreads();
  const uint64_t before = (wid ? ws[wid - 1] : 0) + x - v;
  *total = ws[kScanThreads / kWarp - 1];
  __syncthreads();
  return before;
}

__global__ void __launch_bounds__(kScanThreads) k_tile_sums(const unsigned long long* __restrict__ in, uint64_t n, uint64_t* __restrict__ sums) {
  const uint64_t base = (uint64_t)blockIdx.x * kScanTile;
  uint64_t s = 0;
  for (uint64_t i = base + threadIdx.x; i < n && i < base + kScanTile; i += kScanThreads) s += in[i];
  uint64_t total;
  block_exclusive_u64(s, &total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// one block: sums[0..tiles) -> exclusive offsets in place (tiles <= kScanThreads)
__global__ void __launch_bounds__(kScanThreads) k_tile_offsets(uint64_t* __restrict__ sums, uint64_t tiles) {
  const uint64_t v = threadIdx.x < tiles ? sums[threadIdx.x] : 0;
  uint64_t total;
  const uint64_t ex = block_exclusive_u64(v, &total);
  if (threadIdx.x < tiles) sums[threadIdx.x] = ex;
}

// each thread scans 4 consecutive values of the tile
__global__ void __launch_bounds__(kScanThreads) k_tile_apply(const unsigned long long* __restrict__ in, uint64_t n, const uint64_t* __restrict__ offs,
                                                             uint64_t* __restrict__ out) {
  const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * 4;
  uint64_t v[4], s = 0;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    v[i] = base + i < n ? in[base + i] : 0;
    s += v[i];
  }
  uint64_t total;
  uint64_t run = block_exclusive_u64(s, &total) + offs[blockIdx.x];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    if (base + i < n) out[base + i] = run;
    run += v[i];
  }
  if (base < n && base + 4 >= n) out[n] = run;
}

void scan_chunk(const unsigned long long* in, uint64_t n, uint64_t* out, uint64_t* sums, cudaStream_t st) {
  const uint64_t tiles = (n + kScanTile - 1) / kScanTile;  // n <= 2^20: at most 512 tiles
  k_tile_sums<<<(unsigned)tiles, kScanThreads, 0, st>>>(in, n, sums);
  k_tile_offsets<<<1, kScanThreads, 0, st>>>(sums, tiles);
  k_tile_apply<<<(unsigned)tiles, kScanThreads, 0, st>>>(in, n, sums, out);
  TK(cudaGetLastError());
}

struct PackedBin {
  uint64_t first;    // position of its first source in the order
  uint64_t sources;  // consecutive sources from there
  uint64_t size;     // row entries of its view (ViewBin::total_size)
};

}  // namespace

extern "C" {

int vsgm_features_1hop(int device, uint64_t V, const uint64_t* row_ptrs, const uint32_t* cols, uint64_t* out_row_ptrs, uint32_t* out_cols) {
  if (!row_ptrs || !out_row_ptrs || (!cols && V && row_ptrs[V]) || !out_cols || V == 0 || V >= 0xffffffffull) {
    vsgm::set_host_error("vsgm_features_1hop: bad arguments");
    return VSGM_EINVAL;
  }
  return tool_call(device, [&] {
    const uint64_t E = row_ptrs[V];
    Stream st;
    DevBufs b;
    uint64_t* d_rp = b.take<uint64_t>(V + 1);
    uint32_t* d_ci = b.take<uint32_t>(E);
    uint64_t* d_orp = b.take<uint64_t>(V + 1);
    uint32_t* d_oci = b.take<uint32_t>(E + V);
    TK(cudaMemcpyAsync(d_rp, row_ptrs, (V + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st.s));
    if (E) TK(cudaMemcpyAsync(d_ci, cols, E * sizeof(uint32_t), cudaMemcpyHostToDevice, st.s));
    k_self_loops<<<grid_for(V * kWarp, 256), 256, 0, st.s>>>(d_rp, d_ci, V, d_orp, d_oci);
    TK(cudaGetLastError());
    TK(cudaMemcpyAsync(out_row_ptrs, d_orp, (V + 1) * sizeof(uint64_t), cudaMemcpyDeviceToHost, st.s));
    TK(cudaMemcpyAsync(out_cols, d_oci, (E + V) * sizeof(uint32_t), cudaMemcpyDeviceToHost, st.s));
    TK(cudaStreamSynchronize(st.s));
  });
}

int vsgm_kmeans(int device, uint64_t V, const uint64_t* row_ptrs, const uint32_t* cols, int K, int max_iter, const int32_t* starts, int n_starts,
                int reorder_centroids, int32_t* assignment, int64_t* cluster_sizes, int32_t* n_clusters) {
  if (!row_ptrs || !cols || !starts || !assignment || !cluster_sizes || !n_clusters || V == 0 || V >= 0x7fffffffull || K < 1 ||
      K > 32 * kMaxClusterWords || max_iter < 0 || n_starts < 1) {
    vsgm::set_host_error("vsgm_kmeans: bad arguments (1 <= K <= 128, at least one start)");
    return VSGM_EINVAL;
  }
  for (int p = 0; p < n_starts; p++)
    if (starts[p] < 0 || starts[p] >= K) {
      vsgm::set_host_error("vsgm_kmeans: every start must be a cluster id in [0, K)");
      return VSGM_EINVAL;
    }
  return tool_call(device, [&] {
    const uint64_t E = row_ptrs[V];
    Stream st;
    DevBufs b;
    uint64_t* d_rp = b.take<uint64_t>(V + 1);
    uint32_t* d_ci = b.take<uint32_t>(E);
    double* d_w = b.take<double>(V);
    double* d_cen = b.take<double>(V * (uint64_t)K);
    double* d_sqr = b.take<double>(K);
    int32_t* d_assign = b.take<int32_t>(V);
    int32_t* d_starts = b.take<int32_t>(n_starts);
    unsigned long long* d_cnt = b.take<unsigned long long>(2 * K + 1);  // sizes[K], non-zeros[K], asymmetric entries
    unsigned long long* h = nullptr;
    TK(cudaMallocHost(&h, (2 * K + 1) * sizeof(unsigned long long)));
    struct Pinned {
      void* p;
      ~Pinned() { cudaFreeHost(p); }
    } pin{h};
    TK(cudaMemcpyAsync(d_rp, row_ptrs, (V + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st.s));
    if (E) TK(cudaMemcpyAsync(d_ci, cols, E * sizeof(uint32_t), cudaMemcpyHostToDevice, st.s));
    TK(cudaMemcpyAsync(d_starts, starts, n_starts * sizeof(int32_t), cudaMemcpyHostToDevice, st.s));
    TK(cudaMemsetAsync(d_cnt, 0, (2 * K + 1) * sizeof(unsigned long long), st.s));
    const unsigned gw = grid_for(V * kWarp, 256), gt = grid_for(V, 256);
    k_asymmetric<<<gw, 256, 0, st.s>>>(d_rp, d_ci, V, d_cnt + 2 * K);
    k_row_weights<<<gt, 256, 0, st.s>>>(d_rp, V, d_w);
    k_random_init<<<gt, 256, 0, st.s>>>(V, d_starts, n_starts, K, d_assign);
    TK(cudaGetLastError());
    TK(cudaMemcpyAsync(h + 2 * K, d_cnt + 2 * K, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st.s));
    TK(cudaStreamSynchronize(st.s));
    if (h[2 * K]) throw ToolError{VSGM_EINVAL, "vsgm_kmeans: the graph is not undirected (" + std::to_string(h[2 * K]) + " entries without their reverse)"};
    // UpdateAllCentroids after the initial assignment, then max_iter rounds of
    // UpdateAllAssignments + UpdateAllCentroids (kmeans.cc:398-441)
    for (int it = 0; it <= max_iter; it++) {
      if (it > 0) k_assign<<<gw, 256, 0, st.s>>>(d_rp, d_ci, V, d_w, d_cen, d_sqr, K, d_assign);
      TK(cudaMemsetAsync(d_cnt, 0, K * sizeof(unsigned long long), st.s));
      k_cluster_sizes<<<gt, 256, 0, st.s>>>(d_assign, V, d_cnt);
      k_centroids<<<gw, 256, 0, st.s>>>(d_rp, d_ci, V, d_assign, d_w, d_cnt, K, d_cen);
      if (it < max_iter) k_sqr_sums<<<(unsigned)((K + 7) / 8), 256, 0, st.s>>>(d_cen, V, K, d_sqr);
      TK(cudaGetLastError());
    }
    const int T = std::max(1, reorder_centroids ? std::min(K, n_starts) : 0);
    if (reorder_centroids) {
      TK(cudaMemsetAsync(d_cnt + K, 0, K * sizeof(unsigned long long), st.s));
      k_nonzeros<<<grid_for(V * T, 256), 256, 0, st.s>>>(d_cen, V, K, T, d_cnt + K);
      TK(cudaGetLastError());
    }
    TK(cudaMemcpyAsync(h, d_cnt, 2 * K * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st.s));
    TK(cudaMemcpyAsync(assignment, d_assign, V * sizeof(int32_t), cudaMemcpyDeviceToHost, st.s));
    TK(cudaStreamSynchronize(st.s));
    // cluster renumbering on the host, as the reference does it: the -rc order
    // (centroids by non-zero entries, counted for the first min(K, threads) only,
    // std::sort descending), then RemoveEmptyClusters (kmeans.cc:491-510)
    std::vector<unsigned> old2new(K);
    std::iota(old2new.begin(), old2new.end(), 0u);
    if (reorder_centroids) {
      std::vector<unsigned> nonzero(K, 0), new2old(K);
      for (int c = 0; c < T; c++) nonzero[c] = (unsigned)h[K + c];
      std::iota(new2old.begin(), new2old.end(), 0u);
      std::sort(new2old.begin(), new2old.end(), [&](auto a, auto b) { return nonzero[a] > nonzero[b]; });
      for (int i = 0; i < K; i++) old2new[new2old[i]] = (unsigned)i;
    }
    std::vector<int64_t> size(K, 0);
    for (int k = 0; k < K; k++) size[old2new[k]] = (int64_t)h[k];
    std::vector<int32_t> dense(K, -1);
    int n = 0;
    for (int k = 0; k < K; k++)
      if (size[k]) {
        dense[k] = n;
        cluster_sizes[n++] = size[k];
      }
    for (uint64_t v = 0; v < V; v++) assignment[v] = dense[old2new[assignment[v]]];
    *n_clusters = n;
  });
}

int vsgm_view_packing(int device, uint64_t V, const uint64_t* row_ptrs, const uint32_t* cols, const uint32_t* order, const uint64_t* seq_offsets,
                      int n_seqs, int hop, uint64_t max_bin_size, int32_t* bin_of_vertex, int32_t* n_bins, uint64_t* bin_sizes, uint64_t sizes_cap) {
  if (!row_ptrs || !order || !seq_offsets || !bin_of_vertex || !n_bins || V == 0 || V >= 0xffffffffull || n_seqs < 1 || hop < 1 || hop > 3 ||
      seq_offsets[0] != 0 || seq_offsets[n_seqs] != V) {
    vsgm::set_host_error("vsgm_view_packing: bad arguments (hop 1..3; sequences must cover the V positions of the order)");
    return VSGM_EINVAL;
  }
  for (int q = 0; q < n_seqs; q++)
    if (seq_offsets[q] > seq_offsets[q + 1]) {
      vsgm::set_host_error("vsgm_view_packing: sequence offsets must not decrease");
      return VSGM_EINVAL;
    }
  {
    std::vector<uint8_t> seen(V, 0);  // the order must be a permutation of the vertices
    for (uint64_t i = 0; i < V; i++) {
      if (order[i] >= V || seen[order[i]]) {
        vsgm::set_host_error("vsgm_view_packing: the order must list every vertex exactly once");
        return VSGM_EINVAL;
      }
      seen[order[i]] = 1;
    }
  }
  return tool_call(device, [&] {
    const uint64_t E = row_ptrs[V];
    const uint64_t kMaxChunk = 1ull << 20, kFirstChunk = 4096;
    const uint64_t Lmax = std::min<uint64_t>(kMaxChunk, V);
    Stream st;
    DevBufs b;
    uint64_t* d_rp = b.take<uint64_t>(V + 1);
    uint32_t* d_ci = b.take<uint32_t>(E);
    uint32_t* d_order = b.take<uint32_t>(V);
    unsigned long long* lab1 = b.take<unsigned long long>(V);
    unsigned long long* lab2 = b.take<unsigned long long>(V);
    uint32_t* added = b.take<uint32_t>(V);
    uint32_t* visited = b.take<uint32_t>(V);
    uint32_t* T1 = b.take<uint32_t>(V);
    uint32_t* T2 = b.take<uint32_t>(V);
    unsigned long long* contrib = b.take<unsigned long long>(Lmax);
    uint64_t* prefix = b.take<uint64_t>(Lmax + 1);
    uint64_t* tmp = b.take<uint64_t>(kScanThreads);
    unsigned long long* ctl = b.take<unsigned long long>(4);  // nT1, nT2, boundary, size taken
    unsigned long long* h = nullptr;
    TK(cudaMallocHost(&h, 2 * sizeof(unsigned long long)));
    struct Pinned {
      void* p;
      ~Pinned() { cudaFreeHost(p); }
    } pin{h};
    TK(cudaMemcpyAsync(d_rp, row_ptrs, (V + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st.s));
    if (E) TK(cudaMemcpyAsync(d_ci, cols, E * sizeof(uint32_t), cudaMemcpyHostToDevice, st.s));
    TK(cudaMemcpyAsync(d_order, order, V * sizeof(uint32_t), cudaMemcpyHostToDevice, st.s));
    TK(cudaMemsetAsync(lab1, 0xff, V * sizeof(unsigned long long), st.s));
    TK(cudaMemsetAsync(lab2, 0xff, V * sizeof(unsigned long long), st.s));
    TK(cudaMemsetAsync(added, 0, V * sizeof(uint32_t), st.s));
    TK(cudaMemsetAsync(visited, 0, V * sizeof(uint32_t), st.s));

    std::vector<PackedBin> bins;
    uint32_t pass = 0;
    for (int q = 0; q < n_seqs; q++) {
      // every sequence (a thread of the reference packer) opens its own first bin
      bins.push_back({seq_offsets[q], 0, 0});
      uint64_t a = seq_offsets[q], L = kFirstChunk;
      const uint64_t end = seq_offsets[q + 1];
      while (a < end) {
        PackedBin& bin = bins.back();
        const uint32_t stamp = (uint32_t)bins.size();  // 0 = in no bin
        const uint64_t Lc = std::min({L, Lmax, end - a});
        const uint32_t tag = 0xffffffffu - ++pass;
        TK(cudaMemsetAsync(ctl, 0, 2 * sizeof(unsigned long long), st.s));
        TK(cudaMemsetAsync(contrib, 0, Lc * sizeof(unsigned long long), st.s));
        const uint32_t* ord = d_order + a;
        k_pack_sources<<<grid_for(Lc, 256), 256, 0, st.s>>>(ord, Lc, tag, lab1, T1, ctl);
        if (hop >= 2) k_pack_round1<<<grid_for(Lc * kWarp, 256), 256, 0, st.s>>>(d_rp, d_ci, ord, Lc, tag, lab1, T1, ctl);
        if (hop >= 3) k_pack_round2<<<grid_for(V * kWarp, 256), 256, 0, st.s>>>(d_rp, d_ci, T1, ctl, tag, lab1, lab2, visited, stamp, T2, ctl + 1);
        k_pack_contrib<<<grid_for(V, 256), 256, 0, st.s>>>(d_rp, T1, ctl, T2, ctl + 1, tag, lab1, lab2, added, stamp, contrib);
        TK(cudaGetLastError());
        scan_chunk(contrib, Lc, prefix, tmp, st.s);
        k_set_u64<<<1, 32, 0, st.s>>>(ctl + 2, Lc);
        k_pack_close<<<grid_for(Lc, 256), 256, 0, st.s>>>(prefix, Lc, bin.size, max_bin_size, ctl + 2);
        k_pack_take<<<1, 32, 0, st.s>>>(prefix, Lc, ctl + 2);
        TK(cudaGetLastError());
        TK(cudaMemcpyAsync(h, ctl + 2, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st.s));
        TK(cudaStreamSynchronize(st.s));
        const uint64_t c = h[0];
        if (c == 0 && bin.sources == 0)
          throw ToolError{VSGM_EINVAL, "vsgm_view_packing: the view of source " + std::to_string(order[a]) + " alone exceeds the bin size " +
                                           std::to_string(max_bin_size) + " (the reference packer loses such a source)"};
        if (c > 0) {
          k_pack_commit<<<grid_for(V, 256), 256, 0, st.s>>>(T1, ctl, T2, ctl + 1, tag, lab1, lab2, c, stamp, added, visited);
          TK(cudaGetLastError());
          bin.sources += c;
          bin.size += h[1];
          a += c;
        }
        if (c < Lc) {  // the source at a does not fit: the bin is closed, a new one opens there
          bins.push_back({a, 0, 0});
          L = kFirstChunk;
        } else {
          L = std::min(2 * L, kMaxChunk);
        }
      }
    }
    TK(cudaStreamSynchronize(st.s));
    // the next-fit merge of the packed bins by size (view_packing.cc:247-265),
    // with the reference's own sort of (bin id, size) pairs by size
    std::vector<std::pair<int, size_t>> id_size;
    for (size_t i = 0; i < bins.size(); i++) id_size.push_back({(int)i, (size_t)bins[i].size});
    std::sort(id_size.begin(), id_size.end(), [](const auto& x, const auto& y) { return x.second < y.second; });
    std::vector<int> group_of(bins.size(), 0);
    std::vector<uint64_t> group_size(bins.size() + 1, 0);
    int merged = 0;
    size_t old_size = 0;
    for (const auto& [id, sz] : id_size) {
      if (old_size + sz > max_bin_size) {
        merged++;
        old_size = sz;
      } else {
        old_size += sz;
      }
      group_of[id] = merged;
      group_size[merged] += sz;
    }
    merged++;
    for (size_t i = 0; i < bins.size(); i++)
      for (uint64_t p = bins[i].first; p < bins[i].first + bins[i].sources; p++) bin_of_vertex[order[p]] = group_of[i];
    *n_bins = merged;
    if (bin_sizes)
      for (int i = 0; i < merged && (uint64_t)i < sizes_cap; i++) bin_sizes[i] = group_size[i];
  });
}

}  // extern "C"
