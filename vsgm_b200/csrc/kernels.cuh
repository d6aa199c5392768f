// Device kernels of the enumeration engine (sm_100a).
//
// Partial matches live in HBM as a "frame": SoA columns of matched data-vertex
// ids (one u32 column per materialised pattern vertex) plus, per computed but
// unmaterialised pattern vertex u, a sorted candidate set per path given as
// (address u64, length u32) (the reference keeps an index into a per-parent
// offsets array instead, src/executor/im_data.h:7-90).  A set may point into the
// view's adjacency array: a candidate set that is a slice of one adjacency list,
// or a slice of an earlier set, is never copied; order conditions only narrow
// the slice, and a set is copied only when a NON_EQUAL value actually occurs in
// it.
//
// All kernels are integer-only.  Intersections are warp-per-path: the warp
// restricts every backward neighbour's adjacency list to the value window the
// order conditions allow, takes the shortest restricted list as the pivot, and
// its lanes walk the pivot while galloping forward through the other lists
// (each lane's candidates increase, so every search resumes where the lane's
// previous one ended).  The reference walks the whole pivot list and
// binary-searches every other list from scratch for every element
// (src/gpu/gpu_utils_gpsm_bin_search.h:14-130); the set produced is identical.
#pragma once

#include <cooperative_groups.h>
#include <cstdint>

#include "vsgm_plan.h"

namespace vsgm {
namespace dev {

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;

struct Frame {
  uint64_t P;                    // number of partial matches
  uint32_t* col[VSGM_MAX_QV];    // materialised columns
  uint64_t* cset[VSGM_MAX_QV];   // candidate-set address per path
  uint32_t* clen[VSGM_MAX_QV];   // candidate-set length per path
};

__device__ __forceinline__ const uint32_t* set_of(const Frame& f, int u, uint64_t p) { return (const uint32_t*)__ldg(f.cset[u] + p); }

// Everything a kernel needs about one op, small enough to pass by value.
// Warp kernels load the path's materialised values once (lane i holds the value
// of pattern vertex m[i]) and read them by shuffle: bs[] and cs[] are lane slots.
struct OpDesc {
  uint8_t u;                    // pattern vertex of the op
  uint8_t nb;                   // backward neighbours (intersection inputs)
  uint8_t b[VSGM_MAX_QV];
  uint8_t bs[VSGM_MAX_QV];      // lane slot of b[j]
  uint8_t nc;                   // conditions: candidate cop[i] value(cv[i])
  uint8_t cop[VSGM_MAX_QV];
  uint8_t cv[VSGM_MAX_QV];
  uint8_t cs[VSGM_MAX_QV];      // lane slot of cv[i]
  uint8_t nm;                   // materialised vertices whose columns are read
  uint8_t m[VSGM_MAX_QV];
  int8_t other;                 // COMPUTE_COUNT: computed vertex to count against (-1: none)
  uint8_t other_op;             // relation candidate(u) OP candidate(other)
  uint16_t merge_ratio;         // intersect by merging when list lengths are within this ratio (0: always gallop)
  uint8_t lane_merge;           // counting kernels: lane-partitioned instead of windowed merge
};

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

// first position in a[lo, hi) with a[pos] >= x (hi if none), probing forward from lo
__device__ __forceinline__ uint64_t gallop(const uint32_t* __restrict__ a, uint64_t lo, uint64_t hi, uint32_t x) {
  if (lo >= hi || __ldg(a + lo) >= x) return lo;
  uint64_t step = 1;
  while (lo + step < hi && __ldg(a + lo + step) < x) {
    lo += step;
    step <<= 1;
  }
  uint64_t l = lo + 1, r = (lo + step < hi) ? lo + step : hi;
  while (l < r) {
    uint64_t mid = (l + r) >> 1;
    if (__ldg(a + mid) < x)
      l = mid + 1;
    else
      r = mid;
  }
  return l;
}

__device__ __forceinline__ uint64_t lower_bound(const uint32_t* __restrict__ a, uint64_t lo, uint64_t hi, uint64_t x) {
  while (lo < hi) {
    uint64_t mid = (lo + hi) >> 1;
    if ((uint64_t)__ldg(a + mid) < x)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// Per-path condition state: candidates must lie in [lo, hi) and differ from ne[].
// Lower bound by the whole warp: every round the 32 lanes probe 32 evenly spaced
// positions of [lo, hi), so a range of n shrinks to n/32 per round (4 rounds of
// independent loads for 10^6 elements instead of 20 dependent ones).  All lanes
// must call it with the same arguments; all get the same result.
__device__ __forceinline__ uint64_t warp_lower_bound(const uint32_t* __restrict__ a, uint64_t lo, uint64_t hi, uint64_t x) {
  const unsigned lane = lane_id();
  while (hi - lo > kWarp) {
    const uint64_t step = (hi - lo + kWarp - 1) / kWarp;
    const uint64_t p = lo + lane * step;
    const unsigned below = __ballot_sync(kFull, p < hi && (uint64_t)__ldg(a + p) < x);
    const unsigned cnt = __popc(below);  // a prefix of the lanes: the array is sorted
    if (cnt == 0) return lo;
    const uint64_t nhi = lo + cnt * step;
    lo = lo + (cnt - 1) * step + 1;
    if (nhi < hi) hi = nhi;
  }
  const uint64_t p = lo + lane;
  return lo + __popc(__ballot_sync(kFull, p < hi && (uint64_t)__ldg(a + p) < x));
}

struct Window {
  uint64_t lo, hi;
  uint32_t ne[VSGM_MAX_QV];
  int nne;
};

__device__ __forceinline__ void window_add(Window* w, uint8_t op, uint32_t v, int i) {
  if (op == VSGM_LARGER_THAN) {
    if ((uint64_t)v + 1 > w->lo) w->lo = (uint64_t)v + 1;
  } else if (op == VSGM_LESS_THAN) {
    if ((uint64_t)v < w->hi) w->hi = v;
  } else if (op == VSGM_NON_EQUAL) {
    w->ne[i] = v;  // slot i; unused slots keep a value that never matches
  }
}

// warp version: `mine` is this lane's gathered value (see gather_lane)
__device__ __forceinline__ void make_window(const OpDesc& d, uint32_t mine, Window* w) {
  w->lo = 0;
  w->hi = 0x100000000ull;
  w->nne = d.nc;
#pragma unroll
  for (int i = 0; i < VSGM_MAX_QV; i++) {
    uint32_t v = __shfl_sync(kFull, mine, d.cs[i]);
    w->ne[i] = 0xffffffffu;
    if (i < d.nc) window_add(w, d.cop[i], v, i);
  }
}

// thread version: values read straight from the frame columns
__device__ __forceinline__ void make_window_thread(const OpDesc& d, const Frame& f, uint64_t p, Window* w) {
  w->lo = 0;
  w->hi = 0x100000000ull;
  w->nne = d.nc;
#pragma unroll
  for (int i = 0; i < VSGM_MAX_QV; i++) {
    w->ne[i] = 0xffffffffu;
    if (i < d.nc) window_add(w, d.cop[i], __ldg(f.col[d.cv[i]] + p), i);
  }
}

// NON_EQUAL slots: a candidate can never equal 0xffffffff (ids are < V < 2^32 - 1)
__device__ __forceinline__ bool ne_ok(const Window& w, uint32_t c) {
  bool ok = true;
#pragma unroll
  for (int i = 0; i < VSGM_MAX_QV; i++) ok &= (c != w.ne[i]);
  return ok;
}

// Lane i < nm loads the path's value of pattern vertex m[i].
__device__ __forceinline__ uint32_t gather_lane(const Frame& f, const OpDesc& d, uint64_t p) {
  const unsigned lane = lane_id();
  return lane < d.nm ? __ldg(f.col[d.m[lane]] + p) : 0u;
}

// Restricted ranges of every backward list; pivot = shortest restricted range.
// Lane j < nb computes list j's range; results are broadcast.
struct Lists {
  uint64_t s[VSGM_MAX_QV], e[VSGM_MAX_QV];
  int pivot;
  uint64_t ps, pe;    // the pivot's range
  uint64_t full_min;  // least unrestricted degree (for the algorithmic-byte count)
};

__device__ __forceinline__ void restrict_lists(const OpDesc& d, uint32_t mine, const Window& w, const uint64_t* __restrict__ rp,
                                               const uint32_t* __restrict__ ci, Lists* L) {
  const unsigned lane = lane_id();
  uint64_t s = 0, e = 0, deg = ~0ull;
  const uint32_t v = __shfl_sync(kFull, mine, d.bs[lane < d.nb ? lane : 0]);
  if (lane < d.nb) {
    uint64_t a = __ldg(rp + v), z = __ldg(rp + v + 1);
    deg = z - a;
    s = (w.lo > 0) ? lower_bound(ci, a, z, w.lo) : a;
    e = (w.hi <= 0xffffffffull) ? lower_bound(ci, s, z, w.hi) : z;
    if (e < s) e = s;
  }
  uint64_t best = ~0ull;
  int piv = 0;
  L->full_min = ~0ull;
#pragma unroll
  for (int i = 0; i < VSGM_MAX_QV; i++) {
    uint64_t si = __shfl_sync(kFull, s, i), ei = __shfl_sync(kFull, e, i), di = __shfl_sync(kFull, deg, i);
    L->s[i] = si;
    L->e[i] = ei;
    if (i < d.nb) {
      if (ei - si < best) {
        best = ei - si;
        piv = i;
      }
      if (di < L->full_min) L->full_min = di;
    }
  }
  L->pivot = piv;
  L->ps = L->pe = 0;
#pragma unroll
  for (int i = 0; i < VSGM_MAX_QV; i++)
    if (i == piv) {
      L->ps = L->s[i];
      L->pe = L->e[i];
    }
}

// ---------------------------------------------------------------------------
// sizing: restricted pivot length per path (upper bound of the candidate set)
// ---------------------------------------------------------------------------
__global__ void k_compute_size(Frame f, OpDesc d, const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, uint64_t* __restrict__ ub) {
  const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / kWarp;
  for (uint64_t p = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; p < f.P; p += warps) {
    const uint32_t mine = gather_lane(f, d, p);
    Window w;
    make_window(d, mine, &w);
    Lists L;
    restrict_lists(d, mine, w, rp, ci, &L);
    if (lane_id() == 0) ub[p] = L.pe - L.ps;
  }
}

// ---------------------------------------------------------------------------
// narrow: apply d's conditions to one sorted set per path without copying.
// kFromAdj: the set is the adjacency list of backward neighbour b[0] (COMPUTE
// with one backward neighbour); otherwise the frame's candidates of d.u
// (FILTER_COMPUTE, MATERIALIZE with conditions).  Order conditions cut the
// slice; a NON_EQUAL value found inside it marks the path for copying
// (copy_ub[p] = slice length, else 0).  *total accumulates the exact survivors.
// ---------------------------------------------------------------------------
template <bool kFromAdj>
__global__ void k_narrow(Frame f, OpDesc d, const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, uint64_t* __restrict__ out_set,
                         uint32_t* __restrict__ out_len, uint64_t* __restrict__ copy_ub, unsigned long long* __restrict__ total) {
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
  unsigned long long mine = 0;
  for (uint64_t p = tid; p < f.P; p += nthreads) {
    Window w;
    make_window_thread(d, f, p, &w);
    const uint32_t* base;
    uint64_t n;
    if (kFromAdj) {
      const uint32_t v = __ldg(f.col[d.b[0]] + p);
      const uint64_t a = __ldg(rp + v);
      base = ci + a;
      n = __ldg(rp + v + 1) - a;
    } else {
      base = set_of(f, d.u, p);
      n = __ldg(f.clen[d.u] + p);
    }
    uint64_t s = (w.lo > 0) ? lower_bound(base, 0, n, w.lo) : 0;
    uint64_t e = (w.hi <= 0xffffffffull) ? lower_bound(base, s, n, w.hi) : n;
    if (e < s) e = s;
    uint32_t hits = 0;
#pragma unroll
    for (int i = 0; i < VSGM_MAX_QV; i++) {
      if (w.ne[i] == 0xffffffffu || e == s) continue;
      uint64_t q = lower_bound(base, s, e, w.ne[i]);
      hits += (q < e && __ldg(base + q) == w.ne[i]) ? 1u : 0u;
    }
    out_set[p] = (uint64_t)(base + s);
    out_len[p] = (uint32_t)(e - s);
    copy_ub[p] = hits ? (e - s) : 0;
    mine += (e - s) - hits;
  }
  for (int o = 16; o > 0; o >>= 1) mine += __shfl_down_sync(kFull, mine, o);
  if (lane_id() == 0 && mine) atomicAdd(total, mine);
}

// copy the narrowed sets of the marked paths (off[p+1] > off[p]) without the
// NON_EQUAL values, into pool + off[p]; sets and lengths are updated in place
__global__ void k_copy_marked(Frame f, OpDesc d, const uint64_t* __restrict__ off, uint32_t* __restrict__ pool, uint64_t* __restrict__ set,
                              uint32_t* __restrict__ len) {
  const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / kWarp;
  const unsigned lane = lane_id();
  for (uint64_t p = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; p < f.P; p += warps) {
    const uint64_t o = off[p];
    if (off[p + 1] == o) continue;
    const uint32_t mine = gather_lane(f, d, p);
    Window w;
    make_window(d, mine, &w);
    const uint32_t* in = (const uint32_t*)set[p];
    const uint32_t n = len[p];
    uint32_t* out = pool + o;
    uint32_t written = 0;
    for (uint32_t base = 0; base < n; base += kWarp) {
      const uint32_t k = base + lane;
      uint32_t c = 0;
      bool ok = false;
      if (k < n) {
        c = __ldg(in + k);
        ok = ne_ok(w, c);
      }
      unsigned mask = __ballot_sync(kFull, ok);
      if (ok) out[written + __popc(mask & ((1u << lane) - 1))] = c;
      written += __popc(mask);
    }
    __syncwarp();
    if (lane == 0) {
      set[p] = (uint64_t)out;
      len[p] = written;
    }
  }
}

// ---------------------------------------------------------------------------
// Warp intersection of the backward lists of one path.  emit(ok, c) is called by
// every lane once per step; the lanes with ok hold candidates, in increasing
// order across lanes and steps.
//  - merge: when the second-shortest restricted list is at most merge_ratio
//    times the shortest, both are streamed 32 at a time (coalesced) and each lane
//    finds its element of the shortest list in the other's window by a
//    register binary search over shuffles;
//  - gallop: otherwise lanes walk the shortest list with stride 32 and gallop
//    forward in the longer lists.
// Any remaining lists (three or more backward neighbours) are galloped.
// ---------------------------------------------------------------------------
// kCount: the caller only counts, so emit may be called by single lanes at any
// time (no ballot inside); long similar-length lists then use the lane-partitioned
// merge: the shorter list is cut into 32 equal chunks, each lane finds its start in
// the other list by binary search and merges its chunk sequentially (32
// independent streams per warp instead of one latency-bound window step).
template <int NB, bool kCount = false, typename Emit>
__device__ __forceinline__ void intersect_warp(const Window& w, const Lists& L, const uint32_t* __restrict__ ci, uint32_t merge_ratio, Emit&& emit,
                                               bool lane_merge = false) {
  const unsigned lane = lane_id();
  uint64_t pos[NB];
#pragma unroll
  for (int j = 0; j < NB; j++) pos[j] = L.s[j];
  int jb = -1;
  uint64_t bs = 0, be = 0, blen = ~0ull;
#pragma unroll
  for (int j = 0; j < NB; j++)
    if (j != L.pivot && L.e[j] - L.s[j] < blen) {
      blen = L.e[j] - L.s[j];
      bs = L.s[j];
      be = L.e[j];
      jb = j;
    }
  const uint64_t alen = L.pe - L.ps;
  if (kCount && lane_merge && NB >= 2 && alen >= 256 && blen <= (uint64_t)merge_ratio * alen) {
    const uint64_t chunk = (alen + kWarp - 1) / kWarp;
    uint64_t i = L.ps + lane * chunk;
    const uint64_t i1 = (i + chunk < L.pe) ? i + chunk : L.pe;
    if (i < i1) {
      uint32_t x = __ldg(ci + i);
      uint64_t j = lower_bound(ci, bs, be, x);
      while (i < i1 && j < be) {
        const uint32_t y = __ldg(ci + j);
        if (x < y) {
          if (++i < i1) x = __ldg(ci + i);
        } else if (y < x) {
          j++;
        } else {
          bool ok = ne_ok(w, x);
#pragma unroll
          for (int q = 0; q < NB; q++) {
            if (q == L.pivot || q == jb || !ok) continue;
            uint64_t r = gallop(ci, pos[q], L.e[q], x);
            pos[q] = r;
            ok = (r < L.e[q]) && (__ldg(ci + r) == x);
          }
          if (ok) emit(true, x);
          j++;
          if (++i < i1) x = __ldg(ci + i);
        }
      }
    }
    return;
  }
  if (NB >= 2 && alen >= 64 && blen <= (uint64_t)merge_ratio * alen) {
    uint64_t ia = L.ps, ib = bs;
    while (ia < L.pe && ib < be) {
      const uint32_t nA = (uint32_t)(L.pe - ia < (uint64_t)kWarp ? L.pe - ia : (uint64_t)kWarp);
      const uint32_t nB = (uint32_t)(be - ib < (uint64_t)kWarp ? be - ib : (uint64_t)kWarp);
      const uint32_t x = lane < nA ? __ldg(ci + ia + lane) : 0xffffffffu;
      const uint32_t y = lane < nB ? __ldg(ci + ib + lane) : 0xffffffffu;
      const uint32_t mA = __shfl_sync(kFull, x, nA - 1), mB = __shfl_sync(kFull, y, nB - 1);
      const uint32_t m = mA < mB ? mA : mB;
      int q = 0;
#pragma unroll
      for (int step = 16; step >= 1; step >>= 1) {
        const uint32_t yy = __shfl_sync(kFull, y, q + step - 1);
        if (yy < x) q += step;
      }
      const uint32_t yq = __shfl_sync(kFull, y, q);
      const bool in_a = lane < nA && x <= m;
      bool ok = in_a && yq == x && ne_ok(w, x);
#pragma unroll
      for (int j = 0; j < NB; j++) {
        if (j == L.pivot || j == jb || !ok) continue;
        uint64_t r = gallop(ci, pos[j], L.e[j], x);
        pos[j] = r;
        ok = (r < L.e[j]) && (__ldg(ci + r) == x);
      }
      emit(ok, x);
      ia += __popc(__ballot_sync(kFull, in_a));
      ib += __popc(__ballot_sync(kFull, lane < nB && y <= m));
    }
    return;
  }
  for (uint64_t base = L.ps; base < L.pe; base += kWarp) {
    const uint64_t k = base + lane;
    bool ok = false;
    uint32_t c = 0xffffffffu;
    if (k < L.pe) {
      c = __ldg(ci + k);
      ok = ne_ok(w, c);
#pragma unroll
      for (int j = 0; j < NB; j++) {
        if (j == L.pivot || !ok) continue;
        uint64_t r = gallop(ci, pos[j], L.e[j], c);
        pos[j] = r;
        ok = (r < L.e[j]) && (__ldg(ci + r) == c);
      }
    }
    emit(ok, c);
  }
}

// ---------------------------------------------------------------------------
// COMPUTE: write the sorted candidate set of every path at pool[off[p]...]
// ---------------------------------------------------------------------------
template <int NB>
__global__ void k_compute_write(Frame f, OpDesc d, const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, const uint64_t* __restrict__ off,
                                uint32_t* __restrict__ pool, uint64_t* __restrict__ set, uint32_t* __restrict__ len) {
  const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / kWarp;
  const unsigned lane = lane_id();
  for (uint64_t p = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; p < f.P; p += warps) {
    const uint32_t mine = gather_lane(f, d, p);
    Window w;
    make_window(d, mine, &w);
    Lists L;
    restrict_lists(d, mine, w, rp, ci, &L);
    uint32_t* out = pool + off[p];
    uint32_t written = 0;
    intersect_warp<NB>(w, L, ci, d.merge_ratio, [&](bool ok, uint32_t c) {
      unsigned mask = __ballot_sync(kFull, ok);
      if (ok) out[written + __popc(mask & ((1u << lane) - 1))] = c;
      written += __popc(mask);
    });
    if (lane == 0) {
      set[p] = (uint64_t)out;
      len[p] = written;
    }
  }
}

// ---------------------------------------------------------------------------
// COMPUTE_PATH_COUNT: the size of every path's candidate set, without the set
// (src/executor/ops/compute_path_count.h: IntersectCount with a unit functor)
// ---------------------------------------------------------------------------
template <int NB>
__global__ void k_path_count(Frame f, OpDesc d, const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, uint32_t* __restrict__ len) {
  const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / kWarp;
  const unsigned lane = lane_id();
  for (uint64_t p = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; p < f.P; p += warps) {
    const uint32_t mine = gather_lane(f, d, p);
    Window w;
    make_window(d, mine, &w);
    Lists L;
    restrict_lists(d, mine, w, rp, ci, &L);
    uint32_t n = 0;
    intersect_warp<NB, true>(w, L, ci, d.merge_ratio, [&](bool ok, uint32_t) { n += ok ? 1u : 0u; }, d.lane_merge);
    for (int o = 16; o > 0; o >>= 1) n += __shfl_down_sync(kFull, n, o);
    if (lane == 0) len[p] = n;
  }
}

// ---------------------------------------------------------------------------
// COMPUTE_COUNT: count valid candidates (or, with a computed vertex `other`,
// the candidates of other standing in relation to each) and add to *total.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t count_vs(const uint32_t* __restrict__ a, uint64_t n, uint64_t* cur, uint32_t c, uint8_t op) {
  // elements x of a with  c op x ; *cur is a lower bound of the search position
  uint64_t q = gallop(a, *cur, n, c);
  *cur = q;
  bool eq = q < n && __ldg(a + q) == c;
  if (op == VSGM_LESS_THAN) return n - q - (eq ? 1 : 0);
  if (op == VSGM_LARGER_THAN) return q;
  return n - (eq ? 1 : 0);
}

// pair_mode (same candidate set counted against itself, see the engine's
// set-reuse rule): 0 = plain count, 1 = C(n, 2) per path, 2 = n (n - 1) per path
template <int NB, bool kOther, bool kBytes>
__global__ void __launch_bounds__(256) k_compute_count(Frame f, OpDesc d, const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                                                       unsigned long long* __restrict__ total, unsigned long long* __restrict__ bytes,
                                                       int pair_mode = 0) {
  const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / kWarp;
  const unsigned lane = lane_id();
  unsigned long long acc = 0, acc_bytes = 0;
  for (uint64_t p = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; p < f.P; p += warps) {
    const uint32_t mine = gather_lane(f, d, p);
    Window w;
    make_window(d, mine, &w);
    Lists L;
    restrict_lists(d, mine, w, rp, ci, &L);
    if (kBytes && lane == 0) acc_bytes += 4ull * (L.pe - L.ps) + 16ull * NB + 4ull * d.nm;
    const uint32_t* oset = nullptr;
    uint64_t on = 0, ocur = 0;
    if (kOther) {
      oset = set_of(f, d.other, p);
      on = __ldg(f.clen[d.other] + p);
    }
    if (pair_mode) {
      unsigned long long n = 0;
      intersect_warp<NB, true>(
          w, L, ci, d.merge_ratio, [&](bool ok, uint32_t) { n += ok ? 1ull : 0ull; }, d.lane_merge);
      for (int o = 16; o > 0; o >>= 1) n += __shfl_down_sync(kFull, n, o);
      if (lane == 0 && n > 1) acc += pair_mode == 1 ? n * (n - 1) / 2 : n * (n - 1);
      continue;
    }
    intersect_warp<NB, true>(
        w, L, ci, d.merge_ratio, [&](bool ok, uint32_t c) {
          if (ok) acc += kOther ? count_vs(oset, on, &ocur, c, d.other_op) : 1ull;
        },
        d.lane_merge);
  }
  for (int o = 16; o > 0; o >>= 1) {
    acc += __shfl_down_sync(kFull, acc, o);
    if (kBytes) acc_bytes += __shfl_down_sync(kFull, acc_bytes, o);
  }
  if (lane == 0) {
    if (acc) atomicAdd(total, acc);
    if (kBytes && acc_bytes) atomicAdd(bytes, acc_bytes);
  }
}

// ---------------------------------------------------------------------------
// Fused MATERIALIZE(u) + COMPUTE_COUNT(w) over the parent frame.
//
// The children of one parent share every backward list of w except N(child), so
// the warp intersects the parent-known lists once (restricted by the conditions
// that do not involve u, and by the bound the smallest / largest child puts on
// w) into shared memory.  Then, one child per lane, every child c in the
// parent's candidates of u counts |I ∩ N(c)| under its own condition by probing
// N(c) for the elements of its slice of I; children whose slice is long are
// redone by the whole warp (walk the shorter side, probe the other).  Parents
// whose staged set would not fit fall back to a per-child warp intersection.
// Same result as expanding the children and running COMPUTE_COUNT on them
// (src/executor/ops/materialize.h, src/executor/ops/compute_count.h).
// ---------------------------------------------------------------------------
constexpr int kStageCap = 1536;  // u32 per warp (8 warps: 48 KB of static shared memory per block)
constexpr uint32_t kLaneSlice = 16;  // default: children with longer slices go to the whole-warp pass

struct FusedDesc {
  OpDesc known;        // w's backward lists and conditions that do not involve u (slots into the parent gather)
  uint8_t u;           // materialised vertex (children)
  uint8_t has_cond_u;
  uint8_t cond_u_op;   // condition  candidate(w)  op  c
  int8_t other;        // computed vertex counted against (-1 none)
  uint8_t other_op;
  uint32_t stage_cap;  // <= kStageCap; smaller values force the per-child path
  uint32_t walk_ratio; // a heavy child walks N(c) (probing the stage) unless N(c)'s part is this many times longer
  uint32_t lane_slice; // children whose slice is longer go to the whole-warp pass
  const uint32_t* up;  // per vertex c: offset of the first neighbour > c in N(c) (cond_u_op LARGER_THAN), else null
};

// up[v] = index (within N(v)) of the first neighbour larger than v
__global__ void k_upper_offsets(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, uint64_t V, uint32_t* __restrict__ up) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t a = rp[v];
    up[v] = (uint32_t)(lower_bound(ci, a, rp[v + 1], v + 1) - a);
  }
}

__device__ __forceinline__ uint32_t smem_lower_bound(const uint32_t* a, uint32_t lo, uint32_t hi, uint64_t x) {
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if ((uint64_t)a[mid] < x)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// slice [ia, ib) of the staged set I[0, ni) allowed for child c
__device__ __forceinline__ void child_slice(const FusedDesc& fd, const Window& w, const uint32_t* I, uint32_t ni, uint32_t c, uint32_t* ia,
                                            uint32_t* ib) {
  uint64_t lo = w.lo, hi = w.hi;
  if (fd.has_cond_u) {
    if (fd.cond_u_op == VSGM_LARGER_THAN && (uint64_t)c + 1 > lo) lo = (uint64_t)c + 1;
    if (fd.cond_u_op == VSGM_LESS_THAN && (uint64_t)c < hi) hi = c;
  }
  *ia = (lo > 0) ? smem_lower_bound(I, 0, ni, lo) : 0;
  *ib = (hi <= 0xffffffffull) ? smem_lower_bound(I, *ia, ni, hi) : ni;
}

// kMergeTail: heavy children intersect their slice and their part of N(c) by a
// merge-path split over the 32 lanes (each lane binary-searches its diagonal, then
// merges its share) instead of the walk / gallop of the default instantiation.
template <int NK, bool kOther, bool kMergeTail = false>
__global__ void __launch_bounds__(256, 3) k_mat_count(Frame f, FusedDesc fd, const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                                                   unsigned long long* __restrict__ total, unsigned long long* __restrict__ bytes) {
  __shared__ uint32_t stage[8][kStageCap];
  const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / kWarp;
  const unsigned lane = lane_id();
  uint32_t* I = stage[threadIdx.x / kWarp];
  const OpDesc& d = fd.known;
  const uint32_t excl_child = (fd.has_cond_u && fd.cond_u_op == VSGM_NON_EQUAL) ? 1u : 0u;
  unsigned long long acc = 0, acc_bytes = 0;
  for (uint64_t p = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; p < f.P; p += warps) {
    const uint32_t* cs = set_of(f, fd.u, p);
    const uint32_t nc = __ldg(f.clen[fd.u] + p);
    if (nc == 0) continue;
    const uint32_t mine = gather_lane(f, d, p);
    Window w;
    make_window(d, mine, &w);  // conditions not involving u
    // the children are sorted: an order condition on u bounds what any child can use
    Window ws = w;
    if (fd.has_cond_u && fd.cond_u_op == VSGM_LARGER_THAN) window_add(&ws, VSGM_LARGER_THAN, __ldg(cs), 0);
    if (fd.has_cond_u && fd.cond_u_op == VSGM_LESS_THAN) window_add(&ws, VSGM_LESS_THAN, __ldg(cs + nc - 1), 0);
    Lists L;
    restrict_lists(d, mine, ws, rp, ci, &L);  // the NK parent-known lists
    const uint32_t* oset = nullptr;
    uint32_t on = 0;
    if (kOther) {
      oset = set_of(f, fd.other, p);
      on = __ldg(f.clen[fd.other] + p);
    }
    if ((L.pe - L.ps) <= (uint64_t)fd.stage_cap) {
      // stage I = intersection of the known lists (NON_EQUAL vs parent values applied)
      uint32_t ni = 0;
      if (NK == 1) {
        for (uint64_t base = L.ps; base < L.pe; base += kWarp) {
          const uint64_t k = base + lane;
          uint32_t c = 0;
          bool ok = false;
          if (k < L.pe) {
            c = __ldg(ci + k);
            ok = ne_ok(w, c);
          }
          unsigned mask = __ballot_sync(kFull, ok);
          if (ok) I[ni + __popc(mask & ((1u << lane) - 1))] = c;
          ni += __popc(mask);
        }
      } else {
        intersect_warp<NK>(w, L, ci, d.merge_ratio, [&](bool ok, uint32_t c) {
          unsigned mask = __ballot_sync(kFull, ok);
          if (ok) I[ni + __popc(mask & ((1u << lane) - 1))] = c;
          ni += __popc(mask);
        });
      }
      __syncwarp();
      if (lane == 0) acc_bytes += 4ull * (L.pe - L.ps) + 16ull * NK + 4ull * d.nm;
      if (ni == 0) continue;
      for (uint32_t k0 = 0; k0 < nc; k0 += kWarp) {
        // pass 1, one child per lane; long slices are left for pass 2
        const uint32_t k = k0 + lane;
        bool heavy = false;
        if (k < nc) {
          const uint32_t c = __ldg(cs + k);
          uint32_t ia, ib;
          child_slice(fd, w, I, ni, c, &ia, &ib);
          if (ib - ia > fd.lane_slice) {
            heavy = true;
          } else if (ia < ib) {
            const uint64_t a0 = __ldg(rp + c), z0 = __ldg(rp + c + 1);
            const uint32_t excl = excl_child ? c : 0xffffffffu;
            uint64_t cur = fd.up ? a0 + __ldg(fd.up + c) : a0, ocur = 0;  // the slice lies above c
            acc_bytes += 4ull * (ib - ia) + 16ull;
            for (uint32_t j = ia; j < ib; j++) {
              const uint32_t x = I[j];
              const uint64_t r = gallop(ci, cur, z0, x);
              cur = r;
              if (r < z0 && __ldg(ci + r) == x && x != excl) acc += kOther ? count_vs(oset, on, &ocur, x, fd.other_op) : 1ull;
            }
          }
        }
        // pass 2: the long slices of this group, one child at a time, by the whole warp
        unsigned todo = __ballot_sync(kFull, heavy);
        while (todo) {
          const int src = __ffs(todo) - 1;
          todo &= todo - 1;
          const uint32_t c = __ldg(cs + k0 + src);
          uint32_t ia, ib;
          child_slice(fd, w, I, ni, c, &ia, &ib);
          const uint64_t a0 = __ldg(rp + c), z0 = __ldg(rp + c + 1);
          const uint64_t s2 = warp_lower_bound(ci, fd.up ? a0 + __ldg(fd.up + c) : a0, z0, I[ia]);
          const uint64_t e2 = warp_lower_bound(ci, s2, z0, (uint64_t)I[ib - 1] + 1);
          if (lane == 0) acc_bytes += 4ull * ((uint64_t)(ib - ia) < e2 - s2 ? (uint64_t)(ib - ia) : e2 - s2) + 16ull;
          if (s2 >= e2) continue;
          const uint32_t excl = excl_child ? c : 0xffffffffu;
          uint64_t ocur = 0;
          if (kMergeTail) {
            // A = I[ia, ib) (stage), B = ci[s2, e2); every match is counted by the
            // lane that takes its A element (A goes first on ties)
            const uint64_t na = ib - ia, nb = e2 - s2, tot = na + nb;
            const uint64_t per = (tot + kWarp - 1) / kWarp;
            const uint64_t d0 = (uint64_t)lane * per < tot ? (uint64_t)lane * per : tot;
            const uint64_t d1 = d0 + per < tot ? d0 + per : tot;
            if (d0 < d1) {
              uint64_t lo = d0 > nb ? d0 - nb : 0, hi = d0 < na ? d0 : na;
              while (lo < hi) {
                const uint64_t mid = (lo + hi) >> 1;
                if (I[ia + mid] <= __ldg(ci + s2 + (d0 - 1 - mid)))
                  lo = mid + 1;
                else
                  hi = mid;
              }
              uint64_t i = lo, j = d0 - lo;
              for (uint64_t step = d0; step < d1; step++) {
                if (i < na) {
                  const uint32_t a = I[ia + i];
                  const uint32_t b = j < nb ? __ldg(ci + s2 + j) : 0u;
                  if (j >= nb || a <= b) {
                    if (j < nb && a == b && a != excl) acc += kOther ? count_vs(oset, on, &ocur, a, fd.other_op) : 1ull;
                    i++;
                    continue;
                  }
                }
                j++;
              }
            }
            continue;
          }
          // walk N(c)'s part coalesced, probing the stage, unless it is much longer than the slice
          if ((uint64_t)(ib - ia) * fd.walk_ratio < (e2 - s2)) {
            uint64_t cur = s2;
            for (uint32_t j = ia + lane; j < ib; j += kWarp) {
              const uint32_t x = I[j];
              const uint64_t r = gallop(ci, cur, e2, x);
              cur = r;
              if (r < e2 && __ldg(ci + r) == x && x != excl) acc += kOther ? count_vs(oset, on, &ocur, x, fd.other_op) : 1ull;
            }
          } else {
            uint32_t cur = ia;
            for (uint64_t j = s2 + lane; j < e2; j += kWarp) {
              const uint32_t x = __ldg(ci + j);
              const uint32_t r = smem_lower_bound(I, cur, ib, x);
              cur = r;
              if (r < ib && I[r] == x && x != excl) acc += kOther ? count_vs(oset, on, &ocur, x, fd.other_op) : 1ull;
            }
          }
        }
      }
    } else {
      // too large to stage: per child, intersect the known lists with N(c)
      for (uint32_t k = 0; k < nc; k++) {
        const uint32_t c = __ldg(cs + k);
        Window wc = w;
        if (fd.has_cond_u && fd.cond_u_op == VSGM_NON_EQUAL) {
          // the known conditions leave at least one NON_EQUAL slot free
          bool placed = false;
#pragma unroll
          for (int q = VSGM_MAX_QV - 1; q >= 0; q--)
            if (!placed && wc.ne[q] == 0xffffffffu) {
              wc.ne[q] = c;
              placed = true;
            }
        } else if (fd.has_cond_u) {
          window_add(&wc, fd.cond_u_op, c, 0);
        }
        // lanes < NK: the known lists; lane NK: N(c)
        uint64_t ls = 0, le = 0;
#pragma unroll
        for (int q = 0; q < VSGM_MAX_QV; q++)
          if (q < NK && q == (int)lane) {
            ls = L.s[q];
            le = L.e[q];
          }
        if (lane == NK) {
          ls = __ldg(rp + c);
          le = __ldg(rp + c + 1);
        }
        if (lane <= NK) {
          const uint64_t z = le;
          ls = (wc.lo > 0) ? lower_bound(ci, ls, z, wc.lo) : ls;
          le = (wc.hi <= 0xffffffffull) ? lower_bound(ci, ls, z, wc.hi) : z;
          if (le < ls) le = ls;
        }
        Lists Lc;
        uint64_t best = ~0ull;
        int piv = 0;
#pragma unroll
        for (int q = 0; q < VSGM_MAX_QV; q++) {
          const uint64_t sq = __shfl_sync(kFull, ls, q), eq = __shfl_sync(kFull, le, q);
          Lc.s[q] = sq;
          Lc.e[q] = eq;
          if (q <= NK && eq - sq < best) {
            best = eq - sq;
            piv = q;
          }
        }
        Lc.pivot = piv;
        Lc.ps = Lc.pe = 0;
#pragma unroll
        for (int q = 0; q < VSGM_MAX_QV; q++)
          if (q == piv) {
            Lc.ps = Lc.s[q];
            Lc.pe = Lc.e[q];
          }
        if (lane == 0) acc_bytes += 4ull * (Lc.pe - Lc.ps) + 16ull * (NK + 1);
        uint64_t ocur = 0;
        intersect_warp<NK + 1, true>(
            wc, Lc, ci, d.merge_ratio, [&](bool ok, uint32_t x) {
              if (ok) acc += kOther ? count_vs(oset, on, &ocur, x, fd.other_op) : 1ull;
            },
            d.lane_merge);
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    acc += __shfl_down_sync(kFull, acc, o);
    acc_bytes += __shfl_down_sync(kFull, acc_bytes, o);
  }
  if (lane == 0) {
    if (acc) atomicAdd(total, acc);
    if (bytes && acc_bytes) atomicAdd(bytes, acc_bytes);
  }
}

// ---------------------------------------------------------------------------
// MATERIALIZE: expand every path by its candidates of u (one thread per child;
// the parent is found by binary search over the children offsets)
// ---------------------------------------------------------------------------
struct Expand {
  uint8_t u;
  uint8_t nm;                 // columns copied from the parent
  uint8_t m[VSGM_MAX_QV];
  uint8_t ncu;                // candidate references copied from the parent
  uint8_t cu[VSGM_MAX_QV];
};

// children [c0, c1) of the whole frame; out's pointers are pre-shifted so that
// child c is written at out.*[c]
__global__ void k_expand(Frame in, Expand x, const uint64_t* __restrict__ off, uint64_t c0, uint64_t c1, Frame out) {
  const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t c = c0 + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; c < c1; c += nthreads) {
    // parent = last p with off[p] <= c
    uint64_t lo = 0, hi = in.P;
    while (hi - lo > 1) {
      uint64_t mid = (lo + hi) >> 1;
      if (__ldg(off + mid) <= c)
        lo = mid;
      else
        hi = mid;
    }
    const uint64_t p = lo, r = c - __ldg(off + p);
#pragma unroll
    for (int i = 0; i < VSGM_MAX_QV; i++)
      if (i < x.nm) out.col[x.m[i]][c] = __ldg(in.col[x.m[i]] + p);
    out.col[x.u][c] = __ldg(set_of(in, x.u, p) + r);
#pragma unroll
    for (int i = 0; i < VSGM_MAX_QV; i++)
      if (i < x.ncu) {
        out.cset[x.cu[i]][c] = __ldg(in.cset[x.cu[i]] + p);
        out.clen[x.cu[i]][c] = __ldg(in.clen[x.cu[i]] + p);
      }
  }
}

// ---------------------------------------------------------------------------
// 4-cycle count by wedge aggregation.  Every 4-cycle is counted once, at its
// largest vertex u: for each neighbour v < u and each w in N(v) with w < u,
// L[w] counts the wedges u-v-w; the cycles closed at u are sum C(L[w], 2)
// (pairs of distinct v through the same opposite vertex w).  Work is bounded by
// sum over edges of the smaller degree when ids ascend with degree, instead of
// intersecting the two wedge ends' lists for every wedge (the plan's COMPUTE_COUNT).
// One block per root; each block owns a dense counter array over the ids and a
// list of the ids it touched, used to sum and reset.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long pairs_of_u32(uint32_t c) { return (unsigned long long)c * (c ? c - 1u : 0u) / 2; }
__device__ __forceinline__ unsigned long long pairs_of(uint32_t c) { return pairs_of_u32(c); }

__global__ void __launch_bounds__(256) k_c4_aggregate(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, const uint32_t* __restrict__ roots,
                                                      uint64_t n_roots, uint64_t V, uint32_t* __restrict__ L_all, uint32_t* __restrict__ touched_all,
                                                      unsigned long long* __restrict__ head, unsigned long long* __restrict__ total) {
  __shared__ unsigned long long s_root;
  __shared__ unsigned int s_touched;
  __shared__ unsigned long long s_sum[8];
  uint32_t* L = L_all + (uint64_t)blockIdx.x * V;
  uint32_t* touched = touched_all + (uint64_t)blockIdx.x * V;
  const unsigned lane = lane_id(), warp = threadIdx.x / kWarp, nwarps = blockDim.x / kWarp;
  unsigned long long acc = 0;
  while (true) {
    if (threadIdx.x == 0) {
      s_root = atomicAdd(head, 1ull);
      s_touched = 0;
    }
    __syncthreads();
    const unsigned long long r = s_root;
    if (r >= n_roots) break;
    const uint32_t u = __ldg(roots + r);
    const uint64_t ua = __ldg(rp + u), uz = __ldg(rp + u + 1);
    // wedges: warp per neighbour v < u, lanes over N(v) below u
    for (uint64_t k = ua + warp; k < uz; k += nwarps) {
      const uint32_t v = __ldg(ci + k);
      if (v >= u) break;  // rows are sorted
      const uint64_t va = __ldg(rp + v), vz = __ldg(rp + v + 1);
      for (uint64_t j = va + lane; j < vz; j += kWarp) {
        const uint32_t w = __ldg(ci + j);
        if (w >= u) break;
        if (atomicAdd(L + w, 1u) == 0u) touched[atomicAdd(&s_touched, 1u)] = w;
      }
    }
    __syncthreads();
    const unsigned n = s_touched;
    for (unsigned i = threadIdx.x; i < n; i += blockDim.x) {
      const uint32_t w = touched[i];
      const unsigned long long c = L[w];
      acc += c * (c - 1) / 2;
      L[w] = 0;
    }
    __syncthreads();
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(kFull, acc, o);
  if (lane == 0) s_sum[warp] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (unsigned i = 0; i < nwarps; i++) t += s_sum[i];
    if (t) atomicAdd(total, t);
  }
}

// Light roots of the same count with their counters in a shared-memory hash table
// instead of a dense array over all ids: distinct opposite vertices w are at most
// the root's wedge count, so a table of capacity C holds any root with at most
// 3C/4 wedges (linear probing always ends).  Slots a root used are listed and
// cleared after its sum, so the table starts empty for the next root.
constexpr uint32_t kC4HashWarpCap = 1024;    // per warp: roots with <= 768 wedges
constexpr uint32_t kC4HashBlockCap = 16384;  // per block of 16 warps: roots with <= 12288 wedges
constexpr uint32_t kC4HashWarpMaxW = kC4HashWarpCap / 4 * 3;
constexpr uint32_t kC4HashBlockMaxW = kC4HashBlockCap / 4 * 3;
constexpr int kC4HashWarps = 8;
constexpr size_t kC4HashWarpSmem = (size_t)kC4HashWarps * kC4HashWarpCap * (4 + 4 + 2);
constexpr size_t kC4HashBlockSmem = (size_t)kC4HashBlockCap * (4 + 4 + 2);

__device__ __forceinline__ void c4_hash_add(uint32_t* keys, uint32_t* cnt, uint16_t* used, unsigned* n_used, uint32_t mask, int shift, uint32_t w) {
  uint32_t h = (w * 0x9E3779B1u) >> shift;
  while (true) {
    const uint32_t k = ((volatile uint32_t*)keys)[h];
    if (k == w) break;
    if (k == 0xffffffffu) {
      const uint32_t old = atomicCAS(keys + h, 0xffffffffu, w);
      if (old == 0xffffffffu) {
        used[atomicAdd(n_used, 1u)] = (uint16_t)h;
        break;
      }
      if (old == w) break;
    }
    h = (h + 1) & mask;
  }
  atomicAdd(cnt + h, 1u);
}

// sum C(count, 2) over the listed slots and empty them
__device__ __forceinline__ unsigned long long c4_hash_drain(uint32_t* keys, uint32_t* cnt, const uint16_t* used, unsigned n, unsigned tid, unsigned nthr) {
  unsigned long long acc = 0;
  for (unsigned t = tid; t < n; t += nthr) {
    const uint32_t h = used[t];
    acc += pairs_of_u32(cnt[h]);
    cnt[h] = 0;
    keys[h] = 0xffffffffu;
  }
  return acc;
}

// a warp per root (<= 768 wedges); each lane walks the lower neighbourhoods of
// its own wedge centres v < u
__global__ void __launch_bounds__(kC4HashWarps * 32) k_c4_hash_warp(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                                                                    const uint32_t* __restrict__ up, const uint32_t* __restrict__ roots, uint64_t n,
                                                                    unsigned long long* __restrict__ total) {
  extern __shared__ uint32_t smem[];
  __shared__ unsigned s_used[kC4HashWarps];
  const unsigned lane = lane_id(), wid = threadIdx.x / kWarp;
  uint32_t* keys = smem + (size_t)wid * kC4HashWarpCap;
  uint32_t* cnt = smem + (size_t)kC4HashWarps * kC4HashWarpCap + (size_t)wid * kC4HashWarpCap;
  uint16_t* used = (uint16_t*)(smem + 2 * (size_t)kC4HashWarps * kC4HashWarpCap) + (size_t)wid * kC4HashWarpCap;
  for (uint32_t t = lane; t < kC4HashWarpCap; t += kWarp) {
    keys[t] = 0xffffffffu;
    cnt[t] = 0;
  }
  if (lane == 0) s_used[wid] = 0;
  __syncwarp();
  const int shift = 32 - 10;  // log2(kC4HashWarpCap)
  unsigned long long acc = 0;
  const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / kWarp;
  for (uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; r < n; r += warps) {
    const uint32_t u = __ldg(roots + r);
    const uint64_t ua = __ldg(rp + u), lower = __ldg(up + u);
    for (uint64_t k = lane; k < lower; k += kWarp) {
      const uint32_t v = __ldg(ci + ua + k);
      const uint64_t vz = __ldg(rp + v + 1);
      for (uint64_t j = __ldg(rp + v); j < vz; j++) {
        const uint32_t w = __ldg(ci + j);
        if (w >= u) break;
        c4_hash_add(keys, cnt, used, &s_used[wid], kC4HashWarpCap - 1, shift, w);
      }
    }
    __syncwarp();
    acc += c4_hash_drain(keys, cnt, used, s_used[wid], lane, kWarp);
    __syncwarp();
    if (lane == 0) s_used[wid] = 0;
    __syncwarp();
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(kFull, acc, o);
  if (lane == 0 && acc) atomicAdd(total, acc);
}

// a block per root (<= 12288 wedges): a warp per wedge centre, lanes over its row
__global__ void __launch_bounds__(512, 1) k_c4_hash_block(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, const uint32_t* __restrict__ up,
                                                          const uint32_t* __restrict__ roots, uint64_t n, unsigned long long* __restrict__ head,
                                                          unsigned long long* __restrict__ total) {
  extern __shared__ uint32_t smem[];
  __shared__ unsigned s_used;
  __shared__ unsigned long long s_root;
  __shared__ unsigned long long s_sum[16];
  uint32_t* keys = smem;
  uint32_t* cnt = smem + kC4HashBlockCap;
  uint16_t* used = (uint16_t*)(smem + 2 * kC4HashBlockCap);
  const unsigned lane = lane_id(), wid = threadIdx.x / kWarp, nwarps = blockDim.x / kWarp;
  for (uint32_t t = threadIdx.x; t < kC4HashBlockCap; t += blockDim.x) {
    keys[t] = 0xffffffffu;
    cnt[t] = 0;
  }
  if (threadIdx.x == 0) s_used = 0;
  const int shift = 32 - 14;  // log2(kC4HashBlockCap)
  unsigned long long acc = 0;
  while (true) {
    if (threadIdx.x == 0) s_root = atomicAdd(head, 1ull);
    __syncthreads();
    const unsigned long long r = s_root;
    if (r >= n) break;
    const uint32_t u = __ldg(roots + r);
    const uint64_t ua = __ldg(rp + u), lower = __ldg(up + u);
    for (uint64_t k = wid; k < lower; k += nwarps) {
      const uint32_t v = __ldg(ci + ua + k);
      const uint64_t vz = __ldg(rp + v + 1);
      for (uint64_t base = __ldg(rp + v); base < vz; base += kWarp) {
        const uint64_t j = base + lane;
        const uint32_t w = j < vz ? __ldg(ci + j) : u;
        if (w < u) c4_hash_add(keys, cnt, used, &s_used, kC4HashBlockCap - 1, shift, w);
        if (__any_sync(kFull, w >= u)) break;
      }
    }
    __syncthreads();
    acc += c4_hash_drain(keys, cnt, used, s_used, threadIdx.x, blockDim.x);
    __syncthreads();
    if (threadIdx.x == 0) s_used = 0;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(kFull, acc, o);
  if (lane == 0) s_sum[wid] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (unsigned w = 0; w < nwarps; w++) t += s_sum[w];
    if (t) atomicAdd(total, t);
  }
}

// Heavy roots of the same count.  A root u with many wedges is shared by the whole
// GPU: a group of G such roots keeps G dense counter arrays (one per root, over the
// ids below u) small enough to stay in L2, every warp takes one wedge centre v of
// one root and adds its wedges with fire-and-forget atomics (no return value, so no
// touched list), and a second pass sums C(L[w], 2) over [0, u) and clears the
// counters for the next group.
constexpr int kC4Group = 16;
struct C4Group {
  uint32_t n;                        // roots in the group (<= kC4Group)
  uint32_t root[kC4Group];
  uint32_t lim[kC4Group];            // wedge ends w < lim are counted here (the root itself, or the start of its window)
  uint64_t vbeg[kC4Group + 1];       // prefix of the wedge centres (neighbours below the root) per root
  uint64_t cbase;                    // index of the group's first centre in the centre-degree prefix (balanced kernel)
};



// W[u] += wedges that end at u's lower neighbours: for every edge v-u with v < u,
// the number of neighbours of v below u (u's position in v's sorted row)
__global__ void k_c4_wedge_counts(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, uint64_t V, unsigned long long* __restrict__ W) {
  const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / kWarp;
  const unsigned lane = lane_id();
  for (uint64_t v = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; v < V; v += warps) {
    const uint64_t a = __ldg(rp + v), z = __ldg(rp + v + 1);
    for (uint64_t j = a + lane; j < z; j += kWarp) {
      const uint32_t u = __ldg(ci + j);
      if (u > v && j > a) atomicAdd(W + u, (unsigned long long)(j - a));
    }
  }
}

// light roots by wedge count for the shared-memory hash kernels: wedge-less roots
// dropped, <= warp_max to hash_w, <= block_max to hash_b, the rest stay in light
__global__ void k_c4_split_light(const uint32_t* __restrict__ light, uint64_t n, const unsigned long long* __restrict__ W, unsigned long long warp_max,
                                 unsigned long long block_max, uint32_t* __restrict__ hash_w, uint32_t* __restrict__ hash_b, uint32_t* __restrict__ rest,
                                 unsigned long long* __restrict__ counters) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t u = light[i];
    const unsigned long long w = W[u];
    if (w == 0) continue;
    if (w <= warp_max)
      hash_w[atomicAdd(counters, 1ull)] = u;
    else if (w <= block_max)
      hash_b[atomicAdd(counters + 1, 1ull)] = u;
    else
      rest[atomicAdd(counters + 2, 1ull)] = u;
  }
}

// split roots by wedge count; centres[k] = neighbours of heavy root k below it
// bytes (profiling, may be null): the operator's algorithmic bytes, 8 per wedge (its
// far end read, its counter updated) and 16 per root (row offsets)
__global__ void k_c4_split(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, const uint32_t* __restrict__ roots, uint64_t n,
                           const unsigned long long* __restrict__ W, unsigned long long threshold, uint32_t* __restrict__ heavy,
                           uint64_t* __restrict__ centres, uint32_t* __restrict__ light, unsigned long long* __restrict__ counters,
                           unsigned long long* __restrict__ bytes) {
  unsigned long long b = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t u = roots[i];
    b += 8ull * W[u] + 16;
    if (W[u] >= threshold) {
      const unsigned long long k = atomicAdd(counters, 1ull);
      heavy[k] = u;
      centres[k] = lower_bound(ci, __ldg(rp + u), __ldg(rp + u + 1), u) - __ldg(rp + u);
    } else {
      light[atomicAdd(counters + 1, 1ull)] = u;
    }
  }
  if (bytes) {
    for (int o = 16; o > 0; o >>= 1) b += __shfl_down_sync(kFull, b, o);
    if (lane_id() == 0 && b) atomicAdd(bytes, b);
  }
}

// kPacked: two 16-bit counters per word (w's counter in the low half of word w/2
// when w is even, the high half when odd) - used when every root of the group has
// fewer than 65536 neighbours below it, the bound of any of its counters, so a
// half never carries into the other; stride is in words either way
template <bool kPacked>
__global__ void __launch_bounds__(256) k_c4_group_wedges(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, const C4Group* __restrict__ grp,
                                                         uint32_t* __restrict__ L, uint64_t stride) {
  const C4Group& G = *grp;
  const uint64_t total = G.vbeg[G.n];
  const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / kWarp;
  const unsigned lane = lane_id();
  for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; i < total; i += warps) {
    uint32_t g = 0;
    while (g + 1 < G.n && i >= G.vbeg[g + 1]) g++;
    const uint32_t u = G.root[g], lim = G.lim[g];
    const uint32_t v = __ldg(ci + __ldg(rp + u) + (i - G.vbeg[g]));  // v < u: the row is sorted
    uint32_t* Lg = L + (uint64_t)g * stride;
    const uint64_t z = __ldg(rp + v + 1);
    for (uint64_t base = __ldg(rp + v); base < z; base += kWarp) {
      const uint64_t j = base + lane;
      const uint32_t w = j < z ? __ldg(ci + j) : lim;
      if (w < lim) {
        if (kPacked)
          atomicAdd(Lg + (w >> 1), (w & 1u) ? 0x10000u : 1u);
        else
          atomicAdd(Lg + w, 1u);
      }
      if (__any_sync(kFull, w >= lim)) break;
    }
  }
}

// Row lengths of every group's wedge centres, in group order (centre k of root
// slot i of group g at grp[g].cbase + vbeg[i] + k): the input of the prefix that
// the balanced kernel splits its work by.  One block per group.
__global__ void k_c4_centre_degrees(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, const C4Group* __restrict__ grp,
                                    uint32_t* __restrict__ deg) {
  const C4Group& G = grp[blockIdx.x];
  for (uint32_t i = 0; i < G.n; i++) {
    const uint64_t ua = __ldg(rp + G.root[i]), nc = G.vbeg[i + 1] - G.vbeg[i];
    for (uint64_t k = threadIdx.x; k < nc; k += blockDim.x) {
      const uint32_t v = __ldg(ci + ua + k);
      deg[G.cbase + G.vbeg[i] + k] = (uint32_t)(__ldg(rp + v + 1) - __ldg(rp + v));
    }
  }
}

// k_c4_group_wedges with the work split by adjacency entries instead of by centre:
// P is the exclusive prefix of the centres' row lengths (k_c4_centre_degrees), and
// warp w of the grid takes the group's entries [w*share, (w+1)*share) - one search
// for its first centre, then a walk across centres - so a hub centre's long row is
// shared by many warps and no warp waits on another's tail.  A centre's walk stops
// at the first entry >= lim (rows are sorted); two strides are loaded per step.
template <bool kPacked>
__global__ void __launch_bounds__(256) k_c4_group_wedges_bal(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                                                             const C4Group* __restrict__ grp, const uint64_t* __restrict__ P,
                                                             uint32_t* __restrict__ L, uint64_t stride) {
  const C4Group& G = *grp;
  const uint64_t nc = G.vbeg[G.n];
  const uint64_t* Pg = P + G.cbase;
  const uint64_t E0 = Pg[0], total = Pg[nc] - E0;
  const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / kWarp;
  const uint64_t wid = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp;
  const unsigned lane = lane_id();
  const uint64_t share = (total + warps - 1) / warps;
  const uint64_t s = wid * share, e = min(total, s + share);
  if (s >= e) return;
  // the centre holding entry s: the last c with Pg[c] - E0 <= s (Pg is non-decreasing)
  uint64_t c = 0;
  if (lane == 0) {
    uint64_t lo = 0, hi = nc;  // invariant: Pg[lo] - E0 <= s < Pg[hi] - E0
    while (hi - lo > 1) {
      const uint64_t mid = (lo + hi) / 2;
      if (Pg[mid] - E0 <= s)
        lo = mid;
      else
        hi = mid;
    }
    c = lo;
  }
  c = __shfl_sync(kFull, c, 0);
  uint32_t g = 0;
  while (g + 1 < G.n && c >= G.vbeg[g + 1]) g++;
  uint64_t pos = s;
  while (pos < e && c < nc) {
    const uint64_t rb = Pg[c] - E0, re = Pg[c + 1] - E0;  // this centre's entries
    const uint32_t u = G.root[g], lim = G.lim[g];
    const uint32_t v = __ldg(ci + __ldg(rp + u) + (c - G.vbeg[g]));
    uint32_t* Lg = L + (uint64_t)g * stride;
    const uint64_t row = __ldg(rp + v);
    const uint64_t j0 = row + (pos - rb), jend = row + (min(e, re) - rb);
    for (uint64_t jb = j0; jb < jend; jb += 2 * kWarp) {
      const uint64_t j1 = jb + lane, j2 = j1 + kWarp;
      const uint32_t w1 = j1 < jend ? __ldg(ci + j1) : lim;
      const uint32_t w2 = j2 < jend ? __ldg(ci + j2) : lim;
      if (w1 < lim) {
        if (kPacked)
          atomicAdd(Lg + (w1 >> 1), (w1 & 1u) ? 0x10000u : 1u);
        else
          atomicAdd(Lg + w1, 1u);
      }
      if (w2 < lim) {
        if (kPacked)
          atomicAdd(Lg + (w2 >> 1), (w2 & 1u) ? 0x10000u : 1u);
        else
          atomicAdd(Lg + w2, 1u);
      }
      if (__any_sync(kFull, w2 >= lim)) break;  // w2 >= w1 in every lane that loaded both
    }
    pos = re;
    c++;
    while (g + 1 < G.n && c >= G.vbeg[g + 1]) g++;
  }
}

__device__ __forceinline__ unsigned long long pairs_of_halves(uint32_t c) { return pairs_of_u32(c & 0xffffu) + pairs_of_u32(c >> 16); }

template <bool kPacked>
__global__ void __launch_bounds__(256) k_c4_group_sum(const C4Group* __restrict__ grp, uint32_t* __restrict__ L, uint64_t stride,
                                                      unsigned long long* __restrict__ total) {
  const C4Group& G = *grp;
  unsigned long long acc = 0;
  for (uint32_t g = 0; g < G.n; g++) {
    uint4* Lg = (uint4*)(L + (uint64_t)g * stride);
    // counters below the root, rounded up (the rest are zero): 4 per uint4, 8 packed
    const uint64_t n4 = kPacked ? ((uint64_t)G.lim[g] + 7) / 8 : ((uint64_t)G.lim[g] + 3) / 4;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n4; k += (uint64_t)gridDim.x * blockDim.x) {
      const uint4 c = Lg[k];
      if (c.x | c.y | c.z | c.w) {
        if (kPacked)
          acc += pairs_of_halves(c.x) + pairs_of_halves(c.y) + pairs_of_halves(c.z) + pairs_of_halves(c.w);
        else
          acc += pairs_of(c.x) + pairs_of(c.y) + pairs_of(c.z) + pairs_of(c.w);
        Lg[k] = make_uint4(0u, 0u, 0u, 0u);
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(kFull, acc, o);
  if ((threadIdx.x & (kWarp - 1)) == 0 && acc) atomicAdd(total, acc);
}

// Heavy roots, the top of their range: a cluster of kC4WinCtas blocks takes one root
// u at a time and keeps the counters of the ids [u - kC4Window, u) - where most
// wedges of a heavy root end, the high-degree vertices just below it - as packed
// 16-bit counters in the distributed shared memory of the cluster (block r holds
// ids r*kC4WinPerCta ...).  Every warp of the cluster takes wedge centres v, finds
// the window's start in N(v) and adds its wedges there by shared-memory atomics on
// the owning block; after a cluster barrier each block sums C(L, 2) over its part
// and clears it.  The ids below the window stay with the group kernels (lim).  Only
// roots with fewer than 65536 lower neighbours come here (no counter can overflow).
constexpr int kC4WinCtas = 4;
constexpr uint32_t kC4WinWords = 49152;                      // 192 KB of shared memory per block
constexpr uint32_t kC4WinPerCta = 2 * kC4WinWords;           // ids per block (two per word)
constexpr uint32_t kC4Window = kC4WinCtas * kC4WinPerCta;    // 393,216 ids below the root
constexpr size_t kC4WinSmem = (size_t)kC4WinWords * sizeof(uint32_t);

__global__ void __cluster_dims__(kC4WinCtas, 1, 1) __launch_bounds__(512, 1)
    k_c4_window(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, const uint32_t* __restrict__ roots, uint64_t n,
                unsigned long long* __restrict__ head, unsigned long long* __restrict__ total) {
  namespace cg = cooperative_groups;
  extern __shared__ uint32_t win[];
  __shared__ unsigned long long s_root;
  __shared__ unsigned long long s_sum[16];
  cg::cluster_group cluster = cg::this_cluster();
  const unsigned rank = cluster.block_rank();
  const unsigned lane = lane_id(), wid = threadIdx.x / kWarp, nwarps = blockDim.x / kWarp;
  const unsigned gw = rank * nwarps + wid, nw = kC4WinCtas * nwarps;
  uint32_t* part[kC4WinCtas];
#pragma unroll
  for (int r = 0; r < kC4WinCtas; r++) part[r] = cluster.map_shared_rank(win, r);
  for (uint32_t t = threadIdx.x; t < kC4WinWords; t += blockDim.x) win[t] = 0;
  unsigned long long acc = 0;
  while (true) {
    if (rank == 0 && threadIdx.x == 0) s_root = atomicAdd(head, 1ull);
    cluster.sync();  // the root is popped and every block's window is clear
    const unsigned long long r = *cluster.map_shared_rank(&s_root, 0);
    if (r >= n) break;
    const uint32_t u = __ldg(roots + r);
    const uint32_t lo = u > kC4Window ? u - kC4Window : 0u;
    const uint64_t ua = __ldg(rp + u), uz = __ldg(rp + u + 1);
    for (uint64_t k = ua + gw; k < uz; k += nw) {
      const uint32_t v = __ldg(ci + k);
      if (v >= u) break;  // the row is sorted: the centres below u come first
      const uint64_t vz = __ldg(rp + v + 1);
      for (uint64_t base = warp_lower_bound(ci, __ldg(rp + v), vz, lo); base < vz; base += kWarp) {
        const uint64_t j = base + lane;
        const uint32_t w = j < vz ? __ldg(ci + j) : u;
        if (w < u) {
          const uint32_t x = w - lo;
          atomicAdd(part[x / kC4WinPerCta] + ((x % kC4WinPerCta) >> 1), (x & 1u) ? 0x10000u : 1u);
        }
        if (__any_sync(kFull, w >= u)) break;
      }
    }
    cluster.sync();  // every wedge of u is in the window
    for (uint32_t t = threadIdx.x; t < kC4WinWords; t += blockDim.x) {
      const uint32_t c = win[t];
      if (c) {
        acc += pairs_of_halves(c);
        win[t] = 0;
      }
    }
  }
  cluster.sync();  // no block leaves while another may still read its s_root
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(kFull, acc, o);
  if (lane == 0) s_sum[wid] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (unsigned w = 0; w < nwarps; w++) t += s_sum[w];
    if (t) atomicAdd(total, t);
  }
}

// ---------------------------------------------------------------------------
// View materialisation on the device (ViewBin::Materialize, src/view/view_bin.h:49-142):
// sources of degree >= root_degree start the halo, each further layer adds the
// neighbours of the previous one, then every vertex in the halo gets its full row.
// ---------------------------------------------------------------------------
// flags are one byte per vertex; a word-wide atomicOr of the byte's mask sets one and
// tells the one thread that set it first
__device__ __forceinline__ bool set_flag(uint8_t* flags, uint32_t v) {
  unsigned int* word = (unsigned int*)(flags + (v & ~3u));
  const unsigned int bit = 0xffu << ((v & 3u) * 8);
  unsigned int old = atomicOr(word, bit);
  return (old & bit) == 0;
}

__global__ void k_halo_seed2(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ src, uint64_t n, uint64_t root_degree,
                             uint8_t* __restrict__ in_view, uint32_t* __restrict__ frontier, unsigned long long* __restrict__ n_frontier) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t s = src[i];
    if (root_degree && rp[s + 1] - rp[s] < root_degree) continue;
    if (set_flag(in_view, s)) frontier[atomicAdd(n_frontier, 1ull)] = s;
  }
}

// one warp per frontier vertex: unseen neighbours join the view and the next frontier
__global__ void k_halo_layer(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, uint64_t V, const uint32_t* __restrict__ frontier,
                             uint64_t n, uint8_t* __restrict__ in_view, uint32_t* __restrict__ next, unsigned long long* __restrict__ n_next) {
  const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / kWarp;
  const unsigned lane = lane_id();
  for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; i < n; i += warps) {
    const uint32_t x = frontier[i];
    for (uint64_t j = rp[x] + lane; j < rp[x + 1]; j += kWarp) {
      const uint32_t y = ci[j];
      if (y < V && set_flag(in_view, y)) next[atomicAdd(n_next, 1ull)] = y;  // ids >= V (a corrupt file) are skipped
    }
  }
}

__global__ void k_halo_lengths(const uint64_t* __restrict__ rp, uint64_t V, const uint8_t* __restrict__ in_view, uint64_t* __restrict__ len) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x)
    len[v] = in_view[v] ? rp[v + 1] - rp[v] : 0;
}

// one warp per vertex of the view: copy its row
__global__ void k_halo_copy(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ ci, uint64_t V, const uint8_t* __restrict__ in_view,
                            const uint64_t* __restrict__ out_rp, uint32_t* __restrict__ out_ci) {
  const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / kWarp;
  const unsigned lane = lane_id();
  for (uint64_t v = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; v < V; v += warps) {
    if (!in_view[v]) continue;
    const uint64_t a = rp[v], n = rp[v + 1] - a, o = out_rp[v];
    for (uint64_t j = lane; j < n; j += kWarp) out_ci[o + j] = ci[a + j];
  }
}

// every stride-th root (sampled runs of the autotuner)
__global__ void k_stride_copy(const uint32_t* __restrict__ in, uint64_t n_out, uint64_t stride, uint32_t* __restrict__ out) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_out; i += (uint64_t)gridDim.x * blockDim.x) out[i] = in[i * stride];
}

// ---------------------------------------------------------------------------
// COUNT
// ---------------------------------------------------------------------------
__global__ void k_count_one(Frame f, uint8_t u, unsigned long long* __restrict__ total) {
  const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
  unsigned long long acc = 0;
  for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < f.P; p += nthreads) acc += f.clen[u][p];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(kFull, acc, o);
  if (lane_id() == 0 && acc) atomicAdd(total, acc);
}

// pairs (x0 in set u0, x1 in set u1) with x0 OP x1: walk the smaller set
__global__ void k_count_two(Frame f, uint8_t u0, uint8_t u1, uint8_t op, unsigned long long* __restrict__ total) {
  const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / kWarp;
  const unsigned lane = lane_id();
  unsigned long long acc = 0;
  for (uint64_t p = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; p < f.P; p += warps) {
    const uint32_t* a0 = set_of(f, u0, p);
    const uint32_t* a1 = set_of(f, u1, p);
    uint64_t n0 = f.clen[u0][p], n1 = f.clen[u1][p];
    const uint32_t *walk = a0, *search = a1;
    uint64_t nw = n0, ns = n1;
    uint8_t rel = op;  // relation walked-element OP searched-element
    if (n0 > n1) {
      walk = a1;
      search = a0;
      nw = n1;
      ns = n0;
      rel = op == VSGM_LESS_THAN ? VSGM_LARGER_THAN : (op == VSGM_LARGER_THAN ? VSGM_LESS_THAN : op);
    }
    if (ns == 0) continue;
    uint64_t cur = 0;
    for (uint64_t k = lane; k < nw; k += kWarp) acc += count_vs(search, ns, &cur, __ldg(walk + k), rel);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(kFull, acc, o);
  if (lane == 0 && acc) atomicAdd(total, acc);
}

// ---------------------------------------------------------------------------
// exclusive scan of u64 (three passes over 2048-element tiles)
// ---------------------------------------------------------------------------
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint64_t block_exclusive(uint64_t v, uint64_t* total) {
  __shared__ uint64_t warp_sums[kScanThreads / kWarp];
  const unsigned lane = lane_id(), wid = threadIdx.x / kWarp;
  uint64_t x = v;
  for (int o = 1; o < kWarp; o <<= 1) {
    uint64_t y = __shfl_up_sync(kFull, x, o);
    if (lane >= (unsigned)o) x += y;
  }
  if (lane == kWarp - 1) warp_sums[wid] = x;
  __syncthreads();
  if (wid == 0) {
    uint64_t s = (lane < kScanThreads / kWarp) ? warp_sums[lane] : 0;
    for (int o = 1; o < kWarp; o <<= 1) {
      uint64_t y = __shfl_up_sync(kFull, s, o);
      if (lane >= (unsigned)o) s += y;
    }
    if (lane < kScanThreads / kWarp) warp_sums[lane] = s;
  }
  __syncthreads();
  uint64_t before = (wid > 0 ? warp_sums[wid - 1] : 0) + x - v;
  *total = warp_sums[kScanThreads / kWarp - 1];
  __syncthreads();
  return before;
}

// in may be a u64 or u32 array (kIn32)
template <bool kIn32>
__global__ void k_scan_tiles(const void* __restrict__ in, uint64_t n, uint64_t* __restrict__ tile_sums) {
  const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
  uint64_t s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; i++)
    if (base + i < n) s += kIn32 ? (uint64_t)((const uint32_t*)in)[base + i] : ((const uint64_t*)in)[base + i];
  uint64_t total;
  block_exclusive(s, &total);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

template <bool kIn32>
__global__ void k_scan_apply(const void* __restrict__ in, uint64_t n, const uint64_t* __restrict__ tile_prefix, uint64_t* __restrict__ out) {
  const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
  uint64_t v[kScanItems];
  uint64_t s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    v[i] = (base + i < n) ? (kIn32 ? (uint64_t)((const uint32_t*)in)[base + i] : ((const uint64_t*)in)[base + i]) : 0;
    s += v[i];
  }
  uint64_t total;
  uint64_t run = block_exclusive(s, &total) + tile_prefix[blockIdx.x];
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    if (base + i < n) out[base + i] = run;
    run += v[i];
  }
  // out[n] = grand total, written by the block that owns the last element
  if (base < n && base + kScanItems >= n) out[n] = run;
}

}  // namespace dev
}  // namespace vsgm
