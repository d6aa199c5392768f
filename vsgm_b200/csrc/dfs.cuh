// Persistent depth-first plan interpreter (sm_100a).
//
// One launch runs many (view, plan, root-range) tasks: every warp pops tasks
// from a device queue (one atomicAdd per pop, no waiting) and walks the whole
// execution sequence depth-first for each root of its task, keeping candidate
// sets in a per-warp scratch region instead of materialising partial matches in
// HBM.  The op semantics are the same as the level-wise engine's (and the
// reference's, src/executor/ops/*.h); only the traversal order differs, and
// counts do not depend on it.  This is what keeps many small views and many
// patterns from being launch-bound: the level-wise engine needs a few kernels and
// host synchronisations per op per batch, this needs one launch in total.
#pragma once

#include "kernels.cuh"

namespace vsgm {
namespace dev {

struct DfsOp {
  uint8_t type, u;
  uint8_t nb;
  uint8_t b[VSGM_MAX_QV];
  uint8_t nc;
  uint8_t cop[VSGM_MAX_QV];
  uint8_t cv[VSGM_MAX_QV];
  int8_t other;      // COMPUTE_COUNT: computed vertex counted against (-1 none)
  uint8_t other_op;  // candidate(u) OP candidate(other)
  uint8_t ncu;       // COUNT: computed vertices (1 or 2)
  uint8_t cu0, cu1, cu_op;
};

// The last MATERIALIZE(u) fused with the final COMPUTE_COUNT(w) (same rule as the
// level-wise engine's fused tail): the lists and conditions of w that do not
// involve u are intersected once per parent, then every child c of u counts its
// share of that set in N(c), one child per lane.
struct DfsFused {
  uint8_t on, lvl;     // lvl: the MATERIALIZE's op index
  uint8_t has_cond_u;  // condition  candidate(w)  cond_u_op  c
  uint8_t cond_u_op;
  int8_t other;        // computed vertex counted against (-1 none)
  uint8_t other_op;
  DfsOp known;         // nb/b: backward lists of w without u; nc/cop/cv: conditions of w not on u
};

struct DfsPlan {
  uint32_t n_ops;
  uint32_t root;
  uint32_t split_lvl;  // first MATERIALIZE after the root (n_ops if none): where a root's work can be split
  DfsFused fz;
  DfsOp op[VSGM_MAX_OPS];
};

struct DfsView {
  const uint64_t* rp;
  const uint32_t* ci;
  const uint32_t* sources;
};

struct DfsTask {
  uint32_t plan, view;
  uint64_t r0, r1;  // source index range within the view
  // c1 != 0: a share of one heavy root (r1 == r0 + 1): only the candidates
  // [c0, c1) of the plan's split level are expanded, so several warps share it
  uint32_t c0, c1;
};

constexpr int kDfsWarps = 8;  // warps per block

// per-warp control state (shared memory)
struct DfsState {
  uint32_t M[8];
  const uint32_t* set[8];
  uint32_t len[8];
  const uint32_t* iset[VSGM_MAX_OPS];  // MATERIALIZE: set being iterated; FILTER: saved set
  uint32_t ilen[VSGM_MAX_OPS];
  uint32_t inext[VSGM_MAX_OPS];
  uint32_t ne[VSGM_MAX_OPS][VSGM_MAX_QV];  // MATERIALIZE: values to skip
};

__device__ __forceinline__ void dfs_window(const DfsOp& o, const uint32_t* M, Window* w) {
  w->lo = 0;
  w->hi = 0x100000000ull;
  w->nne = o.nc;
#pragma unroll
  for (int i = 0; i < VSGM_MAX_QV; i++) {
    w->ne[i] = 0xffffffffu;
    if (i < o.nc) window_add(w, o.cop[i], M[o.cv[i]], i);
  }
}

// restricted ranges of the backward lists; lane j < nb searches list j
__device__ __forceinline__ void dfs_lists(const DfsOp& o, const uint32_t* M, const Window& w, const uint64_t* __restrict__ rp,
                                          const uint32_t* __restrict__ ci, Lists* L) {
  const unsigned lane = lane_id();
  uint64_t s = 0, e = 0;
  if (lane < o.nb) {
    uint32_t v = M[o.b[lane]];
    uint64_t a = __ldg(rp + v), z = __ldg(rp + v + 1);
    s = (w.lo > 0) ? lower_bound(ci, a, z, w.lo) : a;
    e = (w.hi <= 0xffffffffull) ? lower_bound(ci, s, z, w.hi) : z;
    if (e < s) e = s;
  }
  uint64_t best = ~0ull;
  int piv = 0;
#pragma unroll
  for (int i = 0; i < VSGM_MAX_QV; i++) {
    uint64_t si = __shfl_sync(kFull, s, i), ei = __shfl_sync(kFull, e, i);
    L->s[i] = si;
    L->e[i] = ei;
    if (i < o.nb && ei - si < best) {
      best = ei - si;
      piv = i;
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

// Walk the pivot; emit(c) for every candidate in all other lists passing the
// NON_EQUAL checks.  Generic over the backward count (<= 6 lists).
template <typename Emit>
__device__ __forceinline__ void dfs_intersect(const DfsOp& o, const Window& w, const Lists& L, const uint32_t* __restrict__ ci, Emit&& emit) {
  const unsigned lane = lane_id();
  uint64_t pos[VSGM_MAX_QV - 1];
#pragma unroll
  for (int j = 0; j < VSGM_MAX_QV - 1; j++) pos[j] = L.s[j];
  for (uint64_t base = L.ps; base < L.pe; base += kWarp) {
    const uint64_t k = base + lane;
    bool ok = false;
    uint32_t c = 0;
    if (k < L.pe) {
      c = __ldg(ci + k);
      ok = ne_ok(w, c);
#pragma unroll
      for (int j = 0; j < VSGM_MAX_QV - 1; j++) {
        if (j >= o.nb || j == L.pivot || !ok) continue;
        uint64_t q = gallop(ci, pos[j], L.e[j], c);
        pos[j] = q;
        ok = (q < L.e[j]) && (__ldg(ci + q) == c);
      }
    }
    emit(ok, c);
  }
}

// candidates x of a (sorted, length n) with  c op x
__device__ __forceinline__ uint64_t dfs_count_vs(const uint32_t* a, uint64_t n, uint32_t c, uint8_t op) {
  uint64_t q = lower_bound(a, 0, n, c);
  bool eq = q < n && __ldg(a + q) == c;
  if (op == VSGM_LESS_THAN) return n - q - (eq ? 1 : 0);
  if (op == VSGM_LARGER_THAN) return q;
  return n - (eq ? 1 : 0);
}

// All-lanes helper: copy set (ptr, n) minus NON_EQUAL values into out; returns written.
__device__ __forceinline__ uint32_t dfs_filter_copy(const uint32_t* in, uint32_t n, const Window& w, uint32_t* out) {
  const unsigned lane = lane_id();
  uint32_t written = 0;
  for (uint32_t base = 0; base < n; base += kWarp) {
    const uint32_t k = base + lane;
    uint32_t c = 0;
    bool ok = false;
    if (k < n) {
      c = __ldg(in + k);
      ok = (uint64_t)c >= w.lo && (uint64_t)c < w.hi && ne_ok(w, c);
    }
    unsigned mask = __ballot_sync(kFull, ok);
    if (ok) out[written + __popc(mask & ((1u << lane) - 1))] = c;
    written += __popc(mask);
  }
  __syncwarp();
  return written;
}

// slice of sorted a[0, n) inside the window's order bounds
__device__ __forceinline__ void dfs_narrow(const uint32_t* a, uint32_t n, const Window& w, const uint32_t** out, uint32_t* out_n) {
  uint64_t s = (w.lo > 0) ? lower_bound(a, 0, n, w.lo) : 0;
  uint64_t e = (w.hi <= 0xffffffffull) ? lower_bound(a, s, n, w.hi) : n;
  if (e < s) e = s;
  *out = a + s;
  *out_n = (uint32_t)(e - s);
}

// does the slice contain one of the window's NON_EQUAL values?
__device__ __forceinline__ bool dfs_has_ne(const uint32_t* a, uint32_t n, const Window& w) {
  bool hit = false;
#pragma unroll
  for (int i = 0; i < VSGM_MAX_QV; i++) {
    if (w.ne[i] == 0xffffffffu || n == 0) continue;
    uint64_t q = lower_bound(a, 0, n, w.ne[i]);
    hit |= (q < n && __ldg(a + q) == w.ne[i]);
  }
  return hit;
}

// Fused tail of one parent (DfsFused): children are cs[k0, n) minus the values in
// skip[]; I is a scratch buffer of at least the largest degree.  Returns the
// matches; *n_children = children expanded (what the unfused walk would enter).
__device__ __forceinline__ unsigned long long dfs_fused(const DfsFused& fz, const uint32_t* M, const uint32_t* cs, uint32_t k0, uint32_t n,
                                                        const uint32_t* skip, const uint32_t* oset, uint32_t on, const uint64_t* __restrict__ rp,
                                                        const uint32_t* __restrict__ ci, uint32_t* I, uint64_t* n_children) {
  const unsigned lane = lane_id();
  unsigned long long acc = 0;
  uint32_t kids = 0;
  for (uint32_t k = k0 + lane; k < n; k += kWarp) {
    const uint32_t c = cs[k];
    bool sk = false;
#pragma unroll
    for (int i = 0; i < VSGM_MAX_QV; i++) sk |= (c == skip[i]);
    kids += sk ? 0u : 1u;
  }
  for (int o = 16; o > 0; o >>= 1) kids += __shfl_xor_sync(kFull, kids, o);
  *n_children = kids;
  if (kids == 0) return 0;
  Window w;
  dfs_window(fz.known, M, &w);  // conditions not involving u
  Window ws = w;
  if (fz.has_cond_u && fz.cond_u_op == VSGM_LARGER_THAN) window_add(&ws, VSGM_LARGER_THAN, cs[k0], 0);
  if (fz.has_cond_u && fz.cond_u_op == VSGM_LESS_THAN) window_add(&ws, VSGM_LESS_THAN, cs[n - 1], 0);
  Lists L;
  dfs_lists(fz.known, M, ws, rp, ci, &L);
  uint32_t ni = 0;
  if (fz.known.nb == 1) {
    ni = dfs_filter_copy(ci + L.ps, (uint32_t)(L.pe - L.ps), w, I);
  } else {
    dfs_intersect(fz.known, w, L, ci, [&](bool ok, uint32_t c) {
      unsigned mask = __ballot_sync(kFull, ok);
      if (ok) I[ni + __popc(mask & ((1u << lane) - 1))] = c;
      ni += __popc(mask);
    });
    __syncwarp();
  }
  if (ni == 0) return 0;
  FusedDesc fd;
  fd.has_cond_u = fz.has_cond_u;
  fd.cond_u_op = fz.cond_u_op;
  const bool excl_child = fz.has_cond_u && fz.cond_u_op == VSGM_NON_EQUAL;
  const bool other = fz.other >= 0;
  for (uint32_t b0 = k0; b0 < n; b0 += kWarp) {
    // pass 1, one child per lane; long slices are left for pass 2
    const uint32_t k = b0 + lane;
    bool heavy = false;
    uint32_t c = 0;
    if (k < n) {
      c = cs[k];
      bool sk = false;
#pragma unroll
      for (int i = 0; i < VSGM_MAX_QV; i++) sk |= (c == skip[i]);
      if (!sk) {
        uint32_t ia, ib;
        child_slice(fd, w, I, ni, c, &ia, &ib);
        if (ib - ia > kLaneSlice) {
          heavy = true;
        } else if (ia < ib) {
          const uint64_t z0 = __ldg(rp + c + 1);
          uint64_t cur = __ldg(rp + c), ocur = 0;
          const uint32_t excl = excl_child ? c : 0xffffffffu;
          for (uint32_t j = ia; j < ib; j++) {
            const uint32_t x = I[j];
            const uint64_t r = gallop(ci, cur, z0, x);
            cur = r;
            if (r < z0 && __ldg(ci + r) == x && x != excl) acc += other ? count_vs(oset, on, &ocur, x, fz.other_op) : 1ull;
          }
        }
      }
    }
    // pass 2: the long slices of this group, one child at a time, by the whole warp
    unsigned todo = __ballot_sync(kFull, heavy);
    while (todo) {
      const int src = __ffs(todo) - 1;
      todo &= todo - 1;
      const uint32_t hc = __shfl_sync(kFull, c, src);
      uint32_t ia, ib;
      child_slice(fd, w, I, ni, hc, &ia, &ib);
      const uint64_t a0 = __ldg(rp + hc), z0 = __ldg(rp + hc + 1);
      const uint64_t s2 = warp_lower_bound(ci, a0, z0, I[ia]);
      const uint64_t e2 = warp_lower_bound(ci, s2, z0, (uint64_t)I[ib - 1] + 1);
      if (s2 >= e2) continue;
      const uint32_t excl = excl_child ? hc : 0xffffffffu;
      uint64_t ocur = 0;
      if ((uint64_t)(ib - ia) <= (e2 - s2)) {
        uint64_t cur = s2;
        for (uint32_t j = ia + lane; j < ib; j += kWarp) {
          const uint32_t x = I[j];
          const uint64_t r = gallop(ci, cur, e2, x);
          cur = r;
          if (r < e2 && __ldg(ci + r) == x && x != excl) acc += other ? count_vs(oset, on, &ocur, x, fz.other_op) : 1ull;
        }
      } else {
        uint32_t cur = ia;
        for (uint64_t j = s2 + lane; j < e2; j += kWarp) {
          const uint32_t x = __ldg(ci + j);
          const uint32_t r = smem_lower_bound(I, cur, ib, x);
          cur = r;
          if (r < ib && I[r] == x && x != excl) acc += other ? count_vs(oset, on, &ocur, x, fz.other_op) : 1ull;
        }
      }
    }
  }
  __syncwarp();
  return acc;
}

// The interpreter.  scratch: per warp, `levels` buffers of `cap` u32 (levels =
// the longest execution sequence, cap = the largest degree of any view).
// counts[task.plan * n_views + task.view] += matches.  *status != 0 on return
// means a candidate set did not fit in cap (the host reports an error; cap is
// the largest degree, which bounds every candidate set, so it does not happen).
// Nothing in the kernel waits on another warp.
// Optional outputs: level_paths[pair * VSGM_MAX_OPS + i] += partial matches
// entering op i (pair = plan * n_views + view); with step_budget > 0 a task stops
// after that many forward steps and sets overflow[pair] (its counts are then
// partial) - a bound on the work of one launch, not a wait.
__global__ void __launch_bounds__(kDfsWarps * kWarp) k_dfs(const DfsPlan* __restrict__ plans, const DfsView* __restrict__ views,
                                                           const DfsTask* __restrict__ tasks, uint64_t n_tasks, unsigned long long* __restrict__ head,
                                                           uint32_t* __restrict__ scratch, uint64_t cap, uint32_t levels, uint32_t n_views,
                                                           unsigned long long* __restrict__ counts, unsigned int* __restrict__ status,
                                                           unsigned long long* __restrict__ level_paths, uint64_t step_budget,
                                                           unsigned int* __restrict__ overflow) {
  __shared__ DfsState sst[kDfsWarps];
  __shared__ DfsOp sop[kDfsWarps][VSGM_MAX_OPS];
  __shared__ unsigned long long svisit[kDfsWarps][VSGM_MAX_OPS];
  const unsigned lane = lane_id(), wib = threadIdx.x / kWarp;
  DfsState& S = sst[wib];
  DfsOp* O = sop[wib];
  const uint64_t gw = (uint64_t)blockIdx.x * kDfsWarps + wib;
  uint32_t* my = scratch + gw * (uint64_t)levels * cap;

  while (true) {
    unsigned long long t = 0;
    if (lane == 0) t = atomicAdd(head, 1ull);
    t = __shfl_sync(kFull, t, 0);
    if (t >= n_tasks) break;
    const DfsTask task = tasks[t];
    const DfsPlan& P = plans[task.plan];
    const DfsView V = views[task.view];
    const uint32_t n_ops = P.n_ops;
    // a share of a split root counts the levels up to the split once (share 0 only)
    const uint32_t split_lvl = task.c1 ? P.split_lvl : n_ops;
    const bool first_share = task.c0 == 0;
    // stage the plan's ops in shared memory
    for (uint32_t i = lane; i < n_ops * (uint32_t)sizeof(DfsOp); i += kWarp) ((uint8_t*)O)[i] = ((const uint8_t*)P.op)[i];
    if (lane < VSGM_MAX_OPS) svisit[wib][lane] = 0;
    __syncwarp();
    unsigned long long acc = 0;
    uint64_t steps = 0;
    bool stopped = false;

    for (uint64_t r = task.r0; r < task.r1 && !stopped; r++) {
      if (lane == 0) {
        S.M[P.root] = __ldg(V.sources + r);
        if (first_share) svisit[wib][0]++;
      }
      __syncwarp();
      int lvl = 1;
      bool forward = true;
      while (lvl >= 1) {
        if (forward) {
          if (lane == 0 && (first_share || (uint32_t)lvl > split_lvl)) svisit[wib][lvl]++;
          if (step_budget && ++steps > step_budget) {
            stopped = true;
            break;
          }
        }
        if (!forward) {
          // backtrack: undo FILTER levels, resume the nearest MATERIALIZE
          const DfsOp& o = O[lvl];
          if (o.type == VSGM_FILTER_COMPUTE) {
            if (lane == 0) {
              S.set[o.u] = S.iset[lvl];
              S.len[o.u] = S.ilen[lvl];
            }
            __syncwarp();
            lvl--;
            continue;
          }
          if (o.type != VSGM_MATERIALIZE) {
            lvl--;
            continue;
          }
        }
        const DfsOp& o = O[lvl];
        if (o.type == VSGM_MATERIALIZE) {
          if (forward) {
            Window w;
            dfs_window(o, S.M, &w);
            if (lane == 0) {
              const uint32_t* a;
              uint32_t n;
              dfs_narrow(S.set[o.u], S.len[o.u], w, &a, &n);
              uint32_t k0 = 0;
              if ((uint32_t)lvl == split_lvl) {  // this task's share of the root's candidates
                n = n < task.c1 ? n : task.c1;
                k0 = task.c0 < n ? task.c0 : n;
              }
              S.iset[lvl] = a;
              S.ilen[lvl] = n;
              S.inext[lvl] = k0;
              for (int i = 0; i < VSGM_MAX_QV; i++) S.ne[lvl][i] = w.ne[i];
            }
            __syncwarp();
            if (P.fz.on && (uint32_t)lvl == P.fz.lvl) {
              // fused tail: all children of this parent at once, then backtrack
              const int8_t ot = P.fz.other;
              uint64_t kids = 0;
              acc += dfs_fused(P.fz, S.M, S.iset[lvl], S.inext[lvl], S.ilen[lvl], S.ne[lvl], ot >= 0 ? S.set[ot] : nullptr,
                               ot >= 0 ? S.len[ot] : 0u, V.rp, V.ci, my + (uint64_t)(lvl + 1) * cap, &kids);
              if (lane == 0 && (first_share || (uint32_t)(lvl + 1) > split_lvl)) svisit[wib][lvl + 1] += kids;
              steps += kids;
              forward = false;
              lvl--;
              continue;
            }
          }
          // next candidate not equal to a NON_EQUAL value
          if (lane == 0) {
            uint32_t k = S.inext[lvl];
            const uint32_t* a = S.iset[lvl];
            while (k < S.ilen[lvl]) {
              uint32_t c = a[k];
              bool skip = false;
              for (int i = 0; i < VSGM_MAX_QV; i++) skip |= (c == S.ne[lvl][i]);
              if (!skip) break;
              k++;
            }
            S.inext[lvl] = k + 1;
            if (k < S.ilen[lvl]) S.M[o.u] = a[k];
          }
          __syncwarp();
          if (S.inext[lvl] > S.ilen[lvl]) {
            forward = false;
            lvl--;
          } else {
            forward = true;
            lvl++;
          }
          continue;
        }
        if (o.type == VSGM_COMPUTE) {
          Window w;
          dfs_window(o, S.M, &w);
          uint32_t* out = my + (uint64_t)lvl * cap;
          if (o.nb == 1) {
            const uint32_t v = S.M[o.b[0]];
            const uint64_t a0 = __ldg(V.rp + v);
            const uint32_t* a;
            uint32_t n;
            dfs_narrow(V.ci + a0, (uint32_t)(__ldg(V.rp + v + 1) - a0), w, &a, &n);
            if (dfs_has_ne(a, n, w)) {
              if (n > cap) {
                if (lane == 0) atomicOr(status, 1u);
                n = 0;
              } else {
                n = dfs_filter_copy(a, n, w, out);
              }
              a = out;
            }
            if (lane == 0) {
              S.set[o.u] = a;
              S.len[o.u] = n;
            }
          } else {
            Lists L;
            dfs_lists(o, S.M, w, V.rp, V.ci, &L);
            uint32_t written = 0;
            if (L.pe - L.ps > cap) {
              if (lane == 0) atomicOr(status, 1u);
            } else {
              dfs_intersect(o, w, L, V.ci, [&](bool ok, uint32_t c) {
                unsigned mask = __ballot_sync(kFull, ok);
                if (ok) out[written + __popc(mask & ((1u << lane) - 1))] = c;
                written += __popc(mask);
              });
            }
            if (lane == 0) {
              S.set[o.u] = out;
              S.len[o.u] = written;
            }
          }
          __syncwarp();
          lvl++;
          forward = true;
          continue;
        }
        if (o.type == VSGM_FILTER_COMPUTE) {
          Window w;
          dfs_window(o, S.M, &w);
          const uint32_t* a;
          uint32_t n;
          dfs_narrow(S.set[o.u], S.len[o.u], w, &a, &n);
          if (dfs_has_ne(a, n, w)) {
            uint32_t* out = my + (uint64_t)lvl * cap;
            n = dfs_filter_copy(a, n, w, out);
            a = out;
          }
          if (lane == 0) {
            S.iset[lvl] = S.set[o.u];
            S.ilen[lvl] = S.len[o.u];
            S.set[o.u] = a;
            S.len[o.u] = n;
          }
          __syncwarp();
          lvl++;
          forward = true;
          continue;
        }
        if (o.type == VSGM_COMPUTE_COUNT) {
          Window w;
          dfs_window(o, S.M, &w);
          Lists L;
          dfs_lists(o, S.M, w, V.rp, V.ci, &L);
          const uint32_t* oset = o.other >= 0 ? S.set[o.other] : nullptr;
          const uint32_t on = o.other >= 0 ? S.len[o.other] : 0;
          dfs_intersect(o, w, L, V.ci, [&](bool ok, uint32_t c) {
            if (ok) acc += (o.other >= 0) ? dfs_count_vs(oset, on, c, o.other_op) : 1ull;
          });
        } else if (o.type == VSGM_COUNT) {
          if (o.ncu == 1) {
            if (lane == 0) acc += S.len[o.cu0];
          } else {
            const uint32_t *a0 = S.set[o.cu0], *a1 = S.set[o.cu1];
            uint32_t n0 = S.len[o.cu0], n1 = S.len[o.cu1];
            uint8_t rel = o.cu_op;
            if (n0 > n1) {
              const uint32_t* t2 = a0;
              a0 = a1;
              a1 = t2;
              uint32_t tn = n0;
              n0 = n1;
              n1 = tn;
              rel = rel == VSGM_LESS_THAN ? VSGM_LARGER_THAN : (rel == VSGM_LARGER_THAN ? VSGM_LESS_THAN : rel);
            }
            if (n1)
              for (uint32_t k = lane; k < n0; k += kWarp) acc += dfs_count_vs(a1, n1, __ldg(a0 + k), rel);
          }
        }
        // counting ops end the branch
        forward = false;
        lvl--;
      }
    }
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(kFull, acc, off);
    const uint64_t pair = (uint64_t)task.plan * n_views + task.view;
    if (lane == 0 && acc) atomicAdd(counts + pair, acc);
    if (lane == 0 && stopped && overflow) atomicOr(overflow + pair, 1u);
    __syncwarp();
    if (level_paths && lane < n_ops && svisit[wib][lane]) atomicAdd(level_paths + pair * VSGM_MAX_OPS + lane, svisit[wib][lane]);
    __syncwarp();
  }
}

}  // namespace dev
}  // namespace vsgm
