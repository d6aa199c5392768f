// The enumeration engine: plan interpreter over device frames with
// memory-bounded batching, and its C ABI.
//
// Control flow follows the reference executor (src/executor/processor.h:24-263):
// one recursive step per op of the execution sequence, depth-first across ops so
// that only one batch per level is alive, breadth-first within a batch.  The
// differences are B200-first:
//   - one device arena (cudaMalloc once) used as a stack, instead of a
//     cudaMalloc/cudaFree per array (src/device/cuda_context.h:163-223);
//   - batches are cut by exact or upper-bound output sizes computed on the
//     device, split points found by bisection over the device prefix sums;
//   - candidate sets that are slices of an adjacency list are not copied;
//   - COMPUTE writes its output in one pass (no count pass followed by a
//     recomputing write pass, src/gpu/gpu_utils_gpsm_bin_search.h:134-171);
//   - every count is an exact uint64 accumulated on the device and read once
//     per match.
#include <cuda.h>  // CUcontext / CUresult types only: driver calls go through cudaGetDriverEntryPointByVersion
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "clique.cuh"
#include "dfs.cuh"
#include "kernels.cuh"
#include "relabel.cuh"
#include "vsgm.h"

using namespace vsgm::dev;

namespace {

struct CudaError {
  cudaError_t code;
  const char* what;
  int line;
};

#define CK(x)                                             \
  do {                                                    \
    cudaError_t e_ = (x);                                 \
    if (e_ != cudaSuccess) throw CudaError{e_, #x, __LINE__}; \
  } while (0)

struct OutOfMemory {
  std::string what;
};

// Stack allocator over one device allocation.
struct Arena {
  char* base = nullptr;
  size_t cap = 0, top = 0, peak = 0;
  static size_t align(size_t x) { return (x + 255) & ~(size_t)255; }
  size_t avail() const { return cap - top; }
  void* take(size_t bytes, const char* what) {
    size_t need = align(bytes ? bytes : 1);
    if (need > cap - top) throw OutOfMemory{std::string("HBM budget exhausted allocating ") + what};
    void* p = base + top;
    top += need;
    peak = std::max(peak, top);
    return p;
  }
  template <typename T>
  T* take_n(uint64_t n, const char* what) {
    return (T*)take(n * sizeof(T), what);
  }
};

struct Mark {
  Arena& a;
  size_t top;
  explicit Mark(Arena& ar) : a(ar), top(ar.top) {}
  ~Mark() { a.top = top; }
};

}  // namespace

namespace {
// full-V row offsets of a view sent in compact form: rp[v] = offsets[number of
// listed vertices below v] (vertices ascending, offsets[0] = 0), rp[V] = the total
__global__ void k_rows_from_compact(const uint32_t* __restrict__ vert, uint64_t n_vert, const uint64_t* __restrict__ off, uint64_t V,
                                    uint64_t* __restrict__ rp) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v <= V; v += (uint64_t)gridDim.x * blockDim.x)
    rp[v] = off[lower_bound(vert, 0, n_vert, v)];
}
}  // namespace

struct vsgm_engine {
  int device = 0;
  cudaStream_t stream = nullptr;
  int sms = 148;
  uint64_t V = 0;
  std::vector<vsgm_plan> plans;
  uint64_t max_sources = 0;

  // view
  uint64_t* d_rp = nullptr;
  uint32_t* d_ci = nullptr;
  uint32_t* d_src = nullptr;
  uint64_t n_cols = 0, n_src = 0, cols_cap = 0, src_cap = 0;
  bool own_cols = false, have_view = false;
  uint64_t* own_rp = nullptr;
  uint32_t* own_ci = nullptr;
  uint32_t* own_src = nullptr;
  // full graph resident for device-side view materialisation (vsgm_upload_graph)
  uint64_t* g_rp = nullptr;
  uint32_t* g_ci = nullptr;
  uint64_t g_cols = 0, g_cap = 0;
  bool relabel = false;         // option "relabel": vsgm_upload_graph orders ids by degree on the device
  uint32_t* g_new = nullptr;    // new id of every caller id of the resident graph (when relabelled)
  // per view: offset of each vertex's first larger neighbour (fused tails with a "> child" condition)
  uint32_t* d_up = nullptr;
  const uint64_t* up_of = nullptr;  // the row_ptrs d_up was computed for
  uint64_t up_cap = 0;

  // second view buffer, filled on the copy stream while the current view is matched
  // (vsgm_prefetch_view / vsgm_swap_view)
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_copy = nullptr;
  // a second compute stream (4-cycle groups alternate between the two), and its fork / join events
  cudaStream_t aux_stream = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  uint64_t* bk_rp = nullptr;
  uint32_t* bk_ci = nullptr;
  uint32_t* bk_src = nullptr;
  uint32_t* bk_vert = nullptr;
  uint64_t* bk_off = nullptr;
  uint64_t bk_cols_cap = 0, bk_src_cap = 0, bk_vert_cap = 0, bk_n_cols = 0, bk_n_src = 0;
  bool bk_pending = false;

  Arena arena;
  unsigned long long* d_counts = nullptr;  // [n_plans]
  unsigned long long* d_bytes = nullptr;   // [1] profiling byte counter
  uint64_t* h_pinned = nullptr;            // small pinned staging

  std::vector<uint64_t> totals;
  std::vector<vsgm_plan_stats> stats;
  bool profiling = false;
  // per-plan tuning knobs (vsgm_set_option / vsgm_set_plan_option)
  struct Knobs {
    bool fuse_tail = true;           // fused MATERIALIZE + COMPUTE_COUNT
    uint32_t stage_cap = kStageCap;  // shared-memory stage of the fused tail, in u32
    uint32_t merge_ratio = 4;        // merge vs gallop threshold of the warp intersection
    bool lane_merge = false;         // counting kernels: lane-partitioned merge
    bool c4_aggregate = true;        // 4-cycle plans: wedge aggregation instead of the op sequence
    bool set_reuse = true;           // COMPUTE o + COMPUTE_COUNT w over the same set: count pairs of one intersection
    uint64_t c4_heavy = kC4HashBlockMaxW + 1;  // 4-cycle roots with at least this many wedges use the L2-resident group kernels
    bool c4_hash = true;             // 4-cycle light roots: counters in a shared-memory hash table
    bool c4_window = false;          // 4-cycle heavy roots: the ids just below the root counted in cluster shared memory
    bool c4_balance = false;         // 4-cycle heavy groups: work split by adjacency entries instead of by wedge centre
    uint32_t walk_ratio = 8;         // fused tail: walk N(c) unless it is this many times longer than the slice
    uint32_t lane_slice = kLaneSlice;  // fused tail: longest slice a lane handles alone
    bool tail_merge = false;           // fused tail: heavy children by a merge-path split over the lanes
    bool clique_bits = true;           // 3- and 4-clique plans: bitmap operator on the roots' out-neighbourhoods
    bool edge_triangles = true;        // diamond plans: pairs of per-edge triangle counts
  };
  std::vector<Knobs> knobs;
  Knobs cur;
  uint64_t root_stride = 1;  // >1: match only every root_stride-th source (autotuning samples)
  uint64_t hybrid_steps = 1ull << 14;  // vsgm_run_batched: pairs whose tasks exceed this many steps rerun level-wise (0: never)
  int streams = 4;                     // those reruns run on this many streams at once (host threads, one helper engine each)
  std::vector<vsgm_engine*> helpers;   // helper engines: own stream, counters, statistics; the resident views and arena slices are ours
  bool helper = false;                 // this engine is a helper: its views and arena belong to its parent
  int only_plan = -1;        // >=0: vsgm_match runs this plan only
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t ev_h0 = nullptr, ev_h1 = nullptr;  // around a hybrid batched run
  std::string err;

  // resident views for batched runs (vsgm_add_view)
  struct ResidentView {
    uint64_t V = 0, n_cols = 0, n_src = 0, max_deg = 0;
    uint64_t* rp = nullptr;
    uint32_t* ci = nullptr;
    uint32_t* src = nullptr;
    std::vector<uint64_t> h_deg_src;  // degree of each source (task costing)
  };
  std::vector<ResidentView> rviews;
  vsgm_batch_stats bstats{};

  // per-match state
  const vsgm_plan* plan = nullptr;
  vsgm_plan_stats* st = nullptr;
  unsigned long long* d_total = nullptr;

  // ------------------------------------------------------------- helpers
  unsigned grid_warps(uint64_t work_items) const {
    // warp-per-item kernels: 8 warps per 256-thread block, enough blocks to fill
    // every SM several times over
    uint64_t blocks = (work_items + 7) / 8;
    uint64_t cap = (uint64_t)sms * 16;
    return (unsigned)std::max<uint64_t>(1, std::min(blocks, cap));
  }
  unsigned grid_threads(uint64_t work_items) const {
    uint64_t blocks = (work_items + 255) / 256;
    uint64_t cap = (uint64_t)sms * 16;
    return (unsigned)std::max<uint64_t>(1, std::min(blocks, cap));
  }

  const uint32_t* upper_offsets() {
    if (up_of != d_rp || !d_up) {
      if (d_up && up_cap < V) {
        CK(cudaFree(d_up));
        d_up = nullptr;
      }
      if (!d_up) {
        CK(cudaMalloc(&d_up, sizeof(uint32_t) * std::max<uint64_t>(V, 1)));
        up_cap = V;
      }
      k_upper_offsets<<<grid_threads(V), 256, 0, stream>>>(d_rp, d_ci, V, d_up);
      CK(cudaGetLastError());
      up_of = d_rp;
    }
    return d_up;
  }

  uint64_t read_u64(const uint64_t* d) {
    CK(cudaMemcpyAsync(h_pinned, d, sizeof(uint64_t), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    return h_pinned[0];
  }

  // exclusive scan of n values (u32 or u64) into out[0..n], out[n] = total
  void scan(const void* in, bool in32, uint64_t n, uint64_t* out) {
    if (n == 0) {
      CK(cudaMemsetAsync(out, 0, sizeof(uint64_t), stream));
      return;
    }
    Mark m(arena);
    uint64_t tiles = (n + kScanTile - 1) / kScanTile;
    uint64_t* sums = arena.take_n<uint64_t>(tiles + 1, "scan tiles");
    if (in32)
      k_scan_tiles<true><<<(unsigned)tiles, kScanThreads, 0, stream>>>(in, n, sums);
    else
      k_scan_tiles<false><<<(unsigned)tiles, kScanThreads, 0, stream>>>(in, n, sums);
    CK(cudaGetLastError());
    if (tiles == 1) {
      CK(cudaMemsetAsync(sums, 0, sizeof(uint64_t), stream));
    } else {
      scan(sums, false, tiles, sums);  // in place is safe: each tile is read before it is written
    }
    if (in32)
      k_scan_apply<true><<<(unsigned)tiles, kScanThreads, 0, stream>>>(in, n, sums, out);
    else
      k_scan_apply<false><<<(unsigned)tiles, kScanThreads, 0, stream>>>(in, n, sums, out);
    CK(cudaGetLastError());
  }

  // Stable radix sort of n (key, value) pairs by the low `bits` bits of the keys,
  // ping-ponging between (k0, v0) and (k1, v1); true when the result is in (k1, v1).
  bool radix_sort(uint32_t* k0, uint32_t* v0, uint32_t* k1, uint32_t* v1, uint64_t n, int bits) {
    if (n == 0) return false;
    const uint64_t tiles = (n + kRadixTile - 1) / kRadixTile;
    Mark m(arena);
    uint32_t* hist = arena.take_n<uint32_t>(256 * tiles, "radix histogram");
    uint64_t* off = arena.take_n<uint64_t>(256 * tiles + 1, "radix offsets");
    bool in1 = false;
    for (int shift = 0; shift < bits; shift += 8) {
      const uint32_t* ks = in1 ? k1 : k0;
      const uint32_t* vs = in1 ? v1 : v0;
      k_radix_hist<<<(unsigned)tiles, kRadixThreads, 0, stream>>>(ks, n, shift, hist, tiles);
      CK(cudaGetLastError());
      scan(hist, true, 256 * tiles, off);
      k_radix_scatter<<<(unsigned)tiles, kRadixThreads, 0, stream>>>(ks, vs, n, shift, off, tiles, in1 ? k0 : k1, in1 ? v0 : v1);
      CK(cudaGetLastError());
      in1 = !in1;
    }
    return in1;
  }

  // The resident graph from the caller's (t_rp, t_ci), relabelled so that ids ascend
  // with degree (relabel.cuh), into g_rp / g_ci, with the caller-id map in g_new.
  void relabel_into_resident(const uint64_t* t_rp, const uint32_t* t_ci, uint64_t E) {
    auto bits_of = [](uint64_t x) {
      int b = 0;
      while (b < 64 && (x >> b)) b++;
      return b;
    };
    Mark m(arena);
    const uint64_t Vn = std::max<uint64_t>(V, 1);
    uint32_t* dk0 = arena.take_n<uint32_t>(Vn, "relabel degree keys");
    uint32_t* dv0 = arena.take_n<uint32_t>(Vn, "relabel ids");
    uint32_t* dk1 = arena.take_n<uint32_t>(Vn, "relabel degree keys");
    uint32_t* dv1 = arena.take_n<uint32_t>(Vn, "relabel ids");
    uint64_t* len = arena.take_n<uint64_t>(Vn, "relabel row lengths");
    unsigned long long* dmax = arena.take_n<unsigned long long>(1, "relabel max degree");
    CK(cudaMemsetAsync(dmax, 0, sizeof(unsigned long long), stream));
    k_degree_pairs<<<grid_threads(V), 256, 0, stream>>>(t_rp, V, dk0, dv0, dmax);
    CK(cudaGetLastError());
    const uint64_t dm = read_u64((const uint64_t*)dmax);
    if (dm >= 0xffffffffull) throw std::invalid_argument("relabel: a degree does not fit 32 bits");
    const uint32_t* order = radix_sort(dk0, dv0, dk1, dv1, V, bits_of(dm)) ? dv1 : dv0;
    k_invert_order<<<grid_threads(V), 256, 0, stream>>>(t_rp, order, V, g_new, len);
    CK(cudaGetLastError());
    scan(len, false, V, g_rp);
    const uint64_t En = std::max<uint64_t>(E, 1);
    uint32_t* ek0 = arena.take_n<uint32_t>(En, "relabel edge keys");
    uint32_t* ev0 = arena.take_n<uint32_t>(En, "relabel edge values");
    uint32_t* ek1 = arena.take_n<uint32_t>(En, "relabel edge keys");
    uint32_t* ev1 = arena.take_n<uint32_t>(En, "relabel edge values");
    k_emit_edges<<<grid_warps(V), 256, 0, stream>>>(t_rp, t_ci, order, g_new, g_rp, V, ek0, ev0);
    CK(cudaGetLastError());
    const uint32_t* sorted = radix_sort(ek0, ev0, ek1, ev1, E, bits_of(V - 1)) ? ev1 : ev0;
    if (E) CK(cudaMemcpyAsync(g_ci, sorted, sizeof(uint32_t) * E, cudaMemcpyDeviceToDevice, stream));
  }

  // largest b in (a, P] with unit * (off[b] - off[a]) + item * (b - a) <= budget;
  // at least a + 1 so that every call makes progress
  uint64_t split_point(const uint64_t* off, uint64_t a, uint64_t P, uint64_t unit, uint64_t item, uint64_t budget) {
    const uint64_t base = read_u64(off + a);
    auto cost = [&](uint64_t b) { return unit * (read_u64(off + b) - base) + item * (b - a); };
    if (cost(P) <= budget) return P;
    uint64_t lo = a + 1, hi = P;
    while (lo < hi) {
      uint64_t mid = lo + (hi - lo + 1) / 2;
      if (cost(mid) <= budget)
        lo = mid;
      else
        hi = mid - 1;
    }
    return lo;
  }

  // bytes this level may keep alive: the rest is left to the levels below,
  // like the reference's available / remaining-levels rule
  // (src/executor/processor.h:68-75)
  uint64_t level_budget(int i) const {
    const uint64_t reserve = std::min<uint64_t>(1 << 20, arena.cap / 64);
    const uint64_t avail = arena.avail() > reserve ? arena.avail() - reserve : 0;
    const int remaining = (int)plan->n_ops - i;
    const uint64_t share = avail / (uint64_t)std::max(2, remaining);
    // small arenas: keep making progress with at least 64 KB while it exists
    return std::max(share, std::min<uint64_t>(avail / 2, 1 << 16));
  }

  void begin_op() {
    if (profiling) CK(cudaEventRecord(ev0, stream));
  }
  void end_op(int i, uint64_t launches) {
    st->op_launches[i] += launches;
    if (profiling) {
      CK(cudaEventRecord(ev1, stream));
      CK(cudaEventSynchronize(ev1));
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, ev0, ev1));
      st->op_ms[i] += ms;
    }
  }

  OpDesc make_desc(int i, const vsgm_conds& conds) const {
    const vsgm_plan& p = *plan;
    OpDesc d;
    std::memset(&d, 0, sizeof(d));
    d.u = p.op_vertex[i];
    d.other = -1;
    d.merge_ratio = (uint16_t)cur.merge_ratio;
    d.lane_merge = cur.lane_merge ? 1 : 0;
    const vsgm_vgroup& mg = p.materialized[i];
    d.nm = mg.count;
    int slot[VSGM_MAX_QV];
    for (int k = 0; k < VSGM_MAX_QV; k++) slot[k] = 0;
    for (int k = 0; k < mg.count; k++) {
      d.m[k] = mg.v[k];
      slot[mg.v[k]] = k;
    }
    if (d.u < p.n_vertices) {
      const vsgm_vgroup& bg = p.backward[d.u];
      d.nb = bg.count;
      for (int k = 0; k < bg.count; k++) {
        d.b[k] = bg.v[k];
        d.bs[k] = (uint8_t)slot[bg.v[k]];
      }
    }
    d.nc = conds.count;
    for (int k = 0; k < conds.count; k++) {
      d.cop[k] = conds.op[k];
      d.cv[k] = conds.v[k];
      d.cs[k] = (uint8_t)slot[conds.v[k]];
    }
    return d;
  }

  // --------------------------------------------------------------- ops
  void process(int i, const Frame& f) {
    const vsgm_plan& p = *plan;
    if (i >= (int)p.n_ops || f.P == 0) return;
    st->op_paths[i] += f.P;
    const int type = p.op_type[i];
    const int u = p.op_vertex[i];
    switch (type) {
      case VSGM_COMPUTE_COUNT: op_compute_count(i, f); break;
      case VSGM_COUNT: op_count(i, f); break;
      case VSGM_COMPUTE: op_compute(i, f, u); break;
      case VSGM_FILTER_COMPUTE: op_filter(i, f, u); break;
      case VSGM_MATERIALIZE: op_materialize(i, f, u); break;
      case VSGM_COMPUTE_PATH_COUNT: op_path_count(i, f, u); break;
      default: throw OutOfMemory{"execution sequence holds an op this engine does not run"};
    }
  }

  static Frame slice(const Frame& f, uint64_t a, uint64_t b) {
    Frame g = f;
    g.P = b - a;
    for (int k = 0; k < VSGM_MAX_QV; k++) {
      if (g.col[k]) g.col[k] += a;
      if (g.cset[k]) g.cset[k] += a;
      if (g.clen[k]) g.clen[k] += a;
    }
    return g;
  }

  void op_compute_count(int i, const Frame& f) {
    const vsgm_plan& p = *plan;
    OpDesc d = make_desc(i, p.compute_cond[p.op_vertex[i]]);
    const vsgm_vgroup& cu = p.computed_unmat[i];
    bool other = cu.count == 1;
    if (other) {
      d.other = (int8_t)cu.v[0];
      d.other_op = p.order[d.u][cu.v[0]];
    }
    begin_op();
    launch_count(d, f, other);
    end_op(i, 1);
  }

  template <int NB>
  void launch_count_nb(const OpDesc& d, const Frame& f, bool other) {
    unsigned g = grid_warps(f.P);
    if (other) {
      if (profiling)
        k_compute_count<NB, true, true><<<g, 256, 0, stream>>>(f, d, d_rp, d_ci, d_total, d_bytes);
      else
        k_compute_count<NB, true, false><<<g, 256, 0, stream>>>(f, d, d_rp, d_ci, d_total, d_bytes);
    } else {
      if (profiling)
        k_compute_count<NB, false, true><<<g, 256, 0, stream>>>(f, d, d_rp, d_ci, d_total, d_bytes);
      else
        k_compute_count<NB, false, false><<<g, 256, 0, stream>>>(f, d, d_rp, d_ci, d_total, d_bytes);
    }
    CK(cudaGetLastError());
  }

  void launch_count(const OpDesc& d, const Frame& f, bool other) {
    switch (d.nb) {
      case 1: launch_count_nb<1>(d, f, other); break;
      case 2: launch_count_nb<2>(d, f, other); break;
      case 3: launch_count_nb<3>(d, f, other); break;
      case 4: launch_count_nb<4>(d, f, other); break;
      case 5: launch_count_nb<5>(d, f, other); break;
      case 6: launch_count_nb<6>(d, f, other); break;
      default: throw OutOfMemory{"pattern vertex with no backward neighbour"};
    }
  }

  void op_count(int i, const Frame& f) {
    const vsgm_plan& p = *plan;
    const vsgm_vgroup& cu = p.computed_unmat[i];
    begin_op();
    if (cu.count == 1) {
      k_count_one<<<grid_threads(f.P), 256, 0, stream>>>(f, cu.v[0], d_total);
    } else {
      k_count_two<<<grid_warps(f.P), 256, 0, stream>>>(f, cu.v[0], cu.v[1], p.order[cu.v[0]][cu.v[1]], d_total);
    }
    CK(cudaGetLastError());
    end_op(i, 1);
  }

  template <int NB>
  void launch_write_nb(const OpDesc& d, const Frame& f, const uint64_t* off, uint32_t* pool, uint64_t* set, uint32_t* len) {
    k_compute_write<NB><<<grid_warps(f.P), 256, 0, stream>>>(f, d, d_rp, d_ci, off, pool, set, len);
  }

  // Apply conditions to one sorted set per path (the adjacency list of the single
  // backward neighbour, or the frame's candidates of u), copying only the sets
  // that contain a NON_EQUAL value; then hand the narrowed frame to `next`.
  template <typename Next>
  void narrow_then(int i, const Frame& f, const OpDesc& d, bool from_adj, int u, Next&& next) {
    const uint64_t per = 8 + 4 + 8;  // set address, length, copy bound / offset
    uint64_t a = 0, cap_paths = ~0ull;
    while (a < f.P) {
      uint64_t room = std::min(cap_paths, level_budget(i) / (per + 4));
      if (room == 0) throw OutOfMemory{"HBM budget exhausted (narrow)"};
      uint64_t b = std::min(f.P, a + room);
      Mark m(arena);
      Frame g = slice(f, a, b);
      uint64_t* set = arena.take_n<uint64_t>(g.P, "candidate sets");
      uint32_t* len = arena.take_n<uint32_t>(g.P, "candidate lengths");
      uint64_t* off = arena.take_n<uint64_t>(g.P + 1, "copy offsets");
      begin_op();
      CK(cudaMemsetAsync(d_bytes + 1, 0, sizeof(unsigned long long), stream));
      if (from_adj)
        k_narrow<true><<<grid_threads(g.P), 256, 0, stream>>>(g, d, d_rp, d_ci, set, len, off, d_bytes + 1);
      else
        k_narrow<false><<<grid_threads(g.P), 256, 0, stream>>>(g, d, d_rp, d_ci, set, len, off, d_bytes + 1);
      CK(cudaGetLastError());
      scan(off, false, g.P, off);
      end_op(i, 3);
      st->op_outputs[i] += read_u64((const uint64_t*)(d_bytes + 1));
      const uint64_t copy = read_u64(off + g.P);
      if (copy && 4 * copy + 4096 > arena.avail() && g.P > 1) {
        // the copies of this slice do not fit: retry with half the paths
        st->op_outputs[i] -= read_u64((const uint64_t*)(d_bytes + 1));
        cap_paths = std::max<uint64_t>(1, g.P / 2);
        continue;
      }
      if (copy) {
        uint32_t* pool = arena.take_n<uint32_t>(copy, "copied candidates");
        begin_op();
        k_copy_marked<<<grid_warps(g.P), 256, 0, stream>>>(g, d, off, pool, set, len);
        CK(cudaGetLastError());
        end_op(i, 1);
      }
      g.cset[u] = set;
      g.clen[u] = len;
      st->batches++;
      next(g);
      a = b;
    }
  }

  // COMPUTE(o) followed by the final COMPUTE_COUNT(w) counted against o, with the
  // same backward lists and the same conditions on the same materialised vertices:
  // both candidate sets are one set S, and the count per path is the number of
  // pairs of S the condition between w and o admits
  int same_set_pairs(int i, int o) const {
    const vsgm_plan& p = *plan;
    if (!cur.set_reuse || i + 1 != (int)p.n_ops - 1 || p.op_type[i + 1] != VSGM_COMPUTE_COUNT) return 0;
    const int w = p.op_vertex[i + 1];
    const vsgm_vgroup& cu = p.computed_unmat[i + 1];
    if (cu.count != 1 || cu.v[0] != o) return 0;
    if (p.materialized[i].count != p.materialized[i + 1].count) return 0;
    const vsgm_vgroup &bw = p.backward[w], &bo = p.backward[o];
    if (bw.count != bo.count) return 0;
    for (int k = 0; k < bw.count; k++)
      if (bw.v[k] != bo.v[k]) return 0;
    const vsgm_conds &cw = p.compute_cond[w], &co = p.compute_cond[o];
    if (cw.count != co.count) return 0;
    for (int k = 0; k < cw.count; k++)
      if (cw.v[k] != co.v[k] || cw.op[k] != co.op[k]) return 0;
    const uint8_t rel = p.order[w][o];
    return (rel == VSGM_LESS_THAN || rel == VSGM_LARGER_THAN) ? 1 : (rel == VSGM_NON_EQUAL ? 2 : 0);
  }

  void op_compute(int i, const Frame& f, int u) {
    const vsgm_plan& p = *plan;
    OpDesc d = make_desc(i, p.compute_cond[u]);
    if (const int mode = same_set_pairs(i, u)) {
      begin_op();
      switch (d.nb) {
#define VSGM_PAIRS(NB)                                                                                              \
  case NB:                                                                                                          \
    k_compute_count<NB, false, false><<<grid_warps(f.P), 256, 0, stream>>>(f, d, d_rp, d_ci, d_total, d_bytes, mode); \
    break;
        VSGM_PAIRS(1)
        VSGM_PAIRS(2)
        VSGM_PAIRS(3)
        VSGM_PAIRS(4)
        VSGM_PAIRS(5)
        VSGM_PAIRS(6)
#undef VSGM_PAIRS
        default: throw OutOfMemory{"pattern vertex with no backward neighbour"};
      }
      CK(cudaGetLastError());
      end_op(i + 1, 1);
      st->op_paths[i + 1] += f.P;
      return;
    }
    if (d.nb == 1) {
      narrow_then(i, f, d, true, u, [&](const Frame& g) { process(i + 1, g); });
      return;
    }
    // general case: size, scan, write
    Mark m(arena);
    uint64_t* off = arena.take_n<uint64_t>(f.P + 1, "candidate offsets");
    begin_op();
    k_compute_size<<<grid_warps(f.P), 256, 0, stream>>>(f, d, d_rp, d_ci, off);
    CK(cudaGetLastError());
    scan(off, false, f.P, off);
    end_op(i, 3);
    uint64_t a = 0;
    while (a < f.P) {
      // each path needs a set address, a length and 4 bytes per candidate
      uint64_t b = split_point(off, a, f.P, 4, 12, level_budget(i));
      Mark mb(arena);
      Frame g = slice(f, a, b);
      uint64_t lo = read_u64(off + a), hi = read_u64(off + b);
      uint32_t* pool = arena.take_n<uint32_t>(hi - lo, "candidate pool");
      uint64_t* set = arena.take_n<uint64_t>(g.P, "candidate sets");
      uint32_t* len = arena.take_n<uint32_t>(g.P, "candidate lengths");
      uint32_t* pool_eff = pool - lo;  // pool_eff + off[p] lies inside pool
      begin_op();
      switch (d.nb) {
        case 2: launch_write_nb<2>(d, g, off + a, pool_eff, set, len); break;
        case 3: launch_write_nb<3>(d, g, off + a, pool_eff, set, len); break;
        case 4: launch_write_nb<4>(d, g, off + a, pool_eff, set, len); break;
        case 5: launch_write_nb<5>(d, g, off + a, pool_eff, set, len); break;
        case 6: launch_write_nb<6>(d, g, off + a, pool_eff, set, len); break;
        default: throw OutOfMemory{"pattern vertex with no backward neighbour"};
      }
      CK(cudaGetLastError());
      end_op(i, 1);
      st->op_outputs[i] += hi - lo;
      g.cset[u] = set;
      g.clen[u] = len;
      st->batches++;
      process(i + 1, g);
      a = b;
    }
  }

  // COMPUTE_PATH_COUNT: only the size of every path's candidate set of u; the set
  // addresses stay zero (plans are checked at vsgm_create: no later op reads them)
  void op_path_count(int i, const Frame& f, int u) {
    const vsgm_plan& p = *plan;
    OpDesc d = make_desc(i, p.compute_cond[u]);
    uint64_t a = 0;
    while (a < f.P) {
      const uint64_t room = std::max<uint64_t>(1, level_budget(i) / 12);
      const uint64_t b = std::min(f.P, a + room);
      Mark m(arena);
      Frame g = slice(f, a, b);
      uint64_t* set = arena.take_n<uint64_t>(g.P, "candidate sets");
      uint32_t* len = arena.take_n<uint32_t>(g.P, "candidate sizes");
      CK(cudaMemsetAsync(set, 0, sizeof(uint64_t) * g.P, stream));
      begin_op();
      switch (d.nb) {
#define VSGM_PATHS(NB) \
  case NB: k_path_count<NB><<<grid_warps(g.P), 256, 0, stream>>>(g, d, d_rp, d_ci, len); break;
        VSGM_PATHS(1)
        VSGM_PATHS(2)
        VSGM_PATHS(3)
        VSGM_PATHS(4)
        VSGM_PATHS(5)
        VSGM_PATHS(6)
#undef VSGM_PATHS
        default: throw OutOfMemory{"pattern vertex with no backward neighbour"};
      }
      CK(cudaGetLastError());
      end_op(i, 1);
      g.cset[u] = set;
      g.clen[u] = len;
      st->batches++;
      process(i + 1, g);
      a = b;
    }
  }

  // FILTER_COMPUTE keeps the candidates of u that satisfy the filter conditions
  void op_filter(int i, const Frame& f, int u) {
    OpDesc d = make_desc(i, plan->filter_cond[u]);
    d.u = (uint8_t)u;
    narrow_then(i, f, d, false, u, [&](const Frame& g) { process(i + 1, g); });
  }

  void op_materialize(int i, const Frame& f, int u) {
    const vsgm_plan& p = *plan;
    const bool fuse = fusable(i, u);
    auto next = [&](const Frame& g) {
      if (fuse)
        fused_count(i, g, u);
      else
        materialize_frame(i, g, u);
    };
    if (p.materialize_cond[u].count > 0) {
      OpDesc d = make_desc(i, p.materialize_cond[u]);
      d.u = (uint8_t)u;
      narrow_then(i, f, d, false, u, next);
    } else {
      next(f);
    }
  }

  // MATERIALIZE(u) directly followed by the final COMPUTE_COUNT(w), u one of w's
  // backward neighbours: count without expanding the children
  bool fusable(int i, int u) const {
    const vsgm_plan& p = *plan;
    if (!cur.fuse_tail || i + 1 != (int)p.n_ops - 1 || p.op_type[i + 1] != VSGM_COMPUTE_COUNT) return false;
    const int w = p.op_vertex[i + 1];
    const vsgm_vgroup& B = p.backward[w];
    bool has_u = false;
    for (int k = 0; k < B.count; k++) has_u |= (B.v[k] == u);
    if (!has_u || B.count < 2 || B.count > 6) return false;
    if (p.computed_unmat[i + 1].count > 1) return false;
    int on_u = 0;
    for (int k = 0; k < p.compute_cond[w].count; k++) on_u += (p.compute_cond[w].v[k] == u);
    return on_u <= 1;
  }

  void fused_count(int i, const Frame& f, int u) {
    const vsgm_plan& p = *plan;
    const int w = p.op_vertex[i + 1];
    FusedDesc fd;
    std::memset(&fd, 0, sizeof(fd));
    // the known part: materialised[i] columns, B(w) minus u, conditions not on u
    vsgm_conds known;
    std::memset(&known, 0, sizeof(known));
    const vsgm_conds& cc = p.compute_cond[w];
    for (int k = 0; k < cc.count; k++) {
      if (cc.v[k] == u) {
        fd.has_cond_u = 1;
        fd.cond_u_op = cc.op[k];
      } else {
        known.op[known.count] = cc.op[k];
        known.v[known.count++] = cc.v[k];
      }
    }
    fd.known = make_desc(i, known);
    fd.known.u = (uint8_t)w;
    {
      const vsgm_vgroup& B = p.backward[w];
      int slot[VSGM_MAX_QV] = {0};
      for (int k = 0; k < p.materialized[i].count; k++) slot[p.materialized[i].v[k]] = k;
      fd.known.nb = 0;
      for (int k = 0; k < B.count; k++)
        if (B.v[k] != u) {
          fd.known.b[fd.known.nb] = B.v[k];
          fd.known.bs[fd.known.nb++] = (uint8_t)slot[B.v[k]];
        }
    }
    fd.u = (uint8_t)u;
    fd.stage_cap = cur.stage_cap;
    fd.walk_ratio = cur.walk_ratio;
    fd.lane_slice = cur.lane_slice;
    fd.up = (fd.has_cond_u && fd.cond_u_op == VSGM_LARGER_THAN) ? upper_offsets() : nullptr;
    fd.other = -1;
    const vsgm_vgroup& cu = p.computed_unmat[i + 1];
    if (cu.count == 1) {
      fd.other = (int8_t)cu.v[0];
      fd.other_op = p.order[w][cu.v[0]];
    }
    // children count, for the statistics
    CK(cudaMemsetAsync(d_bytes + 1, 0, sizeof(unsigned long long), stream));
    k_count_one<<<grid_threads(f.P), 256, 0, stream>>>(f, (uint8_t)u, d_bytes + 1);
    CK(cudaGetLastError());
    const uint64_t children = read_u64((const uint64_t*)(d_bytes + 1));
    st->op_outputs[i] += children;
    st->op_paths[i + 1] += children;
    begin_op();
    const unsigned g = grid_warps(f.P);
    const bool other = fd.other >= 0;
    const bool merge = cur.tail_merge;
    switch (fd.known.nb) {
#define VSGM_FUSED(NK)                                                                          \
  case NK:                                                                                      \
    if (other && merge)                                                                         \
      k_mat_count<NK, true, true><<<g, 256, 0, stream>>>(f, fd, d_rp, d_ci, d_total, d_bytes);  \
    else if (other)                                                                             \
      k_mat_count<NK, true><<<g, 256, 0, stream>>>(f, fd, d_rp, d_ci, d_total, d_bytes);        \
    else if (merge)                                                                             \
      k_mat_count<NK, false, true><<<g, 256, 0, stream>>>(f, fd, d_rp, d_ci, d_total, d_bytes); \
    else                                                                                        \
      k_mat_count<NK, false><<<g, 256, 0, stream>>>(f, fd, d_rp, d_ci, d_total, d_bytes);       \
    break;
      VSGM_FUSED(1)
      VSGM_FUSED(2)
      VSGM_FUSED(3)
      VSGM_FUSED(4)
      VSGM_FUSED(5)
#undef VSGM_FUSED
      default: throw OutOfMemory{"unsupported fused op shape"};
    }
    CK(cudaGetLastError());
    end_op(i + 1, 1);
  }

  void materialize_frame(int i, const Frame& f, int u) {
    const vsgm_plan& p = *plan;
    const vsgm_vgroup& mg = p.materialized[i];
    const vsgm_vgroup& cg = p.computed_unmat[i];
    Expand x;
    std::memset(&x, 0, sizeof(x));
    x.u = (uint8_t)u;
    x.nm = mg.count;
    for (int k = 0; k < mg.count; k++) x.m[k] = mg.v[k];
    for (int k = 0; k < cg.count; k++)
      if (cg.v[k] != u) x.cu[x.ncu++] = cg.v[k];
    const uint64_t child_bytes = 4ull * (x.nm + 1) + 12ull * x.ncu;
    Mark m(arena);
    uint64_t* off = arena.take_n<uint64_t>(f.P + 1, "children offsets");
    begin_op();
    scan(f.clen[u], true, f.P, off);
    end_op(i, 2);
    const uint64_t C = read_u64(off + f.P);
    st->op_outputs[i] += C;
    uint64_t c0 = 0;
    while (c0 < C) {
      uint64_t n = std::min(C - c0, level_budget(i) / (child_bytes + 8));
      if (n == 0) throw OutOfMemory{"HBM budget exhausted (MATERIALIZE)"};
      Mark mb(arena);
      Frame g;
      std::memset(&g, 0, sizeof(g));
      g.P = n;
      for (int k = 0; k < x.nm; k++) g.col[x.m[k]] = arena.take_n<uint32_t>(n, "child column");
      g.col[u] = arena.take_n<uint32_t>(n, "child column");
      for (int k = 0; k < x.ncu; k++) {
        g.cset[x.cu[k]] = arena.take_n<uint64_t>(n, "child candidate sets");
        g.clen[x.cu[k]] = arena.take_n<uint32_t>(n, "child candidate lengths");
      }
      // k_expand writes children [c0, c0+n) at positions [0, n): shift the outputs
      Frame shifted = g;
      for (int k = 0; k < VSGM_MAX_QV; k++) {
        if (shifted.col[k]) shifted.col[k] -= c0;
        if (shifted.cset[k]) shifted.cset[k] -= c0;
        if (shifted.clen[k]) shifted.clen[k] -= c0;
      }
      begin_op();
      launch_expand(f, x, off, c0, n, shifted);
      end_op(i, 1);
      st->batches++;
      process(i + 1, g);
      c0 += n;
    }
  }

  void launch_expand(const Frame& in, const Expand& x, const uint64_t* off, uint64_t c0, uint64_t n, const Frame& out) {
    k_expand<<<grid_threads(n), 256, 0, stream>>>(in, x, off, c0, c0 + n, out);
    CK(cudaGetLastError());
  }

  // the pattern is a 4-cycle: four vertices, four edges, every vertex of degree two
  static bool is_four_cycle(const vsgm_plan& p) {
    if (p.n_vertices != 4 || p.n_edges != 4) return false;
    for (int i = 0; i < 4; i++)
      if (__builtin_popcount(p.adj[i]) != 2) return false;
    return true;
  }

  // 4-cycles rooted at the given sources, by wedge aggregation; each cycle is
  // attributed to its largest vertex, the plan attributes it to its smallest:
  // totals over all sources are the same.  Roots with at least c4_heavy wedges
  // (most of the work on skewed graphs; default 12289) go through the L2-resident
  // group kernels; the others through shared-memory hash tables (knob c4_hash: a
  // warp per root up to 768 wedges, a block per root up to 12288), and whatever is
  // left through k_c4_aggregate (one root per block, dense counters in HBM).
  void c4_aggregate(const uint32_t* roots, uint64_t n) {
    const int last = (int)plan->n_ops - 1;
    Mark m(arena);
    begin_op();
    // split the roots by wedge count
    unsigned long long* W = arena.take_n<unsigned long long>(V, "4-cycle wedge counts");
    uint32_t* heavy = arena.take_n<uint32_t>(std::max<uint64_t>(n, 1), "4-cycle heavy roots");
    uint64_t* centres = arena.take_n<uint64_t>(std::max<uint64_t>(n, 1), "4-cycle wedge centres");
    uint32_t* light = arena.take_n<uint32_t>(std::max<uint64_t>(n, 1), "4-cycle light roots");
    unsigned long long* ctr = arena.take_n<unsigned long long>(2, "4-cycle split counters");
    CK(cudaMemsetAsync(W, 0, V * sizeof(unsigned long long), stream));
    CK(cudaMemsetAsync(ctr, 0, 2 * sizeof(unsigned long long), stream));
    k_c4_wedge_counts<<<grid_warps(V), 256, 0, stream>>>(d_rp, d_ci, V, W);
    k_c4_split<<<grid_threads(n), 256, 0, stream>>>(d_rp, d_ci, roots, n, W, cur.c4_heavy, heavy, centres, light, ctr, profiling ? d_bytes : nullptr);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h_pinned, ctr, 2 * sizeof(uint64_t), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    const uint64_t n_heavy = h_pinned[0];
    uint64_t n_light = h_pinned[1];
    uint64_t launches = 2;
    if (n_light && cur.c4_hash) {
      // light roots with few wedges: counters in shared-memory hash tables
      uint32_t* hw = arena.take_n<uint32_t>(n_light, "4-cycle hashed roots");
      uint32_t* hb = arena.take_n<uint32_t>(n_light, "4-cycle hashed roots");
      uint32_t* rest = arena.take_n<uint32_t>(n_light, "4-cycle light roots");
      unsigned long long* hc = arena.take_n<unsigned long long>(4, "4-cycle hash counters");
      CK(cudaMemsetAsync(hc, 0, 4 * sizeof(unsigned long long), stream));
      k_c4_split_light<<<grid_threads(n_light), 256, 0, stream>>>(light, n_light, W, kC4HashWarpMaxW, kC4HashBlockMaxW, hw, hb, rest, hc);
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(h_pinned, hc, 3 * sizeof(uint64_t), cudaMemcpyDeviceToHost, stream));
      CK(cudaStreamSynchronize(stream));
      const uint64_t nw = h_pinned[0], nb = h_pinned[1];
      const uint32_t* up = upper_offsets();
      if (nb) {
        k_c4_hash_block<<<(unsigned)sms, 512, kC4HashBlockSmem, stream>>>(d_rp, d_ci, up, hb, nb, hc + 3, d_total);
        launches++;
      }
      if (nw) {
        k_c4_hash_warp<<<(unsigned)sms * 2, kC4HashWarps * kWarp, kC4HashWarpSmem, stream>>>(d_rp, d_ci, up, hw, nw, d_total);
        launches++;
      }
      CK(cudaGetLastError());
      light = rest;
      n_light = h_pinned[2];
    }
    if (n_light) {
      launches++;
      const uint64_t per_block = 2ull * V * sizeof(uint32_t);
      uint64_t blocks = std::min<uint64_t>((uint64_t)sms * 4, (arena.avail() > (1u << 20) ? arena.avail() - (1u << 20) : 0) / per_block);
      if (blocks == 0) throw OutOfMemory{"HBM budget exhausted (4-cycle counters)"};
      blocks = std::min<uint64_t>(blocks, n_light);
      Mark ml(arena);
      uint32_t* L = arena.take_n<uint32_t>(blocks * V, "4-cycle counters");
      uint32_t* touched = arena.take_n<uint32_t>(blocks * V, "4-cycle touched ids");
      unsigned long long* head = arena.take_n<unsigned long long>(1, "4-cycle queue head");
      CK(cudaMemsetAsync(L, 0, blocks * V * sizeof(uint32_t), stream));
      CK(cudaMemsetAsync(head, 0, sizeof(unsigned long long), stream));
      k_c4_aggregate<<<(unsigned)blocks, 256, 0, stream>>>(d_rp, d_ci, light, n_light, V, L, touched, head, d_total);
      CK(cudaGetLastError());
    }
    if (n_heavy) {
      std::vector<uint32_t> hr(n_heavy);
      std::vector<uint64_t> hc(n_heavy);
      CK(cudaMemcpyAsync(hr.data(), heavy, n_heavy * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
      CK(cudaMemcpyAsync(hc.data(), centres, n_heavy * sizeof(uint64_t), cudaMemcpyDeviceToHost, stream));
      CK(cudaStreamSynchronize(stream));
      // groups of up to kC4Group roots whose counter arrays fit in about 96 MB (L2):
      // two buffers of 48 MB on two streams, so that one group's sum pass runs while
      // the next group adds its wedges; 16-bit counters for roots with fewer than
      // 65536 neighbours below them (no counter can exceed that), 32-bit for the rest
      std::vector<uint32_t> pr, wr, win_roots;
      std::vector<uint64_t> pc, wc;
      std::vector<uint32_t> plim, wlim;
      for (uint64_t k = 0; k < n_heavy; k++) {
        if (hc[k] < 65536) {
          // with the window on, the ids [u - kC4Window, u) are counted by the cluster kernel
          const uint32_t lim = cur.c4_window ? (hr[k] > kC4Window ? hr[k] - kC4Window : 0u) : hr[k];
          if (cur.c4_window) win_roots.push_back(hr[k]);
          if (lim == 0) continue;
          pr.push_back(hr[k]);
          pc.push_back(hc[k]);
          plim.push_back(lim);
        } else {
          wr.push_back(hr[k]);
          wc.push_back(hc[k]);
          wlim.push_back(hr[k]);
        }
      }
      if (!win_roots.empty()) {
        Mark mw(arena);
        uint32_t* d_win = arena.take_n<uint32_t>(win_roots.size(), "4-cycle window roots");
        unsigned long long* whead = arena.take_n<unsigned long long>(1, "4-cycle window queue");
        CK(cudaMemcpyAsync(d_win, win_roots.data(), win_roots.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        CK(cudaMemsetAsync(whead, 0, sizeof(unsigned long long), stream));
        const unsigned clusters = std::max(1, sms / kC4WinCtas);
        k_c4_window<<<clusters * kC4WinCtas, 512, kC4WinSmem, stream>>>(d_rp, d_ci, d_win, win_roots.size(), whead, d_total);
        CK(cudaGetLastError());
        launches++;
      }
      const uint64_t stride_p = (((V + 1) / 2) + 3) & ~3ull, stride_w = (V + 3) & ~3ull;  // words per root
      const uint64_t buf = 48ull << 20;
      const int Gp = (int)std::max<uint64_t>(1, std::min<uint64_t>(kC4Group, buf / (stride_p * 4)));
      const int Gw = (int)std::max<uint64_t>(1, std::min<uint64_t>(kC4Group, buf / (stride_w * 4)));
      std::vector<C4Group> groups;
      std::vector<uint8_t> packed;
      uint64_t n_centres = 0;  // centres of all groups, in group order (the balanced kernel's prefix)
      auto make_groups = [&](const std::vector<uint32_t>& r, const std::vector<uint64_t>& c, const std::vector<uint32_t>& lim, int G, bool pk) {
        for (uint64_t k = 0; k < r.size(); k += G) {
          C4Group g;
          std::memset(&g, 0, sizeof(g));
          g.n = (uint32_t)std::min<uint64_t>(G, r.size() - k);
          for (uint32_t i = 0; i < g.n; i++) {
            g.root[i] = r[k + i];
            g.lim[i] = lim[k + i];
            g.vbeg[i + 1] = g.vbeg[i] + c[k + i];
          }
          g.cbase = n_centres;
          n_centres += g.vbeg[g.n];
          groups.push_back(g);
          packed.push_back(pk ? 1 : 0);
        }
      };
      make_groups(pr, pc, plim, Gp, true);
      make_groups(wr, wc, wlim, Gw, false);
      const uint64_t words = std::max((uint64_t)Gp * stride_p, (uint64_t)Gw * stride_w);
      if (!groups.empty()) {
        C4Group* d_groups = arena.take_n<C4Group>(groups.size(), "4-cycle groups");
        uint32_t* Lbuf[2] = {arena.take_n<uint32_t>(words, "4-cycle group counters"), arena.take_n<uint32_t>(words, "4-cycle group counters")};
        CK(cudaMemcpyAsync(d_groups, groups.data(), groups.size() * sizeof(C4Group), cudaMemcpyHostToDevice, stream));
        CK(cudaMemsetAsync(Lbuf[0], 0, words * sizeof(uint32_t), stream));
        CK(cudaMemsetAsync(Lbuf[1], 0, words * sizeof(uint32_t), stream));
        uint64_t* P = nullptr;
        if (cur.c4_balance) {
          // prefix of every centre's row length, the entry space the balanced kernel splits
          uint32_t* deg = arena.take_n<uint32_t>(n_centres + 1, "4-cycle centre degrees");
          P = arena.take_n<uint64_t>(n_centres + 1, "4-cycle centre prefix");
          k_c4_centre_degrees<<<(unsigned)groups.size(), 256, 0, stream>>>(d_rp, d_ci, d_groups, deg);
          CK(cudaGetLastError());
          scan(deg, true, n_centres, P);
          launches += 1;
        }
        CK(cudaEventRecord(ev_fork, stream));
        CK(cudaStreamWaitEvent(aux_stream, ev_fork, 0));
        const unsigned gw = (unsigned)sms * 8, gs = (unsigned)sms * 4;
        for (size_t i = 0; i < groups.size(); i++) {
          cudaStream_t st2 = (i & 1) ? aux_stream : stream;  // group i uses buffer i % 2 on stream i % 2
          uint32_t* L = Lbuf[i & 1];
          if (packed[i]) {
            if (P)
              k_c4_group_wedges_bal<true><<<gw, 256, 0, st2>>>(d_rp, d_ci, d_groups + i, P, L, stride_p);
            else
              k_c4_group_wedges<true><<<gw, 256, 0, st2>>>(d_rp, d_ci, d_groups + i, L, stride_p);
            k_c4_group_sum<true><<<gs, 256, 0, st2>>>(d_groups + i, L, stride_p, d_total);
          } else {
            if (P)
              k_c4_group_wedges_bal<false><<<gw, 256, 0, st2>>>(d_rp, d_ci, d_groups + i, P, L, stride_w);
            else
              k_c4_group_wedges<false><<<gw, 256, 0, st2>>>(d_rp, d_ci, d_groups + i, L, stride_w);
            k_c4_group_sum<false><<<gs, 256, 0, st2>>>(d_groups + i, L, stride_w, d_total);
          }
        }
        CK(cudaEventRecord(ev_join, aux_stream));
        CK(cudaStreamWaitEvent(stream, ev_join, 0));
        launches += 2 * groups.size();
      }
      CK(cudaGetLastError());
    }
    end_op(last, launches);
    st->op_paths[last] += n;
  }

  // k when the plan counts k-cliques at their smallest vertex: a complete pattern
  // whose LARGER_THAN / LESS_THAN conditions order every pair of vertices (their
  // transitive closure is a strict total order) with the root first; else 0
  static int clique_order(const vsgm_plan& p) {
    const int n = (int)p.n_vertices;
    if (n < 3 || n > VSGM_MAX_QV || p.n_edges != (uint32_t)(n * (n - 1) / 2)) return 0;
    bool less[VSGM_MAX_QV][VSGM_MAX_QV] = {};  // less[a][b]: a < b
    auto take = [&](int u, const vsgm_conds& c) {
      for (int k = 0; k < c.count; k++) {
        if (c.op[k] == VSGM_LARGER_THAN) less[c.v[k]][u] = true;
        if (c.op[k] == VSGM_LESS_THAN) less[u][c.v[k]] = true;
      }
    };
    for (int u = 0; u < n; u++) {
      take(u, p.compute_cond[u]);
      take(u, p.materialize_cond[u]);
      take(u, p.filter_cond[u]);
    }
    for (int k = 0; k < n; k++)
      for (int a = 0; a < n; a++)
        for (int b = 0; b < n; b++) less[a][b] |= less[a][k] && less[k][b];
    const int root = p.op_vertex[0];
    for (int a = 0; a < n; a++) {
      if (less[a][a]) return 0;
      for (int b = 0; b < n; b++)
        if (a != b && !(less[a][b] || less[b][a])) return 0;
      if (a != root && !less[root][a]) return 0;
    }
    return n;
  }

  // k-cliques (k = 3, 4) at the given roots by the bitmap operator (clique.cuh);
  // roots whose out-neighbourhood is wider than its block tier run the plan.
  void clique_bits(const uint32_t* roots, uint64_t n, int K) {
    const int last = (int)plan->n_ops - 1;
    const uint32_t* up = upper_offsets();
    Mark m(arena);
    begin_op();
    CliqueTiers t;
    for (int k = 0; k < 4; k++) t.root[k] = arena.take_n<uint32_t>(std::max<uint64_t>(n, 1), "clique tier roots");
    t.count = arena.take_n<unsigned long long>(6, "clique tier counters");  // 4 tiers + 2 queue heads
    CK(cudaMemsetAsync(t.count, 0, 6 * sizeof(unsigned long long), stream));
    k_clique_split<<<grid_threads(n), 256, 0, stream>>>(d_rp, up, roots, n, (uint32_t)(K - 1), kCliqueSmall, kCliqueMid, kCliqueLarge, t);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h_pinned, t.count, 4 * sizeof(uint64_t), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    const uint64_t nt[4] = {h_pinned[0], h_pinned[1], h_pinned[2], h_pinned[3]};
    unsigned long long* bytes = profiling ? d_bytes : nullptr;
    uint64_t launches = 1;
    if (nt[2]) {
      if (K == 3)
        k_clique_large<3><<<(unsigned)sms, kCliqueLargeWarps * kWarp, kCliqueLargeSmem, stream>>>(d_rp, d_ci, up, t.root[2], nt[2], t.count + 4, d_total, bytes);
      else
        k_clique_large<4><<<(unsigned)sms, kCliqueLargeWarps * kWarp, kCliqueLargeSmem, stream>>>(d_rp, d_ci, up, t.root[2], nt[2], t.count + 4, d_total, bytes);
      launches++;
    }
    if (nt[1]) {
      if (K == 3)
        k_clique_mid<3><<<(unsigned)sms * 2, kCliqueMidWarps * kWarp, kCliqueMidSmem, stream>>>(d_rp, d_ci, up, t.root[1], nt[1], t.count + 5, d_total, bytes);
      else
        k_clique_mid<4><<<(unsigned)sms * 2, kCliqueMidWarps * kWarp, kCliqueMidSmem, stream>>>(d_rp, d_ci, up, t.root[1], nt[1], t.count + 5, d_total, bytes);
      launches++;
    }
    if (nt[0]) {
      if (K == 3)
        k_clique_small<3><<<grid_warps(nt[0]), 256, 0, stream>>>(d_rp, d_ci, up, t.root[0], nt[0], d_total, bytes);
      else
        k_clique_small<4><<<grid_warps(nt[0]), 256, 0, stream>>>(d_rp, d_ci, up, t.root[0], nt[0], d_total, bytes);
      launches++;
    }
    CK(cudaGetLastError());
    end_op(last, launches);
    st->op_paths[last] += n;
    if (nt[3]) {
      // the widest out-neighbourhoods: the level-wise plan on those roots
      Frame f;
      std::memset(&f, 0, sizeof(f));
      f.P = nt[3];
      f.col[plan->op_vertex[0]] = t.root[3];
      process(1, f);
    }
  }

  // Pair mode (1: C(t, 2), 2: t (t - 1)) when the plan is M(a) C(b) M(b) C(o) CC(w)
  // with b > a the only condition on b, o and w both drawn from N(a) and N(b) with no
  // conditions but "differs from a / b" (which a common neighbour always does), and
  // o, w ordered or distinct: the diamond of pm_pipeline -p 2.  Its count at root a
  // is the sum over edges (a, b), b > a, of the pairs of their t(a, b) common
  // neighbours.  Else 0.
  static int diamond_mode(const vsgm_plan& p) {
    if (p.n_vertices != 4 || p.n_edges != 5 || p.n_ops != 5) return 0;
    const int want[5] = {VSGM_MATERIALIZE, VSGM_COMPUTE, VSGM_MATERIALIZE, VSGM_COMPUTE, VSGM_COMPUTE_COUNT};
    for (int i = 0; i < 5; i++)
      if (p.op_type[i] != want[i]) return 0;
    const int a = p.op_vertex[0], b = p.op_vertex[1], o = p.op_vertex[3], w = p.op_vertex[4];
    if (p.op_vertex[2] != b || a == b || o == w || o == a || o == b || w == a || w == b) return 0;
    if (p.backward[b].count != 1 || p.backward[b].v[0] != a) return 0;
    if (p.compute_cond[b].count != 1 || p.compute_cond[b].op[0] != VSGM_LARGER_THAN || p.compute_cond[b].v[0] != a) return 0;
    if (p.materialize_cond[b].count || p.materialize_cond[a].count) return 0;
    for (int x : {o, w}) {
      const vsgm_vgroup& B = p.backward[x];
      if (B.count != 2 || !((B.v[0] == a && B.v[1] == b) || (B.v[0] == b && B.v[1] == a))) return 0;
      const vsgm_conds& c = p.compute_cond[x];
      for (int k = 0; k < c.count; k++)
        if (c.op[k] != VSGM_NON_EQUAL || (c.v[k] != a && c.v[k] != b)) return 0;
    }
    if (p.computed_unmat[4].count != 1 || p.computed_unmat[4].v[0] != o) return 0;
    const uint8_t rel = p.order[w][o];
    return (rel == VSGM_LESS_THAN || rel == VSGM_LARGER_THAN) ? 1 : (rel == VSGM_NON_EQUAL ? 2 : 0);
  }

  // The diamond plan at the given roots from per-edge triangle counts (clique.cuh):
  // the triangles with their smallest vertex among the roots or their neighbours
  // below them are found once each and added to the slots of their three edges, then
  // every root sums the pairs over its out-edges.  A view with an out-neighbourhood
  // wider than the block tier runs the plan instead.
  void diamond_edges(const uint32_t* roots, uint64_t n, int mode) {
    const int last = (int)plan->n_ops - 1;
    const uint32_t* up = upper_offsets();
    Mark m(arena);
    begin_op();
    uint8_t* flags = (uint8_t*)arena.take_n<uint32_t>((V + 3) / 4 + 1, "triangle root flags");
    uint8_t* is_src = (uint8_t*)arena.take_n<uint32_t>((V + 3) / 4 + 1, "triangle source flags");
    uint32_t* R = arena.take_n<uint32_t>(std::max<uint64_t>(V, 1), "triangle roots");
    CliqueTiers t;
    for (int k = 0; k < 4; k++) t.root[k] = arena.take_n<uint32_t>(std::max<uint64_t>(V, 1), "triangle tier roots");
    t.count = arena.take_n<unsigned long long>(8, "triangle counters");  // 4 tiers, 3 queue heads, the root count
    CK(cudaMemsetAsync(flags, 0, sizeof(uint32_t) * ((V + 3) / 4 + 1), stream));
    CK(cudaMemsetAsync(is_src, 0, sizeof(uint32_t) * ((V + 3) / 4 + 1), stream));
    CK(cudaMemsetAsync(t.count, 0, 8 * sizeof(unsigned long long), stream));
    k_tri_mark_roots<<<grid_warps(n), 256, 0, stream>>>(d_rp, d_ci, up, roots, n, flags, is_src);
    k_flags_to_list<<<grid_threads(V), 256, 0, stream>>>(flags, V, R, t.count + 7);
    CK(cudaGetLastError());
    const uint64_t nR = read_u64((const uint64_t*)(t.count + 7));
    k_clique_split<<<grid_threads(nR), 256, 0, stream>>>(d_rp, up, R, nR, 2u, kTriSmall, kTriMid, kTriLarge, t);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h_pinned, t.count, 4 * sizeof(uint64_t), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    const uint64_t nt[4] = {h_pinned[0], h_pinned[1], h_pinned[2], h_pinned[3]};
    if (nt[3]) {
      end_op(last, 3);
      Frame f;
      std::memset(&f, 0, sizeof(f));
      f.P = n;
      f.col[plan->op_vertex[0]] = const_cast<uint32_t*>(roots);
      process(1, f);
      return;
    }
    uint32_t* tri = arena.take_n<uint32_t>(std::max<uint64_t>(n_cols, 1), "per-edge triangle counts");
    CK(cudaMemsetAsync(tri, 0, sizeof(uint32_t) * std::max<uint64_t>(n_cols, 1), stream));
    unsigned long long* bytes = profiling ? d_bytes : nullptr;
    uint64_t launches = 5;
    if (nt[2]) {
      k_edge_tri_block<<<(unsigned)sms, 512, kTriLargeSmem, stream>>>(d_rp, d_ci, up, is_src, t.root[2], nt[2], t.count + 4, tri, bytes);
      launches++;
    }
    if (nt[1]) {
      k_edge_tri_warp<kTriMid><<<(unsigned)sms * 3, 256, kTriMidSmem, stream>>>(d_rp, d_ci, up, is_src, t.root[1], nt[1], t.count + 5, tri, bytes);
      launches++;
    }
    if (nt[0]) {
      k_edge_tri_warp<kTriSmall><<<(unsigned)sms * 8, 256, 8 * 2 * kTriSmall * sizeof(uint32_t), stream>>>(d_rp, d_ci, up, is_src, t.root[0], nt[0],
                                                                                                       t.count + 6, tri, bytes);
      launches++;
    }
    k_diamond_sum<<<grid_warps(n), 256, 0, stream>>>(d_rp, up, roots, n, tri, mode, d_total, bytes);
    CK(cudaGetLastError());
    end_op(last, launches);
    st->op_paths[last] += n;
  }

  // the DFS fused tail (DfsFused): the level-wise engine's fusable() rule
  static void dfs_fuse(const vsgm_plan& p, DfsPlan* d) {
    if (p.n_ops < 3) return;
    const int i = (int)p.n_ops - 2;
    if (p.op_type[i] != VSGM_MATERIALIZE || p.op_type[i + 1] != VSGM_COMPUTE_COUNT) return;
    const int u = p.op_vertex[i], w = p.op_vertex[i + 1];
    const vsgm_vgroup& B = p.backward[w];
    bool has_u = false;
    for (int k = 0; k < B.count; k++) has_u |= (B.v[k] == u);
    if (!has_u || B.count < 2 || B.count > 6) return;
    if (p.computed_unmat[i + 1].count > 1) return;
    const vsgm_conds& cc = p.compute_cond[w];
    int on_u = 0;
    for (int k = 0; k < cc.count; k++) on_u += (cc.v[k] == u);
    if (on_u > 1) return;
    DfsFused& f = d->fz;
    f.on = 1;
    f.lvl = (uint8_t)i;
    f.other = -1;
    f.known.type = VSGM_COMPUTE_COUNT;
    f.known.u = (uint8_t)w;
    for (int k = 0; k < B.count; k++)
      if (B.v[k] != u) f.known.b[f.known.nb++] = B.v[k];
    for (int k = 0; k < cc.count; k++) {
      if (cc.v[k] == u) {
        f.has_cond_u = 1;
        f.cond_u_op = cc.op[k];
      } else {
        f.known.cop[f.known.nc] = cc.op[k];
        f.known.cv[f.known.nc++] = cc.v[k];
      }
    }
    const vsgm_vgroup& cu = p.computed_unmat[i + 1];
    if (cu.count == 1) {
      f.other = (int8_t)cu.v[0];
      f.other_op = p.order[w][cu.v[0]];
    }
  }

  static DfsPlan to_dfs(const vsgm_plan& p, bool fuse = true) {
    DfsPlan d;
    std::memset(&d, 0, sizeof(d));
    if (fuse) dfs_fuse(p, &d);
    d.n_ops = p.n_ops;
    d.split_lvl = p.n_ops;
    for (uint32_t i = 1; i < p.n_ops; i++)
      if (p.op_type[i] == VSGM_MATERIALIZE) {
        d.split_lvl = i;
        break;
      }
    d.root = p.op_vertex[0];
    for (uint32_t i = 0; i < p.n_ops; i++) {
      DfsOp& o = d.op[i];
      o.type = p.op_type[i];
      o.u = p.op_vertex[i];
      o.other = -1;
      const vsgm_conds* c = nullptr;
      if (o.type == VSGM_COMPUTE_PATH_COUNT) o.type = VSGM_COMPUTE;  // the set's size is all a later COUNT reads
      if (o.type == VSGM_COMPUTE || o.type == VSGM_COMPUTE_COUNT) c = &p.compute_cond[o.u];
      if (o.type == VSGM_MATERIALIZE && i > 0) c = &p.materialize_cond[o.u];
      if (o.type == VSGM_FILTER_COMPUTE) c = &p.filter_cond[o.u];
      if (c) {
        o.nc = c->count;
        for (int k = 0; k < c->count; k++) {
          o.cop[k] = c->op[k];
          o.cv[k] = c->v[k];
        }
      }
      if (o.type == VSGM_COMPUTE || o.type == VSGM_COMPUTE_COUNT) {
        o.nb = p.backward[o.u].count;
        for (int k = 0; k < o.nb; k++) o.b[k] = p.backward[o.u].v[k];
      }
      const vsgm_vgroup& cu = p.computed_unmat[i];
      if (o.type == VSGM_COMPUTE_COUNT && cu.count == 1) {
        o.other = (int8_t)cu.v[0];
        o.other_op = p.order[o.u][cu.v[0]];
      }
      if (o.type == VSGM_COUNT) {
        o.ncu = cu.count;
        o.cu0 = cu.v[0];
        o.cu1 = cu.count > 1 ? cu.v[1] : 0;
        o.cu_op = cu.count > 1 ? p.order[cu.v[0]][cu.v[1]] : 0;
      }
    }
    return d;
  }

  // One persistent launch over every (plan, view) pair: tasks are root ranges of
  // balanced estimated cost, longest first, popped by warps from a device queue.
  // mask (optional): mask[plan * n_views + view] != 0 for the pairs to count; the
  // others get no tasks and count 0
  void run_batched(const int* view_ids, int n_views, const int* plan_ids, int n_plans, uint64_t* out, uint64_t* level_out = nullptr,
                   uint64_t step_budget = 0, uint32_t* overflow_out = nullptr, const uint8_t* mask = nullptr) {
    std::vector<DfsPlan> hp(n_plans);
    uint32_t levels = 1;
    for (int k = 0; k < n_plans; k++) {
      hp[k] = to_dfs(plans[plan_ids[k]], knobs[plan_ids[k]].fuse_tail);
      levels = std::max(levels, hp[k].n_ops);
    }
    std::vector<DfsView> hv(n_views);
    uint64_t cap = 1;
    for (int k = 0; k < n_views; k++) {
      const ResidentView& r = rviews[view_ids[k]];
      hv[k] = DfsView{r.rp, r.ci, r.src};
      cap = std::max(cap, r.max_deg);
    }
    // task costs: sum over roots of deg^2 (wedges through the root), per plan
    const uint64_t warps = (uint64_t)sms * 2 * kDfsWarps;  // two resident blocks per SM
    std::vector<std::pair<double, DfsTask>> tasks;
    double total = 0;
    std::vector<double> work(n_views, 0);
    for (int k = 0; k < n_views; k++) {
      for (uint64_t d : rviews[view_ids[k]].h_deg_src) work[k] += (double)d * (double)d + 1.0;
      total += work[k] * n_plans;
    }
    const double target = std::max(1.0, total / (double)(warps * 16));
    for (int pk = 0; pk < n_plans; pk++)
      for (int k = 0; k < n_views; k++) {
        if (mask && !mask[(size_t)pk * n_views + k]) continue;
        const auto& deg = rviews[view_ids[k]].h_deg_src;
        const bool splittable = hp[pk].split_lvl < hp[pk].n_ops;
        uint64_t r0 = 0;
        double acc = 0;
        for (uint64_t r = 0; r < deg.size(); r++) {
          const double w = (double)deg[r] * (double)deg[r] + 1.0;
          if (splittable && w > 2.0 * target && deg[r] > 1) {
            // a heavy root: close the open range, then split the root's candidates at
            // the split level (a subset of its neighbours) into shares of ~target work
            if (r > r0) tasks.push_back({acc, DfsTask{(uint32_t)pk, (uint32_t)k, r0, r, 0u, 0u}});
            const uint64_t shares = std::min<uint64_t>(deg[r], (uint64_t)std::ceil(w / target));
            const uint64_t per = (deg[r] + shares - 1) / shares;
            for (uint64_t c0 = 0; c0 < deg[r]; c0 += per)
              tasks.push_back({w / (double)shares, DfsTask{(uint32_t)pk, (uint32_t)k, r, r + 1, (uint32_t)c0, (uint32_t)std::min<uint64_t>(c0 + per, deg[r])}});
            r0 = r + 1;
            acc = 0;
            continue;
          }
          acc += w;
          if (acc >= target || r + 1 == deg.size()) {
            tasks.push_back({acc, DfsTask{(uint32_t)pk, (uint32_t)k, r0, r + 1, 0u, 0u}});
            r0 = r + 1;
            acc = 0;
          }
        }
      }
    std::stable_sort(tasks.begin(), tasks.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    std::vector<DfsTask> ht(tasks.size());
    for (size_t k = 0; k < tasks.size(); k++) ht[k] = tasks[k].second;

    Mark m(arena);
    DfsPlan* d_plans = arena.take_n<DfsPlan>(n_plans, "batched plans");
    DfsView* d_views = arena.take_n<DfsView>(n_views, "batched views");
    DfsTask* d_tasks = arena.take_n<DfsTask>(std::max<size_t>(1, ht.size()), "batched tasks");
    const uint64_t pairs = (uint64_t)n_plans * n_views;
    unsigned long long* d_cnt = arena.take_n<unsigned long long>(pairs + 2, "batched counts");
    unsigned long long* d_lvl = level_out ? arena.take_n<unsigned long long>(pairs * VSGM_MAX_OPS, "level paths") : nullptr;
    unsigned int* d_ovf = overflow_out ? arena.take_n<unsigned int>(pairs, "overflow flags") : nullptr;
    if (d_lvl) CK(cudaMemsetAsync(d_lvl, 0, sizeof(unsigned long long) * pairs * VSGM_MAX_OPS, stream));
    if (d_ovf) CK(cudaMemsetAsync(d_ovf, 0, sizeof(unsigned int) * pairs, stream));
    const uint64_t grid = (uint64_t)sms * 2;
    uint32_t* scratch = arena.take_n<uint32_t>(grid * kDfsWarps * levels * cap, "per-warp scratch");
    CK(cudaMemcpyAsync(d_plans, hp.data(), sizeof(DfsPlan) * n_plans, cudaMemcpyHostToDevice, stream));
    CK(cudaMemcpyAsync(d_views, hv.data(), sizeof(DfsView) * n_views, cudaMemcpyHostToDevice, stream));
    if (!ht.empty()) CK(cudaMemcpyAsync(d_tasks, ht.data(), sizeof(DfsTask) * ht.size(), cudaMemcpyHostToDevice, stream));
    CK(cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long) * ((uint64_t)n_plans * n_views + 2), stream));
    unsigned long long* d_head = d_cnt + (uint64_t)n_plans * n_views;
    unsigned int* d_status = (unsigned int*)(d_head + 1);
    if (profiling) CK(cudaEventRecord(ev0, stream));
    k_dfs<<<(unsigned)grid, kDfsWarps * kWarp, 0, stream>>>(d_plans, d_views, d_tasks, ht.size(), d_head, scratch, cap, levels, (uint32_t)n_views, d_cnt,
                                                             d_status, d_lvl, step_budget, d_ovf);
    CK(cudaGetLastError());
    if (profiling) CK(cudaEventRecord(ev1, stream));
    std::vector<uint64_t> hc((uint64_t)n_plans * n_views + 2);
    CK(cudaMemcpyAsync(hc.data(), d_cnt, sizeof(uint64_t) * hc.size(), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    if ((uint32_t)hc[(uint64_t)n_plans * n_views + 1] != 0) throw OutOfMemory{"batched run: a candidate set exceeded the per-warp scratch"};
    bstats.tasks = ht.size();
    bstats.launches = 1;
    bstats.level_pairs = 0;
    bstats.scratch_bytes = grid * kDfsWarps * levels * cap * 4;
    bstats.ms = 0;
    if (profiling) {
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, ev0, ev1));
      bstats.ms = ms;
    }
    for (uint64_t k = 0; k < (uint64_t)n_plans * n_views; k++) out[k] = hc[k];
    if (level_out) CK(cudaMemcpy(level_out, d_lvl, sizeof(uint64_t) * pairs * VSGM_MAX_OPS, cudaMemcpyDeviceToHost));
    if (overflow_out) CK(cudaMemcpy(overflow_out, d_ovf, sizeof(uint32_t) * pairs, cudaMemcpyDeviceToHost));
  }

  // Hybrid batched run (knob hybrid_steps): one persistent launch finishes every
  // pair whose tasks stay within the step bound; the pairs it stopped are counted
  // again by the level-wise engine on their resident view (their partial counts
  // are discarded).
  void run_hybrid(const int* view_ids, int n_views, const int* plan_ids, int n_plans, uint64_t* counts, const uint8_t* mask) {
    if (!hybrid_steps) {
      run_batched(view_ids, n_views, plan_ids, n_plans, counts, nullptr, 0, nullptr, mask);
      return;
    }
    if (profiling) CK(cudaEventRecord(ev_h0, stream));
    std::vector<uint32_t> ovf((size_t)n_plans * n_views, 0);
    run_batched(view_ids, n_views, plan_ids, n_plans, counts, nullptr, hybrid_steps, ovf.data(), mask);
    vsgm_batch_stats bs = bstats;
    std::vector<std::pair<int, int>> rerun;  // (plan index, view index) the persistent launch stopped
    for (int p = 0; p < n_plans; p++)
      for (int v = 0; v < n_views; v++)
        if (ovf[(size_t)p * n_views + v]) rerun.push_back({p, v});
    const int K = (int)std::min<size_t>((size_t)std::max(1, streams), rerun.size());
    if (K <= 1) {
      for (auto [p, v] : rerun) {
        counts[(size_t)p * n_views + v] = run_resident(view_ids[v], plan_ids[p]);
        const vsgm_plan_stats& st = stats[plan_ids[p]];
        for (uint32_t i = 0; i < plans[plan_ids[p]].n_ops; i++) bs.launches += st.op_launches[i];
        bs.level_pairs++;
      }
    } else {
      // K helper engines on their own streams, each with a slice of our arena, take
      // the pairs from a shared index (heaviest pairs are not known in advance)
      CK(cudaStreamSynchronize(stream));
      const auto t0 = std::chrono::steady_clock::now();
      const size_t slice = (arena.cap / (size_t)K) & ~(size_t)255;
      while ((int)helpers.size() < K) helpers.push_back(make_helper());
      std::atomic<size_t> next{0};
      std::vector<std::string> errs(K);
      std::vector<uint64_t> launches(K, 0);
      std::vector<std::thread> th;
      for (int k = 0; k < K; k++) {
        vsgm_engine* h = helpers[k];
        h->knobs = knobs;
        h->profiling = profiling;
        h->rviews = rviews;
        h->arena.base = arena.base + (size_t)k * slice;
        h->arena.cap = slice;
        h->arena.top = h->arena.peak = 0;
        th.emplace_back([&, h, k] {
          try {
            CK(cudaSetDevice(device));
            for (size_t i; (i = next++) < rerun.size();) {
              const auto [p, v] = rerun[i];
              counts[(size_t)p * n_views + v] = h->run_resident(view_ids[v], plan_ids[p]);
              const vsgm_plan_stats& st = h->stats[plan_ids[p]];
              for (uint32_t j = 0; j < plans[plan_ids[p]].n_ops; j++) launches[k] += st.op_launches[j];
            }
          } catch (const CudaError& c) {
            errs[k] = std::string("CUDA error ") + cudaGetErrorString(c.code) + " in " + c.what;
          } catch (const OutOfMemory& o) {
            errs[k] = o.what;
          } catch (const std::exception& x) {
            errs[k] = x.what();
          }
        });
      }
      for (auto& t : th) t.join();
      for (const auto& m : errs)
        if (!m.empty()) throw std::runtime_error("concurrent rerun: " + m);
      for (uint64_t l : launches) bs.launches += l;
      bs.level_pairs += rerun.size();
      if (profiling) {
        // the helpers' streams are not ours: the persistent launch's events plus host time of the reruns
        CK(cudaEventRecord(ev_h1, stream));
        CK(cudaEventSynchronize(ev_h1));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ev_h0, ev_h1));
        bs.ms = ms + std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
        bstats = bs;
        return;
      }
    }
    if (profiling) {
      CK(cudaEventRecord(ev_h1, stream));
      CK(cudaEventSynchronize(ev_h1));
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, ev_h0, ev_h1));
      bs.ms = ms;
    }
    bstats = bs;
  }

  // A helper engine for concurrent reruns: same device, plans and knobs; its own
  // stream, events, counters and pinned staging; views and arena lent per run.
  vsgm_engine* make_helper() {
    vsgm_engine* h = new vsgm_engine();
    h->helper = true;
    h->device = device;
    h->sms = sms;
    h->V = V;
    h->plans = plans;
    h->knobs = knobs;
    h->totals.assign(plans.size(), 0);
    h->stats.assign(plans.size(), vsgm_plan_stats{});
    try {
      CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
      CK(cudaStreamCreateWithFlags(&h->aux_stream, cudaStreamNonBlocking));
      CK(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));
      CK(cudaEventCreate(&h->ev0));
      CK(cudaEventCreate(&h->ev1));
      CK(cudaEventCreate(&h->ev_h0));
      CK(cudaEventCreate(&h->ev_h1));
      CK(cudaMalloc(&h->d_counts, sizeof(unsigned long long) * (plans.size() + 2)));
      h->d_bytes = h->d_counts + plans.size();
      CK(cudaMemset(h->d_counts, 0, sizeof(unsigned long long) * (plans.size() + 2)));
      CK(cudaMallocHost(&h->h_pinned, 64));
    } catch (...) {
      release_helper(h);
      throw;
    }
    return h;
  }

  static void release_helper(vsgm_engine* h) {
    if (h->stream) cudaStreamSynchronize(h->stream);
    cudaFree(h->d_counts);
    cudaFree(h->d_up);
    if (h->h_pinned) cudaFreeHost(h->h_pinned);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->ev_h0) cudaEventDestroy(h->ev_h0);
    if (h->ev_h1) cudaEventDestroy(h->ev_h1);
    if (h->aux_stream) cudaStreamSynchronize(h->aux_stream);
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ev_join) cudaEventDestroy(h->ev_join);
    if (h->aux_stream) cudaStreamDestroy(h->aux_stream);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
  }

  // The level-wise engine on one resident view (the hybrid batched run's heavy
  // pairs): the view temporarily becomes the current one.
  uint64_t run_resident(int vid, int pk) {
    const ResidentView& r = rviews[vid];
    const uint64_t* s_rp = d_rp;
    const uint32_t* s_ci = d_ci;
    const uint32_t* s_src = d_src;
    const uint64_t s_nsrc = n_src, s_ncols = n_cols, s_V = V, s_stride = root_stride;
    root_stride = 1;  // every source of the view, as the persistent launch does
    d_rp = r.rp;
    d_ci = r.ci;
    d_src = r.src;
    n_src = r.n_src;
    n_cols = r.n_cols;
    V = r.V;
    up_of = nullptr;
    uint64_t c = 0;
    try {
      CK(cudaMemsetAsync(d_counts + pk, 0, sizeof(unsigned long long), stream));
      stats[pk] = vsgm_plan_stats{};
      arena.top = 0;
      run_plan(pk);
      c = read_u64((const uint64_t*)(d_counts + pk));
    } catch (...) {
      d_rp = const_cast<uint64_t*>(s_rp);
      d_ci = const_cast<uint32_t*>(s_ci);
      d_src = const_cast<uint32_t*>(s_src);
      n_src = s_nsrc;
      n_cols = s_ncols;
      V = s_V;
      root_stride = s_stride;
      up_of = nullptr;
      throw;
    }
    d_rp = const_cast<uint64_t*>(s_rp);
    d_ci = const_cast<uint32_t*>(s_ci);
    d_src = const_cast<uint32_t*>(s_src);
    n_src = s_nsrc;
    n_cols = s_ncols;
    V = s_V;
    root_stride = s_stride;
    up_of = nullptr;
    return c;
  }

  void run_plan(int pi) {
    plan = &plans[pi];
    st = &stats[pi];
    cur = knobs[pi];
    d_total = d_counts + pi;
    if (n_src == 0) return;
    Frame f;
    std::memset(&f, 0, sizeof(f));
    f.P = n_src;
    f.col[plan->op_vertex[0]] = d_src;
    Mark m(arena);
    if (root_stride > 1) {
      // sampled run: every root_stride-th source only
      f.P = (n_src + root_stride - 1) / root_stride;
      uint32_t* sampled = arena.take_n<uint32_t>(f.P, "sampled roots");
      k_stride_copy<<<grid_threads(f.P), 256, 0, stream>>>(d_src, f.P, root_stride, sampled);
      CK(cudaGetLastError());
      f.col[plan->op_vertex[0]] = sampled;
    }
    st->op_paths[0] += f.P;
    st->op_outputs[0] += f.P;
    const int K = cur.clique_bits ? clique_order(*plan) : 0;
    if (cur.c4_aggregate && is_four_cycle(*plan)) {
      c4_aggregate(f.col[plan->op_vertex[0]], f.P);
    } else if (K == 3 || K == 4) {
      clique_bits(f.col[plan->op_vertex[0]], f.P, K);
    } else if (const int dm = cur.edge_triangles ? diamond_mode(*plan) : 0) {
      diamond_edges(f.col[plan->op_vertex[0]], f.P, dm);
    } else {
      process(1, f);
    }
    if (profiling) {
      // the CC kernel accumulated algorithmic bytes
      uint64_t b = read_u64((const uint64_t*)d_bytes);
      for (uint32_t k = 0; k < plan->n_ops; k++)
        if (plan->op_type[k] == VSGM_COMPUTE_COUNT) st->op_bytes[k] += b;
      CK(cudaMemsetAsync(d_bytes, 0, sizeof(unsigned long long), stream));
    }
  }
};

// ---------------------------------------------------------------- C ABI
namespace {
thread_local std::string g_engine_err;

int engine_fail(vsgm_engine* e, int code, const std::string& msg) {
  if (e) e->err = msg;
  g_engine_err = msg;
  return code;
}

template <typename F>
int guarded(vsgm_engine* e, F&& body) {
  try {
    body();
    return VSGM_OK;
  } catch (const CudaError& c) {
    char buf[512];
    std::snprintf(buf, sizeof(buf), "CUDA error %d (%s) at engine.cu:%d in %s", (int)c.code, cudaGetErrorString(c.code), c.line, c.what);
    return engine_fail(e, VSGM_ECUDA, buf);
  } catch (const OutOfMemory& o) {
    return engine_fail(e, VSGM_ENOMEM, o.what);
  } catch (const std::exception& x) {
    return engine_fail(e, VSGM_EINVAL, x.what());
  }
}
}  // namespace

extern "C" {

int vsgm_create(int device, uint64_t V, const vsgm_plan* plans, int n_plans, uint64_t max_sources, uint64_t hbm_budget_bytes, vsgm_engine** out) {
  if (!out || !plans || n_plans < 1 || V == 0 || V >= 0xffffffffull) return engine_fail(nullptr, VSGM_EINVAL, "bad engine arguments");
  for (int k = 0; k < n_plans; k++) {
    const vsgm_plan& p = plans[k];
    if (p.n_vertices < 2 || p.n_vertices > VSGM_MAX_QV || p.n_ops < 2 || p.n_ops > VSGM_MAX_OPS || p.op_type[0] != VSGM_MATERIALIZE)
      return engine_fail(nullptr, VSGM_EINVAL, "malformed plan");
    // a COMPUTE_PATH_COUNT vertex has sizes only: a later op may count it, never read it
    for (uint32_t i = 0; i < p.n_ops; i++) {
      if (p.op_type[i] != VSGM_COMPUTE_PATH_COUNT) continue;
      const int u = p.op_vertex[i];
      for (uint32_t j = i + 1; j < p.n_ops; j++) {
        const vsgm_vgroup& cu = p.computed_unmat[j];
        bool in_cu = false;
        for (int q = 0; q < cu.count; q++) in_cu |= cu.v[q] == u;
        const int t = p.op_type[j];
        if (((t == VSGM_MATERIALIZE || t == VSGM_FILTER_COMPUTE) && p.op_vertex[j] == u) || (t == VSGM_COMPUTE_COUNT && in_cu) ||
            (t == VSGM_COUNT && in_cu && cu.count > 1))
          return engine_fail(nullptr, VSGM_EINVAL, "a COMPUTE_PATH_COUNT vertex is read by a later op (only a COUNT of it may follow)");
      }
    }
  }
  vsgm_engine* e = new vsgm_engine();
  e->device = device;
  e->V = V;
  e->plans.assign(plans, plans + n_plans);
  e->max_sources = max_sources;
  e->totals.assign(n_plans, 0);
  e->stats.assign(n_plans, vsgm_plan_stats{});
  e->knobs.assign(n_plans, vsgm_engine::Knobs{});
  int rc = guarded(e, [&] {
    CK(cudaSetDevice(device));
    CK(cudaDeviceGetAttribute(&e->sms, cudaDevAttrMultiProcessorCount, device));
    CK(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&e->copy_stream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&e->ev_copy, cudaEventDisableTiming));
    CK(cudaStreamCreateWithFlags(&e->aux_stream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&e->ev_join, cudaEventDisableTiming));
    // the clique operator's tiers keep their rows in more than 48 KB of shared memory
    CK(cudaFuncSetAttribute(k_clique_mid<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCliqueMidSmem));
    CK(cudaFuncSetAttribute(k_clique_mid<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCliqueMidSmem));
    CK(cudaFuncSetAttribute(k_clique_large<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCliqueLargeSmem));
    CK(cudaFuncSetAttribute(k_clique_large<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCliqueLargeSmem));
    CK(cudaFuncSetAttribute(k_edge_tri_warp<kTriMid>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTriMidSmem));
    CK(cudaFuncSetAttribute(k_edge_tri_block, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTriLargeSmem));
    CK(cudaFuncSetAttribute(k_c4_hash_warp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kC4HashWarpSmem));
    CK(cudaFuncSetAttribute(k_c4_hash_block, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kC4HashBlockSmem));
    CK(cudaFuncSetAttribute(k_c4_window, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kC4WinSmem));
    CK(cudaEventCreate(&e->ev0));
    CK(cudaEventCreate(&e->ev1));
    CK(cudaEventCreate(&e->ev_h0));
    CK(cudaEventCreate(&e->ev_h1));
    CK(cudaMalloc(&e->d_counts, sizeof(unsigned long long) * (n_plans + 2)));
    e->d_bytes = e->d_counts + n_plans;
    CK(cudaMemset(e->d_counts, 0, sizeof(unsigned long long) * (n_plans + 2)));
    CK(cudaMallocHost(&e->h_pinned, 64));
    CK(cudaMalloc(&e->own_rp, sizeof(uint64_t) * (V + 1)));
    if (max_sources) {
      CK(cudaMalloc(&e->own_src, sizeof(uint32_t) * max_sources));
      e->src_cap = max_sources;
    }
    size_t free_b = 0, total_b = 0;
    CK(cudaMemGetInfo(&free_b, &total_b));
    size_t budget = hbm_budget_bytes ? hbm_budget_bytes : (size_t)(free_b * 0.9);
    if (budget > free_b) budget = (size_t)(free_b * 0.95);
    e->arena.cap = budget & ~(size_t)255;
    CK(cudaMalloc(&e->arena.base, e->arena.cap));
  });
  if (rc != VSGM_OK) {
    vsgm_destroy(e);
    return rc;
  }
  *out = e;
  return VSGM_OK;
}

int vsgm_transfer_view(vsgm_engine* e, const uint64_t* row_ptrs, const uint32_t* cols, uint64_t n_cols, const uint32_t* sources, uint64_t n_sources) {
  if (!e || !row_ptrs || (n_cols && !cols) || (n_sources && !sources)) return engine_fail(e, VSGM_EINVAL, "null view argument");
  if (row_ptrs[e->V] != n_cols) return engine_fail(e, VSGM_EINVAL, "row_ptrs[V] != n_cols");
  for (uint64_t i = 0; i < n_sources; i++)
    if (sources[i] >= e->V) return engine_fail(e, VSGM_EINVAL, "source id out of range");
  return guarded(e, [&] {
    CK(cudaSetDevice(e->device));
    if (n_cols > e->cols_cap) {
      if (e->own_ci) CK(cudaFree(e->own_ci));
      e->own_ci = nullptr;
      CK(cudaMalloc(&e->own_ci, sizeof(uint32_t) * std::max<uint64_t>(n_cols, 1)));
      e->cols_cap = n_cols;
    }
    if (n_sources > e->src_cap) {
      if (e->own_src) CK(cudaFree(e->own_src));
      e->own_src = nullptr;
      CK(cudaMalloc(&e->own_src, sizeof(uint32_t) * n_sources));
      e->src_cap = n_sources;
    }
    CK(cudaMemcpyAsync(e->own_rp, row_ptrs, sizeof(uint64_t) * (e->V + 1), cudaMemcpyHostToDevice, e->stream));
    if (n_cols) CK(cudaMemcpyAsync(e->own_ci, cols, sizeof(uint32_t) * n_cols, cudaMemcpyHostToDevice, e->stream));
    if (n_sources) CK(cudaMemcpyAsync(e->own_src, sources, sizeof(uint32_t) * n_sources, cudaMemcpyHostToDevice, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    e->d_rp = e->own_rp;
    e->d_ci = e->own_ci;
    e->d_src = e->own_src;
    e->n_cols = n_cols;
    e->n_src = n_sources;
    e->have_view = true;
    e->up_of = nullptr;  // a new view: the upper offsets are stale
  });
}

int vsgm_bind_view_device(vsgm_engine* e, const uint64_t* d_row_ptrs, const uint32_t* d_cols, uint64_t n_cols, const uint32_t* d_sources, uint64_t n_sources) {
  if (!e || !d_row_ptrs || (n_cols && !d_cols) || (n_sources && !d_sources)) return engine_fail(e, VSGM_EINVAL, "null view argument");
  e->d_rp = const_cast<uint64_t*>(d_row_ptrs);
  e->d_ci = const_cast<uint32_t*>(d_cols);
  e->d_src = const_cast<uint32_t*>(d_sources);
  e->n_cols = n_cols;
  e->n_src = n_sources;
  e->have_view = true;
  e->up_of = nullptr;
  return VSGM_OK;
}

int vsgm_upload_graph(vsgm_engine* e, const uint64_t* row_ptrs, const uint32_t* cols, uint64_t n_cols) {
  if (!e || !row_ptrs || (n_cols && !cols)) return engine_fail(e, VSGM_EINVAL, "null graph argument");
  if (row_ptrs[e->V] != n_cols) return engine_fail(e, VSGM_EINVAL, "row_ptrs[V] != n_cols");
  return guarded(e, [&] {
    CK(cudaSetDevice(e->device));
    CK(cudaStreamSynchronize(e->stream));
    // the buffers of an earlier upload are kept when the new graph fits them
    if (!e->g_rp) CK(cudaMalloc(&e->g_rp, sizeof(uint64_t) * (e->V + 1)));
    if (e->g_ci && e->g_cap < n_cols) {
      CK(cudaFree(e->g_ci));
      e->g_ci = nullptr;
    }
    if (!e->g_ci) {
      CK(cudaMalloc(&e->g_ci, sizeof(uint32_t) * std::max<uint64_t>(n_cols, 1)));
      e->g_cap = n_cols;
    }
    if (!e->relabel && e->g_new) {
      CK(cudaFree(e->g_new));
      e->g_new = nullptr;
    }
    if (e->relabel) {
      // the caller's graph goes to the arena first, the relabelled one stays resident
      if (!e->g_new) CK(cudaMalloc(&e->g_new, sizeof(uint32_t) * std::max<uint64_t>(e->V, 1)));
      Mark m(e->arena);
      e->arena.top = 0;
      uint64_t* t_rp = e->arena.take_n<uint64_t>(e->V + 1, "graph row offsets (caller ids)");
      uint32_t* t_ci = e->arena.take_n<uint32_t>(std::max<uint64_t>(n_cols, 1), "graph adjacency (caller ids)");
      CK(cudaMemcpyAsync(t_rp, row_ptrs, sizeof(uint64_t) * (e->V + 1), cudaMemcpyHostToDevice, e->stream));
      if (n_cols) CK(cudaMemcpyAsync(t_ci, cols, sizeof(uint32_t) * n_cols, cudaMemcpyHostToDevice, e->stream));
      e->relabel_into_resident(t_rp, t_ci, n_cols);
    } else {
      CK(cudaMemcpyAsync(e->g_rp, row_ptrs, sizeof(uint64_t) * (e->V + 1), cudaMemcpyHostToDevice, e->stream));
      if (n_cols) CK(cudaMemcpyAsync(e->g_ci, cols, sizeof(uint32_t) * n_cols, cudaMemcpyHostToDevice, e->stream));
    }
    CK(cudaStreamSynchronize(e->stream));
    e->g_cols = n_cols;
  });
}

int vsgm_materialize_view(vsgm_engine* e, const uint32_t* sources, uint64_t n_sources, int hop, uint64_t root_degree) {
  if (!e || (n_sources && !sources)) return engine_fail(e, VSGM_EINVAL, "null view argument");
  if (!e->g_rp) return engine_fail(e, VSGM_EINVAL, "no graph uploaded");
  if (hop < 1) return engine_fail(e, VSGM_EINVAL, "hop must be >= 1");
  for (uint64_t i = 0; i < n_sources; i++)
    if (sources[i] >= e->V) return engine_fail(e, VSGM_EINVAL, "source id out of range");
  return guarded(e, [&] {
    CK(cudaSetDevice(e->device));
    const uint64_t V = e->V;
    if (n_sources > e->src_cap) {
      if (e->own_src) CK(cudaFree(e->own_src));
      e->own_src = nullptr;
      CK(cudaMalloc(&e->own_src, sizeof(uint32_t) * n_sources));
      e->src_cap = n_sources;
    }
    if (n_sources) CK(cudaMemcpyAsync(e->own_src, sources, sizeof(uint32_t) * n_sources, cudaMemcpyHostToDevice, e->stream));
    if (n_sources && e->g_new) k_map_ids<<<e->grid_threads(n_sources), 256, 0, e->stream>>>(e->own_src, n_sources, e->g_new);
    Mark m(e->arena);
    e->arena.top = 0;
    // membership flags: one byte per vertex, whole words so the flag update is a word atomic
    uint8_t* flags = (uint8_t*)e->arena.take_n<uint32_t>((V + 3) / 4 + 1, "view flags");
    uint32_t* cur = e->arena.take_n<uint32_t>(std::max<uint64_t>(V, 1), "view frontier");
    uint32_t* nxt = e->arena.take_n<uint32_t>(std::max<uint64_t>(V, 1), "view frontier");
    unsigned long long* cnt = e->arena.take_n<unsigned long long>(2, "view counters");
    uint64_t* len = e->arena.take_n<uint64_t>(V + 1, "view row lengths");
    CK(cudaMemsetAsync(flags, 0, sizeof(uint32_t) * ((V + 3) / 4 + 1), e->stream));
    CK(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * 2, e->stream));
    k_halo_seed2<<<e->grid_threads(n_sources), 256, 0, e->stream>>>(e->g_rp, e->own_src, n_sources, root_degree, flags, cur, cnt);
    CK(cudaGetLastError());
    uint64_t n_cur = e->read_u64((const uint64_t*)cnt);
    for (int layer = 1; layer < hop && n_cur; layer++) {
      CK(cudaMemsetAsync(cnt + 1, 0, sizeof(unsigned long long), e->stream));
      k_halo_layer<<<e->grid_warps(n_cur), 256, 0, e->stream>>>(e->g_rp, e->g_ci, V, cur, n_cur, flags, nxt, cnt + 1);
      CK(cudaGetLastError());
      n_cur = e->read_u64((const uint64_t*)(cnt + 1));
      std::swap(cur, nxt);
    }
    k_halo_lengths<<<e->grid_threads(V), 256, 0, e->stream>>>(e->g_rp, V, flags, len);
    CK(cudaGetLastError());
    e->scan(len, false, V, e->own_rp);
    const uint64_t total = e->read_u64(e->own_rp + V);
    if (total > e->cols_cap) {
      if (e->own_ci) CK(cudaFree(e->own_ci));
      e->own_ci = nullptr;
      CK(cudaMalloc(&e->own_ci, sizeof(uint32_t) * std::max<uint64_t>(total, 1)));
      e->cols_cap = total;
    }
    k_halo_copy<<<e->grid_warps(V), 256, 0, e->stream>>>(e->g_rp, e->g_ci, V, flags, e->own_rp, e->own_ci);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(e->stream));
    e->d_rp = e->own_rp;
    e->d_ci = e->own_ci;
    e->d_src = e->own_src;
    e->n_cols = total;
    e->n_src = n_sources;
    e->have_view = true;
    e->up_of = nullptr;  // a new view: the upper offsets are stale
  });
}

int vsgm_graph_view(vsgm_engine* e, const uint32_t* sources, uint64_t n_sources) {
  if (!e || (n_sources && !sources)) return engine_fail(e, VSGM_EINVAL, "null view argument");
  if (!e->g_rp) return engine_fail(e, VSGM_EINVAL, "no graph uploaded");
  for (uint64_t i = 0; i < n_sources; i++)
    if (sources[i] >= e->V) return engine_fail(e, VSGM_EINVAL, "source id out of range");
  return guarded(e, [&] {
    CK(cudaSetDevice(e->device));
    if (n_sources > e->src_cap) {
      if (e->own_src) CK(cudaFree(e->own_src));
      e->own_src = nullptr;
      CK(cudaMalloc(&e->own_src, sizeof(uint32_t) * n_sources));
      e->src_cap = n_sources;
    }
    if (n_sources) CK(cudaMemcpyAsync(e->own_src, sources, sizeof(uint32_t) * n_sources, cudaMemcpyHostToDevice, e->stream));
    if (n_sources && e->g_new) k_map_ids<<<e->grid_threads(n_sources), 256, 0, e->stream>>>(e->own_src, n_sources, e->g_new);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(e->stream));
    e->d_rp = e->g_rp;
    e->d_ci = e->g_ci;
    e->d_src = e->own_src;
    e->n_cols = e->g_cols;
    e->n_src = n_sources;
    e->have_view = true;
    e->up_of = nullptr;  // a new view: the upper offsets are stale
  });
}

int vsgm_read_view(vsgm_engine* e, uint64_t* row_ptrs, uint32_t* cols, uint64_t cols_cap, uint64_t* n_cols) {
  if (!e || !row_ptrs || !n_cols) return engine_fail(e, VSGM_EINVAL, "null argument");
  if (!e->have_view) return engine_fail(e, VSGM_EINVAL, "no view transferred");
  *n_cols = e->n_cols;
  if (e->n_cols > cols_cap || (e->n_cols && !cols)) return engine_fail(e, VSGM_ENOMEM, "view has more adjacency entries than cols_cap");
  return guarded(e, [&] {
    CK(cudaSetDevice(e->device));
    CK(cudaMemcpyAsync(row_ptrs, e->d_rp, sizeof(uint64_t) * (e->V + 1), cudaMemcpyDeviceToHost, e->stream));
    if (e->n_cols) CK(cudaMemcpyAsync(cols, e->d_ci, sizeof(uint32_t) * e->n_cols, cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
  });
}

int vsgm_match(vsgm_engine* e) {
  if (!e) return engine_fail(nullptr, VSGM_EINVAL, "null engine");
  if (!e->have_view) return engine_fail(e, VSGM_EINVAL, "no view transferred");
  return guarded(e, [&] {
    CK(cudaSetDevice(e->device));
    const int n = (int)e->plans.size();
    CK(cudaMemsetAsync(e->d_counts, 0, sizeof(unsigned long long) * (n + 2), e->stream));
    for (int k = 0; k < n; k++) {
      if (e->only_plan >= 0 && k != e->only_plan) continue;
      e->stats[k] = vsgm_plan_stats{};
      e->arena.top = 0;
      e->arena.peak = 0;
      e->run_plan(k);
      e->stats[k].peak_bytes = e->arena.peak;
    }
    std::vector<uint64_t> c(n);
    CK(cudaMemcpyAsync(e->h_pinned, e->d_counts, sizeof(uint64_t) * std::min(n, 8), cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    if (n > 8) {
      CK(cudaMemcpy(c.data(), e->d_counts, sizeof(uint64_t) * n, cudaMemcpyDeviceToHost));
    } else {
      for (int k = 0; k < n; k++) c[k] = e->h_pinned[k];
    }
    for (int k = 0; k < n; k++) e->totals[k] += c[k];
  });
}

int vsgm_get_counts(vsgm_engine* e, uint64_t* out) {
  if (!e || !out) return engine_fail(e, VSGM_EINVAL, "null argument");
  for (size_t k = 0; k < e->totals.size(); k++) out[k] = e->totals[k];
  return VSGM_OK;
}

int vsgm_reset_counts(vsgm_engine* e) {
  if (!e) return engine_fail(nullptr, VSGM_EINVAL, "null engine");
  std::fill(e->totals.begin(), e->totals.end(), 0);
  return VSGM_OK;
}

int vsgm_get_stats(vsgm_engine* e, int plan, vsgm_plan_stats* out) {
  if (!e || !out || plan < 0 || plan >= (int)e->plans.size()) return engine_fail(e, VSGM_EINVAL, "bad stats request");
  *out = e->stats[plan];
  return VSGM_OK;
}

int vsgm_set_plan_option(vsgm_engine* e, int plan, const char* name, int64_t value) {
  if (!e || !name) return engine_fail(e, VSGM_EINVAL, "null argument");
  if (plan < -1 || plan >= (int)e->plans.size()) return engine_fail(e, VSGM_EINVAL, "bad plan index");
  const std::string n(name);
  const int lo = plan < 0 ? 0 : plan, hi = plan < 0 ? (int)e->plans.size() : plan + 1;
  if (n == "fuse_tail") {
    for (int k = lo; k < hi; k++) e->knobs[k].fuse_tail = value != 0;
    return VSGM_OK;
  }
  if (n == "stage_cap") {
    if (value < 0 || value > kStageCap) return engine_fail(e, VSGM_EINVAL, "stage_cap must be 0.." + std::to_string(kStageCap));
    for (int k = lo; k < hi; k++) e->knobs[k].stage_cap = (uint32_t)value;
    return VSGM_OK;
  }
  if (n == "set_reuse") {
    for (int k = lo; k < hi; k++) e->knobs[k].set_reuse = value != 0;
    return VSGM_OK;
  }
  if (n == "c4_aggregate") {
    for (int k = lo; k < hi; k++) e->knobs[k].c4_aggregate = value != 0;
    return VSGM_OK;
  }
  if (n == "edge_triangles") {
    for (int k = lo; k < hi; k++) e->knobs[k].edge_triangles = value != 0;
    return VSGM_OK;
  }
  if (n == "clique_bits") {
    for (int k = lo; k < hi; k++) e->knobs[k].clique_bits = value != 0;
    return VSGM_OK;
  }
  if (n == "tail_merge") {
    for (int k = lo; k < hi; k++) e->knobs[k].tail_merge = value != 0;
    return VSGM_OK;
  }
  if (n == "lane_slice") {
    if (value < 0 || value > 4096) return engine_fail(e, VSGM_EINVAL, "lane_slice must be 0..4096");
    for (int k = lo; k < hi; k++) e->knobs[k].lane_slice = (uint32_t)value;
    return VSGM_OK;
  }
  if (n == "walk_ratio") {
    if (value < 0 || value > 65535) return engine_fail(e, VSGM_EINVAL, "walk_ratio must be 0..65535");
    for (int k = lo; k < hi; k++) e->knobs[k].walk_ratio = (uint32_t)value;
    return VSGM_OK;
  }
  if (n == "c4_balance") {
    for (int k = lo; k < hi; k++) e->knobs[k].c4_balance = value != 0;
    return VSGM_OK;
  }
  if (n == "c4_window") {
    for (int k = lo; k < hi; k++) e->knobs[k].c4_window = value != 0;
    return VSGM_OK;
  }
  if (n == "c4_hash") {
    for (int k = lo; k < hi; k++) e->knobs[k].c4_hash = value != 0;
    return VSGM_OK;
  }
  if (n == "c4_heavy") {
    if (value < 0) return engine_fail(e, VSGM_EINVAL, "c4_heavy must be >= 0");
    for (int k = lo; k < hi; k++) e->knobs[k].c4_heavy = (uint64_t)value;
    return VSGM_OK;
  }
  if (n == "lane_merge") {
    for (int k = lo; k < hi; k++) e->knobs[k].lane_merge = value != 0;
    return VSGM_OK;
  }
  if (n == "merge_ratio") {
    if (value < 0 || value > 65535) return engine_fail(e, VSGM_EINVAL, "merge_ratio must be 0..65535");
    for (int k = lo; k < hi; k++) e->knobs[k].merge_ratio = (uint32_t)value;
    return VSGM_OK;
  }
  if (n == "only_plan") {
    if (value < -1 || value >= (int64_t)e->plans.size()) return engine_fail(e, VSGM_EINVAL, "only_plan must be -1 or a plan index");
    e->only_plan = (int)value;
    return VSGM_OK;
  }
  if (n == "streams") {
    if (value < 1 || value > 64) return engine_fail(e, VSGM_EINVAL, "streams must be 1..64");
    e->streams = (int)value;
    return VSGM_OK;
  }
  if (n == "hybrid_steps") {
    if (value < 0) return engine_fail(e, VSGM_EINVAL, "hybrid_steps must be >= 0");
    e->hybrid_steps = (uint64_t)value;
    return VSGM_OK;
  }
  if (n == "relabel") {
    e->relabel = value != 0;
    return VSGM_OK;
  }
  if (n == "root_stride") {
    if (value < 1) return engine_fail(e, VSGM_EINVAL, "root_stride must be >= 1");
    e->root_stride = (uint64_t)value;
    return VSGM_OK;
  }
  return engine_fail(e, VSGM_EINVAL, "unknown option " + n);
}

int vsgm_set_option(vsgm_engine* e, const char* name, int64_t value) { return vsgm_set_plan_option(e, -1, name, value); }

int vsgm_set_profiling(vsgm_engine* e, int on) {
  if (!e) return engine_fail(nullptr, VSGM_EINVAL, "null engine");
  e->profiling = on != 0;
  return VSGM_OK;
}

void* vsgm_engine_stream(vsgm_engine* e) { return e ? (void*)e->stream : nullptr; }

const char* vsgm_engine_error(vsgm_engine* e) { return e ? e->err.c_str() : g_engine_err.c_str(); }

int vsgm_add_view(vsgm_engine* e, uint64_t V, const uint64_t* row_ptrs, const uint32_t* cols, uint64_t n_cols, const uint32_t* sources,
                  uint64_t n_sources, int* view_id) {
  if (!e || !row_ptrs || (n_cols && !cols) || (n_sources && !sources) || !view_id) return engine_fail(e, VSGM_EINVAL, "null view argument");
  if (V == 0 || V >= 0xffffffffull || row_ptrs[V] != n_cols) return engine_fail(e, VSGM_EINVAL, "row_ptrs[V] != n_cols");
  for (uint64_t i = 0; i < n_sources; i++)
    if (sources[i] >= V) return engine_fail(e, VSGM_EINVAL, "source id out of range");
  return guarded(e, [&] {
    CK(cudaSetDevice(e->device));
    vsgm_engine::ResidentView r;
    r.V = V;
    r.n_cols = n_cols;
    r.n_src = n_sources;
    for (uint64_t v = 0; v < V; v++) r.max_deg = std::max<uint64_t>(r.max_deg, row_ptrs[v + 1] - row_ptrs[v]);
    r.h_deg_src.resize(n_sources);
    for (uint64_t i = 0; i < n_sources; i++) r.h_deg_src[i] = row_ptrs[sources[i] + 1] - row_ptrs[sources[i]];
    CK(cudaMalloc(&r.rp, sizeof(uint64_t) * (V + 1)));
    CK(cudaMalloc(&r.ci, sizeof(uint32_t) * std::max<uint64_t>(1, n_cols)));
    CK(cudaMalloc(&r.src, sizeof(uint32_t) * std::max<uint64_t>(1, n_sources)));
    CK(cudaMemcpyAsync(r.rp, row_ptrs, sizeof(uint64_t) * (V + 1), cudaMemcpyHostToDevice, e->stream));
    if (n_cols) CK(cudaMemcpyAsync(r.ci, cols, sizeof(uint32_t) * n_cols, cudaMemcpyHostToDevice, e->stream));
    if (n_sources) CK(cudaMemcpyAsync(r.src, sources, sizeof(uint32_t) * n_sources, cudaMemcpyHostToDevice, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    e->rviews.push_back(std::move(r));
    *view_id = (int)e->rviews.size() - 1;
  });
}

int vsgm_run_batched(vsgm_engine* e, const int* view_ids, int n_views, const int* plan_ids, int n_plans, uint64_t* counts) {
  if (!e || !view_ids || !plan_ids || !counts || n_views < 1 || n_plans < 1) return engine_fail(e, VSGM_EINVAL, "bad batched request");
  for (int k = 0; k < n_views; k++)
    if (view_ids[k] < 0 || view_ids[k] >= (int)e->rviews.size()) return engine_fail(e, VSGM_EINVAL, "unknown view id");
  for (int k = 0; k < n_plans; k++)
    if (plan_ids[k] < 0 || plan_ids[k] >= (int)e->plans.size()) return engine_fail(e, VSGM_EINVAL, "unknown plan id");
  return guarded(e, [&] {
    CK(cudaSetDevice(e->device));
    e->arena.top = 0;
    e->run_hybrid(view_ids, n_views, plan_ids, n_plans, counts, nullptr);
  });
}

int vsgm_run_pairs(vsgm_engine* e, const int* plan_ids, const int* view_ids, int n_pairs, uint64_t* counts) {
  if (!e || !view_ids || !plan_ids || !counts || n_pairs < 1) return engine_fail(e, VSGM_EINVAL, "bad pairs request");
  for (int k = 0; k < n_pairs; k++) {
    if (view_ids[k] < 0 || view_ids[k] >= (int)e->rviews.size()) return engine_fail(e, VSGM_EINVAL, "unknown view id");
    if (plan_ids[k] < 0 || plan_ids[k] >= (int)e->plans.size()) return engine_fail(e, VSGM_EINVAL, "unknown plan id");
  }
  return guarded(e, [&] {
    CK(cudaSetDevice(e->device));
    e->arena.top = 0;
    // the distinct plans and views, and the mask of the requested pairs
    std::vector<int> P, W;
    std::vector<int> pi(n_pairs), wi(n_pairs);
    for (int k = 0; k < n_pairs; k++) {
      auto fp = std::find(P.begin(), P.end(), plan_ids[k]);
      pi[k] = (int)(fp - P.begin());
      if (fp == P.end()) P.push_back(plan_ids[k]);
      auto fw = std::find(W.begin(), W.end(), view_ids[k]);
      wi[k] = (int)(fw - W.begin());
      if (fw == W.end()) W.push_back(view_ids[k]);
    }
    std::vector<uint8_t> mask(P.size() * W.size(), 0);
    for (int k = 0; k < n_pairs; k++) mask[(size_t)pi[k] * W.size() + wi[k]] = 1;
    std::vector<uint64_t> all(P.size() * W.size(), 0);
    e->run_hybrid(W.data(), (int)W.size(), P.data(), (int)P.size(), all.data(), mask.data());
    for (int k = 0; k < n_pairs; k++) counts[k] = all[(size_t)pi[k] * W.size() + wi[k]];
  });
}

int vsgm_run_batched_ex(vsgm_engine* e, const int* view_ids, int n_views, const int* plan_ids, int n_plans, uint64_t step_budget, uint64_t* counts,
                        uint64_t* level_paths, uint32_t* overflow) {
  if (!e || !view_ids || !plan_ids || !counts || n_views < 1 || n_plans < 1) return engine_fail(e, VSGM_EINVAL, "bad batched request");
  for (int k = 0; k < n_views; k++)
    if (view_ids[k] < 0 || view_ids[k] >= (int)e->rviews.size()) return engine_fail(e, VSGM_EINVAL, "unknown view id");
  for (int k = 0; k < n_plans; k++)
    if (plan_ids[k] < 0 || plan_ids[k] >= (int)e->plans.size()) return engine_fail(e, VSGM_EINVAL, "unknown plan id");
  return guarded(e, [&] {
    CK(cudaSetDevice(e->device));
    e->arena.top = 0;
    e->run_batched(view_ids, n_views, plan_ids, n_plans, counts, level_paths, step_budget, overflow);
  });
}

int vsgm_get_batch_stats(vsgm_engine* e, vsgm_batch_stats* out) {
  if (!e || !out) return engine_fail(e, VSGM_EINVAL, "null argument");
  *out = e->bstats;
  return VSGM_OK;
}

int vsgm_host_alloc(uint64_t bytes, void** out) {
  if (!out) return engine_fail(nullptr, VSGM_EINVAL, "null argument");
  *out = nullptr;
  return guarded(nullptr, [&] { CK(cudaMallocHost(out, std::max<uint64_t>(bytes, 1))); });
}

int vsgm_host_free(void* p) {
  return guarded(nullptr, [&] {
    if (p) CK(cudaFreeHost(p));
  });
}

int vsgm_prefetch_view(vsgm_engine* e, const uint32_t* vertices, uint64_t n_vertices, const uint64_t* offsets, const uint32_t* cols,
                       const uint32_t* sources, uint64_t n_sources) {
  if (!e || !offsets || (n_vertices && !vertices) || (n_sources && !sources)) return engine_fail(e, VSGM_EINVAL, "null view argument");
  if (e->bk_pending) return engine_fail(e, VSGM_EINVAL, "a prefetched view is waiting: vsgm_swap_view first");
  const uint64_t n_cols = offsets[n_vertices];
  if (n_cols && !cols) return engine_fail(e, VSGM_EINVAL, "null view argument");
  if (offsets[0] != 0) return engine_fail(e, VSGM_EINVAL, "offsets[0] != 0");
  for (uint64_t i = 0; i < n_vertices; i++) {
    if (vertices[i] >= e->V || (i && vertices[i] <= vertices[i - 1])) return engine_fail(e, VSGM_EINVAL, "vertices must ascend and be < V");
    if (offsets[i + 1] < offsets[i]) return engine_fail(e, VSGM_EINVAL, "offsets must not decrease");
  }
  for (uint64_t i = 0; i < n_sources; i++)
    if (sources[i] >= e->V) return engine_fail(e, VSGM_EINVAL, "source id out of range");
  return guarded(e, [&] {
    CK(cudaSetDevice(e->device));
    auto grow = [](auto** p, uint64_t* cap, uint64_t need) {
      if (*p && *cap >= need) return;
      if (*p) CK(cudaFree(*p));
      *p = nullptr;
      CK(cudaMalloc((void**)p, sizeof(**p) * std::max<uint64_t>(need, 1)));
      *cap = need;
    };
    uint64_t rp_cap = e->bk_rp ? e->V + 1 : 0;
    grow(&e->bk_rp, &rp_cap, e->V + 1);
    grow(&e->bk_ci, &e->bk_cols_cap, n_cols);
    grow(&e->bk_src, &e->bk_src_cap, n_sources);
    uint64_t off_cap = e->bk_off ? e->bk_vert_cap + 1 : 0;
    grow(&e->bk_vert, &e->bk_vert_cap, n_vertices);
    grow(&e->bk_off, &off_cap, n_vertices + 1);
    cudaStream_t cs = e->copy_stream;
    if (n_vertices) CK(cudaMemcpyAsync(e->bk_vert, vertices, sizeof(uint32_t) * n_vertices, cudaMemcpyHostToDevice, cs));
    CK(cudaMemcpyAsync(e->bk_off, offsets, sizeof(uint64_t) * (n_vertices + 1), cudaMemcpyHostToDevice, cs));
    if (n_cols) CK(cudaMemcpyAsync(e->bk_ci, cols, sizeof(uint32_t) * n_cols, cudaMemcpyHostToDevice, cs));
    if (n_sources) CK(cudaMemcpyAsync(e->bk_src, sources, sizeof(uint32_t) * n_sources, cudaMemcpyHostToDevice, cs));
    k_rows_from_compact<<<e->grid_threads(e->V + 1), 256, 0, cs>>>(e->bk_vert, n_vertices, e->bk_off, e->V, e->bk_rp);
    CK(cudaGetLastError());
    CK(cudaEventRecord(e->ev_copy, cs));
    e->bk_n_cols = n_cols;
    e->bk_n_src = n_sources;
    e->bk_pending = true;
  });
}

int vsgm_view_released(vsgm_engine* e) {
  if (!e) return engine_fail(nullptr, VSGM_EINVAL, "null engine");
  return guarded(e, [&] {
    CK(cudaSetDevice(e->device));
    CK(cudaEventSynchronize(e->ev_copy));
  });
}

int vsgm_swap_view(vsgm_engine* e) {
  if (!e) return engine_fail(nullptr, VSGM_EINVAL, "null engine");
  if (!e->bk_pending) return engine_fail(e, VSGM_EINVAL, "no prefetched view");
  return guarded(e, [&] {
    CK(cudaSetDevice(e->device));
    CK(cudaStreamWaitEvent(e->stream, e->ev_copy, 0));  // the engine's stream, not the host, waits for the copies
    std::swap(e->own_rp, e->bk_rp);
    std::swap(e->own_ci, e->bk_ci);
    std::swap(e->cols_cap, e->bk_cols_cap);
    std::swap(e->own_src, e->bk_src);
    std::swap(e->src_cap, e->bk_src_cap);
    e->d_rp = e->own_rp;
    e->d_ci = e->own_ci;
    e->d_src = e->own_src;
    e->n_cols = e->bk_n_cols;
    e->n_src = e->bk_n_src;
    e->have_view = true;
    e->bk_pending = false;
    e->up_of = nullptr;  // a new view (the same address may come back with other rows)
  });
}

int vsgm_destroy(vsgm_engine* e) {
  if (!e) return VSGM_OK;
  cudaSetDevice(e->device);
  for (vsgm_engine* h : e->helpers) vsgm_engine::release_helper(h);
  e->helpers.clear();
  if (e->stream) cudaStreamSynchronize(e->stream);
  cudaFree(e->arena.base);
  cudaFree(e->d_counts);
  cudaFree(e->own_rp);
  cudaFree(e->own_ci);
  cudaFree(e->own_src);
  cudaFree(e->g_rp);
  cudaFree(e->g_ci);
  cudaFree(e->g_new);
  cudaFree(e->d_up);
  for (auto& r : e->rviews) {
    cudaFree(r.rp);
    cudaFree(r.ci);
    cudaFree(r.src);
  }
  if (e->h_pinned) cudaFreeHost(e->h_pinned);
  if (e->ev0) cudaEventDestroy(e->ev0);
  if (e->ev1) cudaEventDestroy(e->ev1);
  if (e->ev_h0) cudaEventDestroy(e->ev_h0);
  if (e->ev_h1) cudaEventDestroy(e->ev_h1);
  if (e->copy_stream) cudaStreamSynchronize(e->copy_stream);
  cudaFree(e->bk_rp);
  cudaFree(e->bk_ci);
  cudaFree(e->bk_src);
  cudaFree(e->bk_vert);
  cudaFree(e->bk_off);
  if (e->ev_copy) cudaEventDestroy(e->ev_copy);
  if (e->copy_stream) cudaStreamDestroy(e->copy_stream);
  if (e->aux_stream) cudaStreamSynchronize(e->aux_stream);
  if (e->ev_fork) cudaEventDestroy(e->ev_fork);
  if (e->ev_join) cudaEventDestroy(e->ev_join);
  if (e->aux_stream) cudaStreamDestroy(e->aux_stream);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
  return VSGM_OK;
}

}  // extern "C"

// ------------------------------------------------- allocation-free entry point
//
// vsgm_count_noalloc counts one plan over one view that is already in device
// memory without allocating anything: it runs the persistent depth-first kernel
// (k_dfs, the kernel behind vsgm_run_batched) with every buffer it needs - task
// list, counters and the per-warp candidate scratch - carved out of one
// file-scope device array of fixed size.  It is meant for callers that must not
// call cudaMalloc: code running inside a memory pool or allocator that owns all
// device memory of the process, code paths whose memory footprint has to be known
// before they run, and embeddings whose host side cannot manage device
// allocations.  Every GPU that loads this library holds the array until the
// process exits.
namespace {

constexpr size_t kNoAllocBytes = 48ull << 20;  // the whole static scratch
constexpr unsigned kNoAllocBlocks = 64;         // 64 blocks x 8 warps
constexpr uint64_t kNoAllocWarps = (uint64_t)kNoAllocBlocks * kDfsWarps;
constexpr uint64_t kNoAllocMaxTasks = 16384;
// layout: [0, 256) counters | [256, 1280) plan + view | tasks | per-warp scratch
constexpr size_t kNoAllocHeader = 256;
constexpr size_t kNoAllocDescOff = kNoAllocHeader;  // the plan and view descriptors follow the counters
constexpr size_t kNoAllocTaskOff = 1280;
constexpr size_t kNoAllocScratchOff = (kNoAllocTaskOff + kNoAllocMaxTasks * sizeof(DfsTask) + 255) & ~(size_t)255;
constexpr uint64_t kNoAllocWarpU32 = (kNoAllocBytes - kNoAllocScratchOff) / (kNoAllocWarps * sizeof(uint32_t));
// the view descriptor (8-byte pointers) follows the plan at the next 16-byte boundary
constexpr size_t kNoAllocViewOff = kNoAllocDescOff + ((sizeof(DfsPlan) + 15) & ~(size_t)15);
static_assert(kNoAllocViewOff % alignof(DfsView) == 0 && kNoAllocTaskOff % alignof(DfsTask) == 0, "descriptor alignment");
static_assert(kNoAllocViewOff + sizeof(DfsView) <= kNoAllocTaskOff, "plan + view must fit their slot");
static_assert(kNoAllocWarpU32 == 24319, "the documented limit (plan ops x max degree) follows the layout");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// device address of g_noalloc_scratch per device (the host-side symbol is not a
// device address; cudaGetSymbolAddress gives the real one), with the id of the
// context it was looked up in: a context that is torn down and rebuilt (for
// example after cudaDeviceReset) loads the module again, and the array may then
// sit at another address
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_ptr[128] = {};
unsigned long long g_noalloc_ctx[128] = {};

// Unique id of the calling thread's current context (ids are never reused within
// a process), or 0 when the driver cannot tell.  The driver calls are reached
// through the runtime's entry-point query so that the library does not link
// against the driver library itself.
unsigned long long current_context_id() {
  typedef CUresult (*GetCurrent)(CUcontext*);
  typedef CUresult (*GetId)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q;
    void* f = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
      get_current = (GetCurrent)f;
    f = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
      get_id = (GetId)f;
  });
  if (!get_current || !get_id) return 0;
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (get_current(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
  return id;
}

struct NoAllocCounters {
  unsigned long long head;
  unsigned long long count;
  unsigned long long max_degree;
  unsigned int status;
};

__global__ void k_noalloc_max_degree(const uint64_t* __restrict__ rp, uint64_t V, NoAllocCounters* c) {
  unsigned long long m = 0;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
    const unsigned long long d = rp[v + 1] - rp[v];
    if (d > m) m = d;
  }
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long y = __shfl_down_sync(kFull, m, o);
    if (y > m) m = y;
  }
  if ((threadIdx.x & 31) == 0 && m) atomicMax(&c->max_degree, m);
}

__global__ void k_noalloc_tasks(DfsTask* tasks, uint64_t n_tasks, uint64_t n_sources, uint64_t chunk) {
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n_tasks; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t r0 = t * chunk;
    tasks[t] = DfsTask{0u, 0u, r0, r0 + chunk < n_sources ? r0 + chunk : n_sources, 0u, 0u};
  }
}

int noalloc_fail(const std::string& msg) { return engine_fail(nullptr, VSGM_EINVAL, msg); }

}  // namespace

extern "C" int vsgm_count_noalloc(int device, const vsgm_plan* plan, uint64_t V, const uint64_t* d_row_ptrs, const uint32_t* d_cols,
                                  const uint32_t* d_sources, uint64_t n_sources, void* stream, uint64_t* count) {
  if (!plan || !count || !d_row_ptrs || (n_sources && !d_sources)) return noalloc_fail("null argument");
  if (V == 0 || V >= 0xffffffffull) return noalloc_fail("vertex count must be 1 .. 2^32-2");
  if (plan->n_vertices < 2 || plan->n_vertices > VSGM_MAX_QV || plan->n_ops < 2 || plan->n_ops > VSGM_MAX_OPS || plan->op_type[0] != VSGM_MATERIALIZE)
    return noalloc_fail("malformed plan");
  if (device < 0 || device >= 128) return noalloc_fail("device index out of range");
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  cudaStream_t s = (cudaStream_t)stream;
  int rc = guarded(nullptr, [&] {
    CK(cudaSetDevice(device));
    unsigned char* base = nullptr;
    {
      std::lock_guard<std::mutex> lock(g_noalloc_mu);
      // once per device (and again whenever the device's context has changed), with
      // that device current; an unknown context id (0) means: look up every call
      const unsigned long long ctx = current_context_id();
      if (!g_noalloc_ptr[device] || ctx == 0 || ctx != g_noalloc_ctx[device]) {
        g_noalloc_ptr[device] = nullptr;
        CK(cudaGetSymbolAddress((void**)&g_noalloc_ptr[device], g_noalloc_scratch));
        g_noalloc_ctx[device] = ctx;
      }
      base = g_noalloc_ptr[device];
    }
    NoAllocCounters* ctr = (NoAllocCounters*)base;
    DfsPlan* d_plan = (DfsPlan*)(base + kNoAllocDescOff);
    DfsView* d_view = (DfsView*)(base + kNoAllocViewOff);
    DfsTask* d_tasks = (DfsTask*)(base + kNoAllocTaskOff);
    uint32_t* scratch = (uint32_t*)(base + kNoAllocScratchOff);
    // the array keeps the previous call's contents: clear the counters
    CK(cudaMemsetAsync(ctr, 0, sizeof(NoAllocCounters), s));
    k_noalloc_max_degree<<<256, 256, 0, s>>>(d_row_ptrs, V, ctr);
    CK(cudaGetLastError());
    NoAllocCounters h{};
    CK(cudaMemcpyAsync(&h, ctr, sizeof(h), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const uint64_t cap = std::max<uint64_t>(1, h.max_degree);
    const uint32_t levels = plan->n_ops;
    if ((uint64_t)levels * cap > kNoAllocWarpU32)
      throw std::invalid_argument("view too large for the allocation-free path: plan ops x maximum degree = " + std::to_string(levels * cap) +
                                  ", limit " + std::to_string(kNoAllocWarpU32));
    if (n_sources == 0) {
      *count = 0;
      return;
    }
    const DfsPlan hp = vsgm_engine::to_dfs(*plan);
    const DfsView hv{d_row_ptrs, d_cols, d_sources};
    CK(cudaMemcpyAsync(d_plan, &hp, sizeof(hp), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d_view, &hv, sizeof(hv), cudaMemcpyHostToDevice, s));
    const uint64_t chunk = std::max<uint64_t>(16, (n_sources + kNoAllocMaxTasks - 1) / kNoAllocMaxTasks);
    const uint64_t n_tasks = (n_sources + chunk - 1) / chunk;
    k_noalloc_tasks<<<64, 256, 0, s>>>(d_tasks, n_tasks, n_sources, chunk);
    CK(cudaGetLastError());
    k_dfs<<<kNoAllocBlocks, kDfsWarps * kWarp, 0, s>>>(d_plan, d_view, d_tasks, n_tasks, &ctr->head, scratch, cap, levels, 1u, &ctr->count,
                                                       &ctr->status, nullptr, 0, nullptr);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(&h, ctr, sizeof(h), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (h.status) throw std::invalid_argument("a candidate set did not fit in the allocation-free scratch");
    *count = h.count;
  });
  if (prev >= 0) cudaSetDevice(prev);
  return rc;
}
