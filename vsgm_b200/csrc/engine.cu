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
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "kernels.cuh"
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

  Arena arena;
  unsigned long long* d_counts = nullptr;  // [n_plans]
  unsigned long long* d_bytes = nullptr;   // [1] profiling byte counter
  uint64_t* h_pinned = nullptr;            // small pinned staging

  std::vector<uint64_t> totals;
  std::vector<vsgm_plan_stats> stats;
  bool profiling = false;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::string err;

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
    const uint64_t reserve = 1 << 20;
    uint64_t avail = arena.avail() > reserve ? arena.avail() - reserve : 0;
    int remaining = (int)plan->n_ops - i;
    return avail / (uint64_t)std::max(2, remaining);
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
      case VSGM_FILTER_COMPUTE: op_filter(i, f, u, p.filter_cond[u], true); break;
      case VSGM_MATERIALIZE: op_materialize(i, f, u); break;
      default: throw OutOfMemory{"execution sequence holds an op this engine does not run"};
    }
  }

  static Frame slice(const Frame& f, uint64_t a, uint64_t b) {
    Frame g = f;
    g.P = b - a;
    for (int k = 0; k < VSGM_MAX_QV; k++) {
      if (g.col[k]) g.col[k] += a;
      if (g.cbeg[k]) g.cbeg[k] += a;
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
  void launch_write_nb(const OpDesc& d, const Frame& f, const uint64_t* off, uint32_t* pool, uint32_t* len) {
    k_compute_write<NB><<<grid_warps(f.P), 256, 0, stream>>>(f, d, d_rp, d_ci, off, pool, len);
  }

  void op_compute(int i, const Frame& f, int u) {
    const vsgm_plan& p = *plan;
    OpDesc d = make_desc(i, p.compute_cond[u]);
    bool has_ne = false;
    for (int k = 0; k < d.nc; k++) has_ne |= (d.cop[k] == VSGM_NON_EQUAL);
    if (d.nb == 1 && !has_ne) {
      // the candidate set is a slice of one adjacency list
      const uint64_t per = sizeof(uint64_t) + sizeof(uint32_t);
      uint64_t a = 0;
      while (a < f.P) {
        uint64_t room = level_budget(i) / per;
        if (room == 0) throw OutOfMemory{"HBM budget exhausted (COMPUTE slice)"};
        uint64_t b = std::min(f.P, a + room);
        Mark m(arena);
        Frame g = slice(f, a, b);
        uint64_t* beg = arena.take_n<uint64_t>(g.P, "candidate begins");
        uint32_t* len = arena.take_n<uint32_t>(g.P, "candidate lengths");
        begin_op();
        CK(cudaMemsetAsync(d_bytes + 1, 0, sizeof(unsigned long long), stream));
        k_compute_slice<<<grid_threads(g.P), 256, 0, stream>>>(g, d, d_rp, d_ci, beg, len, d_bytes + 1);
        CK(cudaGetLastError());
        end_op(i, 1);
        st->op_outputs[i] += read_u64((const uint64_t*)(d_bytes + 1));
        g.cbeg[u] = beg;
        g.clen[u] = len;
        g.pool[u] = d_ci;
        st->batches++;
        process(i + 1, g);
        a = b;
      }
      return;
    }
    // general case: size, scan, write
    Mark m(arena);
    uint64_t* off = arena.take_n<uint64_t>(f.P + 1, "candidate offsets");
    begin_op();
    k_compute_size<<<grid_warps(f.P), 256, 0, stream>>>(f, d, d_rp, d_ci, off);
    CK(cudaGetLastError());
    scan(off, false, f.P, off);
    end_op(i, 2);
    uint64_t a = 0;
    while (a < f.P) {
      // each path needs 4 bytes of length plus 4 per candidate
      uint64_t b = split_point(off, a, f.P, 4, 4 + 256, level_budget(i));
      Mark mb(arena);
      Frame g = slice(f, a, b);
      uint64_t lo = read_u64(off + a), hi = read_u64(off + b);
      uint32_t* pool = arena.take_n<uint32_t>(hi - lo, "candidate pool");
      uint32_t* len = arena.take_n<uint32_t>(g.P, "candidate lengths");
      uint32_t* pool_eff = pool - lo;  // so that pool_eff + off[p] lies inside pool
      begin_op();
      switch (d.nb) {
        case 1: launch_write_nb<1>(d, g, off + a, pool_eff, len); break;
        case 2: launch_write_nb<2>(d, g, off + a, pool_eff, len); break;
        case 3: launch_write_nb<3>(d, g, off + a, pool_eff, len); break;
        case 4: launch_write_nb<4>(d, g, off + a, pool_eff, len); break;
        case 5: launch_write_nb<5>(d, g, off + a, pool_eff, len); break;
        case 6: launch_write_nb<6>(d, g, off + a, pool_eff, len); break;
        default: throw OutOfMemory{"pattern vertex with no backward neighbour"};
      }
      CK(cudaGetLastError());
      end_op(i, 1);
      st->op_outputs[i] += hi - lo;
      g.cbeg[u] = off + a;
      g.clen[u] = len;
      g.pool[u] = pool_eff;
      st->batches++;
      process(i + 1, g);
      a = b;
    }
  }

  // keep the candidates of u that satisfy conds; then continue with op i+1
  // (FILTER_COMPUTE), or return the filtered frame to the caller (MATERIALIZE)
  void op_filter(int i, const Frame& f, int u, const vsgm_conds& conds, bool continue_next) {
    OpDesc d = make_desc(i, conds);
    d.u = (uint8_t)u;
    Mark m(arena);
    uint64_t* off = arena.take_n<uint64_t>(f.P + 1, "filter offsets");
    begin_op();
    scan(f.clen[u], true, f.P, off);
    end_op(i, 2);
    uint64_t a = 0;
    while (a < f.P) {
      uint64_t b = split_point(off, a, f.P, 4, 4 + 256, level_budget(i));
      Mark mb(arena);
      Frame g = slice(f, a, b);
      uint64_t lo = read_u64(off + a), hi = read_u64(off + b);
      uint32_t* pool = arena.take_n<uint32_t>(hi - lo, "filtered pool");
      uint32_t* len = arena.take_n<uint32_t>(g.P, "filtered lengths");
      uint32_t* pool_eff = pool - lo;
      begin_op();
      k_filter<<<grid_warps(g.P), 256, 0, stream>>>(g, d, off + a, pool_eff, len);
      CK(cudaGetLastError());
      end_op(i, 1);
      g.cbeg[u] = off + a;
      g.clen[u] = len;
      g.pool[u] = pool_eff;
      st->batches++;
      if (continue_next) {
        process(i + 1, g);
      } else {
        materialize_frame(i, g, u);
      }
      a = b;
    }
  }

  void op_materialize(int i, const Frame& f, int u) {
    const vsgm_plan& p = *plan;
    if (p.materialize_cond[u].count > 0) {
      op_filter(i, f, u, p.materialize_cond[u], false);
    } else {
      materialize_frame(i, f, u);
    }
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
      for (int k = 0; k < VSGM_MAX_QV; k++) g.pool[k] = f.pool[k];
      for (int k = 0; k < x.nm; k++) g.col[x.m[k]] = arena.take_n<uint32_t>(n, "child column");
      g.col[u] = arena.take_n<uint32_t>(n, "child column");
      for (int k = 0; k < x.ncu; k++) {
        g.cbeg[x.cu[k]] = arena.take_n<uint64_t>(n, "child candidate begins");
        g.clen[x.cu[k]] = arena.take_n<uint32_t>(n, "child candidate lengths");
      }
      g.pool[u] = nullptr;
      // k_expand writes children [c0, c0+n) at positions [0, n): shift the outputs
      Frame shifted = g;
      for (int k = 0; k < VSGM_MAX_QV; k++) {
        if (shifted.col[k]) shifted.col[k] -= c0;
        if (shifted.cbeg[k]) shifted.cbeg[k] -= c0;
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

  void run_plan(int pi) {
    plan = &plans[pi];
    st = &stats[pi];
    d_total = d_counts + pi;
    if (n_src == 0) return;
    Frame f;
    std::memset(&f, 0, sizeof(f));
    f.P = n_src;
    f.col[plan->op_vertex[0]] = d_src;
    st->op_paths[0] += n_src;
    st->op_outputs[0] += n_src;
    process(1, f);
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
  }
  vsgm_engine* e = new vsgm_engine();
  e->device = device;
  e->V = V;
  e->plans.assign(plans, plans + n_plans);
  e->max_sources = max_sources;
  e->totals.assign(n_plans, 0);
  e->stats.assign(n_plans, vsgm_plan_stats{});
  int rc = guarded(e, [&] {
    CK(cudaSetDevice(device));
    CK(cudaDeviceGetAttribute(&e->sms, cudaDevAttrMultiProcessorCount, device));
    CK(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&e->ev0));
    CK(cudaEventCreate(&e->ev1));
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
  return VSGM_OK;
}

int vsgm_match(vsgm_engine* e) {
  if (!e) return engine_fail(nullptr, VSGM_EINVAL, "null engine");
  if (!e->have_view) return engine_fail(e, VSGM_EINVAL, "no view transferred");
  return guarded(e, [&] {
    CK(cudaSetDevice(e->device));
    const int n = (int)e->plans.size();
    CK(cudaMemsetAsync(e->d_counts, 0, sizeof(unsigned long long) * (n + 2), e->stream));
    for (int k = 0; k < n; k++) {
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

int vsgm_set_profiling(vsgm_engine* e, int on) {
  if (!e) return engine_fail(nullptr, VSGM_EINVAL, "null engine");
  e->profiling = on != 0;
  return VSGM_OK;
}

void* vsgm_engine_stream(vsgm_engine* e) { return e ? (void*)e->stream : nullptr; }

const char* vsgm_engine_error(vsgm_engine* e) { return e ? e->err.c_str() : g_engine_err.c_str(); }

int vsgm_destroy(vsgm_engine* e) {
  if (!e) return VSGM_OK;
  cudaSetDevice(e->device);
  if (e->stream) cudaStreamSynchronize(e->stream);
  cudaFree(e->arena.base);
  cudaFree(e->d_counts);
  cudaFree(e->own_rp);
  cudaFree(e->own_ci);
  cudaFree(e->own_src);
  if (e->h_pinned) cudaFreeHost(e->h_pinned);
  if (e->ev0) cudaEventDestroy(e->ev0);
  if (e->ev1) cudaEventDestroy(e->ev1);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
  return VSGM_OK;
}

}  // extern "C"
