"""vsgm_b200: B200-native subgraph enumeration/counting behind VSGM's pm_pipeline surface.

Python is a thin layer over the C ABI (include/vsgm.h); every count comes from
the CUDA engine in libvsgm_b200.so.  Names follow the reference:

    plan_pattern(p)       Pattern((PresetPatternType)p, false) + Plan::Optimize
    plan_clique(k)        Clique(k) + Plan::Optimize                (-kc)
    plan_graphlets(k)     Graphlet(k)->GetQueries(), planned        (-km)
    plan_query(adj)       Query(n, e, adj) + Plan::Optimize
    read_csr_bin / write_csr_bin / read_vbmap                       (src/graph/graph_io.h, src/view)
    materialize_view      ViewBin::Materialize                      (src/view/view_bin.h:66-142)
    Engine                PipelineExecutor                          (src/executor/pipeline_executor.h)
"""
import ctypes as C

import numpy as np

from . import capi
from .capi import Plan, PlanStats, VsgmError

__all__ = [
    "Plan", "PlanStats", "VsgmError", "Graph", "Engine",
    "plan_pattern", "plan_clique", "plan_query", "plan_graphlets", "plan_reorder", "automorphisms",
    "gen_rmat", "gen_chung_lu", "random_pattern", "read_csr_bin", "write_csr_bin", "read_vbmap", "write_vbmap",
    "csr_defects", "materialize_view", "sources_of_bins", "degree_relabel",
]


def _L():
    return capi.lib()


# ------------------------------------------------------------------ planning
def plan_pattern(pattern_id):
    p = Plan()
    capi.check(_L().vsgm_plan_pattern(int(pattern_id), C.byref(p)))
    return p


def plan_clique(k):
    p = Plan()
    capi.check(_L().vsgm_plan_clique(int(k), C.byref(p)))
    return p


def plan_query(neighbours):
    """Plan of a connected pattern given as neighbour lists (Query(n, e, adj), src/query/query.h:62-78)."""
    n = len(neighbours)
    bits = (C.c_uint8 * capi.MAX_QV)()
    for i, row in enumerate(neighbours):
        for j in row:
            bits[i] |= 1 << int(j)
    p = Plan()
    capi.check(_L().vsgm_plan_query(n, bits, C.byref(p)))
    return p


def plan_query_bits(n, bits):
    arr = (C.c_uint8 * capi.MAX_QV)(*[int(b) for b in list(bits)[:capi.MAX_QV]])
    p = Plan()
    capi.check(_L().vsgm_plan_query(int(n), arr, C.byref(p)))
    return p


def plan_graphlets(k):
    arr = (Plan * 64)()
    n = C.c_int()
    capi.check(_L().vsgm_plan_graphlets(int(k), arr, 64, C.byref(n)))
    return [arr[i] for i in range(n.value)]


def plan_reorder(base, seq):
    s = (C.c_uint8 * capi.MAX_QV)(*[int(x) for x in seq])
    p = Plan()
    capi.check(_L().vsgm_plan_reorder(C.byref(base), s, C.byref(p)))
    return p


def automorphisms(plan):
    return int(_L().vsgm_plan_automorphisms(C.byref(plan)))


# -------------------------------------------------------------------- graphs
class Graph:
    """Undirected CSR: row_ptrs (uint64, V+1), cols (uint32, E = 2 x undirected edges)."""

    def __init__(self, row_ptrs, cols):
        self.row_ptrs = np.ascontiguousarray(row_ptrs, dtype=np.uint64)
        self.cols = np.ascontiguousarray(cols, dtype=np.uint32)
        self.V = len(self.row_ptrs) - 1

    @property
    def E(self):
        return len(self.cols)

    def degrees(self):
        return np.diff(self.row_ptrs)


def _take(ptr_u64, ptr_u32, V, E):
    rp = np.ctypeslib.as_array(ptr_u64, shape=(V + 1,)).copy()
    ci = np.ctypeslib.as_array(ptr_u32, shape=(max(E, 1),))[:E].copy() if E else np.zeros(0, np.uint32)
    _L().vsgm_free(C.cast(ptr_u64, C.c_void_p))
    _L().vsgm_free(C.cast(ptr_u32, C.c_void_p))
    return Graph(rp, ci)


def gen_rmat(scale, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=1, threads=0):
    V, E = C.c_uint64(), C.c_uint64()
    rp, ci = C.POINTER(C.c_uint64)(), C.POINTER(C.c_uint32)()
    capi.check(_L().vsgm_gen_rmat(scale, edge_factor, a, b, c, seed, threads, C.byref(V), C.byref(E), C.byref(rp), C.byref(ci)))
    return _take(rp, ci, V.value, E.value)


def gen_chung_lu(V, target_edges, gamma, max_degree, seed, threads=0):
    E = C.c_uint64()
    rp, ci = C.POINTER(C.c_uint64)(), C.POINTER(C.c_uint32)()
    capi.check(_L().vsgm_gen_chung_lu(V, target_edges, gamma, max_degree, seed, threads, C.byref(E), C.byref(rp), C.byref(ci)))
    return _take(rp, ci, V, E.value)


def random_pattern(seed, counter, n_min=3, n_max=6, p=0.5):
    """Returns (n, adj_bits, next_counter)."""
    ctr = C.c_uint64(counter)
    n = C.c_int()
    bits = (C.c_uint8 * capi.MAX_QV)()
    capi.check(_L().vsgm_random_pattern(n_min, n_max, p, seed, C.byref(ctr), C.byref(n), bits))
    return n.value, [bits[i] for i in range(capi.MAX_QV)], ctr.value


def read_csr_bin(path, threads=0):
    """The .bin file straight into numpy arrays (parallel bulk reads, no copy)."""
    V, E = C.c_uint64(), C.c_uint64()
    capi.check(_L().vsgm_csr_bin_header(str(path).encode(), C.byref(V), C.byref(E)))
    rp = np.empty(V.value + 1, np.uint64)
    ci = np.empty(max(E.value, 1), np.uint32)
    capi.check(_L().vsgm_read_csr_bin_into(str(path).encode(), V.value, E.value, capi.ptr(rp, C.c_uint64), capi.ptr(ci, C.c_uint32), threads))
    return Graph(rp, ci[:E.value])


def write_csr_bin(path, g):
    capi.check(_L().vsgm_write_csr_bin(str(path).encode(), g.V, g.E, capi.ptr(g.row_ptrs, C.c_uint64), capi.ptr(g.cols, C.c_uint32)))


def read_vbmap(path, V):
    bins = np.zeros(V, np.int32)
    nb = C.c_int32()
    capi.check(_L().vsgm_read_vbmap(str(path).encode(), V, capi.ptr(bins, C.c_int32), C.byref(nb)))
    return bins, nb.value


def write_vbmap(path, bins, n_bins):
    bins = np.ascontiguousarray(bins, dtype=np.int32)
    capi.check(_L().vsgm_write_vbmap(str(path).encode(), len(bins), capi.ptr(bins, C.c_int32), int(n_bins)))


def csr_defects(g):
    return int(_L().vsgm_csr_defects(g.V, capi.ptr(g.row_ptrs, C.c_uint64), capi.ptr(g.cols, C.c_uint32)))


def degree_relabel(g, ascending=True, threads=0):
    """Relabel by (degree, id) rank; returns (relabelled graph, new_of_old)."""
    perm = np.empty(g.V, np.uint32)  # all three are fully written by the call
    rp = np.empty(g.V + 1, np.uint64)
    ci = np.empty(max(g.E, 1), np.uint32)
    capi.check(_L().vsgm_degree_relabel(g.V, capi.ptr(g.row_ptrs, C.c_uint64), capi.ptr(g.cols, C.c_uint32), 1 if ascending else 0, threads,
                                        capi.ptr(perm, C.c_uint32), capi.ptr(rp, C.c_uint64), capi.ptr(ci, C.c_uint32)))
    return Graph(rp, ci[:g.E]), perm


def sources_of_bins(bins, n_bins):
    """Per-bin ascending source lists (ViewBinManager::LoadViewBinPartition, src/view/view_bin_manager.h:43-60)."""
    order = np.argsort(bins, kind="stable").astype(np.uint32)
    counts = np.bincount(bins, minlength=n_bins)
    out, at = [], 0
    for b in range(n_bins):
        out.append(order[at:at + counts[b]])
        at += counts[b]
    return out


def materialize_view(g, sources, hop, root_degree=0, threads=0):
    """Full-V view CSR holding the rows of the sources' (hop-1)-neighbourhood."""
    sources = np.ascontiguousarray(sources, dtype=np.uint32)
    vrp = np.empty(g.V + 1, np.uint64)  # fully written by the call
    n = C.c_uint64()
    cap = g.E
    vci = np.empty(max(cap, 1), np.uint32)
    capi.check(_L().vsgm_view_materialize(g.V, capi.ptr(g.row_ptrs, C.c_uint64), capi.ptr(g.cols, C.c_uint32),
                                          capi.ptr(sources, C.c_uint32), len(sources), hop, root_degree, threads,
                                          capi.ptr(vrp, C.c_uint64), capi.ptr(vci, C.c_uint32), cap, C.byref(n)))
    return Graph(vrp, vci[:n.value])


# ------------------------------------------------- view-bin tools (device)
def features_1hop(g, device=0):
    """features -h 1 on the GPU: every row gains its own vertex (src/tools/features.cc:177-201)."""
    rp = np.empty(g.V + 1, np.uint64)
    ci = np.empty(g.E + g.V, np.uint32)
    capi.check(_L().vsgm_features_1hop(device, g.V, capi.ptr(g.row_ptrs, C.c_uint64), capi.ptr(g.cols, C.c_uint32), capi.ptr(rp, C.c_uint64),
                                       capi.ptr(ci, C.c_uint32)))
    return Graph(rp, ci)


def reference_rand_starts(k, threads=1):
    """The clusters the reference's random initialisation draws in a fresh process:
    std::rand() % k once per thread (kmeans.cc:125-141) from glibc's generator at
    its default seed 1 (the published additive-feedback recurrence
    r[i] = r[i-31] + r[i-3], output r >> 1).  With threads > 1 the reference's
    threads draw in whatever order they start; this gives thread p the p-th draw."""
    r = [1]
    for i in range(1, 31):
        r.append((16807 * r[i - 1]) % 2147483647)
    r += r[0:3]
    draws = []
    for i in range(34, 344 + threads):
        r.append((r[i - 31] + r[i - 3]) & 0xFFFFFFFF)
        if i >= 344:
            draws.append(r[i] >> 1)
    return np.array([d % k for d in draws], np.int32)


def kmeans(g, k, iters=20, starts=None, reorder=False, device=0):
    """kmeans -k K -i iters -init 1 [-rc 1] on the GPU over the rows of g (use the
    features_1hop graph, as the reference pipeline does).  starts: the cluster each
    reference thread draws (default: reference_rand_starts(k, 1), i.e. -t 1).
    Returns (assignment int32[V], sizes of the non-empty clusters)."""
    starts = np.ascontiguousarray(reference_rand_starts(k, 1) if starts is None else starts, dtype=np.int32)
    assign = np.empty(g.V, np.int32)
    sizes = np.zeros(k, np.int64)
    n = C.c_int32()
    capi.check(_L().vsgm_kmeans(device, g.V, capi.ptr(g.row_ptrs, C.c_uint64), capi.ptr(g.cols, C.c_uint32), k, iters, capi.ptr(starts, C.c_int32),
                                len(starts), 1 if reorder else 0, capi.ptr(assign, C.c_int32), sizes.ctypes.data_as(C.POINTER(C.c_int64)), C.byref(n)))
    return assign, sizes[:n.value].copy()


def packing_order(partition, suffix, threads):
    """The source order and per-thread sequences view_packing -o 0 builds from a
    partition file (src/tools/view_packing.cc:150-190): suffix "K" (K == threads)
    gives thread t the vertices of cluster t in id order; "AxB" (A == threads)
    gives thread t clusters t*B .. t*B+B-1 one after the other."""
    partition = np.asarray(partition)
    if "x" in suffix:
        first, second = (int(x) for x in suffix.split("x"))
    else:
        first, second = int(suffix), 1
    if first != threads:
        raise ValueError(f"partition suffix {suffix!r} needs {first} packing threads, not {threads}")
    key = partition.astype(np.int64)
    seqs = [np.nonzero(key // second == t)[0] for t in range(first)]
    seqs = [s_[np.argsort(key[s_] % second, kind="stable")].astype(np.uint32) for s_ in seqs]
    order = np.concatenate(seqs).astype(np.uint32) if seqs else np.zeros(0, np.uint32)
    offsets = np.zeros(len(seqs) + 1, np.uint64)
    offsets[1:] = np.cumsum([len(x) for x in seqs])
    return order, offsets


def view_packing(g, order, seq_offsets, hop, mem_gb, device=0):
    """view_packing -h hop -m mem_gb -s 1 on the GPU: returns (bin of every vertex,
    number of bins, row entries per bin).  The bin size is mem_gb * 1e9 / 4 row
    entries, computed as the reference computes it."""
    order = np.ascontiguousarray(order, dtype=np.uint32)
    seq_offsets = np.ascontiguousarray(seq_offsets, dtype=np.uint64)
    cap = int(float(mem_gb) * 1000 * 1000 * 1000 / 4)
    bins = np.empty(g.V, np.int32)
    nb = C.c_int32()
    sizes = np.zeros(g.V, np.uint64)
    capi.check(_L().vsgm_view_packing(device, g.V, capi.ptr(g.row_ptrs, C.c_uint64), capi.ptr(g.cols, C.c_uint32), capi.ptr(order, C.c_uint32),
                                      capi.ptr(seq_offsets, C.c_uint64), len(seq_offsets) - 1, hop, cap, capi.ptr(bins, C.c_int32), C.byref(nb),
                                      capi.ptr(sizes, C.c_uint64), g.V))
    return bins, nb.value, sizes[:nb.value].copy()


# -------------------------------------------------------------------- engine
def view_compact(g):
    """Compact form of a full-V view: (ascending vertices with a non-empty row,
    their offsets into g.cols) - what vsgm_prefetch_view sends."""
    vert = np.empty(max(g.V, 1), np.uint32)
    off = np.empty(g.V + 1, np.uint64)
    n = C.c_uint64()
    capi.check(_L().vsgm_view_compact(g.V, capi.ptr(g.row_ptrs, C.c_uint64), capi.ptr(vert, C.c_uint32), capi.ptr(off, C.c_uint64), C.byref(n)))
    return vert[:n.value].copy(), off[:n.value + 1].copy()


class Engine:
    """PipelineExecutor on one GPU: transfer a view, match every plan, read exact counts."""

    def __init__(self, V, plans, device=0, max_sources=0, hbm_budget_bytes=0):
        self.plans = list(plans)
        arr = (Plan * len(self.plans))(*self.plans)
        h = C.c_void_p()
        capi.check(_L().vsgm_create(device, V, arr, len(self.plans), max_sources, hbm_budget_bytes, C.byref(h)))
        self.h = h
        self.V = V

    def transfer_view(self, view, sources):
        sources = np.ascontiguousarray(sources, dtype=np.uint32)
        self._keep = (view, sources)
        capi.check(_L().vsgm_transfer_view(self.h, capi.ptr(view.row_ptrs, C.c_uint64), capi.ptr(view.cols, C.c_uint32),
                                           view.E, capi.ptr(sources, C.c_uint32), len(sources)), self.h)

    def prefetch_view(self, view, sources):
        """Start copying a view (in compact form) into the engine's second view
        buffer; it becomes current at swap_view.  The arrays are kept alive here
        until view_released."""
        vert, off = view_compact(view)
        src = np.ascontiguousarray(sources, dtype=np.uint32)
        cols = np.ascontiguousarray(view.cols, dtype=np.uint32)
        self._prefetch_keep = (vert, off, cols, src)
        capi.check(_L().vsgm_prefetch_view(self.h, capi.ptr(vert, C.c_uint32), len(vert), capi.ptr(off, C.c_uint64), capi.ptr(cols, C.c_uint32),
                                           capi.ptr(src, C.c_uint32), len(src)), self.h)

    def view_released(self):
        capi.check(_L().vsgm_view_released(self.h), self.h)
        self._prefetch_keep = None

    def swap_view(self):
        capi.check(_L().vsgm_swap_view(self.h), self.h)

    def bind_view_device(self, d_row_ptrs, d_cols, n_cols, d_sources, n_sources):
        capi.check(_L().vsgm_bind_view_device(self.h, C.c_void_p(d_row_ptrs), C.c_void_p(d_cols), n_cols,
                                              C.c_void_p(d_sources), n_sources), self.h)

    def upload_graph(self, g):
        """Keep the whole graph on the device; views are then built there by materialize_view."""
        self._graph = g
        capi.check(_L().vsgm_upload_graph(self.h, capi.ptr(g.row_ptrs, C.c_uint64), capi.ptr(g.cols, C.c_uint32), g.E), self.h)

    def materialize_view(self, sources, hop, root_degree=0):
        """ViewBin::Materialize on the device: the sources' halo becomes the current view."""
        sources = np.ascontiguousarray(sources, dtype=np.uint32)
        capi.check(_L().vsgm_materialize_view(self.h, capi.ptr(sources, C.c_uint32), len(sources), int(hop), int(root_degree)), self.h)

    def graph_view(self, sources):
        """The uploaded graph itself is the view; only the roots change."""
        sources = np.ascontiguousarray(sources, dtype=np.uint32)
        self._keep_src = sources
        capi.check(_L().vsgm_graph_view(self.h, capi.ptr(sources, C.c_uint32), len(sources)), self.h)

    def read_view(self):
        """The current view copied back to the host, as a Graph."""
        rp = np.zeros(self.V + 1, np.uint64)
        n = C.c_uint64()
        rc = _L().vsgm_read_view(self.h, capi.ptr(rp, C.c_uint64), None, 0, C.byref(n))
        if rc not in (0, capi.ENOMEM):
            capi.check(rc, self.h)
        ci = np.zeros(max(n.value, 1), np.uint32)
        capi.check(_L().vsgm_read_view(self.h, capi.ptr(rp, C.c_uint64), capi.ptr(ci, C.c_uint32), n.value, C.byref(n)), self.h)
        return Graph(rp, ci[:n.value])

    def match(self):
        capi.check(_L().vsgm_match(self.h), self.h)

    def counts(self):
        out = np.zeros(len(self.plans), np.uint64)
        capi.check(_L().vsgm_get_counts(self.h, capi.ptr(out, C.c_uint64)), self.h)
        return [int(x) for x in out]

    def reset_counts(self):
        capi.check(_L().vsgm_reset_counts(self.h), self.h)

    def stats(self, plan=0):
        s = PlanStats()
        capi.check(_L().vsgm_get_stats(self.h, plan, C.byref(s)), self.h)
        return s

    def add_view(self, view, sources=None):
        """Upload another view and keep it resident for run_batched; returns its id."""
        src = np.arange(view.V, dtype=np.uint32) if sources is None else np.ascontiguousarray(sources, dtype=np.uint32)
        vid = C.c_int()
        capi.check(_L().vsgm_add_view(self.h, view.V, capi.ptr(view.row_ptrs, C.c_uint64), capi.ptr(view.cols, C.c_uint32), view.E,
                                      capi.ptr(src, C.c_uint32), len(src), C.byref(vid)), self.h)
        return vid.value

    def run_batched(self, view_ids, plan_ids=None):
        """Every (plan, view) pair in one persistent launch; returns counts[plan][view]."""
        plan_ids = list(range(len(self.plans))) if plan_ids is None else list(plan_ids)
        v = (C.c_int * len(view_ids))(*view_ids)
        p = (C.c_int * len(plan_ids))(*plan_ids)
        out = np.zeros(len(plan_ids) * len(view_ids), np.uint64)
        capi.check(_L().vsgm_run_batched(self.h, v, len(view_ids), p, len(plan_ids), capi.ptr(out, C.c_uint64)), self.h)
        return [[int(x) for x in out[i * len(view_ids):(i + 1) * len(view_ids)]] for i in range(len(plan_ids))]

    def run_pairs(self, pairs):
        """Counts of an explicit list of (plan id, view id) pairs in one persistent run."""
        n = len(pairs)
        p = (C.c_int * n)(*[int(a) for a, _ in pairs])
        v = (C.c_int * n)(*[int(b) for _, b in pairs])
        out = np.zeros(n, np.uint64)
        capi.check(_L().vsgm_run_pairs(self.h, p, v, n, capi.ptr(out, C.c_uint64)), self.h)
        return [int(x) for x in out]

    def run_batched_ex(self, view_ids, plan_ids=None, step_budget=0):
        """Counts [plan][view], level paths [plan][view][op] and overflow flags [plan][view]."""
        plan_ids = list(range(len(self.plans))) if plan_ids is None else list(plan_ids)
        nv, npl = len(view_ids), len(plan_ids)
        v = (C.c_int * nv)(*view_ids)
        p = (C.c_int * npl)(*plan_ids)
        cnt = np.zeros(npl * nv, np.uint64)
        lvl = np.zeros(npl * nv * capi.MAX_OPS, np.uint64)
        ovf = np.zeros(npl * nv, np.uint32)
        capi.check(_L().vsgm_run_batched_ex(self.h, v, nv, p, npl, step_budget, capi.ptr(cnt, C.c_uint64), capi.ptr(lvl, C.c_uint64),
                                            capi.ptr(ovf, C.c_uint32)), self.h)
        return cnt.reshape(npl, nv), lvl.reshape(npl, nv, capi.MAX_OPS), ovf.reshape(npl, nv)

    def batch_stats(self):
        s = capi.BatchStats()
        capi.check(_L().vsgm_get_batch_stats(self.h, C.byref(s)), self.h)
        return s

    def set_option(self, name, value, plan=None):
        if plan is None:
            capi.check(_L().vsgm_set_option(self.h, name.encode(), int(value)), self.h)
        else:
            capi.check(_L().vsgm_set_plan_option(self.h, int(plan), name.encode(), int(value)), self.h)

    def set_profiling(self, on=True):
        capi.check(_L().vsgm_set_profiling(self.h, 1 if on else 0), self.h)

    def stream(self):
        return _L().vsgm_engine_stream(self.h)

    def close(self):
        if getattr(self, "h", None):
            _L().vsgm_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def canonical_pattern(plan):
    """Canonical form of a planned pattern's graph: the largest upper-triangle
    adjacency bit string over all relabellings of its vertices (n <= 7, so at most
    5040 of them).  Two patterns are isomorphic iff their forms are equal."""
    import itertools
    n = plan.n_vertices
    A = [[(plan.adj[i] >> j) & 1 for j in range(n)] for i in range(n)]
    pairs = [(i, j) for i in range(n) for j in range(i + 1, n)]
    best = max(tuple(A[p[i]][p[j]] for i, j in pairs) for p in itertools.permutations(range(n)))
    return n, best


def query_classes(plans):
    """Isomorphism classes of a batch of queries: (representative plan index per
    class, class of every plan).  A batch often holds the same pattern under
    different vertex labellings (random queries of 3-6 vertices fall into few
    classes); over a view whose every vertex is a source, isomorphic patterns have
    the same exact count whatever their plans, so a batch needs to count each class
    once.  (With views that split the sources, per-view counts of isomorphic
    patterns can differ - their plans may root a match at different pattern
    vertices - and only the totals over all views agree.)"""
    reps, cls, seen = [], [], {}
    for i, p in enumerate(plans):
        key = canonical_pattern(p)
        if key not in seen:
            seen[key] = len(reps)
            reps.append(i)
        cls.append(seen[key])
    return reps, cls


def count_graph(g, plans, sources=None, device=0, hbm_budget_bytes=0, views=None, hop=None):
    """Exact counts of every plan over g (all vertices as sources, one view), or
    over a list of per-view source arrays, each materialised with the plans' hop."""
    with Engine(g.V, plans, device=device, hbm_budget_bytes=hbm_budget_bytes) as e:
        if views is None:
            e.transfer_view(g, np.arange(g.V, dtype=np.uint32) if sources is None else sources)
            e.match()
        else:
            h = hop or max(p.hop for p in plans)
            rd = min(p.root_degree for p in plans)
            for src in views:
                e.transfer_view(materialize_view(g, src, h, rd), src)
                e.match()
        return e.counts()
