"""CPU ORACLE (test infrastructure only): ctypes access to oracle/liboracle.so.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm
use this package, and only to check results or as the timed CPU baseline; the product
never imports it.  See oracle/oracle.c for what each function restates.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
_lib = None


def build():
    """The oracle library; with VSGM_REFERENCE set to a checkout of the reference,
    also the harnesses compiled from its sources (oracle/_ref).  Without the
    variable the reference is treated as absent."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    ref = os.environ.get("VSGM_REFERENCE", "")
    if ref and os.path.isdir(os.path.join(ref, "src")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref}"], check=True)


def lib():
    global _lib
    if _lib is None:
        # make is incremental: this rebuilds only a library older than its source
        subprocess.run(["make", "-s", "-C", HERE], check=True)
        L = C.CDLL(LIB)
        for name in ("oracle_count", "oracle_op_paths", "oracle_bruteforce", "oracle_c4_by_largest", "oracle_c4_by_largest_wedges",
                     "oracle_cliques_by_smallest"):
            getattr(L, name).restype = C.c_uint64
        for name in ("oracle_gen_rmat", "oracle_degree_relabel", "oracle_free"):
            getattr(L, name).restype = None
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def count(plan, g, sources=None, threads=0):
    """Restated reference executor: exact count of plan over g's sources."""
    src = np.arange(g.V, dtype=np.uint32) if sources is None else np.ascontiguousarray(sources, dtype=np.uint32)
    return int(lib().oracle_count(C.byref(plan), C.c_uint64(g.V), _p(g.row_ptrs, C.c_uint64), _p(g.cols, C.c_uint32),
                                  _p(src, C.c_uint32), C.c_uint64(len(src)), threads))


def op_paths(plan, g, sources=None, threads=0):
    src = np.arange(g.V, dtype=np.uint32) if sources is None else np.ascontiguousarray(sources, dtype=np.uint32)
    out = (C.c_uint64 * 24)()
    total = lib().oracle_op_paths(C.byref(plan), C.c_uint64(g.V), _p(g.row_ptrs, C.c_uint64), _p(g.cols, C.c_uint32),
                                  _p(src, C.c_uint32), C.c_uint64(len(src)), threads, out)
    return int(total), [int(out[i]) for i in range(plan.n_ops)]


def bruteforce(plan, g, n_automorphisms, threads=0):
    """Injective edge-preserving maps of the pattern into g divided by |Aut(P)|."""
    return int(lib().oracle_bruteforce(C.byref(plan), C.c_uint64(g.V), _p(g.row_ptrs, C.c_uint64), _p(g.cols, C.c_uint32),
                                       C.c_uint64(n_automorphisms), threads))


def c4_by_largest(g, sources=None, threads=0):
    """4-cycles whose largest vertex is one of `sources` (all vertices by default)."""
    src = np.arange(g.V, dtype=np.uint32) if sources is None else np.ascontiguousarray(sources, dtype=np.uint32)
    return int(lib().oracle_c4_by_largest(C.c_uint64(g.V), _p(g.row_ptrs, C.c_uint64), _p(g.cols, C.c_uint32),
                                          _p(src, C.c_uint32), C.c_uint64(len(src)), threads))


def c4_by_largest_wedges(g, sources=None, threads=0):
    """c4_by_largest by wedge counting (cost ~ wedges below each source, not pairs)."""
    src = np.arange(g.V, dtype=np.uint32) if sources is None else np.ascontiguousarray(sources, dtype=np.uint32)
    return int(lib().oracle_c4_by_largest_wedges(C.c_uint64(g.V), _p(g.row_ptrs, C.c_uint64), _p(g.cols, C.c_uint32),
                                                 _p(src, C.c_uint32), C.c_uint64(len(src)), threads))


def cliques_by_smallest(k, g, sources=None, threads=0):
    """k-cliques whose smallest vertex is one of `sources` (all vertices by default):
    the per-root attribution of the clique plans, counted by definition."""
    src = np.arange(g.V, dtype=np.uint32) if sources is None else np.ascontiguousarray(sources, dtype=np.uint32)
    return int(lib().oracle_cliques_by_smallest(k, C.c_uint64(g.V), _p(g.row_ptrs, C.c_uint64), _p(g.cols, C.c_uint32),
                                                _p(src, C.c_uint32), C.c_uint64(len(src)), threads))


# ------------------------------------------------------------------ plans and inputs
# The reference arm of the benchmark runs on these alone: plans as the reference's
# own planner wrote them (tests/golden/ref_plans.jsonl, dumped by the planner
# compiled from its sources), the workload graph from the restated generator.
MAX_QV, MAX_OPS = 7, 24


class _VGroup(C.Structure):
    _fields_ = [("count", C.c_uint8), ("v", C.c_uint8 * MAX_QV)]


class _Conds(C.Structure):
    _fields_ = [("count", C.c_uint8), ("op", C.c_uint8 * MAX_QV), ("v", C.c_uint8 * MAX_QV)]


class Plan(C.Structure):
    """include/vsgm_plan.h's vsgm_plan, field for field."""
    _fields_ = [("n_vertices", C.c_uint32), ("n_edges", C.c_uint32), ("hop", C.c_int32), ("root_degree", C.c_uint32), ("root", C.c_uint32),
                ("n_ops", C.c_uint32), ("adj", C.c_uint8 * MAX_QV), ("order", (C.c_uint8 * MAX_QV) * MAX_QV), ("seq", C.c_uint8 * MAX_QV),
                ("op_type", C.c_uint8 * MAX_OPS), ("op_vertex", C.c_uint8 * MAX_OPS), ("backward", _VGroup * MAX_QV),
                ("compute_cond", _Conds * MAX_QV), ("materialize_cond", _Conds * MAX_QV), ("filter_cond", _Conds * MAX_QV),
                ("materialized", _VGroup * MAX_OPS), ("computed_unmat", _VGroup * MAX_OPS)]


GOLDEN_PLANS = os.path.join(os.path.dirname(HERE), "tests", "golden", "ref_plans.jsonl")


def golden_plan(name, path=GOLDEN_PLANS):
    """The reference planner's plan `name` ("kc4", "p1", ...) from the golden dump."""
    import json
    with open(path) as f:
        for line in f:
            r = json.loads(line)
            if r["name"] == name:
                break
        else:
            raise KeyError(name)
    p = Plan()
    p.n_vertices, p.n_edges, p.hop, p.root_degree, p.n_ops = r["n"], r["edges"], r["hop"], r["root_degree"], len(r["exec"])
    p.root = r["exec"][0][1]
    for i, nb in enumerate(r["adj"]):
        p.adj[i] = sum(1 << j for j in nb)
    for i, row in enumerate(r["order"]):
        for j, x in enumerate(row):
            p.order[i][j] = x
    seen = []
    for i, (op, v) in enumerate(r["exec"]):
        p.op_type[i], p.op_vertex[i] = op, v
        if v < r["n"] and v not in seen:
            seen.append(v)  # the search sequence: vertices in order of first appearance
    for k, v in enumerate(seen):
        p.seq[k] = v

    def group(dst, lst):
        dst.count = len(lst)
        for k, x in enumerate(lst):
            dst.v[k] = x

    def conds(dst, lst):
        dst.count = len(lst)
        for k, (op, x) in enumerate(lst):
            dst.op[k], dst.v[k] = op, x

    for u in range(r["n"]):
        group(p.backward[u], r["backward"][u])
        conds(p.compute_cond[u], r["compute_cond"][u])
        conds(p.materialize_cond[u], r["materialize_cond"][u])
        conds(p.filter_cond[u], r["filter_cond"][u])
    for i in range(len(r["exec"])):
        group(p.materialized[i], r["materialized"][i])
        group(p.computed_unmat[i], r["computed_unmat"][i])
    return p


class Csr:
    """row_ptrs (u64, V+1) and cols (u32) of an undirected graph."""

    def __init__(self, row_ptrs, cols):
        self.row_ptrs, self.cols, self.V = row_ptrs, cols, len(row_ptrs) - 1


def _take(rp, ci, V):
    E = rp[V]
    out = Csr(np.ctypeslib.as_array(rp, shape=(V + 1,)).copy(), np.ctypeslib.as_array(ci, shape=(max(E, 1),))[:E].copy())
    lib().oracle_free(C.cast(rp, C.c_void_p))
    lib().oracle_free(C.cast(ci, C.c_void_p))
    return out


def gen_rmat(scale, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=1, threads=0):
    """The benchmark's R-MAT graph (same edges as the library's generator)."""
    V, rp, ci = C.c_uint64(), C.POINTER(C.c_uint64)(), C.POINTER(C.c_uint32)()
    lib().oracle_gen_rmat(scale, edge_factor, C.c_double(a), C.c_double(b), C.c_double(c), C.c_uint64(seed), threads, C.byref(V),
                          C.byref(rp), C.byref(ci))
    return _take(rp, ci, V.value)


def degree_relabel(g, threads=0):
    """Ids ascending with (degree, old id)."""
    rp, ci = C.POINTER(C.c_uint64)(), C.POINTER(C.c_uint32)()
    lib().oracle_degree_relabel(C.c_uint64(g.V), _p(g.row_ptrs, C.c_uint64), _p(g.cols, C.c_uint32), threads, C.byref(rp), C.byref(ci))
    return _take(rp, ci, g.V)


def kmeans(g, k, iters, starts, reorder=False):
    """Restated reference kmeans -init 1 (oracle_tools.cc): the cluster of every
    vertex after `iters` rounds from the random start `starts` (one draw per
    reference thread), empty clusters removed."""
    starts = np.ascontiguousarray(starts, dtype=np.int32)
    out = np.zeros(g.V, np.int32)
    n = C.c_int32()
    rc = lib().oracle_kmeans(C.c_uint64(g.V), _p(g.row_ptrs, C.c_uint64), _p(g.cols, C.c_uint32), int(k), int(iters), _p(starts, C.c_int32),
                             len(starts), 1 if reorder else 0, _p(out, C.c_int32), C.byref(n))
    if rc != 0:
        raise ValueError("oracle_kmeans: bad arguments")
    return out


def view_packing(g, order, seq_offsets, hop, cap):
    """Restated reference view_packing -s 1 (oracle_tools.cc): (bin of every vertex,
    number of bins, row entries per bin) for bins of at most `cap` row entries."""
    order = np.ascontiguousarray(order, dtype=np.uint32)
    offs = np.ascontiguousarray(seq_offsets, dtype=np.uint64)
    bins = np.zeros(g.V, np.int32)
    sizes = np.zeros(max(g.V, 1), np.uint64)
    nb = C.c_int32()
    rc = lib().oracle_view_packing(C.c_uint64(g.V), _p(g.row_ptrs, C.c_uint64), _p(g.cols, C.c_uint32), _p(order, C.c_uint32),
                                   _p(offs, C.c_uint64), len(offs) - 1, int(hop), C.c_uint64(int(cap)), _p(bins, C.c_int32), C.byref(nb),
                                   _p(sizes, C.c_uint64))
    if rc == -2:
        raise ValueError("a source's view alone exceeds the bin size")
    return bins, nb.value, sizes[:nb.value].copy()
