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
