"""ctypes binding of the vsgm_b200 C ABI (include/vsgm.h).

The shared library is built in-tree (vsgm_b200/libvsgm_b200.so, see build.py).
Loading fails loudly when it is missing: there is no Python or CPU fallback for
the engine.
"""
import ctypes as C
import os

import numpy as np

MAX_QV = 7
MAX_OPS = 24

COMPUTE, COMPUTE_PATH_COUNT, MATERIALIZE, FILTER_COMPUTE, COUNT, COMPUTE_COUNT = range(6)
LESS_THAN, LARGER_THAN, NON_EQUAL, OPERATOR_NONE = range(4)
OP_NAMES = {COMPUTE: "COMPUTE", COMPUTE_PATH_COUNT: "COMPUTE_PATH_COUNT", MATERIALIZE: "MATERIALIZE",
            FILTER_COMPUTE: "FILTER_COMPUTE", COUNT: "COUNT", COMPUTE_COUNT: "COMPUTE_COUNT"}


class VGroup(C.Structure):
    _fields_ = [("count", C.c_uint8), ("v", C.c_uint8 * MAX_QV)]

    def tolist(self):
        return [int(self.v[i]) for i in range(self.count)]


class Conds(C.Structure):
    _fields_ = [("count", C.c_uint8), ("op", C.c_uint8 * MAX_QV), ("v", C.c_uint8 * MAX_QV)]

    def tolist(self):
        return [[int(self.op[i]), int(self.v[i])] for i in range(self.count)]


class Plan(C.Structure):
    _fields_ = [
        ("n_vertices", C.c_uint32),
        ("n_edges", C.c_uint32),
        ("hop", C.c_int32),
        ("root_degree", C.c_uint32),
        ("root", C.c_uint32),
        ("n_ops", C.c_uint32),
        ("adj", C.c_uint8 * MAX_QV),
        ("order", (C.c_uint8 * MAX_QV) * MAX_QV),
        ("seq", C.c_uint8 * MAX_QV),
        ("op_type", C.c_uint8 * MAX_OPS),
        ("op_vertex", C.c_uint8 * MAX_OPS),
        ("backward", VGroup * MAX_QV),
        ("compute_cond", Conds * MAX_QV),
        ("materialize_cond", Conds * MAX_QV),
        ("filter_cond", Conds * MAX_QV),
        ("materialized", VGroup * MAX_OPS),
        ("computed_unmat", VGroup * MAX_OPS),
    ]

    def exec_seq(self):
        return [(int(self.op_type[i]), int(self.op_vertex[i])) for i in range(self.n_ops)]

    def adjacency(self):
        n = self.n_vertices
        return [[j for j in range(n) if self.adj[i] >> j & 1] for i in range(n)]

    def describe(self):
        short = {COMPUTE: "C", COMPUTE_PATH_COUNT: "CP", MATERIALIZE: "M", FILTER_COMPUTE: "FC", COUNT: "CT", COMPUTE_COUNT: "CC"}
        return " ".join(f"({short[t]},{v})" for t, v in self.exec_seq())

    def to_dict(self):
        """The plan in the layout of tests/golden/ref_plans.jsonl."""
        n = self.n_vertices
        return {
            "n": n,
            "edges": self.n_edges,
            "adj": self.adjacency(),
            "order": [[int(self.order[i][j]) for j in range(n)] for i in range(n)],
            "hop": self.hop,
            "root_degree": self.root_degree,
            "exec": [list(x) for x in self.exec_seq()],
            "backward": [self.backward[i].tolist() for i in range(n)],
            "materialized": [self.materialized[i].tolist() for i in range(self.n_ops)],
            "computed_unmat": [self.computed_unmat[i].tolist() for i in range(self.n_ops)],
            "compute_cond": [self.compute_cond[i].tolist() for i in range(n)],
            "materialize_cond": [self.materialize_cond[i].tolist() for i in range(n)],
            "filter_cond": [self.filter_cond[i].tolist() for i in range(n)],
        }


class BatchStats(C.Structure):
    _fields_ = [("tasks", C.c_uint64), ("launches", C.c_uint64), ("scratch_bytes", C.c_uint64), ("ms", C.c_double),
                ("level_pairs", C.c_uint64)]


class PlanStats(C.Structure):
    _fields_ = [
        ("op_paths", C.c_uint64 * MAX_OPS),
        ("op_outputs", C.c_uint64 * MAX_OPS),
        ("op_ms", C.c_double * MAX_OPS),
        ("op_launches", C.c_uint64 * MAX_OPS),
        ("op_bytes", C.c_uint64 * MAX_OPS),
        ("batches", C.c_uint64),
        ("peak_bytes", C.c_uint64),
    ]


LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libvsgm_b200.so")
_lib = None

_P = C.POINTER
_u8p, _u32p, _u64p, _i32p = _P(C.c_uint8), _P(C.c_uint32), _P(C.c_uint64), _P(C.c_int32)

_SIGS = {
    "vsgm_last_error": (C.c_char_p, []),
    "vsgm_free": (None, [C.c_void_p]),
    "vsgm_plan_pattern": (C.c_int, [C.c_int, _P(Plan)]),
    "vsgm_plan_clique": (C.c_int, [C.c_int, _P(Plan)]),
    "vsgm_plan_query": (C.c_int, [C.c_int, _u8p, _P(Plan)]),
    "vsgm_plan_graphlets": (C.c_int, [C.c_int, _P(Plan), C.c_int, _P(C.c_int)]),
    "vsgm_plan_reorder": (C.c_int, [_P(Plan), _u8p, _P(Plan)]),
    "vsgm_plan_automorphisms": (C.c_uint64, [_P(Plan)]),
    "vsgm_read_csr_bin": (C.c_int, [C.c_char_p, _u64p, _u64p, _P(_u64p), _P(_u32p)]),
    "vsgm_csr_bin_header": (C.c_int, [C.c_char_p, _u64p, _u64p]),
    "vsgm_read_csr_bin_into": (C.c_int, [C.c_char_p, C.c_uint64, C.c_uint64, _u64p, _u32p, C.c_int]),
    "vsgm_write_csr_bin": (C.c_int, [C.c_char_p, C.c_uint64, C.c_uint64, _u64p, _u32p]),
    "vsgm_read_vbmap": (C.c_int, [C.c_char_p, C.c_uint64, _i32p, _i32p]),
    "vsgm_write_vbmap": (C.c_int, [C.c_char_p, C.c_uint64, _i32p, C.c_int32]),
    "vsgm_csr_defects": (C.c_uint64, [C.c_uint64, _u64p, _u32p]),
    "vsgm_gen_rmat": (C.c_int, [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_uint64, C.c_int,
                                _u64p, _u64p, _P(_u64p), _P(_u32p)]),
    "vsgm_gen_chung_lu": (C.c_int, [C.c_uint64, C.c_uint64, C.c_double, C.c_uint64, C.c_uint64, C.c_int,
                                    _u64p, _P(_u64p), _P(_u32p)]),
    "vsgm_degree_relabel": (C.c_int, [C.c_uint64, _u64p, _u32p, C.c_int, C.c_int, _u32p, _u64p, _u32p]),
    "vsgm_random_pattern": (C.c_int, [C.c_int, C.c_int, C.c_double, C.c_uint64, _u64p, _P(C.c_int), _u8p]),
    "vsgm_view_materialize": (C.c_int, [C.c_uint64, _u64p, _u32p, _u32p, C.c_uint64, C.c_int, C.c_uint64, C.c_int,
                                        _u64p, _u32p, C.c_uint64, _u64p]),
    "vsgm_features_1hop": (C.c_int, [C.c_int, C.c_uint64, _u64p, _u32p, _u64p, _u32p]),
    "vsgm_kmeans": (C.c_int, [C.c_int, C.c_uint64, _u64p, _u32p, C.c_int, C.c_int, _i32p, C.c_int, C.c_int, _i32p, _P(C.c_int64), _i32p]),
    "vsgm_view_packing": (C.c_int, [C.c_int, C.c_uint64, _u64p, _u32p, _u32p, _u64p, C.c_int, C.c_int, C.c_uint64, _i32p, _i32p, _u64p,
                                    C.c_uint64]),
    "vsgm_create": (C.c_int, [C.c_int, C.c_uint64, _P(Plan), C.c_int, C.c_uint64, C.c_uint64, _P(C.c_void_p)]),
    "vsgm_transfer_view": (C.c_int, [C.c_void_p, _u64p, _u32p, C.c_uint64, _u32p, C.c_uint64]),
    "vsgm_bind_view_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64]),
    "vsgm_prefetch_view": (C.c_int, [C.c_void_p, _u32p, C.c_uint64, _u64p, _u32p, _u32p, C.c_uint64]),
    "vsgm_view_released": (C.c_int, [C.c_void_p]),
    "vsgm_swap_view": (C.c_int, [C.c_void_p]),
    "vsgm_view_compact": (C.c_int, [C.c_uint64, _u64p, _u32p, _u64p, _u64p]),
    "vsgm_host_alloc": (C.c_int, [C.c_uint64, _P(C.c_void_p)]),
    "vsgm_host_free": (C.c_int, [C.c_void_p]),
    "vsgm_upload_graph": (C.c_int, [C.c_void_p, _u64p, _u32p, C.c_uint64]),
    "vsgm_materialize_view": (C.c_int, [C.c_void_p, _u32p, C.c_uint64, C.c_int, C.c_uint64]),
    "vsgm_graph_view": (C.c_int, [C.c_void_p, _u32p, C.c_uint64]),
    "vsgm_read_view": (C.c_int, [C.c_void_p, _u64p, _u32p, C.c_uint64, _u64p]),
    "vsgm_match": (C.c_int, [C.c_void_p]),
    "vsgm_get_counts": (C.c_int, [C.c_void_p, _u64p]),
    "vsgm_reset_counts": (C.c_int, [C.c_void_p]),
    "vsgm_get_stats": (C.c_int, [C.c_void_p, C.c_int, _P(PlanStats)]),
    "vsgm_set_profiling": (C.c_int, [C.c_void_p, C.c_int]),
    "vsgm_set_option": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int64]),
    "vsgm_set_plan_option": (C.c_int, [C.c_void_p, C.c_int, C.c_char_p, C.c_int64]),
    "vsgm_add_view": (C.c_int, [C.c_void_p, C.c_uint64, _u64p, _u32p, C.c_uint64, _u32p, C.c_uint64, _P(C.c_int)]),
    "vsgm_run_batched": (C.c_int, [C.c_void_p, _P(C.c_int), C.c_int, _P(C.c_int), C.c_int, _u64p]),
    "vsgm_run_pairs": (C.c_int, [C.c_void_p, _P(C.c_int), _P(C.c_int), C.c_int, _u64p]),
    "vsgm_get_batch_stats": (C.c_int, [C.c_void_p, _P(BatchStats)]),
    "vsgm_run_batched_ex": (C.c_int, [C.c_void_p, _P(C.c_int), C.c_int, _P(C.c_int), C.c_int, C.c_uint64, _u64p, _u64p, _u32p]),
    "vsgm_engine_stream": (C.c_void_p, [C.c_void_p]),
    "vsgm_engine_error": (C.c_char_p, [C.c_void_p]),
    "vsgm_destroy": (C.c_int, [C.c_void_p]),
    "vsgm_count_noalloc": (C.c_int, [C.c_int, _P(Plan), C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, _u64p]),
    "vsgm_mlp_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, _P(C.c_void_p)]),
    "vsgm_mlp_num_params": (C.c_uint64, [C.c_void_p]),
    "vsgm_mlp_get_params": (C.c_int, [C.c_void_p, _P(C.c_float)]),
    "vsgm_mlp_set_params": (C.c_int, [C.c_void_p, _P(C.c_float)]),
    "vsgm_mlp_forward": (C.c_int, [C.c_void_p, _P(C.c_float), C.c_int, _P(C.c_float)]),
    "vsgm_mlp_gradients": (C.c_int, [C.c_void_p, _P(C.c_float), _P(C.c_float), _P(C.c_float), C.c_int, _P(C.c_float), _P(C.c_float)]),
    "vsgm_mlp_train_step": (C.c_int, [C.c_void_p, _P(C.c_float), _P(C.c_float), _P(C.c_float), C.c_int, C.c_float, _P(C.c_float)]),
    "vsgm_mlp_error": (C.c_char_p, [C.c_void_p]),
    "vsgm_mlp_destroy": (C.c_int, [C.c_void_p]),
}

EXPORTED = sorted(_SIGS)


def lib(path=None):
    """Load (once) and return the shared library."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"vsgm_b200 native library not built: {p} is missing (run `python -m vsgm_b200.build`)")
    L = C.CDLL(p)
    for name, (res, args) in _SIGS.items():
        fn = getattr(L, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = L
    return L


class VsgmError(RuntimeError):
    pass


ENOMEM = -4  # VSGM_ENOMEM


def check(rc, engine=None):
    if rc != 0:
        L = lib()
        msg = (L.vsgm_engine_error(engine) if engine else L.vsgm_last_error()) or b""
        raise VsgmError(f"vsgm error {rc}: {msg.decode(errors='replace')}")


def ptr(a, ctype):
    return a.ctypes.data_as(_P(ctype))
