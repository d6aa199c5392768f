import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the native engine")


@pytest.fixture(scope="session")
def vs():
    """The package with its native library built in-tree."""
    from vsgm_b200 import build
    build.build()
    import vsgm_b200
    return vsgm_b200


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.lib()  # builds (incrementally) and loads the oracle library
    return oracle


def small_graphs(vs):
    """Seeded small inputs: R-MAT, Chung-Lu, and degenerate shapes."""
    out = {
        "rmat7": vs.gen_rmat(7, 8, seed=11),
        "rmat8": vs.gen_rmat(8, 8, seed=7),
        "chunglu": vs.gen_chung_lu(400, 2400, 2.3, 60, seed=5),
    }
    return out


def complete_graph(vs, n):
    rp = np.arange(0, n * (n - 1) + 1, n - 1, dtype=np.uint64)
    cols = np.array([j for i in range(n) for j in range(n) if j != i], dtype=np.uint32)
    return vs.Graph(rp, cols)


def cycle_graph(vs, n):
    rows = [sorted({(i - 1) % n, (i + 1) % n}) for i in range(n)]
    rp = np.zeros(n + 1, np.uint64)
    rp[1:] = np.cumsum([len(r) for r in rows])
    return vs.Graph(rp, np.array([x for r in rows for x in r], dtype=np.uint32))


def empty_graph(vs, n):
    return vs.Graph(np.zeros(n + 1, np.uint64), np.zeros(0, np.uint32))


def all_plans(vs):
    plans = [(f"p{i}", vs.plan_pattern(i)) for i in range(19)]
    plans += [(f"kc{k}", vs.plan_clique(k)) for k in range(3, 8)]
    for k in (3, 4, 5):
        plans += [(f"km{k}_{i}", p) for i, p in enumerate(vs.plan_graphlets(k))]
    return plans


def with_path_count(vs, p):
    """The same plan with its final COMPUTE_COUNT(u) (no computed vertex counted
    against) split into COMPUTE_PATH_COUNT(u) and a COUNT of u: the op pair the
    reference's executor runs for it (src/executor/ops/compute_path_count.h,
    src/executor/ops/count.h); the reference planner itself never emits it."""
    q = type(p).from_buffer_copy(bytes(p))
    i = q.n_ops - 1
    assert q.op_type[i] == vs.capi.COMPUTE_COUNT and q.computed_unmat[i].count == 0
    u = q.op_vertex[i]
    q.op_type[i] = vs.capi.COMPUTE_PATH_COUNT
    q.op_type[i + 1] = vs.capi.COUNT
    q.op_vertex[i + 1] = q.n_vertices
    q.materialized[i + 1] = type(q.materialized[i]).from_buffer_copy(bytes(q.materialized[i]))
    q.computed_unmat[i + 1].count = 1
    q.computed_unmat[i + 1].v[0] = u
    q.n_ops += 1
    return q
