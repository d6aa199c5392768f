"""Pin the CPU oracle before trusting it.

The reference ships no golden counts and its matching path cannot be built here,
so the restatement of its executor (oracle/oracle.c) is pinned to (a) an
independent brute-force counter (injective edge-preserving maps / |Aut(P)|) on
every preset pattern, clique, graphlet and random pattern, and (b) closed forms.
"""
from math import comb

import numpy as np
import pytest

from conftest import all_plans, complete_graph, cycle_graph, empty_graph


@pytest.fixture(scope="module")
def g(vs):
    return vs.gen_rmat(7, 8, seed=11)


def test_restatement_equals_bruteforce_all_named_queries(vs, orc, g):
    bad = []
    for name, p in all_plans(vs):
        a = orc.count(p, g)
        b = orc.bruteforce(p, g, vs.automorphisms(p))
        if a != b:
            bad.append((name, a, b))
    assert not bad, bad


def test_restatement_equals_bruteforce_random_patterns(vs, orc):
    g = vs.gen_chung_lu(300, 1500, 2.2, 40, seed=2)
    ctr = 0
    for _ in range(40):
        n, bits, ctr = vs.random_pattern(seed=3, counter=ctr, n_min=3, n_max=6)
        p = vs.plan_query_bits(n, bits)
        assert orc.count(p, g) == orc.bruteforce(p, g, vs.automorphisms(p)), p.describe()


def test_closed_forms(vs, orc):
    k7 = complete_graph(vs, 7)
    for k in range(3, 8):
        assert orc.count(vs.plan_clique(k), k7) == comb(7, k)
    for n in (4, 5, 6):
        c = cycle_graph(vs, n)
        pid = {4: 1, 5: 16, 6: 17}[n]
        assert orc.count(vs.plan_pattern(pid), c) == 1
        assert orc.count(vs.plan_clique(3), c) == 0
    assert orc.count(vs.plan_pattern(2), empty_graph(vs, 10)) == 0


def test_automorphism_counts(vs):
    assert vs.automorphisms(vs.plan_clique(4)) == 24
    assert vs.automorphisms(vs.plan_pattern(1)) == 8   # 4-cycle
    assert vs.automorphisms(vs.plan_pattern(2)) == 4   # diamond
    assert vs.automorphisms(vs.plan_pattern(4)) == 2   # house
    assert vs.automorphisms(vs.plan_pattern(16)) == 10  # 5-cycle


def test_oracle_counts_are_view_invariant(vs, orc, g):
    p = vs.plan_pattern(4)
    whole = orc.count(p, g)
    bins = np.arange(g.V) % 3
    total = 0
    for src in vs.sources_of_bins(bins.astype(np.int32), 3):
        v = vs.materialize_view(g, src, p.hop, p.root_degree)
        total += orc.count(p, v, src)
    assert total == whole


def test_four_cycles_by_largest_vertex(vs, orc, g):
    """The largest-vertex attribution of 4-cycles: over all vertices it is the
    4-cycle count (brute force), over a partition of the vertices it sums to it,
    and on C_n / K_n it has closed forms."""
    p = vs.plan_pattern(1)
    for h in (g, vs.gen_chung_lu(300, 1500, 2.3, 40, seed=6), vs.degree_relabel(g)[0]):
        total = orc.bruteforce(p, h, vs.automorphisms(p))
        assert orc.c4_by_largest(h) == total == orc.count(p, h)
        parts = [np.arange(b, h.V, 3, dtype=np.uint32) for b in range(3)]
        assert sum(orc.c4_by_largest(h, s) for s in parts) == total
    c = cycle_graph(vs, 4)
    assert orc.c4_by_largest(c, np.array([3], np.uint32)) == 1 and orc.c4_by_largest(c, np.array([0, 1, 2], np.uint32)) == 0
    k = complete_graph(vs, 6)  # 3 * C(6, 4) cycles; the one whose largest vertex is u: 3 * C(u, 3)
    for u in range(6):
        assert orc.c4_by_largest(k, np.array([u], np.uint32)) == 3 * (u * (u - 1) * (u - 2) // 6)


def test_four_cycle_wedge_oracle_equals_pairwise(vs, orc, g):
    """The wedge-counting form of the largest-vertex 4-cycle count (used on hub roots
    of the full-size graphs) equals the pairwise form root by root."""
    hub = complete_graph(vs, 8)
    for h in (g, vs.gen_chung_lu(400, 2400, 2.2, 80, seed=9), vs.degree_relabel(g)[0], hub, cycle_graph(vs, 4)):
        for v in range(h.V):
            s = np.array([v], np.uint32)
            assert orc.c4_by_largest_wedges(h, s) == orc.c4_by_largest(h, s), v
        assert orc.c4_by_largest_wedges(h) == orc.c4_by_largest(h)


def test_rooted_clique_oracle_equals_plan_oracle(vs, orc, g):
    """Cliques counted by definition at their smallest vertex equal the clique plans'
    per-root counts (the plans chain v0 < v1 < ... by their order conditions), and
    closed forms on K_n: the cliques whose smallest vertex is u number C(n-1-u, k-1)."""
    from math import comb
    for h in (g, vs.gen_chung_lu(400, 2400, 2.2, 80, seed=9), vs.degree_relabel(g)[0], vs.degree_relabel(g, ascending=False)[0]):
        for k in (3, 4, 5):
            p = vs.plan_clique(k)
            for v in range(0, h.V, 7):
                s = np.array([v], np.uint32)
                assert orc.cliques_by_smallest(k, h, s) == orc.count(p, h, s), (k, v)
            assert orc.cliques_by_smallest(k, h) == orc.count(p, h)
    kn = complete_graph(vs, 8)
    for k in (3, 4, 5, 6, 7):
        for u in range(8):
            assert orc.cliques_by_smallest(k, kn, np.array([u], np.uint32)) == comb(7 - u, k - 1)


def test_restated_workload_and_golden_plans(vs, orc):
    """The reference arm's inputs, built without the product library, equal the
    library's: the R-MAT graph and its degree relabelling edge for edge, and the
    plans of the benchmark's queries table for table."""
    for scale, ef, seed in ((10, 16, 2), (12, 8, 5)):
        g = vs.gen_rmat(scale, ef, 0.57, 0.19, 0.19, seed=seed)
        h = orc.gen_rmat(scale, ef, 0.57, 0.19, 0.19, seed=seed)
        assert np.array_equal(g.row_ptrs, h.row_ptrs) and np.array_equal(g.cols, h.cols)
        gr, _ = vs.degree_relabel(g, ascending=True)
        hr = orc.degree_relabel(h)
        assert np.array_equal(gr.row_ptrs, hr.row_ptrs) and np.array_equal(gr.cols, hr.cols)
    import ctypes as C
    for name, p in (("kc4", vs.plan_clique(4)), ("p1", vs.plan_pattern(1)), ("p2", vs.plan_pattern(2))):
        q = orc.golden_plan(name)
        assert bytes(q)[:C.sizeof(q)] == bytes(p)[:C.sizeof(p)], name
        assert orc.count(q, hr) == orc.count(p, hr)



def test_oracle_compute_path_count(vs, orc, g):
    """COMPUTE_PATH_COUNT + COUNT counts what the fused COMPUTE_COUNT counts."""
    from conftest import with_path_count
    for p in (vs.plan_clique(3), vs.plan_clique(4), vs.plan_pattern(1), vs.plan_clique(5)):
        assert orc.count(with_path_count(vs, p), g) == orc.count(p, g)
