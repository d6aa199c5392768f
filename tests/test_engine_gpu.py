"""GPU parity: the CUDA engine's exact counts equal the CPU oracle's.

Every test calls the engine through the C ABI (vsgm_create / vsgm_transfer_view
/ vsgm_match / vsgm_get_counts) and compares with the oracle restatement of the
reference executor (oracle/oracle.c), itself pinned to brute force in
tests/test_oracle.py.  Integer counts: the bar is bit-exact equality.
"""
import numpy as np
import pytest

from conftest import all_plans, complete_graph, cycle_graph, empty_graph, small_graphs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def graphs(vs):
    return small_graphs(vs)


@pytest.mark.parametrize("gname", ["rmat7", "rmat8", "chunglu"])
def test_every_preset_clique_and_graphlet(vs, orc, graphs, gname):
    g = graphs[gname]
    plans = all_plans(vs)
    got = vs.count_graph(g, [p for _, p in plans])
    want = [orc.count(p, g) for _, p in plans]
    bad = [(n, w, x) for (n, _), w, x in zip(plans, want, got) if w != x]
    assert not bad, bad


def test_random_patterns(vs, orc, graphs):
    g = graphs["rmat8"]
    ctr = 0
    plans = []
    for _ in range(48):
        n, bits, ctr = vs.random_pattern(seed=3, counter=ctr, n_min=3, n_max=6, p=0.5)
        plans.append(vs.plan_query_bits(n, bits))
    got = vs.count_graph(g, plans)
    want = [orc.count(p, g) for p in plans]
    assert got == want


def test_closed_forms(vs):
    from math import comb
    k7 = complete_graph(vs, 7)
    got = vs.count_graph(k7, [vs.plan_clique(k) for k in range(3, 8)])
    assert got == [comb(7, k) for k in range(3, 8)]
    c9 = cycle_graph(vs, 9)
    assert vs.count_graph(c9, [vs.plan_clique(3), vs.plan_pattern(1)]) == [0, 0]
    c4 = cycle_graph(vs, 4)
    assert vs.count_graph(c4, [vs.plan_pattern(1)]) == [1]  # exactly one 4-cycle
    assert vs.count_graph(empty_graph(vs, 16), [vs.plan_clique(3), vs.plan_pattern(2)]) == [0, 0]


def test_views_partition_invariance(vs, orc, graphs):
    """Counts summed over views equal the whole-graph count (src/view/view_bin.h:49-142)."""
    g = graphs["rmat8"]
    plans = [vs.plan_clique(3), vs.plan_clique(4), vs.plan_pattern(1), vs.plan_pattern(2), vs.plan_pattern(4)]
    whole = vs.count_graph(g, plans)
    rng = np.random.default_rng(5)
    bins = rng.integers(0, 4, size=g.V).astype(np.int32)
    views = vs.sources_of_bins(bins, 4)
    assert vs.count_graph(g, plans, views=views) == whole
    assert whole == [orc.count(p, g) for p in plans]


def test_tiny_budget_forces_batches(vs, orc, graphs):
    """Memory-bounded batching must not change a count."""
    g = graphs["rmat8"]
    plans = [vs.plan_clique(4), vs.plan_pattern(1), vs.plan_pattern(4), vs.plan_pattern(13)]
    want = [orc.count(p, g) for p in plans]
    with vs.Engine(g.V, plans, hbm_budget_bytes=1 << 21) as e:
        e.transfer_view(g, np.arange(g.V, dtype=np.uint32))
        e.match()
        assert e.counts() == want
        assert max(e.stats(i).batches for i in range(len(plans))) > 4


def test_stats_match_oracle_paths(vs, orc, graphs):
    g = graphs["rmat7"]
    for p in [vs.plan_clique(4), vs.plan_pattern(1), vs.plan_pattern(3)]:
        total, paths = orc.op_paths(p, g)
        with vs.Engine(g.V, [p]) as e:
            e.set_option("c4_aggregate", 0)  # the op sequence itself
            e.set_option("clique_bits", 0)
            e.transfer_view(g, np.arange(g.V, dtype=np.uint32))
            e.match()
            assert e.counts() == [total]
            s = e.stats(0)
            assert [s.op_paths[i] for i in range(p.n_ops)] == paths


def test_counts_accumulate_across_views_and_reset(vs, graphs):
    g = graphs["rmat7"]
    p = vs.plan_clique(3)
    with vs.Engine(g.V, [p]) as e:
        src = np.arange(g.V, dtype=np.uint32)
        e.transfer_view(g, src)
        e.match()
        one = e.counts()[0]
        e.match()
        assert e.counts()[0] == 2 * one
        e.reset_counts()
        e.match()
        assert e.counts()[0] == one


def test_engine_rejects_bad_views(vs, graphs):
    g = graphs["rmat7"]
    with vs.Engine(g.V, [vs.plan_clique(3)]) as e:
        with pytest.raises(vs.VsgmError):
            e.transfer_view(g, np.array([g.V + 5], dtype=np.uint32))
        with pytest.raises(vs.VsgmError):
            e.match()  # no view transferred yet


def test_pm_pipeline_driver(vs, orc, graphs, tmp_path):
    """The drop-in CLI reads a .bin and its .vbmap and prints the reference's lines."""
    import re
    import subprocess

    from vsgm_b200 import build

    g = graphs["rmat8"]
    path = tmp_path / "g.bin"
    vs.write_csr_bin(path, g)
    bins = (np.arange(g.V) * 7 % 3).astype(np.int32)
    vs.write_vbmap(str(path) + ".2.hop.vbmap", bins, 3)
    for args, plan in [(["-kc", "4"], vs.plan_clique(4)), (["-p", "4"], vs.plan_pattern(4)), (["-kc", "4", "-rl", "0"], vs.plan_clique(4)),
                       (["-p", "1", "-rl", "0"], vs.plan_pattern(1)), (["-p", "2", "-gv", "0"], vs.plan_pattern(2))]:
        out = subprocess.run([build.DRIVER, "-f", str(path), "-m", "1", "-t", "2", "-qs", "2", "-pn", "2", "-cn", "1", "-ds", "1"] + args,
                             capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stderr
        got = int(re.search(r"total count for query 0: (\d+)", out.stdout).group(1))
        assert got == orc.count(plan, g)
        assert re.search(r"finish total time, elapsed_time=[0-9.]+ms", out.stdout)


def test_batched_persistent_run_matches_oracle(vs, orc, graphs):
    """Many plans x many views in one persistent launch (vsgm_run_batched)."""
    views = [graphs["rmat7"], graphs["rmat8"], graphs["chunglu"], complete_graph(vs, 9), cycle_graph(vs, 12)]
    named = all_plans(vs)
    ctr = 0
    for _ in range(16):
        n, bits, ctr = vs.random_pattern(seed=3, counter=ctr, n_min=3, n_max=6)
        named.append(("rand", vs.plan_query_bits(n, bits)))
    plans = [p for _, p in named]
    V = max(g.V for g in views)
    with vs.Engine(V, plans) as e:
        ids = [e.add_view(g) for g in views]
        e.set_option("hybrid_steps", 0)  # the persistent launch alone
        got = e.run_batched(ids)
        st = e.batch_stats()
        assert st.launches == 1 and st.tasks >= len(plans) * len(views) and st.level_pairs == 0
        # hybrid: pairs whose tasks exceed the step bound are counted level-wise
        e.set_option("hybrid_steps", 1)
        every = e.run_batched(ids)  # every pair recounted level-wise, 4 at a time on their own streams
        assert e.batch_stats().level_pairs == len(plans) * len(views)
        e.set_option("streams", 1)
        assert e.run_batched(ids) == every  # one after the other
        e.set_option("streams", 4)
        e.set_option("hybrid_steps", 1 << 17)
        default = e.run_batched(ids)
        # an explicit pair list gives the same counts as the cross product
        rng = np.random.default_rng(2)
        pairs = [(int(a), int(b)) for a, b in zip(rng.integers(0, len(plans), 40), rng.integers(0, len(views), 40))]
        for steps in (0, 1, 1 << 17):
            e.set_option("hybrid_steps", steps)
            assert e.run_pairs(pairs) == [got[a][b] for a, b in pairs], steps
    assert every == got and default == got
    for pi, (name, p) in enumerate(named):
        want = [orc.count(p, g) for g in views]
        assert got[pi] == want, (name, p.describe())


def test_batched_run_with_partial_sources(vs, orc, graphs):
    g = graphs["rmat8"]
    p = vs.plan_pattern(4)
    src = np.arange(0, g.V, 3, dtype=np.uint32)
    with vs.Engine(g.V, [p]) as e:
        vid = e.add_view(g, src)
        assert e.run_batched([vid]) == [[orc.count(p, g, src)]]


@pytest.mark.parametrize("fuse", [0, 1])
def test_fused_tail_on_and_off(vs, orc, graphs, fuse):
    """MATERIALIZE + COMPUTE_COUNT fused or expanded: same counts."""
    g = graphs["chunglu"]
    plans = [vs.plan_clique(3), vs.plan_clique(4), vs.plan_clique(5), vs.plan_pattern(1), vs.plan_pattern(5),
             vs.plan_pattern(8), vs.plan_pattern(16), vs.plan_pattern(18)]
    with vs.Engine(g.V, plans) as e:
        e.set_option("fuse_tail", fuse)
        e.set_option("clique_bits", 0)  # the cliques through the plan's fused tail too
        e.transfer_view(g, np.arange(g.V, dtype=np.uint32))
        e.match()
        assert e.counts() == [orc.count(p, g) for p in plans]


def _hub_graph(vs, leaves=2000, chords=3000, seed=4):
    """One hub joined to every leaf, leaves on a ring plus random chords."""
    rng = np.random.default_rng(seed)
    edges = {(0, i) for i in range(1, leaves + 1)}
    edges |= {(i, i % leaves + 1) for i in range(1, leaves + 1)}
    for a, b in rng.integers(1, leaves + 1, size=(chords, 2)):
        if a != b:
            edges.add((min(a, b), max(a, b)))
    n = leaves + 1
    rows = [[] for _ in range(n)]
    for a, b in edges:
        rows[a].append(b)
        rows[b].append(a)
    rp = np.zeros(n + 1, np.uint64)
    rp[1:] = np.cumsum([len(r) for r in rows])
    return vs.Graph(rp, np.array([x for r in rows for x in sorted(r)], dtype=np.uint32))


def test_fused_tail_large_staged_sets(vs, orc, graphs):
    """Shared lists larger than the stage take the per-child path (natural hub, and forced)."""
    hub, _ = vs.degree_relabel(_hub_graph(vs))
    assert hub.degrees().max() > 1536
    plans = [vs.plan_clique(3), vs.plan_clique(4), vs.plan_pattern(1), vs.plan_pattern(8)]
    for g in (hub, graphs["rmat8"]):
        want = [orc.count(p, g) for p in plans]
        for cap in (1536, 16, 0):
            with vs.Engine(g.V, plans) as e:
                e.set_option("stage_cap", cap)
                e.set_option("clique_bits", 0)
                e.transfer_view(g, np.arange(g.V, dtype=np.uint32))
                e.match()
                assert e.counts() == want, cap


@pytest.mark.parametrize("gname", ["rmat8", "chunglu", "hub"])
def test_tail_merge_matches_oracle(vs, orc, graphs, gname):
    """The merge-path split of heavy children in the fused tail (knob tail_merge):
    every preset, clique and graphlet, with every child sent to the heavy pass
    (lane_slice 0) and with the default split, equals the oracle."""
    g = vs.degree_relabel(_hub_graph(vs))[0] if gname == "hub" else graphs[gname]
    # on the hub graph the oracle is slow for the 6- and 7-vertex presets: patterns up to 5 vertices there
    plans = [p for _, p in all_plans(vs) if gname != "hub" or p.n_vertices <= 5]
    want = [orc.count(p, g) for p in plans]
    for ls in (0, 16):
        with vs.Engine(g.V, plans) as e:
            e.set_option("tail_merge", 1)
            e.set_option("clique_bits", 0)
            e.set_option("lane_slice", ls)
            e.transfer_view(g, np.arange(g.V, dtype=np.uint32))
            e.match()
            assert e.counts() == want, ls


def test_relabelled_graph_same_counts(vs, orc, graphs):
    g = graphs["rmat8"]
    plans = [vs.plan_clique(4), vs.plan_pattern(1), vs.plan_pattern(2)]
    want = [orc.count(p, g) for p in plans]
    for asc in (True, False):
        h, perm = vs.degree_relabel(g, ascending=asc)
        assert sorted(perm.tolist()) == list(range(g.V))
        assert vs.count_graph(h, plans) == want


def test_batched_level_paths_and_step_budget(vs, orc, graphs):
    """Per-op partial-match counts of the persistent run equal the oracle's; a step budget stops tasks."""
    g = graphs["rmat7"]
    plans = [vs.plan_clique(4), vs.plan_pattern(1), vs.plan_pattern(3), vs.plan_pattern(13)]
    with vs.Engine(g.V, plans) as e:
        vid = e.add_view(g)
        cnt, lvl, ovf = e.run_batched_ex([vid])
        for i, p in enumerate(plans):
            total, paths = orc.op_paths(p, g)
            assert int(cnt[i][0]) == total
            assert [int(x) for x in lvl[i][0][:p.n_ops]] == paths
        assert not ovf.any()
        cnt2, _, ovf2 = e.run_batched_ex([vid], step_budget=5)
        assert ovf2.all()
        assert all(int(cnt2[i][0]) <= int(cnt[i][0]) for i in range(len(plans)))


@pytest.mark.parametrize("fuse", [0, 1])
def test_batched_heavy_roots_and_fused_tail(vs, orc, graphs, fuse):
    """The persistent run splits a hub root's candidates over several warps and fuses
    the last MATERIALIZE with the final count: counts and per-op partial matches
    still equal the oracle's."""
    plans = [vs.plan_clique(3), vs.plan_clique(4), vs.plan_pattern(1), vs.plan_pattern(2), vs.plan_pattern(3),
             vs.plan_pattern(4), vs.plan_pattern(13)]
    ctr = 0
    for _ in range(6):
        n, bits, ctr = vs.random_pattern(seed=5, counter=ctr, n_min=4, n_max=5)
        plans.append(vs.plan_query_bits(n, bits))
    hub = _hub_graph(vs, leaves=1200, chords=1500)
    views = [vs.degree_relabel(hub, ascending=True)[0], vs.degree_relabel(hub, ascending=False)[0], graphs["rmat7"]]
    V = max(g.V for g in views)
    with vs.Engine(V, plans) as e:
        e.set_option("fuse_tail", fuse)
        ids = [e.add_view(g) for g in views]
        cnt, lvl, ovf = e.run_batched_ex(ids)
        assert e.batch_stats().tasks > len(plans) * len(views)
        assert not ovf.any()
    for i, p in enumerate(plans):
        for v, g in enumerate(views):
            total, paths = orc.op_paths(p, g)
            assert int(cnt[i][v]) == total, (p.describe(), v)
            assert [int(x) for x in lvl[i][v][:p.n_ops]] == paths, (p.describe(), v)


def test_knobs_and_autotuner_keep_counts(vs, orc, graphs):
    """Every intersection variant / fusion setting gives the same counts; the autotuner picks one."""
    from vsgm_b200.autotune import autotune
    g = graphs["rmat8"]
    plans = [vs.plan_clique(4), vs.plan_pattern(1), vs.plan_pattern(2), vs.plan_pattern(4)]
    want = [orc.count(p, g) for p in plans]
    with vs.Engine(g.V, plans) as e:
        e.transfer_view(g, np.arange(g.V, dtype=np.uint32))
        e.set_option("clique_bits", 0)  # the 4-clique through the plan's intersections
        for ratio in (0, 1, 2, 64):
            for lane in (0, 1):
                e.set_option("merge_ratio", ratio)
                e.set_option("lane_merge", lane)
                e.reset_counts()
                e.match()
                assert e.counts() == want, (ratio, lane)
        for walk in (0, 1, 8, 1000):
            for ls in (0, 16, 4096):
                e.set_option("walk_ratio", walk)
                e.set_option("lane_slice", ls)
                e.reset_counts()
                e.match()
                assert e.counts() == want, (walk, ls)
        e.set_option("lane_slice", 16)
        e.set_option("clique_bits", 1)
        from vsgm_b200.autotune import TuneCache
        cache = TuneCache()
        report = autotune(e, len(plans), stride=4, cache=cache, plans=plans, degrees=g.degrees())
        assert [r["plan"] for r in report] == list(range(len(plans))) and not any(r["cached"] for r in report)
        e.match()
        assert e.counts() == want
        again = autotune(e, len(plans), stride=4, cache=cache, plans=plans, degrees=g.degrees())  # same view class
        assert all(r["cached"] for r in again) and [r["best"] for r in again] == [r["best"] for r in report]
        e.reset_counts()
        e.match()
        assert e.counts() == want
        e.set_option("root_stride", 3)
        e.set_option("only_plan", 1)
        e.set_option("c4_aggregate", 0)  # a root sample counts like the plan only without aggregation
        e.reset_counts()
        e.match()
        assert e.counts()[1] == orc.count(plans[1], g, np.arange(0, g.V, 3, dtype=np.uint32))


def test_four_cycle_aggregation_equals_plan(vs, orc, graphs):
    """Wedge aggregation (each 4-cycle at its largest vertex) gives the plan's total, on any labels."""
    p = vs.plan_pattern(1)
    hub, _ = vs.degree_relabel(_hub_graph(vs))
    for g in (graphs["rmat7"], graphs["rmat8"], graphs["chunglu"], vs.degree_relabel(graphs["rmat8"])[0],
              vs.degree_relabel(graphs["rmat8"], ascending=False)[0], hub, cycle_graph(vs, 4), complete_graph(vs, 6)):
        want = orc.count(p, g)
        # c4_heavy 0: every root through the group kernels; 2^40: none; c4_hash 0:
        # light roots through dense counters in HBM instead of shared-memory tables
        # c4_balance 1: heavy groups split by adjacency entry instead of by centre
        for agg, heavy, hashed, window, bal in ((1, 1 << 40, 1, 0, 1), (1, 1 << 40, 0, 0, 1), (1, 0, 1, 0, 1), (1, 0, 1, 0, 0), (1, 0, 1, 1, 1),
                                                (1, 64, 1, 1, 1), (1, 64, 0, 0, 1), (1, 64, 0, 0, 0), (1, 12289, 1, 0, 1), (0, 0, 1, 0, 1)):
            with vs.Engine(g.V, [p]) as e:
                e.set_option("c4_aggregate", agg)
                e.set_option("c4_heavy", heavy)
                e.set_option("c4_hash", hashed)
                e.set_option("c4_window", window)
                e.set_option("c4_balance", bal)
                e.transfer_view(g, np.arange(g.V, dtype=np.uint32))
                e.match()
                assert e.counts() == [want], (agg, heavy, hashed, window, bal)
    # views: per-view attribution differs, totals do not
    g = graphs["rmat8"]
    bins = (np.arange(g.V) % 3).astype(np.int32)
    assert vs.count_graph(g, [p], views=vs.sources_of_bins(bins, 3)) == [orc.count(p, g)]
    # each view counts the cycles whose largest vertex is one of its sources
    for heavy, hashed in ((1 << 18, 1), (1 << 18, 0), (0, 1)):
        with vs.Engine(g.V, [p]) as e:
            e.set_option("c4_heavy", heavy)
            e.set_option("c4_hash", hashed)
            for src in vs.sources_of_bins(bins, 3):
                e.reset_counts()
                e.transfer_view(g, src)
                e.match()
                assert e.counts() == [orc.c4_by_largest(g, src)], heavy


@pytest.mark.parametrize("reuse", [0, 1])
def test_set_reuse_pairs(vs, orc, graphs, reuse):
    """Diamond-like tails (count against an identical candidate set): pairs of one set."""
    g = graphs["chunglu"]
    plans = [vs.plan_pattern(2)] + [p for _, p in all_plans(vs) if _.startswith("km")]
    with vs.Engine(g.V, plans) as e:
        e.set_option("set_reuse", reuse)
        e.set_option("edge_triangles", 0)  # the diamond through the plan's ops
        e.transfer_view(g, np.arange(g.V, dtype=np.uint32))
        e.match()
        assert e.counts() == [orc.count(p, g) for p in plans]


def _star_of_cliques(vs, sizes=(20, 150, 600, 2000), chords=3, seed=8):
    """Disjoint hubs, hub h joined to its leaves, the leaves on a ring with random
    chords, ids kept as built (each hub below its leaves): the hubs' out-degrees are
    the sizes, one per tier of the clique operator (<= 32, <= 256, <= 1024, wider)."""
    rng = np.random.default_rng(seed)
    edges, base = set(), 0
    for n in sizes:
        h = base
        leaves = list(range(base + 1, base + n + 1))
        edges |= {(h, x) for x in leaves}
        edges |= {(leaves[i], leaves[(i + 1) % n]) for i in range(n)}
        for a, b in rng.integers(0, n, size=(chords * n, 2)):
            if a != b:
                edges.add((leaves[min(a, b)], leaves[max(a, b)]))
        base += n + 1
    rows = [[] for _ in range(base)]
    for a, b in edges:
        rows[a].append(b)
        rows[b].append(a)
    rp = np.zeros(base + 1, np.uint64)
    rp[1:] = np.cumsum([len(r) for r in rows])
    return vs.Graph(rp, np.array([x for r in rows for x in sorted(set(r))], dtype=np.uint32))


def test_clique_bits_every_tier(vs, orc, graphs):
    """The bitmap clique operator (each root's out-neighbourhood as bit rows) in all
    of its tiers and its fallback to the plan, per root and in total, against the
    rooted clique oracle; dense rows on complete graphs against closed forms."""
    from math import comb
    star = _star_of_cliques(vs)
    kc = [vs.plan_clique(3), vs.plan_clique(4)]
    for g in (star, graphs["rmat8"], graphs["chunglu"], vs.degree_relabel(graphs["rmat8"])[0], complete_graph(vs, 300)):
        want = [orc.cliques_by_smallest(3, g), orc.cliques_by_smallest(4, g)]
        for bits in (1, 0):
            with vs.Engine(g.V, kc) as e:
                e.set_option("clique_bits", bits)
                e.transfer_view(g, np.arange(g.V, dtype=np.uint32))
                e.match()
                assert e.counts() == want, (bits, g.V)
                # root subsets: the per-root attribution (smallest vertex)
                for src in (np.arange(0, g.V, 3, dtype=np.uint32), np.array([0, 21, 172, 773], np.uint32) % g.V):
                    src = np.unique(src)
                    e.reset_counts()
                    e.transfer_view(g, src)
                    e.match()
                    assert e.counts() == [orc.cliques_by_smallest(3, g, src), orc.cliques_by_smallest(4, g, src)], (bits, g.V)
    # K_1100: every row full, roots 0..74 wider than the block tier
    k = complete_graph(vs, 1100)
    with vs.Engine(k.V, kc) as e:
        e.transfer_view(k, np.arange(k.V, dtype=np.uint32))
        e.match()
        assert e.counts() == [comb(1100, 3), comb(1100, 4)]
        # out-degree 1099 - u: 1025 / 1024 / 257 / 256 / 33 / 32 / 3 / 2 at the tier edges
        for u in (0, 74, 75, 842, 843, 1066, 1067, 1096, 1097, 1099):
            e.reset_counts()
            e.transfer_view(k, np.array([u], np.uint32))
            e.match()
            assert e.counts() == [comb(1099 - u, 2), comb(1099 - u, 3)], u


def test_diamond_from_edge_triangles(vs, orc, graphs):
    """The diamond (-p 2) from per-edge triangle counts: per root (any source subset,
    so the triangles whose smallest vertex is a lower neighbour of a source count
    too), on views built by halo, in every tier of the triangle kernels and with the
    fallback to the plan when an out-neighbourhood is wider than the block tier."""
    p = vs.plan_pattern(2)
    star = _star_of_cliques(vs, sizes=(20, 150, 2000, 17000), chords=1)
    for g in (star, graphs["rmat8"], graphs["chunglu"], vs.degree_relabel(graphs["rmat8"])[0], complete_graph(vs, 60)):
        rng = np.random.default_rng(g.V)
        subsets = [np.arange(g.V, dtype=np.uint32), np.sort(rng.choice(g.V, size=max(1, g.V // 5), replace=False)).astype(np.uint32),
                   np.array([0, 21, 172, 2173], np.uint32) % g.V]
        for src in subsets:
            src = np.unique(src)
            want = orc.count(p, g, src)
            for tri in (1, 0):
                with vs.Engine(g.V, [p]) as e:
                    e.set_option("edge_triangles", tri)
                    e.transfer_view(g, src)
                    e.match()
                    assert e.counts() == [want], (tri, g.V, len(src))
    # views built by halo around interleaved bins (rows beyond the halo are empty)
    g = graphs["chunglu"]
    with vs.Engine(g.V, [p]) as e:
        e.upload_graph(g)
        for b in range(3):
            src = np.arange(b, g.V, 3, dtype=np.uint32)
            e.reset_counts()
            e.materialize_view(src, p.hop)
            e.match()
            assert e.counts() == [orc.count(p, g, src)], b


def test_compute_path_count_op(vs, orc, graphs):
    """COMPUTE_PATH_COUNT (sizes only) followed by COUNT, level-wise and in the
    persistent batched launch, equals the oracle; a plan that would read such a
    vertex's set later is rejected at vsgm_create."""
    from conftest import with_path_count
    g = graphs["chunglu"]
    base = [vs.plan_clique(3), vs.plan_clique(4), vs.plan_pattern(1), vs.plan_clique(5)]
    plans = [with_path_count(vs, p) for p in base]
    want = [orc.count(p, g) for p in base]
    assert [orc.count(p, g) for p in plans] == want
    with vs.Engine(g.V, plans, hbm_budget_bytes=1 << 22) as e:  # a small budget: the sizes come in batches
        e.set_option("clique_bits", 0)
        e.set_option("c4_aggregate", 0)
        e.transfer_view(g, np.arange(g.V, dtype=np.uint32))
        e.match()
        assert e.counts() == want
    with vs.Engine(g.V, plans) as e:
        vid = e.add_view(g)
        e.set_option("hybrid_steps", 0)
        assert [row[0] for row in e.run_batched([vid])] == want
    bad = with_path_count(vs, vs.plan_clique(3))
    bad.op_type[bad.n_ops - 1] = vs.capi.COMPUTE_COUNT  # would read the sizes-only set as a set
    bad.computed_unmat[bad.n_ops - 1].count = 1
    with pytest.raises(vs.VsgmError):
        vs.Engine(g.V, [bad])


def test_four_cycle_wide_and_packed_counters(vs, orc):
    """Heavy 4-cycle roots count with 16-bit counters when they have fewer than 65536
    neighbours below them and with 32-bit counters otherwise: a wheel whose hub has
    70000 lower neighbours (each rim vertex closes one cycle through the hub) plus
    a smaller wheel of 3000, against the oracle, with every root in the groups."""
    def wheel(n, base):
        edges = {(base, base + 1 + i) for i in range(n)} | {(base + 1 + i, base + 1 + (i + 1) % n) for i in range(n)}
        return edges, n + 1
    e1, n1 = wheel(70000, 0)
    e2, n2 = wheel(3000, n1)
    n = n1 + n2
    rows = [[] for _ in range(n)]
    for a, b in e1 | e2:
        rows[a].append(b)
        rows[b].append(a)
    rp = np.zeros(n + 1, np.uint64)
    rp[1:] = np.cumsum([len(r) for r in rows])
    g, _ = vs.degree_relabel(vs.Graph(rp, np.array([x for r in rows for x in sorted(r)], dtype=np.uint32)))
    want = orc.c4_by_largest_wedges(g)
    for heavy in (0, 1 << 10, 12289):
        for window, bal in ((0, 1), (1, 1), (0, 0)):
            with vs.Engine(g.V, [vs.plan_pattern(1)]) as e:
                e.set_option("c4_heavy", heavy)
                e.set_option("c4_window", window)
                e.set_option("c4_balance", bal)
                e.transfer_view(g, np.arange(g.V, dtype=np.uint32))
                e.match()
                assert e.counts() == [want], (heavy, window, bal)


def test_isomorphic_queries_count_alike(vs, orc, graphs):
    """The batched runs count one pattern per isomorphism class of the batch: on a
    view whose every vertex is a source, relabelled copies of a pattern (different
    plans, different roots) have the same exact count, and it is the oracle's."""
    from vsgm_b200 import workloads as wl
    pats = [p for p in wl.random_patterns(64, seed=3) if p.n_vertices <= 5]
    reps, cls = vs.query_classes(pats)
    assert len(reps) < len(pats)
    g = graphs["rmat7"]
    with vs.Engine(g.V, pats) as e:
        e.transfer_view(g, np.arange(g.V, dtype=np.uint32))
        e.match()
        got = e.counts()
    for i, p in enumerate(pats):
        assert got[i] == got[reps[cls[i]]], i
    for r in reps:
        assert got[r] == orc.count(pats[r], g), r
