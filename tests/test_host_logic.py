"""Host-side logic that needs no GPU: bench query parsing, the autotuner's search
space, the learned planner's order bookkeeping and its verified choice (driven by
a stand-in sampler and network), and root sharding."""
import numpy as np
import pytest


def test_bench_query_flags():
    import bench
    assert bench.parse_queries("kc4,p1,p2") == ["-kc 4", "-p 1", "-p 2"]
    assert bench.parse_queries(" kc3 ") == ["-kc 3"]
    with pytest.raises(SystemExit):
        bench.parse_queries("q7")


def test_autotune_space_has_no_redundant_settings():
    from vsgm_b200.autotune import CANDIDATES, _settings
    cfgs = list(_settings(CANDIDATES))
    keys = [tuple(sorted(c.items())) for c in cfgs]
    assert len(keys) == len(set(keys))
    for c in cfgs:
        if not c["fuse_tail"]:
            assert c["stage_cap"] == CANDIDATES["stage_cap"][0] and c["walk_ratio"] == CANDIDATES["walk_ratio"][0]
        if c["lane_merge"]:
            assert c["merge_ratio"]
    # every knob value is reachable
    for k, vals in CANDIDATES.items():
        assert {c[k] for c in cfgs} == set(vals)


def test_valid_orders_and_ranks(vs):
    from vsgm_b200 import planner as lp
    p = vs.plan_pattern(1)  # 4-cycle
    orders = lp.valid_orders(p)
    assert lp.heuristic_order(p) in orders
    for o in orders:  # every later vertex has an earlier neighbour
        seen = 1 << o[0]
        for v in o[1:]:
            assert p.adj[v] & seen
            seen |= 1 << v
    ranks = [lp.order_index(o) for o in orders]
    assert len(set(ranks)) == len(ranks) and max(ranks) < 24
    x = lp.features(p, np.full(32, 1 / 32, np.float32), np.arange(24))
    assert x.shape == (lp.N_IN,) and x.dtype == np.float32


class _Sampler:
    """Stand-in sampler: per-op work of an order is a fixed function of the order."""

    def __init__(self, work_of):
        self.work_of = work_of
        self.hist = [np.full(32, 1 / 32, np.float32)]
        self.calls = 0

    def evaluate(self, plans, view_index):
        self.calls += 1
        lvl = np.zeros((len(plans), 1, 24), np.uint64)
        ovf = np.zeros((len(plans), 1), np.uint32)
        for i, p in enumerate(plans):
            seq = tuple(int(p.seq[j]) for j in range(p.n_vertices))
            w = self.work_of(seq)
            if w is None:
                ovf[i][0] = 1
                w = 10
            lvl[i][0][0] = w
        return np.zeros((len(plans), 1), np.uint64), lvl, ovf


def _stub_model(scores):
    from vsgm_b200 import planner as lp
    m = lp.LearnedPlanner.__new__(lp.LearnedPlanner)  # no device network: predictions are given
    m.h = None
    m.predict = lambda X: np.tile(scores, (len(X), 1))
    return m


def test_verified_choice_takes_measured_gain_and_falls_back(vs):
    from vsgm_b200 import planner as lp
    p = vs.plan_pattern(1)
    h = lp.heuristic_order(p)
    others = [o for o in lp.valid_orders(p) if o != h]
    good, bad = others[0], others[1]
    scores = np.full(lp.N_OUT, 10.0, np.float32)
    scores[lp.order_index(good)] = 1.0  # the network ranks `good` and `bad` first
    scores[lp.order_index(bad)] = 2.0
    model = _stub_model(scores)
    # measured: good does half the heuristic's work -> chosen
    s = _Sampler(lambda o: 500 if o == good else (2000 if o == bad else 1000))
    assert model.choose_verified(p, s, 0, k=2) == (good, True)
    assert model.choose_verified_many([p, p], s, 0, k=2) == [(good, True), (good, True)]
    assert s.calls == 2 + 2  # one features run + one candidates run per call
    # measured: no proposal beats the heuristic by the margin -> heuristic kept
    s = _Sampler(lambda o: 980 if o in (good, bad) else 1000)
    assert model.choose_verified(p, s, 0, k=2) == (h, False)
    # a proposal stopped by the step budget is never preferred
    s = _Sampler(lambda o: None if o == good else (400 if o == bad else 1000))
    assert model.choose_verified(p, s, 0, k=2) == (bad, True)


def test_strided_shards_partition_the_sources():
    from vsgm_b200.shard import roots_of_rank
    src = np.arange(1000, 1037, dtype=np.uint32)
    for world in (1, 2, 3, 8):
        parts = [roots_of_rank(len(src), r, world, src) for r in range(world)]
        allr = np.sort(np.concatenate(parts))
        assert np.array_equal(allr, src)
        assert max(len(x) for x in parts) - min(len(x) for x in parts) <= 1


def test_autotune_view_classes():
    """The tuner's view signature: degree histograms of the same shape share a class,
    a heavier tail or a larger hub does not."""
    import numpy as np

    from vsgm_b200.autotune import TuneCache, view_class
    rng = np.random.default_rng(1)
    a = rng.zipf(2.2, size=20000).clip(1, 5000)
    b = rng.zipf(2.2, size=20000).clip(1, 5000)
    assert view_class(a) == view_class(b)
    assert view_class(a) != view_class(np.full(20000, 64))
    assert view_class(np.full(100, 3)) != view_class(np.concatenate([np.full(99, 3), [100000]]))
    c = TuneCache()
    c.put(b"plan", view_class(a), {"fuse_tail": 0})
    assert c.get(b"plan", view_class(b)) == {"fuse_tail": 0} and c.get(b"other", view_class(b)) is None


def test_query_classes_group_isomorphic_patterns(vs):
    """Relabelled copies of a pattern fall into one class, different patterns into
    different classes (the batched runs count each class once)."""
    import itertools
    import random

    def bits_of(n, edges):
        b = [0] * 7
        for i, j in edges:
            b[i] |= 1 << j
            b[j] |= 1 << i
        return b

    rng = random.Random(5)
    shapes = {"house": (5, [(0, 1), (1, 2), (2, 3), (3, 4), (4, 0), (1, 4)]), "c5": (5, [(0, 1), (1, 2), (2, 3), (3, 4), (4, 0)]),
              "path4": (4, [(0, 1), (1, 2), (2, 3)]), "star4": (4, [(0, 1), (0, 2), (0, 3)]), "tri": (3, [(0, 1), (1, 2), (0, 2)])}
    plans, truth = [], []
    for name, (n, edges) in shapes.items():
        for _ in range(3):
            perm = list(range(n))
            rng.shuffle(perm)
            plans.append(vs.plan_query_bits(n, bits_of(n, [(perm[i], perm[j]) for i, j in edges])))
            truth.append(name)
    reps, cls = vs.query_classes(plans)
    assert len(reps) == len(shapes)
    for a, b in itertools.combinations(range(len(plans)), 2):
        assert (cls[a] == cls[b]) == (truth[a] == truth[b])
