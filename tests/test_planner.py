"""Planner parity: the product planner reproduces the reference planner's plans.

tests/golden/ref_plans.jsonl was produced by the reference's own Plan::Optimize
(src/query/plan.h:548-561), compiled from source by oracle/Makefile (see
tests/golden/make_plan_golden.py): all preset patterns, cliques 3..7, graphlets
3..5 and 400 seeded random connected patterns of 3..7 vertices.
"""
import json
import os

import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_plans.jsonl")


def _rows():
    with open(GOLDEN) as f:
        return [json.loads(line) for line in f]


def _plan_for(vs, row, cache):
    name = row["name"]
    if name.startswith("kc"):
        return vs.plan_clique(int(name[2:]))
    if name.startswith("km"):
        k, i = int(name[2]), int(name.split("_")[1])
        if k not in cache:
            cache[k] = vs.plan_graphlets(k)
        return cache[k][i]
    if name.startswith("p"):
        return vs.plan_pattern(int(name[1:]))
    n, b = row["input_n"], row["input_bits"]
    return vs.plan_query([[j for j in range(n) if b[i * n + j] == "1"] for i in range(n)])


def test_golden_covers_every_query_family():
    names = [r["name"] for r in _rows()]
    assert sum(n.startswith("rand") for n in names) == 400
    assert {f"p{i}" for i in range(19)} <= set(names)
    assert {f"kc{k}" for k in range(3, 8)} <= set(names)
    assert sum(n.startswith("km") for n in names) == 2 + 6 + 21


def test_plans_match_reference_planner(vs):
    cache = {}
    bad = []
    for row in _rows():
        mine = _plan_for(vs, row, cache).to_dict()
        for key, val in mine.items():
            if row[key] != val:
                bad.append((row["name"], key, row[key], val))
                break
    assert not bad, bad[:5]


def test_reorder_keeps_heuristic_tables_for_heuristic_sequence(vs):
    for p in [vs.plan_pattern(i) for i in range(19)] + [vs.plan_clique(k) for k in range(3, 8)]:
        q = vs.plan_reorder(p, [p.seq[i] for i in range(p.n_vertices)])
        assert q.to_dict() == p.to_dict()


def test_reorder_rejects_disconnected_prefix(vs):
    p = vs.plan_pattern(1)  # 4-cycle: 0-1, 0-2, 1-3, 2-3 after re-mapping
    adj = p.adjacency()
    bad_seq = [0, 3, 1, 2] if 3 not in adj[0] else [1, 2, 0, 3]
    with pytest.raises(vs.VsgmError):
        vs.plan_reorder(p, bad_seq)


def test_bad_pattern_ids_fail_cleanly(vs):
    with pytest.raises(vs.VsgmError):
        vs.plan_pattern(19)
    with pytest.raises(vs.VsgmError):
        vs.plan_clique(2)
    with pytest.raises(vs.VsgmError):
        vs.plan_query([[1], [0], []])  # disconnected
