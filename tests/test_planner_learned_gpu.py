"""Learned planner: trained by the library's own MLP kernels on costs measured by
the batched engine; the plans it picks give identical exact counts, and on held-out
(pattern, view) pairs they do no more work than the heuristic order overall.

The reference's only order is Plan::GenerateSearchSequence (src/query/plan.h:210-265).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(vs):
    from vsgm_b200 import planner as lp
    from vsgm_b200 import workloads as wl

    views = [vs.degree_relabel(vs.gen_chung_lu(V, E, gam, 600, seed=40 + i))[0]
             for i, (V, E, gam) in enumerate(wl.chung_lu_specs(4, seed=4, e_min=5e3, e_max=4e4))]
    pats = wl.random_patterns(48, seed=4)
    sampler = lp.Sampler(views, roots_per_view=256, seed=1, step_budget=400_000)
    pairs = [(pi, vi) for pi in range(len(pats)) for vi in range(len(views))]
    rng = np.random.default_rng(0)
    rng.shuffle(pairs)
    cut = int(0.75 * len(pairs))
    train = lp.make_examples(sampler, pats, pairs[:cut], orders_per_pair=8, seed=1)
    model = lp.LearnedPlanner()
    losses = model.train(*train[:3], epochs=150)
    yield vs, lp, views, pats, sampler, model, losses, pairs[cut:]
    model.close()


def test_training_converges(setup):
    *_, losses, _ = setup
    assert losses[-1] < 0.5 * losses[0]


def test_held_out_work_not_above_heuristic(setup):
    """On held-out (pattern, view) pairs the verified choice does no more work than
    the heuristic order, measured on a second, independent root sample."""
    vs, lp, views, pats, sampler, model, losses, held = setup
    check = lp.Sampler(views, roots_per_view=256, seed=99, step_budget=4_000_000)
    heur = learned = 0.0
    used = 0
    for pi, vi in held:
        base = pats[pi]
        order, took = model.choose_verified(base, sampler, vi, k=4)
        used += took
        plans = [lp.plan_reorder(base, lp.heuristic_order(base)), lp.plan_reorder(base, order)]
        # a different order roots each match at a different pattern vertex, so the
        # counts of one root sample differ; the work on a uniform root sample is an
        # unbiased estimate of each order's whole-view work
        cnt, lvl, ovf = check.evaluate(plans, vi)
        w = [sum(int(x) for x in lvl[i][0][:plans[i].n_ops]) for i in range(2)]
        heur += w[0]
        learned += w[1]
    print(f"held-out work ({len(held)} pairs, model order used on {used}): heuristic {heur:.4g}, learned {learned:.4g} "
          f"({heur / max(learned, 1):.2f}x)")
    assert learned <= heur * 1.02


def test_chosen_plans_count_exactly(setup):
    vs, lp, views, pats, sampler, model, losses, held = setup
    g = views[0]
    for pi in range(12):
        base = pats[pi]
        order, _ = model.choose_verified(base, sampler, 0, k=4)
        chosen = vs.plan_reorder(base, order)
        assert vs.count_graph(g, [chosen]) == vs.count_graph(g, [base])


def test_plan_error_on_held_out_pairs(setup):
    """The plain engine judges the network: on held-out pairs its predicted log
    intermediate sizes are compared with the measured ones of up to 8 orders per
    pair.  The report is the point (mean absolute error in log units, top-1 against
    chance, rank correlation); the network's ranking must correlate with the
    measurement.  Its top-1 pick is not reliably better than chance on this small
    training set, which is why choose_verified measures its proposals before using
    any of them."""
    vs, lp, views, pats, sampler, model, losses, held = setup
    X, Y, M, _ = lp.make_examples(sampler, pats, held, orders_per_pair=8, seed=2)
    err = lp.plan_error(model.predict(X), Y, M)
    print("plan error on held-out pairs:", err)
    assert err["pairs"] == len(held)
    assert err["mae_log"] is not None and np.isfinite(err["mae_log"])
    assert err["spearman"] is not None and err["spearman"] > 0.2
