"""Run one of the five workload configurations on one GPU; print one JSON line.

    python -m vsgm_b200.run_configs c1 | c3 | c4 | c5 [options]

c1  -kc 3 on R-MAT scale 16, edge factor 16, seed 1, ids ascending with degree
    (the degree-ordered orientation), one view holding every source.
c3  64 random connected patterns (3-6 vertices, p = 0.5, seed 3) x 16 Chung-Lu
    views (exponent U[2.1, 2.8], edges log-uniform in [1e5, e_max] (default 1e6;
    the configuration's 1e7 with --e-max 1e7), max degree 1e4, seed 3): the
    persistent batched (hybrid) run and, with --learned, the batched run over the
    learned planner's orders, against the plain level-wise engine with the
    heuristic order view after view, at identical counts.  The batched runs count
    each isomorphism class of the batch once (every view holds all its vertices as
    sources, so isomorphic patterns have equal counts; --no-dedup counts every
    pattern).  Patterns whose sampled work exceeds --max-work on some view are left
    out and listed.
c4  the learned planner on c3-distributed (pattern, view) pairs (seed 4): the
    network is trained by the library's MLP kernels on measured per-op work of
    candidate orders; held-out pairs report the work of the heuristic order and
    of the verified learned choice on an independent root sample.
views  the view-bin chain (features, kmeans, view_packing) of C2 on the device,
    timed and, with --reference, compared with the reference's own tools.
c5  Chung-Lu, 65M vertices, ~1.8B edges, exponent 2.2, max degree 5000, seed 5
    (use --scale-down k for a 1/k-size graph of the same shape): -kc 3, -kc 4,
    -p 4 (house), whole graph as one view, plus the same totals over 4
    interleaved source bins as a size-independent consistency check.

Counts are exact u64; times are device times from the engine's CUDA events
(value) and wall time around the C ABI calls (wall).  No oracle is used here:
parity is the test suite's job.
"""
import argparse
import json
import sys
import time

import numpy as np

from . import Engine, Graph, degree_relabel, gen_rmat, plan_clique, plan_pattern, query_classes
from . import planner as lp
from . import workloads as wl


def _match_all(g, plans, device=0, sources=None, options=()):
    src = np.arange(g.V, dtype=np.uint32) if sources is None else sources
    with Engine(g.V, plans, device=device) as e:
        for k, v in options:
            e.set_option(k, v)
        e.transfer_view(g, src)
        e.set_profiling(True)
        e.match()  # warm-up (first-touch of the arena, module load)
        e.reset_counts()
        t = time.perf_counter()
        e.match()
        wall = time.perf_counter() - t
        per = []
        for i, p in enumerate(plans):
            s = e.stats(i)
            per.append(sum(s.op_ms[j] for j in range(p.n_ops)))
        return e.counts(), per, wall


def run_c1(args):
    g = gen_rmat(16, 16, *wl.RMAT_ABC, seed=1)
    g, _ = degree_relabel(g, ascending=True)
    counts, per, wall = _match_all(g, [plan_clique(3)])
    return {"config": "c1", "graph": f"R-MAT 16 ef16 seed 1, V={g.V}, E={g.E}", "query": "-kc 3", "count": counts[0],
            "device_ms": per[0], "wall_ms": wall * 1e3, "matches_per_s": counts[0] / (per[0] / 1e3) if per[0] else None}


def _screen(plans, views, stride, step_budget, device=0):
    V = max(g.V for g in views)
    with Engine(V, plans, device=device) as e:
        ids = [e.add_view(g, np.arange(0, g.V, stride, dtype=np.uint32)) for g in views]
        cnt, lvl, ovf = e.run_batched_ex(ids, step_budget=step_budget)
    return lvl.sum(axis=2) * stride, ovf


def _train_planner(args):
    """A planner trained on c4-distributed pairs (seed 4), or loaded from --model."""
    model = lp.LearnedPlanner()
    if args.model:
        model.load(args.model)
        return model, 0.0
    views = [degree_relabel(g)[0] for g in wl.chung_lu_views(args.views, seed=4, e_min=2e4, e_max=2e5, max_degree=2000)]
    pats = wl.random_patterns(args.patterns, seed=4)
    sampler = lp.Sampler(views, roots_per_view=256, seed=1, step_budget=500_000)
    pairs = [(pi, vi) for pi in range(len(pats)) for vi in range(len(views))]
    t = time.perf_counter()
    X, Y, M, _ = lp.make_examples(sampler, pats, pairs, orders_per_pair=8, seed=1)
    model.train(X, Y, M, epochs=150)
    return model, time.perf_counter() - t


def run_c3(args):
    views = [degree_relabel(g)[0] for g in wl.chung_lu_views(16, seed=3, e_max=args.e_max)]
    pats = wl.random_patterns(64, seed=3)
    work, ovf = _screen(pats, views, stride=97, step_budget=200_000)
    keep = [i for i in range(len(pats)) if not ovf[i].any() and work[i].max() < args.max_work]
    plans = [pats[i] for i in keep]
    V = max(g.V for g in views)
    # the batch's isomorphism classes: every view holds all its vertices as sources,
    # so one count per class and view serves every pattern of the class
    if args.no_dedup:
        reps, cls = list(range(len(plans))), list(range(len(plans)))
    else:
        reps, cls = query_classes(plans)
    rplans = [plans[i] for i in reps]
    # batched: every (class representative, view) pair in one persistent (hybrid) run
    with Engine(V, rplans) as e:
        ids = [e.add_view(g) for g in views]
        e.set_profiling(True)
        e.run_batched(ids)  # warm-up
        t = time.perf_counter()
        rb = e.run_batched(ids)
        b_wall = time.perf_counter() - t
        st = e.batch_stats()
        b_ms, tasks, b_level = st.ms, st.tasks, st.level_pairs
    batched = [rb[cls[pi]] for pi in range(len(plans))]
    learned = None
    if args.learned:
        # batched + learned: the planner proposes orders per (class, view), the
        # level-wise engine times them on a root sample of that view, then one
        # hybrid run over the chosen plans
        model, t_train = _train_planner(args)
        sampler = lp.Sampler(views, roots_per_view=256, seed=1, step_budget=500_000)
        t = time.perf_counter()
        chosen = [model.choose_timed_many(rplans, sampler, vi, k=4) for vi in range(len(views))]
        t_plan = time.perf_counter() - t
        model.close()
        uniq, pair_list = [], []
        for vi in range(len(views)):
            for ri, (order, _) in enumerate(chosen[vi]):
                key = (ri, tuple(order))
                if key not in uniq:
                    uniq.append(key)
                pair_list.append((uniq.index(key), vi))
        lplans = [lp.plan_reorder(rplans[ri], o) for ri, o in uniq]
        with Engine(V, lplans) as e:
            ids = [e.add_view(g) for g in views]
            e.set_profiling(True)
            e.run_pairs([(a, ids[b]) for a, b in pair_list])  # warm-up
            t = time.perf_counter()
            got = e.run_pairs([(a, ids[b]) for a, b in pair_list])
            l_wall = time.perf_counter() - t
            lst = e.batch_stats()
        rcounts = [[0] * len(views) for _ in rplans]
        for (a, vi), c in zip(pair_list, got):
            rcounts[uniq[a][0]][vi] = c
        lcounts = [rcounts[cls[pi]] for pi in range(len(plans))]
        learned = {"changed_pairs": [[int(keep[reps[ri]]), vi] for vi in range(len(views)) for ri, (_, took) in enumerate(chosen[vi]) if took],
                   "wall_ms": l_wall * 1e3, "device_ms": lst.ms, "level_pairs": int(lst.level_pairs), "tasks": int(lst.tasks),
                   "orders_changed": sum(int(took) for row in chosen for _, took in row), "plan_s": t_plan, "train_s": t_train,
                   "counts": lcounts}
    # plain: the level-wise engine, one view after the other (uploads outside the timing)
    plain = [[0] * len(views) for _ in plans]
    pair_ms = np.zeros((len(plans), len(views)))
    p_ms = p_wall = 0.0
    launches = 0
    with Engine(V, plans) as e:
        e.set_profiling(True)
        for vi, g in enumerate(views):
            rp = np.concatenate([g.row_ptrs, np.full(V - g.V, g.row_ptrs[-1], np.uint64)])
            e.transfer_view(Graph(rp, g.cols), np.arange(g.V, dtype=np.uint32))
            e.reset_counts()
            t = time.perf_counter()
            e.match()
            p_wall += time.perf_counter() - t
            c = e.counts()
            for pi, p in enumerate(plans):
                plain[pi][vi] = c[pi]
                s = e.stats(pi)
                pair_ms[pi, vi] = sum(s.op_ms[j] for j in range(p.n_ops))
                p_ms += pair_ms[pi, vi]
                launches += sum(s.op_launches[j] for j in range(p.n_ops))
    total = sum(sum(r) for r in plain)
    out = {"config": "c3", "views": [(g.V, g.E) for g in views], "patterns_run": len(keep), "pattern_classes": len(reps),
           "dedup": not args.no_dedup,
           "patterns_left_out": [i for i in range(len(pats)) if i not in keep],
           "identical_counts": [list(map(int, r)) for r in batched] == plain, "matches": int(total),
           "batched": {"device_ms": b_ms, "wall_ms": b_wall * 1e3, "tasks": int(tasks), "level_pairs": int(b_level)},
           "plain": {"device_ms": p_ms, "wall_ms": p_wall * 1e3, "launches": int(launches)},
           "speedup_wall": p_wall / b_wall if b_wall else None}
    # where the plain engine's time goes: the heaviest (pattern, view) pairs
    top = np.argsort(pair_ms, axis=None)[::-1][:16]
    out["plain_top_pairs"] = [{"pattern": int(keep[i // len(views)]), "view": int(i % len(views)), "ms": float(pair_ms.flat[i]),
                               "vertices": int(plans[i // len(views)].n_vertices), "edges": int(plans[i // len(views)].n_edges),
                               "count": int(plain[i // len(views)][i % len(views)])} for i in top]
    out["plain_top16_share"] = float(pair_ms.flat[top].sum() / max(pair_ms.sum(), 1e-9))
    if learned:
        out["learned_identical_counts"] = learned.pop("counts") == plain
        out["batched_learned"] = learned
        out["speedup_learned_wall"] = p_wall / (learned["wall_ms"] / 1e3) if learned["wall_ms"] else None
    return out


def run_c4(args):
    views = [degree_relabel(g)[0] for g in wl.chung_lu_views(args.views, seed=4, e_min=2e4, e_max=args.e_max, max_degree=2000)]
    pats = wl.random_patterns(args.patterns, seed=4)
    sampler = lp.Sampler(views, roots_per_view=256, seed=1, step_budget=500_000)
    check = lp.Sampler(views, roots_per_view=256, seed=99, step_budget=4_000_000)
    pairs = [(pi, vi) for pi in range(len(pats)) for vi in range(len(views))]
    rng = np.random.default_rng(0)
    rng.shuffle(pairs)
    cut = int(0.8 * len(pairs))
    t = time.perf_counter()
    X, Y, M, _ = lp.make_examples(sampler, pats, pairs[:cut], orders_per_pair=8, seed=1)
    t_logs = time.perf_counter() - t
    model = lp.LearnedPlanner()
    t = time.perf_counter()
    losses = model.train(X, Y, M, epochs=150)
    t_train = time.perf_counter() - t
    heur = learned = 0.0
    used = 0
    for pi, vi in pairs[cut:]:
        base = pats[pi]
        order, took = model.choose_verified(base, sampler, vi, k=4)
        used += took
        plans = [lp.plan_reorder(base, lp.heuristic_order(base)), lp.plan_reorder(base, order)]
        cnt, lvl, ovf = check.evaluate(plans, vi)
        heur += sum(int(x) for x in lvl[0][0][:plans[0].n_ops])
        learned += sum(int(x) for x in lvl[1][0][:plans[1].n_ops])
    # plan error: predicted against measured log intermediate sizes of several orders
    # of every held-out pair
    Xh, Yh, Mh, _ = lp.make_examples(sampler, pats, pairs[cut:], orders_per_pair=8, seed=2)
    err = lp.plan_error(model.predict(Xh), Yh, Mh)
    if args.save:
        model.save(args.save)
    model.close()
    return {"config": "c4", "plan_error": err, "train_pairs": cut, "held_out_pairs": len(pairs) - cut, "examples": int(len(X)), "log_s": t_logs, "train_s": t_train,
            "loss_first": losses[0], "loss_last": losses[-1], "model_order_used": used,
            "held_out_work": {"heuristic": heur, "learned": learned, "gain": heur / learned if learned else None}}


def run_c5(args):
    """C5: generate, relabel on the host and (the engine's resident copy) on the
    device - the two must agree - count the three queries over every source with
    their device times, and check that 4 interleaved source bins sum to the totals.
    (Exact parity on a root sample with the hubs: tests/test_configs_gpu.py.)"""
    k = args.scale_down
    t = time.perf_counter()
    raw = wl.social_chung_lu(V=65_000_000 // k, edges=1_800_000_000 // k)
    t_gen = time.perf_counter() - t
    t = time.perf_counter()
    g, new_of_old = degree_relabel(raw, ascending=True)
    t_host_relabel = time.perf_counter() - t
    plans = [plan_clique(3), plan_clique(4), plan_pattern(4)]
    out = {"config": "c5", "graph": f"Chung-Lu V={g.V} E={g.E} (exponent 2.2, max degree 5000, seed 5)", "scale_down": k, "gen_s": t_gen,
           "host_relabel_s": t_host_relabel, "queries": ["-kc 3", "-kc 4", "-p 4"]}
    print(json.dumps({"progress": out}), flush=True)
    with Engine(g.V, plans) as e:
        e.set_option("relabel", 1)
        t = time.perf_counter()
        e.upload_graph(raw)
        out["upload_and_device_relabel_s"] = time.perf_counter() - t
        e.graph_view(np.arange(g.V, dtype=np.uint32))
        r = e.read_view()
        out["device_relabel_equals_host"] = bool(np.array_equal(r.row_ptrs, g.row_ptrs) and np.array_equal(r.cols, g.cols))
        del r
        e.set_profiling(True)
        counts, per = [], []
        for i in range(len(plans)):
            e.set_option("only_plan", i)
            # the house (-p 4) first on every args.house_stride-th root, to bound its time
            stride = args.house_stride if i == 2 else 1
            e.set_option("root_stride", stride)
            e.reset_counts()
            t = time.perf_counter()
            e.match()
            wall = time.perf_counter() - t
            counts.append(e.counts()[i])
            s = e.stats(i)
            per.append({"query": out["queries"][i], "count": counts[-1], "device_ms": sum(s.op_ms[j] for j in range(plans[i].n_ops)),
                        "wall_ms": wall * 1e3, "root_stride": stride})
            print(json.dumps({"progress": per[-1]}), flush=True)
        e.set_option("only_plan", -1)
        e.set_option("root_stride", 1)
        e.set_profiling(False)
        out["per_query"] = per
        out["counts"] = counts
        # the same totals over 4 interleaved source bins (caller ids)
        e.reset_counts()
        t = time.perf_counter()
        for b in range(4):
            e.graph_view(np.arange(b, g.V, 4, dtype=np.uint32))
            for i in (0, 1):
                e.set_option("only_plan", i)
                e.match()
        e.set_option("only_plan", -1)
        out["bins_wall_ms"] = (time.perf_counter() - t) * 1e3
        out["bins_total_equal_kc3_kc4"] = e.counts()[:2] == counts[:2]
    return out


def run_views(args):
    """The view-bin chain of C2 on the device: features -h 1, kmeans -k 4 -i
    --kmeans-iters -init 1, view_packing -h 2 at 40 GB and at 0.45 GB, on R-MAT 22
    in the generator's ids; with --reference the reference's own tools (built in
    oracle/_ref) run on the same files with all host threads, their outputs are
    compared and both are timed.  The reference kmeans runs with -t 1 when
    --reference-kmeans-t1 is given (its random start is then the same draw)."""
    import os
    import shutil
    import subprocess
    import tempfile

    from . import features_1hop, kmeans, packing_order, reference_rand_starts, view_packing, write_csr_bin
    g = gen_rmat(22, 16, *wl.RMAT_ABC, seed=2)
    out = {"config": "views", "graph": f"R-MAT 22 ef 16 seed 2, V={g.V}, E={g.E}", "kmeans_iters": args.kmeans_iters}
    t = time.perf_counter()
    h = features_1hop(g)
    out["features_ms"] = (time.perf_counter() - t) * 1e3
    t = time.perf_counter()
    part, sizes = kmeans(h, 4, args.kmeans_iters, starts=reference_rand_starts(4, 1))
    out["kmeans_ms"] = (time.perf_counter() - t) * 1e3
    out["cluster_sizes"] = sizes.tolist()
    order, offs = packing_order(part, "1x4", 1)
    for mem in (40, 0.45):
        t = time.perf_counter()
        bins, nb, _ = view_packing(g, order, offs, 2, mem)
        out[f"packing_{mem}GB_ms"] = (time.perf_counter() - t) * 1e3
        out[f"packing_{mem}GB_bins"] = nb
    if args.reference:
        ref = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")
        threads = str(os.cpu_count() or 1)
        with tempfile.TemporaryDirectory() as d:
            write_csr_bin(os.path.join(d, "g.bin"), g)

            def timed(*cmd):
                t0 = time.perf_counter()
                r = subprocess.run(list(cmd), cwd=d, capture_output=True, text=True, timeout=3600)
                if r.returncode != 0:
                    raise RuntimeError(r.stderr[-500:])
                return (time.perf_counter() - t0) * 1e3

            out["reference_threads"] = int(threads)
            out["reference_features_ms"] = timed(os.path.join(ref, "features"), "-f", "g.bin", "-h", "1", "-t", threads)
            kt = "1" if args.reference_kmeans_t1 else threads
            out["reference_kmeans_threads"] = int(kt)
            out["reference_kmeans_ms"] = timed(os.path.join(ref, "kmeans"), "-f", "g.bin.1hop.bin", "-k", "4", "-i", str(args.kmeans_iters), "-t", kt,
                                               "-init", "1")
            want = np.loadtxt(os.path.join(d, "g.bin.1hop.bin.kmeans.4"), dtype=np.int32)
            if kt == "1":
                out["kmeans_equal_reference"] = bool(np.array_equal(want, part))
            shutil.copy(os.path.join(d, "g.bin.1hop.bin.kmeans.4"), os.path.join(d, "g.bin.kmeans.1x4"))
            r_order, r_offs = packing_order(want, "1x4", 1)
            for mem in (40, 0.45):
                out[f"reference_packing_{mem}GB_ms"] = timed(os.path.join(ref, "view_packing"), "-gf", "g.bin", "-pf", "g.bin.kmeans.1x4", "-h", "2",
                                                             "-m", str(mem), "-t", "1", "-s", "1")
                wb = np.loadtxt(os.path.join(d, "g.bin.2.hop.vbmap"), dtype=np.int32)
                bins, nb, _ = view_packing(g, r_order, r_offs, 2, mem)
                out[f"packing_{mem}GB_equal_reference"] = bool(int(wb[0]) == nb and np.array_equal(wb[1:], bins))
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("config", choices=["c1", "c3", "c4", "c5", "views"])
    ap.add_argument("--kmeans-iters", type=int, default=10, help="views: k-means iterations")
    ap.add_argument("--reference", action="store_true", help="views: also run and compare the reference's tools from oracle/_ref")
    ap.add_argument("--reference-kmeans-t1", action="store_true", help="views: run the reference kmeans with -t 1 (same random start)")
    ap.add_argument("--e-max", type=float, default=None)
    ap.add_argument("--max-work", type=float, default=5e9)
    ap.add_argument("--views", type=int, default=8)
    ap.add_argument("--patterns", type=int, default=96)
    ap.add_argument("--scale-down", type=int, default=1)
    ap.add_argument("--house-stride", type=int, default=1, help="c5: count the house on every k-th root only")
    ap.add_argument("--learned", action="store_true", help="c3: also run batched + learned orders")
    ap.add_argument("--no-dedup", action="store_true", help="c3: batched runs count every pattern, not one per isomorphism class")
    ap.add_argument("--model", default=None, help="c3 --learned: planner parameters (.npy from c4 --save)")
    ap.add_argument("--save", default=None, help="c4: write the trained planner's parameters here")
    args = ap.parse_args(argv)
    if args.e_max is None:
        args.e_max = {"c3": 1e6, "c4": 2e5}.get(args.config, 1e7)
    out = {"c1": run_c1, "c3": run_c3, "c4": run_c4, "c5": run_c5, "views": run_views}[args.config](args)
    print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
