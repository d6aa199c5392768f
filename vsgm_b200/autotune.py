"""Autotuner for the engine's per-plan knobs (intersection variant and tail fusion).

For every plan it times each candidate setting of (clique_bits, c4_aggregate, fuse_tail,
merge_ratio, lane_merge, stage_cap, walk_ratio) on a strided sample of the view's roots (engine option root_stride)
and keeps the fastest; the choice is written back as per-plan options, and kept per
(plan, degree-histogram class of the view) in a TuneCache for views of the same
class.  Counts
never depend on these knobs, so tuning on a sample is safe; the sample only has
to rank the settings.
"""
import itertools
import time

import numpy as np

CANDIDATES = {
    "clique_bits": (1, 0),
    "c4_aggregate": (1, 0),
    "fuse_tail": (1, 0),
    "merge_ratio": (0, 4, 16),
    "lane_merge": (0, 1),
    "stage_cap": (1536, 384),
    "walk_ratio": (8, 1),
}


def _settings(space):
    keys = list(space)
    for vals in itertools.product(*(space[k] for k in keys)):
        cfg = dict(zip(keys, vals))
        if not cfg["fuse_tail"] and (cfg["stage_cap"] != space["stage_cap"][0] or cfg.get("walk_ratio", 0) != space.get("walk_ratio", (0,))[0]):
            continue  # the stage and the walk only matter for the fused tail
        if cfg.get("lane_merge") and not cfg["merge_ratio"]:
            continue  # no merge, nothing to partition
        if cfg.get("clique_bits") and not cfg.get("c4_aggregate", 1):
            continue  # a plan is a clique or a 4-cycle, never both: one of the two settings suffices
        if cfg.get("c4_aggregate") and (cfg["fuse_tail"] != space["fuse_tail"][0] or cfg["merge_ratio"] != space["merge_ratio"][0]
                                        or cfg.get("lane_merge") or cfg["stage_cap"] != space["stage_cap"][0]
                                        or cfg.get("walk_ratio", 0) != space.get("walk_ratio", (0,))[0]):
            continue  # the other knobs do not matter when a 4-cycle is aggregated
        yield cfg


def view_class(degrees, buckets=8):
    """A coarse signature of a view's degree histogram: the share of vertices in each
    of `buckets` degree bands of a factor 4 each (rounded to tenths) and the band of
    the largest degree.  Views with the same signature get the same knobs from a TuneCache."""
    d = np.asarray(degrees, dtype=np.float64)
    band = np.minimum(buckets - 1, np.floor(np.log2(np.maximum(d, 1)) / 2).astype(np.int64))
    share = np.bincount(band, minlength=buckets)[:buckets] / max(1, len(d))
    top = int(np.floor(np.log2(max(1.0, float(d.max()) if len(d) else 1.0)) / 2))  # factor-4 bands, like the histogram
    return tuple(int(round(10 * x)) for x in share) + (top,)


class TuneCache:
    """Tuned knobs per (plan, view class): autotune() fills it, and a plan met again
    on a view of the same class is set from it without timing."""

    def __init__(self):
        self.best = {}

    @staticmethod
    def key(plan, cls):
        return (bytes(plan).hex(), cls)

    def get(self, plan, cls):
        return self.best.get(self.key(plan, cls))

    def put(self, plan, cls, cfg):
        self.best[self.key(plan, cls)] = dict(cfg)


def autotune(engine, n_plans, stride=64, space=None, cache=None, plans=None, degrees=None):
    """Tune every plan of an engine whose view is already transferred; returns
    [{"plan": i, "best": cfg, "ms": {cfg-key: ms}, "cached": bool}] and applies the
    best settings.  With a TuneCache, the plan objects and the view's degrees, a
    (plan, view class) already tuned is applied from the cache."""
    space = space or CANDIDATES
    cls = view_class(degrees) if cache is not None and degrees is not None else None
    report = []
    engine.set_profiling(True)
    engine.set_option("root_stride", stride)
    try:
        for i in range(n_plans):
            if cls is not None and plans is not None:
                hit = cache.get(plans[i], cls)
                if hit is not None:
                    for k, v in hit.items():
                        engine.set_option(k, v, plan=i)
                    report.append({"plan": i, "best": hit, "ms": {}, "cached": True})
                    continue
            engine.set_option("only_plan", i)
            timings = {}
            best, best_ms = None, float("inf")
            for cfg in _settings(space):
                for k, v in cfg.items():
                    engine.set_option(k, v, plan=i)
                t = time.perf_counter()
                engine.match()
                wall = (time.perf_counter() - t) * 1e3
                s = engine.stats(i)
                ms = sum(s.op_ms[j] for j in range(len(s.op_ms))) or wall
                key = ",".join(f"{k}={v}" for k, v in cfg.items())
                timings[key] = ms
                if ms < best_ms:
                    best, best_ms = cfg, ms
            for k, v in best.items():
                engine.set_option(k, v, plan=i)
            if cls is not None and plans is not None:
                cache.put(plans[i], cls, best)
            report.append({"plan": i, "best": best, "ms": timings, "cached": False})
    finally:
        engine.set_option("only_plan", -1)
        engine.set_option("root_stride", 1)
        engine.reset_counts()
    return report
