"""Learned matching-order planner.

The reference picks one search sequence per pattern with a fixed heuristic
(Plan::GenerateSearchSequence, src/query/plan.h:210-265).  Here a small MLP
predicts, for a (pattern, view) pair, the log intermediate-result size of every
candidate search sequence, and the planner runs the predicted cheapest one.  The
network only chooses the plan: every order of a pattern yields the same exact
count.  choose() trusts the prediction beyond a confidence margin;
choose_verified() (the planner's default) lets the network propose a few orders
and keeps the heuristic one unless a sampled run of the proposals beats it.

Features (76 values):
  36  pattern adjacency bits (6 x 6, after the query's vertex re-mapping)
  32  log2-degree histogram of the view (fractions of its vertices)
   8  log1p of the partial matches entering ops 1..8 of the heuristic plan on a
      sample of the view's roots (the "sampled per-level candidate counts")
Output: 720 values, one per permutation of 6 pattern vertices (lexicographic
rank); a pattern with n < 6 vertices uses the first n! units.

Training targets come from the engine itself: the persistent batched run
(vsgm_run_batched_ex) executes the heuristic order and several random valid
orders of each pair on the same root sample and reports the partial matches
entering every op; the target is log1p of their sum scaled to the whole view.
"""
import ctypes as C
import itertools
import math

import numpy as np

from . import Engine, capi, plan_reorder

N_IN, N_HIDDEN, N_OUT = 76, 128, 720
MAX_N = 6


def _perms(n):
    return list(itertools.permutations(range(n)))


_RANK = {n: {p: i for i, p in enumerate(_perms(n))} for n in range(1, MAX_N + 1)}


def order_index(seq):
    return _RANK[len(seq)][tuple(seq)]


def valid_orders(plan):
    """Every search sequence whose later vertices each have an earlier neighbour."""
    n = plan.n_vertices
    adj = [plan.adj[i] for i in range(n)]
    out = []
    for perm in _perms(n):
        seen = 1 << perm[0]
        ok = True
        for v in perm[1:]:
            if not adj[v] & seen:
                ok = False
                break
            seen |= 1 << v
        if ok:
            out.append(perm)
    return out


def heuristic_order(plan):
    return tuple(int(plan.seq[i]) for i in range(plan.n_vertices))


def degree_histogram(g):
    d = g.degrees().astype(np.float64)
    b = np.minimum(31, np.floor(np.log2(np.maximum(d, 1))).astype(np.int64) + (d > 0))
    h = np.bincount(b, minlength=32)[:32].astype(np.float32)
    return h / max(1.0, h.sum())


def pattern_bits(plan):
    x = np.zeros(36, np.float32)
    for i in range(plan.n_vertices):
        for j in range(plan.n_vertices):
            if plan.adj[i] >> j & 1:
                x[i * 6 + j] = 1.0
    return x


def features(plan, hist, level_paths):
    lv = np.zeros(8, np.float32)
    for i in range(1, min(9, plan.n_ops)):
        lv[i - 1] = math.log1p(float(level_paths[i]))
    return np.concatenate([pattern_bits(plan), hist, lv / 20.0]).astype(np.float32)


def plan_cost(plan, level_paths, scale):
    """log1p of the partial matches the plan touches, scaled to the whole view."""
    return math.log1p(scale * float(sum(int(level_paths[i]) for i in range(plan.n_ops))))


class Sampler:
    """Evaluates plans (orders) of many patterns over sampled roots of resident views."""

    def __init__(self, views, roots_per_view=512, seed=0, device=0, step_budget=2_000_000):
        self.views = views
        self.hist = [degree_histogram(g) for g in views]
        rng = np.random.default_rng(seed)
        self.samples = [np.sort(rng.choice(g.V, size=min(roots_per_view, g.V), replace=False)).astype(np.uint32) for g in views]
        self.scale = [g.V / len(s) for g, s in zip(views, self.samples)]
        self.device = device
        self.step_budget = step_budget

    def evaluate(self, plans, view_index):
        """(counts, level_paths, overflow) of every plan on one view's root sample."""
        g = self.views[view_index]
        with Engine(g.V, plans, device=self.device) as e:
            vid = e.add_view(g, self.samples[view_index])
            return e.run_batched_ex([vid], step_budget=self.step_budget)


def make_examples(sampler, patterns, pairs, orders_per_pair=8, seed=0):
    """Training rows (features, target vector, mask) for (pattern index, view index) pairs."""
    rng = np.random.default_rng(seed)
    X, Y, M, meta = [], [], [], []
    by_view = {}
    for pi, vi in pairs:
        by_view.setdefault(vi, []).append(pi)
    for vi, pis in by_view.items():
        plans, owners = [], []
        for pi in pis:
            base = patterns[pi]
            orders = valid_orders(base)
            h = heuristic_order(base)
            pick = [h] + [orders[k] for k in rng.permutation(len(orders))[:orders_per_pair] if orders[k] != h]
            for o in pick[:orders_per_pair]:
                plans.append(plan_reorder(base, o))
                owners.append((pi, o))
        cnt, lvl, ovf = sampler.evaluate(plans, vi)
        rows = {}
        for k, (pi, o) in enumerate(owners):
            rows.setdefault(pi, []).append((o, plans[k], lvl[k][0], bool(ovf[k][0])))
        for pi, items in rows.items():
            hplan = items[0][1]
            x = features(hplan, sampler.hist[vi], items[0][2])
            y = np.zeros(N_OUT, np.float32)
            m = np.zeros(N_OUT, np.float32)
            for o, p, lp, over in items:
                cost = plan_cost(p, lp, sampler.scale[vi])
                if over:  # stopped by the step budget: a lower bound, still a ranking signal
                    cost += 1.0
                y[order_index(o)] = cost
                m[order_index(o)] = 1.0
            X.append(x)
            Y.append(y)
            M.append(m)
            meta.append((pi, vi, [(o, plan_cost(p, lp, sampler.scale[vi]), over) for o, p, lp, over in items]))
    return np.array(X), np.array(Y), np.array(M), meta


def plan_error(pred, Y, M):
    """The network judged against measured costs on examples it was not trained on:
    pred / Y / M are predicted log intermediate sizes, measured ones (plan_cost, from
    the plain engine's per-op partial-match counts) and the mask of measured orders,
    one row per (pattern, view) pair.  Returns the mean absolute error in log units
    over every measured (pair, order), the share of pairs whose predicted cheapest
    measured order is the measured cheapest (and what chance gives), and the mean
    Spearman rank correlation over pairs with at least 3 measured orders."""
    errs, top1, chance, rhos = [], 0, 0.0, []
    for p, y, m in zip(pred, Y, M):
        idx = np.nonzero(m > 0)[0]
        if len(idx) == 0:
            continue
        errs.extend(np.abs(p[idx] - y[idx]).tolist())
        top1 += int(idx[np.argmin(p[idx])] == idx[np.argmin(y[idx])])
        chance += 1.0 / len(idx)
        if len(idx) >= 3:
            rp = np.argsort(np.argsort(p[idx])).astype(np.float64)
            ry = np.argsort(np.argsort(y[idx])).astype(np.float64)
            if rp.std() > 0 and ry.std() > 0:
                rhos.append(float(np.corrcoef(rp, ry)[0, 1]))
    n = sum(1 for m in M if (m > 0).any())
    return {"pairs": n, "mae_log": float(np.mean(errs)) if errs else None, "top1": top1 / max(n, 1), "top1_chance": chance / max(n, 1),
            "spearman": float(np.mean(rhos)) if rhos else None}


class LearnedPlanner:
    """The MLP, trained and evaluated by the library's own BF16/FP32 kernels."""

    def __init__(self, device=0, seed=7):
        L = capi.lib()
        h = C.c_void_p()
        capi.check(L.vsgm_mlp_create(device, N_IN, N_HIDDEN, N_OUT, seed, C.byref(h)))
        self.h = h
        self.L = L

    def close(self):
        if self.h:
            self.L.vsgm_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _p(a):
        return np.ascontiguousarray(a, np.float32).ctypes.data_as(C.POINTER(C.c_float))

    def train(self, X, Y, M, epochs=200, batch=256, lr=3e-3, seed=0):
        rng = np.random.default_rng(seed)
        X, Y, M = (np.ascontiguousarray(a, np.float32) for a in (X, Y, M))
        losses = []
        loss = C.c_float()
        for _ in range(epochs):
            idx = rng.permutation(len(X))
            for s in range(0, len(X), batch):
                b = idx[s:s + batch]
                xb, yb, mb = X[b].copy(), Y[b].copy(), M[b].copy()
                capi.check(self.L.vsgm_mlp_train_step(self.h, self._p(xb), self._p(yb), self._p(mb), len(b), lr, C.byref(loss)))
            losses.append(loss.value)
        return losses

    def save(self, path):
        """Write the FP32 master parameters (packed as the C ABI packs them) to a .npy file."""
        n = int(self.L.vsgm_mlp_num_params(self.h))
        w = np.zeros(n, np.float32)
        capi.check(self.L.vsgm_mlp_get_params(self.h, self._p(w)))
        np.save(path, w)

    def load(self, path):
        w = np.ascontiguousarray(np.load(path), np.float32)
        if w.size != int(self.L.vsgm_mlp_num_params(self.h)):
            raise ValueError("parameter file does not match the network's shape")
        capi.check(self.L.vsgm_mlp_set_params(self.h, self._p(w)))

    def predict(self, X):
        X = np.ascontiguousarray(X, np.float32)
        y = np.zeros((len(X), N_OUT), np.float32)
        capi.check(self.L.vsgm_mlp_forward(self.h, self._p(X), len(X), y.ctypes.data_as(C.POINTER(C.c_float))))
        return y

    def propose(self, plan, x, k=4):
        """The k valid orders with the lowest predicted cost (heuristic order excluded)."""
        pred = self.predict(x[None, :])[0]
        h = heuristic_order(plan)
        ranked = sorted((o for o in valid_orders(plan) if o != h), key=lambda o: pred[order_index(o)])
        return ranked[:k]

    def choose_verified(self, plan, sampler, view_index, k=4, margin=0.05):
        """(order, used_model): the network proposes its k cheapest-looking orders, one
        batched run over the view's root sample measures them beside the heuristic
        order, and the measured cheapest wins if it does at least `margin` (relative)
        less work than the heuristic; otherwise the heuristic order is kept.  A wrong
        prediction therefore costs one sampled run, never a slow full run."""
        h = heuristic_order(plan)
        _, lvl0, _ = sampler.evaluate([plan], view_index)
        x = features(plan, sampler.hist[view_index], lvl0[0][0])
        cands = [h] + self.propose(plan, x, k)
        plans = [plan_reorder(plan, o) for o in cands]
        _, lvl, ovf = sampler.evaluate(plans, view_index)
        work = [sum(int(lvl[i][0][j]) for j in range(plans[i].n_ops)) for i in range(len(plans))]
        # an order stopped by the step budget did at least that much work: never prefer it
        work = [w if not ovf[i][0] else float("inf") for i, w in enumerate(work)]
        best = min(range(len(cands)), key=lambda i: work[i])
        if best != 0 and work[best] < (1.0 - margin) * work[0]:
            return cands[best], True
        return h, False

    def choose_verified_many(self, plans, sampler, view_index, k=4, margin=0.05):
        """choose_verified for many patterns on one view with two sampled runs in
        total (features of every heuristic plan, then every pattern's candidates)."""
        hs = [heuristic_order(p) for p in plans]
        _, lvl0, _ = sampler.evaluate(list(plans), view_index)
        X = np.stack([features(p, sampler.hist[view_index], lvl0[i][0]) for i, p in enumerate(plans)])
        pred = self.predict(X)
        cands, owner = [], []
        for i, p in enumerate(plans):
            ranked = sorted((o for o in valid_orders(p) if o != hs[i]), key=lambda o: pred[i][order_index(o)])
            for o in [hs[i]] + ranked[:k]:
                cands.append(plan_reorder(p, o))
                owner.append((i, o))
        _, lvl, ovf = sampler.evaluate(cands, view_index)
        best = {}
        for j, (i, o) in enumerate(owner):
            w = float("inf") if ovf[j][0] else float(sum(int(x) for x in lvl[j][0][:cands[j].n_ops]))
            best.setdefault(i, []).append((w, o))
        out = []
        for i in range(len(plans)):
            h_work = best[i][0][0]
            w, o = min(best[i], key=lambda t: t[0])
            out.append((o, True) if o != hs[i] and w < (1.0 - margin) * h_work else (hs[i], False))
        return out

    def choose_timed_many(self, plans, sampler, view_index, k=4, stride=16, margin=0.1):
        """Like choose_verified_many, but the proposals are judged by time: the
        level-wise engine (the one the heavy pairs run on) times the heuristic order
        and the network's k proposals of every pattern on every stride-th root of the
        view, and the fastest replaces the heuristic order if it saves at least
        `margin` of its time.  Partial-match counts ignore how long the intersected
        lists are; time does not."""
        g = sampler.views[view_index]
        hs = [heuristic_order(p) for p in plans]
        _, lvl0, _ = sampler.evaluate(list(plans), view_index)
        X = np.stack([features(p, sampler.hist[view_index], lvl0[i][0]) for i, p in enumerate(plans)])
        pred = self.predict(X)
        cands, owner = [], []
        for i, p in enumerate(plans):
            ranked = sorted((o for o in valid_orders(p) if o != hs[i]), key=lambda o: pred[i][order_index(o)])
            for o in [hs[i]] + ranked[:k]:
                cands.append(plan_reorder(p, o))
                owner.append((i, o))
        with Engine(g.V, cands, device=sampler.device) as e:
            e.transfer_view(g, np.arange(0, g.V, stride, dtype=np.uint32))
            e.set_profiling(True)
            e.match()
            ms = []
            for j, c in enumerate(cands):
                st = e.stats(j)
                ms.append(sum(st.op_ms[t] for t in range(c.n_ops)))
        best = {}
        for j, (i, o) in enumerate(owner):
            best.setdefault(i, []).append((ms[j], o))
        out = []
        for i in range(len(plans)):
            h_ms = best[i][0][0]
            t, o = min(best[i], key=lambda x: x[0])
            out.append((o, True) if o != hs[i] and t < (1.0 - margin) * h_ms else (hs[i], False))
        return out

    def choose(self, plan, x, margin=0.25):
        """(order, used_model): the predicted cheapest valid order, or the heuristic
        one when it is not predicted to be cheaper by at least `margin` (log units)."""
        pred = self.predict(x[None, :])[0]
        h = heuristic_order(plan)
        best = min(valid_orders(plan), key=lambda o: pred[order_index(o)])
        if pred[order_index(best)] + margin < pred[order_index(h)]:
            return best, True
        return h, False
