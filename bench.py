"""Benchmark: exact subgraph counting on one B200 (matches/s), pm_pipeline workload.

Workload (N=1): synthetic R-MAT scale 22 (4.19M vertices), edge factor 16,
a/b/c/d = 0.57/0.19/0.19/0.05, seed 2, self-loops and duplicates removed,
symmetrised, uint32 CSR with sorted rows; queries: 4-clique (-kc 4), 4-cycle
(-p 1) and diamond (-p 2), planned by the reference heuristic; one view holding
every source (what view_packing produces for this graph under a 40 GB budget).
A step is one match of all three queries over the resident view.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--scale S] [--queries kc4,p1,p2] [--option knob=value ...]

(--scale / --queries / --option / --hbm-gb select smaller or single-query cases
for profiling; the default is the workload above.)

value   = sum of the exact counts / device time per step (inputs resident in HBM)
e2e     = the same through the C ABI from pinned host buffers: the graph in the
          generator's ids uploaded, relabelled by degree on the device, matched,
          counts read back - all inside the timed region
roofline: dominant kernel (COMPUTE_COUNT) algorithmic bytes / its device time
cpu_baseline / --impl reference: the CPU restatement of the reference executor
          (oracle/) on a time-boxed random sample of roots, all host cores (the
          reference arm builds its graph and plans without the product library);
          cpu_baseline.view_stages: the reference's own .bin reader and view
          materialisation (compiled from its sources) beside ours, on host and device.
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = {"workload": "rmat22_ef16_seed2_kc4_p1_p2", "graph": "R-MAT scale 22, edge factor 16, a/b/c=0.57/0.19/0.19, seed 2",
            "queries": ["-kc 4", "-p 1", "-p 2"], "views": 1,
            "relabel": "degree-ascending ids (exact counts are invariant to relabelling)"}


# DRAM bytes per step of the dominant op, from one ncu capture of the same bench
# command (the launch list of one step kept under profiles/: cold-cache
# dram__bytes_read.sum + dram__bytes_write.sum of the 4-cycle operator's kernels,
# its heavy-root groups scaled from the 288 captured to all 5,940).  Only for the
# workload it was taken on.
MEASURED_TRAFFIC = {("rmat22_ef16_seed2_kc4_p1_p2", "-p 1"): 3.5e11}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def parse_queries(text):
    """"kc4,p1,p2" -> reference flags ["-kc 4", "-p 1", "-p 2"]."""
    flags = []
    for q in text.split(","):
        q = q.strip()
        if q.startswith("kc"):
            flags.append(f"-kc {int(q[2:])}")
        elif q.startswith("p"):
            flags.append(f"-p {int(q[1:])}")
        else:
            raise SystemExit(f"unknown query {q!r} (kcK or pN)")
    return flags


def plan_of(vs, flag):
    kind, k = flag.split()
    return vs.plan_clique(int(k)) if kind == "-kc" else vs.plan_pattern(int(k))


def make_workload(vs, scale=22, edge_factor=16, seed=2, relabel="asc", queries=None):
    """(relabelled graph, plans, graph in the generator's ids)."""
    t = time.time()
    raw = vs.gen_rmat(scale, edge_factor, 0.57, 0.19, 0.19, seed=seed)
    g = raw
    if relabel != "none":
        g, _ = vs.degree_relabel(raw, ascending=(relabel == "asc"))
    plans = [plan_of(vs, f) for f in (queries or WORKLOAD["queries"])]
    log(f"graph V={g.V} E={g.E} generated+relabelled in {time.time() - t:.1f}s; plans:", [p.describe() for p in plans])
    return g, plans, raw


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, path, device=0):
        self.path = path
        self.device = device
        self.p = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200", "-i", str(self.device)],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            self.p.wait()
            self.f.close()

    def summary(self):
        try:
            rows = [l.split(",") for l in open(self.path).read().strip().splitlines() if l.strip()]
        except Exception:
            return None
        if not rows:
            return None
        sm = sorted(float(r[1]) for r in rows)
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for n, v in zip(names, r[5:9]):
                if v.strip() == "Active":
                    reasons.add(n)
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": float(rows[0][2]), "reasons": sorted(reasons), "samples": len(rows)}


def cpu_sample_rate(g, plans, seconds, threads):
    """Time-boxed oracle run: random roots in chunks until `seconds` elapse."""
    import oracle
    rng = np.random.default_rng(12345)
    roots = rng.permutation(g.V).astype(np.uint32)
    per_plan = seconds / len(plans)
    total_count, total_time, roots_done = 0, 0.0, 0
    chunk = 8
    for p in plans:
        t_plan, i = 0.0, 0
        while t_plan < per_plan and i < len(roots):
            src = np.sort(roots[i:i + chunk])
            t = time.perf_counter()
            c = oracle.count(p, g, src, threads=threads)
            dt = time.perf_counter() - t
            total_count += c
            t_plan += dt
            i += chunk
            roots_done += len(src)
            chunk = min(chunk * 2, 1 << 16) if dt < 0.5 else max(chunk // 2, 1)
        total_time += t_plan
    return total_count / total_time, total_count, total_time, roots_done


def view_stage_times(vs, eng, g, threads):
    """The view-producing stages beside the match: the reference's own .bin reader
    and ViewBin::Materialize (compiled from its sources into oracle/_ref, when that
    build exists), against this library's bulk reader, host halo build and device
    halo build, on the workload graph as one 2-hop view bin.  Milliseconds."""
    import tempfile
    out = {"view": "1 bin holding every source, hop 2"}
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "g.bin")
        vs.write_csr_bin(path, g)
        vs.write_vbmap(path + ".2.hop.vbmap", np.zeros(g.V, np.int32), 1)
        t = time.perf_counter()
        h = vs.read_csr_bin(path)
        out["read_bin_ms"] = (time.perf_counter() - t) * 1e3
        src = np.arange(g.V, dtype=np.uint32)
        t = time.perf_counter()
        vs.materialize_view(h, src, 2, 0, threads)
        out["materialize_host_ms"] = (time.perf_counter() - t) * 1e3
        import torch
        eng.set_option("relabel", 0)  # the file's ids, as the reference builds its halos
        eng.upload_graph(h)
        eng.materialize_view(src, 2)  # warm-up
        torch.cuda.synchronize()
        t = time.perf_counter()
        eng.materialize_view(src, 2)
        out["materialize_device_ms"] = (time.perf_counter() - t) * 1e3
        stages = os.path.join(ROOT, "oracle", "_ref", "ref_cpu_stages")
        if os.path.exists(stages):
            r = subprocess.run([stages, "read", path], capture_output=True, text=True, timeout=600)
            out["reference_read_bin_ms"] = float(r.stdout.strip().splitlines()[-1].split()[-1])
            r = subprocess.run([stages, "views", path, path + ".2.hop.vbmap", "2", "0", str(threads)], capture_output=True, text=True, timeout=600)
            out["reference_materialize_ms"] = float(r.stdout.strip().splitlines()[-1].split()[-1])
            out["reference"] = "GraphIO::ReadCSRBinFile, ViewBin::Materialize compiled from the reference sources"
    return out


def bench_config(args, world):
    """The config dict both arms print (the driver compares them)."""
    return dict(WORKLOAD, scale=args.scale, l2="inputs larger than L2 (cols 0.5 GB)", parallelism=f"roots strided over {world} GPU(s)")


def run_reference(args):
    """The reference arm: the CPU restatement of the reference executor (oracle/) on
    all host cores, over the same graph (built by the oracle's restatement of the
    generator) and the reference planner's own plans (its dump in tests/golden), on
    a time-boxed random root sample per step.  Nothing of the product is loaded."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle
    if args.relabel == "desc":
        raise SystemExit("the reference arm restates ascending or no relabelling only")
    t = time.time()
    g = oracle.gen_rmat(args.scale, 16, 0.57, 0.19, 0.19, seed=2)
    if args.relabel == "asc":
        g = oracle.degree_relabel(g)
    plans = [oracle.golden_plan(f.replace("-", "").replace(" ", "")) for f in args.query_flags]
    log(f"reference arm: graph V={g.V} E={len(g.cols)} built in {time.time() - t:.1f}s from the oracle's generator; plans from the reference planner's dump")
    threads = os.cpu_count() or 1
    per_step = []
    for s in range(args.warmup + args.steps):
        rate, cnt, secs, nroots = cpu_sample_rate(g, plans, args.ref_seconds, threads)
        if s >= args.warmup:
            per_step.append((rate, cnt, secs, nroots))
    rate = float(np.mean([r[0] for r in per_step]))
    secs = float(np.mean([r[2] for r in per_step]))
    sample = (f"{per_step[-1][3]} random roots of {g.V} per step (time-boxed {args.ref_seconds}s, summed over the {len(plans)} queries); "
              f"matches/s = sampled matches / sampled seconds")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    out = {"impl": "reference", "metric": "matches/s", "value": rate, "unit": "matches/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": secs * 1e3, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
           "dtype": "u32", "data": "synthetic", "config": bench_config(args, world),
           "cpu_baseline": {"value": rate, "unit": "matches/s", "cores": threads, "kind": "port", "sample": sample},
           "e2e": {"value": rate, "unit": "matches/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--ref-seconds", type=float, default=20.0)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--scale", type=int, default=22)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--relabel", default="asc", choices=["asc", "desc", "none"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--queries", default="kc4,p1,p2", help="comma list of kcK / pN (default: the workload's three)")
    ap.add_argument("--option", action="append", default=[], help="engine knob name=value (vsgm_set_option), repeatable")
    ap.add_argument("--no-stages", action="store_true", help="skip the view-stage timings of the CPU leg")
    ap.add_argument("--no-profile", action="store_true", help="skip the profiled pass (roofline fields become null); for launch lists")
    ap.add_argument("--hbm-gb", type=float, default=0.0,
                    help="engine working budget in GB (0: 90%% of free HBM); profiler captures use a few GB")
    args = ap.parse_args()
    args.query_flags = parse_queries(args.queries)
    if args.query_flags != WORKLOAD["queries"] or args.scale != 22:
        WORKLOAD["workload"] = f"rmat{args.scale}_ef16_seed2_" + "_".join(q.strip() for q in args.queries.split(","))
        WORKLOAD["queries"] = args.query_flags
        WORKLOAD["graph"] = WORKLOAD["graph"].replace("scale 22", f"scale {args.scale}")
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import vsgm_b200 as vs

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    g, plans, raw = make_workload(vs, scale=args.scale, relabel=args.relabel, queries=args.query_flags)
    # roots of this rank: a strided share of the vertices (one view per rank)
    from vsgm_b200.shard import allreduce_counts, roots_of_rank
    roots = roots_of_rank(g.V, rank, world)
    eng = vs.Engine(g.V, plans, device=local, hbm_budget_bytes=int(args.hbm_gb * 1e9))
    stream = torch.cuda.ExternalStream(eng.stream(), device=local)
    for kv in args.option:
        name, val = kv.split("=")
        eng.set_option(name, int(val))

    # ---------------- device-resident timing (value): production kernels, no
    # profiling events or byte accounting inside the timed region
    eng.transfer_view(g, roots)
    eng.set_profiling(False)
    for _ in range(args.warmup):
        eng.match()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    eng.reset_counts()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    import tempfile
    with Clocks(os.path.join(tempfile.gettempdir(), f"vsgm_bench_clocks_{os.getpid()}.csv"), device=local) as ck:
        ev0.record(stream)
        for _ in range(args.steps):
            eng.match()
            launches += sum(eng.stats(pi).op_launches[i] for pi, p in enumerate(plans) for i in range(p.n_ops))
        ev1.record(stream)
        torch.cuda.synchronize()
    clocks = ck.summary()
    step_ms = ev0.elapsed_time(ev1) / args.steps
    counts = [c // args.steps for c in eng.counts()]

    # ---------------- one profiled pass (outside the timed region): per-op device
    # time on the engine's stream and the algorithmic bytes for the roofline
    op_ms, op_bytes = {(0, 0): 0.0}, {}
    if not args.no_profile:
        eng.set_profiling(True)
        eng.reset_counts()
        eng.match()
        eng.set_profiling(False)
        if eng.counts() != counts and world == 1:
            raise SystemExit(f"profiled pass counted {eng.counts()} against {counts}")
        for pi, p in enumerate(plans):
            s = eng.stats(pi)
            for i in range(p.n_ops):
                op_ms[(pi, i)] = s.op_ms[i]
                op_bytes[(pi, i)] = s.op_bytes[i]
    if world > 1:
        t = torch.tensor([step_ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        step_ms = float(t.item())
        counts = allreduce_counts(counts, device="cuda")
    matches = sum(counts)
    value = matches / (step_ms / 1e3)

    # dominant kernel: the op with the largest device time
    (dom_plan, dom_op), dom_ms = max(op_ms.items(), key=lambda kv: kv[1])
    dom_bytes = op_bytes.get((dom_plan, dom_op), 0)
    peak, peak_kind = load_peaks()
    achieved = (dom_bytes / (dom_ms / 1e3)) / 1e9 if dom_ms > 0 and dom_bytes > 0 else None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
                "traffic": MEASURED_TRAFFIC.get((WORKLOAD["workload"], WORKLOAD["queries"][dom_plan])) if world == 1 else None,
                "traffic_source": "ncu launch list of one step (profiles/), bytes per step of the op",
                "kernel": f"plan {dom_plan} op {dom_op} ({vs.capi.OP_NAMES[plans[dom_plan].op_type[dom_op]]})",
                "kernel_ms_per_step": dom_ms, "peak_kind": peak_kind, "timed_in": "one profiled pass after the timed steps"}
    per_query = []
    for pi, p in enumerate(plans):
        ms = sum(v for (a, _), v in op_ms.items() if a == pi)
        per_query.append({"query": WORKLOAD["queries"][pi], "count": counts[pi], "device_ms": ms})

    # ---------------- end to end through the C ABI from pinned host buffers: the
    # graph in the generator's ids goes up, is relabelled by degree on the device
    # (option "relabel", vsgm_upload_graph), every source of this rank (caller ids)
    # becomes the view's roots (vsgm_graph_view), then match and count read-back
    eng.set_profiling(False)
    h_rp = torch.from_numpy(raw.row_ptrs.view(np.int64)).pin_memory()
    h_ci = torch.from_numpy(raw.cols.view(np.int32)).pin_memory()
    h_src = torch.from_numpy(roots.view(np.int32)).pin_memory()
    L = vs.capi.lib()
    import ctypes as C
    eng.set_option("relabel", 0 if args.relabel == "none" else 1)
    if args.relabel == "desc":
        raise SystemExit("the end-to-end pass relabels ascending only")
    e2e_ms, e2e_counts = [], counts
    for s in range(1 + args.e2e_steps if args.e2e_steps > 0 else 0):
        eng.reset_counts()
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        vs.capi.check(L.vsgm_upload_graph(eng.h, C.cast(h_rp.data_ptr(), C.POINTER(C.c_uint64)), C.cast(h_ci.data_ptr(), C.POINTER(C.c_uint32)),
                                          raw.E), eng.h)
        vs.capi.check(L.vsgm_graph_view(eng.h, C.cast(h_src.data_ptr(), C.POINTER(C.c_uint32)), len(roots)), eng.h)
        eng.match()
        e2e_counts = eng.counts()
        t1.record(stream)
        torch.cuda.synchronize()
        if s >= 1:  # the first pass is a warm-up
            e2e_ms.append(t0.elapsed_time(t1))
    if world == 1 and e2e_counts != counts:
        raise SystemExit(f"end-to-end pass counted {e2e_counts} against {counts}")
    e2e_step = float(np.mean(e2e_ms)) if e2e_ms else float("nan")
    if world > 1:
        t = torch.tensor([e2e_step], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_step = float(t.item())
    e2e = {"value": matches / (e2e_step / 1e3), "unit": "matches/s", "h2d_bytes_per_step": int(8 * (g.V + 1) + 4 * g.E + 4 * len(roots)),
           "d2h_bytes_per_step": 8 * len(plans), "ms_per_step": e2e_step, "steps": args.e2e_steps, "warmup": 1,
           "scope": "generator-id graph from pinned host memory -> device relabel by degree -> all sources -> match -> counts to host"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        rate, cnt, secs, nroots = cpu_sample_rate(g, plans, args.cpu_seconds, threads)
        cpu = {"value": rate, "unit": "matches/s", "cores": threads, "kind": "port",
               "sample": f"{nroots} random roots (time-boxed {args.cpu_seconds}s over the {len(plans)} queries), matches/s = sampled matches / seconds"}
        if not args.no_stages:
            try:
                cpu["view_stages"] = view_stage_times(vs, eng, g, threads)
            except Exception as ex:  # the stages are a side measurement; the line still prints
                cpu["view_stages"] = {"error": str(ex)}

    if rank == 0:
        out = {"metric": "matches/s", "value": value, "unit": "matches/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
               "ms_per_step": step_ms, "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "u32",
               "data": "synthetic", "config": bench_config(args, world),
               "counts": counts, "per_query": per_query, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
               "gpu_launches": int(launches), "clocks": clocks}
        print(json.dumps(out), flush=True)
    eng.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
