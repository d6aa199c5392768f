"""Regenerate tests/golden/ref_view_tools.npz from the reference's offline view tools.

Runs oracle/_ref/{features,kmeans,view_packing} (built by `make -C oracle ref` from
the reference sources, as its tools Makefile builds them) on two small seeded
graphs written in the .bin layout by this project's writer, and stores the
graphs and the tools' outputs:

  features -h 1                        the self-loop graph (row_ptrs, cols)
  kmeans -k K -i I -t 1 -init 1 -rc R  the cluster of every vertex (K, I, R per case)
  view_packing -t T -s 1 -h H -m M     the .vbmap and the .vbstat sizes, over the
                                       -k 4 partition as 1x4 (T = 1) and as 4 (T = 4)

Budgets M are a fraction of the graph's row entries, raised to just above the
largest single ball where that is bigger (below it the reference packer loses the
source and stops on its own assertion).

    python tests/golden/make_view_tools_golden.py
"""
import os
import re
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.join(HERE, "..", "..")
REF = os.path.join(ROOT, "oracle", "_ref")
KMEANS_CASES = [(4, 10, 0), (4, 10, 1), (7, 6, 0), (3, 0, 0)]  # (K, iterations, -rc)
# (hop, threads, -o, row entries per bin as a fraction of the graph's)
PACK_CASES = [(2, 1, 0, 0.12), (2, 1, 0, 1.5), (1, 1, 0, 0.05), (3, 1, 0, 0.2), (2, 4, 0, 0.08), (2, 1, 1, 0.12), (3, 4, 0, 0.2), (2, 4, 1, 0.3)]


def max_ball(g, hop):
    """Row entries of the largest (hop-1)-ball of one source: a budget below it makes
    the reference packer lose that source and stop on its vertex-count assertion."""
    deg = np.diff(g.row_ptrs).astype(np.int64)
    best = 0
    for s in range(g.V):
        ball = {s}
        frontier = [s]
        for _ in range(hop - 1):
            nxt = []
            for x in frontier:
                for y in g.cols[g.row_ptrs[x]:g.row_ptrs[x + 1]]:
                    if int(y) not in ball:
                        ball.add(int(y))
                        nxt.append(int(y))
            frontier = nxt
        best = max(best, int(deg[list(ball)].sum()))
    return best


def run(args, cwd):
    return subprocess.run(args, cwd=cwd, capture_output=True, text=True, timeout=600)


def main():
    sys.path.insert(0, ROOT)
    import vsgm_b200 as vs
    graphs = {"rmat": vs.gen_rmat(11, 8, seed=5), "chunglu": vs.gen_chung_lu(3000, 18000, 2.3, 250, seed=7)}
    out = {}
    for name, g in graphs.items():
        out[f"{name}_rp"], out[f"{name}_ci"] = g.row_ptrs, g.cols
        with tempfile.TemporaryDirectory() as d:
            vs.write_csr_bin(os.path.join(d, "g.bin"), g)
            r = run([os.path.join(REF, "features"), "-f", "g.bin", "-h", "1", "-t", "1"], d)
            assert r.returncode == 0, r.stderr
            h = vs.read_csr_bin(os.path.join(d, "g.bin.1hop.bin"))
            out[f"{name}_1hop_rp"], out[f"{name}_1hop_ci"] = h.row_ptrs, h.cols
            for c, (k, iters, rc) in enumerate(KMEANS_CASES):
                r = run([os.path.join(REF, "kmeans"), "-f", "g.bin.1hop.bin", "-k", str(k), "-i", str(iters), "-t", "1", "-init", "1",
                         "-rc", str(rc), "-o", f"g.km{c}."], d)
                assert r.returncode == 0, r.stderr
                out[f"{name}_kmeans_{c}"] = np.loadtxt(os.path.join(d, f"g.km{c}.{k}"), dtype=np.int32)
            # the -k 4 partition (case 0) drives the packer, as "1x4" and as "4"
            shutil.copy(os.path.join(d, "g.km0.4"), os.path.join(d, "g.bin.kmeans.1x4"))
            shutil.copy(os.path.join(d, "g.km0.4"), os.path.join(d, "g.bin.kmeans.4"))
            kept = []
            balls = {h: max_ball(g, h) for h in (1, 2, 3)}
            for c, (hop, threads, opt, frac) in enumerate(PACK_CASES):
                mem = max(frac * g.E, 1.02 * balls[hop]) * 4 / 1e9
                pf = "g.bin.kmeans.1x4" if threads == 1 else "g.bin.kmeans.4"
                r = run([os.path.join(REF, "view_packing"), "-gf", "g.bin", "-pf", pf, "-h", str(hop), "-m", repr(mem), "-t", str(threads),
                         "-s", "1", "-o", str(opt), "-d", "1"], d)
                if r.returncode != 0:
                    print(f"{name} packing case {c} left out: the reference packer stopped ({r.stderr.strip()[-120:]})")
                    continue
                lines = open(os.path.join(d, f"g.bin.{hop}.hop.vbmap")).read().split()
                out[f"{name}_pack_{c}_nbins"] = np.array([int(lines[0])], np.int32)
                out[f"{name}_pack_{c}_vbmap"] = np.array(lines[1:], np.int32)
                stat = open(os.path.join(d, f"g.bin.{hop}.hop.vbstat")).read()
                out[f"{name}_pack_{c}_sizes"] = np.array([int(x) for x in re.findall(r"total size: (\d+)", stat)], np.uint64)
                out[f"{name}_pack_{c}_mem"] = np.array([mem], np.float64)
                kept.append(c)
                os.remove(os.path.join(d, "g.bin.degrees.bin"))
            out[f"{name}_pack_cases"] = np.array(kept, np.int32)
            print(name, "V", g.V, "E", g.E, "packing cases", kept, "bins", [int(out[f"{name}_pack_{c}_nbins"][0]) for c in kept])
    out["kmeans_cases"] = np.array(KMEANS_CASES, np.int64)
    out["pack_cases"] = np.array(PACK_CASES, np.float64)
    np.savez_compressed(os.path.join(HERE, "ref_view_tools.npz"), **out)
    print("wrote", os.path.join(HERE, "ref_view_tools.npz"))


if __name__ == "__main__":
    main()
