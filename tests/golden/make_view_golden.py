"""Regenerate tests/golden/ref_views.npz from the reference's own CPU stages.

Runs oracle/_ref/ref_cpu_stages (built by `make -C oracle ref` from the reference
sources: GraphIO::ReadCSRBinFile, ViewBinManager::LoadViewBinPartition and
ViewBin::Materialize) on a small seeded R-MAT graph written in the .bin layout by
this project's writer, with a 3-bin .vbmap, for several (hop, root_degree)
settings, and stores the graph, the bins, the reference reader's (V, E, sum of
cols) and every materialised view.

    python tests/golden/make_view_golden.py
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.join(HERE, "..", "..")
STAGES = os.path.join(ROOT, "oracle", "_ref", "ref_cpu_stages")
CASES = [(2, 0), (3, 0), (2, 4), (3, 6), (1, 0)]


def main():
    sys.path.insert(0, ROOT)
    import vsgm_b200 as vs
    g = vs.gen_rmat(8, 6, seed=9)
    bins = (np.arange(g.V) * 5 % 3).astype(np.int32)
    out = {"row_ptrs": g.row_ptrs, "cols": g.cols, "bins": bins, "cases": np.array(CASES, np.int64)}
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "g.bin")
        vs.write_csr_bin(path, g)
        vs.write_vbmap(path + ".vbmap", bins, 3)
        r = subprocess.run([STAGES, "read", path], capture_output=True, text=True, check=True)
        _, V, E, s, _ = r.stdout.split("\n")[-2].split()
        out["read"] = np.array([int(V), int(E), int(s)], np.uint64)
        for c, (hop, rd) in enumerate(CASES):
            subprocess.run([STAGES, "views", path, path + ".vbmap", str(hop), str(rd), "1", d], capture_output=True, text=True, check=True)
            for b in range(3):
                raw = open(os.path.join(d, f"view_{b}.bin"), "rb").read()
                V, n = (int(x) for x in np.frombuffer(raw[:16], np.uint64))
                out[f"rp_{c}_{b}"] = np.frombuffer(raw[16:16 + 8 * (V + 1)], np.uint64).copy()
                out[f"ci_{c}_{b}"] = np.frombuffer(raw[16 + 8 * (V + 1):], np.uint32).copy()
    np.savez_compressed(os.path.join(HERE, "ref_views.npz"), **out)
    print("wrote", os.path.join(HERE, "ref_views.npz"), "graph", g.V, g.E)


if __name__ == "__main__":
    main()
