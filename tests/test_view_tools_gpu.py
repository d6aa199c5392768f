"""The offline view-bin chain on the GPU against the reference's own tools.

tests/golden/ref_view_tools.npz holds what the reference's features -h 1,
kmeans -init 1 -t 1 and view_packing -s 1 (compiled from its sources into
oracle/_ref by oracle/Makefile; tests/golden/make_view_tools_golden.py) wrote for
two seeded graphs.  The device versions must give the same graph, the same
cluster of every vertex and the same .vbmap and bin sizes, bit for bit
(src/tools/features.cc:177-201, src/tools/kmeans.cc:54-510,
src/tools/view_packing.cc:141-324).
"""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "ref_view_tools.npz")
REF_TOOLS = os.path.join(os.path.dirname(HERE), "oracle", "_ref")
NAMES = ["rmat", "chunglu"]


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def _graph(vs, z, name, suffix=""):
    return vs.Graph(z[f"{name}{suffix}_rp"], z[f"{name}{suffix}_ci"])


@pytest.mark.parametrize("name", NAMES)
def test_features_1hop_equals_reference(vs, gold, name):
    h = vs.features_1hop(_graph(vs, gold, name))
    np.testing.assert_array_equal(h.row_ptrs, gold[f"{name}_1hop_rp"])
    np.testing.assert_array_equal(h.cols, gold[f"{name}_1hop_ci"])


@pytest.mark.parametrize("name", NAMES)
def test_kmeans_equals_reference(vs, gold, name):
    h = _graph(vs, gold, name, "_1hop")
    for c, (k, iters, rc) in enumerate(gold["kmeans_cases"]):
        got, sizes = vs.kmeans(h, int(k), int(iters), starts=vs.reference_rand_starts(int(k), 1), reorder=bool(rc))
        want = gold[f"{name}_kmeans_{c}"]
        np.testing.assert_array_equal(got, want, err_msg=f"case {c}")
        np.testing.assert_array_equal(sizes, np.bincount(want))


@pytest.mark.parametrize("name", NAMES)
def test_view_packing_equals_reference(vs, gold, name):
    g = _graph(vs, gold, name)
    part = gold[f"{name}_kmeans_0"]
    cases = gold["pack_cases"]
    ran = 0
    for c in gold[f"{name}_pack_cases"]:
        hop, threads, opt, _ = (int(x) if i < 3 else x for i, x in enumerate(cases[c]))
        if opt:
            continue  # degree-sorted orders are built by the view_tools driver (test below)
        order, offs = vs.packing_order(part, "1x4" if threads == 1 else "4", threads)
        bins, nb, sizes = vs.view_packing(g, order, offs, hop, float(gold[f"{name}_pack_{c}_mem"][0]))
        assert nb == int(gold[f"{name}_pack_{c}_nbins"][0]), c
        np.testing.assert_array_equal(bins, gold[f"{name}_pack_{c}_vbmap"], err_msg=f"case {c}")
        np.testing.assert_array_equal(sizes, gold[f"{name}_pack_{c}_sizes"], err_msg=f"case {c}")
        ran += 1
    assert ran >= 5


def test_view_packing_rejects_a_ball_above_the_bin_size(vs, gold):
    g = _graph(vs, gold, "rmat")
    order, offs = vs.packing_order(gold["rmat_kmeans_0"], "1x4", 1)
    cap_gb = int(np.diff(g.row_ptrs).max()) * 4 / 1e9  # the largest closed neighbourhood is bigger than any single row
    with pytest.raises(vs.capi.VsgmError, match="alone exceeds"):
        vs.view_packing(g, order, offs, 2, cap_gb)


def test_view_tools_driver_writes_the_reference_files(vs, gold, tmp_path):
    """The drop-in driver with the reference tools' flags: features, kmeans -t 1
    -init 1, view_packing (-o 0 and the degree-sorted -o 1) write the files the
    reference tools write, with the same content."""
    from vsgm_b200 import build
    name = "chunglu"
    g = _graph(vs, gold, name)
    vs.write_csr_bin(tmp_path / "g.bin", g)
    tool = build.VIEW_TOOLS

    def run(*args):
        r = subprocess.run([tool, *args], cwd=tmp_path, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        return r.stdout

    run("features", "-f", "g.bin", "-h", "1")
    h = vs.read_csr_bin(tmp_path / "g.bin.1hop.bin")
    np.testing.assert_array_equal(h.cols, gold[f"{name}_1hop_ci"])
    run("kmeans", "-f", "g.bin.1hop.bin", "-k", "4", "-i", "10", "-t", "1", "-init", "1", "-rc", "0")
    km = np.loadtxt(tmp_path / "g.bin.1hop.bin.kmeans.4", dtype=np.int32)
    np.testing.assert_array_equal(km, gold[f"{name}_kmeans_0"])
    shutil.copy(tmp_path / "g.bin.1hop.bin.kmeans.4", tmp_path / "g.bin.kmeans.1x4")
    shutil.copy(tmp_path / "g.bin.1hop.bin.kmeans.4", tmp_path / "g.bin.kmeans.4")
    cases = gold["pack_cases"]
    for c in gold[f"{name}_pack_cases"]:
        hop, threads, opt = (int(x) for x in cases[c][:3])
        pf = "g.bin.kmeans.1x4" if threads == 1 else "g.bin.kmeans.4"
        run("view_packing", "-gf", "g.bin", "-pf", pf, "-h", str(hop), "-m", repr(float(gold[f"{name}_pack_{c}_mem"][0])), "-t", str(threads),
            "-s", "1", "-o", str(opt))
        bins, nb = vs.read_vbmap(tmp_path / f"g.bin.{hop}.hop.vbmap", g.V)
        assert nb == int(gold[f"{name}_pack_{c}_nbins"][0]), c
        np.testing.assert_array_equal(bins, gold[f"{name}_pack_{c}_vbmap"], err_msg=f"case {c}")
        stat = open(tmp_path / f"g.bin.{hop}.hop.vbstat").read()
        np.testing.assert_array_equal(np.array([int(x) for x in re.findall(r"total size: (\d+)", stat)], np.uint64),
                                      gold[f"{name}_pack_{c}_sizes"])


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_TOOLS, "kmeans")), reason="the reference's view tools are not built")
def test_chain_equals_reference_tools_on_rmat16(vs, tmp_path):
    """A larger graph than the fixtures (R-MAT 16, ef 16): the reference tools built
    in oracle/_ref run beside the device chain on the same files."""
    g = vs.gen_rmat(16, 16, seed=1)
    vs.write_csr_bin(tmp_path / "g.bin", g)

    def ref(tool, *args):
        r = subprocess.run([os.path.join(REF_TOOLS, tool), *args], cwd=tmp_path, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr

    ref("features", "-f", "g.bin", "-h", "1", "-t", "1")
    h = vs.features_1hop(g)
    hr = vs.read_csr_bin(tmp_path / "g.bin.1hop.bin")
    np.testing.assert_array_equal(h.cols, hr.cols)
    ref("kmeans", "-f", "g.bin.1hop.bin", "-k", "4", "-i", "5", "-t", "1", "-init", "1")
    want = np.loadtxt(tmp_path / "g.bin.1hop.bin.kmeans.4", dtype=np.int32)
    got, _ = vs.kmeans(h, 4, 5)
    np.testing.assert_array_equal(got, want)
    shutil.copy(tmp_path / "g.bin.1hop.bin.kmeans.4", tmp_path / "g.bin.kmeans.1x4")
    for hop, frac in ((2, 0.02), (3, 0.6)):
        mem = frac * g.E * 4 / 1e9
        r = subprocess.run([os.path.join(REF_TOOLS, "view_packing"), "-gf", "g.bin", "-pf", "g.bin.kmeans.1x4", "-h", str(hop), "-m", repr(mem),
                            "-t", "1", "-s", "1"], cwd=tmp_path, capture_output=True, text=True, timeout=600)
        order, offs = vs.packing_order(want, "1x4", 1)
        if r.returncode != 0:  # the reference lost a source whose ball exceeds the budget
            with pytest.raises(vs.capi.VsgmError, match="alone exceeds"):
                vs.view_packing(g, order, offs, hop, mem)
            continue
        wb, wn = vs.read_vbmap(tmp_path / f"g.bin.{hop}.hop.vbmap", g.V)
        bins, nb, _ = vs.view_packing(g, order, offs, hop, mem)
        assert nb == wn
        np.testing.assert_array_equal(bins, wb)
