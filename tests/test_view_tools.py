"""Host-side pieces of the device view-bin chain and its golden fixture (no GPU).

The fixture (tests/golden/ref_view_tools.npz) is the reference tools' own output;
here it is checked for internal consistency against definitions that need no GPU:
the self-loop graph by numpy, every vertex in exactly one packed bin, each bin's
size within the budget and equal to the row entries of its sources' balls.  The
helpers that rebuild the reference's inputs are checked too: the random start
against glibc's rand() in a fresh process, and the packing order from a
partition file's suffix.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "ref_view_tools.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


@pytest.mark.parametrize("name", ["rmat", "chunglu"])
def test_fixture_self_loop_graph(gold, name):
    rp, ci = gold[f"{name}_rp"], gold[f"{name}_ci"]
    V = len(rp) - 1
    rows = [np.sort(np.append(ci[rp[v]:rp[v + 1]], v)) for v in range(V)]
    np.testing.assert_array_equal(gold[f"{name}_1hop_rp"], np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.uint64))
    np.testing.assert_array_equal(gold[f"{name}_1hop_ci"], np.concatenate(rows).astype(np.uint32))


def _ball(rp, ci, s, radius):
    ball, frontier = {s}, [s]
    for _ in range(radius):
        nxt = []
        for x in frontier:
            for y in ci[rp[x]:rp[x + 1]]:
                if int(y) not in ball:
                    ball.add(int(y))
                    nxt.append(int(y))
        frontier = nxt
    return ball


@pytest.mark.parametrize("name", ["rmat", "chunglu"])
def test_fixture_bins_cover_the_vertices_within_budget(gold, name):
    rp, ci = gold[f"{name}_rp"], gold[f"{name}_ci"]
    V = len(rp) - 1
    deg = np.diff(rp).astype(np.int64)
    cases = gold["pack_cases"]
    for c in gold[f"{name}_pack_cases"][:3]:
        hop = int(cases[c][0])
        bins = gold[f"{name}_pack_{c}_vbmap"]
        nb = int(gold[f"{name}_pack_{c}_nbins"][0])
        cap = int(float(gold[f"{name}_pack_{c}_mem"][0]) * 1000 * 1000 * 1000 / 4)
        assert len(bins) == V and bins.min() == 0 and bins.max() == nb - 1
        sizes = gold[f"{name}_pack_{c}_sizes"]
        assert len(sizes) == nb
        # a merged bin's size is the sum over its packed bins: at least its own
        # sources' union of balls, and each packed bin is within the budget
        for b in range(nb):
            members = np.nonzero(bins == b)[0]
            union = set()
            for s in members:
                union |= _ball(rp, ci, int(s), hop - 1)
            assert deg[list(union)].sum() <= int(sizes[b])
        assert all(int(s) <= cap for s in sizes)


def test_reference_rand_starts_are_glibc_draws(vs):
    code = "import ctypes, ctypes.util; c = ctypes.CDLL(ctypes.util.find_library('c')); print([c.rand() for _ in range(5)])"
    draws = eval(subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True).stdout)
    for k in (2, 3, 4, 7, 64):
        np.testing.assert_array_equal(vs.reference_rand_starts(k, 5), np.array(draws) % k)


def test_packing_order_follows_the_partition_suffix(vs):
    part = np.array([1, 0, 3, 2, 1, 0, 2, 3])
    order, offs = vs.packing_order(part, "1x4", 1)
    np.testing.assert_array_equal(order, [1, 5, 0, 4, 3, 6, 2, 7])
    np.testing.assert_array_equal(offs, [0, 8])
    order, offs = vs.packing_order(part, "4", 4)
    np.testing.assert_array_equal(order, [1, 5, 0, 4, 3, 6, 2, 7])
    np.testing.assert_array_equal(offs, [0, 2, 4, 6, 8])
    order, offs = vs.packing_order(part, "2x2", 2)
    np.testing.assert_array_equal(offs, [0, 4, 8])
    with pytest.raises(ValueError):
        vs.packing_order(part, "4", 1)


def test_view_tools_driver_refuses_unsupported_forms(vs, tmp_path):
    """The drop-in driver stops with exit code 2 and a message, before touching a
    GPU, for the forms it does not build: features beyond -h 1, kmeans -init 0
    (the reference seeds it from the clock) and multi-level -k, view_packing -s > 1."""
    from vsgm_b200 import build
    cases = [["features", "-f", "g.bin", "-h", "2"], ["kmeans", "-f", "g.bin", "-k", "4", "-init", "0"],
             ["kmeans", "-f", "g.bin", "-k", "2^3", "-init", "1"], ["kmeans", "-f", "g.bin", "-k", "4x4", "-init", "1"],
             ["view_packing", "-gf", "g.bin", "-pf", "g.bin.kmeans.4", "-s", "2"], ["no_such_tool"]]
    for args in cases:
        r = subprocess.run([build.VIEW_TOOLS, *args], cwd=tmp_path, capture_output=True, text=True, timeout=60)
        assert r.returncode == 2, (args, r.returncode, r.stderr)
        assert "view_tools" in r.stderr


def test_view_tool_entry_points_reject_bad_arguments(vs):
    """Argument checks run on the host before any device work (no GPU needed): a
    cluster count out of range, a start outside [0, K), an order that is not a
    permutation, sequences that do not cover the vertices, an unsupported hop."""
    import ctypes as C
    L = vs.capi.lib()
    g = vs.gen_rmat(6, 4, seed=3)
    rp, ci = vs.capi.ptr(g.row_ptrs, C.c_uint64), vs.capi.ptr(g.cols, C.c_uint32)
    assign = np.zeros(g.V, np.int32)
    sizes = np.zeros(200, np.int64)
    n = C.c_int32()

    def km(k, starts):
        st = np.asarray(starts, np.int32)
        return L.vsgm_kmeans(0, g.V, rp, ci, k, 3, vs.capi.ptr(st, C.c_int32), len(st), 0, vs.capi.ptr(assign, C.c_int32),
                             sizes.ctypes.data_as(C.POINTER(C.c_int64)), C.byref(n))

    assert km(0, [0]) == -1
    assert km(129, [0]) == -1
    assert km(4, [4]) == -1 and b"start" in L.vsgm_last_error()
    assert km(4, [-1]) == -1

    bins = np.zeros(g.V, np.int32)
    nb = C.c_int32()

    def pack(order, offs, hop=2):
        order = np.asarray(order, np.uint32)
        offs = np.asarray(offs, np.uint64)
        return L.vsgm_view_packing(0, g.V, rp, ci, vs.capi.ptr(order, C.c_uint32), vs.capi.ptr(offs, C.c_uint64), len(offs) - 1, hop, 10**6,
                                   vs.capi.ptr(bins, C.c_int32), C.byref(nb), None, 0)

    ident = np.arange(g.V)
    assert pack(np.zeros(g.V), [0, g.V]) == -1 and b"every vertex exactly once" in L.vsgm_last_error()
    assert pack(ident, [0, g.V - 1]) == -1
    assert pack(ident, [0, g.V // 2 + 1, g.V // 2, g.V]) == -1 and b"must not decrease" in L.vsgm_last_error()
    assert pack(ident, [0, g.V], hop=4) == -1
    out_rp = np.zeros(g.V + 1, np.uint64)
    out_ci = np.zeros(g.E + g.V, np.uint32)
    assert L.vsgm_features_1hop(0, 0, rp, ci, vs.capi.ptr(out_rp, C.c_uint64), vs.capi.ptr(out_ci, C.c_uint32)) == -1


def test_oracle_restatement_reproduces_the_reference_fixtures(vs, gold):
    """The oracle's restatement of kmeans and view_packing (oracle/oracle_tools.cc)
    gives the reference tools' own outputs on every fixture case."""
    import oracle
    for name in ["rmat", "chunglu"]:
        h = vs.Graph(gold[f"{name}_1hop_rp"], gold[f"{name}_1hop_ci"])
        for c, (k, iters, rc) in enumerate(gold["kmeans_cases"]):
            got = oracle.kmeans(h, int(k), int(iters), vs.reference_rand_starts(int(k), 1), bool(rc))
            np.testing.assert_array_equal(got, gold[f"{name}_kmeans_{c}"], err_msg=f"{name} kmeans {c}")
        g = vs.Graph(gold[f"{name}_rp"], gold[f"{name}_ci"])
        for c in gold[f"{name}_pack_cases"]:
            hop, threads, opt = (int(x) for x in gold["pack_cases"][c][:3])
            if opt:
                continue
            order, offs = vs.packing_order(gold[f"{name}_kmeans_0"], "1x4" if threads == 1 else "4", threads)
            cap = int(float(gold[f"{name}_pack_{c}_mem"][0]) * 1000 * 1000 * 1000 / 4)
            bins, nb, sizes = oracle.view_packing(g, order, offs, hop, cap)
            assert nb == int(gold[f"{name}_pack_{c}_nbins"][0])
            np.testing.assert_array_equal(bins, gold[f"{name}_pack_{c}_vbmap"], err_msg=f"{name} pack {c}")
            np.testing.assert_array_equal(sizes, gold[f"{name}_pack_{c}_sizes"], err_msg=f"{name} pack {c}")


REF_TOOLS = os.path.join(os.path.dirname(HERE), "oracle", "_ref")


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_TOOLS, "view_packing")), reason="the reference's view tools are not built")
def test_oracle_restatement_equals_reference_tools_on_random_graphs(vs, tmp_path):
    """Beyond the fixtures: seeded graphs of other shapes, the reference binaries
    (oracle/_ref) against the restatement, kmeans -t 1 and packing at hop 2 and 3."""
    import oracle
    graphs = [vs.gen_rmat(10, 6, seed=s) for s in (21, 22)] + [vs.gen_chung_lu(1500, 7000, g, 120, seed=9) for g in (2.2, 2.7)]
    for i, g in enumerate(graphs):
        d = tmp_path / f"g{i}"
        d.mkdir()
        vs.write_csr_bin(d / "g.bin", g)
        subprocess.run([os.path.join(REF_TOOLS, "features"), "-f", "g.bin", "-h", "1", "-t", "1"], cwd=d, check=True, capture_output=True)
        subprocess.run([os.path.join(REF_TOOLS, "kmeans"), "-f", "g.bin.1hop.bin", "-k", "5", "-i", "4", "-t", "1", "-init", "1"], cwd=d,
                       check=True, capture_output=True)
        want = np.loadtxt(d / "g.bin.1hop.bin.kmeans.5", dtype=np.int32)
        h = vs.read_csr_bin(d / "g.bin.1hop.bin")
        np.testing.assert_array_equal(oracle.kmeans(h, 5, 4, vs.reference_rand_starts(5, 1)), want)
        (d / "g.bin.kmeans.1x5").write_bytes((d / "g.bin.1hop.bin.kmeans.5").read_bytes())
        order, offs = vs.packing_order(want, "1x5", 1)
        for hop in (2, 3):
            for frac in (0.05, 0.3, 1.0):
                mem = frac * g.E * 4 / 1e9
                cap = int(mem * 1000 * 1000 * 1000 / 4)  # the bin size as the reference derives it from -m
                try:
                    bins, nb, _ = oracle.view_packing(g, order, offs, hop, cap)
                    break
                except ValueError:
                    continue
            r = subprocess.run([os.path.join(REF_TOOLS, "view_packing"), "-gf", "g.bin", "-pf", "g.bin.kmeans.1x5", "-h", str(hop), "-m",
                                repr(mem), "-t", "1", "-s", "1"], cwd=d, capture_output=True, text=True)
            assert r.returncode == 0, r.stderr
            wb, wn = vs.read_vbmap(d / f"g.bin.{hop}.hop.vbmap", g.V)
            assert nb == wn, (i, hop)
            np.testing.assert_array_equal(bins, wb, err_msg=f"graph {i} hop {hop}")
