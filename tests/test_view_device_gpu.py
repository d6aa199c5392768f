"""View bins built on the device (vsgm_upload_graph + vsgm_materialize_view).

ViewBin::Materialize (src/view/view_bin.h:66-142) builds, for a bin's sources,
the full-V CSR holding the rows of every vertex within hop-1 steps of a source
of degree >= root_degree.  The device build must equal the host build byte for
byte, and matching over it must give the same exact counts.
"""
import re
import subprocess

import numpy as np
import pytest

from conftest import complete_graph, cycle_graph, small_graphs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def graphs(vs):
    return small_graphs(vs)


def _same(a, b):
    assert a.V == b.V
    np.testing.assert_array_equal(a.row_ptrs, b.row_ptrs)
    np.testing.assert_array_equal(a.cols, b.cols)


@pytest.mark.parametrize("name", ["rmat7", "rmat8", "chunglu"])
def test_device_halo_equals_host(vs, graphs, name):
    g = graphs[name]
    rng = np.random.default_rng(5)
    with vs.Engine(g.V, [vs.plan_clique(3)]) as e:
        e.upload_graph(g)
        for hop in (1, 2, 3):
            for root_degree in (0, 3, 9):
                src = np.sort(rng.choice(g.V, size=max(1, g.V // 7), replace=False)).astype(np.uint32)
                e.materialize_view(src, hop, root_degree)
                _same(e.read_view(), vs.materialize_view(g, src, hop, root_degree))


def test_device_halo_matches_reference_golden(vs):
    """Device-built views equal the reference's ViewBin::Materialize output
    (tests/golden/ref_views.npz, made from the reference sources)."""
    import os
    from conftest import ROOT
    z = np.load(os.path.join(ROOT, "tests", "golden", "ref_views.npz"))
    g = vs.Graph(z["row_ptrs"], z["cols"])
    src = vs.sources_of_bins(z["bins"], 3)
    with vs.Engine(g.V, [vs.plan_clique(3)]) as e:
        e.upload_graph(g)
        for c, (hop, rd) in enumerate(z["cases"]):
            for b in range(3):
                e.materialize_view(src[b], int(hop), int(rd))
                v = e.read_view()
                np.testing.assert_array_equal(v.row_ptrs, z[f"rp_{c}_{b}"])
                np.testing.assert_array_equal(v.cols, z[f"ci_{c}_{b}"])


def test_device_halo_edge_cases(vs, graphs):
    g = graphs["rmat8"]
    with vs.Engine(g.V, [vs.plan_clique(3)]) as e:
        e.upload_graph(g)
        # no sources: an empty view, zero matches
        e.materialize_view(np.zeros(0, np.uint32), 2)
        v = e.read_view()
        assert v.E == 0 and v.row_ptrs.shape == (g.V + 1,)
        e.match()
        assert e.counts() == [0]
        # duplicated sources and every vertex as a source
        dup = np.array([3, 3, 5, 3], np.uint32)
        e.materialize_view(dup, 2)
        _same(e.read_view(), vs.materialize_view(g, dup, 2))
        every = np.arange(g.V, dtype=np.uint32)
        e.materialize_view(every, 2)
        _same(e.read_view(), g)
        # out-of-range source is rejected on the host
        with pytest.raises(vs.VsgmError):
            e.materialize_view(np.array([g.V], np.uint32), 2)
        with pytest.raises(vs.VsgmError):
            e.materialize_view(every, 0)


def test_device_views_count_like_host_views(vs, orc, graphs):
    """Matching bin by bin over device-built views sums to the whole-graph count."""
    g = graphs["chunglu"]
    plans = [vs.plan_clique(4), vs.plan_pattern(1), vs.plan_pattern(4)]
    hop = max(p.hop for p in plans)
    bins = vs.sources_of_bins((np.arange(g.V) * 5 % 4).astype(np.int32), 4)
    with vs.Engine(g.V, plans) as e:
        e.upload_graph(g)
        for src in bins:
            e.materialize_view(src, hop)
            e.match()
        got = e.counts()
    assert got == [orc.count(p, g) for p in plans]
    # the resident graph as the view of every bin: same totals, no halo built
    with vs.Engine(g.V, plans) as e:
        e.upload_graph(g)
        for src in bins:
            e.graph_view(src)
            e.match()
        assert e.counts() == got
    for G in (complete_graph(vs, 8), cycle_graph(vs, 10)):
        with vs.Engine(G.V, plans) as e:
            e.upload_graph(G)
            e.materialize_view(np.arange(G.V, dtype=np.uint32), hop)
            e.match()
            assert e.counts() == [orc.count(p, G) for p in plans]


def test_pm_pipeline_device_views(vs, orc, graphs, tmp_path):
    """The CLI gives the same counts with host-built halos (-gv 0), device-built halos
    (-gv 1) and the resident whole graph as every bin's view (-gv 2)."""
    from vsgm_b200 import build

    g = graphs["rmat8"]
    path = tmp_path / "g.bin"
    vs.write_csr_bin(path, g)
    bins = (np.arange(g.V) * 7 % 5).astype(np.int32)
    vs.write_vbmap(str(path) + ".2.hop.vbmap", bins, 5)
    want = orc.count(vs.plan_pattern(2), g)
    for gv in ("0", "1", "2"):
        out = subprocess.run([build.DRIVER, "-f", str(path), "-m", "1", "-p", "2", "-pn", "2", "-cn", "1", "-gv", gv],
                             capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stderr
        assert int(re.search(r"total count for query 0: (\d+)", out.stdout).group(1)) == want


def test_device_relabel_equals_host(vs, orc, graphs):
    """vsgm_upload_graph with the "relabel" option: the resident graph equals the host
    relabelling (ids ascending with (degree, id)) entry for entry, totals do not
    change, and a bin given in the caller's ids counts what the oracle counts on the
    relabelled graph at the mapped sources (4-cycles by their largest vertex)."""
    from conftest import complete_graph, empty_graph
    kc4, p1, p2 = vs.plan_clique(4), vs.plan_pattern(1), vs.plan_pattern(2)
    for g in (graphs["rmat8"], graphs["chunglu"], vs.gen_rmat(12, 16, seed=3), empty_graph(vs, 9), complete_graph(vs, 12)):
        h, new_of_old = vs.degree_relabel(g, ascending=True)
        with vs.Engine(g.V, [kc4, p1, p2]) as e:
            e.set_option("relabel", 1)
            e.upload_graph(g)
            e.graph_view(np.arange(g.V, dtype=np.uint32))
            r = e.read_view()
            assert np.array_equal(r.row_ptrs, h.row_ptrs) and np.array_equal(r.cols, h.cols)
            e.match()
            assert e.counts() == [orc.count(p, g) for p in (kc4, p1, p2)]
            src = np.arange(0, g.V, 3, dtype=np.uint32)
            mapped = np.sort(new_of_old[src]).astype(np.uint32)
            e.reset_counts()
            e.graph_view(src)
            e.match()
            assert e.counts() == [orc.count(kc4, h, mapped), orc.c4_by_largest(h, mapped), orc.count(p2, h, mapped)]
            e.reset_counts()
            e.materialize_view(src, 2)
            e.match()
            assert e.counts() == [orc.count(kc4, h, mapped), orc.c4_by_largest(h, mapped), orc.count(p2, h, mapped)]


def test_prefetched_compact_views(vs, orc, graphs):
    """Views sent in compact form and copied while the previous view is matched
    (vsgm_prefetch_view / vsgm_swap_view / vsgm_view_released) count what the
    synchronous full-V transfer counts, bin by bin; pinned host buffers allocate
    and free."""
    import ctypes as C
    g = graphs["rmat8"]
    plans = [vs.plan_clique(4), vs.plan_pattern(1), vs.plan_pattern(2), vs.plan_pattern(4)]
    bins = [np.arange(b, g.V, 4, dtype=np.uint32) for b in range(4)]
    views = [vs.materialize_view(g, src, 2) for src in bins]
    with vs.Engine(g.V, plans) as e:
        want = []
        for v, src in zip(views, bins):
            e.reset_counts()
            e.transfer_view(v, src)
            e.match()
            want.append(e.counts())
        got = []
        e.prefetch_view(views[0], bins[0])
        e.swap_view()
        e.view_released()
        for k in range(4):
            if k + 1 < 4:
                e.prefetch_view(views[k + 1], bins[k + 1])  # copies while view k is matched
            e.reset_counts()
            e.match()
            got.append(e.counts())
            if k + 1 < 4:
                e.swap_view()
                e.view_released()
        assert got == want
        assert [sum(c[i] for c in got) for i in range(len(plans))] == [orc.count(p, g) for p in plans]
        with pytest.raises(vs.VsgmError):
            e.swap_view()  # nothing prefetched
    p = C.c_void_p()
    vs.capi.check(vs.capi.lib().vsgm_host_alloc(1 << 20, C.byref(p)))
    assert p.value
    vs.capi.check(vs.capi.lib().vsgm_host_free(p))
