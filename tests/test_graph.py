"""Host layers: file formats, generators, view materialisation, ABI surface (CPU only)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, complete_graph


def test_rmat_is_simple_sorted_symmetric(vs):
    g = vs.gen_rmat(10, 16, seed=1)
    assert g.V == 1024
    assert vs.csr_defects(g) == 0
    src = np.repeat(np.arange(g.V), np.diff(g.row_ptrs).astype(np.int64))
    fwd = set(zip(src.tolist(), g.cols.tolist()))
    assert all((b, a) in fwd for a, b in fwd)


def test_generators_are_deterministic(vs):
    a, b = vs.gen_rmat(9, 8, seed=3), vs.gen_rmat(9, 8, seed=3)
    assert np.array_equal(a.row_ptrs, b.row_ptrs) and np.array_equal(a.cols, b.cols)
    c = vs.gen_rmat(9, 8, seed=4)
    assert not np.array_equal(a.cols, c.cols)
    d1, d2 = vs.gen_chung_lu(5000, 40000, 2.4, 300, seed=9), vs.gen_chung_lu(5000, 40000, 2.4, 300, seed=9)
    assert np.array_equal(d1.cols, d2.cols)
    assert vs.csr_defects(d1) == 0
    assert d1.degrees().max() < 600  # capped expected degree


def test_chung_lu_degree_skew(vs):
    g = vs.gen_chung_lu(20000, 200000, 2.1, 2000, seed=1)
    deg = g.degrees()
    assert deg[:10].mean() > 20 * deg[10000:].mean()


def test_csr_bin_round_trip_and_layout(vs, tmp_path):
    g = vs.gen_rmat(8, 8, seed=2)
    p = tmp_path / "g.bin"
    vs.write_csr_bin(p, g)
    raw = p.read_bytes()
    hdr = np.frombuffer(raw[:32], np.uint64)
    assert hdr.tolist() == [4, 8, g.V, g.E]
    assert len(raw) == 32 + 8 * (g.V + 1) + 4 * g.E
    h = vs.read_csr_bin(p)
    assert np.array_equal(h.row_ptrs, g.row_ptrs) and np.array_equal(h.cols, g.cols)


def test_csr_bin_rejects_truncated_file(vs, tmp_path):
    g = vs.gen_rmat(6, 4, seed=2)
    p = tmp_path / "g.bin"
    vs.write_csr_bin(p, g)
    p.write_bytes(p.read_bytes()[:-4])
    with pytest.raises(vs.VsgmError):
        vs.read_csr_bin(p)
    with pytest.raises(vs.VsgmError):
        vs.read_csr_bin(tmp_path / "missing.bin")


def test_csr_bin_size_must_match_header(vs, tmp_path):
    """Like the reference reader, the file must end right after the cols; the
    allocating reader, the two-step reader and the driver's path agree."""
    from vsgm_b200 import capi
    g = vs.gen_rmat(7, 4, seed=3)
    p = tmp_path / "g.bin"
    vs.write_csr_bin(p, g)
    good = p.read_bytes()
    p.write_bytes(good + b"\0")  # one byte too many
    with pytest.raises(vs.VsgmError):
        vs.read_csr_bin(p)
    bad = bytearray(good)
    bad[16:24] = np.uint64(g.V + 1).tobytes()  # V that does not fit the size
    p.write_bytes(bytes(bad))
    with pytest.raises(vs.VsgmError):
        vs.read_csr_bin(p)
    p.write_bytes(good)
    L = capi.lib()
    import ctypes as C
    rp = np.empty(g.V + 1, np.uint64)
    ci = np.empty(g.E, np.uint32)
    # the caller's sizes must be the file's
    assert L.vsgm_read_csr_bin_into(str(p).encode(), g.V, g.E - 1, capi.ptr(rp, C.c_uint64), capi.ptr(ci, C.c_uint32), 2) != 0
    V, E = C.c_uint64(), C.c_uint64()
    rpp, cip = C.POINTER(C.c_uint64)(), C.POINTER(C.c_uint32)()
    assert L.vsgm_read_csr_bin(str(p).encode(), C.byref(V), C.byref(E), C.byref(rpp), C.byref(cip)) == 0
    assert (V.value, E.value) == (g.V, g.E)
    assert np.array_equal(np.ctypeslib.as_array(cip, shape=(g.E,)), g.cols)
    L.vsgm_free(C.cast(rpp, C.c_void_p))
    L.vsgm_free(C.cast(cip, C.c_void_p))


def test_csr_bin_multi_chunk_parallel_read(vs, tmp_path):
    """A file larger than one read chunk (64 MB), read with several threads."""
    g = vs.gen_rmat(20, 16, seed=4)
    assert 4 * g.E > (64 << 20)
    p = tmp_path / "big.bin"
    vs.write_csr_bin(p, g)
    for threads in (1, 3, 0):
        h = vs.read_csr_bin(p, threads=threads)
        assert np.array_equal(h.row_ptrs, g.row_ptrs) and np.array_equal(h.cols, g.cols)


def test_vbmap_round_trip(vs, tmp_path):
    bins = np.array([0, 2, 1, 1, 0, 2, 2], np.int32)
    p = tmp_path / "g.bin.2.hop.vbmap"
    vs.write_vbmap(p, bins, 3)
    assert p.read_text().split() == ["3"] + [str(b) for b in bins]
    got, nb = vs.read_vbmap(p, 7)
    assert nb == 3 and got.tolist() == bins.tolist()
    srcs = vs.sources_of_bins(got, nb)
    assert [s.tolist() for s in srcs] == [[0, 4], [2, 3], [1, 5, 6]]
    p.write_text("2\n0\n5\n")
    with pytest.raises(vs.VsgmError):
        vs.read_vbmap(p, 2)
    # Windows line ends and spare whitespace parse like the reference's operator>>
    p.write_bytes(b"3\r\n0\r\n2 \t\n1\r\n\n")
    got, nb = vs.read_vbmap(p, 3)
    assert nb == 3 and got.tolist() == [0, 2, 1]
    for bad in (b"2\n0\n-1\n", b"2\n0\nx\n", b"-2\n0\n", b"2\n0\n"):
        p.write_bytes(bad)
        with pytest.raises(vs.VsgmError):
            vs.read_vbmap(p, 2)


def _halo(g, sources, hop, root_degree):
    deg = g.degrees()
    keep = set()
    frontier = [s for s in sources if root_degree == 0 or deg[s] >= root_degree]
    keep.update(frontier)
    for _ in range(hop - 1):
        nxt = []
        for x in frontier:
            for y in g.cols[g.row_ptrs[x]:g.row_ptrs[x + 1]]:
                if y not in keep:
                    keep.add(int(y))
                    nxt.append(int(y))
        frontier = nxt
    return keep


@pytest.mark.parametrize("hop,root_degree", [(1, 0), (2, 0), (3, 0), (2, 4)])
def test_view_materialize_matches_halo(vs, hop, root_degree):
    g = vs.gen_rmat(9, 8, seed=5)
    rng = np.random.default_rng(hop)
    sources = np.sort(rng.choice(g.V, size=40, replace=False)).astype(np.uint32)
    v = vs.materialize_view(g, sources, hop, root_degree)
    keep = _halo(g, sources.tolist(), hop, root_degree)
    for x in range(g.V):
        row = v.cols[v.row_ptrs[x]:v.row_ptrs[x + 1]]
        if x in keep:
            assert np.array_equal(row, g.cols[g.row_ptrs[x]:g.row_ptrs[x + 1]])
        else:
            assert len(row) == 0


def _ref_views():
    return np.load(os.path.join(ROOT, "tests", "golden", "ref_views.npz"))


def test_view_materialize_matches_reference_golden(vs, tmp_path):
    """Byte-identical to the reference's own ViewBin::Materialize (fixture made by
    tests/golden/make_view_golden.py from the reference sources), and our .bin file
    reads back in the reference reader with the same V, E and column sum."""
    z = _ref_views()
    g = vs.Graph(z["row_ptrs"], z["cols"])
    V, E, colsum = (int(x) for x in z["read"])
    assert (g.V, g.E, int(g.cols.astype(np.uint64).sum())) == (V, E, colsum)
    path = tmp_path / "g.bin"
    vs.write_csr_bin(path, g)
    h = vs.read_csr_bin(path)
    assert np.array_equal(h.row_ptrs, g.row_ptrs) and np.array_equal(h.cols, g.cols)
    src = vs.sources_of_bins(z["bins"], 3)
    for c, (hop, rd) in enumerate(z["cases"]):
        for b in range(3):
            v = vs.materialize_view(g, src[b], int(hop), int(rd))
            np.testing.assert_array_equal(v.row_ptrs, z[f"rp_{c}_{b}"])
            np.testing.assert_array_equal(v.cols, z[f"ci_{c}_{b}"])


def test_view_capacity_error(vs):
    g = complete_graph(vs, 6)
    L = vs.capi.lib()
    vrp = np.zeros(g.V + 1, np.uint64)
    vci = np.zeros(4, np.uint32)
    n = C.c_uint64()
    src = np.array([0], np.uint32)
    rc = L.vsgm_view_materialize(g.V, vs.capi.ptr(g.row_ptrs, C.c_uint64), vs.capi.ptr(g.cols, C.c_uint32), vs.capi.ptr(src, C.c_uint32),
                                 1, 2, 0, 1, vs.capi.ptr(vrp, C.c_uint64), vs.capi.ptr(vci, C.c_uint32), 4, C.byref(n))
    assert rc != 0 and n.value == 30


def test_random_patterns_are_connected_and_seeded(vs):
    ctr = 0
    seen = []
    for _ in range(64):
        n, bits, ctr = vs.random_pattern(seed=3, counter=ctr)
        assert 3 <= n <= 6
        p = vs.plan_query_bits(n, bits)  # raises if disconnected
        assert p.n_vertices == n
        seen.append((n, tuple(bits)))
    ctr2 = 0
    again = []
    for _ in range(64):
        n, bits, ctr2 = vs.random_pattern(seed=3, counter=ctr2)
        again.append((n, tuple(bits)))
    assert seen == again
    assert len({s for s in seen}) > 20


def test_library_exports_every_declared_symbol(vs):
    """Every function include/*.h declares is exported by libvsgm_b200.so (no GPU needed)."""
    decl = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        text = open(os.path.join(ROOT, "include", h)).read()
        decl |= set(re.findall(r"\b(vsgm_[a-z0-9_]+)\s*\(", text))
    L = C.CDLL(vs.capi.LIB_PATH)
    missing = [d for d in sorted(decl) if not hasattr(L, d)]
    assert not missing, missing
    assert set(vs.capi.EXPORTED) <= decl


def test_engine_create_fails_cleanly_without_gpu(vs):
    import torch

    if torch.cuda.is_available():
        pytest.skip("GPU present")
    p = vs.plan_clique(3)
    with pytest.raises(vs.VsgmError):
        vs.Engine(16, [p])


def test_pm_pipeline_fails_cleanly_without_gpu(vs, tmp_path):
    """With no usable GPU the driver reports the error and exits non-zero instead
    of hanging its producer/consumer threads (every -gv mode)."""
    import subprocess

    import torch

    from vsgm_b200 import build
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    g = vs.gen_rmat(7, 8, seed=2)
    path = tmp_path / "g.bin"
    vs.write_csr_bin(path, g)
    vs.write_vbmap(str(path) + ".2.hop.vbmap", (np.arange(g.V) % 3).astype(np.int32), 3)
    for gv in ("0", "1", "2"):
        out = subprocess.run([build.DRIVER, "-f", str(path), "-kc", "3", "-pn", "2", "-qs", "1", "-gv", gv],
                             capture_output=True, text=True, timeout=120)
        assert out.returncode != 0
        assert "error" in out.stderr
    # a partition file that exists but cannot be read is an error, not a fallback
    vb = str(path) + ".2.hop.vbmap"
    os.remove(vb)
    os.mkdir(vb)
    out = subprocess.run([build.DRIVER, "-f", str(path), "-kc", "3"], capture_output=True, text=True, timeout=120)
    assert out.returncode != 0 and "error" in out.stderr and "one view bin of every vertex" not in out.stdout
    os.rmdir(vb)
    # without a partition file the driver uses one bin of every vertex, and says so
    out = subprocess.run([build.DRIVER, "-f", str(path), "-kc", "3"], capture_output=True, text=True, timeout=120)
    assert "no view bin partition file" in out.stdout and "one view bin of every vertex" in out.stdout
    assert "loaded view bin partition file" not in out.stdout
    # ... and a halo of the whole graph (-gv 0 / 1) must fit the -m budget
    out = subprocess.run([build.DRIVER, "-f", str(path), "-kc", "3", "-gv", "0", "-m", "1e-9"], capture_output=True, text=True, timeout=120)
    assert out.returncode != 0 and "exceeds -m" in out.stderr


def test_view_compact_roundtrip(vs):
    """The compact view form (vertices with a non-empty row and their offsets)
    expands back to the full-V row offsets the way the device expands it."""
    g = vs.gen_rmat(9, 8, seed=4)
    for src in (np.arange(0, g.V, 5, dtype=np.uint32), np.arange(g.V, dtype=np.uint32), np.zeros(0, np.uint32)):
        v = vs.materialize_view(g, src, 2)
        vert, off = vs.view_compact(v)
        assert off[0] == 0 and off[-1] == v.row_ptrs[-1] and np.all(np.diff(vert.astype(np.int64)) > 0)
        rp = off[np.searchsorted(vert, np.arange(v.V + 1), side="left")]
        assert np.array_equal(rp, v.row_ptrs)
