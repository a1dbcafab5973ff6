"""Host side of libdmf.so (no GPU): the .bin formats, the create_bin-equivalent
builder, validation errors and the seeded generators."""
import os

import numpy as np
import pytest


def test_graph_load_save_roundtrip(dmf, golden_dir, tmp_path):
    src = os.path.join(golden_dir, "johnson8-2-4.bin")
    g = dmf.Graph.load(src)
    assert (g.num_nodes(), g.num_edges()) == (29, 420)
    out = tmp_path / "j.bin"
    g.save(str(out))
    assert out.read_bytes() == open(src, "rb").read()


def test_from_edges_byte_identical_to_reference_tool(dmf, golden_dir, tmp_path):
    t = np.loadtxt(os.path.join(golden_dir, "johnson8-2-4.txt"), dtype=np.int64)
    g = dmf.Graph.from_edges(t[:, 0], t[:, 1], t[:, 2])
    g.save(str(tmp_path / "b.bin"))
    assert (tmp_path / "b.bin").read_bytes() == open(os.path.join(golden_dir, "johnson8-2-4.bin"), "rb").read()


@pytest.mark.parametrize("seed", range(5))
def test_from_edges_matches_oracle_builder(dmf, oracle, seed):
    rng = np.random.default_rng(seed)
    k = 3000
    u = rng.integers(0, 300, k)
    v = rng.integers(0, 300, k)
    u[:200] = v[:200]                  # self-loops: dropped
    u[200:600], v[200:600] = u[600:1000], v[600:1000]  # duplicates: summed
    w = rng.integers(0, 50, k)
    g = dmf.Graph.from_edges(u, v, w)
    n, m, off, adj, cap, par = oracle.build_csr(u, v, w)
    assert (g.num_nodes(), g.num_edges()) == (n, m)
    for a, b in zip(g.arrays(), (off, adj, cap, par)):
        np.testing.assert_array_equal(a, b)


def test_find_arc_and_set_caps(dmf, golden_dir):
    g = dmf.Graph.load(os.path.join(golden_dir, "johnson8-2-4.bin"))
    off, adj, w, par = g.arrays()
    for v in range(g.num_nodes()):
        for e in range(off[v], off[v + 1]):
            assert g.find_arc(v, int(adj[e])) == e
    assert g.find_arc(0, 0) == -1
    e = g.find_arc(3, 4)
    g.set_caps([3], [4], [77])
    assert g.arrays()[2][e] == 77
    missing = next((a, b) for a in range(g.num_nodes()) for b in range(g.num_nodes())
                   if a != b and g.find_arc(a, b) < 0)
    with pytest.raises(dmf.DmfError) as ei:
        g.set_caps([missing[0]], [missing[1]], [5])
    assert ei.value.status == 3


def _write(path, arrs):
    with open(path, "wb") as f:
        for a in arrs:
            f.write(np.asarray(a, dtype=np.int32).tobytes())


def test_load_rejects_bad_files(dmf, golden_dir, tmp_path):
    raw = open(os.path.join(golden_dir, "johnson8-2-4.bin"), "rb").read()
    (tmp_path / "trunc.bin").write_bytes(raw[:-4])
    (tmp_path / "empty.bin").write_bytes(b"")
    for name in ("trunc.bin", "empty.bin", "missing.bin"):
        with pytest.raises(dmf.DmfError) as ei:
            dmf.Graph.load(str(tmp_path / name))
        assert ei.value.status == 2
    # broken partner involution
    a = np.frombuffer(raw, dtype=np.int32).copy()
    n, m = a[0], a[1]
    par_ofs = 2 + (n + 1) + 2 * m
    a[par_ofs] = a[par_ofs + 1]
    (tmp_path / "par.bin").write_bytes(a.tobytes())
    with pytest.raises(dmf.DmfError) as ei:
        dmf.Graph.load(str(tmp_path / "par.bin"))
    assert ei.value.status == 2 and "partner" in str(ei.value)
    # negative capacity
    b = np.frombuffer(raw, dtype=np.int32).copy()
    b[2 + (n + 1) + m] = -5
    (tmp_path / "neg.bin").write_bytes(b.tobytes())
    with pytest.raises(dmf.DmfError):
        dmf.Graph.load(str(tmp_path / "neg.bin"))
    # capacity + partner capacity overflow
    _write(tmp_path / "ovf.bin", [[2, 2], [0, 1, 2], [1, 0], [2**31 - 1, 1], [1, 0]])
    with pytest.raises(dmf.DmfError) as ei:
        dmf.Graph.load(str(tmp_path / "ovf.bin"))
    assert ei.value.status == 9
    # a valid two-vertex graph loads
    _write(tmp_path / "ok.bin", [[2, 2], [0, 1, 2], [1, 0], [5, 0], [1, 0]])
    assert dmf.Graph.load(str(tmp_path / "ok.bin")).num_edges() == 2


def test_int32_arguments_never_wrap(dmf, golden_dir):
    """Host arrays are converted to int32 only when every value fits exactly."""
    g = dmf.Graph.load(os.path.join(golden_dir, "johnson8-2-4.bin"))
    with pytest.raises(OverflowError):
        g.set_caps(np.array([2**32 + 1], np.int64), [2], [5])
    with pytest.raises(ValueError):
        g.set_caps([1.5], [2], [5])
    with pytest.raises(TypeError):
        g.set_caps(["a"], [2], [5])
    off, adj, _, _ = g.arrays()
    u = int(np.argmax(np.diff(off) > 0))  # a vertex with an out-arc
    v = int(adj[off[u]])
    g.set_caps(np.array([u], np.int64), np.array([v], np.uint8), np.array([7.0]))  # exact: accepted
    assert g.arrays()[2][g.find_arc(u, v)] == 7


def test_largest_vertex_id_is_rejected(dmf):
    """A vertex id of 2^31-1 would make the vertex count overflow int32: the
    builder says so instead of wrapping.  A self-loop on it is dropped before
    the count, as create_bin drops every self-loop."""
    with pytest.raises(dmf.DmfError) as ei:
        dmf.Graph.from_edges([2**31 - 1], [1], [5])
    assert ei.value.status == 1 and "no room for the vertex count" in str(ei.value)
    g = dmf.Graph.from_edges([0, 2**31 - 1], [1, 2**31 - 1], [5, 7])
    assert g.num_nodes() == 2 and g.num_edges() == 2


def test_validation_names_the_lowest_bad_arc(dmf, golden_dir):
    """With several defects of one kind, the message names the lowest arc,
    whatever the number of host threads that checked them."""
    g = dmf.Graph.load(os.path.join(golden_dir, "johnson8-2-4.bin"))
    off, adj, w, par = g.arrays()
    bad = w.copy()
    bad[[7, 40, g.num_edges() - 1]] = -1
    for _ in range(5):
        with pytest.raises(dmf.DmfError) as ei:
            dmf.Graph.from_csr(off, adj, bad, par)
        assert ei.value.status == 2 and "arc 7: negative capacity" in str(ei.value)


def test_updates_roundtrip_and_errors(dmf, tmp_path, oracle):
    p = str(tmp_path / "u.bin")
    dmf.save_updates(p, [1, 2, 3], [4, 5, 6], [7, 8, 9])
    s, d, w = dmf.load_updates(p)
    assert s.tolist() == [1, 2, 3] and d.tolist() == [4, 5, 6] and w.tolist() == [7, 8, 9]
    so, do, wo = oracle.read_updates(p)
    assert so.tolist() == [1, 2, 3] and wo.tolist() == [7, 8, 9]
    dmf.save_updates(p, [], [], [])
    assert len(dmf.load_updates(p)[0]) == 0
    with open(p, "wb") as f:
        f.write(np.array([5, 1, 2], np.int32).tobytes())
    with pytest.raises(dmf.DmfError):
        dmf.load_updates(p)


def test_grid_generator(dmf):
    g, s, t = dmf.gen_grid(256, 256, seed=0)
    assert (g.num_nodes(), s, t) == (65536, 0, 65535)
    off, adj, w, par = g.arrays()
    assert g.num_edges() == 2 * 2 * 256 * 255 + 2 * 254 * 2
    assert (w[par[par]] == w).all() and (par[par] == np.arange(g.num_edges())).all()
    grid_caps = w[w < 1000]
    assert grid_caps.min() >= 0 and grid_caps.max() <= 100
    g2, _, _ = dmf.gen_grid(256, 256, seed=0)
    for a, b in zip(g.arrays(), g2.arrays()):
        np.testing.assert_array_equal(a, b)


def test_rmat_generator(dmf):
    g, s, t = dmf.gen_rmat(12, seed=3, reserve=50)
    off, adj, w, par = g.arrays()
    n = g.num_nodes()
    assert n == 4096 and s != t
    tail = np.repeat(np.arange(n), np.diff(off))
    assert (tail != adj).all()
    assert w.min() >= 0 and w.max() <= 1000
    outdeg = np.bincount(tail[w > 0], minlength=n)
    assert outdeg[s] == outdeg.max()
    # reserved slots: zero-capacity arcs whose partner is zero too
    assert ((w == 0) & (w[par] == 0)).sum() >= 50
    g2, s2, t2 = dmf.gen_rmat(12, seed=3, reserve=50)
    assert (s2, t2) == (s, t) and (g2.arrays()[1] == adj).all()


def test_batch_generator(dmf):
    g, s, t = dmf.gen_rmat(12, seed=0, reserve=200)
    batches = dmf.gen_batches(g, 4, frac=0.01, p_inc=0.4, p_dec=0.4, p_ins=0.1, delta_hi=500, seed=9)
    off, adj, w, par = g.arrays()
    cur = w.copy()
    npos = (w > 0).sum()
    for src, dst, nw in batches:
        assert abs(len(src) - round(0.01 * (cur > 0).sum())) <= 2
        arcs = [g.find_arc(int(a), int(b)) for a, b in zip(src, dst)]
        assert min(arcs) >= 0 and len(set(arcs)) == len(arcs)  # existing, distinct
        old = cur[arcs]
        ins = (old == 0).sum()
        dele = ((old > 0) & (nw == 0)).sum()
        assert ins >= 1 and dele >= 1
        cur[arcs] = nw
    assert npos > 0
