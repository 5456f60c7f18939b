"""GPU parity of incremental single-source BFS / SSSP (GIR::trackIncremental / updateIncremental /
incDist, gir_query.cpp:867-996) through the C ABI. After every update the tracked result equals
both the reference's own incremental result (compiled from its sources, driven through the same
updates) and the oracle's from-scratch BFS / SSSP of the current graph. The rounds follow the
reference's IncTest (gir_test.cpp:1043-1083): batches of mostly deletions of existing edges,
applied as one batch, as single directed updates or as single undirected updates."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NONE = np.uint64(2**64 - 1)


@pytest.fixture(scope="module")
def s16(pkg, orc):
    g = pkg.graphs.rmat_s16()
    fb, fa = orc.normalize(g.V, g.fw_beg, g.fw_adj)
    return g, fb, fa


def _scratch(orc, V, cb, ca, src):
    lv = orc.bfs(V, cb, ca, [src])
    return np.where(lv < 0, NONE, lv.astype(np.uint64)), orc.sssp(V, cb, ca, [src])


def _round_ops(rng, V, cb, ca, n):
    """Two in three ops delete an existing edge (they cut dependence trees), the rest insert a
    random pair (gir_test.cpp:1052-1062)."""
    u, v, ins = [], [], []
    for _ in range(n):
        if rng.integers(3):
            a = int(rng.integers(V))
            row = ca[cb[a]:cb[a + 1]]
            if len(row):
                u.append(a)
                v.append(int(row[rng.integers(len(row))]))
                ins.append(0)
                continue
        a, b = int(rng.integers(V)), int(rng.integers(V))
        if a != b:
            u.append(a)
            v.append(b)
            ins.append(1)
    return np.array(u, np.int32), np.array(v, np.int32), np.array(ins, np.uint8)


@pytest.mark.parametrize("scale,rounds,max_ops", [(10, 40, 40), (14, 12, 2000)])
def test_incremental_matches_reference_and_scratch(pkg, orc, scale, rounds, max_ops):
    g = pkg.graphs.rmat(scale, seed=scale, weights=None)
    V = g.V
    gir = pkg.GIR(graph=g)
    gir.buildWCC()
    gir.buildSCC_DAG()
    gir.buildBCT()
    d = gir.device
    cb, ca = d.csr(0)
    ref = orc.RefGIR(V, cb.astype(np.int32), ca, *orc.transpose(V, cb, ca))
    ref.build(7)  # (the reference's applyBatch expects all three layers)
    rng = np.random.default_rng(scale)
    src = int(np.argmax(np.diff(g.fw_beg)))
    for w in (False, True):
        gir.trackIncremental(src, w)
        ref.inc_track(src, w)
    cut_total = 0
    for r in range(rounds):
        cb, ca = d.csr(0)
        u, v, ins = _round_ops(rng, V, cb, ca, int(rng.integers(1, max_ops + 1)))
        how = r % 3
        if how == 0:
            gir.applyBatch(zip(u.tolist(), v.tolist(), ins.tolist()))
            ref.apply_batch(u, v, ins)
        else:
            u, v, ins = u[:200], v[:200], ins[:200]
            for a, b, i in zip(u.tolist(), v.tolist(), ins.tolist()):
                if how == 1:
                    gir.updateEdgeDirected(a, b, bool(i))
                else:
                    gir.updateEdgeUndirected(a, b, bool(i))
                ref.update_edge(a, b, bool(i), undirected=how == 2)
        for w in (False, True):
            gir.updateIncremental(w)
            if w:
                cut_total += d.query_stats()["reached"]
            ref.inc_update(w)
        cb, ca = d.csr(0)
        rb, ra = ref.out_csr()
        np.testing.assert_array_equal(cb, rb)
        np.testing.assert_array_equal(ca, ra)
        want_b, want_w = _scratch(orc, V, cb, ca, src)
        got_b, got_w = d.inc_dist(False), d.inc_dist(True)
        np.testing.assert_array_equal(got_b, want_b, err_msg=f"bfs, round {r}")
        np.testing.assert_array_equal(got_w, want_w, err_msg=f"sssp, round {r}")
        np.testing.assert_array_equal(got_b, ref.inc_dist(False))
        np.testing.assert_array_equal(got_w, ref.inc_dist(True))
        assert gir.incDist(True, src) == 0
    assert cut_total > 0  # some deletion did cut a dependence subtree
    ref.close()
    d.close()


def test_incremental_cut_at_the_source(pkg, orc, s16):
    """Deleting every out-edge of the source cuts the whole reached set (one list of many
    levels); putting them back restores it."""
    g, fb, fa = s16
    V = g.V
    d = pkg.DeviceGraph.from_graph(g)
    src = int(np.argmax(np.diff(fb)))
    d.inc_track(src, True)
    d.inc_track(src, False)
    outs = fa[fb[src]:fb[src + 1]]
    d.apply_batch(np.full(len(outs), src, np.int32), outs, np.zeros(len(outs), np.uint8))
    d.inc_update(True)
    st = d.query_stats()
    assert st["reached"] > 1000
    d.inc_update(False)
    got = d.inc_dist(True)
    assert got[src] == 0 and np.all(np.delete(got, src) == NONE)
    d.apply_batch(np.full(len(outs), src, np.int32), outs, np.ones(len(outs), np.uint8))
    d.inc_update(True)
    d.inc_update(False)
    want_b, want_w = _scratch(orc, V, fb, fa, src)
    np.testing.assert_array_equal(d.inc_dist(True), want_w)
    np.testing.assert_array_equal(d.inc_dist(False), want_b)
    d.close()


def test_incremental_edge_cases(pkg, orc, s16):
    g, fb, fa = s16
    V = g.V
    n = pkg.native
    d = pkg.DeviceGraph.from_graph(g)
    # a mode never tracked has no result
    with pytest.raises(n.GirError) as e:
        d.inc_dist(True)
    assert e.value.code == 6
    # sources out of range track an all-unreachable result, which updates keep
    for bad in (-1, V + 3):
        d.inc_track(bad, True)
        d.apply_batch(np.array([0, 1], np.int32), np.array([5, 7], np.int32), np.ones(2, np.uint8))
        d.inc_update(True)
        assert np.all(d.inc_dist(True) == NONE)
    # nothing logged: the update does nothing
    cb, ca = d.csr(0)
    d.inc_track(3, False)
    d.inc_update(False)
    assert d.query_stats()["iterations"] == 0
    want_b, _ = _scratch(orc, V, cb, ca, 3)
    np.testing.assert_array_equal(d.inc_dist(False), want_b)
    # tracking again drops what was logged before and starts from the current graph
    u = np.array([3] * 4, np.int32)
    v = ca[cb[3]:cb[3] + 4].astype(np.int32)
    d.apply_batch(u[:len(v)], v, np.zeros(len(v), np.uint8))
    d.inc_track(3, False)
    cb, ca = d.csr(0)
    want_b, want_w = _scratch(orc, V, cb, ca, 3)
    np.testing.assert_array_equal(d.inc_dist(False), want_b)
    d.inc_update(False)
    np.testing.assert_array_equal(d.inc_dist(False), want_b)
    # a batch that changes nothing logs nothing
    d.inc_track(3, True)
    d.apply_batch(np.array([0], np.int32), np.array([0], np.int32), np.ones(1, np.uint8))  # self-loop: invalid
    d.inc_update(True)
    assert d.query_stats()["iterations"] == 0
    np.testing.assert_array_equal(d.inc_dist(True), want_w)
    d.close()


def test_incremental_large_batches(pkg, orc):
    """1M vertices, 16M draws: rounds of 20K-op batches against the oracle's from-scratch results."""
    g = pkg.graphs.rmat(20, seed=11, weights=None)
    V = g.V
    d = pkg.DeviceGraph.from_graph(g, weights=False)
    rng = np.random.default_rng(20)
    src = int(np.argmax(np.diff(g.fw_beg)))
    d.inc_track(src, True)
    d.inc_track(src, False)
    for r in range(3):
        cb, ca = d.csr(0)
        k = 14000
        a = rng.integers(0, V, k)
        deg = cb[a + 1] - cb[a]
        a = a[deg > 0]
        b = ca[cb[a] + rng.integers(0, 1 << 30, len(a)) % (cb[a + 1] - cb[a])]
        iu = rng.integers(0, V, 6000)
        iv = rng.integers(0, V, 6000)
        u = np.concatenate([a, iu]).astype(np.int32)
        v = np.concatenate([b, iv]).astype(np.int32)
        ins = np.concatenate([np.zeros(len(a)), np.ones(6000)]).astype(np.uint8)
        d.apply_batch(u, v, ins)
        d.inc_update(True)
        d.inc_update(False)
        cb, ca = d.csr(0)
        want_b, want_w = _scratch(orc, V, cb, ca, src)
        np.testing.assert_array_equal(d.inc_dist(True), want_w, err_msg=f"round {r}")
        np.testing.assert_array_equal(d.inc_dist(False), want_b, err_msg=f"round {r}")
    d.close()
