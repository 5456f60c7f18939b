"""Pins the C restatement of the oracle: against the golden vectors made by the reference itself
(tests/golden/make_golden.py) and, where the reference was compiled here, against the reference
on larger generated graphs. CPU only."""
import os

import numpy as np
import pytest

from conftest import golden_cases


def _layers_match(orc, V, fb, fa, exp, key):
    L = orc.Layers(V, fb, fa)
    np.testing.assert_array_equal(L.wcc, exp[f"{key}/wcc"], err_msg=f"{key} wcc")
    np.testing.assert_array_equal(L.scc, exp[f"{key}/scc"], err_msg=f"{key} scc")
    np.testing.assert_array_equal(L.dag, exp[f"{key}/dag"], err_msg=f"{key} dag")
    np.testing.assert_array_equal(L.blocks, exp[f"{key}/blocks"], err_msg=f"{key} blocks")
    np.testing.assert_array_equal(L.ap, exp[f"{key}/ap"], err_msg=f"{key} ap")
    np.testing.assert_array_equal(L.sb, exp[f"{key}/sym_beg"], err_msg=f"{key} sym beg")
    np.testing.assert_array_equal(L.sa, exp[f"{key}/sym_adj"], err_msg=f"{key} sym adj")
    src = exp[f"{key.split('/')[0]}/sources"]
    for i, s in enumerate(src):
        np.testing.assert_array_equal(orc.bfs(V, fb, fa, [s]), exp[f"{key}/bfs"][i], err_msg=f"{key} bfs {s}")
        np.testing.assert_array_equal(orc.sssp(V, fb, fa, [s]), exp[f"{key}/sssp"][i], err_msg=f"{key} sssp {s}")


def test_oracle_replays_every_golden_case(orc, golden):
    for case in golden_cases(golden):
        V = int(golden[f"{case}/V"][0])
        fb, fa = orc.normalize(V, golden[f"{case}/in_fw_beg"], golden[f"{case}/in_fw_adj"])
        np.testing.assert_array_equal(fb, golden[f"{case}/s0/fw_beg"])
        np.testing.assert_array_equal(fa, golden[f"{case}/s0/fw_adj"])
        _layers_match(orc, V, fb, fa, golden, f"{case}/s0")
        for k in range(1, int(golden[f"{case}/steps"][0]) + 1):
            key = f"{case}/s{k}"
            fb, fa, _, _ = orc.apply_batch(V, fb, fa, golden[f"{key}/ops_u"], golden[f"{key}/ops_v"],
                                           golden[f"{key}/ops_ins"])
            np.testing.assert_array_equal(fb, golden[f"{key}/fw_beg"], err_msg=key)
            np.testing.assert_array_equal(fa, golden[f"{key}/fw_adj"], err_msg=key)
            _layers_match(orc, V, fb, fa, golden, key)


def test_targeted_split_known_answers(golden):
    """runTargetedSplitTest (gir_test.cpp:704-753) and the selftest regressions
    (gir_selftest.cpp:209-233), as recorded from the reference."""
    wccs = lambda key: len(np.unique(golden[f"{key}/wcc"]))
    sccs = lambda key: len(np.unique(golden[f"{key}/scc"]))
    assert wccs("example/s1") == wccs("example/s0") - 1  # insert 3->12 joins two WCCs
    assert wccs("example/s2") == wccs("example/s0")      # deleting it splits them again
    s2, s3 = golden["example/s2/scc"], golden["example/s3/scc"]
    assert s2[0] == s2[9] and s3[0] != s3[9]              # delete 9->2 splits {0,1,2,9,10,11}
    assert s3[0] == s3[1] == s3[2] and s3[9] == s3[10] == s3[11]
    assert sccs("example/s3") == sccs("example/s2") + 1
    d = golden["example_del01/s1/scc"]
    assert d[0] != d[1]                                   # delete 0->1 splits the 3-cycle
    r = golden["example_rev/s2/sym_beg"], golden["example_rev/s2/sym_adj"]
    assert 1 in r[1][r[0][0]:r[0][1]]                     # {0,1} survives while 1->0 exists


def test_edge_weight_restatement(orc):
    rng = np.random.default_rng(0)
    for u, v in rng.integers(0, 2**31 - 1, size=(200, 2)):
        w = orc.edge_weight(int(u), int(v))
        assert 1 <= w <= 100
    if orc.ref_available():
        for u, v in rng.integers(0, 2**31 - 1, size=(200, 2)):
            assert orc.edge_weight(int(u), int(v)) == orc.ref().ref_edge_weight(int(u), int(v))


def test_loader_error_codes(orc, tmp_path):
    """graph.cpp:95-114 checks, as error codes: malformed offsets, ids out of range, fw/bw sizes."""
    d = str(tmp_path) + "/"
    def write(fb, fa, bb, ba):
        for name, a in (("fw_begin", fb), ("fw_adjacent", fa), ("bw_begin", bb), ("bw_adjacent", ba)):
            np.asarray(a, np.int32).tofile(d + name + ".bin")
    def load():
        V, E, Vb, Eb = (orc.ctypes.c_int64() for _ in range(4))
        rc = orc.lib().or_file_sizes(d.encode(), *(orc.ctypes.byref(x) for x in (V, E, Vb, Eb)))
        if rc:
            return rc
        arrs = [np.zeros(max(n, 1), np.int32) for n in (V.value + 1, E.value, V.value + 1, E.value)]
        return orc.lib().or_load(d.encode(), V.value, E.value, *[orc.ptr(a) for a in arrs])
    write([0, 1, 2], [1, 0], [0, 1, 2], [1, 0])
    assert load() == 0
    write([0, 2, 1], [1, 0], [0, 1, 2], [1, 0])
    assert load() == 3  # forward offsets decrease
    write([0, 1, 2], [1, 5], [0, 1, 2], [1, 0])
    assert load() == 3  # id out of range
    write([0, 1, 2], [1, 0], [0, 1, 2], [1, 7])
    assert load() == 4  # backward id out of range
    write([0, 1, 2], [1, 0], [0, 1, 1, 2], [1, 0])
    assert load() == 2  # bw has another V


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref",
                                                    "libgirref.so")), reason="reference not compiled here")
def test_oracle_matches_reference_on_rmat(orc, pkg):
    g = pkg.graphs.rmat(12, seed=11, weights=None)
    fb, fa = orc.normalize(g.V, g.fw_beg, g.fw_adj)
    L = orc.Layers(g.V, fb, fa)
    r = orc.RefGIR(g.V, g.fw_beg, g.fw_adj, g.bw_beg, g.bw_adj)
    r.build(7)
    np.testing.assert_array_equal(L.wcc, r.wcc())
    np.testing.assert_array_equal(L.scc, r.scc())
    np.testing.assert_array_equal(L.dag, r.dag())
    np.testing.assert_array_equal(L.blocks, r.blocks())
    np.testing.assert_array_equal(L.ap, r.ap())
    for s in (0, 17, 1234):
        np.testing.assert_array_equal(orc.bfs(g.V, fb, fa, [s]), r.bfs(s))
        np.testing.assert_array_equal(orc.sssp(g.V, fb, fa, [s]), r.sssp(s))
    u, v, ins = pkg.graphs.updates(g, 500, 500, 2)
    r.apply_batch(u, v, ins)
    fb2, fa2, _, _ = orc.apply_batch(g.V, fb, fa, u, v, ins)
    rb, ra = r.out_csr()
    np.testing.assert_array_equal(fb2, rb)
    np.testing.assert_array_equal(fa2, ra)
    L2 = orc.Layers(g.V, fb2, fa2)
    np.testing.assert_array_equal(L2.scc, r.scc())
    np.testing.assert_array_equal(L2.wcc, r.wcc())
    np.testing.assert_array_equal(L2.blocks, r.blocks())
    r.close()


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref",
                                                    "libgirref.so")), reason="reference not compiled here")
def test_reference_incremental_matches_oracle(orc, pkg):
    """Pins the incremental checker: the reference's own updateIncremental (gir_query.cpp:894-996)
    equals the oracle's from-scratch BFS / SSSP after every batch of its IncTest pattern
    (gir_test.cpp:1043-1083: mostly deletions of existing edges)."""
    g = pkg.graphs.rmat(12, seed=7, weights=None)
    fb, fa = orc.normalize(g.V, g.fw_beg, g.fw_adj)
    r = orc.RefGIR(g.V, fb.astype(np.int32), fa, *orc.transpose(g.V, fb, fa))
    r.build(7)
    rng = np.random.default_rng(3)
    src = int(np.argmax(np.diff(fb)))
    r.inc_track(src, False)
    r.inc_track(src, True)
    none = np.uint64(2**64 - 1)
    for _ in range(20):
        beg, adj = r.out_csr()
        a = rng.integers(0, g.V, 300)
        a = a[beg[a + 1] > beg[a]]
        b = adj[beg[a] + rng.integers(0, 1 << 30, len(a)) % (beg[a + 1] - beg[a])]
        u = np.concatenate([a, rng.integers(0, g.V, 100)]).astype(np.int32)
        v = np.concatenate([b, rng.integers(0, g.V, 100)]).astype(np.int32)
        ins = np.concatenate([np.zeros(len(a)), np.ones(100)]).astype(np.uint8)
        r.apply_batch(u, v, ins)
        r.inc_update(False)
        r.inc_update(True)
        beg, adj = r.out_csr()
        lv = orc.bfs(g.V, beg, adj, [src])
        np.testing.assert_array_equal(r.inc_dist(False), np.where(lv < 0, none, lv.astype(np.uint64)))
        np.testing.assert_array_equal(r.inc_dist(True), orc.sssp(g.V, beg, adj, [src]))
    r.close()


def test_reference_ingest_defers_layers_until_sync(orc, pkg):
    """Pins the checker of the deferred-maintenance test: the reference's own ingestBatch leaves its
    layer getters at the last sync, and sync() brings them to the oracle's answer for the new
    graph."""
    if not orc.ref_available():
        import pytest
        pytest.skip("the reference library is not built")
    g = pkg.graphs.rmat(11, seed=4, weights=None)
    fb, fa = orc.normalize(g.V, g.fw_beg, g.fw_adj)
    r = orc.RefGIR(g.V, g.fw_beg, g.fw_adj, g.bw_beg, g.bw_adj)
    r.build(7)
    scc0 = r.scc()
    u, v, ins = pkg.graphs.updates(g, 300, 600, 8)
    r.ingest_batch(u, v, ins)
    assert not r.synced()
    np.testing.assert_array_equal(r.scc(), scc0)
    r.sync()
    fb2, fa2, _, _ = orc.apply_batch(g.V, fb, fa, u, v, ins)
    L2 = orc.Layers(g.V, fb2, fa2)
    np.testing.assert_array_equal(r.scc(), L2.scc)
    np.testing.assert_array_equal(r.wcc(), L2.wcc)
    np.testing.assert_array_equal(r.blocks(), L2.blocks)
    r.close()
