"""GPU parity: edge store, WCC, BFS and SSSP through the C ABI against the golden vectors made
by the reference and against the oracle restatement. Bit-exact (integer work)."""
import numpy as np
import pytest

from conftest import golden_cases

pytestmark = pytest.mark.gpu


def _dev(pkg, golden, case, weights=None):
    V = int(golden[f"{case}/V"][0])
    return pkg.DeviceGraph.create(golden[f"{case}/in_fw_beg"], golden[f"{case}/in_fw_adj"],
                                  golden[f"{case}/in_bw_beg"], golden[f"{case}/in_bw_adj"], V, weights)


def _check_store(d, golden, key):
    fb, fa = d.csr(0)
    np.testing.assert_array_equal(fb, golden[f"{key}/fw_beg"], err_msg=key)
    np.testing.assert_array_equal(fa, golden[f"{key}/fw_adj"], err_msg=key)
    sb, sa = d.csr(2)
    np.testing.assert_array_equal(sb, golden[f"{key}/sym_beg"], err_msg=key)
    np.testing.assert_array_equal(sa, golden[f"{key}/sym_adj"], err_msg=key)


def _check_queries(d, golden, case, key):
    src = golden[f"{case}/sources"]
    np.testing.assert_array_equal(d.bfs(src), golden[f"{key}/bfs"], err_msg=f"{key} bfs")
    for delta in (1, 16, 1000):
        np.testing.assert_array_equal(d.sssp(src, delta=delta), golden[f"{key}/sssp"], err_msg=f"{key} sssp {delta}")


def test_golden_store_wcc_and_queries_after_every_step(pkg, golden):
    for case in golden_cases(golden):
        d = _dev(pkg, golden, case)
        d.build(pkg.native.LAYER_WCC)
        _check_store(d, golden, f"{case}/s0")
        np.testing.assert_array_equal(d.labels(pkg.native.LABEL_WCC), golden[f"{case}/s0/wcc"])
        _check_queries(d, golden, case, f"{case}/s0")
        for k in range(1, int(golden[f"{case}/steps"][0]) + 1):
            key = f"{case}/s{k}"
            d.apply_batch(golden[f"{key}/ops_u"], golden[f"{key}/ops_v"], golden[f"{key}/ops_ins"])
            _check_store(d, golden, key)
            np.testing.assert_array_equal(d.labels(pkg.native.LABEL_WCC), golden[f"{key}/wcc"], err_msg=key)
            _check_queries(d, golden, case, key)
        d.close()


def test_four_file_loader_matches(pkg, golden, tmp_path):
    case = "example"
    dd = str(tmp_path) + "/"
    for name in ("fw_beg", "fw_adj", "bw_beg", "bw_adj"):
        fname = {"fw_beg": "fw_begin", "fw_adj": "fw_adjacent", "bw_beg": "bw_begin", "bw_adj": "bw_adjacent"}[name]
        golden[f"{case}/in_{name}"].astype(np.int32).tofile(dd + fname + ".bin")
    d = pkg.DeviceGraph.load(dd)
    assert d.V == 18 and d.E == 26
    _check_store(d, golden, f"{case}/s0")
    d.close()


def test_malformed_inputs_rejected(pkg):
    fb = np.array([0, 2, 1], np.int32)  # offsets decrease
    fa = np.array([1, 0], np.int32)
    with pytest.raises(pkg.GirError) as e:
        pkg.DeviceGraph.create(fb, fa, np.array([0, 1, 2], np.int32), fa, 2)
    assert e.value.code == 5
    with pytest.raises(pkg.GirError):
        pkg.DeviceGraph.create(np.array([0, 1, 2], np.int32), np.array([1, 9], np.int32),
                               np.array([0, 1, 2], np.int32), np.array([1, 0], np.int32), 2)
    # fw and bw disagree after de-duplication (gir.cpp:122-126)
    with pytest.raises(pkg.GirError) as e:
        pkg.DeviceGraph.create(np.array([0, 2, 2], np.int32), np.array([1, 1], np.int32),
                               np.array([0, 0, 2], np.int32), np.array([0, 1], np.int32), 2)
    assert e.value.code == 5


def test_unsorted_rows_and_duplicates_normalised(pkg, orc):
    rng = np.random.default_rng(3)
    V = 300
    src = rng.integers(0, V, 3000).astype(np.int32)
    dst = rng.integers(0, V, 3000).astype(np.int32)  # duplicates and self-loops included
    order = np.argsort(src, kind="stable")
    src, dst = src[order], dst[order]
    fb = np.zeros(V + 1, np.int32)
    np.add.at(fb, src + 1, 1)
    fb = np.cumsum(fb).astype(np.int32)
    o2 = np.argsort(dst, kind="stable")
    bb = np.zeros(V + 1, np.int32)
    np.add.at(bb, dst + 1, 1)
    bb = np.cumsum(bb).astype(np.int32)
    d = pkg.DeviceGraph.create(fb, dst, bb, src[o2], V)
    eb, ea = orc.normalize(V, fb, dst)
    gb, ga = d.csr(0)
    np.testing.assert_array_equal(gb, eb)
    np.testing.assert_array_equal(ga, ea)
    d.close()


def test_empty_graph_and_bad_sources(pkg):
    V = 10
    z = np.zeros(V + 1, np.int32)
    d = pkg.DeviceGraph.create(z, np.zeros(0, np.int32), z, np.zeros(0, np.int32), V)
    d.build(pkg.native.LAYER_WCC)
    np.testing.assert_array_equal(d.labels(pkg.native.LABEL_WCC), np.arange(V))
    lv = d.bfs([3, -1, 10])
    assert lv[0, 3] == 0 and (lv[0] == -1).sum() == V - 1
    assert np.all(lv[1] == -1) and np.all(lv[2] == -1)  # out-of-range source: all -1 (gir_query.cpp:112)
    ds = d.sssp([3, 99])
    assert ds[0, 3] == 0 and np.all(ds[1] == np.iinfo(np.uint64).max)
    d.close()


@pytest.fixture(scope="module")
def s16(pkg, orc):
    g = pkg.graphs.rmat_s16()
    fb, fa = orc.normalize(g.V, g.fw_beg, g.fw_adj)
    return g, fb, fa


def test_rmat_s16_bfs_64_sources(pkg, orc, s16):
    g, fb, fa = s16
    d = pkg.DeviceGraph.from_graph(g)
    src = pkg.graphs.sources(g.V, 64, 1)
    lv = d.bfs(src)
    st = d.query_stats()
    exp_edges = 0
    for i, s in enumerate(src):
        e = orc.bfs(g.V, fb, fa, [s])
        np.testing.assert_array_equal(lv[i], e, err_msg=f"source {s}")
        exp_edges += int(np.diff(fb)[e >= 0].sum())
    assert st["edges"] == exp_edges
    d.close()


def test_rmat_s16_bfs_both_directions_forced(pkg, orc, s16):
    """Same levels whatever the direction schedule: all top-down, all bottom-up, mixed."""
    g, fb, fa = s16
    d = pkg.DeviceGraph.from_graph(g)
    src = pkg.graphs.sources(g.V, 7, 5)
    exp = np.stack([orc.bfs(g.V, fb, fa, [s]) for s in src])
    for alpha, beta in ((1e-9, 1e9), (1e9, 1e-9), (15, 18), (1, 2)):
        d.set_param(pkg.native.PARAM_ALPHA, alpha)
        d.set_param(pkg.native.PARAM_BETA, beta)
        np.testing.assert_array_equal(d.bfs(src), exp, err_msg=f"alpha={alpha} beta={beta}")
    for small, large in ((1, 2), (1000000, 2000000), (4, 64)):
        d.set_param(pkg.native.PARAM_SMALL_DEG, small)
        d.set_param(pkg.native.PARAM_LARGE_DEG, large)
        d.set_param(pkg.native.PARAM_ALPHA, 1e9)
        np.testing.assert_array_equal(d.bfs(src), exp, err_msg=f"bins {small}/{large}")
    d.close()


def test_rmat_s16_multi_source_sets(pkg, orc, s16):
    g, fb, fa = s16
    d = pkg.DeviceGraph.from_graph(g)
    rng = np.random.default_rng(9)
    sets = [rng.integers(0, g.V, int(k)).astype(np.int32) for k in (1, 3, 17, 200, 4096)] + [np.array([], np.int32)]
    lv = d.bfs_sets(sets)
    for i, s in enumerate(sets):
        np.testing.assert_array_equal(lv[i], orc.bfs(g.V, fb, fa, s), err_msg=f"set {i}")
    ds = d.sssp_sets(sets[:3], weights=pkg.native.WEIGHT_STORED)
    for i, s in enumerate(sets[:3]):
        np.testing.assert_array_equal(ds[i], orc.sssp(g.V, fb, fa, s, w=_weights_sorted(g, orc)), err_msg=f"sssp set {i}")
    d.close()


def _weights_sorted(g, orc):
    # generator rows are sorted and duplicate-free, so the forward weights already line up
    return g.w


def test_rmat_s16_sssp_hash_and_stored(pkg, orc, s16):
    g, fb, fa = s16
    d = pkg.DeviceGraph.from_graph(g)
    src = pkg.graphs.sources(g.V, 8, 2)
    for delta in (16, 64, 300):
        dh = d.sssp(src, delta=delta, weights=pkg.native.WEIGHT_HASH)
        ds = d.sssp(src, delta=delta, weights=pkg.native.WEIGHT_STORED)
        for i, s in enumerate(src):
            np.testing.assert_array_equal(dh[i], orc.sssp(g.V, fb, fa, [s]), err_msg=f"hash {s} delta {delta}")
            np.testing.assert_array_equal(ds[i], orc.sssp(g.V, fb, fa, [s], w=g.w), err_msg=f"stored {s} {delta}")
    d.close()


def test_rmat_s16_batches_against_oracle(pkg, orc, s16):
    g, fb, fa = s16
    d = pkg.DeviceGraph.from_graph(g)
    d.build(pkg.native.LAYER_WCC)
    for step, (ni, nd) in enumerate(((1000, 0), (0, 1000), (5000, 5000), (1, 1))):
        cur_fb, cur_fa = d.csr(0)
        gg = pkg.graphs.Graph(g.V, cur_fb.astype(np.int32), cur_fa, None, None)
        u, v, ins = pkg.graphs.updates(gg, ni, nd, 100 + step)
        d.apply_batch(u, v, ins)
        fb, fa, n_ins, n_del = orc.apply_batch(g.V, fb, fa, u, v, ins)
        st = d.batch_stats()
        assert (st["inserted"], st["deleted"]) == (n_ins, n_del)
        gb, ga = d.csr(0)
        np.testing.assert_array_equal(gb, fb)
        np.testing.assert_array_equal(ga, fa)
        tb, ta = orc.transpose(g.V, fb, fa)
        gb, ga = d.csr(1)
        np.testing.assert_array_equal(gb, tb)
        np.testing.assert_array_equal(ga, ta)
        sb, sa = orc.sym(g.V, fb, fa, tb, ta)
        gb, ga = d.csr(2)
        np.testing.assert_array_equal(gb, sb)
        np.testing.assert_array_equal(ga, sa)
        np.testing.assert_array_equal(d.labels(pkg.native.LABEL_WCC), orc.wcc(g.V, fb, fa))
        src = pkg.graphs.sources(g.V, 4, step)
        lv = d.bfs(src)
        for i, s in enumerate(src):
            np.testing.assert_array_equal(lv[i], orc.bfs(g.V, fb, fa, [s]))
    d.close()


def test_has_edges(pkg, s16):
    g, fb, fa = s16
    d = pkg.DeviceGraph.from_graph(g)
    rows = np.repeat(np.arange(g.V), np.diff(fb)).astype(np.int32)
    pick = np.arange(0, len(fa), 997)
    assert d.has_edges(rows[pick], fa[pick]).all()
    assert d.has_edges(fa[pick], rows[pick], undirected=True).all()
    assert not d.has_edges([0, -1, g.V], [0, 1, 2]).any()
    d.close()


def test_autotune_keeps_results(pkg, s16):
    g, _, _ = s16
    d = pkg.DeviceGraph.from_graph(g)
    src = pkg.graphs.sources_with_edges(g, 32, 44)
    before = d.bfs(src)
    res = d.autotune(src, reps=1)
    assert res["ctas_per_sm"] in (2, 4, 8) and res["small_deg"] in (8, 32, 128)
    assert res["large_deg"] in (1024, 4096, 32768) and res["bfs_ms"] > 0
    np.testing.assert_array_equal(d.bfs(src), before)
    with pytest.raises(pkg.GirError):
        d.autotune(np.zeros(65, np.int32))
    d.close()


def test_persistent_levels_on_a_lattice(pkg, orc):
    """A high-diameter graph runs most BFS levels inside the persistent top-down launch; levels
    equal the oracle's, with the fixed switch and with the learned schedule, for single sources
    and multi-source sets, and the schedule trace still holds a decision per level."""
    lat = pkg.graphs.lattice(side=300, seed=12)
    fb, fa = orc.normalize(lat.V, lat.fw_beg, lat.fw_adj)
    d = pkg.DeviceGraph.from_graph(lat)
    src = pkg.graphs.sources_with_edges(lat, 64, 5)
    exp = np.stack([orc.bfs(lat.V, fb, fa, [s]) for s in src[:8]])
    for mode in ("fixed", "top-down", "learned"):
        if mode == "top-down":  # a tiny alpha never switches: every level can run persistent
            d.set_param(pkg.native.PARAM_ALPHA, 1e-6)
        if mode == "learned":
            d.set_param(pkg.native.PARAM_ALPHA, 15)
            d.use_learned_schedule()
        lv = d.bfs(src)
        st = d.query_stats()
        assert st["persistent_levels"] > 0, st
        if mode == "top-down":
            assert st["persistent_levels"] > 0.9 * st["iterations"] and st["bottom_up"] <= 2, st
        np.testing.assert_array_equal(lv[:8], exp)
        x, y = d.sched_trace()
        assert len(y) >= st["iterations"] and x.shape[1] == pkg.native.SCHED_IN
        sets = [src[:3], src[3:4], src[4:40]]
        ls = d.bfs_sets(sets)
        for i, s in enumerate(sets):
            np.testing.assert_array_equal(ls[i], orc.bfs(lat.V, fb, fa, list(s)))
    d.close()


def test_betweenness_matches_reference(pkg, orc, s16):
    """Brandes betweenness (GIR::bc) against the reference's own implementation: two graphs, more
    sources than one 64-lane group, repeated and out-of-range sources. Doubles: the sums run in
    another order than the reference's, so the bar is a relative 1e-9."""
    small = pkg.graphs.rmat(12, seed=14, weights=None)
    g, _, _ = s16
    # Rows longer than 4,096 entries are summed in 1,024-entry chunks: vertex 0 points to 6,001
    # vertices, 6,001 vertices point to vertex 1, over a sparse random graph of 3 out-edges each.
    rng = np.random.default_rng(21)
    V = 12_000
    su = np.concatenate([np.repeat(np.arange(V, dtype=np.int64), 3), np.zeros(6001, np.int64),
                         np.arange(2, 6003)])
    sv = np.concatenate([rng.integers(0, V, 3 * V), np.arange(V - 6001, V), np.ones(6001, np.int64)])
    key = np.unique(su * V + sv)
    hubs = pkg.graphs.from_edges(V, key // V, key % V, name="hubs")
    assert np.diff(hubs.fw_beg).max() > 4096 and np.diff(hubs.bw_beg).max() > 4096
    for gr, n in ((small, 70), (g, 100), (hubs, 80)):
        d = pkg.DeviceGraph.from_graph(gr, weights=False)
        src = np.concatenate([pkg.graphs.sources_with_edges(gr, n, 3), [0, 0, -5, gr.V + 2]]).astype(np.int32)
        got = d.bc(src)
        ref = orc.RefGIR(gr.V, gr.fw_beg, gr.fw_adj, gr.bw_beg, gr.bw_adj)
        exp = ref.bc(src)
        ref.close()
        np.testing.assert_allclose(got, exp, rtol=1e-9, atol=1e-9)
        assert exp.max() > 0
        d.close()


def test_sssp_lane_order_and_groups_map_back_to_query_rows(pkg, orc, s16):
    """70 queries (a group of 64 lanes, then 6) with repeats and an out-of-range source: lanes are
    placed by the sources' distance to the hub, and every lane must land in its own query's row."""
    g, fb, fa = s16
    d = pkg.DeviceGraph.from_graph(g)
    src = pkg.graphs.sources(g.V, 70, 9)
    src[5] = src[40]
    src[66] = g.V + 3
    exp = {0: [orc.sssp(g.V, fb, fa, [s]) for s in src], 1: [orc.sssp(g.V, fb, fa, [s], w=g.w) for s in src]}
    for bits in (0, 16, 32, 64):
        for order in (1, 0):
            d.set_param(pkg.native.PARAM_LANE_BITS, bits)
            d.set_param(pkg.native.PARAM_LANE_ORDER, order)
            for weights in (pkg.native.WEIGHT_HASH, pkg.native.WEIGHT_STORED):
                ds = d.sssp(src, delta=16, weights=weights)
                for i, s in enumerate(src):
                    np.testing.assert_array_equal(ds[i], exp[weights][i],
                                                  err_msg=f"query {i}, source {s}, {bits} bits, order {order}")
    d.close()


def test_sssp_16bit_lane_overflow_reruns_wider(pkg, orc):
    """The distances to the hub are tiny (so 16-bit lane distances are tried first), but a chain of
    20,000-weight edges holds distances far beyond 65,535: the group must be rerun with wider lanes
    and still equal the oracle."""
    V = 200
    es, ed, ew = [], [], []
    for i in range(1, 61):
        es += [i, 0]; ed += [0, i]; ew += [1, 1]
    es.append(0); ed.append(100); ew.append(1)
    for i in range(100, 120):
        es.append(i); ed.append(i + 1); ew.append(20000)
    g = pkg.graphs.from_edges(V, np.array(es), np.array(ed), np.array(ew, np.uint32))
    fb, fa = orc.normalize(g.V, g.fw_beg, g.fw_adj)
    d = pkg.DeviceGraph.from_graph(g)
    d.set_param(pkg.native.PARAM_LANE_BITS, 16)
    src = np.array([1, 100, 5, 0, 150], np.int32)
    for _ in range(2):  # the second call starts from the handle's remembered overflow
        ds = d.sssp(src, delta=16, weights=pkg.native.WEIGHT_STORED)
        for i, s in enumerate(src):
            np.testing.assert_array_equal(ds[i], orc.sssp(g.V, fb, fa, [s], w=g.w), err_msg=f"source {s}")
    assert ds[0, 120] > 65535
    d.close()
