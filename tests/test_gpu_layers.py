"""GPU parity of the structural layers (buildWCC / buildSCC_DAG / buildBCT and their upkeep under
updates) through the C ABI: canonical WCC and SCC partitions, condensation-DAG edge sets, blocks
and articulation points, bit-exact against the reference's golden vectors after every update
step and against the oracle on R-MAT graphs."""
import numpy as np
import pytest

from conftest import golden_cases

pytestmark = pytest.mark.gpu


def _layers(pkg, orc, d):
    n = pkg.native
    scc = d.labels(n.LABEL_SCC)
    src, dst = d.dag()
    dag = (src.astype(np.int64) << 32) | dst.astype(np.int64)
    label, head = d.blocks()
    blocks = orc.canon_blocks_from_device(label, head)
    ap = d.labels(n.LABEL_BCNT) >= 2
    return d.labels(n.LABEL_WCC), scc, dag, blocks, ap


def _check_ranks(pkg, d):
    scc = d.labels(pkg.native.LABEL_SCC)
    rank = d.labels(pkg.native.LABEL_SCC_RANK)
    src, dst = d.dag()
    # rank is per SCC and respects every condensation edge (gir.h:54-57)
    assert np.all(rank == rank[scc])
    assert np.all(rank[src] < rank[dst])
    reps = np.nonzero(scc == np.arange(len(scc)))[0]
    assert len(np.unique(rank[reps])) == len(reps)


def _check_block_invariants(pkg, d):
    """checkBlockForestInvariants (gir.cpp:4159-4211), in this representation: every block has
    at least one vertex whose parent block it is, heads of non-root blocks are APs, and the
    count array matches the memberships."""
    label, head = d.blocks()
    bcnt = d.labels(pkg.native.LABEL_BCNT)
    V = len(label)
    assert label.min(initial=0) >= 0 and (V == 0 or label.max() < len(head))
    counts = np.bincount(label, minlength=len(head))
    assert np.all(counts >= 1)
    exp = np.ones(V, np.int64)
    np.add.at(exp, head[head >= 0], 1)
    np.testing.assert_array_equal(bcnt, exp)
    assert np.all(bcnt[head[head >= 0]] >= 2)


def _match(pkg, orc, d, golden, key):
    wcc, scc, dag, blocks, ap = _layers(pkg, orc, d)
    np.testing.assert_array_equal(wcc, golden[f"{key}/wcc"], err_msg=f"{key} wcc")
    np.testing.assert_array_equal(scc, golden[f"{key}/scc"], err_msg=f"{key} scc")
    np.testing.assert_array_equal(dag, golden[f"{key}/dag"], err_msg=f"{key} dag")
    np.testing.assert_array_equal(blocks, golden[f"{key}/blocks"], err_msg=f"{key} blocks")
    np.testing.assert_array_equal(ap, golden[f"{key}/ap"], err_msg=f"{key} ap")
    _check_ranks(pkg, d)
    _check_block_invariants(pkg, d)


def test_golden_layers_after_every_step(pkg, orc, golden):
    for case in golden_cases(golden):
        V = int(golden[f"{case}/V"][0])
        d = pkg.DeviceGraph.create(golden[f"{case}/in_fw_beg"], golden[f"{case}/in_fw_adj"],
                                   golden[f"{case}/in_bw_beg"], golden[f"{case}/in_bw_adj"], V)
        d.build(pkg.native.LAYER_ALL)
        _match(pkg, orc, d, golden, f"{case}/s0")
        for k in range(1, int(golden[f"{case}/steps"][0]) + 1):
            key = f"{case}/s{k}"
            d.apply_batch(golden[f"{key}/ops_u"], golden[f"{key}/ops_v"], golden[f"{key}/ops_ins"])
            _match(pkg, orc, d, golden, key)
        d.close()


def test_call_order_enforced(pkg, golden):
    case = "example"
    d = pkg.DeviceGraph.create(golden[f"{case}/in_fw_beg"], golden[f"{case}/in_fw_adj"],
                               golden[f"{case}/in_bw_beg"], golden[f"{case}/in_bw_adj"], 18)
    with pytest.raises(pkg.GirError) as e:
        d.build(pkg.native.LAYER_BCT)
    assert e.value.code == 6
    with pytest.raises(pkg.GirError):
        d.labels(pkg.native.LABEL_SCC)
    d.close()


def test_gir_class_surface(pkg, golden):
    """The reference surface (getNodeToScc, getDAG, getBCTComponents, ...) on the example graph."""
    case = "example"
    g = pkg.graphs.Graph(18, golden[f"{case}/in_fw_beg"], golden[f"{case}/in_fw_adj"],
                         golden[f"{case}/in_bw_beg"], golden[f"{case}/in_bw_adj"])
    G = pkg.GIR(graph=g)
    G.buildWCC(); G.buildSCC_DAG(); G.buildBCT()
    n2s = G.getNodeToScc()
    assert n2s[0] == n2s[9] and n2s[0] != n2s[12]
    wccs_before = len(G.getWCCs())
    G.insertEdge(3, 12)
    assert len(G.getWCCs()) == wccs_before - 1
    G.deleteEdge(3, 12)
    assert len(G.getWCCs()) == wccs_before
    G.updateEdgeUndirected(9, 2, False)  # routes as directed 9->2 (gir.cpp:3134)
    n2s = G.getNodeToScc()
    assert n2s[0] != n2s[9] and n2s[9] == n2s[10] == n2s[11]
    dag = G.getDAG()
    assert any(dag[r] for r in range(18))
    comps = G.getBCTComponents(G.sccOf(0))
    assert sorted(map(sorted, comps)) == sorted(map(sorted, [[0, 1, 2]]))
    assert G.hasDirectedEdge(2, 9) and not G.hasDirectedEdge(9, 2) and G.hasUndirectedEdge(9, 2)
    assert G.bfs(0)[9] == 3  # 0 -> 1 -> 2 -> 9
    assert G.sssp(0)[0] == 0 and G.sssp(0)[1] == G.edgeWeight(0, 1)
    # structure queries (gir.h:131-138, 153)
    assert G.sameScc(0, 1) and not G.sameScc(0, 9) and G.sameWcc(0, 9)
    assert G.biconnected(0, 1) and not G.biconnected(0, 9) and G.biconnected(4, 4)
    assert all(G.reachableNoIndex(0, v) == G.reachable(0, v) for v in range(18))
    assert G.checkBlockForestInvariants()
    assert not any(G.articulationPoint(v) for v in (0, 1, 2))
    # deferred maintenance: the layers wait for sync (gir.h:107-116)
    wccs = len(G.getWCCs())
    G.ingestBatch([(3, 12, True)])
    assert not G.synced() and len(G.getWCCs()) == wccs and G.bfs(3)[12] == 1
    G.sync()
    assert G.synced() and len(G.getWCCs()) == wccs - 1


@pytest.fixture(scope="module")
def s16(pkg, orc):
    g = pkg.graphs.rmat_s16()
    fb, fa = orc.normalize(g.V, g.fw_beg, g.fw_adj)
    return g, fb, fa


def _oracle_match(pkg, orc, d, V, fb, fa, what):
    L = orc.Layers(V, fb, fa)
    wcc, scc, dag, blocks, ap = _layers(pkg, orc, d)
    np.testing.assert_array_equal(wcc, L.wcc, err_msg=f"{what} wcc")
    np.testing.assert_array_equal(scc, L.scc, err_msg=f"{what} scc")
    np.testing.assert_array_equal(dag, L.dag, err_msg=f"{what} dag")
    np.testing.assert_array_equal(blocks, L.blocks, err_msg=f"{what} blocks")
    np.testing.assert_array_equal(ap, L.ap, err_msg=f"{what} ap")
    _check_ranks(pkg, d)
    _check_block_invariants(pkg, d)


def test_rmat_s16_layers_and_batches(pkg, orc, s16):
    g, fb, fa = s16
    d = pkg.DeviceGraph.from_graph(g)
    d.build(pkg.native.LAYER_ALL)
    _oracle_match(pkg, orc, d, g.V, fb, fa, "build")
    for step, (ni, nd) in enumerate(((1000, 0), (0, 1000), (20000, 20000))):
        cb, ca = d.csr(0)
        gg = pkg.graphs.Graph(g.V, cb.astype(np.int32), ca, None, None)
        u, v, ins = pkg.graphs.updates(gg, ni, nd, 200 + step)
        d.apply_batch(u, v, ins)
        fb, fa, _, _ = orc.apply_batch(g.V, fb, fa, u, v, ins)
        _oracle_match(pkg, orc, d, g.V, fb, fa, f"batch {step}")
    d.close()


def test_shapes_high_diameter_and_dense(pkg, orc):
    """A long directed cycle (one SCC, deep BFS tree, no AP), a path of 2-cycles (every inner
    vertex an AP), a lattice (symmetric, many blocks), a dense random graph, and 2-cycles with
    self-loops, some closed and some tied into larger SCCs (trim-2)."""
    cases = []
    n = 3000
    cases.append(("cycle", n, np.arange(n), (np.arange(n) + 1) % n))
    m = 2000
    a = np.arange(m - 1)
    cases.append(("path2", m, np.concatenate([a, a + 1]), np.concatenate([a + 1, a])))
    lat = pkg.graphs.lattice(side=40, seed=8)
    rows = np.repeat(np.arange(lat.V), np.diff(lat.fw_beg))
    cases.append(("lattice", lat.V, rows, lat.fw_adj))
    rng = np.random.default_rng(5)
    cases.append(("dense", 500, rng.integers(0, 500, 20000), rng.integers(0, 500, 20000)))
    # 2-cycles (the trim-2 case): 500 pairs, some closed, others tied to the rest by one-way
    # edges or merged into larger SCCs by random edges, several with self-loops
    p = np.arange(500)
    rs, rt = rng.integers(0, 1000, 350), rng.integers(0, 1000, 350)
    loops = rng.integers(0, 1000, 40)
    ring = np.arange(30)  # pairs 0..30 chained into one SCC of 62 vertices
    cases.append(("pairs", 1000, np.concatenate([2 * p, 2 * p + 1, rs, loops, 2 * ring + 1, [61]]),
                  np.concatenate([2 * p + 1, 2 * p, rt, loops, 2 * ring + 2, [0]])))
    for name, V, s, t in cases:
        s = np.asarray(s, np.int32)
        t = np.asarray(t, np.int32)
        keep = (s != t) | (name == "pairs")
        gg = pkg.graphs.from_edges(V, s[keep], t[keep])
        d = pkg.DeviceGraph.from_graph(gg, weights=False)
        d.build(pkg.native.LAYER_ALL)
        fb, fa = orc.normalize(V, gg.fw_beg, gg.fw_adj)
        _oracle_match(pkg, orc, d, V, fb, fa, name)
        d.close()


def test_batch_repair_plans_match_oracle(pkg, orc, s16):
    """Small batches built to reach each repair decision (layers kept, WCC unioned, DAG-only SCC
    refresh, full rebuilds), checked against the oracle after every batch; every decision the
    batches are built for must be taken at least once."""
    g, fb, fa = s16
    V = g.V
    d = pkg.DeviceGraph.from_graph(g)
    d.build(pkg.native.LAYER_ALL)
    rng = np.random.default_rng(77)
    seen = {"wcc": set(), "scc": set(), "bct": set()}

    def apply(u, v, ins, what):
        nonlocal fb, fa
        u = np.asarray(u, np.int32)
        v = np.asarray(v, np.int32)
        ins = np.asarray(ins, np.uint8)
        d.apply_batch(u, v, ins)
        for k, x in d.batch_plan().items():
            seen[k].add(x)
        fb, fa, _, _ = orc.apply_batch(V, fb, fa, u, v, ins)
        _oracle_match(pkg, orc, d, V, fb, fa, what)

    for step in range(4):
        scc = d.labels(pkg.native.LABEL_SCC)
        rank = d.labels(pkg.native.LABEL_SCC_RANK)
        label, head = d.blocks()
        # inserts inside one block of the giant SCC: every layer kept or WCC-unioned
        big = np.bincount(scc).argmax()
        members = np.nonzero(scc == big)[0]
        blk = label[members]
        b = np.bincount(blk).argmax()
        inb = members[blk == b]
        u, v = rng.choice(inb, 8), rng.choice(inb, 8)
        keep = u != v
        apply(u[keep], v[keep], np.ones(keep.sum()), f"same-block inserts {step}")
        # inserts between SCCs that follow the rank order: labels kept, DAG refreshed
        a, c = rng.integers(0, V, 64), rng.integers(0, V, 64)
        fwd = (scc[a] != scc[c]) & (rank[a] < rank[c])
        apply(a[fwd][:6], c[fwd][:6], np.ones(min(6, fwd.sum())), f"rank-forward inserts {step}")
        # deletions of cross-SCC edges: labels kept, DAG refreshed
        cb, ca = d.csr(0)
        rows = np.repeat(np.arange(V), np.diff(cb))
        cross = np.nonzero(scc[rows] != scc[ca])[0]
        pick = rng.choice(cross, min(6, len(cross)), replace=False)
        apply(rows[pick], ca[pick], np.zeros(len(pick)), f"cross deletions {step}")
        # a random mixed batch (usually rebuilds)
        gg = pkg.graphs.Graph(V, cb.astype(np.int32), ca, None, None)
        u, v, ins = pkg.graphs.updates(gg, 20, 20, 300 + step)
        apply(u, v, ins, f"random batch {step}")
    d.close()
    assert {"kept", "rebuilt"} <= seen["bct"], seen
    assert {"kept", "patched", "rebuilt"} <= seen["scc"], seen
    assert "patched" in seen["wcc"] or "kept" in seen["wcc"], seen


def test_single_edge_checks_match_oracle(pkg, orc):
    """One-op batches (the single-edge latency path, insertEdge / deleteEdge) whose layer decisions
    come from the exact device searches, checked against the oracle after every op: deletions of
    existing edges inside SCCs and anywhere, inserts against the rank order (closing a cycle or
    not) and random inserts, on a dense R-MAT (one big SCC and block) and a sparse one (bridges,
    articulation points, small SCCs). The searches must keep layers many times, split weakly
    connected components in place (the handle's component count follows), and SCCs and blocks
    must still be patched and rebuilt where the searches say so."""
    seen = {"wcc": set(), "scc": set(), "bct": set()}
    checked = kept = wcc_splits = 0
    for ef, n_ops in ((16, 120), (2, 200)):
        g = pkg.graphs.rmat(11, n_draws=ef << 11, seed=40 + ef, weights=None)
        V = g.V
        fb, fa = orc.normalize(V, g.fw_beg, g.fw_adj)
        d = pkg.DeviceGraph.from_graph(g, weights=False)
        d.build(pkg.native.LAYER_ALL)
        rng = np.random.default_rng(ef)
        for i in range(n_ops):
            scc = d.labels(pkg.native.LABEL_SCC)
            rank = d.labels(pkg.native.LABEL_SCC_RANK)
            kind = i % 4
            if kind in (0, 1):  # delete an existing edge (kind 0: one inside an SCC if any)
                rows = np.repeat(np.arange(V), np.diff(fb))
                cand = np.nonzero(scc[rows] == scc[fa])[0] if kind == 0 else np.arange(len(fa))
                if len(cand) == 0:
                    cand = np.arange(len(fa))
                j = int(rng.choice(cand))
                u, v, ins = int(rows[j]), int(fa[j]), 0
            elif kind == 2:  # insert against the rank order
                a, c = rng.integers(0, V, 256), rng.integers(0, V, 256)
                back = np.nonzero((scc[a] != scc[c]) & (rank[a] > rank[c]))[0]
                if len(back) == 0:
                    continue
                u, v, ins = int(a[back[0]]), int(c[back[0]]), 1
            else:
                u, v, ins = int(rng.integers(V)), int(rng.integers(V)), 1
                if u == v:
                    continue
            n_wcc = d.counts()["n_wcc"]
            d.apply_batch(np.array([u], np.int32), np.array([v], np.int32), np.array([ins], np.uint8))
            for k, x in d.batch_plan().items():
                seen[k].add(x)
            assert d.counts()["n_wcc"] == len(np.unique(d.labels(pkg.native.LABEL_WCC)))
            wcc_splits += d.counts()["n_wcc"] > n_wcc
            fb, fa, _, _ = orc.apply_batch(V, fb, fa, [u], [v], [ins])
            _oracle_match(pkg, orc, d, V, fb, fa, f"op {i} ({u} -> {v}, insert {ins}), edge factor {ef}")
            if i % 40 == 39:  # reachability after the condensation DAG was patched in place
                srcs = rng.integers(0, V, 6)
                tgt = rng.integers(0, V, 50).astype(np.int32)
                for s_ in srcs:
                    got = d.reachable(np.full(len(tgt), s_, np.int32), tgt)
                    np.testing.assert_array_equal(got, orc.bfs(V, fb, fa, [int(s_)])[tgt] >= 0)
        st = d.single_stats()
        checked += st["checked"]
        kept += st["kept"]
        d.close()
    assert checked > 100 and kept > 50, (checked, kept)
    assert wcc_splits > 0
    assert {"kept", "patched"} <= seen["wcc"], seen
    assert {"kept", "patched", "rebuilt"} <= seen["scc"], seen
    assert {"kept", "rebuilt"} <= seen["bct"], seen


def test_reachable_matches_reference(pkg, orc, s16):
    """Batched reachability against the reference's own GIR::reachable (compiled from its
    sources) and the oracle's BFS, before and after a batch: random pairs, same-SCC pairs,
    pairs along the DAG, out-of-range ids and u == v."""
    g, fb, fa = s16
    d = pkg.DeviceGraph.from_graph(g)
    d.build(pkg.native.LAYER_WCC | pkg.native.LAYER_SCC)
    rng = np.random.default_rng(9)
    for step in range(2):
        cb, ca = d.csr(0)
        scc = d.labels(pkg.native.LABEL_SCC)
        src, dst = d.dag()
        u = np.concatenate([rng.integers(0, g.V, 3000), src[:500], np.array([0, 5, -1, g.V])]).astype(np.int32)
        v = np.concatenate([rng.integers(0, g.V, 3000), dst[:500], np.array([0, g.V + 3, 2, 1])]).astype(np.int32)
        big = np.bincount(scc).argmax()
        m = np.nonzero(scc == big)[0]
        u = np.concatenate([u, m[:100]]).astype(np.int32)
        v = np.concatenate([v, m[100:200]]).astype(np.int32)
        got = d.reachable(u, v)
        ok = (u >= 0) & (u < g.V) & (v >= 0) & (v < g.V)
        ref = orc.RefGIR(g.V, cb.astype(np.int32), ca, *orc.transpose(g.V, cb, ca))
        ref.build(3)
        exp = np.zeros(len(u), bool)
        exp[ok] = ref.reachable(u[ok], v[ok])
        ref.close()
        np.testing.assert_array_equal(got, exp)
        for i in np.nonzero(ok)[0][:40]:  # a few through the oracle's BFS as well
            assert got[i] == (orc.bfs(g.V, cb, ca, [int(u[i])])[v[i]] >= 0)
        assert got.any() and not got.all()
        gg = pkg.graphs.Graph(g.V, cb.astype(np.int32), ca, None, None)
        bu, bv, bi = pkg.graphs.updates(gg, 3000, 3000, 41)
        d.apply_batch(bu, bv, bi)
    d.close()


def test_ingest_and_sync_match_reference(pkg, orc, s16):
    """GIR::ingestBatch / sync (gir.h:107-116): ingested batches change the edge store at once (BFS
    sees them) while the layer getters keep describing the last sync, like the reference's own
    ingestBatch; sync() repairs every layer for all of them at once; applyBatch and reachability
    sync first."""
    if not orc.ref_available():
        pytest.skip("the reference library oracle/_ref/libgirref.so is not built")
    g, fb, fa = s16
    ref = orc.RefGIR(g.V, g.fw_beg, g.fw_adj, g.bw_beg, g.bw_adj)
    ref.build(7)
    d = pkg.DeviceGraph.from_graph(g)
    d.build(pkg.native.LAYER_ALL)
    before = _layers(pkg, orc, d)
    assert d.synced()
    src = pkg.graphs.sources(g.V, 3, 5)
    for k, (ni, nd) in enumerate(((300, 300), (0, 2000), (1500, 0))):
        cb, ca = d.csr(0)
        u, v, ins = pkg.graphs.updates(pkg.graphs.Graph(g.V, cb.astype(np.int32), ca, None, None), ni, nd, 900 + k)
        d.ingest_batch(u, v, ins)
        ref.ingest_batch(u, v, ins)
        assert not d.synced() and not ref.synced()
        now = _layers(pkg, orc, d)
        for a, b, what in zip(before, now, ("wcc", "scc", "dag", "blocks", "ap")):
            np.testing.assert_array_equal(a, b, err_msg=f"ingest {k}: {what} changed before sync")
        np.testing.assert_array_equal(now[0], ref.wcc(), err_msg=f"ingest {k}: WCC vs the reference before sync")
        np.testing.assert_array_equal(now[1], ref.scc(), err_msg=f"ingest {k}: SCC vs the reference before sync")
        lv = d.bfs(src)
        for i, s in enumerate(src):
            np.testing.assert_array_equal(lv[i], ref.bfs(int(s)), err_msg=f"ingest {k}: BFS sees the store")
    d.sync()
    ref.sync()
    assert d.synced() and ref.synced()
    cb, ca = d.csr(0)
    _oracle_match(pkg, orc, d, g.V, cb, ca, "after sync")
    wcc, scc, dag, blocks, ap = _layers(pkg, orc, d)
    np.testing.assert_array_equal(scc, ref.scc())
    np.testing.assert_array_equal(wcc, ref.wcc())
    np.testing.assert_array_equal(dag, ref.dag())
    np.testing.assert_array_equal(blocks, ref.blocks())
    # reachability and applyBatch sync pending batches first
    cb, ca = d.csr(0)
    u, v, ins = pkg.graphs.updates(pkg.graphs.Graph(g.V, cb.astype(np.int32), ca, None, None), 200, 200, 950)
    d.ingest_batch(u, v, ins)
    d.reachable([0], [1])
    assert d.synced()
    d.ingest_batch(v, u, ins)
    d.apply_batch(u[:10], v[:10], 1 - ins[:10])
    assert d.synced()
    cb, ca = d.csr(0)
    _oracle_match(pkg, orc, d, g.V, cb, ca, "after apply_batch on pending batches")
    ref.close()
    d.close()


def test_single_edge_in_place_edits_keep_the_store_exact(pkg, orc):
    """One-op batches edit the forward, backward and symmetric rows in place (one CTA) while a row
    has room, and fall back to the batch merge when it has none: 14 inserts into one row (its
    slack runs out), deletions, re-inserts, no-ops and invalid ops, on a graph with stored weights.
    After every op the three CSRs equal the oracle's; at the end SSSP over the stored weights
    (new edges take the hash weight, the default weight rule) equals the oracle's Dijkstra."""
    g = pkg.graphs.rmat(10, seed=77)
    V = g.V
    fb, fa = orc.normalize(V, g.fw_beg, g.fw_adj)
    w = {}
    rows = np.repeat(np.arange(V), np.diff(g.fw_beg))
    for r, x, wt in zip(rows, g.fw_adj, g.w):
        w[(int(r), int(x))] = int(wt)
    d = pkg.DeviceGraph.from_graph(g)
    d.build(pkg.native.LAYER_ALL)
    deg = np.diff(fb)
    small = int(np.nonzero(deg == 4)[0][0])  # capacity 8: room for 4 inserts, then the fallback
    rng = np.random.default_rng(3)
    ops = [(small, int(x), 1) for x in rng.choice(V, 14, replace=False) if x != small]
    ops += [(int(rows[j]), int(g.fw_adj[j]), 0) for j in rng.choice(len(g.fw_adj), 10, replace=False)]
    ops += [ops[0], (ops[1][0], ops[1][1], 0), (ops[1][0], ops[1][1], 1), (5, 5, 1), (-1, 3, 1), (3, V, 0)]
    for i, (u, v, ins) in enumerate(ops):
        d.apply_batch(np.array([u], np.int32), np.array([v], np.int32), np.array([ins], np.uint8))
        fb, fa, _, _ = orc.apply_batch(V, fb, fa, [u], [v], [ins])
        if 0 <= u < V and 0 <= v < V and u != v:
            if ins:
                w.setdefault((u, v), orc.edge_weight(u, v))
            else:
                w.pop((u, v), None)
        cb, ca = d.csr(0)
        np.testing.assert_array_equal(cb, fb, err_msg=f"op {i}: fw offsets")
        np.testing.assert_array_equal(ca, fa, err_msg=f"op {i}: fw")
        bb, ba = orc.transpose(V, fb, fa)
        np.testing.assert_array_equal(d.csr(1)[1], ba, err_msg=f"op {i}: bw")
        sb, sa = orc.sym(V, fb, fa, bb, ba)
        np.testing.assert_array_equal(d.csr(2)[1], sa, err_msg=f"op {i}: sym")
    _oracle_match(pkg, orc, d, V, fb, fa, "after the single ops")
    rows = np.repeat(np.arange(V), np.diff(fb))
    wf = np.array([w[(int(r), int(x))] for r, x in zip(rows, fa)], np.uint32)
    src = pkg.graphs.sources(V, 5, 9)
    ds = d.sssp(src, delta=16, weights=pkg.native.WEIGHT_STORED)
    for i, s in enumerate(src):
        np.testing.assert_array_equal(ds[i], orc.sssp(V, fb, fa, [s], w=wf), err_msg=f"stored-weight SSSP from {s}")
    d.close()
