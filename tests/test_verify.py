"""The size-independent result checks (used where the CPU oracle cannot run, at full sizes):
the weight hash equals the oracle's GIR::edgeWeight, and every check passes on the oracle's
exact answers and catches planted mistakes (on the CPU, in copies of those answers)."""
import importlib

import numpy as np
import torch


def _verify():
    return importlib.import_module("graph-intermedia-representation_b200.verify")


def test_edge_weight_matches_oracle(orc):
    rng = np.random.default_rng(3)
    u = rng.integers(0, 2**31 - 1, 2000)
    v = rng.integers(0, 2**31 - 1, 2000)
    got = _verify().edge_weight(torch.from_numpy(u), torch.from_numpy(v)).numpy()
    exp = np.array([orc.edge_weight(int(a), int(b)) for a, b in zip(u, v)])
    np.testing.assert_array_equal(got, exp)


def test_certificates_pass_exact_and_catch_mistakes(pkg, orc):
    vf = _verify()
    g = pkg.graphs.rmat(11, seed=6, weights=None)
    fb, fa = orc.normalize(g.V, g.fw_beg, g.fw_adj)
    src = pkg.graphs.sources_with_edges(pkg.graphs.Graph(g.V, fb.astype(np.int32), fa, None, None), 3, 1)
    lv = orc.bfs(g.V, fb, fa, [src[0]])
    assert vf.bfs_levels(fb, fa, [src[0]], lv, "cpu") == 0
    bad = lv.copy()
    r = np.nonzero(lv > 1)[0][0]
    bad[r] += 1
    assert vf.bfs_levels(fb, fa, [src[0]], bad, "cpu") > 0
    d = orc.sssp(g.V, fb, fa, [src[1]])
    assert vf.sssp_dists(fb, fa, [src[1]], d, "cpu") == 0
    bad = d.copy()
    r = np.nonzero((d > 0) & (d != np.iinfo(np.uint64).max))[0][0]
    bad[r] -= 1
    assert vf.sssp_dists(fb, fa, [src[1]], bad, "cpu") > 0
    L = orc.Layers(g.V, fb, fa)
    assert vf.wcc_labels(fb, fa, L.wcc, "cpu") == 0
    bad = L.wcc.copy()
    bad[np.nonzero(bad != np.arange(g.V))[0][0]] = g.V - 1
    assert vf.wcc_labels(fb, fa, bad, "cpu") > 0
    # ranks: any topological order of the condensation (Kahn on the oracle's DAG edges)
    src_d, dst_d = (L.dag >> 32).astype(np.int64), (L.dag & 0xFFFFFFFF).astype(np.int64)
    indeg = np.bincount(dst_d, minlength=g.V)
    order, stack = [], [x for x in range(g.V) if L.scc[x] == x and indeg[x] == 0]
    adj = {}
    for a, b in zip(src_d, dst_d):
        adj.setdefault(int(a), []).append(int(b))
    while stack:
        x = stack.pop()
        order.append(x)
        for y in adj.get(x, []):
            indeg[y] -= 1
            if indeg[y] == 0:
                stack.append(y)
    rank_of = np.zeros(g.V, np.int64)
    rank_of[order] = np.arange(len(order))
    rank = rank_of[L.scc]
    assert vf.scc_dag(fb, fa, L.scc, rank, src_d, dst_d, "cpu") == 0
    assert vf.scc_dag(fb, fa, L.scc, rank, src_d[1:], dst_d[1:], "cpu") > 0  # a DAG edge missing


def _merge_two_classes(lab, pick):
    """Relabel the class of `pick` to a smaller existing class label: canonical form and label
    constancy along edges may survive, only the partition is wrong."""
    lab = lab.copy()
    roots = np.unique(lab)
    big = lab[pick]
    small = roots[roots < big]
    assert len(small), "need a smaller class"
    lab[lab == big] = small[0]
    return lab


def test_wcc_certificate_catches_over_merge(pkg, orc):
    vf = _verify()
    # two components with no edge between them, plus isolated vertices
    g = pkg.graphs.from_edges(12, np.array([0, 1, 2, 5, 6, 7]), np.array([1, 2, 0, 6, 7, 5]))
    fb, fa = orc.normalize(g.V, g.fw_beg, g.fw_adj)
    L = orc.Layers(g.V, fb, fa)
    assert vf.wcc_labels(fb, fa, L.wcc, "cpu") == 0
    merged = L.wcc.copy()
    merged[[5, 6, 7]] = 0  # labels stay canonical (label <= v, root labels itself), no edge disagrees
    assert vf.wcc_labels(fb, fa, merged, "cpu") > 0
    g2 = pkg.graphs.rmat(11, seed=8, weights=None)
    fb2, fa2 = orc.normalize(g2.V, g2.fw_beg, g2.fw_adj)
    L2 = orc.Layers(g2.V, fb2, fa2)
    assert vf.wcc_labels(fb2, fa2, L2.wcc, "cpu") == 0
    nonroot = np.nonzero(L2.wcc != np.arange(g2.V))[0]
    lonely = np.nonzero((np.bincount(L2.wcc, minlength=g2.V) == 1) & (np.arange(g2.V) > L2.wcc.min()))[0]
    assert len(lonely)
    assert vf.wcc_labels(fb2, fa2, _merge_two_classes(L2.wcc, lonely[-1]), "cpu") > 0
    assert len(nonroot)


def _ranks(L, V):
    src_d, dst_d = (L.dag >> 32).astype(np.int64), (L.dag & 0xFFFFFFFF).astype(np.int64)
    indeg = np.bincount(dst_d, minlength=V)
    order, stack = [], [x for x in range(V) if L.scc[x] == x and indeg[x] == 0]
    adj = {}
    for a, b in zip(src_d, dst_d):
        adj.setdefault(int(a), []).append(int(b))
    while stack:
        x = stack.pop()
        order.append(x)
        for y in adj.get(x, []):
            indeg[y] -= 1
            if indeg[y] == 0:
                stack.append(y)
    rank_of = np.zeros(V, np.int64)
    rank_of[order] = np.arange(len(order))
    return src_d, dst_d, rank_of


def test_scc_certificate_catches_over_merge_and_extra_keys(pkg, orc):
    vf = _verify()
    # cycle {0,1,2} -> edge 2->3 -> cycle {3,4}: one-way connection between two SCCs
    g = pkg.graphs.from_edges(6, np.array([0, 1, 2, 2, 3, 4]), np.array([1, 2, 0, 3, 4, 3]))
    fb, fa = orc.normalize(g.V, g.fw_beg, g.fw_adj)
    L = orc.Layers(g.V, fb, fa)
    src_d, dst_d, rank_of = _ranks(L, g.V)
    rank = rank_of[L.scc]
    assert vf.scc_dag(fb, fa, L.scc, rank, src_d, dst_d, "cpu") == 0
    # {0,1,2} and {3,4} merged into one class: no cross edge is left to break a rank, the DAG
    # loses its key consistently -- only the strong connectivity of the class catches it
    merged = L.scc.copy()
    merged[[3, 4]] = 0
    keep = np.ones(len(src_d), bool)
    keep &= ~((merged[src_d] == merged[dst_d]))
    assert vf.scc_dag(fb, fa, merged, rank_of[merged], src_d[keep], dst_d[keep], "cpu") > 0
    # an extra condensation key that no edge has
    assert vf.scc_dag(fb, fa, L.scc, rank, np.r_[src_d, 5], np.r_[dst_d, 0], "cpu") > 0
    # a key missing
    assert vf.scc_dag(fb, fa, L.scc, rank, src_d[1:], dst_d[1:], "cpu") > 0


def test_block_certificate(pkg, orc):
    vf = _verify()
    g = pkg.graphs.rmat(10, seed=12, weights=None)
    fb, fa = orc.normalize(g.V, g.fw_beg, g.fw_adj)
    bb, ba = orc.transpose(g.V, fb, fa)
    sb, sa = orc.sym(g.V, fb, fa, bb, ba)
    L = orc.Layers(g.V, fb, fa)
    t = L.blocks  # sorted (k1, k2, v) triples
    # the oracle's blocks in the device library's block-cut forest representation
    label, head, bcnt = orc.block_forest(g.V, sb, sa, L.scc)
    assert vf.blocks(sb, sa, L.scc, label, head, bcnt, "cpu") == 0
    np.testing.assert_array_equal(orc.canon_blocks_from_device(label, head), t)
    big = np.bincount(label).argmax()
    members = np.nonzero(label == big)[0]
    assert len(members) >= 3
    bad = label.copy()
    bad[members[1]] = big + 1 if big + 1 < len(head) else big - 1  # a vertex moved to another block
    assert vf.blocks(sb, sa, L.scc, bad, head, bcnt, "cpu") > 0
    badc = bcnt.copy()
    badc[members[0]] += 1  # a block count that does not match the heads
    assert vf.blocks(sb, sa, L.scc, label, head, badc, "cpu") > 0
