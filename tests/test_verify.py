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
