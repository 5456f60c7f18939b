"""Parity at the full configuration size (4.8M vertices / 69M edges).

test_full_size_certificates: the device results pass the size-independent certificates of
verify.py -- BFS levels and SSSP distances of all 64 lanes (every edge relaxed, every reached
vertex with a tight in-edge), WCC labels equal to an independent recomputation, SCC classes
strongly connected with every cross edge forward in rank and the condensation keys exactly the
cross-edge class pairs, the block-cut forest's necessary conditions -- after the build and after a
1M-edge batch.

test_full_size_parity_against_reference: every layer, BFS and SSSP rows compared with the
reference itself (compiled from its sources) on the same graph and batch."""
import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_full_size_certificates(pkg):
    vf = importlib.import_module("graph-intermedia-representation_b200.verify")
    n = pkg.native
    g = pkg.graphs.rmat_lj()
    d = pkg.DeviceGraph.from_graph(g)
    d.build(n.LAYER_ALL)
    for step in range(2):
        fb, fa = d.csr(0)
        src = pkg.graphs.sources_with_edges(pkg.graphs.Graph(g.V, fb.astype(np.int32), fa, None, None), 64, 7 + step)
        lv = torch.empty((64, g.V), dtype=torch.int32, device="cuda")
        ds = torch.empty((64, g.V), dtype=torch.int64, device="cuda")
        d.bfs(torch.from_numpy(src).cuda(), out=lv)
        d.sssp(torch.from_numpy(src).cuda(), delta=16, out=ds)
        fb_d, fa_d = torch.from_numpy(fb).cuda(), torch.from_numpy(fa).cuda()
        for lane in range(64):
            assert vf.bfs_levels(fb_d, fa_d, [src[lane]], lv[lane]) == 0, (step, lane)
            assert vf.sssp_dists(fb_d, fa_d, [src[lane]], ds[lane]) == 0, (step, lane)
        assert vf.wcc_labels(fb_d, fa_d, d.labels(n.LABEL_WCC)) == 0, step
        s, t = d.dag()
        scc = d.labels(n.LABEL_SCC)
        assert vf.scc_dag(fb_d, fa_d, scc, d.labels(n.LABEL_SCC_RANK), s, t) == 0, step
        sb, sa = d.csr(2)
        label, head = d.blocks()
        assert vf.blocks(torch.from_numpy(sb).cuda(), torch.from_numpy(sa).cuda(), scc, label, head,
                         d.labels(n.LABEL_BCNT)) == 0, step
        gg = pkg.graphs.Graph(g.V, fb.astype(np.int32), fa, None, None)
        u, v, ins = pkg.graphs.updates(gg, 500_000, 500_000, 31)
        d.apply_batch(u, v, ins)
    d.close()


def _layers_equal(pkg, orc, d, ref, step):
    n = pkg.native
    np.testing.assert_array_equal(d.labels(n.LABEL_WCC), ref.wcc(), err_msg=f"{step}: WCC")
    np.testing.assert_array_equal(d.labels(n.LABEL_SCC), ref.scc(), err_msg=f"{step}: SCC")
    s, t = d.dag()
    keys = np.unique((s.astype(np.int64) << 32) | t.astype(np.int64))
    np.testing.assert_array_equal(keys, ref.dag(), err_msg=f"{step}: condensation DAG")
    label, head = d.blocks()
    np.testing.assert_array_equal(orc.canon_blocks_from_device(label, head), ref.blocks(), err_msg=f"{step}: blocks")
    np.testing.assert_array_equal(d.labels(n.LABEL_BCNT) >= 2, ref.ap(), err_msg=f"{step}: articulation points")


def test_full_size_parity_against_reference(pkg, orc):
    """The 4.8M-vertex / 69M-edge R-MAT (seed 3, ids permuted) in the device library and in the
    reference compiled from its own sources: canonical WCC, SCC, condensation-DAG key set, blocks
    and articulation points after the build and again after one 1M-edge batch (500K inserts,
    500K deletions of existing edges), plus BFS levels and SSSP distances (delta 16, the
    reference's hash weights) from 4 sources each, all bit-exact."""
    if not orc.ref_available():
        pytest.skip("the reference library oracle/_ref/libgirref.so is not built")
    n = pkg.native
    g = pkg.graphs.rmat_lj()
    ref = orc.RefGIR(g.V, g.fw_beg, g.fw_adj, g.bw_beg, g.bw_adj)
    ref.build(7)
    d = pkg.DeviceGraph.from_graph(g)
    d.build(n.LAYER_ALL)
    for step in ("build", "1M batch"):
        _layers_equal(pkg, orc, d, ref, step)
        fb, fa = d.csr(0)
        src = pkg.graphs.sources_with_edges(pkg.graphs.Graph(g.V, fb.astype(np.int32), fa, None, None), 4, 17)
        lv = d.bfs(src)
        ds = d.sssp(src, delta=16, weights=n.WEIGHT_HASH)
        for i, s in enumerate(src):
            np.testing.assert_array_equal(lv[i], ref.bfs(int(s)), err_msg=f"{step}: BFS from {s}")
            np.testing.assert_array_equal(ds[i], ref.sssp(int(s), 16), err_msg=f"{step}: SSSP from {s}")
        if step == "build":
            gg = pkg.graphs.Graph(g.V, fb.astype(np.int32), fa, None, None)
            u, v, ins = pkg.graphs.updates(gg, 500_000, 500_000, 31)
            d.apply_batch(u, v, ins)
            ref.apply_batch(u, v, ins)
            rb, ra = ref.out_csr()
            fb2, fa2 = d.csr(0)
            np.testing.assert_array_equal(fb2, rb, err_msg="edge store offsets after the batch")
            np.testing.assert_array_equal(fa2, ra, err_msg="edge store after the batch")
    ref.close()
    d.close()
