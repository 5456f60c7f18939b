"""Parity at the full configuration size (4.8M vertices / 69M edges), where the CPU oracle is
too slow for every query: the device results must pass the size-independent certificates of
verify.py -- BFS levels and SSSP distances (every edge relaxed, every reached vertex with a
tight in-edge), WCC labels constant along edges, every cross-SCC edge a condensation edge going
forward in rank -- after the build and after a 1M-edge batch."""
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
        for lane in (0, 21, 63):
            assert vf.bfs_levels(fb, fa, [src[lane]], lv[lane]) == 0, (step, lane)
            assert vf.sssp_dists(fb, fa, [src[lane]], ds[lane]) == 0, (step, lane)
        assert vf.wcc_labels(fb, fa, d.labels(n.LABEL_WCC)) == 0, step
        s, t = d.dag()
        assert vf.scc_dag(fb, fa, d.labels(n.LABEL_SCC), d.labels(n.LABEL_SCC_RANK), s, t) == 0, step
        gg = pkg.graphs.Graph(g.V, fb.astype(np.int32), fa, None, None)
        u, v, ins = pkg.graphs.updates(gg, 500_000, 500_000, 31)
        d.apply_batch(u, v, ins)
    d.close()
