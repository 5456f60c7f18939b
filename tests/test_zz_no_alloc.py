"""gir_dev_bfs_noalloc: the BFS entry point for callers that cannot allocate memory at call time
(an engine whose own arena owns the GPU's memory, or a latency-critical thread that cannot take
the device-wide synchronization a cudaMalloc / cudaFree can cause). Called through the C ABI on a
caller-owned CSR in device memory, its levels must equal those of gir_dev_bfs, on two calls in a
row (the calls share one static working array, which keeps the previous call's contents)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def test_noalloc_bfs_matches_bfs_on_two_calls(pkg):
    import torch

    lib = pkg.native.dev_lib()
    g = pkg.graphs.rmat_s16()
    d = pkg.DeviceGraph.from_graph(g)
    beg, adj = d.csr(0)
    beg_d = torch.from_numpy(beg).to("cuda:0")
    adj_d = torch.from_numpy(adj).to("cuda:0")
    src = pkg.graphs.sources_with_edges(g, 2, 77)
    expect = d.bfs(src)
    out = torch.full((g.V,), 7, dtype=torch.int32, device="cuda:0")
    for i, s in enumerate(src):
        rc = lib.gir_dev_bfs_noalloc(_p(beg_d), _p(adj_d), g.V, int(s), _p(out), None)
        assert rc == 0, lib.gir_dev_last_error(None)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy(), expect[i], err_msg=f"call {i}, source {s}")
    d.close()


def test_noalloc_bfs_rejects_sizes_beyond_its_maximum(pkg):
    import torch

    lib = pkg.native.dev_lib()
    beg = torch.zeros(4, dtype=torch.int64, device="cuda:0")
    adj = torch.zeros(1, dtype=torch.int32, device="cuda:0")
    out = torch.zeros(4, dtype=torch.int32, device="cuda:0")
    rc = lib.gir_dev_bfs_noalloc(_p(beg), _p(adj), (1 << 21) + 1, 0, _p(out), None)
    assert rc == 8  # GIR_ERR_CAPACITY
    assert b"GIR_NOALLOC_MAX_V" in lib.gir_dev_last_error(None)
