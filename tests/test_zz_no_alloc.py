"""gir_dev_bfs_noalloc: the BFS entry point for callers that cannot allocate memory at call time
(an engine whose own arena owns the GPU's memory, or a latency-critical thread that cannot take
the device-wide synchronization a cudaMalloc / cudaFree can cause).

Called through the C ABI on a caller-owned CSR in device memory, its levels must equal the
oracle's BFS (oracle/gir_oracle.c, restating GIR::bfs, gir_query.cpp:108-294) and those of
gir_dev_bfs, on two calls in a row: the calls share one static working array, which keeps the
previous call's contents. A source outside [0, V) gives all -1 (gir_query.cpp:112). Malformed
CSRs that lie inside their allocations, and a beg[V] beyond the given adj length, are rejected
with GIR_ERR_MALFORMED before any level runs. This file is collected last."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GIR_ERR_MALFORMED = 5
GIR_ERR_CAPACITY = 8


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _oracle_bfs(orc, beg, adj, V, s):
    out = np.empty(V, np.int32)
    orc.lib().or_bfs(V, orc.ptr(np.ascontiguousarray(beg, np.int64)), orc.ptr(np.ascontiguousarray(adj, np.int32)),
                     orc.ptr(np.array([s], np.int32)), 1, orc.ptr(out))
    return out


def test_noalloc_bfs_matches_oracle_and_bfs_on_two_calls(pkg, orc):
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
        rc = lib.gir_dev_bfs_noalloc(_p(beg_d), _p(adj_d), len(adj), g.V, int(s), _p(out), None)
        assert rc == 0, lib.gir_dev_last_error(None)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        np.testing.assert_array_equal(got, _oracle_bfs(orc, beg, adj, g.V, int(s)), err_msg=f"call {i}: oracle")
        np.testing.assert_array_equal(got, expect[i], err_msg=f"call {i}, source {s}: gir_dev_bfs")
    # a source out of range: every level -1, status 0
    for bad_src in (-1, g.V):
        rc = lib.gir_dev_bfs_noalloc(_p(beg_d), _p(adj_d), len(adj), g.V, bad_src, _p(out), None)
        assert rc == 0, lib.gir_dev_last_error(None)
        torch.cuda.synchronize()
        assert (out.cpu().numpy() == -1).all()
    d.close()


def test_noalloc_bfs_rejects_malformed_csr(pkg):
    import torch

    lib = pkg.native.dev_lib()
    V = 6
    out = torch.zeros(V, dtype=torch.int32, device="cuda:0")
    good_beg = np.array([0, 2, 3, 5, 5, 6, 6], np.int64)
    good_adj = np.array([1, 2, 3, 4, 0, 5], np.int32)
    cases = {
        "beg decreasing": (np.array([0, 2, 1, 5, 5, 6, 6], np.int64), good_adj, len(good_adj)),
        "beg[0] not 0": (np.array([1, 2, 3, 5, 5, 6, 6], np.int64), good_adj, len(good_adj)),
        "id >= V": (good_beg, np.array([1, 2, 3, 4, 0, 6], np.int32), len(good_adj)),
        "negative id": (good_beg, np.array([1, 2, -3, 4, 0, 5], np.int32), len(good_adj)),
        # beg[V] = 6 entries claimed, only 4 given: nothing past entry 4 is read
        "beg[V] beyond n_adj": (good_beg, good_adj, 4),
    }
    for name, (b, a, n_adj) in cases.items():
        b_d = torch.from_numpy(b).to("cuda:0")
        a_d = torch.from_numpy(a).to("cuda:0")
        rc = lib.gir_dev_bfs_noalloc(_p(b_d), _p(a_d), n_adj, V, 0, _p(out), None)
        assert rc == GIR_ERR_MALFORMED, (name, rc, lib.gir_dev_last_error(None))
    # the well-formed graph still runs after the rejections
    b_d = torch.from_numpy(good_beg).to("cuda:0")
    a_d = torch.from_numpy(good_adj).to("cuda:0")
    rc = lib.gir_dev_bfs_noalloc(_p(b_d), _p(a_d), len(good_adj), V, 0, _p(out), None)
    assert rc == 0, lib.gir_dev_last_error(None)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), [0, 1, 1, 2, 2, 3])


def test_noalloc_bfs_rejects_sizes_beyond_its_maximum(pkg):
    import torch

    lib = pkg.native.dev_lib()
    beg = torch.zeros(4, dtype=torch.int64, device="cuda:0")
    adj = torch.zeros(1, dtype=torch.int32, device="cuda:0")
    out = torch.zeros(4, dtype=torch.int32, device="cuda:0")
    rc = lib.gir_dev_bfs_noalloc(_p(beg), _p(adj), 1, (1 << 21) + 1, 0, _p(out), None)
    assert rc == GIR_ERR_CAPACITY
    assert b"GIR_NOALLOC_MAX_V" in lib.gir_dev_last_error(None)


def test_noalloc_bfs_rejects_host_memory(pkg):
    import torch

    lib = pkg.native.dev_lib()
    beg = torch.zeros(4, dtype=torch.int64)
    adj = torch.zeros(1, dtype=torch.int32)
    out = torch.zeros(3, dtype=torch.int32, device="cuda:0")
    rc = lib.gir_dev_bfs_noalloc(_p(beg), _p(adj), 1, 3, 0, _p(out), None)
    assert rc == 1  # GIR_ERR_INVALID
