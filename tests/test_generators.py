"""Synthetic workload generators: deterministic, well-formed four-file CSR. CPU only."""
import numpy as np


def _well_formed(g):
    assert g.fw_beg[0] == 0 and g.fw_beg[-1] == len(g.fw_adj)
    assert np.all(np.diff(g.fw_beg) >= 0) and np.all(np.diff(g.bw_beg) >= 0)
    assert g.fw_adj.min(initial=0) >= 0 and g.fw_adj.max(initial=0) < g.V
    # bw is the transpose of fw
    rows = np.repeat(np.arange(g.V), np.diff(g.fw_beg))
    fw = np.sort(rows.astype(np.int64) << 32 | g.fw_adj)
    rows_b = np.repeat(np.arange(g.V), np.diff(g.bw_beg))
    bw = np.sort(g.bw_adj.astype(np.int64) << 32 | rows_b)
    np.testing.assert_array_equal(fw, bw)


def test_rmat_s16_shape(pkg):
    g = pkg.graphs.rmat_s16()
    assert g.V == 65536
    assert 900_000 < g.E < 1_048_576  # self-loops and duplicates dropped from 2^20 draws
    _well_formed(g)
    rows = np.repeat(np.arange(g.V), np.diff(g.fw_beg))
    assert not np.any(rows == g.fw_adj)  # no self-loops
    assert g.w.min() >= 1 and g.w.max() <= 255
    g2 = pkg.graphs.rmat_s16()
    np.testing.assert_array_equal(g.fw_adj, g2.fw_adj)
    np.testing.assert_array_equal(g.w, g2.w)


def test_rmat_target_count_and_permutation(pkg):
    g = pkg.graphs.rmat(14, V=12000, n_draws=0, target_unique=100_000, seed=3, permute=True)
    assert g.E == 100_000 and g.V == 12000
    _well_formed(g)


def test_lattice_small(pkg):
    g = pkg.graphs.lattice(side=60, seed=4)
    _well_formed(g)
    # symmetric with equal weights both ways
    rows = np.repeat(np.arange(g.V), np.diff(g.fw_beg))
    k = rows.astype(np.int64) << 32 | g.fw_adj
    kt = g.fw_adj.astype(np.int64) << 32 | rows
    order = np.argsort(k)
    ordert = np.argsort(kt)
    np.testing.assert_array_equal(k[order], kt[ordert])
    np.testing.assert_array_equal(g.w[order], g.w[ordert])
    assert g.E < 2 * 2 * 60 * 59 * 1.01


def test_updates_batch(pkg):
    g = pkg.graphs.rmat(10, seed=2)
    u, v, ins = pkg.graphs.updates(g, 300, 200, 5)
    assert len(u) == 500 and ins.sum() == 300
    d = ins == 0
    # deletions are existing edges
    rows = np.repeat(np.arange(g.V), np.diff(g.fw_beg))
    keys = set((rows.astype(np.int64) << 32 | g.fw_adj).tolist())
    assert all(((int(a) << 32) | int(b)) in keys for a, b in zip(u[d], v[d]))
    assert np.all(u[~d] != v[~d])


def test_four_files_roundtrip(pkg, orc, tmp_path):
    g = pkg.graphs.rmat(8, seed=9)
    d = str(tmp_path) + "/"
    pkg.graphs.write_four_files(g, d)
    np.testing.assert_array_equal(np.fromfile(d + "fw_adjacent.bin", np.int32), g.fw_adj)
    np.testing.assert_array_equal(np.fromfile(d + "bw_begin.bin", np.int32), g.bw_beg)
