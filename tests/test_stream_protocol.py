"""The streaming protocol (the reference's experiments/baselines/gir/gir_stream.cpp, DZiG's
setting): protocol files written by stream.export_protocol, consumed by the reference's own driver
(compiled from its sources, on the CPU) and by this package's gir_stream (on the GPU), in the four
modes -- applyBatch, lazy (ingestBatch + one sync), inc (incremental BFS / SSSP), lazy-inc."""
import importlib
import os

import numpy as np
import pytest

MODES = ("", "lazy", "inc", "lazy-inc")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DRIVER = os.path.join(ROOT, "oracle", "_ref", "gir_stream_ref")


def _stream():
    return importlib.import_module("graph-intermedia-representation_b200.stream")


def _ops(path):
    tags, u, v = [], [], []
    with open(path) as f:
        for line in f:
            a, b, c = line.split()
            tags.append(a)
            u.append(int(b))
            v.append(int(c))
    return np.array(tags), np.array(u, np.int64), np.array(v, np.int64)


@pytest.fixture(scope="module")
def proto(pkg, tmp_path_factory):
    g = pkg.graphs.rmat(12, seed=5, weights=None)
    d = str(tmp_path_factory.mktemp("proto12"))
    info = _stream().export_protocol(g, d, ops_per_stream=2000)
    return g, d, info


def test_exported_protocol_files(proto):
    g, d, info = proto
    el = np.loadtxt(os.path.join(d, "loaded.el"), dtype=np.int64)
    loaded = set(map(tuple, el.tolist()))
    assert len(loaded) == info["loaded"] == info["E"] // 2
    rows = np.repeat(np.arange(g.V), np.diff(g.fw_beg))
    allk = set(zip(rows.tolist(), g.fw_adj.tolist())) - {(x, x) for x in range(g.V)}
    assert loaded <= allk and len(allk) == info["E"]
    t, u, v = _ops(os.path.join(d, "insert.ops"))
    assert (t == "a").all() and len(t) == info["ops_per_phase"]
    assert all((a, b) in allk and (a, b) not in loaded for a, b in zip(u.tolist(), v.tolist()))
    t, u, v = _ops(os.path.join(d, "delete.ops"))
    assert (t == "d").all() and all((a, b) in loaded for a, b in zip(u.tolist(), v.tolist()))
    t, u, v = _ops(os.path.join(d, "mixed.ops"))
    k = info["ops_per_phase"]
    assert (t == "a").sum() == k // 2 and (t == "d").sum() == k // 2
    src = np.loadtxt(os.path.join(d, "sources.txt"), dtype=np.int64, ndmin=1)
    assert (np.diff(g.fw_beg)[src] > 0).all()


@pytest.mark.skipif(not os.path.exists(REF_DRIVER), reason="the reference's driver is not built")
def test_reference_driver_runs_the_exported_protocol(proto, tmp_path):
    """Pins the protocol files: the reference's own driver reads them in every mode, and its
    incremental results equal its from-scratch ones."""
    _, d, _ = proto
    for mode in MODES:
        rows = _stream().run_driver(REF_DRIVER, d, "rmat12", str(tmp_path / "ref.csv"), 500, 4, mode)
        names = {r["metric"] for r in rows}
        for s in ("insert", "delete", "mixed"):
            assert f"{s}_mutation_MEPS" in names and f"sssp_{s}_endtoend_ms" in names
            if "inc" in mode:
                assert [r["value"] for r in rows if r["metric"] == f"inc_mismatch_{s}"] == [0.0]
            if "lazy" in mode:
                assert f"sync_{s}_ms" in names


@pytest.mark.gpu
def test_device_driver_matches_the_reference_protocol(proto, tmp_path):
    """This package's gir_stream on the GPU: the reference's metric rows in every mode, incremental
    results equal to from-scratch ones after every stream."""
    st = _stream()
    _, d, _ = proto
    for mode in MODES:
        rows = st.run_driver(st.DRIVER, d, "rmat12", str(tmp_path / "dev.csv"), 500, 4, mode)
        names = {r["metric"] for r in rows}
        assert all(r["system"].startswith("GIR-B200") for r in rows)
        for s in ("insert", "delete", "mixed"):
            assert f"{s}_mutation_MEPS" in names and f"bfs_{s}_recompute_ms" in names
            assert [r["value"] for r in rows if r["metric"] == f"{s}_mutation_MEPS"][0] > 0
            if "inc" in mode:
                assert [r["value"] for r in rows if r["metric"] == f"inc_mismatch_{s}"] == [0.0]
            if "lazy" in mode:
                assert f"sync_{s}_ms" in names
        if os.path.exists(REF_DRIVER):
            ref = st.run_driver(REF_DRIVER, d, "rmat12", str(tmp_path / "ref.csv"), 500, 4, mode)
            assert names == {r["metric"] for r in ref}


@pytest.mark.gpu
def test_stream_batches_keep_layers_equal_to_the_reference(pkg, orc, proto):
    """The mixed stream's batches through the GIR class (applyBatch, then ingestBatch + sync) and
    through the reference: every layer equal after each batch / sync."""
    if not orc.ref_available():
        pytest.skip("the reference library is not built")
    g, d, _ = proto
    el = np.loadtxt(os.path.join(d, "loaded.el"), dtype=np.int64)
    t, u, v = _ops(os.path.join(d, "mixed.ops"))
    gl = pkg.graphs.from_edges(g.V, el[:, 0], el[:, 1])
    for lazy in (False, True):
        G = pkg.GIR(graph=gl)
        G.buildWCC(); G.buildSCC_DAG(); G.buildBCT()
        ref = orc.RefGIR(g.V, gl.fw_beg, gl.fw_adj, gl.bw_beg, gl.bw_adj)
        ref.build(7)
        for i in range(0, len(t), 500):
            batch = list(zip(u[i:i + 500].tolist(), v[i:i + 500].tolist(), (t[i:i + 500] == "a").tolist()))
            if lazy:
                G.ingestBatch(batch)
                ref.ingest_batch(u[i:i + 500], v[i:i + 500], (t[i:i + 500] == "a").astype(np.uint8))
            else:
                G.applyBatch(batch)
                ref.apply_batch(u[i:i + 500], v[i:i + 500], (t[i:i + 500] == "a").astype(np.uint8))
        if lazy:
            G.sync()
            ref.sync()
        lab = G._d.labels
        np.testing.assert_array_equal(lab(pkg.native.LABEL_SCC), ref.scc())
        np.testing.assert_array_equal(lab(pkg.native.LABEL_WCC), ref.wcc())
        blk, head = G._d.blocks()
        np.testing.assert_array_equal(orc.canon_blocks_from_device(blk, head), ref.blocks())
        ref.close()
