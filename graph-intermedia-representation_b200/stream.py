"""The streaming protocol of the reference's baseline drivers (DZiG's setting; the reference's
experiments/baselines/common/protocol.h and gir_constructor/bench_main.cpp:263-345).

export_protocol writes a protocol directory for a graph, in the reference's file formats:
  loaded.el     half of the graph's distinct non-loop edges, "u v" per line (the initial graph)
  insert.ops    k held-out edges as inserts, "a u v" per line
  delete.ops    k loaded edges as deletions, "d u v" per line
  mixed.ops     k/2 further held-out inserts and k/2 further loaded deletions, shuffled
  sources.txt   query sources (vertices with out-edges); bc_sources.txt  betweenness sources
  meta.txt      V, E, loaded, ops_per_phase, max_weight, symmetric
with k = min(ops_per_stream, half / 2). The split is seeded (numpy), not the reference's
mt19937 shuffle, so the files are of the same kind, not the same draws.

run_driver runs a protocol driver binary -- this package's gir_stream (csrc/gir_stream.cpp, on the
GPU) or the reference's own gir_stream built from its sources -- with the reference's command line
(<dir> <dataset> <csv> <batch> <batches> <mode>) and returns its result rows.
"""
import csv as _csv
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DRIVER = os.path.join(HERE, "gir_stream")


def _write_pairs(path, u, v, prefix=None):
    u = np.asarray(u, np.int64)
    v = np.asarray(v, np.int64)
    with open(path, "w") as f:
        if prefix is None:
            np.savetxt(f, np.column_stack([u, v]), fmt="%d %d")
        else:
            lines = np.char.add(np.char.add(np.char.add(np.asarray(prefix, dtype="U1"), " "),
                                            np.char.add(u.astype("U11"), " ")), v.astype("U11"))
            if len(lines):
                f.write("\n".join(lines.tolist()))
                f.write("\n")


def export_protocol(g, directory, ops_per_stream=10000, n_sources=4, n_bc=4, seed=2027):
    """Writes the protocol files for graph g (a graphs.Graph) into `directory` (created)."""
    os.makedirs(directory, exist_ok=True)
    rows = np.repeat(np.arange(g.V, dtype=np.int64), np.diff(np.asarray(g.fw_beg, np.int64)))
    cols = np.asarray(g.fw_adj, np.int64)
    keys = np.unique((rows << 32) | cols)
    keys = keys[(keys >> 32) != (keys & 0xFFFFFFFF)]  # no self-loops
    rng = np.random.default_rng(seed)
    keys = keys[rng.permutation(len(keys))]
    half = len(keys) // 2
    loaded, held = keys[:half], keys[half:]
    k = min(ops_per_stream, half // 2)
    uv = lambda a: (a >> 32, a & 0xFFFFFFFF)  # noqa: E731
    _write_pairs(os.path.join(directory, "loaded.el"), *uv(loaded))
    ins = held[:k]
    dele = loaded[:k]
    mix_i = held[k:k + k // 2]
    mix_d = loaded[k:k + k // 2]
    _write_pairs(os.path.join(directory, "insert.ops"), *uv(ins), prefix=np.full(len(ins), "a"))
    _write_pairs(os.path.join(directory, "delete.ops"), *uv(dele), prefix=np.full(len(dele), "d"))
    mk = np.concatenate([mix_i, mix_d])
    tag = np.concatenate([np.full(len(mix_i), "a"), np.full(len(mix_d), "d")])
    perm = rng.permutation(len(mk))
    _write_pairs(os.path.join(directory, "mixed.ops"), *uv(mk[perm]), prefix=tag[perm])
    outdeg = np.bincount((keys >> 32).astype(np.int64), minlength=g.V)
    cand = np.nonzero(outdeg > 0)[0]
    src = cand[rng.integers(0, len(cand), n_sources)] if len(cand) else np.zeros(n_sources, np.int64)
    np.savetxt(os.path.join(directory, "sources.txt"), src, fmt="%d")
    np.savetxt(os.path.join(directory, "bc_sources.txt"), rng.integers(0, g.V, n_bc), fmt="%d")
    with open(os.path.join(directory, "meta.txt"), "w") as f:
        f.write(f"V {g.V}\nE {len(keys)}\nloaded {half}\nops_per_phase {k}\nmax_weight 100\nsymmetric 0\n")
    return {"V": g.V, "E": int(len(keys)), "loaded": int(half), "ops_per_phase": int(k), "sources": src.tolist()}


def run_driver(binary, directory, dataset, csv_path, batch=10000, batches=10, mode="", timeout=1800, env=None):
    """Runs a protocol driver and returns its rows as dicts (metric, mode, value, unit, count, system)."""
    if os.path.exists(csv_path):
        os.remove(csv_path)
    args = [binary, directory, dataset, csv_path, str(batch), str(batches)] + ([mode] if mode else [])
    subprocess.run(args, check=True, capture_output=True, text=True, timeout=timeout, env=env)
    out = []
    with open(csv_path) as f:
        for r in _csv.reader(f):
            if len(r) >= 8:
                out.append({"dataset": r[0], "system": r[1], "metric": r[2], "mode": r[3], "value": float(r[4]),
                            "unit": r[5], "count": int(r[6]), "threads": int(r[7])})
    return out
