"""Generates tests/golden/golden.npz from the reference itself.

Run where the reference sources are (the oracle Makefile compiles them into
oracle/_ref/libgirref.so):
  make -C oracle REF=<checkout>/gir_constructor && python tests/golden/make_golden.py <checkout>
(or set GIR_REFERENCE_DIR=<checkout> instead of the argument).

Cases (the reference's own fixtures and known answers, gir_constructor/gir_test.cpp:704-753
and gir_selftest.cpp:94-233, plus seeded graphs of the self-test's shapes):
  example        data/example_graph (18 vertices, 26 edges) read by the reference's loader;
                 steps: insert 3->12, delete 3->12, delete 9->2 (runTargetedSplitTest)
  example_del01  example graph, delete 0->1 (splits SCC {0,1,2})
  example_rev    example graph, insert 1->0 then delete 0->1 ({0,1} stays undirected)
  bridge300      fromEdges(300, 15<->299, 299<->178, 15<->296), one batch deleting 15<->299
  sparse_60 .. cactus_150   random graphs of the self-test's shapes, each with 6 batches of 25
                 ops (duplicates, cancelling pairs, invalid ops)
  rmat_s10       R-MAT scale 10, 3 batches of 200 ops
For every step the canonical WCC / SCC labels, condensation edges, blocks, articulation points,
BFS levels and hash-weight SSSP distances from 4 sources are recorded, as the reference computes
them (build once, then applyBatch / insertEdge / deleteEdge).
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402

# The reference's example graph (data/example_graph/ of its checkout), given as the first argument
# or by the environment variable GIR_REFERENCE_DIR (the checkout's root).
REF_EXAMPLE = None
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.npz")


def csr_from_edges(V, edges):
    edges = sorted(set(edges))
    fb = np.zeros(V + 1, np.int32)
    for u, _ in edges:
        fb[u + 1] += 1
    fb = np.cumsum(fb).astype(np.int32)
    fa = np.array([v for _, v in edges], np.int32)
    tb = np.zeros(V + 1, np.int32)
    for _, v in edges:
        tb[v + 1] += 1
    tb = np.cumsum(tb).astype(np.int32)
    rev = sorted((v, u) for u, v in edges)
    ta = np.array([u for _, u in rev], np.int32)
    return fb, fa, tb, ta


def random_edges(rng, n, m):
    e = set()
    while len(e) < m:
        u, v = int(rng.integers(n)), int(rng.integers(n))
        if u != v:
            e.add((u, v))
    return e


def cycle_chain(rng, n):
    e = set()
    start = 0
    while start < n:
        L = min(int(rng.integers(2, 7)), n - start)
        if L > 1:
            for i in range(L):
                e.add((start + i, start + (i + 1) % L))
        if start > 0:
            a, b = start - 1 - int(rng.integers(3)), start
            if a >= 0:
                e.add((a, b))
                if rng.integers(3) == 0:
                    e.add((b, a))
        start += L
    return e


def cactus(rng, n, chords):
    e = set()
    placed = [0]
    nxt = 1
    while nxt < n:
        anchor = placed[int(rng.integers(len(placed)))]
        L = min(int(rng.integers(3, 8)), n - nxt + 1)
        cyc = [anchor]
        for _ in range(1, L):
            cyc.append(nxt)
            placed.append(nxt)
            nxt += 1
        for i in range(len(cyc)):
            e.add((cyc[i], cyc[(i + 1) % len(cyc)]))
    for _ in range(chords):
        u, v = int(rng.integers(n)), int(rng.integers(n))
        if u != v:
            e.add((u, v))
    return e


def random_batch(rng, V, fb, fa, size):
    """Mixed batch with duplicates, cancelling pairs and invalid ops (runBatchDifferentialTest
    style, gir_test.cpp:758-783)."""
    u, v, ins = [], [], []
    E = int(fb[-1])
    for _ in range(size):
        r = rng.random()
        if r < 0.45 and E > 0:
            e = int(rng.integers(E))
            a = int(np.searchsorted(fb, e, side="right") - 1)
            u.append(a); v.append(int(fa[e])); ins.append(0)
        elif r < 0.9:
            a, b = int(rng.integers(V)), int(rng.integers(V))
            u.append(a); v.append(b); ins.append(1)
        elif r < 0.95:
            u.append(int(rng.integers(V))); v.append(V + 3); ins.append(1)  # invalid
        else:
            a = int(rng.integers(V))
            u.append(a); v.append(a); ins.append(1)  # self-loop: dropped
        if rng.random() < 0.15:  # duplicate or cancelling op on the same edge
            u.append(u[-1]); v.append(v[-1]); ins.append(int(rng.integers(2)))
    return np.array(u, np.int32), np.array(v, np.int32), np.array(ins, np.uint8)


def record(store, key, g, sources):
    store[f"{key}/wcc"] = g.wcc()
    store[f"{key}/scc"] = g.scc()
    store[f"{key}/dag"] = g.dag()
    store[f"{key}/blocks"] = g.blocks()
    store[f"{key}/ap"] = g.ap()
    fb, fa = g.out_csr()
    store[f"{key}/fw_beg"] = fb
    store[f"{key}/fw_adj"] = fa
    sb, sa = g.und_csr()
    store[f"{key}/sym_beg"] = sb
    store[f"{key}/sym_adj"] = sa
    store[f"{key}/bfs"] = np.stack([g.bfs(int(s)) for s in sources]) if len(sources) else np.zeros((0, g.V), np.int32)
    store[f"{key}/sssp"] = np.stack([g.sssp(int(s)) for s in sources]) if len(sources) else np.zeros((0, g.V), np.uint64)


def run_case(store, name, V, fb, fa, bb, ba, steps, sources, directory=None):
    """steps: list of ("batch", u, v, ins) or ("insert"/"delete", u, v)."""
    store[f"{name}/V"] = np.array([V], np.int64)
    store[f"{name}/in_fw_beg"] = fb
    store[f"{name}/in_fw_adj"] = fa
    store[f"{name}/in_bw_beg"] = bb
    store[f"{name}/in_bw_adj"] = ba
    store[f"{name}/sources"] = np.asarray(sources, np.int32)
    g = oracle.RefGIR(directory=directory) if directory else oracle.RefGIR(V, fb, fa, bb, ba)
    g.build(7)
    record(store, f"{name}/s0", g, sources)
    for k, st in enumerate(steps, start=1):
        if st[0] == "batch":
            _, u, v, ins = st
            g.apply_batch(u, v, ins)
        else:
            u = np.array([st[1]], np.int32)
            v = np.array([st[2]], np.int32)
            ins = np.array([1 if st[0] == "insert" else 0], np.uint8)
            if st[0] == "insert":
                g.update_edge(st[1], st[2], True)
            else:
                g.update_edge(st[1], st[2], False)
        store[f"{name}/s{k}/ops_u"] = u
        store[f"{name}/s{k}/ops_v"] = v
        store[f"{name}/s{k}/ops_ins"] = ins
        record(store, f"{name}/s{k}", g, sources)
    store[f"{name}/steps"] = np.array([len(steps)], np.int64)
    g.close()


def main():
    store = {}
    names = []
    # the reference's example graph, through its own four-file loader
    fb = np.fromfile(REF_EXAMPLE + "fw_begin.bin", np.int32)
    fa = np.fromfile(REF_EXAMPLE + "fw_adjacent.bin", np.int32)
    bb = np.fromfile(REF_EXAMPLE + "bw_begin.bin", np.int32)
    ba = np.fromfile(REF_EXAMPLE + "bw_adjacent.bin", np.int32)
    V = len(fb) - 1
    src = [0, 3, 9, 12]
    run_case(store, "example", V, fb, fa, bb, ba, [("insert", 3, 12), ("delete", 3, 12), ("delete", 9, 2)], src,
             directory=REF_EXAMPLE)
    run_case(store, "example_del01", V, fb, fa, bb, ba, [("delete", 0, 1)], src, directory=REF_EXAMPLE)
    run_case(store, "example_rev", V, fb, fa, bb, ba, [("insert", 1, 0), ("delete", 0, 1)], src,
             directory=REF_EXAMPLE)
    names += ["example", "example_del01", "example_rev"]
    E = [(15, 299), (299, 15), (299, 178), (178, 299), (15, 296), (296, 15)]
    b = csr_from_edges(300, E)
    run_case(store, "bridge300", 300, *b,
             [("batch", np.array([15, 299], np.int32), np.array([299, 15], np.int32), np.array([0, 0], np.uint8))],
             [15, 299, 178, 0])
    names.append("bridge300")
    rng = np.random.default_rng(12345)
    shapes = [("sparse_60", 60, random_edges(rng, 60, 80)), ("dense_40", 40, random_edges(rng, 40, 160)),
              ("cycles_80", 80, cycle_chain(rng, 80)), ("medium_200", 200, random_edges(rng, 200, 320)),
              ("empty_30", 30, set()), ("dense_120", 120, random_edges(rng, 120, 600)),
              ("cactus_150", 150, cactus(rng, 150, 40))]
    for name, n, edges in shapes:
        b = csr_from_edges(n, edges)
        steps = []
        cur = oracle.RefGIR(n, *b)
        cur.build(7)  # (the reference maintains layers only once they are built)
        for _ in range(6):
            cb, ca = cur.out_csr()
            u, v, ins = random_batch(rng, n, cb, ca, 25)
            cur.apply_batch(u, v, ins)
            steps.append(("batch", u, v, ins))
        cur.close()
        run_case(store, name, n, *b, steps, [0, 1, n // 2, n - 1])
        names.append(name)
    # R-MAT scale 10 (the benchmark shape, small)
    sys.path.insert(0, ROOT)
    import importlib
    pkg = importlib.import_module("graph-intermedia-representation_b200")
    g = pkg.graphs.rmat(10, seed=7, weights=None)
    steps = []
    cur = oracle.RefGIR(g.V, g.fw_beg, g.fw_adj, g.bw_beg, g.bw_adj)
    cur.build(7)
    for k in range(3):
        cb, ca = cur.out_csr()
        u, v, ins = random_batch(rng, g.V, cb, ca, 200)
        cur.apply_batch(u, v, ins)
        steps.append(("batch", u, v, ins))
    cur.close()
    run_case(store, "rmat_s10", g.V, g.fw_beg, g.fw_adj, g.bw_beg, g.bw_adj, steps, [0, 5, 100, 1000])
    names.append("rmat_s10")
    store["cases"] = np.array(names)
    np.savez_compressed(OUT, **store)
    print(f"wrote {OUT}: {len(names)} cases, {os.path.getsize(OUT)} bytes")


if __name__ == "__main__":
    checkout = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GIR_REFERENCE_DIR")
    if not checkout:
        sys.exit("usage: make_golden.py <reference checkout> (or set GIR_REFERENCE_DIR)")
    REF_EXAMPLE = os.path.join(checkout, "data", "example_graph") + os.sep
    main()
