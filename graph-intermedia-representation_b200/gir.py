"""Python mirror of the reference GIR class surface (gir_constructor/gir.h:72-671) over the
gir_dev_* C ABI. Every computation runs in libgir_b200.so on the GPU; this module only moves
arguments and results.

Differences from the reference that a caller can see:
  - component ids are canonical: the id of a WCC / SCC is its smallest vertex (the reference
    uses union-find roots and Tarjan emission order, gir.cpp:646-653, 809-816), so getSCCs()
    has one slot per vertex id, empty for ids that are not an SCC's smallest vertex (the
    reference's list also has empty slots, for retired ids);
  - single-edge updates are applied at once as one-edge batches (the reference's
    Scope-Prune-Update path, gir.cpp:3043-3131, has the same effect on every layer);
  - malformed input raises GirError instead of ending the process (graph.cpp:95-114).
"""
import ctypes

import numpy as np

from . import native
from .native import GirError, dev_lib, ptr


def _raise(handle, rc, what):
    if rc != 0:
        lib = dev_lib()
        msg = lib.gir_dev_last_error(handle).decode() if handle is not None else lib.gir_dev_last_error(None).decode()
        raise GirError(rc, f"{what}: {msg}")


class DeviceGraph:
    """One graph resident in HBM (a gir_dev_t handle)."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def create(cls, fw_beg, fw_adj, bw_beg, bw_adj, V, w=None):
        lib = dev_lib()
        h = ctypes.c_void_p()
        E = int(len(fw_adj))
        rc = lib.gir_dev_create(ptr(fw_beg), ptr(fw_adj), ptr(bw_beg), ptr(bw_adj), int(V), E, ptr(w), ctypes.byref(h))
        _raise(None, rc, "gir_dev_create")
        return cls(h)

    @classmethod
    def from_graph(cls, g, weights=True):
        return cls.create(g.fw_beg, g.fw_adj, g.bw_beg, g.bw_adj, g.V, g.w if weights else None)

    @classmethod
    def load(cls, directory):
        lib = dev_lib()
        h = ctypes.c_void_p()
        rc = lib.gir_dev_load(directory.encode(), ctypes.byref(h))
        _raise(None, rc, "gir_dev_load")
        return cls(h)

    def close(self):
        if self._h is not None:
            dev_lib().gir_dev_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc, what):
        _raise(self._h, rc, what)

    @property
    def handle(self):
        return self._h

    def counts(self):
        vals = [ctypes.c_int64() for _ in range(6)]
        self._ck(dev_lib().gir_dev_counts(self._h, *[ctypes.byref(v) for v in vals]), "counts")
        keys = ("V", "E", "n_wcc", "n_scc", "n_dag", "n_blocks")
        return dict(zip(keys, (v.value for v in vals)))

    @property
    def V(self):
        return self.counts()["V"]

    @property
    def E(self):
        return self.counts()["E"]

    def build(self, layers=native.LAYER_ALL):
        self._ck(dev_lib().gir_dev_build(self._h, layers), "build")

    def labels(self, which):
        out = np.empty(self.V, np.int32)
        self._ck(dev_lib().gir_dev_get_labels(self._h, which, ptr(out)), "get_labels")
        return out

    def dag(self):
        n = ctypes.c_int64()
        self._ck(dev_lib().gir_dev_get_dag(self._h, None, None, 0, ctypes.byref(n)), "get_dag")
        src = np.empty(n.value, np.int32)
        dst = np.empty(n.value, np.int32)
        self._ck(dev_lib().gir_dev_get_dag(self._h, ptr(src), ptr(dst), n.value, ctypes.byref(n)), "get_dag")
        return src, dst

    def blocks(self):
        """(label_block[V], head[n_blocks]): block b = {v : label_block[v] == b} + {head[b]} (head -1: root)."""
        n = ctypes.c_int64()
        self._ck(dev_lib().gir_dev_get_blocks(self._h, None, 0, ctypes.byref(n)), "get_blocks")
        head = np.empty(n.value, np.int32)
        self._ck(dev_lib().gir_dev_get_blocks(self._h, ptr(head), n.value, ctypes.byref(n)), "get_blocks")
        return self.labels(native.LABEL_BLOCK), head

    def csr(self, direction=0):
        """Current edge set as a compact CSR: 0 forward, 1 backward, 2 symmetrized."""
        n = ctypes.c_int64()
        self._ck(dev_lib().gir_dev_get_csr(self._h, direction, None, None, 0, ctypes.byref(n)), "get_csr")
        beg = np.empty(self.V + 1, np.int64)
        adj = np.empty(max(n.value, 1), np.int32)
        self._ck(dev_lib().gir_dev_get_csr(self._h, direction, ptr(beg), ptr(adj), n.value, ctypes.byref(n)), "get_csr")
        return beg, adj[:n.value]

    def has_edges(self, u, v, undirected=False):
        u = np.ascontiguousarray(u, np.int32)
        v = np.ascontiguousarray(v, np.int32)
        out = np.empty(len(u), np.uint8)
        self._ck(dev_lib().gir_dev_has_edges(self._h, int(undirected), ptr(u), ptr(v), len(u), ptr(out)), "has_edges")
        return out.astype(bool)

    @staticmethod
    def _ids(a):
        """int32 ids as an array the C ABI can read: numpy (host) or a torch tensor (host or device)."""
        if hasattr(a, "data_ptr"):
            assert str(a.dtype) == "torch.int32" and a.is_contiguous()
            return a, int(a.numel())
        a = np.ascontiguousarray(a, np.int32)
        return a, len(a)

    def bfs(self, sources, out=None):
        s, n = self._ids(sources)
        if out is None:
            out = np.empty((n, self.V), np.int32)
        self._ck(dev_lib().gir_dev_bfs(self._h, ptr(s), n, ptr(out)), "bfs")
        return out

    def bfs_sets(self, sets, out=None):
        beg = np.zeros(len(sets) + 1, np.int64)
        beg[1:] = np.cumsum([len(x) for x in sets])
        src = np.concatenate([np.asarray(x, np.int32) for x in sets]) if sets else np.zeros(0, np.int32)
        if out is None:
            out = np.empty((len(sets), self.V), np.int32)
        self._ck(dev_lib().gir_dev_bfs_sets(self._h, ptr(beg), ptr(src), len(sets), ptr(out)), "bfs_sets")
        return out

    def sssp(self, sources, delta=16, weights=native.WEIGHT_HASH, out=None):
        s, n = self._ids(sources)
        if out is None:
            out = np.empty((n, self.V), np.uint64)
        self._ck(dev_lib().gir_dev_sssp(self._h, ptr(s), n, int(delta), weights, ptr(out)), "sssp")
        return out

    def sssp_sets(self, sets, delta=16, weights=native.WEIGHT_HASH, out=None):
        beg = np.zeros(len(sets) + 1, np.int64)
        beg[1:] = np.cumsum([len(x) for x in sets])
        src = np.concatenate([np.asarray(x, np.int32) for x in sets]) if sets else np.zeros(0, np.int32)
        if out is None:
            out = np.empty((len(sets), self.V), np.uint64)
        self._ck(dev_lib().gir_dev_sssp_sets(self._h, ptr(beg), ptr(src), len(sets), int(delta), weights, ptr(out)),
                 "sssp_sets")
        return out

    def apply_batch(self, u, v, ins):
        u = np.ascontiguousarray(u, np.int32)
        v = np.ascontiguousarray(v, np.int32)
        ins = np.ascontiguousarray(ins, np.uint8)
        self._ck(dev_lib().gir_dev_apply_batch(self._h, ptr(u), ptr(v), ptr(ins), len(u)), "apply_batch")

    def ingest_batch(self, u, v, ins):
        """Edge store only; the layers wait for sync() (gir_dev_ingest_batch)."""
        u = np.ascontiguousarray(u, np.int32)
        v = np.ascontiguousarray(v, np.int32)
        ins = np.ascontiguousarray(ins, np.uint8)
        self._ck(dev_lib().gir_dev_ingest_batch(self._h, ptr(u), ptr(v), ptr(ins), len(u)), "ingest_batch")

    def sync(self):
        self._ck(dev_lib().gir_dev_sync(self._h), "sync")

    def synced(self):
        out = ctypes.c_int()
        self._ck(dev_lib().gir_dev_synced(self._h, ctypes.byref(out)), "synced")
        return bool(out.value)

    def batch_stats(self):
        vals = [ctypes.c_int64() for _ in range(4)]
        self._ck(dev_lib().gir_dev_batch_stats(self._h, *[ctypes.byref(v) for v in vals]), "batch_stats")
        return dict(zip(("inserted", "deleted", "noop", "invalid"), (v.value for v in vals)))

    def batch_times(self):
        """Wall ms of the last batch's phases: store merge, WCC, SCC + DAG, blocks."""
        out = np.zeros(4, np.float64)
        self._ck(dev_lib().gir_dev_batch_times(self._h, ptr(out)), "batch_times")
        return dict(zip(("store", "wcc", "scc", "bct"), out.tolist()))

    def autotune(self, sources, reps=2):
        """Picks the grid size and degree-bin thresholds by timing BFS from `sources` (1..64);
        returns the chosen parameters and the winner's ms per call."""
        s, n = self._ids(sources)
        best = ctypes.c_double()
        self._ck(dev_lib().gir_dev_autotune(self._h, ptr(s), n, int(reps), ctypes.byref(best)), "autotune")
        P = native
        return {"ctas_per_sm": self.get_param(P.PARAM_CTAS_PER_SM), "small_deg": self.get_param(P.PARAM_SMALL_DEG),
                "large_deg": self.get_param(P.PARAM_LARGE_DEG), "bfs_ms": best.value}

    def reachable(self, u, v, out=None):
        """GIR::reachable for every pair (u[i], v[i]): a bool array (or fills `out`, uint8)."""
        su, n = self._ids(u)
        sv, n2 = self._ids(v)
        if n != n2:
            raise ValueError("reachable: u and v differ in length")
        res = np.empty(n, np.uint8) if out is None else out
        self._ck(dev_lib().gir_dev_reachable(self._h, ptr(su), ptr(sv), n, ptr(res)), "reachable")
        return res.astype(bool) if out is None else res

    def bc(self, sources, out=None):
        """GIR::bc: betweenness of every vertex over `sources` (float64[V], or fills `out`)."""
        s, n = self._ids(sources)
        res = np.empty(self.V, np.float64) if out is None else out
        self._ck(dev_lib().gir_dev_bc(self._h, ptr(s), n, ptr(res)), "bc")
        return res

    def inc_track(self, source, weighted):
        """GIR::trackIncremental: BFS (weighted False) or SSSP (True, GIR::edgeWeight) of one
        source, kept up to date by inc_update under later batches."""
        self._ck(dev_lib().gir_dev_inc_track(self._h, int(source), 1 if weighted else 0), "inc_track")

    def inc_update(self, weighted):
        """GIR::updateIncremental: corrects the tracked result for the edges changed since."""
        self._ck(dev_lib().gir_dev_inc_update(self._h, 1 if weighted else 0), "inc_update")

    def inc_dist(self, weighted, out=None):
        """The tracked levels / distances of every vertex (uint64[V], UINT64_MAX = unreachable)."""
        res = np.empty(self.V, np.uint64) if out is None else out
        self._ck(dev_lib().gir_dev_inc_dist(self._h, 1 if weighted else 0, ptr(res)), "inc_dist")
        return res

    def single_stats(self):
        """One-op batches that ran the exact single-edge checks, and the layer rebuilds they avoided."""
        c, k = ctypes.c_int64(), ctypes.c_int64()
        self._ck(dev_lib().gir_dev_single_stats(self._h, ctypes.byref(c), ctypes.byref(k)), "single_stats")
        return {"checked": c.value, "kept": k.value}

    def batch_plan(self):
        """Per layer, what the last batch did: 'kept', 'patched' or 'rebuilt'."""
        out = np.zeros(3, np.int32)
        self._ck(dev_lib().gir_dev_batch_plan(self._h, ptr(out)), "batch_plan")
        names = ("kept", "patched", "rebuilt")
        return dict(zip(("wcc", "scc", "bct"), (names[i] for i in out.tolist())))

    def set_weight_rule(self, seed, lo, hi):
        self._ck(dev_lib().gir_dev_set_weight_rule(self._h, seed, lo, hi), "set_weight_rule")

    def set_schedule(self, mode):
        self._ck(dev_lib().gir_dev_set_schedule(self._h, mode), "set_schedule")

    def set_param(self, which, value):
        self._ck(dev_lib().gir_dev_set_param(self._h, which, float(value)), "set_param")

    def get_param(self, which):
        v = ctypes.c_double()
        self._ck(dev_lib().gir_dev_get_param(self._h, which, ctypes.byref(v)), "get_param")
        return v.value

    def query_stats(self):
        st = native.QueryStats()
        self._ck(dev_lib().gir_dev_query_stats(self._h, ctypes.byref(st)), "query_stats")
        return {f: getattr(st, f) for f, _ in native.QueryStats._fields_}

    def stream(self):
        s = ctypes.c_void_p()
        self._ck(dev_lib().gir_dev_stream(self._h, ctypes.byref(s)), "stream")
        return s.value

    # ---- schedule network ----
    def sched_param_count(self):
        return int(dev_lib().gir_dev_sched_param_count())

    def sched_set_weights(self, params):
        p = np.ascontiguousarray(params, np.float32)
        self._ck(dev_lib().gir_dev_sched_set_weights(self._h, ptr(p), len(p)), "sched_set_weights")

    def sched_get_weights(self):
        p = np.empty(self.sched_param_count(), np.float32)
        self._ck(dev_lib().gir_dev_sched_get_weights(self._h, ptr(p), len(p)), "sched_get_weights")
        return p

    def sched_forward(self, x):
        x = np.ascontiguousarray(x, np.float32)
        out = np.empty((len(x), native.SCHED_OUT), np.float32)
        self._ck(dev_lib().gir_dev_sched_forward(self._h, ptr(x), len(x), ptr(out)), "sched_forward")
        return out

    def sched_grad(self, x, y):
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.int32)
        grad = np.empty(self.sched_param_count(), np.float32)
        loss = ctypes.c_float()
        self._ck(dev_lib().gir_dev_sched_grad(self._h, ptr(x), ptr(y), len(x), ptr(grad), ctypes.byref(loss)),
                 "sched_grad")
        return grad, loss.value

    def use_learned_schedule(self, path=None):
        """Loads the trained schedule network (schedule_weights.npy, written by
        train_schedule.py) and switches the traversal choices to it."""
        import os
        path = path or os.path.join(os.path.dirname(os.path.abspath(__file__)), "schedule_weights.npy")
        self.sched_set_weights(np.load(path))
        self.set_schedule(native.SCHEDULE_LEARNED)

    def sched_trace(self):
        """(features[n][8], class[n]) of the schedule decisions of the last query call."""
        n = ctypes.c_int64()
        self._ck(dev_lib().gir_dev_sched_trace(self._h, None, None, 0, ctypes.byref(n)), "sched_trace")
        x = np.empty((n.value, native.SCHED_IN), np.float32)
        y = np.empty(n.value, np.int32)
        self._ck(dev_lib().gir_dev_sched_trace(self._h, ptr(x), ptr(y), n.value, ctypes.byref(n)), "sched_trace")
        return x, y

    @staticmethod
    def delta_choices():
        out = np.empty(6, np.uint64)
        rc = dev_lib().gir_dev_sched_delta_choices(ptr(out))
        if rc != 0:
            raise GirError(rc, "sched_delta_choices")
        return out

    def sched_train(self, x, y, steps, lr):
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.int32)
        loss = ctypes.c_float()
        self._ck(dev_lib().gir_dev_sched_train(self._h, ptr(x), ptr(y), len(x), int(steps), float(lr),
                                               ctypes.byref(loss)), "sched_train")
        return loss.value


class GIR:
    """The reference's GIR class surface (gir.h:72-240) on the GPU."""

    kMaxWeight = 100

    def __init__(self, path_directed=None, path_undirected=None, graph=None, weights=False):
        if graph is not None:
            self._d = DeviceGraph.from_graph(graph, weights=weights)  # GIR(graph*) (gir.h:95)
        else:
            self._d = DeviceGraph.load(path_directed)  # GIR(dir, und_dir) (gir.h:93)
        self._V = self._d.V
        self._inc = {False: None, True: None}

    @property
    def device(self):
        return self._d

    # construction (gir.h:98-101)
    def buildWCC(self):
        self._d.build(native.LAYER_WCC)

    def buildSCC_DAG(self):
        self._d.build(native.LAYER_SCC)

    def buildBCT(self):
        self._d.build(native.LAYER_BCT)

    # updates (gir.h:104-119)
    def applyBatch(self, batch):
        """batch: iterable of (u, v, insert)."""
        arr = np.asarray(list(batch), dtype=np.int64).reshape(-1, 3)
        self._d.apply_batch(arr[:, 0], arr[:, 1], arr[:, 2] != 0)

    def insertEdge(self, u, v):
        self._d.apply_batch([u], [v], [1])

    def deleteEdge(self, u, v):
        self._d.apply_batch([u], [v], [0])

    def updateEdgeDirected(self, u, v, insert):
        self._d.apply_batch([u], [v], [1 if insert else 0])

    def updateEdgeUndirected(self, u, v, insert):
        # gir.cpp:3134: the reference routes the undirected entry point through the directed one
        self._d.apply_batch([u], [v], [1 if insert else 0])

    # deferred maintenance (gir.h:107-116): the edge store takes the batch now, the layers at sync()
    def ingestBatch(self, batch):
        arr = np.asarray(list(batch), dtype=np.int64).reshape(-1, 3)
        self._d.ingest_batch(arr[:, 0], arr[:, 1], arr[:, 2] != 0)

    def sync(self):
        self._d.sync()

    def synced(self):
        return self._d.synced()

    # per-vertex queries (gir.h:122-125)
    def vertexCount(self):
        return self._V

    def sccOf(self, v):
        return int(self._d.labels(native.LABEL_SCC)[v])

    def wccOf(self, v):
        return int(self._d.labels(native.LABEL_WCC)[v])

    def sccRank(self, s):
        return int(self._d.labels(native.LABEL_SCC_RANK)[s])

    def isArticulationPoint(self, v):
        return bool(self._d.labels(native.LABEL_BCNT)[v] >= 2)

    # materialized views (gir.h:142-150)
    def getNodeToScc(self):
        return dict(enumerate(self._d.labels(native.LABEL_SCC).tolist()))

    def getNodeToWcc(self):
        return dict(enumerate(self._d.labels(native.LABEL_WCC).tolist()))

    def _groups(self, lab):
        order = np.argsort(lab, kind="stable")
        out = [[] for _ in range(self._V)]
        for v in order.tolist():
            out[lab[v]].append(v)
        return out

    def getSCCs(self):
        return self._groups(self._d.labels(native.LABEL_SCC))

    def getWCCs(self):
        return [g for g in self._groups(self._d.labels(native.LABEL_WCC)) if g]

    def getDAG(self):
        src, dst = self._d.dag()
        rows = [[] for _ in range(self._V)]
        for a, b in zip(src.tolist(), dst.tolist()):
            rows[a].append(b)
        return rows

    def getBCTComponents(self, scc_id):
        scc = self._d.labels(native.LABEL_SCC)
        label, head = self._d.blocks()
        members = np.nonzero(scc == scc_id)[0]
        out = {}
        for v in members.tolist():
            out.setdefault(int(label[v]), set()).add(v)
        for b in list(out):
            if head[b] >= 0:
                out[b].add(int(head[b]))
        return [sorted(x) for x in out.values()]

    # edge store (gir.h:160-164)
    def getDirectedOutNeighbors(self, v):
        beg, adj = self._d.csr(0)
        return adj[beg[v]:beg[v + 1]].tolist()

    def getDirectedInNeighbors(self, v):
        beg, adj = self._d.csr(1)
        return adj[beg[v]:beg[v + 1]].tolist()

    def getUndirectedNeighborsPublic(self, v):
        beg, adj = self._d.csr(2)
        return adj[beg[v]:beg[v + 1]].tolist()

    def hasDirectedEdge(self, u, v):
        return bool(self._d.has_edges([u], [v])[0])

    def hasUndirectedEdge(self, u, v):
        return bool(self._d.has_edges([u], [v], undirected=True)[0])

    # queries (gir.h:204-216)
    def bfs(self, source):
        return self._d.bfs([source])[0]

    def sssp(self, source, delta=16):
        return self._d.sssp([source], delta=delta)[0]

    def reachable(self, u, v):
        """gir.h:128-130 (gir_query.cpp:789-825); batches go through DeviceGraph.reachable."""
        return bool(self._d.reachable([u], [v])[0])

    def reachableNoIndex(self, u, v):
        """gir.h:138: the same answer without the index (a BFS from u over the edge store)."""
        if not (0 <= u < self._V and 0 <= v < self._V):
            return False
        return u == v or bool(self._d.bfs([u])[0][v] >= 0)

    # structure-based queries sync first (gir.h:131-135)
    def sameScc(self, u, v):
        self.sync()
        lab = self._d.labels(native.LABEL_SCC)
        return bool(lab[u] == lab[v])

    def sameWcc(self, u, v):
        self.sync()
        lab = self._d.labels(native.LABEL_WCC)
        return bool(lab[u] == lab[v])

    def articulationPoint(self, v):
        self.sync()
        return self.isArticulationPoint(v)

    def biconnected(self, u, v):
        """u and v share a block of one SCC's undirected view (a vertex lies in its own block and
        in every block it heads)."""
        self.sync()
        if u == v:
            return True
        scc = self._d.labels(native.LABEL_SCC)
        if scc[u] != scc[v]:
            return False
        blk, head = self._d.blocks()
        return bool(blk[u] == blk[v] or head[blk[v]] == u or head[blk[u]] == v)

    def checkBlockForestInvariants(self):
        """gir.h:153 (gir.cpp:4159-4211): the block-cut forest's structural rules -- every block
        non-empty and inside one SCC with its head, heads are articulation points, block counts
        equal 1 + the blocks a vertex heads."""
        scc = self._d.labels(native.LABEL_SCC).astype(np.int64)
        blk, head = self._d.blocks()
        cnt = self._d.labels(native.LABEL_BCNT).astype(np.int64)
        blk = blk.astype(np.int64)
        head = head.astype(np.int64)
        nb = len(head)
        if len(blk) and (blk.min() < 0 or blk.max() >= nb):
            return False
        members = np.bincount(blk, minlength=nb)
        if np.any(members == 0):
            return False
        lo = np.full(nb, np.iinfo(np.int64).max)
        hi = np.full(nb, -1)
        np.minimum.at(lo, blk, scc)
        np.maximum.at(hi, blk, scc)
        if np.any(lo != hi):
            return False
        hh = head >= 0
        if np.any(scc[head[hh]] != lo[hh]):
            return False
        exp = np.ones(self._V, np.int64)
        np.add.at(exp, head[hh], 1)
        return bool(np.array_equal(cnt, exp) and np.all(cnt[head[hh]] >= 2))

    # gir.h:208-216: the reference's task-parallel formulations of the same queries (a wavefront
    # over the condensation DAG with block tasks inside SCCs) return what bfs / sssp return; on
    # the device the flat lane-parallel traversal is that computation.
    def bc(self, sources):
        """gir.h:217-219 (gir_query.cpp:728-778)."""
        return self._d.bc(sources)

    # gir.h:220-232 (gir_query.cpp:867-996). incDist reads a host copy of the tracked result,
    # taken after each track / update (the result changes only there).
    def trackIncremental(self, source, weighted):
        self._d.inc_track(source, weighted)
        self._inc[bool(weighted)] = None

    def updateIncremental(self, weighted):
        self._d.inc_update(weighted)
        self._inc[bool(weighted)] = None

    def incDist(self, weighted, v):
        w = bool(weighted)
        if self._inc[w] is None:
            self._inc[w] = self._d.inc_dist(w)
        return int(self._inc[w][v])

    def bfsTwoLevel(self, source):
        return self.bfs(source)

    def bfsTaskParallel(self, source):
        return self.bfs(source)

    def ssspTwoLevel(self, source, delta=16):
        return self.sssp(source, delta)

    @staticmethod
    def edgeWeight(u, v):
        """gir_query.cpp:50-54 (computed on the host here only to answer this static call)."""
        x = ((u & 0xffffffff) << 32) | (v & 0xffffffff)
        m = (1 << 64) - 1
        x ^= x >> 33
        x = (x * 0xff51afd7ed558ccd) & m
        x ^= x >> 33
        x = (x * 0xc4ceb9fe1a85ec53) & m
        x ^= x >> 33
        return 1 + x % GIR.kMaxWeight
