"""Python access to the test oracle -- TEST INFRASTRUCTURE ONLY.

Two libraries, both built by oracle/Makefile:
  liboracle.so       the C restatement of the reference algorithms (gir_oracle.c)
  _ref/libgirref.so  the reference GIR itself, compiled from its own sources (ref_shim.cpp)

Only tests/, the smoke check of __graft_entry__.py and bench.py's CPU-baseline / reference arm
use this module; the product (graph-intermedia-representation_b200/) never does.
Also the canonical forms every comparison is made in (the normalizePartition idea of
gir_constructor/gir_test.cpp:365-374): component label = smallest vertex of the component,
condensation edges as sorted (label, label) pairs, blocks as sorted (k1, k2, v) triples.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_lib = None
_ref = None


def ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise ImportError(f"{path} missing: run `make -C {HERE}`")
        L = ctypes.CDLL(path)
        L.or_file_sizes.argtypes = [ctypes.c_char_p] + [ctypes.POINTER(_I64)] * 4
        L.or_load.argtypes = [ctypes.c_char_p, _I64, _I64, _P, _P, _P, _P]
        L.or_normalize.argtypes = [_I64, _P, _P]
        L.or_normalize.restype = _I64
        L.or_sym.argtypes = [_I64, _P, _P, _P, _P, _P, _P]
        L.or_sym.restype = _I64
        L.or_wcc.argtypes = [_I64, _P, _P, _P]
        L.or_wcc.restype = None
        L.or_scc.argtypes = [_I64, _P, _P, _P]
        L.or_scc.restype = None
        L.or_dag.argtypes = [_I64, _P, _P, _P, _P]
        L.or_dag.restype = _I64
        L.or_bicc.argtypes = [_I64, _P, _P, _P, _P, _P, _P, _P]
        L.or_bicc.restype = _I64
        L.or_bfs.argtypes = [_I64, _P, _P, _P, _I64, _P]
        L.or_bfs.restype = None
        L.or_edge_weight.argtypes = [ctypes.c_int32, ctypes.c_int32]
        L.or_edge_weight.restype = ctypes.c_uint32
        L.or_sssp.argtypes = [_I64, _P, _P, _P, _P, _I64, _P]
        L.or_sssp.restype = None
        L.or_apply_batch.argtypes = [_I64, _P, _P, _P, _P, _P, _I64, _P, _P, ctypes.POINTER(_I64),
                                     ctypes.POINTER(_I64)]
        L.or_apply_batch.restype = _I64
        L.or_transpose.argtypes = [_I64, _P, _P, _P, _P]
        L.or_transpose.restype = None
        _lib = L
    return _lib


def ref_available():
    return os.path.exists(os.path.join(HERE, "_ref", "libgirref.so"))


def ref():
    """The reference GIR compiled from its sources (raises if it was not built)."""
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libgirref.so")
        if not os.path.exists(path):
            raise ImportError(f"{path} missing: run `make -C {HERE}` where the reference sources exist")
        R = ctypes.CDLL(path)
        R.ref_create.argtypes = [ctypes.c_int32, _I64, _P, _P, _P, _P]
        R.ref_create.restype = _P
        R.ref_load.argtypes = [ctypes.c_char_p]
        R.ref_load.restype = _P
        R.ref_destroy.argtypes = [_P]
        R.ref_build.argtypes = [_P, ctypes.c_int]
        R.ref_vertex_count.argtypes = [_P]
        R.ref_vertex_count.restype = ctypes.c_int32
        R.ref_out_csr.argtypes = [_P, _P, _P]
        R.ref_out_csr.restype = _I64
        R.ref_und_csr.argtypes = [_P, _P, _P]
        R.ref_und_csr.restype = _I64
        R.ref_bfs.argtypes = [_P, ctypes.c_int32, _P]
        R.ref_reachable.argtypes = [_P, _P, _P, _I64, _P]
        R.ref_bc.argtypes = [_P, _P, _I64, _P]
        R.ref_bc.restype = None
        R.ref_ingest_batch.argtypes = [_P, _P, _P, _P, _I64]
        R.ref_ingest_batch.restype = None
        R.ref_sync.argtypes = [_P]
        R.ref_sync.restype = None
        R.ref_synced.argtypes = [_P]
        R.ref_synced.restype = ctypes.c_int
        R.ref_inc_track.argtypes = [_P, ctypes.c_int32, ctypes.c_int]
        R.ref_inc_track.restype = None
        R.ref_inc_update.argtypes = [_P, ctypes.c_int]
        R.ref_inc_update.restype = None
        R.ref_inc_dist.argtypes = [_P, ctypes.c_int, _P]
        R.ref_inc_dist.restype = None
        R.ref_reachable.restype = None
        R.ref_sssp.argtypes = [_P, ctypes.c_int32, ctypes.c_uint64, _P]
        R.ref_bfs_two_level.argtypes = [_P, ctypes.c_int32, _P]
        R.ref_bfs_two_level.restype = None
        R.ref_sssp_two_level.argtypes = [_P, ctypes.c_int32, ctypes.c_uint64, _P]
        R.ref_sssp_two_level.restype = None
        R.ref_edge_weight.argtypes = [ctypes.c_int32, ctypes.c_int32]
        R.ref_edge_weight.restype = ctypes.c_uint32
        R.ref_apply_batch.argtypes = [_P, _P, _P, _P, _I64]
        R.ref_update_edge.argtypes = [_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int, ctypes.c_int]
        R.ref_scc_raw.argtypes = [_P, _P]
        R.ref_wcc_raw.argtypes = [_P, _P]
        R.ref_dag_raw.argtypes = [_P, _P, _P]
        R.ref_dag_raw.restype = _I64
        R.ref_blocks.argtypes = [_P, _P, _P, ctypes.POINTER(_I64)]
        R.ref_blocks.restype = _I64
        R.ref_ap.argtypes = [_P, _P]
        R.ref_bct_shape.argtypes = [_P, ctypes.c_int32, ctypes.POINTER(_I64), ctypes.POINTER(_I64)]
        _ref = R
    return _ref


# ---------------------------------------------------------------------------------------------
# canonical forms
# ---------------------------------------------------------------------------------------------

def canon_labels(lab):
    """Relabel every class to its smallest vertex id."""
    lab = np.asarray(lab, np.int64)
    V = len(lab)
    if V == 0:
        return lab.astype(np.int32)
    top = int(lab.max()) + 1
    mins = np.full(top, V, np.int64)
    np.minimum.at(mins, lab, np.arange(V, dtype=np.int64))
    return mins[lab].astype(np.int32)


def canon_dag_from_labels(canon_scc, src_vertex_scc_ids, dst_vertex_scc_ids):
    keys = (np.asarray(src_vertex_scc_ids, np.int64) << 32) | np.asarray(dst_vertex_scc_ids, np.int64)
    return np.unique(keys)


def canon_blocks(blocks):
    """blocks: iterable of vertex lists -> sorted (k1, k2, v) triples as an int64 array [n, 3]."""
    rows = []
    for b in blocks:
        s = sorted(set(int(x) for x in b))
        k1 = s[0]
        k2 = s[1] if len(s) > 1 else -1
        rows.extend((k1, k2, v) for v in s)
    if not rows:
        return np.zeros((0, 3), np.int64)
    a = np.array(rows, np.int64)
    return a[np.lexsort((a[:, 2], a[:, 1], a[:, 0]))]


def canon_blocks_csr(beg, verts):
    """Blocks as a CSR of vertex lists (block i = verts[beg[i]:beg[i+1]]) -> the same sorted
    (k1, k2, v) triples as canon_blocks, vectorized for millions of blocks (empty blocks are
    dropped, repeated vertices within a block counted once)."""
    beg = np.asarray(beg, np.int64)
    verts = np.asarray(verts, np.int64)
    nb = len(beg) - 1
    if nb <= 0 or len(verts) == 0:
        return np.zeros((0, 3), np.int64)
    b = np.repeat(np.arange(nb, dtype=np.int64), np.diff(beg))
    key = np.unique((b << 32) | verts[:len(b)])
    b, v = key >> 32, key & 0xffffffff
    starts = np.r_[0, np.nonzero(np.diff(b))[0] + 1]
    cnt = np.diff(np.r_[starts, len(b)])
    first = v[starts]
    second = np.where(cnt > 1, v[np.minimum(starts + 1, len(v) - 1)], -1)
    idx = np.repeat(np.arange(len(starts)), cnt)
    t = np.stack([first[idx], second[idx], v], axis=1)
    return t[np.lexsort((t[:, 2], t[:, 1], t[:, 0]))]


def block_forest(V, sb, sa, scc_lab):
    """The oracle's blocks in the block-cut forest representation the device library returns
    (v_block / blk_parent_ap / v_bcnt, gir_constructor/gir.h:420-423): every vertex labelled with
    one block, every block headed by the articulation point through which it hangs off its
    parent block (-1 for the root block of an SCC), and the number of blocks holding each vertex.
    Blocks are walked breadth-first from the block of each SCC's smallest vertex. Small graphs
    only (Python loops)."""
    t = bicc(V, sb, sa, scc_lab)[0]
    blocks = {}
    for k1, k2, v in t:
        blocks.setdefault((int(k1), int(k2)), []).append(int(v))
    blist = sorted(blocks.values(), key=lambda b: min(b))
    of = {}
    for i, b in enumerate(blist):
        for v in b:
            of.setdefault(v, []).append(i)
    nb = len(blist)
    label = np.full(V, -1, np.int64)
    head = np.full(nb, -2, np.int64)
    bcnt = np.zeros(V, np.int64)
    for v, bs in of.items():
        bcnt[v] = len(bs)
    for r in range(nb):
        if head[r] != -2:
            continue
        head[r] = -1
        queue = [r]
        while queue:
            b = queue.pop(0)
            for v in blist[b]:
                if v == head[b]:
                    continue
                label[v] = b
                for c in of[v]:
                    if head[c] == -2:
                        head[c] = v
                        queue.append(c)
    return label.astype(np.int32), head.astype(np.int32), bcnt.astype(np.int32)


def canon_blocks_from_device(label_block, head):
    """Device representation (block of every vertex + head AP of every block) -> triples."""
    label_block = np.asarray(label_block, np.int64)
    head = np.asarray(head, np.int64)
    V = len(label_block)
    b = np.concatenate([label_block, np.nonzero(head >= 0)[0]])
    v = np.concatenate([np.arange(V, dtype=np.int64), head[head >= 0]])
    order = np.lexsort((v, b))
    b, v = b[order], v[order]
    nb = len(head)
    # two smallest vertices per block
    first = np.full(nb, -1, np.int64)
    second = np.full(nb, -1, np.int64)
    starts = np.r_[0, np.nonzero(np.diff(b))[0] + 1]
    first[b[starts]] = v[starts]
    has2 = starts + 1 < len(b)
    nxt = np.minimum(starts + 1, len(b) - 1)
    same = has2 & (b[nxt] == b[starts])
    second[b[starts[same]]] = v[nxt[same]]
    t = np.stack([first[b], second[b], v], axis=1)
    return t[np.lexsort((t[:, 2], t[:, 1], t[:, 0]))]


def sort_rows(beg, adj):
    """Sorts every row of a CSR (the canonical row order)."""
    beg = np.asarray(beg, np.int64)
    rows = np.repeat(np.arange(len(beg) - 1, dtype=np.int64), np.diff(beg))
    order = np.lexsort((np.asarray(adj, np.int64), rows))
    return np.asarray(adj)[order]


def ap_from_triples(t, V):
    cnt = np.bincount(t[:, 2], minlength=V) if len(t) else np.zeros(V, np.int64)
    return cnt >= 2


# ---------------------------------------------------------------------------------------------
# the C restatement
# ---------------------------------------------------------------------------------------------

def normalize(V, beg, adj):
    beg = np.asarray(beg, np.int64).copy()
    adj = np.asarray(adj, np.int32).copy()
    E = lib().or_normalize(V, ptr(beg), ptr(adj))
    return beg, adj[:E].copy()


def transpose(V, beg, adj):
    tb = np.zeros(V + 1, np.int64)
    ta = np.zeros(max(len(adj), 1), np.int32)
    lib().or_transpose(V, ptr(np.ascontiguousarray(beg, np.int64)), ptr(np.ascontiguousarray(adj, np.int32)),
                       ptr(tb), ptr(ta))
    return tb, ta[:len(adj)]


def sym(V, fb, fa, bb, ba):
    fb, bb = np.ascontiguousarray(fb, np.int64), np.ascontiguousarray(bb, np.int64)
    fa, ba = np.ascontiguousarray(fa, np.int32), np.ascontiguousarray(ba, np.int32)
    n = lib().or_sym(V, ptr(fb), ptr(fa), ptr(bb), ptr(ba), None, None)
    sb = np.zeros(V + 1, np.int64)
    sa = np.zeros(max(n, 1), np.int32)
    lib().or_sym(V, ptr(fb), ptr(fa), ptr(bb), ptr(ba), ptr(sb), ptr(sa))
    return sb, sa[:n]


def wcc(V, beg, adj):
    out = np.zeros(max(V, 1), np.int32)
    lib().or_wcc(V, ptr(np.ascontiguousarray(beg, np.int64)), ptr(np.ascontiguousarray(adj, np.int32)), ptr(out))
    return out[:V]


def scc(V, beg, adj):
    out = np.zeros(max(V, 1), np.int32)
    lib().or_scc(V, ptr(np.ascontiguousarray(beg, np.int64)), ptr(np.ascontiguousarray(adj, np.int32)), ptr(out))
    return out[:V]


def dag(V, beg, adj, scc_lab):
    beg = np.ascontiguousarray(beg, np.int64)
    adj = np.ascontiguousarray(adj, np.int32)
    s = np.ascontiguousarray(scc_lab, np.int32)
    n = lib().or_dag(V, ptr(beg), ptr(adj), ptr(s), None)
    out = np.zeros(max(n, 1), np.int64)
    lib().or_dag(V, ptr(beg), ptr(adj), ptr(s), ptr(out))
    return out[:n]


def bicc(V, sb, sa, scc_lab):
    sb = np.ascontiguousarray(sb, np.int64)
    sa = np.ascontiguousarray(sa, np.int32)
    s = np.ascontiguousarray(scc_lab, np.int32)
    n = lib().or_bicc(V, ptr(sb), ptr(sa), ptr(s), None, None, None, None)
    k1 = np.zeros(max(n, 1), np.int32)
    k2 = np.zeros(max(n, 1), np.int32)
    v = np.zeros(max(n, 1), np.int32)
    ap = np.zeros(max(V, 1), np.uint8)
    lib().or_bicc(V, ptr(sb), ptr(sa), ptr(s), ptr(k1), ptr(k2), ptr(v), ptr(ap))
    t = np.stack([k1[:n], k2[:n], v[:n]], axis=1).astype(np.int64)
    return t, ap[:V].astype(bool)


def bfs(V, beg, adj, sources):
    s = np.ascontiguousarray(sources, np.int32)
    out = np.zeros(max(V, 1), np.int32)
    lib().or_bfs(V, ptr(np.ascontiguousarray(beg, np.int64)), ptr(np.ascontiguousarray(adj, np.int32)), ptr(s),
                 len(s), ptr(out))
    return out[:V]


def sssp(V, beg, adj, sources, w=None):
    s = np.ascontiguousarray(sources, np.int32)
    out = np.zeros(max(V, 1), np.uint64)
    wp = None if w is None else np.ascontiguousarray(w, np.uint32)
    lib().or_sssp(V, ptr(np.ascontiguousarray(beg, np.int64)), ptr(np.ascontiguousarray(adj, np.int32)), ptr(wp),
                  ptr(s), len(s), ptr(out))
    return out[:V]


def edge_weight(u, v):
    return int(lib().or_edge_weight(u, v))


def apply_batch(V, beg, adj, u, v, ins):
    beg = np.ascontiguousarray(beg, np.int64)
    adj = np.ascontiguousarray(adj, np.int32)
    u = np.ascontiguousarray(u, np.int32)
    v = np.ascontiguousarray(v, np.int32)
    ins = np.ascontiguousarray(ins, np.uint8)
    nb = np.zeros(V + 1, np.int64)
    na = np.zeros(len(adj) + len(u) + 1, np.int32)
    ni, nd = _I64(), _I64()
    E = lib().or_apply_batch(V, ptr(beg), ptr(adj), ptr(u), ptr(v), ptr(ins), len(u), ptr(nb), ptr(na),
                             ctypes.byref(ni), ctypes.byref(nd))
    return nb, na[:E].copy(), ni.value, nd.value


class Layers:
    """Canonical layers of a graph computed by the C restatement (forward CSR with sorted rows)."""

    def __init__(self, V, fb, fa):
        self.V = V
        self.fb = np.ascontiguousarray(fb, np.int64)
        self.fa = np.ascontiguousarray(fa, np.int32)
        self.bb, self.ba = transpose(V, self.fb, self.fa)
        self.sb, self.sa = sym(V, self.fb, self.fa, self.bb, self.ba)
        self.wcc = wcc(V, self.fb, self.fa)
        self.scc = scc(V, self.fb, self.fa)
        self.dag = dag(V, self.fb, self.fa, self.scc)
        self.blocks, self.ap = bicc(V, self.sb, self.sa, self.scc)


# ---------------------------------------------------------------------------------------------
# the reference itself
# ---------------------------------------------------------------------------------------------

class RefGIR:
    """The reference GIR (built from its sources) on host memory."""

    def __init__(self, V=None, fb=None, fa=None, bb=None, ba=None, directory=None):
        R = ref()
        if directory is not None:
            self.h = R.ref_load(directory.encode())
        else:
            arrs = [np.ascontiguousarray(x, np.int32) for x in (fb, fa, bb, ba)]
            self._keep = arrs
            self.h = R.ref_create(V, len(arrs[1]), *[ptr(x) for x in arrs])
        self.V = R.ref_vertex_count(self.h)

    def close(self):
        if self.h:
            ref().ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def build(self, mask=7):
        ref().ref_build(self.h, mask)

    def out_csr(self):
        """Current edges (getDirectedOutNeighbors), every row sorted: the reference lists a
        vertex's inserted edges after its base edges (gir_iter.h:8-72)."""
        n = ref().ref_out_csr(self.h, None, None)
        beg = np.zeros(self.V + 1, np.int64)
        adj = np.zeros(max(n, 1), np.int32)
        ref().ref_out_csr(self.h, ptr(beg), ptr(adj))
        return beg, sort_rows(beg, adj[:n])

    def und_csr(self):
        n = ref().ref_und_csr(self.h, None, None)
        beg = np.zeros(self.V + 1, np.int64)
        adj = np.zeros(max(n, 1), np.int32)
        ref().ref_und_csr(self.h, ptr(beg), ptr(adj))
        return beg, sort_rows(beg, adj[:n])

    def bfs(self, s):
        out = np.zeros(max(self.V, 1), np.int32)
        ref().ref_bfs(self.h, s, ptr(out))
        return out[:self.V]

    def bc(self, sources):
        """GIR::bc over the sources (float64[V])."""
        s = np.ascontiguousarray(sources, np.int32)
        out = np.zeros(max(self.V, 1), np.float64)
        ref().ref_bc(self.h, ptr(s), len(s), ptr(out))
        return out[:self.V]

    def inc_track(self, source, weighted):
        """GIR::trackIncremental."""
        ref().ref_inc_track(self.h, int(source), 1 if weighted else 0)

    def inc_update(self, weighted):
        """GIR::updateIncremental."""
        ref().ref_inc_update(self.h, 1 if weighted else 0)

    def inc_dist(self, weighted):
        """GIR::incDist of every vertex (uint64[V])."""
        out = np.zeros(max(self.V, 1), np.uint64)
        ref().ref_inc_dist(self.h, 1 if weighted else 0, ptr(out))
        return out[:self.V]

    def reachable(self, u, v):
        """GIR::reachable for every pair (after the SCC layer is built)."""
        u = np.ascontiguousarray(u, np.int32)
        v = np.ascontiguousarray(v, np.int32)
        out = np.zeros(max(len(u), 1), np.uint8)
        ref().ref_reachable(self.h, ptr(u), ptr(v), len(u), ptr(out))
        return out[:len(u)].astype(bool)

    def sssp(self, s, delta=16):
        out = np.zeros(max(self.V, 1), np.uint64)
        ref().ref_sssp(self.h, s, delta, ptr(out))
        return out[:self.V]

    def bfs_two_level(self, s):
        """GIR::bfsTwoLevel (the DAG wavefront; needs the layers built)."""
        out = np.zeros(max(self.V, 1), np.int32)
        ref().ref_bfs_two_level(self.h, s, ptr(out))
        return out[:self.V]

    def sssp_two_level(self, s, delta=16):
        """GIR::ssspTwoLevel."""
        out = np.zeros(max(self.V, 1), np.uint64)
        ref().ref_sssp_two_level(self.h, s, delta, ptr(out))
        return out[:self.V]

    def apply_batch(self, u, v, ins):
        u = np.ascontiguousarray(u, np.int32)
        v = np.ascontiguousarray(v, np.int32)
        ins = np.ascontiguousarray(ins, np.uint8)
        ref().ref_apply_batch(self.h, ptr(u), ptr(v), ptr(ins), len(u))

    def ingest_batch(self, u, v, ins):
        """GIR::ingestBatch: edge store and incremental logs only (layers wait for sync)."""
        u = np.ascontiguousarray(u, np.int32)
        v = np.ascontiguousarray(v, np.int32)
        ins = np.ascontiguousarray(ins, np.uint8)
        ref().ref_ingest_batch(self.h, ptr(u), ptr(v), ptr(ins), len(u))

    def sync(self):
        """GIR::sync: the layers catch up with the ingested batches."""
        ref().ref_sync(self.h)

    def synced(self):
        return bool(ref().ref_synced(self.h))

    def update_edge(self, u, v, insert, undirected=False):
        ref().ref_update_edge(self.h, u, v, int(insert), int(undirected))

    def scc_raw(self):
        out = np.zeros(max(self.V, 1), np.int32)
        ref().ref_scc_raw(self.h, ptr(out))
        return out[:self.V]

    def wcc_raw(self):
        out = np.zeros(max(self.V, 1), np.int32)
        ref().ref_wcc_raw(self.h, ptr(out))
        return out[:self.V]

    def scc(self):
        return canon_labels(self.scc_raw())

    def wcc(self):
        return canon_labels(self.wcc_raw())

    def dag(self):
        """Condensation edges as sorted canonical keys (min vertex of source SCC << 32 | of target)."""
        n = ref().ref_dag_raw(self.h, None, None)
        a = np.zeros(max(n, 1), np.int32)
        b = np.zeros(max(n, 1), np.int32)
        ref().ref_dag_raw(self.h, ptr(a), ptr(b))
        raw = self.scc_raw()
        canon = canon_labels(raw)
        # raw scc id -> min vertex
        top = int(max(raw.max(initial=0), a[:n].max(initial=0), b[:n].max(initial=0))) + 1
        m = np.full(top, -1, np.int64)
        m[raw] = canon
        return np.unique((m[a[:n]] << 32) | m[b[:n]])

    def blocks(self):
        nbk = _I64()
        n = ref().ref_blocks(self.h, None, None, ctypes.byref(nbk))
        beg = np.zeros(nbk.value + 1, np.int64)
        verts = np.zeros(max(n, 1), np.int32)
        ref().ref_blocks(self.h, ptr(beg), ptr(verts), ctypes.byref(nbk))
        return canon_blocks_csr(beg, verts[:n])

    def ap(self):
        out = np.zeros(max(self.V, 1), np.uint8)
        ref().ref_ap(self.h, ptr(out))
        return out[:self.V].astype(bool)
