"""Synthetic workloads of the benchmark and tests, built by libgir_gen.so.

A Graph holds the four int32 arrays of the reference's four-file CSR (fw_begin, fw_adjacent,
bw_begin, bw_adjacent; gir_constructor/graph.h:14-18) plus optional uint32 forward weights.

Named workloads (shapes of the reference's benchmark graphs; the datasets themselves are not
available, so seeded synthetic graphs of the same shape stand in for them):
  rmat_s16      R-MAT scale 16, 2^20 draws, a,b,c = .57/.19/.19, seed 1 (65,536 vertices, isolated
                vertices kept), weights U[1,255]
  rmat_lj       4.8M vertices / 69M distinct edges, R-MAT drawn at scale 23 with ids >= V
                rejected, ids permuted, seed 3 (stands in for soc-LiveJournal1), weights U[1,255]
  lattice       side x side 4-neighbour lattice, 5% edges removed, 0.1% Pareto(1.5) long-range
                edges, weights 100 x length + U[0,50] (stands in for road graphs)
  rmat_tw       41.6M vertices / 1.47B edges, R-MAT, seed 5 (stands in for twitter), U[1,1023]
"""
import ctypes
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import native


@dataclass
class Graph:
    V: int
    fw_beg: np.ndarray
    fw_adj: np.ndarray
    bw_beg: np.ndarray
    bw_adj: np.ndarray
    w: Optional[np.ndarray] = None
    name: str = ""

    @property
    def E(self):
        return int(self.fw_beg[-1])

    def fw_beg64(self):
        return self.fw_beg.astype(np.int64)

    def bw_beg64(self):
        return self.bw_beg.astype(np.int64)


def _check(rc):
    if rc != 0:
        raise RuntimeError(native.gen_lib().gir_gen_last_error().decode())


def _take(p, n, dtype):
    lib = native.gen_lib()
    arr = np.ctypeslib.as_array(p, shape=(max(n, 1),))[:n].astype(dtype, copy=True)
    lib.gir_gen_free(ctypes.cast(p, ctypes.c_void_p))
    return arr


def rmat_edges(scale, V, n_draws, target_unique, a, b, c, seed, permute):
    lib = native.gen_lib()
    n = ctypes.c_int64(0)
    s = ctypes.POINTER(ctypes.c_int32)()
    t = ctypes.POINTER(ctypes.c_int32)()
    _check(lib.gir_gen_rmat(scale, V, n_draws, target_unique, a, b, c, seed, int(permute), ctypes.byref(n),
                            ctypes.byref(s), ctypes.byref(t)))
    return _take(s, n.value, np.int32), _take(t, n.value, np.int32)


def from_edges(V, src, dst, w=None, name=""):
    """Forward + backward CSR of an edge list (rows sorted); graph::fromEdges (graph.cpp:123-136)."""
    lib = native.gen_lib()
    src = np.ascontiguousarray(src, dtype=np.int32)
    dst = np.ascontiguousarray(dst, dtype=np.int32)
    n = len(src)
    fb = np.zeros(V + 1, np.int32)
    fa = np.zeros(max(n, 1), np.int32)
    bb = np.zeros(V + 1, np.int32)
    ba = np.zeros(max(n, 1), np.int32)
    wf = np.zeros(max(n, 1), np.uint32) if w is not None else None
    w_in = np.ascontiguousarray(w, dtype=np.uint32) if w is not None else None
    _check(lib.gir_gen_csr(V, n, native.ptr(src), native.ptr(dst), native.ptr(w_in), native.ptr(fb), native.ptr(fa),
                           native.ptr(bb), native.ptr(ba), native.ptr(wf)))
    return Graph(V, fb, fa[:n], bb, ba[:n], None if wf is None else wf[:n], name)


def uniform_weights(g, lo, hi, seed):
    lib = native.gen_lib()
    w = np.zeros(max(g.E, 1), np.uint32)
    lib.gir_gen_uniform_weights(g.V, native.ptr(g.fw_beg), native.ptr(g.fw_adj), lo, hi, seed, native.ptr(w))
    return w[:g.E]


def sources(V, n, seed):
    out = np.zeros(max(n, 1), np.int32)
    native.gen_lib().gir_gen_sources(V, n, seed, native.ptr(out))
    return out[:n]


def sources_with_edges(g, n, seed):
    """n sources drawn uniformly among the vertices with at least one out-edge (as Graph500
    draws its search keys), so a query is never trivially empty."""
    cand = np.nonzero(np.diff(g.fw_beg) > 0)[0].astype(np.int32)
    if len(cand) == 0:
        return sources(g.V, n, seed)
    lib = native.gen_lib()
    return np.array([cand[lib.gir_gen_hash3(seed, i, 98) % len(cand)] for i in range(n)], np.int32)


def updates(g, n_ins, n_del, seed):
    """A batch of n_ins uniform inserts and n_del deletions sampled from g's edges, shuffled."""
    n = n_ins + n_del
    u = np.zeros(max(n, 1), np.int32)
    v = np.zeros(max(n, 1), np.int32)
    ins = np.zeros(max(n, 1), np.uint8)
    native.gen_lib().gir_gen_updates(g.V, native.ptr(g.fw_beg), native.ptr(g.fw_adj), n_ins, n_del, seed,
                                     native.ptr(u), native.ptr(v), native.ptr(ins))
    return u[:n], v[:n], ins[:n]


def hash3(seed, a, b):
    return native.gen_lib().gir_gen_hash3(seed, a, b)


def rmat(scale, V=None, n_draws=None, target_unique=0, seed=1, permute=False, weights=(1, 255), name="rmat"):
    V = (1 << scale) if V is None else V
    n_draws = 16 * (1 << scale) if n_draws is None else n_draws
    s, t = rmat_edges(scale, V, n_draws, target_unique, 0.57, 0.19, 0.19, seed, permute)
    g = from_edges(V, s, t, name=name)
    if weights:
        g.w = uniform_weights(g, weights[0], weights[1], seed)
    return g


def rmat_s16():
    """R-MAT scale 16, 1,048,576 draws, seed 1, weights U[1,255]."""
    return rmat(16, seed=1, name="rmat_s16")


def rmat_lj(V=4_800_000, E=69_000_000, seed=3):
    """4.8M vertices / 69M distinct edges, ids permuted, seed 3, weights U[1,255]."""
    return rmat(23, V=V, n_draws=0, target_unique=E, seed=seed, permute=True, name="rmat_lj")


def rmat_tw(V=41_652_231, E=1_468_365_182, seed=5):
    """41.6M vertices / 1.47B edges, seed 5, weights U[1,1023]."""
    return rmat(26, V=V, n_draws=0, target_unique=E, seed=seed, permute=True, weights=(1, 1023), name="rmat_tw")


def lattice(side=4900, remove=0.05, longrange=0.001, shape=1.5, seed=4):
    lib = native.gen_lib()
    n = ctypes.c_int64(0)
    s = ctypes.POINTER(ctypes.c_int32)()
    t = ctypes.POINTER(ctypes.c_int32)()
    w = ctypes.POINTER(ctypes.c_uint32)()
    _check(lib.gir_gen_lattice(side, remove, longrange, shape, seed, ctypes.byref(n), ctypes.byref(s),
                               ctypes.byref(t), ctypes.byref(w)))
    src, dst, wt = _take(s, n.value, np.int32), _take(t, n.value, np.int32), _take(w, n.value, np.uint32)
    return from_edges(side * side, src, dst, wt, name=f"lattice_{side}")


def write_four_files(g, directory):
    """Writes g in the reference's on-disk layout; `directory` ends with '/'."""
    _check(native.gen_lib().gir_write_four_files(directory.encode(), g.V, native.ptr(g.fw_beg), native.ptr(g.fw_adj),
                                                  native.ptr(g.bw_beg), native.ptr(g.bw_adj)))
