"""ctypes bindings of the two native libraries built in this directory.

libgir_b200.so  -- the CUDA library behind the gir_dev_* C ABI (include/gir_dev.h)
libgir_gen.so   -- host-only synthetic-input generators (include/gir_gen.h)

Loading fails loudly: there is no fallback implementation of any gir_dev_* call.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

GIR_OK = 0
ERRORS = {
    1: "GIR_ERR_INVALID", 2: "GIR_ERR_CUDA", 3: "GIR_ERR_OOM", 4: "GIR_ERR_FILE", 5: "GIR_ERR_MALFORMED",
    6: "GIR_ERR_STATE", 7: "GIR_ERR_TIMEOUT", 8: "GIR_ERR_CAPACITY", 9: "GIR_ERR_NODEVICE",
}
LAYER_WCC, LAYER_SCC, LAYER_BCT, LAYER_ALL = 1, 2, 4, 7
LABEL_WCC, LABEL_SCC, LABEL_BLOCK, LABEL_BCNT, LABEL_SCC_RANK = 0, 1, 2, 3, 4
WEIGHT_HASH, WEIGHT_STORED = 0, 1
SCHEDULE_FIXED, SCHEDULE_LEARNED = 0, 1
(PARAM_ALPHA, PARAM_BETA, PARAM_DELTA, PARAM_BLOCK, PARAM_SMALL_DEG, PARAM_LARGE_DEG, PARAM_CTAS_PER_SM,
 PARAM_PROFILE, PARAM_PIVOT, PARAM_LANE_BITS, PARAM_LANE_ORDER) = range(11)
SCHED_IN, SCHED_HID, SCHED_OUT = 8, 32, 12

# Every symbol include/gir_dev.h declares (checked by the CPU test suite).
DEV_SYMBOLS = (
    "gir_dev_create", "gir_dev_load", "gir_dev_destroy", "gir_dev_last_error", "gir_dev_counts", "gir_dev_build",
    "gir_dev_get_labels", "gir_dev_get_dag", "gir_dev_get_blocks", "gir_dev_get_csr", "gir_dev_has_edges",
    "gir_dev_bfs", "gir_dev_bfs_sets", "gir_dev_sssp", "gir_dev_sssp_sets", "gir_dev_apply_batch",
    "gir_dev_set_weight_rule", "gir_dev_batch_stats", "gir_dev_set_schedule", "gir_dev_set_param",
    "gir_dev_get_param", "gir_dev_query_stats", "gir_dev_stream", "gir_dev_sched_set_weights",
    "gir_dev_sched_get_weights", "gir_dev_sched_param_count", "gir_dev_sched_train", "gir_dev_sched_forward",
    "gir_dev_sched_grad", "gir_dev_bfs_noalloc", "gir_dev_sched_trace", "gir_dev_sched_delta_choices",
    "gir_dev_batch_times", "gir_dev_batch_plan", "gir_dev_autotune", "gir_dev_reachable", "gir_dev_bc",
    "gir_dev_inc_track", "gir_dev_inc_update", "gir_dev_inc_dist", "gir_dev_single_stats",
    "gir_dev_ingest_batch", "gir_dev_sync", "gir_dev_synced",
)
GEN_SYMBOLS = (
    "gir_gen_last_error", "gir_gen_free", "gir_gen_hash3", "gir_gen_rmat", "gir_gen_lattice", "gir_gen_csr",
    "gir_gen_uniform_weights", "gir_gen_sources", "gir_gen_updates", "gir_write_four_files",
)


class GirError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class QueryStats(ctypes.Structure):
    _fields_ = [("edges", ctypes.c_int64), ("reached", ctypes.c_int64), ("iterations", ctypes.c_int64),
                ("bottom_up", ctypes.c_int64), ("launches", ctypes.c_int64), ("kernel_ms", ctypes.c_double),
                ("total_ms", ctypes.c_double), ("main_ms", ctypes.c_double), ("main_launches", ctypes.c_int64),
                ("persistent_levels", ctypes.c_int64)]


_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_I32 = ctypes.c_int32
_dev = None
_gen = None


def lib_path(name):
    return os.path.join(HERE, name)


def dev_lib():
    """The CUDA library (raises if it was not built)."""
    global _dev
    if _dev is None:
        path = lib_path("libgir_b200.so")
        if not os.path.exists(path):
            raise ImportError(f"{path} is missing: build it with `make -C {HERE}` (no CPU fallback exists)")
        lib = ctypes.CDLL(path)
        sig = {
            "gir_dev_create": [_P, _P, _P, _P, _I64, _I64, _P, ctypes.POINTER(_P)],
            "gir_dev_load": [ctypes.c_char_p, ctypes.POINTER(_P)],
            "gir_dev_destroy": [_P],
            "gir_dev_counts": [_P] + [ctypes.POINTER(_I64)] * 6,
            "gir_dev_build": [_P, ctypes.c_uint],
            "gir_dev_get_labels": [_P, ctypes.c_int, _P],
            "gir_dev_get_dag": [_P, _P, _P, _I64, ctypes.POINTER(_I64)],
            "gir_dev_get_blocks": [_P, _P, _I64, ctypes.POINTER(_I64)],
            "gir_dev_get_csr": [_P, ctypes.c_int, _P, _P, _I64, ctypes.POINTER(_I64)],
            "gir_dev_has_edges": [_P, ctypes.c_int, _P, _P, _I64, _P],
            "gir_dev_bfs": [_P, _P, _I64, _P],
            "gir_dev_bfs_sets": [_P, _P, _P, _I64, _P],
            "gir_dev_sssp": [_P, _P, _I64, ctypes.c_uint64, ctypes.c_int, _P],
            "gir_dev_sssp_sets": [_P, _P, _P, _I64, ctypes.c_uint64, ctypes.c_int, _P],
            "gir_dev_apply_batch": [_P, _P, _P, _P, _I64],
            "gir_dev_ingest_batch": [_P, _P, _P, _P, _I64],
            "gir_dev_sync": [_P],
            "gir_dev_synced": [_P, _P],
            "gir_dev_set_weight_rule": [_P, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32],
            "gir_dev_batch_stats": [_P] + [ctypes.POINTER(_I64)] * 4,
            "gir_dev_set_schedule": [_P, ctypes.c_int],
            "gir_dev_set_param": [_P, ctypes.c_int, ctypes.c_double],
            "gir_dev_get_param": [_P, ctypes.c_int, ctypes.POINTER(ctypes.c_double)],
            "gir_dev_query_stats": [_P, ctypes.POINTER(QueryStats)],
            "gir_dev_stream": [_P, ctypes.POINTER(_P)],
            "gir_dev_sched_set_weights": [_P, _P, _I64],
            "gir_dev_sched_get_weights": [_P, _P, _I64],
            "gir_dev_sched_train": [_P, _P, _P, _I64, ctypes.c_int, ctypes.c_float, ctypes.POINTER(ctypes.c_float)],
            "gir_dev_sched_forward": [_P, _P, _I64, _P],
            "gir_dev_sched_grad": [_P, _P, _P, _I64, _P, ctypes.POINTER(ctypes.c_float)],
            "gir_dev_bfs_noalloc": [_P, _P, _I64, _I64, ctypes.c_int32, _P, _P],
            "gir_dev_sched_trace": [_P, _P, _P, _I64, ctypes.POINTER(_I64)],
            "gir_dev_sched_delta_choices": [_P],
            "gir_dev_batch_times": [_P, _P],
            "gir_dev_batch_plan": [_P, _P],
            "gir_dev_autotune": [_P, _P, _I64, ctypes.c_int, ctypes.POINTER(ctypes.c_double)],
            "gir_dev_reachable": [_P, _P, _P, _I64, _P],
            "gir_dev_bc": [_P, _P, _I64, _P],
            "gir_dev_inc_track": [_P, _I32, ctypes.c_int],
            "gir_dev_inc_update": [_P, ctypes.c_int],
            "gir_dev_inc_dist": [_P, ctypes.c_int, _P],
            "gir_dev_single_stats": [_P, ctypes.POINTER(_I64), ctypes.POINTER(_I64)],
        }
        for name, args in sig.items():
            f = getattr(lib, name)
            f.argtypes = args
            f.restype = ctypes.c_int
        lib.gir_dev_last_error.argtypes = [_P]
        lib.gir_dev_last_error.restype = ctypes.c_char_p
        lib.gir_dev_sched_param_count.argtypes = []
        lib.gir_dev_sched_param_count.restype = _I64
        _dev = lib
    return _dev


def gen_lib():
    global _gen
    if _gen is None:
        path = lib_path("libgir_gen.so")
        if not os.path.exists(path):
            raise ImportError(f"{path} is missing: build it with `make -C {HERE}`")
        lib = ctypes.CDLL(path)
        pp32 = ctypes.POINTER(ctypes.POINTER(ctypes.c_int32))
        ppu32 = ctypes.POINTER(ctypes.POINTER(ctypes.c_uint32))
        lib.gir_gen_last_error.restype = ctypes.c_char_p
        lib.gir_gen_free.argtypes = [_P]
        lib.gir_gen_hash3.argtypes = [ctypes.c_uint64] * 3
        lib.gir_gen_hash3.restype = ctypes.c_uint64
        lib.gir_gen_rmat.argtypes = [ctypes.c_int, _I64, _I64, _I64, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(_I64), pp32, pp32]
        lib.gir_gen_lattice.argtypes = [_I64, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_uint64,
                                        ctypes.POINTER(_I64), pp32, pp32, ppu32]
        lib.gir_gen_csr.argtypes = [_I64, _I64, _P, _P, _P, _P, _P, _P, _P, _P]
        lib.gir_gen_uniform_weights.argtypes = [_I64, _P, _P, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, _P]
        lib.gir_gen_uniform_weights.restype = None
        lib.gir_gen_sources.argtypes = [_I64, _I64, ctypes.c_uint64, _P]
        lib.gir_gen_sources.restype = None
        lib.gir_gen_updates.argtypes = [_I64, _P, _P, _I64, _I64, ctypes.c_uint64, _P, _P, _P]
        lib.gir_gen_updates.restype = None
        lib.gir_write_four_files.argtypes = [ctypes.c_char_p, _I64, _P, _P, _P, _P]
        _gen = lib
    return _gen


def ptr(a):
    """Data pointer of a numpy array or a torch tensor (host or device), or None."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return a.ctypes.data_as(ctypes.c_void_p)
