"""GIR-B200: the data-parallel hot path of GIR (graph intermediate representation) on one B200.

The graph lives in HBM as forward / backward / symmetrized slack CSRs; the WCC, SCC +
condensation DAG and per-SCC block-cut layers, BFS and Delta-stepping SSSP, and batched edge
updates run as CUDA kernels for sm_100a behind the gir_dev_* C ABI (include/gir_dev.h).
Import name: importlib.import_module("graph-intermedia-representation_b200").
"""
from . import graphs, native
from .gir import GIR, DeviceGraph
from .native import GirError

__all__ = ["GIR", "DeviceGraph", "GirError", "graphs", "native"]
