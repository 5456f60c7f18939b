"""The replica logic of several GPUs, run as two gloo ranks on the CPU: rank 0's update batches
reach every rank, the source split covers every source once, the replicas' layer checksums
agree after every batch, and a replica that drifts (a mistake planted in rank 1's CPU stand-in,
which applies one extra edge) is caught by the checksum exchange on every rank."""
import importlib
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


class OracleReplica:
    """CPU stand-in for one rank's DeviceGraph: the oracle's batch merge and layers."""

    def __init__(self, orc, V, fb, fa):
        self.orc, self.V, self.fb, self.fa = orc, V, fb, fa

    def apply_batch(self, u, v, ins):
        self.fb, self.fa, _, _ = self.orc.apply_batch(self.V, self.fb, self.fa, u, v, ins)

    def counts(self):
        return {"E": len(self.fa)}

    def labels(self, which):
        L = self.orc.Layers(self.V, self.fb, self.fa)
        return L.wcc if which == 0 else L.scc


def _worker(rank, world, port, out_dir):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import torch.distributed as dist
    import oracle
    pkg = importlib.import_module("graph-intermedia-representation_b200")
    from importlib import import_module
    replicas = import_module("graph-intermedia-representation_b200.replicas")
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        g = pkg.graphs.rmat(9, seed=4, weights=None)
        fb, fa = oracle.normalize(g.V, g.fw_beg, g.fw_adj)
        rep = replicas.Replicas(OracleReplica(oracle, g.V, fb, fa))
        mine = rep.sources(np.arange(101))
        sums = []
        for k in range(3):
            if rank == 0:
                gg = pkg.graphs.Graph(g.V, rep.g.fb.astype(np.int32), rep.g.fa, None, None)
                u, v, ins = pkg.graphs.updates(gg, 40, 40, 10 + k)
                n = rep.apply_batch(u, v, ins)
            else:
                n = rep.apply_batch()
            sums.append((n, rep.check_agree()))
        if rank == 1:  # planted drift: one edge only this replica has
            rep.g.apply_batch(np.array([0], np.int32), np.array([g.V - 1], np.int32), np.array([1], np.uint8))
        caught = False
        try:
            rep.check_agree()
        except RuntimeError:
            caught = True
        np.save(os.path.join(out_dir, f"r{rank}.npy"),
                np.array([len(mine), int(mine[0]) if len(mine) else -1, int(caught)] + [x for s in sums for x in s],
                         dtype=object), allow_pickle=True)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_replicas_two_gloo_ranks(tmp_path, orc):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0
    r0 = np.load(tmp_path / "r0.npy", allow_pickle=True)
    r1 = np.load(tmp_path / "r1.npy", allow_pickle=True)
    assert r0[0] + r1[0] == 101 and r0[1] == 0 and r1[1] == r0[0]  # contiguous split, every source once
    assert r0[2] == 1 and r1[2] == 1  # the drift is seen on both ranks
    assert list(r0[3:]) == list(r1[3:])  # same batch sizes and checksums after every batch
    assert all(n > 0 for n in r0[3::2])
