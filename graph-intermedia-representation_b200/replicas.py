"""Replicas on several GPUs of one node: every rank (one process per GPU) holds the whole graph
in its own HBM, so BFS / SSSP queries are independent units split across the ranks with no
collective on the traversal path. An update batch must change every replica identically: rank 0
owns the batch and broadcasts it (length, then the u / v / insert arrays), every rank applies the
same normalised batch, and a checksum of the layers, all-gathered, shows that the replicas still
agree. The reference runs on one host with OpenMP and has no counterpart of this module.

Works with any process group: NCCL between GPUs (tensors go through the GPU of the rank) or gloo
on CPUs. The graph object only needs apply_batch(u, v, ins), labels(which) and counts()["E"].
"""
import numpy as np
import torch
import torch.distributed as dist

from . import native


def shard(items, rank, world):
    """The contiguous share of `items` (a sequence or array) that `rank` of `world` runs."""
    n = len(items)
    lo = (n * rank) // world
    hi = (n * (rank + 1)) // world
    return items[lo:hi]


def layer_checksum(labels):
    """64-bit checksum of a list of int32 label arrays (order-sensitive, so two replicas agree
    only when every label agrees)."""
    h = np.uint64(1469598103934665603)
    mult = np.uint64(1099511628211)
    for a in labels:
        a = np.ascontiguousarray(a, np.int64).astype(np.uint64)
        idx = np.arange(1, len(a) + 1, dtype=np.uint64)
        with np.errstate(over="ignore"):
            part = np.bitwise_xor.reduce((a + np.uint64(0x9E3779B97F4A7C15)) * (idx * mult), initial=np.uint64(0))
            h = (h ^ part) * mult + np.uint64(len(a))
    return int(h & np.uint64((1 << 63) - 1))


class Replicas:
    """One rank's view of the replica set (call collectively on every rank, in the same order)."""

    def __init__(self, graph, group=None, device=None):
        self.g = graph
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        backend = dist.get_backend(group)
        self.device = torch.device(device) if device is not None else (
            torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu"))

    def _bcast(self, t):
        dist.broadcast(t, src=0, group=self.group)
        return t

    def broadcast_batch(self, u=None, v=None, ins=None):
        """Rank 0's batch on every rank (the other ranks pass nothing)."""
        n = torch.zeros(1, dtype=torch.int64, device=self.device)
        if self.rank == 0:
            n[0] = len(u)
        n = int(self._bcast(n).item())
        if self.rank == 0:
            tu = torch.as_tensor(np.ascontiguousarray(u, np.int32)).to(self.device)
            tv = torch.as_tensor(np.ascontiguousarray(v, np.int32)).to(self.device)
            ti = torch.as_tensor(np.ascontiguousarray(ins, np.uint8)).to(self.device)
        else:
            tu = torch.empty(n, dtype=torch.int32, device=self.device)
            tv = torch.empty(n, dtype=torch.int32, device=self.device)
            ti = torch.empty(n, dtype=torch.uint8, device=self.device)
        for t in (tu, tv, ti):
            self._bcast(t)
        return tu.cpu().numpy(), tv.cpu().numpy(), ti.cpu().numpy()

    def apply_batch(self, u=None, v=None, ins=None):
        """Broadcasts rank 0's batch and applies it to this rank's replica."""
        u, v, ins = self.broadcast_batch(u, v, ins)
        self.g.apply_batch(u, v, ins)
        return len(u)

    def sources(self, srcs):
        """This rank's share of the query sources."""
        return shard(srcs, self.rank, self.world)

    def check_agree(self, which=(native.LABEL_WCC, native.LABEL_SCC)):
        """All-gathers a checksum of the edge count and the given layers; raises if any two
        replicas differ."""
        e = np.array([self.g.counts()["E"]], np.int64)
        c = layer_checksum([e] + [self.g.labels(w) for w in which])
        t = torch.tensor([c], dtype=torch.int64, device=self.device)
        out = [torch.zeros_like(t) for _ in range(self.world)]
        dist.all_gather(out, t, group=self.group)
        vals = [int(x.item()) for x in out]
        if len(set(vals)) != 1:
            raise RuntimeError(f"replicas disagree after the batch: layer checksums {vals}")
        return vals[0]
