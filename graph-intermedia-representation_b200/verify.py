"""Size-independent checks of results on the device (torch), for graphs too large for the CPU
oracle: certificates that hold for the exact answer and fail for almost any wrong one.

  bfs_levels    every edge (u, v) from a reached u reaches v with level(v) <= level(u) + 1;
                every reached non-source v has an in-edge from level(v) - 1; sources are 0
  sssp_dists    the same with distances and weights: dist(v) <= dist(u) + w(u, v) on every
                edge, and every reached non-source has a tight in-edge (dist(u) + w = dist(v))
  wcc_labels    labels are canonical (label(v) <= v, labels are their own labels) and agree
                along every edge
  scc_dag       every edge between two SCCs is a condensation edge and goes forward in rank
                (so no cycle crosses SCCs); labels are canonical

Edges are streamed in chunks, so only the per-vertex arrays and one chunk are on the GPU. The
weights of hash mode are GIR::edgeWeight (gir_query.cpp:50-54), computed here in 64-bit integer
arithmetic. Each check returns the number of violations (0 = passed).
"""
import numpy as np
import torch

CHUNK = 1 << 26
_M31 = (1 << 31) - 1


def _lsr33(x):
    return (x >> 33) & _M31


def edge_weight(u, v):
    """GIR::edgeWeight(u, v) for int64 tensors u, v: 1 + mix64(u << 32 | v) % 100."""
    x = (u << 32) | (v & 0xFFFFFFFF)
    x = x ^ _lsr33(x)
    x = x * -49064778989728563  # 0xff51afd7ed558ccd as a signed 64-bit value (wrapping multiply)
    x = x ^ _lsr33(x)
    x = x * -4265267296055464877  # 0xc4ceb9fe1a85ec53
    x = x ^ _lsr33(x)
    hi = (x >> 32) & 0xFFFFFFFF
    lo = x & 0xFFFFFFFF
    return 1 + ((hi % 100) * 96 + lo % 100) % 100  # (2^32 mod 100 = 96)


def _edges(beg, adj, device):
    """(u, v) int64 chunks of a CSR given as host arrays or tensors."""
    beg = torch.as_tensor(np.asarray(beg) if not torch.is_tensor(beg) else beg).to(device, torch.int64)
    adj_t = adj if torch.is_tensor(adj) else torch.from_numpy(np.ascontiguousarray(adj))
    E = int(beg[-1].item())
    V = beg.numel() - 1
    for e0 in range(0, E, CHUNK):
        e1 = min(E, e0 + CHUNK)
        idx = torch.arange(e0, e1, device=device, dtype=torch.int64)
        u = torch.searchsorted(beg, idx, right=True) - 1
        v = adj_t[e0:e1].to(device, torch.int64)
        yield u.clamp_(0, V - 1), v


def bfs_levels(beg, adj, sources, level, device="cuda"):
    lv = torch.as_tensor(level).to(device, torch.int64)
    bad = 0
    src = torch.as_tensor(np.asarray(sources, np.int64)).to(device)
    bad += int((lv[src] != 0).sum().item())
    has_parent = torch.zeros_like(lv, dtype=torch.bool)
    has_parent[src] = True
    for u, v in _edges(beg, adj, device):
        lu, lw = lv[u], lv[v]
        r = lu >= 0
        bad += int((r & ((lw < 0) | (lw > lu + 1))).sum().item())
        tight = r & (lw == lu + 1)
        has_parent[v[tight]] = True
    bad += int(((lv > 0) & ~has_parent).sum().item())
    return bad


def sssp_dists(beg, adj, sources, dist, device="cuda"):
    """`dist` as uint64 numpy or int64 tensor (UINT64_MAX / -1 = unreachable); hash weights."""
    d = torch.as_tensor(np.asarray(dist).view(np.int64) if not torch.is_tensor(dist) else dist).to(device, torch.int64)
    bad = 0
    src = torch.as_tensor(np.asarray(sources, np.int64)).to(device)
    bad += int((d[src] != 0).sum().item())
    has_parent = torch.zeros_like(d, dtype=torch.bool)
    has_parent[src] = True
    for u, v in _edges(beg, adj, device):
        du, dv = d[u], d[v]
        w = edge_weight(u, v)
        r = du >= 0
        cand = du + w
        bad += int((r & ((dv < 0) | (dv > cand))).sum().item())
        tight = r & (dv == cand)
        has_parent[v[tight]] = True
    bad += int(((d > 0) & ~has_parent).sum().item())
    return bad


def wcc_labels(beg, adj, label, device="cuda"):
    lab = torch.as_tensor(label).to(device, torch.int64)
    ids = torch.arange(lab.numel(), device=device)
    bad = int(((lab > ids) | (lab[lab] != lab)).sum().item())
    for u, v in _edges(beg, adj, device):
        bad += int((lab[u] != lab[v]).sum().item())
    return bad


def scc_dag(beg, adj, scc, rank, dag_src, dag_dst, device="cuda"):
    s = torch.as_tensor(scc).to(device, torch.int64)
    rk = torch.as_tensor(rank).to(device, torch.int64)
    ids = torch.arange(s.numel(), device=device)
    bad = int(((s > ids) | (s[s] != s)).sum().item())
    keys = torch.as_tensor(np.asarray(dag_src, np.int64) << 32 | np.asarray(dag_dst, np.int64)).to(device)
    keys, _ = torch.sort(keys)
    for u, v in _edges(beg, adj, device):
        cross = s[u] != s[v]
        a, b = s[u][cross], s[v][cross]
        bad += int((rk[a] >= rk[b]).sum().item())
        k = (a << 32) | b
        pos = torch.searchsorted(keys, k).clamp_(max=max(keys.numel() - 1, 0))
        bad += int((keys.numel() == 0 and k.numel() > 0)) if keys.numel() == 0 else int((keys[pos] != k).sum().item())
    return bad
