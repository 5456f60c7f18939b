"""Size-independent checks of results on the device (torch), for graphs too large for the CPU
oracle. Each returns the number of violations (0 = passed).

  bfs_levels    every edge (u, v) from a reached u reaches v with level(v) <= level(u) + 1;
                every reached non-source v has an in-edge from level(v) - 1; sources are 0.
                Together these pin the exact levels.
  sssp_dists    the same with distances and weights: dist(v) <= dist(u) + w(u, v) on every
                edge, and every reached non-source has a tight in-edge (dist(u) + w = dist(v)).
                With positive weights these pin the exact distances.
  wcc_labels    an independent recomputation of the weakly connected components (hook the
                larger label under the smaller along every edge, then compress, until nothing
                changes), compared label by label with the given canonical labels: exact, so
                both a split and an over-merged component are caught.
  scc_dag       labels canonical; every edge between two classes goes forward in rank (no
                cycle crosses classes, so no two classes belong together); every class is
                strongly connected (the forward and the backward search from its root, each
                staying inside the class, reach all of it); and the condensation edges are
                exactly the distinct class pairs of the edges between classes (a missing or an
                extra key is caught). Together: the exact SCC partition and condensation.
  blocks        necessary conditions of the per-SCC blocks (block-cut forest representation:
                block of every vertex, head articulation point of every block, block count per
                vertex): every block and its head lie in one SCC; every undirected edge inside
                an SCC lies inside one block; a vertex's block count is 1 + the blocks it heads,
                and a head is an articulation point. (That each block is biconnected is not
                checked here; at the 69M-edge size the blocks are compared with the reference
                itself.)

Edges are streamed in chunks, so only the per-vertex arrays and one chunk are on the GPU. The
weights of hash mode are GIR::edgeWeight (gir_query.cpp:50-54), computed here in 64-bit integer
arithmetic.
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
    V = lab.numel()
    ids = torch.arange(V, device=device)
    bad = int(((lab > ids) | (lab[lab] != lab)).sum().item())
    # independent components: parents hooked to the smaller label along every edge, then
    # compressed; the smallest vertex of a component never moves, so this ends with every
    # vertex pointing at its component's smallest id
    m = ids.clone()
    while True:
        before = m.clone()
        for u, v in _edges(beg, adj, device):
            mu, mv = m[u], m[v]
            lo = torch.minimum(mu, mv)
            m.scatter_reduce_(0, mu, lo, "amin")
            m.scatter_reduce_(0, mv, lo, "amin")
            m.scatter_reduce_(0, u, lo, "amin")
            m.scatter_reduce_(0, v, lo, "amin")
        while True:
            mm = m[m]
            if torch.equal(mm, m):
                break
            m = mm
        if torch.equal(m, before):
            break
    bad += int((m != lab).sum().item())
    return bad


def _inside_reach(beg, adj, cls, roots, device, reverse):
    """Vertices reached from `roots` along edges (u -> v, or v -> u with reverse) whose two ends
    have the same class."""
    seen = torch.zeros(cls.numel(), dtype=torch.bool, device=device)
    seen[roots] = True
    while True:
        n0 = int(seen.sum().item())
        for u, v in _edges(beg, adj, device):
            a, b = (v, u) if reverse else (u, v)
            hop = seen[a] & ~seen[b] & (cls[a] == cls[b])
            seen[b[hop]] = True
        if int(seen.sum().item()) == n0:
            return seen


def scc_dag(beg, adj, scc, rank, dag_src, dag_dst, device="cuda"):
    s = torch.as_tensor(scc).to(device, torch.int64)
    rk = torch.as_tensor(rank).to(device, torch.int64)
    ids = torch.arange(s.numel(), device=device)
    bad = int(((s > ids) | (s[s] != s)).sum().item())
    keys = torch.as_tensor(np.asarray(dag_src, np.int64) << 32 | np.asarray(dag_dst, np.int64)).to(device)
    keys = torch.unique(keys)
    cross_keys = []
    for u, v in _edges(beg, adj, device):
        cross = s[u] != s[v]
        a, b = s[u][cross], s[v][cross]
        bad += int((rk[a] >= rk[b]).sum().item())
        cross_keys.append(torch.unique((a << 32) | b))
    want = torch.unique(torch.cat(cross_keys)) if cross_keys else torch.zeros(0, dtype=torch.int64, device=device)
    if want.numel() != keys.numel():
        bad += abs(want.numel() - keys.numel()) + int(want.numel() > 0 and keys.numel() > 0)
    else:
        bad += int((want != keys).sum().item())
    # every class strongly connected: its root reaches all of it and all of it reaches the root
    roots = torch.nonzero(s == ids).flatten()
    for rev in (False, True):
        bad += int((~_inside_reach(beg, adj, s, roots, device, rev)).sum().item())
    return bad


def blocks(sym_beg, sym_adj, scc, label_block, head, bcnt, device="cuda"):
    """See the module text: necessary conditions of the per-SCC block-cut forest."""
    s = torch.as_tensor(scc).to(device, torch.int64)
    blk = torch.as_tensor(label_block).to(device, torch.int64)
    hd = torch.as_tensor(head).to(device, torch.int64)
    cnt = torch.as_tensor(bcnt).to(device, torch.int64)
    V, nb = s.numel(), hd.numel()
    bad = int(((blk < 0) | (blk >= nb)).sum().item())
    if bad:
        return bad
    # every block inside one SCC (its members and its head)
    bscc = torch.full((nb,), -1, dtype=torch.int64, device=device)
    bscc.scatter_reduce_(0, blk, s, "amax", include_self=False)
    bmin = torch.full((nb,), 1 << 62, dtype=torch.int64, device=device)
    bmin.scatter_reduce_(0, blk, s, "amin", include_self=False)
    used = torch.zeros(nb, dtype=torch.bool, device=device)
    used[blk] = True
    bad += int((~used).sum().item())  # every block has a member besides its head
    bad += int((used & (bscc != bmin)).sum().item())
    has_head = hd >= 0
    bad += int((has_head & (s[hd.clamp(min=0)] != bscc)).sum().item())
    # block counts: 1 + blocks headed; heads are articulation points
    headed = torch.bincount(hd[has_head], minlength=V)
    bad += int((cnt != 1 + headed).sum().item())
    bad += int((cnt[hd[has_head]] < 2).sum().item())
    # every undirected edge inside an SCC lies inside one block
    for u, v in _edges(sym_beg, sym_adj, device):
        inside = s[u] == s[v]
        bu, bv = blk[u], blk[v]
        ok = (bu == bv) | (hd[bv] == u) | (hd[bu] == v)
        bad += int((inside & ~ok).sum().item())
    return bad
