"""The decision rules of the single-edge latency path (csrc/single.cu), restated in Python and
checked against the oracle on random graphs. This pins the rules the device searches implement,
not the CUDA code (the GPU test test_single_edge_checks_match_oracle does that):

- an undirected edge {u, v} removed inside an SCC that stays whole leaves every block as it was
  exactly when two internally vertex-disjoint u-v paths remain in the SCC's undirected subgraph
  (Menger), found as one path P1 plus one augmenting search in P1's residual graph with every
  vertex split into an entered and a left state;
- a path found by a plain search around P1's inner vertices is always such a second path (the
  device tries that first), and where it finds none the residual search still may;
- a deleted edge u -> v inside SCC C leaves C whole exactly when u still reaches v.
"""
from collections import deque

import numpy as np


def _csr(V, keys):
    s = (keys // V).astype(np.int32)
    d = (keys % V).astype(np.int32)
    beg = np.zeros(V + 1, np.int64)
    np.add.at(beg, s + 1, 1)
    return np.cumsum(beg), d


def _sym(orc, V, fb, fa):
    tb, ta = orc.transpose(V, fb, fa)
    return orc.sym(V, fb, fa, tb, ta)


def _path(sb, sa, ok, s, t):
    par = {s: s}
    q = deque([s])
    while q:
        x = q.popleft()
        for y in sa[sb[x]:sb[x + 1]].tolist():
            if not ok(y) or y in par:
                continue
            par[y] = x
            if y == t:
                p = [t]
                while p[-1] != s:
                    p.append(par[p[-1]])
                return p[::-1]
            q.append(y)
    return None


def _second_path(sb, sa, ok, P):
    """Residual search from u's left state to v's entered state (csrc/single.cu second_path)."""
    u, v, k = P[0], P[-1], len(P) - 1
    pos = {x: i for i, x in enumerate(P)}
    inner = lambda x: x in pos and 0 < pos[x] < k
    seen = {(u, 1)}
    q = deque([(u, 1)])
    while q:
        x, left = q.popleft()
        nxt = []
        if left:
            if inner(x):
                nxt.append((x, 0))
            for y in sa[sb[x]:sb[x + 1]].tolist():
                if ok(y) and not (x in pos and pos[x] < k and P[pos[x] + 1] == y):
                    nxt.append((y, 0))
        else:
            nxt.append((x, 1) if not inner(x) else (P[pos[x] - 1], 1))
        for st in nxt:
            if st == (v, 0):
                return True
            if st not in seen:
                seen.add(st)
                q.append(st)
    return False


def _two_paths(sb, sa, lab, C, u, v):
    ok = lambda y: lab[y] == C
    P = _path(sb, sa, ok, u, v)
    if P is None:
        return False, False
    inner = set(P[1:-1])
    plain = _path(sb, sa, lambda y: ok(y) and y not in inner, u, v) is not None
    return plain, _second_path(sb, sa, ok, P)


def test_single_edge_rules_against_oracle(orc):
    rng = np.random.default_rng(5)
    agree = changed = plain_missed = split_checks = 0
    for _ in range(700):
        V = int(rng.integers(10, 120))
        E = int(V * rng.uniform(0.9, 2.5))
        a, b = rng.integers(0, V, E), rng.integers(0, V, E)
        keys = np.unique(a[a != b].astype(np.int64) * V + b[a != b])
        if len(keys) == 0:
            continue
        fb, fa = _csr(V, keys)
        scc = orc.scc(V, fb, fa)
        kset = set(keys.tolist())
        inside = [k for k in keys.tolist() if scc[k // V] == scc[k % V]]
        for k in [inside[j] for j in rng.choice(len(inside), min(3, len(inside)), replace=False)] if inside else []:
            u, v = k // V, k % V
            fb2, fa2 = _csr(V, np.array(sorted(kset - {k}), np.int64))
            scc2 = orc.scc(V, fb2, fa2)
            # SCC rule: C stays whole iff u still reaches v
            reach = orc.bfs(V, fb2, fa2, [u])[v] >= 0
            assert reach == np.array_equal(scc2, scc), (u, v)
            split_checks += 1
            if not reach or (v * V + u) in kset:
                continue  # blocks are rebuilt with the SCC / the undirected view did not change
            sb, sa = _sym(orc, V, fb, fa)
            sb2, sa2 = _sym(orc, V, fb2, fa2)
            same = np.array_equal(orc.bicc(V, sb, sa, scc)[0], orc.bicc(V, sb2, sa2, scc2)[0])
            plain, residual = _two_paths(sb2, sa2, scc2, scc2[u], u, v)
            assert residual == same, (u, v)
            assert not plain or residual
            plain_missed += residual and not plain
            changed += not same
            agree += 1
    assert agree > 300 and changed > 5 and split_checks > 500, (agree, changed, split_checks)
    assert plain_missed > 0  # the residual search is needed, not only the plain one
