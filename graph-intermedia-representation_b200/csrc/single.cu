// Exact checks of the single-edge latency path (the Scope-Prune-Update entry points
// insertEdge / deleteEdge, gir.cpp:3043-3134). A batch with one effective edge change asks
// these before the repair plan falls back to rebuilding a layer:
//  - WCC, an undirected pair removed: are u and v still connected in the symmetrized view?
//    (yes: the components are unchanged);
//  - SCC, u -> v deleted inside SCC C: does u still reach v? (yes: C stays strongly connected; a
//    path from u to v never leaves C, so the search is confined to C);
//  - SCC, u -> v inserted against the rank order: does v reach u? (no: no cycle closes, only the
//    condensation edges and ranks change; every vertex on such a path has an SCC rank between
//    rank(v) and rank(u), so the search is confined to that window);
//  - BCT, the undirected edge {u, v} removed inside an SCC that stays whole: are there still two
//    internally vertex-disjoint u-v paths in the SCC's undirected subgraph? By Menger's theorem
//    the block that held {u, v} stays biconnected exactly then, so every block is unchanged.
//    One path P1 comes from a bidirectional search. The second is first sought by a plain
//    bidirectional search around P1's inner vertices (usually enough); only where that finds
//    none does one augmenting search run in the residual graph of P1, with every vertex split
//    into an entered and a left state.
// A WCC split found this way is applied in place (the search that ran out holds the whole new
// component). All searches run in one CTA of one launch (no host round trip per level) with
// visited marks stamped by generation, so nothing is cleared between calls, and with budgets on
// visited vertices and scanned edges: a search that exceeds them reports "unknown" and the layer
// is rebuilt as before.
#include "common.cuh"

namespace gir {

namespace {

constexpr int kThreads = 1024;
constexpr int kBigDeg = 512;  // rows longer than this are swept by the whole CTA
constexpr int kBig = 256;     // deferred long rows per level (overflow: the warp sweeps it)
constexpr unsigned long long kEdgeBudget = 1ull << 20;
constexpr int kVisitBudget = 1 << 20;
constexpr unsigned kFull = 0xffffffffu;

// R_SPLIT: not connected, and the WCC labels were split in place
enum { R_NOT_RUN = 0, R_FOUND = 1, R_NONE = 2, R_UNKNOWN = 3, R_SPLIT = 4 };

// Working arrays (int32 each), sections of one buffer of kWords * V entries.
struct Work {
    int32_t *stamp_f, *stamp_b, *par_f, *par_b, *q_f, *q_b;  // V each
    int32_t *stamp_r, *q_r;                                   // 2V each (vertex-split states)
    int32_t *path, *path_stamp, *path_pos;                    // V each
};
constexpr int kWords = 13;

struct Filter {
    const int32_t* lab;   // vertex allowed iff lab[x] == L (lab null: no label test)
    int32_t L;
    const int32_t* rank;  // and rank[x] in [rlo, rhi] (rank null: no rank test)
    int32_t rlo, rhi;
    const int32_t* pstamp = nullptr;  // and x not inside P1 (stamped pgen at a position in (0, pk))
    const int32_t* ppos = nullptr;
    int32_t pgen = 0, pk = 0;
    __device__ bool ok(int32_t x) const {
        if (lab && lab[x] != L) return false;
        if (pstamp && pstamp[x] == pgen) {
            const int32_t p = ppos[x];
            if (p > 0 && p < pk) return false;
        }
        if (rank) {
            const int32_t r = rank[x];
            return r >= rlo && r <= rhi;
        }
        return true;
    }
};

struct Shared {
    int tail;                  // queue length of the side being expanded (appends go here)
    int stop;                  // set when the search can end (found)
    int found;                 // meeting vertex (or target state) + 1
    int nbig;
    unsigned long long edges;  // scanned edges (budget)
    unsigned long long fe, be, ne;  // row entries of the forward / backward frontier; of the next one
    int lo_f, hi_f, lo_b, hi_b;
    int result;
    int mn;
    int32_t big[kBig];
};

// Expands queue entries [lo, hi) by one level: visit(x, y) for every row entry y of the vertex
// x = row_of(entry) of every entry (entries with row_of < 0 have no row to sweep). Warps take the
// short rows; rows longer than kBigDeg are deferred to the whole CTA. The level stops early when
// the search is over (S.stop) or past its edge budget; the caller then reads the budget first, so
// a level cut short never counts as a frontier that ran out.
template <class RowOf, class Visit>
__device__ void cta_expand(const CSRView& c, const int32_t* q, int lo, int hi, Shared& S, RowOf&& row_of,
                           Visit&& visit) {
    const int warp = threadIdx.x >> 5, ln = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (threadIdx.x == 0) S.nbig = 0;
    __syncthreads();
    for (int i = lo + warp; i < hi; i += nw) {
        const int stop = __shfl_sync(
            kFull, ln == 0 ? (*(volatile int*)&S.stop || *(volatile unsigned long long*)&S.edges > kEdgeBudget) : 0, 0);
        if (stop) break;
        const int32_t x = row_of(q[i]);
        if (x < 0) continue;
        const int64_t b = c.beg[x];
        const int32_t d = c.deg[x];
        if (d > kBigDeg) {
            int deferred = 0;
            if (ln == 0) {
                const int k = atomicAdd(&S.nbig, 1);
                deferred = k < kBig;
                if (deferred) S.big[k] = x;
            }
            if (__shfl_sync(kFull, deferred, 0)) continue;
        }
        for (int64_t k = b + ln; k < b + d; k += 32) visit(x, c.adj[k]);
        if (ln == 0) atomicAdd(&S.edges, (unsigned long long)d);
    }
    __syncthreads();
    const int nbig = S.nbig < kBig ? S.nbig : kBig;
    for (int j = 0; j < nbig; ++j) {
        if (*(volatile int*)&S.stop || *(volatile unsigned long long*)&S.edges > kEdgeBudget) break;
        const int32_t x = S.big[j];
        const int64_t b = c.beg[x];
        const int32_t d = c.deg[x];
        for (int64_t k = b + threadIdx.x; k < b + d; k += blockDim.x) visit(x, c.adj[k]);
        if (threadIdx.x == 0) atomicAdd(&S.edges, (unsigned long long)d);
    }
    __syncthreads();
}

// Claims y for one side (first claimer wins); returns true for the claimer.
__device__ __forceinline__ bool claim(int32_t* stamp, int32_t y, int32_t gen) {
    return stamp[y] != gen && atomicExch(&stamp[y], gen) != gen;
}

__device__ __forceinline__ int32_t same_vertex(int32_t x) { return x; }

// Bidirectional search from s (over fwd) and t (over bwd), both sides limited by the filter,
// expanding each level the side whose frontier has fewer row entries (the work of the level, so
// a side that has reached a hub waits while the other side catches up). R_FOUND with S.found =
// meeting vertex + 1; R_NONE when one side ran out first (t is not reachable from s); R_UNKNOWN
// over budget.
__device__ int bidir(const CSRView& fwd, const CSRView& bwd, const Filter& F, int32_t s, int32_t t, int32_t gen,
                     const Work& W, Shared& S) {
    if (threadIdx.x == 0) {
        W.stamp_f[s] = gen;
        W.par_f[s] = s;
        W.q_f[0] = s;
        W.stamp_b[t] = gen;
        W.par_b[t] = t;
        W.q_b[0] = t;
        S.found = s == t ? s + 1 : 0;
        S.stop = S.found != 0;
        S.edges = 0;
        S.fe = (unsigned long long)fwd.deg[s];
        S.be = (unsigned long long)bwd.deg[t];
        S.lo_f = S.lo_b = 0;
        S.hi_f = S.hi_b = 1;
        S.result = S.found ? R_FOUND : R_NOT_RUN;
    }
    __syncthreads();
    while (true) {
        if (S.stop) break;
        if (S.edges > kEdgeBudget || S.hi_f + S.hi_b > kVisitBudget) {  // (before the next test)
            if (threadIdx.x == 0) S.result = R_UNKNOWN;
            break;
        }
        if (S.hi_f == S.lo_f || S.hi_b == S.lo_b) {
            if (threadIdx.x == 0) S.result = R_NONE;
            break;
        }
        const bool fside = S.fe <= S.be;
        const int lo = fside ? S.lo_f : S.lo_b, hi = fside ? S.hi_f : S.hi_b;
        __syncthreads();  // (every thread has read the bounds before thread 0 moves them)
        if (threadIdx.x == 0) {
            S.tail = hi;
            S.ne = 0;
        }
        if (fside) {
            cta_expand(fwd, W.q_f, lo, hi, S, same_vertex, [&](int32_t x, int32_t y) {
                if (!F.ok(y) || !claim(W.stamp_f, y, gen)) return;
                W.par_f[y] = x;
                W.q_f[atomicAdd(&S.tail, 1)] = y;
                atomicAdd(&S.ne, (unsigned long long)fwd.deg[y]);
                if (W.stamp_b[y] == gen) {
                    S.found = y + 1;
                    S.stop = 1;
                }
            });
        } else {
            cta_expand(bwd, W.q_b, lo, hi, S, same_vertex, [&](int32_t x, int32_t y) {
                if (!F.ok(y) || !claim(W.stamp_b, y, gen)) return;
                W.par_b[y] = x;
                W.q_b[atomicAdd(&S.tail, 1)] = y;
                atomicAdd(&S.ne, (unsigned long long)bwd.deg[y]);
                if (W.stamp_f[y] == gen) {
                    S.found = y + 1;
                    S.stop = 1;
                }
            });
        }
        if (threadIdx.x == 0) {
            if (fside) {
                S.lo_f = hi;
                S.hi_f = S.tail;
                S.fe = S.ne;
            } else {
                S.lo_b = hi;
                S.hi_b = S.tail;
                S.be = S.ne;
            }
            if (S.stop) S.result = R_FOUND;
        }
        __syncthreads();
    }
    __syncthreads();
    const int r = S.result;
    __syncthreads();
    return r;
}

// Second internally vertex-disjoint u-v path in sym (limited by F), given P1 = path[0..k]
// (path[0] = u, path[k] = v; positions stamped with gen): one search of the residual graph of
// P1 with every vertex x split into an entered state 2x and a left state 2x + 1. Moves:
//  - entered 2y, y not inside P1: through y to 2y + 1; y inside P1 (its capacity is used): back
//    along P1's arc into y, to the left state of its predecessor;
//  - left 2x + 1, x inside P1: back through x to 2x (reverse of its capacity arc);
//  - left 2x + 1: to the entered state of every allowed neighbour y, except P1's next vertex
//    (that arc is used).
// R_FOUND when v's entered state is reached.
__device__ int second_path(const CSRView& sym, const Filter& F, int32_t u, int32_t v, int k, int32_t gen,
                           const Work& W, Shared& S) {
    auto internal = [&](int32_t x) {
        if (W.path_stamp[x] != gen) return false;
        const int p = W.path_pos[x];
        return p > 0 && p < k;
    };
    auto push = [&](int32_t st) {
        if (!claim(W.stamp_r, st, gen)) return;
        W.q_r[atomicAdd(&S.tail, 1)] = st;
        if (st == 2 * v) {
            S.found = st + 1;
            S.stop = 1;
        }
    };
    if (threadIdx.x == 0) {
        W.stamp_r[2 * u + 1] = gen;
        W.q_r[0] = 2 * u + 1;
        S.stop = 0;
        S.found = 0;
        S.edges = 0;
        S.lo_f = 0;
        S.hi_f = 1;
        S.result = R_NOT_RUN;
    }
    __syncthreads();
    while (true) {
        if (S.stop) break;
        if (S.edges > kEdgeBudget || S.hi_f > kVisitBudget) {  // (before the next test)
            if (threadIdx.x == 0) S.result = R_UNKNOWN;
            break;
        }
        if (S.hi_f == S.lo_f) {
            if (threadIdx.x == 0) S.result = R_NONE;
            break;
        }
        const int lo = S.lo_f, hi = S.hi_f;
        __syncthreads();
        if (threadIdx.x == 0) S.tail = hi;
        __syncthreads();
        for (int i = lo + (int)threadIdx.x; i < hi; i += blockDim.x) {
            const int32_t st = W.q_r[i];
            const int32_t x = st >> 1;
            if (!(st & 1)) {
                if (!internal(x)) push(2 * x + 1);
                else push(2 * W.path[W.path_pos[x] - 1] + 1);
            } else if (internal(x)) {
                push(2 * x);
            }
        }
        cta_expand(sym, W.q_r, lo, hi, S, [](int32_t st) { return (st & 1) ? (st >> 1) : -1; },
                   [&](int32_t x, int32_t y) {
                       if (!F.ok(y)) return;
                       if (W.path_stamp[x] == gen && W.path_pos[x] < k && W.path[W.path_pos[x] + 1] == y) return;
                       push(2 * y);
                   });
        if (threadIdx.x == 0) {
            S.lo_f = hi;
            S.hi_f = S.tail;
            if (S.stop) S.result = R_FOUND;
        }
        __syncthreads();
    }
    __syncthreads();
    const int r = S.result;
    __syncthreads();
    return r;
}

// A removed undirected pair split its weakly connected component (label L) in two. The side of
// the search that ran out first visited all of its part (set[0..n), stamped gen), so: that part
// takes its smallest id as label, unless L itself lies in it, in which case the part keeps L and
// the rest of the old component takes the rest's smallest id (one CTA pass over the labels).
__device__ void wcc_split(int32_t* label, int64_t V, int32_t L, const int32_t* set, int n, const int32_t* stamp,
                          int32_t gen, Shared& S) {
    if (threadIdx.x == 0) S.mn = INT32_MAX;
    __syncthreads();
    int32_t m = INT32_MAX;
    for (int i = threadIdx.x; i < n; i += blockDim.x) m = set[i] < m ? set[i] : m;
    atomicMin(&S.mn, m);
    __syncthreads();
    const int32_t ms = S.mn;
    __syncthreads();
    if (ms != L) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) label[set[i]] = ms;
    } else {
        if (threadIdx.x == 0) S.mn = INT32_MAX;
        __syncthreads();
        int32_t m2 = INT32_MAX;
        for (int64_t x = threadIdx.x; x < V; x += blockDim.x)
            if (label[x] == L && stamp[x] != gen) m2 = (int32_t)x < m2 ? (int32_t)x : m2;
        atomicMin(&S.mn, m2);
        __syncthreads();
        const int32_t mr = S.mn;
        if (mr != INT32_MAX)
            for (int64_t x = threadIdx.x; x < V; x += blockDim.x)
                if (label[x] == L && stamp[x] != gen) label[x] = mr;
    }
    __syncthreads();
}

struct CheckArgs {
    CSRView fw, bw, sym;
    const int32_t* scc;
    const int32_t* rank;
    int32_t* wcc_label;  // split in place when the WCC check finds u, v disconnected
    int64_t V;
    int32_t u, v;
    int wcc, split, cycle, twopath;
    int32_t gen0;
    Work W;
    int32_t* out;  // one result per check
};

__global__ void __launch_bounds__(kThreads, 1) k_single_checks(CheckArgs a) {
    __shared__ Shared S;
    const int32_t u = a.u, v = a.v;
    const Filter none{nullptr, 0, nullptr, 0, 0};
    int r = R_NOT_RUN;
    bool p1 = false;  // a u-v path inside the SCC's undirected subgraph was found (also a WCC path)
    if (a.twopath) {
        const int32_t gen = a.gen0 + 3;
        const Filter f{a.scc, a.scc[u], nullptr, 0, 0};
        r = bidir(a.sym, a.sym, f, u, v, gen, a.W, S);
        p1 = r == R_FOUND;
        if (r == R_FOUND) {
            // P1 = u .. m along the forward tree, then m .. v along the backward tree (simple:
            // the search stopped at the first vertex both sides held)
            if (threadIdx.x == 0) {
                // (a simple path has at most V vertices; the guard keeps every write in bounds)
                const int32_t m = S.found - 1;
                const int64_t cap = a.V;
                int64_t n = 0;
                for (int32_t x = m; n < cap;) {
                    a.W.path[n++] = x;
                    if (x == u) break;
                    x = a.W.par_f[x];
                }
                for (int64_t i = 0, j = n - 1; i < j; ++i, --j) {
                    const int32_t t = a.W.path[i];
                    a.W.path[i] = a.W.path[j];
                    a.W.path[j] = t;
                }
                for (int32_t x = m; x != v && n < cap;) {
                    x = a.W.par_b[x];
                    a.W.path[n++] = x;
                }
                const bool ok = n >= 2 && a.W.path[0] == u && a.W.path[n - 1] == v;
                for (int64_t i = 0; ok && i < n; ++i) {
                    a.W.path_stamp[a.W.path[i]] = gen;
                    a.W.path_pos[a.W.path[i]] = (int32_t)i;
                }
                S.tail = ok ? (int)(n - 1) : -1;
            }
            __syncthreads();
            const int k = S.tail;
            __syncthreads();
            if (k <= 0) {
                r = R_UNKNOWN;
            } else {
                // a path found around P1's inner vertices is disjoint from P1 by construction
                Filter f2 = f;
                f2.pstamp = a.W.path_stamp;
                f2.ppos = a.W.path_pos;
                f2.pgen = gen;
                f2.pk = k;
                r = bidir(a.sym, a.sym, f2, u, v, a.gen0 + 4, a.W, S);
                if (r != R_FOUND) r = second_path(a.sym, f, u, v, k, gen, a.W, S);
            }
        }
    }
    if (threadIdx.x == 0) a.out[3] = r;
    r = R_NOT_RUN;
    if (a.wcc) {
        r = p1 ? R_FOUND : bidir(a.sym, a.sym, none, u, v, a.gen0, a.W, S);
        if (r == R_NONE && a.wcc_label) {
            const bool fwd_done = S.hi_f == S.lo_f;  // (read by every thread after bidir's barriers)
            const int n = fwd_done ? S.hi_f : S.hi_b;
            __syncthreads();
            wcc_split(a.wcc_label, a.V, a.wcc_label[u], fwd_done ? a.W.q_f : a.W.q_b, n,
                      fwd_done ? a.W.stamp_f : a.W.stamp_b, a.gen0, S);
            r = R_SPLIT;
        }
    }
    if (threadIdx.x == 0) a.out[0] = r;
    r = R_NOT_RUN;
    if (a.split) {
        const Filter f{a.scc, a.scc[u], nullptr, 0, 0};
        r = bidir(a.fw, a.bw, f, u, v, a.gen0 + 1, a.W, S);
    }
    if (threadIdx.x == 0) a.out[1] = r;
    r = R_NOT_RUN;
    if (a.cycle) {
        const Filter f{nullptr, 0, a.rank, a.rank[v], a.rank[u]};
        r = bidir(a.fw, a.bw, f, v, u, a.gen0 + 2, a.W, S);
    }
    if (threadIdx.x == 0) a.out[2] = r;
}

}  // namespace

int single_op_checks(gir_dev* g, int32_t u, int32_t v, const SingleChecks& want, int32_t out[4]) {
    const int64_t V = g->V;
    for (int i = 0; i < 4; ++i) out[i] = R_NOT_RUN;
    if (!(want.wcc || want.split || want.cycle || want.twopath)) return GIR_OK;
    if (V <= 0 || V >= (1ll << 30) || u < 0 || v < 0 || u >= V || v >= V) return GIR_OK;  // (states 2x + 1 in int32)
    const size_t words = (size_t)kWords * (size_t)V + 8;
    if (g->single_ws.bytes < words * sizeof(int32_t) || g->single_gen > INT32_MAX - 16) {
        GIR_TRY(ensure(g, g->single_ws, words * sizeof(int32_t)));
        GIR_CUDA(g, cudaMemsetAsync(g->single_ws.p, 0, words * sizeof(int32_t), g->stream));
        g->single_gen = 1;
    }
    int32_t* p = static_cast<int32_t*>(g->single_ws.p);
    Work W;
    W.stamp_f = p; p += V;
    W.stamp_b = p; p += V;
    W.par_f = p; p += V;
    W.par_b = p; p += V;
    W.q_f = p; p += V;
    W.q_b = p; p += V;
    W.stamp_r = p; p += 2 * V;
    W.q_r = p; p += 2 * V;
    W.path = p; p += V;
    W.path_stamp = p; p += V;
    W.path_pos = p; p += V;
    int32_t* res = p;  // 4 results (within the 8 spare words)
    CheckArgs a;
    a.fw = view(g->fw);
    a.bw = view(g->bw);
    a.sym = view(g->sym);
    a.scc = static_cast<const int32_t*>(g->scc.p);
    a.rank = static_cast<const int32_t*>(g->scc_rank.p);
    a.wcc_label = want.wcc ? static_cast<int32_t*>(g->wcc.p) : nullptr;
    a.V = V;
    a.u = u;
    a.v = v;
    a.wcc = want.wcc;
    a.split = want.split && a.scc;
    a.cycle = want.cycle && a.rank;
    a.twopath = want.twopath && a.scc;
    a.gen0 = g->single_gen;
    a.W = W;
    a.out = res;
    g->single_gen += 5;
    k_single_checks<<<1, kThreads, 0, g->stream>>>(a);
    GIR_LAUNCH(g, "k_single_checks");
    void* hp = nullptr;
    GIR_TRY(pinned(g, 64, &hp));
    GIR_CUDA(g, cudaMemcpyAsync(hp, res, 4 * sizeof(int32_t), cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    for (int i = 0; i < 4; ++i) out[i] = static_cast<const int32_t*>(hp)[i];
    return GIR_OK;
}

}  // namespace gir
