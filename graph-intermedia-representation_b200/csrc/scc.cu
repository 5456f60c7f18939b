// Strongly connected components and the condensation DAG (buildSCC_DAG, gir.cpp:798-839).
//
// The reference runs one sequential iterative Tarjan over all vertices (gir.cpp:494-537) and
// counts cross-SCC edges into per-SCC hash maps (gir.cpp:825-831). The partition is unique,
// so any exact algorithm gives the same SCCs; here it is the data-parallel decomposition
// (as in iSpan / Multistep, gir_constructor/includes/scc_cpu):
//  1. trim-1 as a worklist: a vertex without an in- or out-neighbour among the unassigned
//     vertices (self-loops ignored) is a singleton SCC; removing it lowers its neighbours'
//     counts, which may trim them in turn; then trim-2: two vertices that are each other's only
//     unassigned in- (or out-) neighbour form an SCC of two;
//  2. forward-backward from a pivot of maximal out-degree x in-degree (the giant SCC of a
//     power-law graph): SCC(pivot) = forward reach ∩ backward reach over unassigned vertices;
//  3. colour propagation for the rest, repeated until every vertex is assigned: every
//     unassigned vertex starts with its own id as colour, colours spread along forward edges
//     by max until stable, so colour(v) = largest id that reaches v; a vertex r with
//     colour(r) = r is a root, and SCC(r) = the vertices of colour r that reach r (a backward
//     search restricted to colour r);
//  4. labels are made canonical (smallest member id) and the condensation edges are the
//     distinct (scc(u), scc(v)) keys of all cross edges: radix sort + unique;
//  5. topological ranks: Kahn levels over the condensation DAG, rank = position in
//     (level, label) order, so rank(a) < rank(b) for every DAG edge a -> b (the invariant of
//     scc_rank, gir.h:54-57).
#include "common.cuh"

namespace gir {

namespace {

constexpr int kBlock = 256;
constexpr int kWarps = kBlock / 32;

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

enum { C_Q = 0, C_ACT = 1, C_ROOTS = 2, C_PIV = 3, C_ACT_E = 4, C_N = 8 };

// Active in/out degree counts (self-loops excluded) and the first trim frontier.
__global__ void k_trim_init(int64_t V, CSRView fw, CSRView bw, int32_t* label, int32_t* indeg, int32_t* outdeg,
                            int32_t* q, unsigned long long* cnt) {
    __shared__ int32_t s_st[kBlock / 32][kStage];
    int n_st = 0;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < V; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = base + threadIdx.x;
        bool trim = false;
        if (v < V) {
            int32_t o = fw.deg[v], in = bw.deg[v];
            // self-loop: rows are sorted, binary search for v
            const int64_t fb = fw.beg[v];
            const int64_t p = lower_bound_dev(fw.adj, fb, fb + o, (int32_t)v);
            if (p < fb + o && fw.adj[p] == (int32_t)v) { --o; --in; }
            outdeg[v] = o;
            indeg[v] = in;
            trim = (o == 0 || in == 0);
            label[v] = trim ? (int32_t)v : -1;
        }
        stage_append(trim, (int32_t)v, s_st[threadIdx.x >> 5], n_st, q, &cnt[C_Q]);
    }
    stage_flush(s_st[threadIdx.x >> 5], n_st, q, &cnt[C_Q]);
}

// One trim round over the removed vertices of the last round: lower the counts of their
// neighbours; a neighbour whose count reaches 0 is removed (claimed once by CAS).
__global__ void __launch_bounds__(kBlock) k_trim_out(const int32_t* q, const unsigned long long* qlen, CSRView fw,
                                                     int32_t* label, int32_t* indeg, int32_t* nq,
                                                     unsigned long long* cnt) {
    warp_expand(q, (int64_t)*qlen, fw, nq, &cnt[C_Q], [&](int32_t u, int32_t w) {
        if (w == u) return false;
        if (atomicSub(&indeg[w], 1) == 1) return atomicCAS(&label[w], -1, w) == -1;
        return false;
    });
}

__global__ void __launch_bounds__(kBlock) k_trim_in(const int32_t* q, const unsigned long long* qlen, CSRView bw,
                                                    int32_t* label, int32_t* outdeg, int32_t* nq,
                                                    unsigned long long* cnt) {
    warp_expand(q, (int64_t)*qlen, bw, nq, &cnt[C_Q], [&](int32_t u, int32_t w) {
        if (w == u) return false;
        if (atomicSub(&outdeg[w], 1) == 1) return atomicCAS(&label[w], -1, w) == -1;
        return false;
    });
}

// Trim-2 (iSpan's trim_2_from_fq, gir_constructor/includes/scc_cpu/trim_2_3.h:161, as an
// algorithm source): u and v form an SCC of two when each is the other's only unassigned in-
// neighbour (or, in the second pass, only unassigned out-neighbour): no other unassigned vertex
// reaches either, and the two edges close the cycle. Two launches per direction, so labels are
// never read while they change: k_trim2_pair records each vertex's only unassigned neighbour in
// rows `c` when its count (`deg_act`, exact or an over-count of the unassigned neighbours) is 1,
// then k_trim2_apply labels the mutual pairs with the smaller id.
__global__ void k_trim2_pair(int64_t V, CSRView c, const int32_t* label, const int32_t* deg_act, int32_t* partner) {
    GRID_STRIDE(u, V) {
        int32_t p = -1;
        if (label[u] == -1 && deg_act[u] == 1) {
            const int64_t b = c.beg[u], e = b + c.deg[u];
            for (int64_t k = b; k < e; ++k) {
                const int32_t w = c.adj[k];
                if (w != (int32_t)u && label[w] == -1) {
                    p = w;
                    break;
                }
            }
        }
        partner[u] = p;
    }
}

__global__ void k_trim2_apply(int64_t V, const int32_t* partner, int32_t* label, unsigned long long* n_pairs) {
    unsigned long long c = 0;
    GRID_STRIDE(u, V) {
        const int32_t p = partner[u];
        if (p >= 0 && partner[p] == (int32_t)u) {
            label[u] = p < (int32_t)u ? p : (int32_t)u;
            c += p > (int32_t)u;
        }
    }
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane_id() == 0 && c) atomicAdd(n_pairs, c);
}

// Pivot: the unassigned vertex with the largest score (ties: larger id). Rules: 0 out x in
// degree (iSpan's pivot_selection_from_fq, gir_constructor/includes/scc_cpu/scc_common.h:98-146,
// the fixed schedule), 1 out + in, 2 in-degree. Also counts the unassigned vertices (C_ACT) and
// their edges (C_ROOTS + 1: out-degrees summed), the schedule's features.
__global__ void k_pivot(int64_t V, const int32_t* label, const int32_t* indeg, const int32_t* outdeg, int rule,
                        unsigned long long* cnt) {
    unsigned long long best = 0;
    unsigned long long act = 0, act_e = 0;
    GRID_STRIDE(v, V) {
        if (label[v] != -1) continue;
        ++act;
        act_e += (uint32_t)outdeg[v];
        const unsigned long long o = (uint32_t)outdeg[v], i = (uint32_t)indeg[v];
        const unsigned long long s = rule == 1 ? o + i : (rule == 2 ? i : o * i);
        const unsigned long long k = ((s < (1ull << 31) ? s : (1ull << 31)) << 32) | (unsigned long long)v;
        if (k + 1 > best) best = k + 1;
    }
    for (int o = 16; o; o >>= 1) {
        const unsigned long long t = __shfl_xor_sync(0xffffffffu, best, o);
        best = t > best ? t : best;
        act += __shfl_xor_sync(0xffffffffu, act, o);
        act_e += __shfl_xor_sync(0xffffffffu, act_e, o);
    }
    if (lane_id() == 0) {
        if (best) atomicMax(&cnt[C_PIV], best);
        if (act) atomicAdd(&cnt[C_ACT], act);
        if (act_e) atomicAdd(&cnt[C_ACT_E], act_e);
    }
}

// Edge-balanced reach from the pivot, both directions in one level-synchronous traversal: a
// queue entry e >= 0 is vertex e searched forward (out-rows), e < 0 is vertex ~e searched
// backward (in-rows). The frontier's rows are cut into equal chunks after a scan of their
// lengths, so hubs do not serialize a warp. An unassigned w joins a direction once (mark bit 1
// forward, 2 backward); afterwards the vertices with both bits are SCC(pivot). Paths inside the
// pivot's SCC never pass through trimmed (already labelled) vertices, so restricting both searches
// to unassigned vertices keeps FW ∩ BW exact.
__global__ void k_frontier_deg(const int32_t* q, int64_t n, const int32_t* fdeg, const int32_t* bdeg, int64_t* pref) {
    GRID_STRIDE(i, n) {
        const int32_t e = q[i];
        pref[i] = e >= 0 ? fdeg[e] : bdeg[~e];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) pref[n] = 0;
}

constexpr int kReachChunk = 32 * 16;

__global__ void __launch_bounds__(kBlock) k_reach_both(const int32_t* q, int64_t nq, const int64_t* pref, CSRView fw,
                                                       CSRView bw, const int32_t* label, int32_t* mark, int32_t* out,
                                                       unsigned long long* cnt) {
    __shared__ int32_t s_st[kBlock / 32][kStage];
    int n_st = 0;
    const int64_t total = pref[nq];
    const int lane = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c0 = warp * kReachChunk; c0 < total; c0 += nwarps * kReachChunk) {
        const int64_t c1 = c0 + kReachChunk < total ? c0 + kReachChunk : total;
        const int64_t key = c0 + lane < total ? c0 + lane : total - 1;
        int64_t lo = 0, hi = nq - 1;
        while (lo < hi) {
            const int64_t m = (lo + hi + 1) >> 1;
            if (pref[m] <= key) lo = m; else hi = m - 1;
        }
        int64_t i = lo;
        for (int64_t base = c0; base < c1; base += 32) {
            const int64_t p = base + lane;
            bool push = false;
            int32_t ent = 0;
            if (p < c1) {
                while (pref[i + 1] <= p) ++i;
                const int32_t e = q[i];
                const bool back = e < 0;
                const int32_t u = back ? ~e : e;
                const int32_t w = back ? bw.adj[bw.beg[u] + (p - pref[i])] : fw.adj[fw.beg[u] + (p - pref[i])];
                const int32_t bit = back ? 2 : 1;
                if (label[w] == -1 && (mark[w] & bit) == 0) push = (atomicOr(&mark[w], bit) & bit) == 0;
                ent = back ? ~w : w;
            }
            stage_append(push, ent, s_st[threadIdx.x >> 5], n_st, out, &cnt[C_Q]);
        }
    }
    stage_flush(s_st[threadIdx.x >> 5], n_st, out, &cnt[C_Q]);
}

// SCC(pivot): the unassigned vertices reached both ways.
__global__ void k_reach_label(int64_t V, const int32_t* mark, int32_t pivot, int32_t* label) {
    GRID_STRIDE(v, V) if (mark[v] == 3 && label[v] == -1) label[v] = pivot;
}

// Colour propagation: colour(w) = max(colour(w), colour(u)) along forward edges between
// unassigned vertices. `inq` de-duplicates the next queue per round.
__global__ void k_color_init(int64_t V, const int32_t* label, int32_t* color, int32_t* q, unsigned long long* cnt) {
    __shared__ int32_t s_st[kBlock / 32][kStage];
    int n_st = 0;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < V; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = base + threadIdx.x;
        const bool on = v < V && label[v] == -1;
        if (v < V) color[v] = (int32_t)v;
        stage_append(on, (int32_t)v, s_st[threadIdx.x >> 5], n_st, q, &cnt[C_Q]);
    }
    stage_flush(s_st[threadIdx.x >> 5], n_st, q, &cnt[C_Q]);
}

__global__ void __launch_bounds__(kBlock) k_color_prop(const int32_t* q, const unsigned long long* qlen, CSRView fw,
                                                       const int32_t* label, int32_t* color, int32_t* inq,
                                                       int32_t round, int32_t* nq, unsigned long long* cnt) {
    warp_expand(q, (int64_t)*qlen, fw, nq, &cnt[C_Q], [&](int32_t u, int32_t w) {
        if (label[w] != -1) return false;
        const int32_t cu = color[u];
        if (cu <= color[w]) return false;
        if (atomicMax(&color[w], cu) >= cu) return false;
        return atomicExch(&inq[w], round) != round;
    });
}

__global__ void k_color_roots(int64_t V, int32_t* label, const int32_t* color, int32_t* q, unsigned long long* cnt) {
    __shared__ int32_t s_st[kBlock / 32][kStage];
    int n_st = 0;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < V; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = base + threadIdx.x;
        bool root = false;
        if (v < V && label[v] == -1 && color[v] == (int32_t)v) {
            label[v] = (int32_t)v;
            root = true;
        }
        stage_append(root, (int32_t)v, s_st[threadIdx.x >> 5], n_st, q, &cnt[C_Q]);
    }
    stage_flush(s_st[threadIdx.x >> 5], n_st, q, &cnt[C_Q]);
}

// Backward search inside each colour class from its root.
__global__ void __launch_bounds__(kBlock) k_color_bw(const int32_t* q, const unsigned long long* qlen, CSRView bw,
                                                     int32_t* label, const int32_t* color, int32_t* nq,
                                                     unsigned long long* cnt) {
    warp_expand(q, (int64_t)*qlen, bw, nq, &cnt[C_Q], [&](int32_t u, int32_t w) {
        const int32_t c = color[u];
        if (label[w] != -1 || color[w] != c) return false;
        return atomicCAS(&label[w], -1, c) == -1;
    });
}

// Canonical labels: smallest member of every class.
__global__ void k_fill(int32_t* p, int64_t n, int32_t v) { GRID_STRIDE(i, n) p[i] = v; }

// Smallest member of every class. The lanes of a warp that share a label (consecutive vertices
// of the giant SCC mostly do) send one atomicMin, from their smallest vertex, and only when a
// plain read says it can still lower the minimum: otherwise the millions of members of one
// class would serialize on one address.
__global__ void k_class_min(int64_t V, const int32_t* label, int32_t* mn) {
    GRID_STRIDE(v, V) {
        const int32_t l = label[v];
        const unsigned grp = __match_any_sync(__activemask(), l);
        const bool leader = (int)(__ffs(grp) - 1) == lane_id();  // the group's smallest vertex
        if (leader && *(volatile int32_t*)&mn[l] > (int32_t)v) atomicMin(&mn[l], (int32_t)v);
    }
}

__global__ void k_apply_min(int64_t V, int32_t* label, const int32_t* mn, unsigned long long* n_classes) {
    unsigned long long c = 0;
    GRID_STRIDE(v, V) {
        const int32_t m = mn[label[v]];
        label[v] = m;
        c += (m == (int32_t)v);
    }
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane_id() == 0 && c) atomicAdd(n_classes, c);
}

// Cross-SCC edge keys (label(u) << 32 | label(w)) at the edge's own slot, flagged; the flags of
// slack slots stay 0 (cleared by the caller), so a compaction over the capacity collects them.
__global__ void __launch_bounds__(kBlock) k_cross_keys(int64_t V, CSRView fw, const int32_t* label, uint64_t* keys,
                                                       uint8_t* flag) {
    __shared__ int64_t s_excl[kWarps][33];
    __shared__ int32_t s_u[kWarps][32];
    const int wib = threadIdx.x >> 5;
    warp_sweep_rows(
        fw.beg, fw.deg, fw.adj, 0, V, s_excl[wib], s_u[wib],
        [&](int32_t u, int32_t w, int64_t e) {
            const int32_t a = label[u], b = label[w];
            keys[e] = ((uint64_t)(uint32_t)a << 32) | (uint32_t)b;
            flag[e] = a != b;
        },
        kHeavyRow);
}

// The rows k_cross_keys leaves out (longer than kHeavyRow), their entries spread over the grid.
__global__ void k_cross_keys_heavy(const int32_t* rows, const int64_t* pref, int64_t n, CSRView fw, const int32_t* label,
                                   uint64_t* keys, uint8_t* flag) {
    grid_sweep_heavy_rows(rows, pref, n, fw.beg, fw.adj, [&](int32_t u, int32_t w, int64_t e) {
        const int32_t a = label[u], b = label[w];
        keys[e] = ((uint64_t)(uint32_t)a << 32) | (uint32_t)b;
        flag[e] = a != b;
    });
}

__global__ void k_distinct_u64(const uint64_t* keys, int64_t n, uint8_t* flag) {
    GRID_STRIDE(i, n) flag[i] = (i == 0 || keys[i] != keys[i - 1]);
}

// One round of longest-path levels over the condensation edges: level(b) >= level(a) + 1 for
// every edge a -> b. Edge-parallel with a plain pre-check, so only raises take an atomic (no
// hot counter: a node with many in-edges, like the giant SCC, is raised a few times, not
// decremented once per edge as in Kahn's algorithm).
__global__ void k_dag_level_round(const uint64_t* keys, int64_t n, int32_t* level, unsigned long long* changed) {
    unsigned long long c = 0;
    GRID_STRIDE(i, n) {
        const uint64_t k = keys[i];
        const int32_t a = (int32_t)(k >> 32), b = (int32_t)(k & 0xffffffffULL);
        const int32_t cand = level[a] + 1;
        if (cand > level[b] && atomicMax(&level[b], cand) < cand) ++c;
    }
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane_id() == 0 && c) atomicAdd(changed, c);
}

__global__ void k_rank_keys(int64_t V, const int32_t* label, const int32_t* level, uint64_t* keys,
                            unsigned long long* n) {
    GRID_STRIDE(v, V) {
        if (label[v] == (int32_t)v) keys[atomicAdd(n, 1ull)] = ((uint64_t)(uint32_t)level[v] << 32) | (uint32_t)v;
    }
}

__global__ void k_rank_scatter(const uint64_t* keys, int64_t n, int32_t* rank_of) {
    GRID_STRIDE(i, n) rank_of[(int64_t)(keys[i] & 0xffffffffULL)] = (int32_t)i;
}

__global__ void k_rank_gather(int64_t V, const int32_t* label, const int32_t* rank_of, int32_t* rank) {
    GRID_STRIDE(v, V) rank[v] = rank_of[label[v]];
}

struct Loop {
    gir_dev* g;
    unsigned long long* cnt;
    unsigned long long* hc;
    int read(int64_t* out) {
        GIR_CUDA(g, cudaMemcpyAsync(hc, cnt, sizeof(unsigned long long) * C_N, cudaMemcpyDeviceToHost, g->stream));
        GIR_CUDA(g, cudaStreamSynchronize(g->stream));
        *out = (int64_t)hc[C_Q];
        return GIR_OK;
    }
};

}  // namespace

int scc_labels(gir_dev* g, int32_t* label, int64_t* n_scc) {
    const int64_t V = g->V;
    const CSRView fw = view(g->fw), bw = view(g->bw);
    int32_t *indeg = nullptr, *outdeg = nullptr, *qa = nullptr, *qb = nullptr, *mark = nullptr, *color = nullptr;
    unsigned long long* cnt = nullptr;
    GIR_TRY(ensure_n(g, g->scratch[0], V + 1, &indeg));
    GIR_TRY(ensure_n(g, g->scratch[1], V + 1, &outdeg));
    // (the queues hold up to 2V entries in the two-way reach from the pivot)
    GIR_TRY(ensure_n(g, g->scratch[2], 2 * V + 2, &qa));
    GIR_TRY(ensure_n(g, g->scratch[3], 2 * V + 2, &qb));
    GIR_TRY(ensure_n(g, g->scratch[4], V + 1, &mark));
    GIR_TRY(ensure_n(g, g->scratch[5], V + 1, &color));
    GIR_TRY(ensure_n(g, g->scratch[6], 2 * C_N, &cnt));
    unsigned long long* qlen = cnt + C_N;
    void* hp = nullptr;
    GIR_TRY(pinned(g, 256, &hp));
    Loop lp{g, cnt, static_cast<unsigned long long*>(hp)};
    *n_scc = 0;
    if (V == 0) return GIR_OK;
    const int grid = g->num_sms * (int)g->params[GIR_PARAM_CTAS_PER_SM];
    auto blocks_for_queue = [&](int64_t n) {
        const int64_t b = (n + 32 * kWarps - 1) / (32 * kWarps);
        return (int)(b < 1 ? 1 : (b < grid ? b : grid));
    };
    // One level-synchronous pass: `launch(in, inlen, out)` for each round until the queue empties.
    auto run_queue = [&](int32_t*& in, int32_t*& out, int64_t n, auto&& launch) -> int {
        while (n > 0) {
            GIR_CUDA(g, cudaMemcpyAsync(qlen, &cnt[C_Q], sizeof(unsigned long long), cudaMemcpyDeviceToDevice, g->stream));
            GIR_CUDA(g, cudaMemsetAsync(&cnt[C_Q], 0, sizeof(unsigned long long), g->stream));
            GIR_TRY(launch(in, out, n));
            std::swap(in, out);
            GIR_TRY(lp.read(&n));
        }
        return GIR_OK;
    };

    trace_mark(g, "scc: start");
    // 1. trim-1
    GIR_CUDA(g, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * 2 * C_N, g->stream));
    k_trim_init<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, fw, bw, label, indeg, outdeg, qa, cnt);
    GIR_LAUNCH(g, "k_trim_init");
    int64_t n = 0;
    GIR_TRY(lp.read(&n));
    GIR_TRY(run_queue(qa, qb, n, [&](int32_t* in, int32_t* out, int64_t m) -> int {
        // removed vertices lower both neighbour counts; both kernels append to `out`
        k_trim_out<<<blocks_for_queue(m), kBlock, 0, g->stream>>>(in, qlen, fw, label, indeg, out, cnt);
        GIR_LAUNCH(g, "k_trim_out");
        k_trim_in<<<blocks_for_queue(m), kBlock, 0, g->stream>>>(in, qlen, bw, label, outdeg, out, cnt);
        GIR_LAUNCH(g, "k_trim_in");
        return GIR_OK;
    }));

    // trim-2: SCCs of two vertices, through in-neighbours, then through out-neighbours
    {
        int32_t* partner = color;  // (colours are set up later)
        GIR_CUDA(g, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * C_N, g->stream));
        for (int dir = 0; dir < 2; ++dir) {
            k_trim2_pair<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, dir ? fw : bw, label, dir ? outdeg : indeg,
                                                                           partner);
            GIR_LAUNCH(g, "k_trim2_pair");
            k_trim2_apply<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, partner, label, &cnt[C_ROOTS]);
            GIR_LAUNCH(g, "k_trim2_apply");
        }
        if (g->trace_marks) {
            GIR_CUDA(g, cudaMemcpyAsync(lp.hc, cnt, sizeof(unsigned long long) * C_N, cudaMemcpyDeviceToHost, g->stream));
            GIR_CUDA(g, cudaStreamSynchronize(g->stream));
            std::fprintf(stderr, "[gir] scc: trim-2 pairs %llu\n", (unsigned long long)lp.hc[C_ROOTS]);
        }
    }

    trace_mark(g, "scc: trim");
    // 2. forward-backward from the max-degree pivot
    GIR_CUDA(g, cudaMemsetAsync(mark, 0, sizeof(int32_t) * V, g->stream));
    GIR_CUDA(g, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * C_N, g->stream));
    k_pivot<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, label, indeg, outdeg, 0, cnt);
    GIR_LAUNCH(g, "k_pivot");
    GIR_CUDA(g, cudaMemcpyAsync(lp.hc, cnt, sizeof(unsigned long long) * C_N, cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    // The pivot rule: forced by GIR_PARAM_PIVOT, else the fixed max out x in degree or the
    // schedule network (rule 3: no forward-backward pass, colour propagation does everything).
    // Any rule gives the same SCCs; only the time differs.
    int rule = (int)g->params[GIR_PARAM_PIVOT];
    {
        float feat[GIR_SCHED_IN];
        sched_scc_features(g, (double)lp.hc[C_ACT], (double)lp.hc[C_ACT_E],
                           lp.hc[C_PIV] ? (double)((lp.hc[C_PIV] - 1) >> 32) : 0.0, feat);
        if (rule < 0) {
            rule = 0;
            if (g->schedule == GIR_SCHEDULE_LEARNED && g->sched_loaded) GIR_TRY(sched_choose_pivot(g, feat, &rule));
        }
        g->trace_x.clear();
        g->trace_y.clear();
        sched_trace(g, feat, 8 + rule);
    }
    if (rule == 1 || rule == 2) {
        GIR_CUDA(g, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * C_N, g->stream));
        k_pivot<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, label, indeg, outdeg, rule, cnt);
        GIR_LAUNCH(g, "k_pivot");
        GIR_CUDA(g, cudaMemcpyAsync(lp.hc, cnt, sizeof(unsigned long long) * C_N, cudaMemcpyDeviceToHost, g->stream));
        GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    }
    if (rule != 3 && lp.hc[C_PIV] != 0) {
        const int32_t pivot = (int32_t)((lp.hc[C_PIV] - 1) & 0xffffffffULL);
        // both searches seeded with the pivot (marked both ways)
        int32_t *fa = qa, *fb = qb;
        int64_t* pref = nullptr;
        GIR_TRY(ensure_n(g, g->scratch[7], 2 * V + 2, &pref));
        const int32_t seed[2] = {pivot, ~pivot}, both = 3;
        GIR_CUDA(g, cudaMemcpyAsync(mark + pivot, &both, sizeof(int32_t), cudaMemcpyHostToDevice, g->stream));
        GIR_CUDA(g, cudaMemcpyAsync(fa, seed, sizeof(seed), cudaMemcpyHostToDevice, g->stream));
        GIR_CUDA(g, cudaStreamSynchronize(g->stream));  // (seed is a host stack array)
        int64_t n = 2;
        while (n > 0) {
            k_frontier_deg<<<grid_for(g, n, kBlock), kBlock, 0, g->stream>>>(fa, n, fw.deg, bw.deg, pref);
            GIR_LAUNCH(g, "k_frontier_deg");
            GIR_TRY(exclusive_scan_i64(g, pref, pref, n + 1));
            GIR_CUDA(g, cudaMemsetAsync(&cnt[C_Q], 0, sizeof(unsigned long long), g->stream));
            k_reach_both<<<grid, kBlock, 0, g->stream>>>(fa, n, pref, fw, bw, label, mark, fb, cnt);
            GIR_LAUNCH(g, "k_reach_both");
            std::swap(fa, fb);
            GIR_TRY(lp.read(&n));
        }
        k_reach_label<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, mark, pivot, label);
        GIR_LAUNCH(g, "k_reach_label");
    }

    trace_mark(g, "scc: fw-bw");
    // 3. colour propagation rounds until every vertex is assigned
    int32_t* inq = mark;
    int32_t round = 1;
    GIR_CUDA(g, cudaMemsetAsync(inq, 0, sizeof(int32_t) * V, g->stream));
    for (int outer = 0; outer < (1 << 30); ++outer) {
        GIR_CUDA(g, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * C_N, g->stream));
        k_color_init<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, label, color, qa, cnt);
        GIR_LAUNCH(g, "k_color_init");
        GIR_TRY(lp.read(&n));
        if (n == 0) break;
        GIR_TRY(run_queue(qa, qb, n, [&](int32_t* in, int32_t* out, int64_t m) -> int {
            ++round;
            k_color_prop<<<blocks_for_queue(m), kBlock, 0, g->stream>>>(in, qlen, fw, label, color, inq, round, out, cnt);
            GIR_LAUNCH(g, "k_color_prop");
            return GIR_OK;
        }));
        GIR_CUDA(g, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * C_N, g->stream));
        k_color_roots<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, label, color, qa, cnt);
        GIR_LAUNCH(g, "k_color_roots");
        GIR_TRY(lp.read(&n));
        GIR_TRY(run_queue(qa, qb, n, [&](int32_t* in, int32_t* out, int64_t m) -> int {
            k_color_bw<<<blocks_for_queue(m), kBlock, 0, g->stream>>>(in, qlen, bw, label, color, out, cnt);
            GIR_LAUNCH(g, "k_color_bw");
            return GIR_OK;
        }));
    }

    if (g->trace_marks) std::fprintf(stderr, "[gir] scc: colour rounds %d\n", (int)round);
    trace_mark(g, "scc: colour");
    // 4. canonical labels
    int32_t* mn = color;
    k_fill<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(mn, V, INT32_MAX);
    GIR_LAUNCH(g, "k_fill");
    k_class_min<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, label, mn);
    GIR_LAUNCH(g, "k_class_min");
    GIR_CUDA(g, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * C_N, g->stream));
    k_apply_min<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, label, mn, &cnt[C_Q]);
    GIR_LAUNCH(g, "k_apply_min");
    GIR_TRY(lp.read(n_scc));
    return GIR_OK;
}

int scc_build(gir_dev* g) {
    const int64_t V = g->V;
    int32_t* label = nullptr;
    GIR_TRY(ensure_n(g, g->scc, V + 1, &label));
    GIR_TRY(scc_labels(g, label, &g->n_scc));
    trace_mark(g, "scc: labels");
    return scc_build_dag(g);
}

// One edge u -> v between two SCCs (u's SCC before v's in rank order), inserted or just deleted:
// out[0] = position of its condensation key in the sorted keys (lower bound), out[1] = the key is
// there; out[2] bit 0 = another edge joins the two SCCs from u's forward row or v's backward
// row, bit 1 = u has an out-neighbour in its own SCC, bit 2 = v has an in-neighbour in its own
// SCC (a vertex of a non-trivial SCC always has both, so without them both SCCs are singletons
// and the two rows are every edge between them).
__global__ void k_dag_probe(const uint64_t* dag, int64_t n, uint64_t key, CSRView fw, CSRView bw,
                            const int32_t* label, int32_t u, int32_t v, unsigned long long* out) {
    const int32_t cu = label[u], cv = label[v];
    unsigned long long bits = 0;
    for (int64_t k = fw.beg[u] + threadIdx.x; k < fw.beg[u] + fw.deg[u]; k += blockDim.x) {
        const int32_t y = label[fw.adj[k]];
        if (y == cv) bits |= 1;
        if (y == cu) bits |= 2;
    }
    for (int64_t k = bw.beg[v] + threadIdx.x; k < bw.beg[v] + bw.deg[v]; k += blockDim.x) {
        const int32_t x = label[bw.adj[k]];
        if (x == cu) bits |= 1;
        if (x == cv) bits |= 4;
    }
    if (bits) atomicOr(&out[2], bits);
    if (threadIdx.x == 0) {
        int64_t lo = 0, hi = n;
        while (lo < hi) {
            const int64_t m = (lo + hi) >> 1;
            if (dag[m] < key) lo = m + 1; else hi = m;
        }
        out[0] = (unsigned long long)lo;
        out[1] = lo < n && dag[lo] == key;
    }
}

__global__ void k_dag_put(uint64_t* dag, int64_t p, uint64_t key) { dag[p] = key; }

int scc_dag_patch_one(gir_dev* g, int32_t u, int32_t v, bool insert, bool* patched) {
    *patched = false;
    const int32_t* label = static_cast<const int32_t*>(g->scc.p);
    const int64_t n = g->n_dag;
    if (n < 0 || !g->dag.p || u < 0 || v < 0 || u >= g->V || v >= g->V) return scc_build_dag(g);
    unsigned long long* cnt = nullptr;
    GIR_TRY(ensure_n(g, g->scratch[6], 2 * C_N, &cnt));
    void* hp = nullptr;
    GIR_TRY(pinned(g, 256, &hp));
    unsigned long long* hc = static_cast<unsigned long long*>(hp);
    int32_t lab[2];
    GIR_CUDA(g, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * 3, g->stream));
    GIR_CUDA(g, cudaMemcpyAsync(&lab[0], label + u, sizeof(int32_t), cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaMemcpyAsync(&lab[1], label + v, sizeof(int32_t), cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    const uint64_t key = ((uint64_t)(uint32_t)lab[0] << 32) | (uint32_t)lab[1];
    k_dag_probe<<<1, kBlock, 0, g->stream>>>(static_cast<const uint64_t*>(g->dag.p), n, key, view(g->fw), view(g->bw),
                                             label, u, v, cnt);
    GIR_LAUNCH(g, "k_dag_probe");
    GIR_CUDA(g, cudaMemcpyAsync(hc, cnt, sizeof(unsigned long long) * 3, cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    const int64_t p = (int64_t)hc[0];
    const bool present = hc[1] != 0;
    const unsigned long long bits = hc[2];
    uint64_t* dag = static_cast<uint64_t*>(g->dag.p);
    if (insert) {
        if (present) {
            *patched = true;  // the SCCs were joined already
            return GIR_OK;
        }
        if (g->dag.bytes < sizeof(uint64_t) * (size_t)(n + 2)) return scc_build_dag(g);
        uint64_t* tmp = nullptr;
        GIR_TRY(ensure_n(g, g->scratch[8], n - p + 1, &tmp));
        if (n > p) {
            GIR_CUDA(g, cudaMemcpyAsync(tmp, dag + p, sizeof(uint64_t) * (n - p), cudaMemcpyDeviceToDevice, g->stream));
            GIR_CUDA(g, cudaMemcpyAsync(dag + p + 1, tmp, sizeof(uint64_t) * (n - p), cudaMemcpyDeviceToDevice, g->stream));
        }
        k_dag_put<<<1, 1, 0, g->stream>>>(dag, p, key);
        GIR_LAUNCH(g, "k_dag_put");
        g->n_dag = n + 1;
    } else {
        if (!present || (bits & 1)) {
            *patched = true;  // another edge still joins the two SCCs (or none was recorded)
            return GIR_OK;
        }
        if (bits & 6) return scc_build_dag(g);  // a non-trivial SCC: its other members' rows count too
        if (n - p - 1 > 0) {
            uint64_t* tmp = nullptr;
            GIR_TRY(ensure_n(g, g->scratch[8], n - p, &tmp));
            GIR_CUDA(g, cudaMemcpyAsync(tmp, dag + p + 1, sizeof(uint64_t) * (n - p - 1), cudaMemcpyDeviceToDevice,
                                        g->stream));
            GIR_CUDA(g, cudaMemcpyAsync(dag + p, tmp, sizeof(uint64_t) * (n - p - 1), cudaMemcpyDeviceToDevice,
                                        g->stream));
        }
        g->n_dag = n - 1;
    }
    // the ranks stay a topological order (the edge respects them); reachability changed
    g->dag_rows_valid = false;
    g->reach_hub_valid = false;
    *patched = true;
    return GIR_OK;
}

int scc_build_dag(gir_dev* g) {
    const int64_t V = g->V;
    int32_t* label = static_cast<int32_t*>(g->scc.p);
    // condensation edges: cross keys, radix sort, unique
    const int64_t cap = g->fw.cap;
    uint64_t *keys = nullptr, *tmp = nullptr;
    uint8_t* flag = nullptr;
    unsigned long long* cnt = nullptr;
    GIR_TRY(ensure_n(g, g->scratch[7], cap + 1, &keys));
    GIR_TRY(ensure_n(g, g->scratch[8], cap + 1, &tmp));
    GIR_TRY(ensure_n(g, g->scratch[9], cap + 1, &flag));
    GIR_TRY(ensure_n(g, g->scratch[6], 2 * C_N, &cnt));
    void* hp = nullptr;
    GIR_TRY(pinned(g, 256, &hp));
    unsigned long long* hc = static_cast<unsigned long long*>(hp);
    GIR_CUDA(g, cudaMemsetAsync(flag, 0, cap + 1, g->stream));
    if (V > 0) {
        // the long rows' list in tmp (free until the compaction; cap >= 4V, every row has room
        // for 4 entries): rows int32[V], their length scan int64[V + 1], flags uint8[V]
        int32_t* heavy = reinterpret_cast<int32_t*>(tmp);
        int64_t* hpref = reinterpret_cast<int64_t*>(tmp) + (V + 1) / 2 + 1;
        uint8_t* hflag = reinterpret_cast<uint8_t*>(hpref + V + 2);
        int64_t n_heavy = 0;
        GIR_TRY(heavy_rows(g, g->fw.deg, V, kHeavyRow, hflag, heavy, hpref, &n_heavy));
        k_cross_keys<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, view(g->fw), label, keys, flag);
        GIR_LAUNCH(g, "k_cross_keys");
        if (n_heavy > 0) {
            k_cross_keys_heavy<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(heavy, hpref, n_heavy, view(g->fw), label,
                                                                               keys, flag);
            GIR_LAUNCH(g, "k_cross_keys_heavy");
        }
    }
    int64_t n_cross = 0;
    GIR_TRY(select_flagged_u64(g, keys, flag, tmp, cap, &n_cross));
    std::swap(keys, tmp);
    GIR_TRY(sort_keys_u64(g, keys, tmp, n_cross, 64));
    int64_t n_dag = 0;
    uint64_t* dag = nullptr;
    GIR_TRY(ensure_n(g, g->dag, n_cross + 1, &dag));
    if (n_cross > 0) {
        k_distinct_u64<<<grid_for(g, n_cross, kBlock), kBlock, 0, g->stream>>>(keys, n_cross, flag);
        GIR_LAUNCH(g, "k_distinct_u64");
        GIR_TRY(select_flagged_u64(g, keys, flag, dag, n_cross, &n_dag));
    }
    g->n_dag = n_dag;
    g->dag_rows_valid = false;
    g->reach_hub_valid = false;
    trace_mark(g, "scc: dag edges");

    // topological ranks: longest-path levels over the condensation edges, rounds until stable
    // (at most the DAG's depth + 1 rounds)
    int32_t *level = nullptr, *rank_of = nullptr, *rank = nullptr;
    GIR_TRY(ensure_n(g, g->scratch[1], V + 1, &level));
    GIR_TRY(ensure_n(g, g->scratch[5], V + 1, &rank_of));
    GIR_TRY(ensure_n(g, g->scc_rank, V + 1, &rank));
    GIR_CUDA(g, cudaMemsetAsync(level, 0, sizeof(int32_t) * V, g->stream));
    for (int64_t round = 0; n_dag > 0 && round <= V; ++round) {
        GIR_CUDA(g, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * C_N, g->stream));
        k_dag_level_round<<<grid_for(g, n_dag, kBlock), kBlock, 0, g->stream>>>(dag, n_dag, level, &cnt[C_Q]);
        GIR_LAUNCH(g, "k_dag_level_round");
        GIR_CUDA(g, cudaMemcpyAsync(hc, cnt, sizeof(unsigned long long) * C_N, cudaMemcpyDeviceToHost, g->stream));
        GIR_CUDA(g, cudaStreamSynchronize(g->stream));
        if (hc[C_Q] == 0) break;
    }
    trace_mark(g, "scc: levels");
    // rank = position in (level, label) order
    GIR_CUDA(g, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * C_N, g->stream));
    if (V > 0) {
        k_rank_keys<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, label, level, keys, &cnt[C_Q]);
        GIR_LAUNCH(g, "k_rank_keys");
    }
    GIR_CUDA(g, cudaMemcpyAsync(hc, cnt, sizeof(unsigned long long) * C_N, cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    const int64_t ns = (int64_t)hc[C_Q];
    GIR_TRY(sort_keys_u64(g, keys, tmp, ns, 64));
    if (ns > 0) {
        k_rank_scatter<<<grid_for(g, ns, kBlock), kBlock, 0, g->stream>>>(keys, ns, rank_of);
        GIR_LAUNCH(g, "k_rank_scatter");
        k_rank_gather<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, label, rank_of, rank);
        GIR_LAUNCH(g, "k_rank_gather");
    }
    trace_mark(g, "scc: ranks");
    g->scc_built = true;
    return GIR_OK;
}

}  // namespace gir
