// Per-SCC biconnected blocks and the block-cut forest (buildBCT, gir.cpp:2063-2089).
//
// The layer is defined on H, the undirected graph of the symmetrized edges whose endpoints lie
// in the same SCC (gir.h:45-46): its connected components are the SCCs, and its biconnected
// components are the blocks the reference computes SCC by SCC (sequential Hopcroft-Tarjan for
// small SCCs, gir.cpp:541-587; Tarjan-Vishkin over a BFS tree for large ones, gir.cpp:1804-2022).
// An SCC of one vertex is a singleton block (gir.cpp:584). Here Tarjan-Vishkin runs on every
// SCC at once:
//  1. BFS spanning forest of H from every SCC's smallest vertex (level-synchronous);
//  2. subtree sizes nd (levels bottom-up) and preorder numbers pre (children grouped by parent
//     by a radix sort, sibling offsets by a scan, levels top-down);
//  3. low / high: min / max pre over each subtree and its non-tree neighbours;
//  4. union-find over tree edges (edge (p(v), v) is named by v): rule 1 joins the edges of
//     v and w for a non-tree edge {v, w} between unrelated vertices; rule 2 joins (p(v), v)
//     with (p(p(v)), p(v)) when v's subtree reaches outside p(v)'s subtree;
//  5. every class is a block: its vertices are the child ends of its tree edges plus the
//     parent of the topmost one (the block's head). Output in the reference's representation
//     (gir.h:58-64): every vertex has one parent block (label_block), every block one head
//     articulation point (-1 for the block a tree root belongs to first), bcnt = number of
//     blocks containing the vertex (AP iff >= 2).
#include "common.cuh"

namespace gir {

namespace {

constexpr int kBlock = 256;

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

enum { C_Q = 0, C_ERR = 1, C_N = 4 };

// H row filter: neighbour w of u is in H iff same SCC (sym rows never contain u itself).
struct HView {
    CSRView sym;
    const int32_t* scc;
};

// SCCs with more than one vertex: every non-smallest member marks its SCC's smallest vertex
// (plain stores behind a read, so a giant SCC costs a few writes, not one per member).
__global__ void k_mark_nontrivial(int64_t V, const int32_t* scc, uint8_t* nontrivial) {
    GRID_STRIDE(v, V) {
        const int32_t r = scc[v];
        if (r != (int32_t)v && !nontrivial[r]) nontrivial[r] = 1;
    }
}

// Row lengths of H for the sweeps: 0 for the vertices of singleton SCCs (isolated in H).
__global__ void k_h_deg(int64_t V, const int32_t* scc, const uint8_t* nontrivial, const int32_t* sym_deg,
                        int32_t* hdeg) {
    GRID_STRIDE(v, V) hdeg[v] = nontrivial[scc[v]] ? sym_deg[v] : 0;
}

// Forest roots: every SCC's smallest vertex; only those of non-singleton SCCs start the BFS.
__global__ void k_roots(int64_t V, const int32_t* scc, const uint8_t* nontrivial, int32_t* parent, int32_t* depth,
                        int32_t* order, unsigned long long* cnt) {
    __shared__ int32_t s_st[kBlock / 32][kStage];
    int n_st = 0;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < V; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = base + threadIdx.x;
        bool root = false;
        if (v < V) {
            const bool r = scc[v] == (int32_t)v;
            root = r && nontrivial[v];
            parent[v] = r ? (int32_t)v : -1;
            depth[v] = r ? 0 : -1;
        }
        stage_append(root, (int32_t)v, s_st[threadIdx.x >> 5], n_st, order, &cnt[C_Q]);
    }
    stage_flush(s_st[threadIdx.x >> 5], n_st, order, &cnt[C_Q]);
}

// One BFS level of the spanning forest: the level's vertices are order[lo, lo + n); new ones are
// appended to order after it. Edge-balanced: the level's H rows are cut into equal chunks after
// a scan of their lengths, so hubs of the giant SCC do not serialize a warp.
__global__ void k_level_deg(const int32_t* q, int64_t n, const int32_t* deg, int64_t* pref) {
    GRID_STRIDE(i, n) pref[i] = deg[q[i]];
    if (blockIdx.x == 0 && threadIdx.x == 0) pref[n] = 0;
}

constexpr int kForestChunk = 32 * 16;

__global__ void __launch_bounds__(kBlock) k_forest_balanced(const int32_t* q, int64_t nq, const int64_t* pref, HView h,
                                                            int32_t* parent, int32_t* depth, int32_t L, int32_t* out,
                                                            unsigned long long* cnt) {
    __shared__ int32_t s_st[kBlock / 32][kStage];
    int n_st = 0;
    const int64_t total = pref[nq];
    const int lane = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c0 = warp * kForestChunk; c0 < total; c0 += nwarps * kForestChunk) {
        const int64_t c1 = c0 + kForestChunk < total ? c0 + kForestChunk : total;
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
            int32_t w = 0;
            if (p < c1) {
                while (pref[i + 1] <= p) ++i;
                const int32_t u = q[i];
                w = h.sym.adj[h.sym.beg[u] + (p - pref[i])];
                if (parent[w] == -1 && h.scc[w] == h.scc[u] && atomicCAS(&parent[w], -1, u) == -1) {
                    depth[w] = L + 1;
                    push = true;
                }
            }
            stage_append(push, w, s_st[threadIdx.x >> 5], n_st, out, &cnt[C_Q]);
        }
    }
    stage_flush(s_st[threadIdx.x >> 5], n_st, out, &cnt[C_Q]);
}

__global__ void k_fill_i32(int32_t* p, int64_t n, int32_t v) { GRID_STRIDE(i, n) p[i] = v; }

// nd[parent] += nd[v] for the vertices of one level (deepest level first).
__global__ void k_nd_level(const int32_t* q, int64_t n, const int32_t* parent, int32_t* nd) {
    GRID_STRIDE(i, n) {
        const int32_t v = q[i];
        atomicAdd(&nd[parent[v]], nd[v]);
    }
}

// Children grouped by parent: key (parent << 32 | v) for non-root vertices.
__global__ void k_child_keys(int64_t V, const int32_t* parent, uint64_t* keys, uint8_t* flag) {
    GRID_STRIDE(v, V) {
        const int32_t p = parent[v];
        keys[v] = ((uint64_t)(uint32_t)p << 32) | (uint64_t)v;
        flag[v] = p >= 0 && p != (int32_t)v;
    }
}

// Sibling offsets: off[v] = sum of nd over the earlier children of parent(v).
__global__ void k_child_nd(const uint64_t* keys, int64_t n, const int32_t* nd, int64_t* scan_in) {
    GRID_STRIDE(i, n) scan_in[i] = nd[(int64_t)(keys[i] & 0xffffffffULL)];
    if (blockIdx.x == 0 && threadIdx.x == 0) scan_in[n] = 0;
}

__global__ void k_group_first(const uint64_t* keys, int64_t n, int64_t* first_of_parent) {
    GRID_STRIDE(i, n) {
        const int64_t p = (int64_t)(keys[i] >> 32);
        if (i == 0 || (int64_t)(keys[i - 1] >> 32) != p) first_of_parent[p] = i;
    }
}

__global__ void k_sibling_off(const uint64_t* keys, int64_t n, const int64_t* scan, const int64_t* first_of_parent,
                              int32_t* off) {
    GRID_STRIDE(i, n) {
        const int64_t p = (int64_t)(keys[i] >> 32);
        const int64_t v = (int64_t)(keys[i] & 0xffffffffULL);
        off[v] = (int32_t)(scan[i] - scan[first_of_parent[p]]);
    }
}

__global__ void k_pre_level(const int32_t* q, int64_t n, const int32_t* parent, const int32_t* off, int32_t* pre) {
    GRID_STRIDE(i, n) {
        const int32_t v = q[i];
        pre[v] = pre[parent[v]] + 1 + off[v];
    }
}

__global__ void k_pre_roots(const int32_t* q, int64_t n, int32_t* pre) { GRID_STRIDE(i, n) pre[q[i]] = 0; }

// low / high from non-tree edges of H, and rule 1 unions.
__device__ __forceinline__ int32_t uf_find(int32_t* uf, int32_t x) {
    int32_t p = uf[x];
    while (p != x) {
        const int32_t gp = uf[p];
        if (gp != p) uf[x] = gp;
        x = p;
        p = uf[x];
    }
    return x;
}

__device__ __forceinline__ void uf_union(int32_t* uf, int32_t a, int32_t b, unsigned long long* err) {
    for (int iter = 0; iter < (1 << 22); ++iter) {
        int32_t ra = uf_find(uf, a), rb = uf_find(uf, b);
        if (ra == rb) return;
        if (ra > rb) { const int32_t t = ra; ra = rb; rb = t; }
        if (atomicCAS(&uf[rb], rb, ra) == rb) return;
    }
    atomicAdd(err, 1ull);
}

// Per-vertex tree data packed for the non-tree sweep: one 16-byte gather per neighbour instead of
// four scattered 4-byte ones. x = pre, y = nd, z = parent, w = scc.
__global__ void k_pack_vinfo(int64_t V, const int32_t* pre, const int32_t* nd, const int32_t* parent,
                             const int32_t* scc, int4* vinfo) {
    GRID_STRIDE(v, V) vinfo[v] = make_int4(pre[v], nd[v], parent[v], scc[v]);
}

// Rule-1 unions from a sample before the full sweep: every vertex of H takes the first kSample
// entries of its row, and the non-tree edges among them whose ends are unrelated in the forest
// (neither an ancestor of the other) union the two ends' tree edges. After a flatten (every uf
// entry its root), the full sweep's cheap uf[u] != uf[w] test rejects nearly every pair the
// sample already joined (on a power-law graph the giant block takes most vertices), instead of
// each pair walking two find chains. Unions are idempotent, so the sample changes no class.
constexpr int kSample = 4;

__global__ void k_nontree_sample(int64_t V, HView h, const int4* vinfo, int32_t* uf, unsigned long long* err) {
    GRID_STRIDE(u, V) {
        const int32_t d = h.sym.deg[u];
        if (d == 0) continue;
        const int4 iu = vinfo[u];
        const int64_t b = h.sym.beg[u];
        for (int j = 0; j < kSample && j < d; ++j) {
            const int32_t w = h.sym.adj[b + j];
            const int4 iw = vinfo[w];
            if (iu.w != iw.w || iw.z == (int32_t)u || iu.z == w) continue;  // other SCC, or a tree edge
            const bool w_under_u = iw.x >= iu.x && iw.x < iu.x + iu.y;
            const bool u_under_w = iu.x >= iw.x && iu.x < iw.x + iw.y;
            if (!w_under_u && !u_under_w && uf[u] != uf[w]) uf_union(uf, (int32_t)u, w, err);
        }
    }
}

// Every uf entry to its root (read-only walks, then one write; no union runs meanwhile).
__global__ void k_uf_flatten(int32_t* uf, int64_t V) {
    GRID_STRIDE(v, V) {
        int32_t x = uf[v];
        while (uf[x] != x) x = uf[x];
        uf[v] = x;
    }
}

// One sweep over the non-tree edges of H: low / high of every vertex from its own non-tree
// neighbours, and rule 1 (once per edge, from its endpoint with the smaller pre) for edges
// between unrelated endpoints.
__device__ __forceinline__ void nontree_entry(int32_t u, int32_t w, const int4* vinfo, int32_t* low, int32_t* high,
                                              int32_t* uf, unsigned long long* err) {
    const int4 iu = vinfo[u], iw = vinfo[w];
    if (iu.w != iw.w || iw.z == u || iu.z == w) return;  // other SCC, or a tree edge
    const int32_t pw = iw.x;
    if (pw < low[u]) atomicMin(&low[u], pw);  // (plain pre-checks: a hub's row is swept by many
    if (pw > high[u]) atomicMax(&high[u], pw);  //  threads, most of which change nothing)
    if (iu.x < pw && iu.x + iu.y <= pw && uf[u] != uf[w]) uf_union(uf, u, w, err);
}

// Rows of at most kHeavyRow entries, a warp per 32 rows; the longer rows go to k_nontree_heavy,
// which spreads their entries over the whole grid.
__global__ void __launch_bounds__(kBlock) k_nontree(int64_t V, HView h, const int4* vinfo, int32_t* low, int32_t* high,
                                                    int32_t* uf, unsigned long long* err) {
    __shared__ int64_t s_excl[kBlock / 32][33];
    __shared__ int32_t s_u[kBlock / 32][32];
    const int wib = threadIdx.x >> 5;
    warp_sweep_rows(
        h.sym.beg, h.sym.deg, h.sym.adj, 0, V, s_excl[wib], s_u[wib],
        [&](int32_t u, int32_t w, int64_t) { nontree_entry(u, w, vinfo, low, high, uf, err); }, kHeavyRow);
}

__global__ void k_nontree_heavy(const int32_t* rows, const int64_t* pref, int64_t n, HView h, const int4* vinfo,
                                int32_t* low, int32_t* high, int32_t* uf, unsigned long long* err) {
    grid_sweep_heavy_rows(rows, pref, n, h.sym.beg, h.sym.adj,
                          [&](int32_t u, int32_t w, int64_t) { nontree_entry(u, w, vinfo, low, high, uf, err); });
}

__global__ void k_lowhigh_level(const int32_t* q, int64_t n, const int32_t* parent, int32_t* low, int32_t* high) {
    GRID_STRIDE(i, n) {
        const int32_t v = q[i];
        const int32_t p = parent[v];
        atomicMin(&low[p], low[v]);
        atomicMax(&high[p], high[v]);
    }
}

// rule 2 for every non-root v whose parent u is not a root.
__global__ void k_rule2(int64_t V, const int32_t* parent, const int32_t* pre, const int32_t* nd, const int32_t* low,
                        const int32_t* high, int32_t* uf, unsigned long long* err) {
    GRID_STRIDE(v, V) {
        const int32_t u = parent[v];
        if (u < 0 || u == (int32_t)v) continue;  // unreached (cannot happen) or root
        if (parent[u] == u) continue;            // u is a root
        if (low[v] < pre[u] || high[v] >= pre[u] + nd[u]) uf_union(uf, (int32_t)v, u, err);
    }
}

__global__ void k_uf_init(int32_t* uf, int64_t V) { GRID_STRIDE(v, V) uf[v] = (int32_t)v; }

// Block representatives: non-root vertices that are their class root, and isolated tree roots.
// (Read-only root walk: path-halving writes of other threads could otherwise replace a root
// just stored in uf[v] by an intermediate ancestor; here the only writes are final roots.)
__global__ void k_block_flags(int64_t V, const int32_t* parent, const int32_t* nd, int32_t* uf, uint8_t* flag) {
    GRID_STRIDE(v, V) {
        const int32_t p = parent[v];
        const bool root = p == (int32_t)v;
        int32_t r = (int32_t)v;
        while (uf[r] != r) r = uf[r];
        uf[v] = r;
        flag[v] = root ? (nd[v] == 1) : (r == (int32_t)v);
    }
}

__global__ void k_block_ids(const int32_t* reps, int64_t nb, int32_t* id_of_rep) {
    GRID_STRIDE(b, nb) id_of_rep[reps[b]] = (int32_t)b;
}

// label_block and heads. A tree root's first block (that of its child with pre 1) is its parent
// block (head -1); its other blocks hang from it.
// Pass 1: the block of every tree root's first child (pre 1) becomes the root's parent block.
__global__ void k_root_block(int64_t V, const int32_t* parent, const int32_t* pre, const int32_t* uf,
                             const int32_t* id_of_rep, int32_t* label) {
    GRID_STRIDE(v, V) {
        const int32_t p = parent[v];
        if (p != (int32_t)v && parent[p] == p && pre[v] == 1) label[p] = id_of_rep[uf[v]];
    }
}

// Pass 2: parent blocks of the other vertices, and heads: a block's head is the parent p of its
// topmost child ends (p is a tree root, or p's own parent edge is in another block); the root's
// parent block has head -1.
__global__ void k_block_assign(int64_t V, const int32_t* parent, const int32_t* nd, const int32_t* uf,
                               const int32_t* id_of_rep, int32_t* label, int32_t* head) {
    GRID_STRIDE(v, V) {
        const int32_t p = parent[v];
        if (p == (int32_t)v) {
            if (nd[v] == 1) {  // isolated: singleton block
                const int32_t b = id_of_rep[v];
                label[v] = b;
                head[b] = -1;
            }
            continue;
        }
        const int32_t b = id_of_rep[uf[v]];
        label[v] = b;
        const bool p_root = parent[p] == p;
        if (p_root || uf[p] != uf[v]) head[b] = (p_root && label[p] == b) ? -1 : p;
    }
}

__global__ void k_bcnt(int64_t V, const int32_t* head, int64_t nb, int32_t* bcnt) {
    GRID_STRIDE(v, V) bcnt[v] = 1;
}

__global__ void k_bcnt_heads(const int32_t* head, int64_t nb, int32_t* bcnt) {
    GRID_STRIDE(b, nb) {
        const int32_t h = head[b];
        if (h >= 0) atomicAdd(&bcnt[h], 1);
    }
}

}  // namespace

int bct_build(gir_dev* g) {
    if (!g->scc_built) return fail(g, GIR_ERR_STATE, "buildBCT needs buildSCC_DAG first");
    const int64_t V = g->V;
    const int32_t* scc = static_cast<const int32_t*>(g->scc.p);
    HView h{view(g->sym), scc};  // (row lengths replaced by the H lengths below)
    int32_t *parent = nullptr, *depth = nullptr, *order = nullptr, *nd = nullptr, *pre = nullptr, *off = nullptr;
    int32_t *low = nullptr, *high = nullptr, *uf = nullptr, *reps = nullptr, *id_of_rep = nullptr;
    uint64_t *keys = nullptr, *ktmp = nullptr;
    uint8_t* flag = nullptr;
    int64_t *scan = nullptr, *first = nullptr;
    unsigned long long* cnt = nullptr;
    GIR_TRY(ensure_n(g, g->scratch[0], V + 1, &parent));
    GIR_TRY(ensure_n(g, g->scratch[1], V + 1, &depth));
    GIR_TRY(ensure_n(g, g->scratch[2], V + 1, &order));
    GIR_TRY(ensure_n(g, g->scratch[3], V + 1, &nd));
    GIR_TRY(ensure_n(g, g->scratch[4], V + 1, &pre));
    GIR_TRY(ensure_n(g, g->scratch[5], V + 1, &off));
    GIR_TRY(ensure_n(g, g->scratch[6], V + 1, &low));
    GIR_TRY(ensure_n(g, g->scratch[7], V + 1, &high));
    GIR_TRY(ensure_n(g, g->scratch[8], V + 1, &uf));
    GIR_TRY(ensure_n(g, g->scratch[9], V + 1, &keys));
    GIR_TRY(ensure_n(g, g->scratch[10], V + 1, &ktmp));
    GIR_TRY(ensure_n(g, g->scratch[11], V + 1, &flag));
    GIR_TRY(ensure_n(g, g->scratch[12], V + 2, &scan));
    GIR_TRY(ensure_n(g, g->scratch[13], V + 1, &first));
    GIR_TRY(ensure_n(g, g->scratch[14], 2 * C_N, &cnt));
    void* hp = nullptr;
    GIR_TRY(pinned(g, 256, &hp));
    unsigned long long* hc = static_cast<unsigned long long*>(hp);
    int32_t *label = nullptr, *head = nullptr, *bcnt = nullptr;
    GIR_TRY(ensure_n(g, g->blk_label, V + 1, &label));
    GIR_TRY(ensure_n(g, g->bcnt, V + 1, &bcnt));
    if (V == 0) {
        g->n_blocks = 0;
        g->bct_built = true;
        return GIR_OK;
    }
    auto read = [&]() -> int {
        GIR_CUDA(g, cudaMemcpyAsync(hc, cnt, sizeof(unsigned long long) * C_N, cudaMemcpyDeviceToHost, g->stream));
        GIR_CUDA(g, cudaStreamSynchronize(g->stream));
        return GIR_OK;
    };
    trace_mark(g, "bct: start");
    // 1. BFS forest; order[] holds the levels back to back, lvl_off their boundaries
    GIR_CUDA(g, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * 2 * C_N, g->stream));
    uint8_t* nontrivial = nullptr;
    int32_t* hdeg = nullptr;
    GIR_TRY(ensure_n(g, g->work[6], V + 1, &nontrivial));
    GIR_TRY(ensure_n(g, g->work[7], V + 1, &hdeg));
    GIR_CUDA(g, cudaMemsetAsync(nontrivial, 0, V, g->stream));
    k_mark_nontrivial<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, scc, nontrivial);
    GIR_LAUNCH(g, "k_mark_nontrivial");
    k_h_deg<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, scc, nontrivial, g->sym.deg, hdeg);
    GIR_LAUNCH(g, "k_h_deg");
    h.sym.deg = hdeg;
    k_roots<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, scc, nontrivial, parent, depth, order, cnt);
    GIR_LAUNCH(g, "k_roots");
    GIR_TRY(read());
    std::vector<int64_t> lvl_off{0, (int64_t)hc[C_Q]};
    for (int32_t L = 0;; ++L) {
        const int64_t lo = lvl_off[L], n = lvl_off[L + 1] - lo;
        if (n == 0) break;
        GIR_CUDA(g, cudaMemsetAsync(&cnt[C_Q], 0, sizeof(unsigned long long), g->stream));
        // (`scan` serves as the level's row-length prefix here; the preorder step reuses it later)
        k_level_deg<<<grid_for(g, n, kBlock), kBlock, 0, g->stream>>>(order + lo, n, h.sym.deg, scan);
        GIR_LAUNCH(g, "k_level_deg");
        GIR_TRY(exclusive_scan_i64(g, scan, scan, n + 1));
        k_forest_balanced<<<g->num_sms * 8, kBlock, 0, g->stream>>>(order + lo, n, scan, h, parent, depth, L,
                                                                    order + lo + n, cnt);
        GIR_LAUNCH(g, "k_forest_balanced");
        GIR_TRY(read());
        lvl_off.push_back(lvl_off.back() + (int64_t)hc[C_Q]);
    }
    const int D = (int)lvl_off.size() - 1;  // levels 0..D-1 (the last entry repeats the end)
    trace_mark(g, "bct: forest");
    // 2. subtree sizes, bottom-up
    k_fill_i32<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(nd, V, 1);
    GIR_LAUNCH(g, "k_fill_i32");
    for (int L = D - 1; L >= 1; --L) {
        const int64_t n = lvl_off[L + 1] - lvl_off[L];
        if (n == 0) continue;
        k_nd_level<<<grid_for(g, n, kBlock), kBlock, 0, g->stream>>>(order + lvl_off[L], n, parent, nd);
        GIR_LAUNCH(g, "k_nd_level");
    }
    //    preorder: children grouped by parent, sibling offsets, then levels top-down
    k_child_keys<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, parent, keys, flag);
    GIR_LAUNCH(g, "k_child_keys");
    int64_t nc = 0;
    GIR_TRY(select_flagged_u64(g, keys, flag, ktmp, V, &nc));
    GIR_TRY(sort_keys_u64(g, ktmp, keys, nc, 64));
    if (nc > 0) {
        k_child_nd<<<grid_for(g, nc, kBlock), kBlock, 0, g->stream>>>(ktmp, nc, nd, scan);
        GIR_LAUNCH(g, "k_child_nd");
        GIR_TRY(exclusive_scan_i64(g, scan, scan, nc + 1));
        k_group_first<<<grid_for(g, nc, kBlock), kBlock, 0, g->stream>>>(ktmp, nc, first);
        GIR_LAUNCH(g, "k_group_first");
        k_sibling_off<<<grid_for(g, nc, kBlock), kBlock, 0, g->stream>>>(ktmp, nc, scan, first, off);
        GIR_LAUNCH(g, "k_sibling_off");
    }
    k_pre_roots<<<grid_for(g, lvl_off[1], kBlock), kBlock, 0, g->stream>>>(order, lvl_off[1], pre);
    GIR_LAUNCH(g, "k_pre_roots");
    for (int L = 1; L < D; ++L) {
        const int64_t n = lvl_off[L + 1] - lvl_off[L];
        if (n == 0) continue;
        k_pre_level<<<grid_for(g, n, kBlock), kBlock, 0, g->stream>>>(order + lvl_off[L], n, parent, off, pre);
        GIR_LAUNCH(g, "k_pre_level");
    }
    trace_mark(g, "bct: subtree sizes + preorder");
    // 3. low / high and rule 1
    GIR_CUDA(g, cudaMemcpyAsync(low, pre, sizeof(int32_t) * V, cudaMemcpyDeviceToDevice, g->stream));
    GIR_CUDA(g, cudaMemcpyAsync(high, pre, sizeof(int32_t) * V, cudaMemcpyDeviceToDevice, g->stream));
    k_uf_init<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(uf, V);
    GIR_LAUNCH(g, "k_uf_init");
    int4* vinfo = nullptr;
    GIR_TRY(ensure_n(g, g->work[5], V + 1, &vinfo));
    k_pack_vinfo<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, pre, nd, parent, scc, vinfo);
    GIR_LAUNCH(g, "k_pack_vinfo");
    k_nontree_sample<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, h, vinfo, uf, &cnt[C_ERR]);
    GIR_LAUNCH(g, "k_nontree_sample");
    k_uf_flatten<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(uf, V);
    GIR_LAUNCH(g, "k_uf_flatten");
    k_nontree<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, h, vinfo, low, high, uf, &cnt[C_ERR]);
    GIR_LAUNCH(g, "k_nontree");
    {
        int64_t n_heavy = 0;  // (first / scan are free after the preorder)
        int32_t* heavy = reinterpret_cast<int32_t*>(first);
        GIR_TRY(heavy_rows(g, h.sym.deg, V, kHeavyRow, flag, heavy, scan, &n_heavy));
        if (n_heavy > 0) {
            k_nontree_heavy<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(heavy, scan, n_heavy, h, vinfo, low, high,
                                                                             uf, &cnt[C_ERR]);
            GIR_LAUNCH(g, "k_nontree_heavy");
        }
    }
    for (int L = D - 1; L >= 1; --L) {
        const int64_t n = lvl_off[L + 1] - lvl_off[L];
        if (n == 0) continue;
        k_lowhigh_level<<<grid_for(g, n, kBlock), kBlock, 0, g->stream>>>(order + lvl_off[L], n, parent, low, high);
        GIR_LAUNCH(g, "k_lowhigh_level");
    }
    trace_mark(g, "bct: low/high + rule 1");
    // 4. rule 2
    k_rule2<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, parent, pre, nd, low, high, uf, &cnt[C_ERR]);
    GIR_LAUNCH(g, "k_rule2");
    trace_mark(g, "bct: rule 2");
    // 5. blocks
    k_block_flags<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, parent, nd, uf, flag);
    GIR_LAUNCH(g, "k_block_flags");
    reps = off;  // (sibling offsets are no longer needed)
    int64_t nb = 0;
    GIR_TRY(select_flagged_iota(g, flag, reps, V, &nb));
    id_of_rep = low;
    k_block_ids<<<grid_for(g, nb, kBlock), kBlock, 0, g->stream>>>(reps, nb, id_of_rep);
    GIR_LAUNCH(g, "k_block_ids");
    GIR_TRY(ensure_n(g, g->blk_head, nb + 1, &head));
    k_root_block<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, parent, pre, uf, id_of_rep, label);
    GIR_LAUNCH(g, "k_root_block");
    k_block_assign<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, parent, nd, uf, id_of_rep, label, head);
    GIR_LAUNCH(g, "k_block_assign");
    k_bcnt<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, head, nb, bcnt);
    GIR_LAUNCH(g, "k_bcnt");
    k_bcnt_heads<<<grid_for(g, nb, kBlock), kBlock, 0, g->stream>>>(head, nb, bcnt);
    GIR_LAUNCH(g, "k_bcnt_heads");
    GIR_TRY(read());
    if (hc[C_ERR]) return fail(g, GIR_ERR_TIMEOUT, "bct: union-find exceeded its retry bound");
    g->n_blocks = nb;
    g->bct_built = true;
    trace_mark(g, "bct: blocks");
    return GIR_OK;
}

}  // namespace gir
