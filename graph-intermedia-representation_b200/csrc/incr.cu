// Incremental single-source BFS / SSSP (GIR::trackIncremental / updateIncremental / incDist,
// gir_query.cpp:867-996, gir.h:220-232 and 524-533), KickStarter-style.
//
// State per mode ([0] BFS, weight 1; [1] SSSP, GIR::edgeWeight): one 64-bit word per vertex,
// dist << 32 | parent (the reference's own word, so a 64-bit atomicMin orders candidates by
// distance, then by parent id), all ones = unreachable; and the edge keys (u << 32 | v) that
// batches changed since the last update.
//
// Update, every step a grid-wide kernel over HBM-resident arrays:
//  1. presence of every logged edge now (binary search of u's sorted forward row);
//  2. invalidation: a deleted tree edge u -> v cuts v; the cut spreads down the dependence tree
//     (out-neighbours whose parent is a cut vertex) level by level. All cut vertices land in one
//     list, each level appended behind the previous one, so the list needs no second pass;
//  3. every cut vertex restarts from its valid in-neighbours (one warp per vertex, min-reduce of
//     the candidate words);
//  4. seeds: the re-seeded cut vertices and the heads of inserted edges that improve;
//  5. propagation: frontier Bellman-Ford. A vertex is queued at most once per round (a flag
//     set by compare-and-swap); the flags of a round's frontier are cleared in their own launch
//     before the round reads any distance, so an improvement that lands after a vertex has
//     read its own distance finds the flag clear and queues it again.
// Distances only fall during propagation and every word is the length of a real path, so the
// result is the exact shortest-distance vector whatever the order of the relaxations (parents
// may differ from the reference's where several in-neighbours tie; distances cannot).
#include <algorithm>

#include "common.cuh"

namespace gir {

namespace {

constexpr int kBlock = 256;
constexpr uint64_t kNone = ~0ull;
enum : uint32_t { FLAG_CLEAR = 0, FLAG_CUT = 1, FLAG_QUEUED = 2 };

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

__device__ __forceinline__ uint64_t weight_of(int weighted, int32_t a, int32_t b) {
    return weighted ? (uint64_t)hash_weight(a, b) : 1ull;
}
__device__ __forceinline__ int32_t parent_of(uint64_t k) { return (int32_t)(uint32_t)k; }
__device__ __forceinline__ uint64_t pack(uint64_t d, int32_t p) { return (d << 32) | (uint32_t)p; }

__device__ __forceinline__ uint64_t warp_min_u64(uint64_t x) {
    for (int o = 16; o; o >>= 1) {
        const uint64_t t = __shfl_xor_sync(0xffffffffu, x, o);
        x = t < x ? t : x;
    }
    return x;
}

// BFS levels (int32, -1 = unreached) as distances.
__global__ void k_inc_levels(const int32_t* level, int64_t V, uint64_t* d) {
    GRID_STRIDE(v, V) d[v] = level[v] < 0 ? kNone : (uint64_t)level[v];
}

// Tree words from one traversal's distances (trackIncremental, gir_query.cpp:879-891): the
// parent of a reached v != source is its smallest in-neighbour p with d[p] + w(p, v) = d[v].
// One warp per vertex.
__global__ void k_inc_tree(int64_t V, CSRView bw, const uint64_t* d, int32_t src, int weighted, uint64_t* st) {
    const int ln = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t v = warp; v < V; v += nwarps) {
        const uint64_t dv = d[v];
        if (dv == kNone || v == src) {
            if (ln == 0) st[v] = dv == kNone ? kNone : (uint64_t)(uint32_t)src;
            continue;
        }
        const int64_t b = bw.beg[v], e = b + bw.deg[v];
        uint64_t best = kNone;
        for (int64_t k = b + ln; k < e; k += 32) {
            const int32_t p = bw.adj[k];
            const uint64_t dp = d[p];
            if (dp != kNone && dp + weight_of(weighted, p, (int32_t)v) == dv) {
                const uint64_t c = (uint64_t)(uint32_t)p;
                best = c < best ? c : best;
            }
        }
        best = warp_min_u64(best);
        if (ln == 0) st[v] = pack(dv, best == kNone ? -1 : (int32_t)best);
    }
}

// present[i] = the edge of key i is in the graph now.
__global__ void k_inc_present(const uint64_t* keys, int64_t n, CSRView fw, uint8_t* present) {
    GRID_STRIDE(i, n) {
        const int32_t u = (int32_t)(keys[i] >> 32), v = (int32_t)(uint32_t)keys[i];
        const int64_t b = fw.beg[u], e = b + fw.deg[u];
        const int64_t k = lower_bound_dev(fw.adj, b, e, v);
        present[i] = k < e && fw.adj[k] == v;
    }
}

// Step 2 seeds (gir_query.cpp:934-940): a logged edge that is absent now and was v's tree edge.
__global__ void k_inc_cut(const uint64_t* keys, const uint8_t* present, int64_t n, int32_t src, const uint64_t* st,
                          uint32_t* flag, int32_t* cut, unsigned long long* cnt) {
    __shared__ int32_t s_q[kBlock / 32][kStage];
    int n_q = 0;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < n; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = base + threadIdx.x;  // (block-uniform trip count: every lane joins the appends)
        bool push = false;
        int32_t v = 0;
        if (i < n && !present[i]) {
            const int32_t u = (int32_t)(keys[i] >> 32);
            v = (int32_t)(uint32_t)keys[i];
            const uint64_t k = st[v];
            push = v != src && k != kNone && parent_of(k) == u && atomicCAS(&flag[v], FLAG_CLEAR, FLAG_CUT) == FLAG_CLEAR;
        }
        stage_append(push, v, s_q[threadIdx.x >> 5], n_q, cut, cnt);
    }
    stage_flush(s_q[threadIdx.x >> 5], n_q, cut, cnt);
}

// One level of the cut (gir_query.cpp:941-953): out-neighbours whose parent is a cut vertex
// of the level, appended behind it in the same list.
__global__ void k_inc_cut_level(const int32_t* level_q, int64_t n, CSRView fw, int32_t src, const uint64_t* st,
                                uint32_t* flag, int32_t* cut, unsigned long long* cnt) {
    warp_expand(level_q, n, fw, cut, cnt, [&](int32_t x, int32_t y) {
        if (y == src) return false;
        const uint64_t k = st[y];
        return k != kNone && parent_of(k) == x && atomicCAS(&flag[y], FLAG_CLEAR, FLAG_CUT) == FLAG_CLEAR;
    });
}

__global__ void k_inc_unset(const int32_t* cut, int64_t n, uint64_t* st) {
    GRID_STRIDE(i, n) st[cut[i]] = kNone;
}

// Step 3 (gir_query.cpp:955-968): a cut vertex restarts from its best valid in-neighbour. One
// warp per cut vertex; the cut vertices' own words (kNone or being rewritten) are skipped by flag.
__global__ void k_inc_reseed(const int32_t* cut, int64_t n, CSRView bw, const uint32_t* flag, int weighted,
                             uint64_t* st) {
    const int ln = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = warp; i < n; i += nwarps) {
        const int32_t x = cut[i];
        const int64_t b = bw.beg[x], e = b + bw.deg[x];
        uint64_t best = kNone;
        for (int64_t k = b + ln; k < e; k += 32) {
            const int32_t p = bw.adj[k];
            if (flag[p] == FLAG_CUT) continue;
            const uint64_t kp = st[p];
            if (kp == kNone) continue;
            const uint64_t c = pack((kp >> 32) + weight_of(weighted, p, x), p);
            best = c < best ? c : best;
        }
        best = warp_min_u64(best);
        if (ln == 0) st[x] = best;
    }
}

// Step 4a (gir_query.cpp:969-972): the cut vertices' flags are cleared; the re-seeded ones are queued.
__global__ void k_inc_seed_cut(const int32_t* cut, int64_t n, const uint64_t* st, uint32_t* flag, int32_t* q,
                               unsigned long long* cnt) {
    __shared__ int32_t s_q[kBlock / 32][kStage];
    int n_q = 0;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < n; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = base + threadIdx.x;
        bool push = false;
        int32_t x = 0;
        if (i < n) {
            x = cut[i];
            push = st[x] != kNone;
            flag[x] = push ? FLAG_QUEUED : FLAG_CLEAR;
        }
        stage_append(push, x, s_q[threadIdx.x >> 5], n_q, q, cnt);
    }
    stage_flush(s_q[threadIdx.x >> 5], n_q, q, cnt);
}

// Step 4b (gir_query.cpp:973-981): logged edges present now relax once.
__global__ void k_inc_seed_edges(const uint64_t* keys, const uint8_t* present, int64_t n, int weighted, uint64_t* st,
                                 uint32_t* flag, int32_t* q, unsigned long long* cnt) {
    __shared__ int32_t s_q[kBlock / 32][kStage];
    int n_q = 0;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < n; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = base + threadIdx.x;
        bool push = false;
        int32_t v = 0;
        if (i < n && present[i]) {
            const int32_t u = (int32_t)(keys[i] >> 32);
            v = (int32_t)(uint32_t)keys[i];
            const uint64_t k = __ldcg(&st[u]);
            if (k != kNone) {
                const uint64_t c = pack((k >> 32) + weight_of(weighted, u, v), u);
                push = c < atomicMin((unsigned long long*)&st[v], (unsigned long long)c) &&
                       atomicCAS(&flag[v], FLAG_CLEAR, FLAG_QUEUED) == FLAG_CLEAR;
            }
        }
        stage_append(push, v, s_q[threadIdx.x >> 5], n_q, q, cnt);
    }
    stage_flush(s_q[threadIdx.x >> 5], n_q, q, cnt);
}

__global__ void k_inc_unflag(const int32_t* q, int64_t n, uint32_t* flag) {
    GRID_STRIDE(i, n) flag[q[i]] = FLAG_CLEAR;
}

// Step 5, one round (gir_query.cpp:983-995): every frontier vertex relaxes its out-edges with its
// current word (read through L2: other CTAs lower it during the round).
__global__ void k_inc_round(const int32_t* q, int64_t n, CSRView fw, int weighted, uint64_t* st, uint32_t* flag,
                            int32_t* nq, unsigned long long* ncnt) {
    warp_expand(q, n, fw, nq, ncnt, [&](int32_t x, int32_t y) {
        const uint64_t c = pack((__ldcg(&st[x]) >> 32) + weight_of(weighted, x, y), x);
        return c < __ldcg(&st[y]) && c < atomicMin((unsigned long long*)&st[y], (unsigned long long)c) &&
               atomicCAS(&flag[y], FLAG_CLEAR, FLAG_QUEUED) == FLAG_CLEAR;
    });
}

__global__ void k_inc_dist(const uint64_t* st, int64_t V, uint64_t* out) {
    GRID_STRIDE(v, V) {
        const uint64_t k = st[v];
        out[v] = k == kNone ? kNone : k >> 32;
    }
}

// Reads cnt[0] (after the stream's queued work).
int read_count(gir_dev* g, const unsigned long long* cnt, unsigned long long* host, int64_t* out) {
    GIR_CUDA(g, cudaMemcpyAsync(host, cnt, sizeof(unsigned long long), cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    *out = (int64_t)host[0];
    return GIR_OK;
}

}  // namespace

int inc_track(gir_dev* g, int32_t source, int weighted) {
    const int m = weighted ? 1 : 0;
    const int64_t V = g->V;
    const double t0 = now_ms();
    GIR_TRY(ensure(g, g->inc_st[m], sizeof(uint64_t) * (size_t)(V > 0 ? V : 1)));
    g->inc_src[m] = source;
    g->inc_on[m] = true;
    g->inc_npend[m] = 0;
    if (V == 0) return GIR_OK;
    uint64_t* st = static_cast<uint64_t*>(g->inc_st[m].p);
    uint64_t* d = nullptr;
    int32_t* src_d = nullptr;
    GIR_TRY(dev_alloc_n(g, &d, (size_t)V));
    GIR_TRY(dev_alloc_n(g, &src_d, 4));
    int rc = GIR_OK;
    const QueryStats keep = g->qstats;
    const int64_t set_beg[2] = {0, 1};
    if (!(rc = cuda_check(g, cudaMemcpyAsync(src_d, &source, sizeof(int32_t), cudaMemcpyHostToDevice, g->stream),
                          "inc source"))) {
        if (weighted) {
            rc = sssp_run(g, set_beg, src_d, 1, (uint64_t)g->params[GIR_PARAM_DELTA], GIR_WEIGHT_HASH, d);
        } else {
            int32_t* level = nullptr;
            if (!(rc = dev_alloc_n(g, &level, (size_t)V)) && !(rc = bfs_run(g, set_beg, src_d, 1, level))) {
                k_inc_levels<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(level, V, d);
                rc = cuda_check(g, cudaGetLastError(), "k_inc_levels");
            }
            if (level) dev_free(g, level);
        }
    }
    if (!rc) {
        k_inc_tree<<<grid_for(g, V * 32, kBlock), kBlock, 0, g->stream>>>(V, view(g->bw), d, source, weighted, st);
        rc = cuda_check(g, cudaGetLastError(), "k_inc_tree");
    }
    if (!rc) rc = cuda_check(g, cudaStreamSynchronize(g->stream), "inc track");
    dev_free(g, src_d);
    dev_free(g, d);
    g->qstats = keep;
    g->qstats.total_ms = now_ms() - t0;
    return rc;
}

int inc_log(gir_dev* g, const uint64_t* ins, int64_t n_ins, const uint64_t* del, int64_t n_del) {
    for (int m = 0; m < 2; ++m) {
        if (!g->inc_on[m] || g->inc_src[m] < 0 || n_ins + n_del == 0) continue;
        const int64_t need = g->inc_npend[m] + n_ins + n_del;
        DevBuf& b = g->inc_pend[m];
        if ((size_t)need * sizeof(uint64_t) > b.bytes) {
            // grow with the logged keys kept
            const size_t cap = std::max<size_t>((size_t)need, b.bytes / sizeof(uint64_t) * 2) * sizeof(uint64_t);
            void* p = nullptr;
            GIR_TRY(dev_alloc(g, &p, cap));
            if (g->inc_npend[m] > 0)
                GIR_CUDA(g, cudaMemcpyAsync(p, b.p, sizeof(uint64_t) * g->inc_npend[m], cudaMemcpyDeviceToDevice, g->stream));
            release(g, b);
            b.p = p;
            b.bytes = cap;
        }
        uint64_t* k = static_cast<uint64_t*>(b.p) + g->inc_npend[m];
        if (n_ins > 0) GIR_CUDA(g, cudaMemcpyAsync(k, ins, sizeof(uint64_t) * n_ins, cudaMemcpyDeviceToDevice, g->stream));
        if (n_del > 0)
            GIR_CUDA(g, cudaMemcpyAsync(k + n_ins, del, sizeof(uint64_t) * n_del, cudaMemcpyDeviceToDevice, g->stream));
        g->inc_npend[m] = need;
    }
    return GIR_OK;
}

int inc_update(gir_dev* g, int weighted) {
    const int m = weighted ? 1 : 0;
    const int64_t V = g->V, np = g->inc_npend[m];
    const double t0 = now_ms();
    g->qstats = QueryStats{};
    if (!g->inc_on[m] || g->inc_src[m] < 0 || np == 0 || V == 0) return GIR_OK;
    const int32_t src = g->inc_src[m];
    uint64_t* st = static_cast<uint64_t*>(g->inc_st[m].p);
    const uint64_t* keys = static_cast<const uint64_t*>(g->inc_pend[m].p);
    uint8_t* present = nullptr;
    uint32_t* flag = nullptr;
    int32_t *cut = nullptr, *qa = nullptr, *qb = nullptr;
    unsigned long long* cnt = nullptr;
    void* hp = nullptr;
    GIR_TRY(pinned(g, 256, &hp));
    unsigned long long* hc = static_cast<unsigned long long*>(hp);
    int rc = GIR_OK;
    auto cleanup = [&]() {
        for (void* p : {(void*)present, (void*)flag, (void*)cut, (void*)qa, (void*)qb, (void*)cnt})
            if (p) dev_free(g, p);
    };
    if ((rc = dev_alloc_n(g, &present, (size_t)np)) || (rc = dev_alloc_n(g, &flag, (size_t)V)) ||
        (rc = dev_alloc_n(g, &cut, (size_t)V)) || (rc = dev_alloc_n(g, &qa, (size_t)V)) ||
        (rc = dev_alloc_n(g, &qb, (size_t)V)) || (rc = dev_alloc_n(g, &cnt, 4))) {
        cleanup();
        return rc;
    }
    int64_t launches = 0, rounds = 0, n_cut = 0, relaxed_from = 0;
    auto launched = [&](const char* what) {
        ++launches;
        return cuda_check(g, cudaGetLastError(), what);
    };
    const CSRView fw = view(g->fw), bw = view(g->bw);
    do {
        if ((rc = cuda_check(g, cudaMemsetAsync(flag, 0, sizeof(uint32_t) * (size_t)V, g->stream), "inc flags")) ||
            (rc = cuda_check(g, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * 4, g->stream), "inc counters")))
            break;
        k_inc_present<<<grid_for(g, np, kBlock), kBlock, 0, g->stream>>>(keys, np, fw, present);
        if ((rc = launched("k_inc_present"))) break;
        // 2. the cut, level by level into one list
        k_inc_cut<<<grid_for(g, np, kBlock), kBlock, 0, g->stream>>>(keys, present, np, src, st, flag, cut, cnt);
        if ((rc = launched("k_inc_cut"))) break;
        int64_t lo = 0, hi = 0;
        if ((rc = read_count(g, cnt, hc, &hi))) break;
        while (hi > lo) {
            k_inc_cut_level<<<grid_for(g, (hi - lo) * 32, kBlock), kBlock, 0, g->stream>>>(cut + lo, hi - lo, fw, src, st,
                                                                                          flag, cut, cnt);
            if ((rc = launched("k_inc_cut_level"))) break;
            lo = hi;
            if ((rc = read_count(g, cnt, hc, &hi))) break;
        }
        if (rc) break;
        n_cut = hi;
        // 3. re-seed the cut from valid in-neighbours
        if (n_cut > 0) {
            k_inc_unset<<<grid_for(g, n_cut, kBlock), kBlock, 0, g->stream>>>(cut, n_cut, st);
            if ((rc = launched("k_inc_unset"))) break;
            k_inc_reseed<<<grid_for(g, n_cut * 32, kBlock), kBlock, 0, g->stream>>>(cut, n_cut, bw, flag, weighted, st);
            if ((rc = launched("k_inc_reseed"))) break;
        }
        // 4. seeds
        if ((rc = cuda_check(g, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), g->stream), "inc counters"))) break;
        if (n_cut > 0) {
            k_inc_seed_cut<<<grid_for(g, n_cut, kBlock), kBlock, 0, g->stream>>>(cut, n_cut, st, flag, qa, cnt);
            if ((rc = launched("k_inc_seed_cut"))) break;
        }
        k_inc_seed_edges<<<grid_for(g, np, kBlock), kBlock, 0, g->stream>>>(keys, present, np, weighted, st, flag, qa,
                                                                            cnt);
        if ((rc = launched("k_inc_seed_edges"))) break;
        int64_t nq = 0;
        if ((rc = read_count(g, cnt, hc, &nq))) break;
        // 5. propagation rounds; distances strictly fall, so every vertex is queued at most V times
        const int64_t max_rounds = V + 2;
        while (nq > 0) {
            if (++rounds > max_rounds) {
                rc = fail(g, GIR_ERR_TIMEOUT, "inc update: propagation did not converge");
                break;
            }
            relaxed_from += nq;
            k_inc_unflag<<<grid_for(g, nq, kBlock), kBlock, 0, g->stream>>>(qa, nq, flag);
            if ((rc = launched("k_inc_unflag"))) break;
            if ((rc = cuda_check(g, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), g->stream), "inc counters"))) break;
            k_inc_round<<<grid_for(g, nq * 32, kBlock), kBlock, 0, g->stream>>>(qa, nq, fw, weighted, st, flag, qb, cnt);
            if ((rc = launched("k_inc_round"))) break;
            std::swap(qa, qb);
            if ((rc = read_count(g, cnt, hc, &nq))) break;
        }
    } while (false);
    if (!rc) {
        g->inc_npend[m] = 0;
        rc = cuda_check(g, cudaStreamSynchronize(g->stream), "inc update");
    }
    cleanup();
    g->qstats.iterations = rounds;
    g->qstats.reached = n_cut;
    g->qstats.edges = relaxed_from;
    g->qstats.launches = launches;
    g->qstats.total_ms = now_ms() - t0;
    return rc;
}

int inc_dist(gir_dev* g, int weighted, uint64_t* out_d) {
    const int m = weighted ? 1 : 0;
    if (g->V == 0) return GIR_OK;
    k_inc_dist<<<grid_for(g, g->V, kBlock), kBlock, 0, g->stream>>>(static_cast<const uint64_t*>(g->inc_st[m].p), g->V,
                                                                   out_d);
    GIR_LAUNCH(g, "k_inc_dist");
    return GIR_OK;
}

}  // namespace gir
