// Incremental single-source BFS / SSSP (GIR::trackIncremental / updateIncremental / incDist,
// gir_query.cpp:867-996, gir.h:220-232 and 524-533), KickStarter-style.
//
// State per mode ([0] BFS, weight 1; [1] SSSP, GIR::edgeWeight): one 64-bit word per vertex,
// dist << 32 | parent (the reference's own word, so a 64-bit atomicMin orders candidates by
// distance, then by parent id), all ones = unreachable; and the edge keys (u << 32 | v) that
// batches changed since the last update.
//
// Update, one cooperative launch over HBM-resident arrays whose phases are these steps:
//  1. presence of every logged edge now (binary search of u's sorted forward row);
//  2. invalidation: a deleted tree edge u -> v cuts v; the cut spreads down the dependence tree
//     (out-neighbours whose parent is a cut vertex) level by level. All cut vertices land in one
//     list, each level appended behind the previous one, so the list needs no second pass;
//  3. every cut vertex restarts from its valid in-neighbours (one warp per vertex, min-reduce of
//     the candidate words);
//  4. seeds: the re-seeded cut vertices and the heads of inserted edges that improve;
//  5. propagation: frontier Bellman-Ford. A vertex is queued at most once per round (a flag
//     set by compare-and-swap); the flags of a round's frontier are cleared in their own phase
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

__global__ void k_inc_dist(const uint64_t* st, int64_t V, uint64_t* out) {
    GRID_STRIDE(v, V) {
        const uint64_t k = st[v];
        out[v] = k == kNone ? kNone : k >> 32;
    }
}

// The whole update in one cooperative launch: the phases below are those of the steps in the
// file comment, separated by bounded grid barriers instead of launches and host reads (a small
// update's cost was its round trips: a cut level or a propagation round each waited for the
// host). Counts live in rings of three words: level (or round) k reads slot k % 3, appends behind
// itself counting in slot (k + 1) % 3, and zeroes slot (k + 2) % 3, which every CTA last read
// before the barrier that opened level k, so one barrier per level suffices. Data other CTAs
// write during the launch is read through L2 (ld.cg).
constexpr int kIncThreads = 256;
constexpr unsigned kIncSpins = 1u << 25;  // bounded barrier wait (a few seconds)
enum { I_ERR = 0, I_CUTC = 1, I_QC = 4, I_NCUT = 8, I_ROUNDS = 9, I_RELAXED = 10, I_BAR = 32, I_WORDS = 64 };

struct IncArgs {
    const uint64_t* keys;
    int64_t np;
    CSRView fw, bw;
    int32_t src;
    int weighted;
    uint64_t* st;
    uint32_t* flag;
    uint8_t* present;
    int32_t* cut;
    int32_t* q[2];
    unsigned long long* ctl;  // I_* words, zeroed by the host; the barrier at I_BAR
    int64_t max_rounds;
};

// Warp-uniform append: the warp's pushed values go to out[base + slot], slots from one atomicAdd.
__device__ __forceinline__ void warp_push(bool push, int32_t v, int32_t* out, int64_t base, unsigned long long* cnt) {
    const unsigned m = __ballot_sync(0xffffffffu, push);
    if (!m) return;
    const int leader = __ffs(m) - 1;
    unsigned long long b0 = 0;
    if (lane_id() == leader) b0 = atomicAdd(cnt, (unsigned long long)__popc(m));
    b0 = __shfl_sync(0xffffffffu, b0, leader);
    if (push) out[base + (int64_t)b0 + __popc(m & ((1u << lane_id()) - 1))] = v;
}

__global__ void __launch_bounds__(kIncThreads) k_inc_persistent(IncArgs a) {
    unsigned long long* const ctl = a.ctl;
    unsigned long long* const err = ctl + I_ERR;
    unsigned int* const bar = reinterpret_cast<unsigned int*>(ctl + I_BAR);
    const int ln = lane_id();
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t nthr = (int64_t)gridDim.x * blockDim.x;
    const int64_t warp = tid >> 5, nwarps = nthr >> 5;
    // 1. presence of every logged edge; 2a. an absent tree edge u -> v cuts v (cut level 0)
    for (int64_t base = warp * 32; base < a.np; base += nwarps * 32) {
        const int64_t i = base + ln;
        bool push = false;
        int32_t v = 0;
        if (i < a.np) {
            const int32_t u = (int32_t)(a.keys[i] >> 32);
            v = (int32_t)(uint32_t)a.keys[i];
            const int64_t b = a.fw.beg[u], e = b + a.fw.deg[u];
            const int64_t k = lower_bound_dev(a.fw.adj, b, e, v);
            const bool pr = k < e && a.fw.adj[k] == v;
            a.present[i] = pr;
            if (!pr && v != a.src) {
                const uint64_t w = a.st[v];
                push = w != kNone && parent_of(w) == u && atomicCAS(&a.flag[v], FLAG_CLEAR, FLAG_CUT) == FLAG_CLEAR;
            }
        }
        warp_push(push, v, a.cut, 0, ctl + I_CUTC);
    }
    if (!grid_barrier(bar, err, kIncSpins)) return;
    // 2b. the cut spreads down the dependence tree, level by level, behind itself in one list
    int64_t lo = 0, hi = (int64_t)__ldcg(ctl + I_CUTC);
    for (int k = 0; hi > lo; ++k) {
        unsigned long long* const nc = ctl + I_CUTC + (k + 1) % 3;
        if (tid == 0) ctl[I_CUTC + (k + 2) % 3] = 0ull;
        for (int64_t i = lo + warp; i < hi; i += nwarps) {
            const int32_t x = __ldcg(&a.cut[i]);
            const int64_t b = a.fw.beg[x], e = b + a.fw.deg[x];
            for (int64_t c = b; c < e; c += 32) {
                bool push = false;
                int32_t y = 0;
                if (c + ln < e) {
                    y = a.fw.adj[c + ln];
                    if (y != a.src) {
                        const uint64_t w = a.st[y];
                        push = w != kNone && parent_of(w) == x &&
                               atomicCAS(&a.flag[y], FLAG_CLEAR, FLAG_CUT) == FLAG_CLEAR;
                    }
                }
                warp_push(push, y, a.cut, hi, nc);
            }
        }
        if (!grid_barrier(bar, err, kIncSpins)) return;
        lo = hi;
        hi += (int64_t)__ldcg(nc);
    }
    const int64_t n_cut = hi;
    // 3. the cut vertices restart from their best valid in-neighbour (cut words are skipped by flag)
    for (int64_t i = tid; i < n_cut; i += nthr) a.st[__ldcg(&a.cut[i])] = kNone;
    if (!grid_barrier(bar, err, kIncSpins)) return;
    for (int64_t i = warp; i < n_cut; i += nwarps) {
        const int32_t x = __ldcg(&a.cut[i]);
        const int64_t b = a.bw.beg[x], e = b + a.bw.deg[x];
        uint64_t best = kNone;
        for (int64_t k = b + ln; k < e; k += 32) {
            const int32_t p = a.bw.adj[k];
            if (__ldcg(&a.flag[p]) == FLAG_CUT) continue;
            const uint64_t kp = __ldcg(&a.st[p]);
            if (kp == kNone) continue;
            const uint64_t c = pack((kp >> 32) + weight_of(a.weighted, p, x), p);
            best = c < best ? c : best;
        }
        best = warp_min_u64(best);
        if (ln == 0) a.st[x] = best;
    }
    if (!grid_barrier(bar, err, kIncSpins)) return;
    // 4a. the re-seeded cut vertices start the first frontier (round 0 counts in ring slot 0)
    for (int64_t base = warp * 32; base < n_cut; base += nwarps * 32) {
        const int64_t i = base + ln;
        bool push = false;
        int32_t x = 0;
        if (i < n_cut) {
            x = __ldcg(&a.cut[i]);
            push = __ldcg(&a.st[x]) != kNone;
            a.flag[x] = push ? FLAG_QUEUED : FLAG_CLEAR;
        }
        warp_push(push, x, a.q[0], 0, ctl + I_QC);
    }
    if (!grid_barrier(bar, err, kIncSpins)) return;
    // 4b. logged edges present now relax once
    for (int64_t base = warp * 32; base < a.np; base += nwarps * 32) {
        const int64_t i = base + ln;
        bool push = false;
        int32_t v = 0;
        if (i < a.np && __ldcg(&a.present[i])) {
            const int32_t u = (int32_t)(a.keys[i] >> 32);
            v = (int32_t)(uint32_t)a.keys[i];
            const uint64_t k = __ldcg(&a.st[u]);
            if (k != kNone) {
                const uint64_t c = pack((k >> 32) + weight_of(a.weighted, u, v), u);
                push = c < atomicMin((unsigned long long*)&a.st[v], (unsigned long long)c) &&
                       atomicCAS(&a.flag[v], FLAG_CLEAR, FLAG_QUEUED) == FLAG_CLEAR;
            }
        }
        warp_push(push, v, a.q[0], 0, ctl + I_QC);
    }
    if (!grid_barrier(bar, err, kIncSpins)) return;
    // 5. propagation rounds: the frontier's flags are cleared before any of its distances is read
    int64_t n = (int64_t)__ldcg(ctl + I_QC), r = 0, relaxed = 0;
    for (; n > 0; ++r) {
        if (r >= a.max_rounds) {
            if (tid == 0) atomicExch(err, 2ull);  // (distances strictly fall: cannot happen)
            return;
        }
        const int32_t* in = a.q[r & 1];
        int32_t* out = a.q[(r + 1) & 1];
        unsigned long long* const nc = ctl + I_QC + (r + 1) % 3;
        if (tid == 0) ctl[I_QC + (r + 2) % 3] = 0ull;
        relaxed += n;
        for (int64_t i = tid; i < n; i += nthr) a.flag[__ldcg(&in[i])] = FLAG_CLEAR;
        if (!grid_barrier(bar, err, kIncSpins)) return;
        for (int64_t i = warp; i < n; i += nwarps) {
            const int32_t x = __ldcg(&in[i]);
            const int64_t b = a.fw.beg[x], e = b + a.fw.deg[x];
            for (int64_t c = b; c < e; c += 32) {
                bool push = false;
                int32_t y = 0;
                if (c + ln < e) {
                    y = a.fw.adj[c + ln];
                    const uint64_t cand = pack((__ldcg(&a.st[x]) >> 32) + weight_of(a.weighted, x, y), x);
                    push = cand < __ldcg(&a.st[y]) &&
                           cand < atomicMin((unsigned long long*)&a.st[y], (unsigned long long)cand) &&
                           atomicCAS(&a.flag[y], FLAG_CLEAR, FLAG_QUEUED) == FLAG_CLEAR;
                }
                warp_push(push, y, out, 0, nc);
            }
        }
        if (!grid_barrier(bar, err, kIncSpins)) return;
        n = (int64_t)__ldcg(nc);
    }
    if (tid == 0) {
        ctl[I_NCUT] = (unsigned long long)n_cut;
        ctl[I_ROUNDS] = (unsigned long long)r;
        ctl[I_RELAXED] = (unsigned long long)relaxed;
    }
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
        (rc = dev_alloc_n(g, &qb, (size_t)V)) || (rc = dev_alloc_n(g, &cnt, I_WORDS))) {
        cleanup();
        return rc;
    }
    int64_t launches = 0, rounds = 0, n_cut = 0, relaxed_from = 0;
    do {
        if ((rc = cuda_check(g, cudaMemsetAsync(flag, 0, sizeof(uint32_t) * (size_t)V, g->stream), "inc flags")) ||
            (rc = cuda_check(g, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * I_WORDS, g->stream), "inc counters")))
            break;
        // one cooperative launch: every CTA of the grid must be resident at once
        int per_sm = 0;
        if ((rc = cuda_check(g, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_inc_persistent, kIncThreads, 0),
                             "inc occupancy")))
            break;
        const int grid = g->num_sms * std::max(1, std::min(per_sm, 4));
        IncArgs ia;
        ia.keys = keys;
        ia.np = np;
        ia.fw = view(g->fw);
        ia.bw = view(g->bw);
        ia.src = src;
        ia.weighted = weighted;
        ia.st = st;
        ia.flag = flag;
        ia.present = present;
        ia.cut = cut;
        ia.q[0] = qa;
        ia.q[1] = qb;
        ia.ctl = cnt;
        ia.max_rounds = V + 2;  // distances strictly fall, so every vertex is queued at most V times
        void* kargs[] = {&ia};
        if ((rc = cuda_check(g, cudaLaunchCooperativeKernel((const void*)k_inc_persistent, grid, kIncThreads, kargs, 0,
                                                            g->stream), "k_inc_persistent")))
            break;
        ++launches;
        if ((rc = cuda_check(g, cudaMemcpyAsync(hc, cnt, sizeof(unsigned long long) * 16, cudaMemcpyDeviceToHost, g->stream),
                             "inc counters")) ||
            (rc = cuda_check(g, cudaStreamSynchronize(g->stream), "inc update")))
            break;
        if (hc[I_ERR] == 2ull) {
            rc = fail(g, GIR_ERR_TIMEOUT, "inc update: propagation did not converge");
            break;
        }
        if (hc[I_ERR]) {
            rc = fail(g, GIR_ERR_TIMEOUT, "inc update: a grid barrier ran out its bound");
            break;
        }
        n_cut = (int64_t)hc[I_NCUT];
        rounds = (int64_t)hc[I_ROUNDS];
        relaxed_from = (int64_t)hc[I_RELAXED];
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
