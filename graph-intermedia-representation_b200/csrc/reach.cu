// Reachability queries on the SCC / condensation layer (GIR::reachable, gir_query.cpp:789-825).
//
// u ~> v iff u and v share an SCC, or SCC(v) is reachable from SCC(u) in the condensation DAG.
// Every DAG edge goes from a lower to a higher rank, so a path SCC(u) ~> SCC(v) only visits SCCs
// whose rank lies in [rank(SCC(u)), rank(SCC(v))]; a query with rank(SCC(u)) > rank(SCC(v)) is
// false at once. The reference answers one query by a bidirectional search over the DAG; here a
// batch of queries is answered together:
//  1. one kernel settles the queries that need no search and queues the rest. Besides the same
//     SCC (true), ranks in the wrong order (false) and ids out of range, a landmark index settles
//     most pairs: 64 hub vertices (largest out x in degree, distinct SCCs), and for every vertex
//     F(v) = the hubs that reach v and R(v) = the hubs v reaches (two 64-lane BFS, forward and on
//     the transposed graph, built once per condensation). Then u ~> v if R(u) & F(v) != 0 (through
//     a hub); not if some hub reaches u but not v (F(u) & ~F(v)), or v reaches a hub u does not
//     (R(v) & ~R(u));
//  2. the queued ones run 64 at a time as lanes of one level-synchronous forward search over the
//     DAG (its rows are the sorted condensation keys), every lane pruned to the SCCs whose rank is
//     at most its target's, until every lane has reached its target or run out of frontier.
#include <algorithm>
#include <vector>

#include "common.cuh"

namespace gir {

namespace {

constexpr int kBlock = 256;
constexpr int kChunk = 32 * 16;

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

// counters: [0] pending queries / frontier length, [1] candidates, [2] lanes found (mask)
enum { R_Q = 0, R_CAND = 1, R_FOUND = 2, R_N = 4 };

// Row starts of the DAG over labels: beg[a] = first key with source label >= a.
__global__ void k_dag_rows(const uint64_t* keys, int64_t n, int64_t V, int64_t* beg) {
    GRID_STRIDE(a, V + 1) {
        const uint64_t key = (uint64_t)a << 32;
        int64_t lo = 0, hi = n;
        while (lo < hi) {
            const int64_t m = (lo + hi) >> 1;
            if (keys[m] < key) lo = m + 1; else hi = m;
        }
        beg[a] = lo;
    }
}

// Masks of the landmark index from the 64 lanes' BFS levels (lane-major): bit s iff reached.
__global__ void k_levels_to_mask(const int32_t* level, int64_t V, int nl, uint64_t* mask) {
    GRID_STRIDE(v, V) {
        uint64_t m = 0;
        for (int s = 0; s < nl; ++s) m |= (uint64_t)(level[(int64_t)s * V + v] >= 0) << s;
        mask[v] = m;
    }
}

__global__ void k_reach_classify(const int32_t* u, const int32_t* v, int64_t n, int64_t V, const int32_t* scc,
                                 const int32_t* rank, const uint64_t* F, const uint64_t* R, uint8_t* out, int32_t* pend,
                                 unsigned long long* cnt) {
    __shared__ int32_t s_st[kBlock / 32][kStage];
    int n_st = 0;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < n; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = base + threadIdx.x;
        bool queue = false;
        if (i < n) {
            const int32_t a = u[i], b = v[i];
            uint8_t r = 0;
            if (a >= 0 && b >= 0 && a < V && b < V) {
                if (a == b || scc[a] == scc[b]) {
                    r = 1;
                } else if (rank[a] < rank[b]) {
                    const uint64_t fa = F[a], fb = F[b], ra = R[a], rb = R[b];
                    if (ra & fb) r = 1;
                    else queue = !((fa & ~fb) || (rb & ~ra));
                }
            }
            out[i] = r;
        }
        stage_append(queue, (int32_t)i, s_st[threadIdx.x >> 5], n_st, pend, &cnt[R_Q]);
    }
    stage_flush(s_st[threadIdx.x >> 5], n_st, pend, &cnt[R_Q]);
}

struct Lanes {
    int32_t src[64], dst[64];      // source and target labels
    int32_t sorted_bound[64];      // targets' ranks, ascending
    unsigned long long suffix[65]; // lanes at sorted positions k.. (those with bound >= sorted_bound[k])
};

// Lane setup for queries pend[g0 .. g0 + nl): labels, rank bounds sorted for the pruning masks, and
// the start of every lane (seen / frontier bit at its source label, the label queued once).
__global__ void k_reach_lanes(const int32_t* pend, int64_t g0, int nl, const int32_t* u, const int32_t* v,
                              const int32_t* scc, const int32_t* rank, Lanes* L, uint64_t* seen, uint64_t* front,
                              int32_t* q, unsigned long long* cnt) {
    __shared__ int32_t s_b[64], s_l[64];
    const int s = threadIdx.x;
    if (s < nl) {
        const int32_t qi = pend[g0 + s];
        const int32_t a = scc[u[qi]], b = scc[v[qi]];
        L->src[s] = a;
        L->dst[s] = b;
        s_b[s] = rank[v[qi]];
        s_l[s] = s;
        atomicOr((unsigned long long*)&seen[a], 1ull << s);
        if (atomicOr((unsigned long long*)&front[a], 1ull << s) == 0ull) q[atomicAdd(&cnt[R_Q], 1ull)] = a;
    }
    __syncthreads();
    if (s == 0) {
        for (int i = 1; i < nl; ++i) {  // insertion sort of at most 64 (bound, lane) pairs
            const int32_t b = s_b[i], l = s_l[i];
            int j = i - 1;
            while (j >= 0 && s_b[j] > b) {
                s_b[j + 1] = s_b[j];
                s_l[j + 1] = s_l[j];
                --j;
            }
            s_b[j + 1] = b;
            s_l[j + 1] = l;
        }
        unsigned long long m = 0;
        L->suffix[nl] = 0;
        for (int k = nl - 1; k >= 0; --k) {
            m |= 1ull << s_l[k];
            L->suffix[k] = m;
            L->sorted_bound[k] = s_b[k];
        }
    }
}

// Lanes allowed to enter an SCC of rank r: those whose target's rank is at least r.
__device__ __forceinline__ unsigned long long allowed(const Lanes* L, int nl, int32_t r) {
    int lo = 0, hi = nl;
    while (lo < hi) {
        const int m = (lo + hi) >> 1;
        if (L->sorted_bound[m] < r) lo = m + 1; else hi = m;
    }
    return L->suffix[lo];
}

__global__ void k_reach_degrees(const int32_t* q, int64_t nq, const int64_t* beg, int64_t* pref) {
    GRID_STRIDE(i, nq) pref[i] = beg[q[i] + 1] - beg[q[i]];
    if (blockIdx.x == 0 && threadIdx.x == 0) pref[nq] = 0;
}

// Edge-balanced expand over the frontier's DAG rows (as the BFS top-down expand); lanes already
// found stop spreading.
__global__ void k_reach_expand(const int32_t* q, int64_t nq, const int64_t* pref, const int64_t* beg,
                               const uint64_t* keys, const int32_t* rank, const Lanes* L, int nl, const uint64_t* front,
                               const uint64_t* seen, uint64_t* next, int32_t* cand, unsigned long long* cnt) {
    __shared__ int32_t s_st[kBlock / 32][kStage];
    int n_st = 0;
    const int64_t total = pref[nq];
    const unsigned long long live = ~cnt[R_FOUND];
    const int lane = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c0 = warp * kChunk; c0 < total; c0 += nwarps * kChunk) {
        const int64_t c1 = c0 + kChunk < total ? c0 + kChunk : total;
        const int64_t key = c0 + lane < total ? c0 + lane : total - 1;
        int64_t lo = 0, hi = nq - 1;
        while (lo < hi) {
            const int64_t m = (lo + hi + 1) >> 1;
            if (pref[m] <= key) lo = m; else hi = m - 1;
        }
        int64_t i = lo;
        for (int64_t base = c0; base < c1; base += 32) {
            const int64_t p = base + lane;
            bool fresh = false;
            int32_t y = 0;
            if (p < c1) {
                while (pref[i + 1] <= p) ++i;
                const int32_t x = q[i];
                y = (int32_t)(keys[beg[x] + (p - pref[i])] & 0xffffffffULL);
                const unsigned long long bits = front[x] & live & allowed(L, nl, rank[y]) & ~seen[y];
                if (bits) fresh = atomicOr((unsigned long long*)&next[y], bits) == 0ull;
            }
            stage_append(fresh, y, s_st[threadIdx.x >> 5], n_st, cand, &cnt[R_CAND]);
        }
    }
    stage_flush(s_st[threadIdx.x >> 5], n_st, cand, &cnt[R_CAND]);
}

__global__ void k_reach_clear(const int32_t* q, int64_t nq, uint64_t* front) { GRID_STRIDE(i, nq) front[q[i]] = 0; }

__global__ void k_reach_commit(const unsigned long long* n_cand, const int32_t* cand, uint64_t* seen, uint64_t* front,
                               uint64_t* next, int32_t* q, unsigned long long* cnt) {
    __shared__ int32_t s_st[kBlock / 32][kStage];
    int n_st = 0;
    const int64_t nc = (int64_t)*n_cand;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < nc; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = base + threadIdx.x;
        bool on = false;
        int32_t y = 0;
        if (i < nc) {
            y = cand[i];
            const uint64_t s = seen[y];
            const uint64_t nb = next[y] & ~s;
            next[y] = 0;
            if (nb) {
                seen[y] = s | nb;
                front[y] = nb;
                on = true;
            }
        }
        stage_append(on, y, s_st[threadIdx.x >> 5], n_st, q, &cnt[R_Q]);
    }
    stage_flush(s_st[threadIdx.x >> 5], n_st, q, &cnt[R_Q]);
}

// Lanes whose target now carries their bit.
__global__ void k_reach_found(const Lanes* L, int nl, const uint64_t* seen, unsigned long long* cnt) {
    const int s = threadIdx.x;
    const bool f = s < nl && ((seen[L->dst[s]] >> s) & 1ull);
    const unsigned m = __ballot_sync(0xffffffffu, f);
    if ((threadIdx.x & 31) == 0 && m)
        atomicOr(&cnt[R_FOUND], (unsigned long long)m << (threadIdx.x & 32));
}

__global__ void k_reach_write(const int32_t* pend, int64_t g0, int nl, const unsigned long long* cnt, uint8_t* out) {
    const int s = threadIdx.x;
    if (s < nl) out[pend[g0 + s]] = (uint8_t)((cnt[R_FOUND] >> s) & 1ull);
}

}  // namespace

// The landmark index: hubs chosen on the host from the degrees, then a 64-lane BFS from them on
// the forward graph (F) and on the transposed graph (R, the forward and backward stores swapped
// for the call).
static int build_hub_index(gir_dev* g) {
    const int64_t V = g->V;
    uint64_t* F = nullptr;
    GIR_TRY(ensure_n(g, g->reach_hub, 2 * (size_t)V + 1, &F));
    uint64_t* R = F + V;
    std::vector<int32_t> od((size_t)V), id((size_t)V), lab((size_t)V);
    GIR_CUDA(g, cudaMemcpyAsync(od.data(), g->fw.deg, sizeof(int32_t) * V, cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaMemcpyAsync(id.data(), g->bw.deg, sizeof(int32_t) * V, cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaMemcpyAsync(lab.data(), g->scc.p, sizeof(int32_t) * V, cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    std::vector<std::pair<uint64_t, int32_t>> score((size_t)V);
    for (int64_t v = 0; v < V; ++v) score[v] = {(uint64_t)(uint32_t)od[v] * (uint64_t)(uint32_t)id[v], (int32_t)v};
    std::sort(score.begin(), score.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
    std::vector<int32_t> hubs;
    std::vector<int32_t> used;
    for (const auto& sv : score) {
        if ((int)hubs.size() == 64 || sv.first == 0) break;
        const int32_t l = lab[sv.second];
        if (std::find(used.begin(), used.end(), l) != used.end()) continue;
        used.push_back(l);
        hubs.push_back(sv.second);
    }
    const int nl = (int)hubs.size();
    if (nl == 0) {
        GIR_CUDA(g, cudaMemsetAsync(F, 0, sizeof(uint64_t) * 2 * V, g->stream));
        g->reach_hub_valid = true;
        return GIR_OK;
    }
    int32_t *hubs_d = nullptr, *level = nullptr;
    GIR_TRY(dev_alloc_n(g, &hubs_d, 64));
    GIR_TRY(dev_alloc_n(g, &level, (size_t)nl * V + 1));
    GIR_CUDA(g, cudaMemcpyAsync(hubs_d, hubs.data(), sizeof(int32_t) * nl, cudaMemcpyHostToDevice, g->stream));
    std::vector<int64_t> sb((size_t)nl + 1);
    for (int i = 0; i <= nl; ++i) sb[i] = i;
    const QueryStats keep = g->qstats;
    const int sched = g->schedule;
    g->schedule = GIR_SCHEDULE_FIXED;
    int rc = bfs_run(g, sb.data(), hubs_d, nl, level);
    if (rc == GIR_OK) {
        k_levels_to_mask<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(level, V, nl, F);
        rc = cuda_check(g, cudaGetLastError(), "k_levels_to_mask");
    }
    if (rc == GIR_OK) {  // the transposed graph: swap the two stores around one more BFS
        std::swap(g->fw, g->bw);
        g->bins_valid = false;
        rc = bfs_run(g, sb.data(), hubs_d, nl, level);
        std::swap(g->fw, g->bw);
        g->bins_valid = false;
        if (rc == GIR_OK) {
            k_levels_to_mask<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(level, V, nl, R);
            rc = cuda_check(g, cudaGetLastError(), "k_levels_to_mask");
        }
    }
    g->schedule = sched;
    g->qstats = keep;
    dev_free(g, level);
    dev_free(g, hubs_d);
    GIR_TRY(rc);
    g->reach_hub_valid = true;
    return GIR_OK;
}

int reach_run(gir_dev* g, const int32_t* u_d, const int32_t* v_d, int64_t n, uint8_t* out_d) {
    const int64_t V = g->V;
    if (n <= 0) return GIR_OK;
    if (!g->reach_hub_valid) GIR_TRY(build_hub_index(g));
    const uint64_t* hubF = static_cast<const uint64_t*>(g->reach_hub.p);
    const uint64_t* hubR = hubF + V;
    const int32_t* scc = static_cast<const int32_t*>(g->scc.p);
    const int32_t* rank = static_cast<const int32_t*>(g->scc_rank.p);
    const uint64_t* keys = static_cast<const uint64_t*>(g->dag.p);
    const int64_t n_dag = g->n_dag > 0 ? g->n_dag : 0;
    int64_t* beg = nullptr;
    GIR_TRY(ensure_n(g, g->dag_rows, V + 2, &beg));
    if (!g->dag_rows_valid) {
        k_dag_rows<<<grid_for(g, V + 1, kBlock), kBlock, 0, g->stream>>>(keys, n_dag, V, beg);
        GIR_LAUNCH(g, "k_dag_rows");
        g->dag_rows_valid = true;
    }
    int32_t *pend = nullptr, *qa = nullptr, *qb = nullptr;
    uint64_t *seen = nullptr, *front = nullptr, *next = nullptr;
    int64_t* pref = nullptr;
    unsigned long long* cnt = nullptr;
    Lanes* L = nullptr;
    GIR_TRY(ensure_n(g, g->scratch[0], (size_t)n + 1, &pend));
    GIR_TRY(ensure_n(g, g->scratch[1], V + 1, &qa));
    GIR_TRY(ensure_n(g, g->scratch[2], V + 1, &qb));
    GIR_TRY(ensure_n(g, g->scratch[3], V, &seen));
    GIR_TRY(ensure_n(g, g->scratch[4], V, &front));
    GIR_TRY(ensure_n(g, g->scratch[5], V, &next));
    GIR_TRY(ensure_n(g, g->scratch[6], V + 2, &pref));
    GIR_TRY(ensure_n(g, g->scratch[7], R_N, &cnt));
    GIR_TRY(ensure_n(g, g->scratch[8], 1, &L));
    void* hp = nullptr;
    GIR_TRY(pinned(g, 256, &hp));
    unsigned long long* hc = static_cast<unsigned long long*>(hp);
    auto read = [&]() -> int {
        GIR_CUDA(g, cudaMemcpyAsync(hc, cnt, sizeof(unsigned long long) * R_N, cudaMemcpyDeviceToHost, g->stream));
        GIR_CUDA(g, cudaStreamSynchronize(g->stream));
        return GIR_OK;
    };
    GIR_CUDA(g, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * R_N, g->stream));
    k_reach_classify<<<grid_for(g, n, kBlock), kBlock, 0, g->stream>>>(u_d, v_d, n, V, scc, rank, hubF, hubR, out_d,
                                                                       pend, cnt);
    GIR_LAUNCH(g, "k_reach_classify");
    GIR_TRY(read());
    const int64_t n_pend = (int64_t)hc[R_Q];
    if (n_pend > 0) {
        GIR_CUDA(g, cudaMemsetAsync(seen, 0, sizeof(uint64_t) * V, g->stream));
        GIR_CUDA(g, cudaMemsetAsync(front, 0, sizeof(uint64_t) * V, g->stream));
        GIR_CUDA(g, cudaMemsetAsync(next, 0, sizeof(uint64_t) * V, g->stream));
    }
    const int grid = g->num_sms * (int)g->params[GIR_PARAM_CTAS_PER_SM];
    for (int64_t g0 = 0; g0 < n_pend; g0 += 64) {
        const int nl = (int)std::min<int64_t>(64, n_pend - g0);
        const unsigned long long all = nl == 64 ? ~0ull : ((1ull << nl) - 1);
        GIR_CUDA(g, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * R_N, g->stream));
        k_reach_lanes<<<1, 64, 0, g->stream>>>(pend, g0, nl, u_d, v_d, scc, rank, L, seen, front, qa, cnt);
        GIR_LAUNCH(g, "k_reach_lanes");
        GIR_TRY(read());
        int64_t nq = (int64_t)hc[R_Q];
        while (nq > 0 && hc[R_FOUND] != all) {
            GIR_CUDA(g, cudaMemsetAsync(&cnt[R_CAND], 0, sizeof(unsigned long long), g->stream));
            k_reach_degrees<<<grid_for(g, nq, kBlock), kBlock, 0, g->stream>>>(qa, nq, beg, pref);
            GIR_LAUNCH(g, "k_reach_degrees");
            GIR_TRY(exclusive_scan_i64(g, pref, pref, nq + 1));
            k_reach_expand<<<grid, kBlock, 0, g->stream>>>(qa, nq, pref, beg, keys, rank, L, nl, front, seen, next, qb,
                                                           cnt);
            GIR_LAUNCH(g, "k_reach_expand");
            k_reach_clear<<<grid_for(g, nq, kBlock), kBlock, 0, g->stream>>>(qa, nq, front);
            GIR_LAUNCH(g, "k_reach_clear");
            GIR_CUDA(g, cudaMemsetAsync(&cnt[R_Q], 0, sizeof(unsigned long long), g->stream));
            k_reach_commit<<<grid, kBlock, 0, g->stream>>>(&cnt[R_CAND], qb, seen, front, next, qa, cnt);
            GIR_LAUNCH(g, "k_reach_commit");
            k_reach_found<<<1, 64, 0, g->stream>>>(L, nl, seen, cnt);
            GIR_LAUNCH(g, "k_reach_found");
            GIR_TRY(read());
            nq = (int64_t)hc[R_Q];
        }
        k_reach_write<<<1, 64, 0, g->stream>>>(pend, g0, nl, cnt, out_d);
        GIR_LAUNCH(g, "k_reach_write");
        // reset the masks for the next group (the frontier left behind on an early stop included)
        if (g0 + 64 < n_pend) {
            GIR_CUDA(g, cudaMemsetAsync(seen, 0, sizeof(uint64_t) * V, g->stream));
            GIR_CUDA(g, cudaMemsetAsync(front, 0, sizeof(uint64_t) * V, g->stream));
        }
    }
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    return GIR_OK;
}

}  // namespace gir
