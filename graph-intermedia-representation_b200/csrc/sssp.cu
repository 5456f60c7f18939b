// Delta-stepping single-source shortest paths on the device (GIR::sssp / deltaStepping,
// gir_query.cpp:629-703): uint64 distances, UINT64_MAX = unreachable.
//
// Buckets of width Delta are processed in increasing order. Within bucket k the near queue is
// relaxed through its light edges (weight < Delta) round after round until no vertex re-enters
// the bucket; then every vertex settled in the bucket relaxes its heavy edges (weight >= Delta)
// once -- those can only land in later buckets. (The reference relaxes all edges every round and
// has no light/heavy split, gir_query.cpp:674-688; the split changes the work, not the result.)
// Relaxations that land beyond the bucket go to a far queue, which is split by the next
// non-empty bucket (dist / Delta of its smallest live entry).
//
// Rows are read from a weight-sorted copy of the forward CSR, so the light edges of a row are a
// prefix of it and the heavy edges the rest. Shortest distances are unique, so the result is
// the same for every Delta and every schedule.
#include "common.cuh"

namespace gir {

namespace {

constexpr int kBlock = 256;
constexpr int kWarps = kBlock / 32;

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

// counters: [0] near queue length being built, [1] far queue length, [2] settled list length,
// [3] min far distance (atomicMin), [4] far queue length after a split, [8] length of the queue
// being relaxed; accumulated over the queries: [16] reached vertices, [17] their out-edges
enum { S_NEAR = 0, S_FAR = 1, S_SET = 2, S_MIN = 3, S_FAR2 = 4, S_QLEN = 8, S_REACHED = 16, S_EDGES = 17, S_N = 8 };

__global__ void k_ws_keys(int64_t V, int64_t E, const int64_t* cb, CSRView c, int hash, uint64_t* keys,
                          uint32_t* cols) {
    GRID_STRIDE(i, E) {
        int64_t lo = 0, hi = V - 1;
        while (lo < hi) {
            const int64_t m = (lo + hi + 1) >> 1;
            if (cb[m] <= i) lo = m; else hi = m - 1;
        }
        const int64_t u = lo;
        const int64_t p = c.beg[u] + (i - cb[u]);
        const int32_t v = c.adj[p];
        const uint32_t w = hash ? hash_weight((int32_t)u, v) : c.w[p];
        keys[i] = ((uint64_t)u << 32) | w;
        cols[i] = (uint32_t)v;
    }
}

__global__ void k_ws_split(int64_t E, const uint64_t* keys, const uint32_t* cols, int32_t* adj, uint32_t* w) {
    GRID_STRIDE(i, E) {
        adj[i] = (int32_t)cols[i];
        w[i] = (uint32_t)(keys[i] & 0xffffffffULL);
    }
}

__global__ void k_deg_i64(int64_t V, const int32_t* deg, int64_t* out) {
    GRID_STRIDE(v, V) out[v] = deg[v];
    if (blockIdx.x == 0 && threadIdx.x == 0) out[V] = 0;
}

__global__ void k_sssp_init(const int32_t* srcs, int64_t n, int64_t V, uint64_t* dist, int32_t* near_mark,
                            int32_t epoch, int32_t* nearq, unsigned long long* cnt) {
    GRID_STRIDE(i, n) {
        const int32_t s = srcs[i];
        if (s < 0 || s >= V) continue;
        dist[s] = 0;
        if (atomicExch(&near_mark[s], epoch) != epoch) nearq[atomicAdd(&cnt[S_NEAR], 1ull)] = s;
    }
}

struct RelaxArgs {
    const int64_t* wb;      // weight-sorted rows (compact offsets)
    const int32_t* wdeg;
    const int32_t* wadj;
    const uint32_t* ww;
    uint64_t delta, kend;   // bucket width; end of the current bucket
    uint64_t* dist;
    int32_t* near_mark; int32_t near_epoch; int32_t* nearq;
    int32_t* far_mark; int32_t far_epoch; int32_t* farq;
    int32_t* settle_mark; int32_t settle_epoch; int32_t* setq;
    unsigned long long* cnt;
};

// Relaxes the light (heavy = 0) or heavy (heavy = 1) edges of the queue's vertices. A warp takes
// 32 queue entries at a time and walks their edge ranges together: lane l handles positions
// l, l+32, ... of the concatenated ranges (owner found by binary search in shared memory).
__global__ void __launch_bounds__(kBlock) k_relax(const int32_t* q, const unsigned long long* qlen, int heavy,
                                                  RelaxArgs a) {
    __shared__ int64_t s_excl[kWarps][33];
    __shared__ int64_t s_eb[kWarps][32];
    __shared__ uint64_t s_du[kWarps][32];
    __shared__ int32_t s_u[kWarps][32];
    const int lane = lane_id(), wib = threadIdx.x >> 5;
    const int64_t n = (int64_t)*qlen;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = warp * 32; base < n; base += nwarps * 32) {
        const int64_t i = base + lane;
        int64_t eb = 0, ecount = 0;
        uint64_t du = 0;
        int32_t u = -1;
        if (i < n) {
            u = q[i];
            du = a.dist[u];
            const int64_t b = a.wb[u], e = b + a.wdeg[u];
            int64_t lo = b, hi = e;  // light edges: the prefix with weight < delta
            while (lo < hi) {
                const int64_t m = (lo + hi) >> 1;
                if ((uint64_t)a.ww[m] < a.delta) lo = m + 1; else hi = m;
            }
            if (heavy) { eb = lo; ecount = e - lo; }
            else { eb = b; ecount = lo - b; }
            if (!heavy && atomicExch(&a.settle_mark[u], a.settle_epoch) != a.settle_epoch)
                a.setq[atomicAdd(&a.cnt[S_SET], 1ull)] = u;
        }
        int64_t incl = ecount;
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        s_excl[wib][lane] = incl - ecount;
        if (lane == 31) s_excl[wib][32] = incl;
        s_eb[wib][lane] = eb;
        s_du[wib][lane] = du;
        s_u[wib][lane] = u;
        __syncwarp();
        const int64_t total = s_excl[wib][32];
        for (int64_t p0 = 0; p0 < total; p0 += 32) {
            const int64_t p = p0 + lane;
            bool to_near = false, to_far = false;
            int32_t w = 0;
            if (p < total) {
                int lo = 0, hi = 31;  // largest l with excl[l] <= p
                while (lo < hi) {
                    const int m = (lo + hi + 1) >> 1;
                    if (s_excl[wib][m] <= p) lo = m; else hi = m - 1;
                }
                const int64_t k = s_eb[wib][lo] + (p - s_excl[wib][lo]);
                w = a.wadj[k];
                const uint64_t nd = s_du[wib][lo] + (uint64_t)a.ww[k];
                const unsigned long long old = atomicMin((unsigned long long*)&a.dist[w], (unsigned long long)nd);
                if (nd < old) {
                    if (nd < a.kend) to_near = atomicExch(&a.near_mark[w], a.near_epoch) != a.near_epoch;
                    else to_far = atomicExch(&a.far_mark[w], a.far_epoch) != a.far_epoch;
                }
            }
            warp_append(to_near, w, a.nearq, &a.cnt[S_NEAR]);
            warp_append(to_far, w, a.farq, &a.cnt[S_FAR]);
        }
        __syncwarp();
    }
}

// Smallest distance among live far entries (dist >= kend; smaller ones are settled already).
__global__ void k_far_min(const int32_t* farq, const unsigned long long* nfar, const uint64_t* dist, uint64_t kend,
                          unsigned long long* cnt) {
    unsigned long long m = ~0ull;
    const int64_t n = (int64_t)*nfar;
    GRID_STRIDE(i, n) {
        const uint64_t d = dist[farq[i]];
        if (d >= kend && d < m) m = d;
    }
    for (int o = 16; o; o >>= 1) {
        const unsigned long long t = __shfl_xor_sync(0xffffffffu, m, o);
        m = t < m ? t : m;
    }
    if (lane_id() == 0 && m != ~0ull) atomicMin(&cnt[S_MIN], m);
}

// Splits the far queue at the new bucket [lo, hi): entries in it go to the near queue, later
// ones to farq2, settled (stale) ones are dropped; duplicates are dropped by the marks.
__global__ void k_far_split(const int32_t* farq, const unsigned long long* nfar, const uint64_t* dist, uint64_t lo,
                            uint64_t hi, int32_t* near_mark, int32_t near_epoch, int32_t* nearq, int32_t* far_mark,
                            int32_t far_epoch, int32_t* farq2, unsigned long long* cnt) {
    const int64_t n = (int64_t)*nfar;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < n; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = base + threadIdx.x;
        bool to_near = false, to_far = false;
        int32_t v = 0;
        if (i < n) {
            v = farq[i];
            const uint64_t d = dist[v];
            if (d >= lo && d < hi) to_near = atomicExch(&near_mark[v], near_epoch) != near_epoch;
            else if (d >= hi) to_far = atomicExch(&far_mark[v], far_epoch) != far_epoch;
        }
        warp_append(to_near, v, nearq, &cnt[S_NEAR]);
        warp_append(to_far, v, farq2, &cnt[S_FAR2]);
    }
}

// Reached vertices and their out-degrees (the traversed edges of the GTEPS figure).
__global__ void k_sssp_reached(const uint64_t* dist, int64_t V, const int32_t* outdeg, unsigned long long* cnt) {
    unsigned long long r = 0, e = 0;
    GRID_STRIDE(v, V) {
        if (dist[v] != ~0ull) { ++r; e += (unsigned long long)outdeg[v]; }
    }
    for (int o = 16; o; o >>= 1) {
        r += __shfl_xor_sync(0xffffffffu, r, o);
        e += __shfl_xor_sync(0xffffffffu, e, o);
    }
    if (lane_id() == 0) {
        if (r) atomicAdd(&cnt[S_REACHED], r);
        if (e) atomicAdd(&cnt[S_EDGES], e);
    }
}

}  // namespace

// Weight-sorted copy of the forward CSR for one weight mode (compact rows).
static int build_weight_sorted(gir_dev* g, int hash, DevCSR& ws) {
    const int64_t V = g->V, E = g->fw.E;
    store_free(ws);
    int64_t* cb = nullptr;
    uint64_t *keys = nullptr, *ktmp = nullptr;
    uint32_t *cols = nullptr, *ctmp = nullptr;
    GIR_CUDA(g, cudaMalloc(&ws.beg, sizeof(int64_t) * (V + 1)));
    GIR_CUDA(g, cudaMalloc(&ws.deg, sizeof(int32_t) * (V > 0 ? V : 1)));
    GIR_CUDA(g, cudaMalloc(&ws.adj, sizeof(int32_t) * (E > 0 ? E : 1)));
    GIR_CUDA(g, cudaMalloc(&ws.w, sizeof(uint32_t) * (E > 0 ? E : 1)));
    ws.cap = ws.E = E;
    cb = ws.beg;
    k_deg_i64<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, g->fw.deg, cb);
    GIR_LAUNCH(g, "k_deg_i64");
    GIR_TRY(exclusive_scan_i64(g, cb, cb, V + 1));
    GIR_CUDA(g, cudaMemcpyAsync(ws.deg, g->fw.deg, sizeof(int32_t) * V, cudaMemcpyDeviceToDevice, g->stream));
    if (E == 0) return GIR_OK;
    GIR_TRY(ensure_n(g, g->scratch[8], E, &keys));
    GIR_TRY(ensure_n(g, g->scratch[9], E, &ktmp));
    GIR_TRY(ensure_n(g, g->scratch[10], E, &cols));
    GIR_TRY(ensure_n(g, g->scratch[11], E, &ctmp));
    k_ws_keys<<<grid_for(g, E, kBlock), kBlock, 0, g->stream>>>(V, E, cb, view(g->fw), hash, keys, cols);
    GIR_LAUNCH(g, "k_ws_keys");
    GIR_TRY(sort_pairs_u64(g, keys, ktmp, cols, ctmp, E, 64));
    k_ws_split<<<grid_for(g, E, kBlock), kBlock, 0, g->stream>>>(E, keys, cols, ws.adj, ws.w);
    GIR_LAUNCH(g, "k_ws_split");
    return GIR_OK;
}

int sssp_run(gir_dev* g, const int64_t* set_beg_h, const int32_t* srcs_d, int64_t n_sets, uint64_t delta,
             int weight_mode, uint64_t* dist_d) {
    const int64_t V = g->V;
    QueryStats& st = g->qstats;
    st = QueryStats{};
    if (n_sets <= 0) return GIR_OK;
    GIR_CUDA(g, cudaMemsetAsync(dist_d, 0xff, sizeof(uint64_t) * V * n_sets, g->stream));
    if (V == 0) return GIR_OK;
    const int hash = weight_mode == GIR_WEIGHT_HASH;
    if (!hash && !g->has_weights) return fail(g, GIR_ERR_STATE, "sssp: the graph has no stored weights");
    DevCSR& ws = g->ws[hash ? 0 : 1];
    if (!g->ws_valid[hash ? 0 : 1]) {
        GIR_TRY(build_weight_sorted(g, hash, ws));
        g->ws_valid[hash ? 0 : 1] = true;
    }
    int32_t *nearq = nullptr, *nearq2 = nullptr, *farq = nullptr, *farq2 = nullptr, *setq = nullptr;
    int32_t *near_mark = nullptr, *far_mark = nullptr, *settle_mark = nullptr;
    unsigned long long* cnt = nullptr;
    GIR_TRY(ensure_n(g, g->scratch[0], V + 1, &nearq));
    GIR_TRY(ensure_n(g, g->scratch[1], V + 1, &nearq2));
    GIR_TRY(ensure_n(g, g->scratch[2], 2 * V + 2, &farq));
    GIR_TRY(ensure_n(g, g->scratch[3], 2 * V + 2, &farq2));
    GIR_TRY(ensure_n(g, g->scratch[4], V + 1, &setq));
    GIR_TRY(ensure_n(g, g->scratch[5], V + 1, &near_mark));
    GIR_TRY(ensure_n(g, g->scratch[6], V + 1, &far_mark));
    GIR_TRY(ensure_n(g, g->scratch[7], V + 1, &settle_mark));
    GIR_TRY(ensure_n(g, g->scratch[12], 32, &cnt));
    unsigned long long* hc = nullptr;
    {
        void* h = nullptr;
        GIR_TRY(pinned(g, 256, &h));
        hc = static_cast<unsigned long long*>(h);
    }
    const int grid = g->num_sms * (int)g->params[GIR_PARAM_CTAS_PER_SM];
    GIR_CUDA(g, cudaEventRecord(g->ev0, g->stream));
    GIR_CUDA(g, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * 32, g->stream));
    for (int64_t s = 0; s < n_sets; ++s) {
        uint64_t* dist = dist_d + s * V;
        uint64_t D = delta;
        if (D == 0) {
            if (g->schedule == GIR_SCHEDULE_LEARNED && g->sched_loaded) {
                const double E = (double)g->fw.E;
                float feat[GIR_SCHED_IN] = {(float)(E / V / 64.0), hash ? 0.5f : 1.f, (float)(g->num_sms / 148.0),
                                            0.f, 0.f, 0.f, 0.f, 1.f};
                GIR_TRY(sched_choose_delta(g, feat, &D));
            } else {
                D = (uint64_t)g->params[GIR_PARAM_DELTA];
            }
            if (D == 0) D = 16;
        }
        GIR_CUDA(g, cudaMemsetAsync(near_mark, 0, sizeof(int32_t) * V, g->stream));
        GIR_CUDA(g, cudaMemsetAsync(far_mark, 0, sizeof(int32_t) * V, g->stream));
        GIR_CUDA(g, cudaMemsetAsync(settle_mark, 0, sizeof(int32_t) * V, g->stream));
        GIR_CUDA(g, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * S_N, g->stream));
        int32_t near_epoch = 1, far_epoch = 1, settle_epoch = 1;
        const int64_t n_src = set_beg_h[s + 1] - set_beg_h[s];
        if (n_src > 0) {
            k_sssp_init<<<grid_for(g, n_src, kBlock), kBlock, 0, g->stream>>>(srcs_d + set_beg_h[s], n_src, V, dist,
                                                                             near_mark, near_epoch, nearq, cnt);
            GIR_LAUNCH(g, "k_sssp_init");
        }
        unsigned long long* qlen = cnt + S_QLEN;
        GIR_CUDA(g, cudaMemcpyAsync(hc, cnt, sizeof(unsigned long long) * S_N, cudaMemcpyDeviceToHost, g->stream));
        GIR_CUDA(g, cudaStreamSynchronize(g->stream));
        uint64_t k = 0;
        int64_t n_near = (int64_t)hc[S_NEAR], n_far = 0;
        RelaxArgs a;
        a.wb = ws.beg; a.wdeg = ws.deg; a.wadj = ws.adj; a.ww = ws.w; a.delta = D; a.dist = dist;
        a.near_mark = near_mark; a.far_mark = far_mark; a.settle_mark = settle_mark; a.setq = setq; a.cnt = cnt;
        while (true) {
            // ---- bucket k ----
            a.kend = (k + 1) * D;
            a.settle_epoch = ++settle_epoch;
            GIR_CUDA(g, cudaMemsetAsync(cnt + S_SET, 0, sizeof(unsigned long long), g->stream));
            while (n_near > 0) {
                // near queue (length cnt[S_NEAR]) -> move its length to qlen, reset the counter
                GIR_CUDA(g, cudaMemcpyAsync(qlen, cnt + S_NEAR, sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
                                            g->stream));
                GIR_CUDA(g, cudaMemsetAsync(cnt + S_NEAR, 0, sizeof(unsigned long long), g->stream));
                a.near_epoch = ++near_epoch;
                a.nearq = nearq2;
                a.far_epoch = far_epoch;
                a.farq = farq;
                const int64_t blocks = (n_near + 31) / 32 / kWarps + 1;
                k_relax<<<(int)(blocks < grid ? blocks : grid), kBlock, 0, g->stream>>>(nearq, qlen, 0, a);
                GIR_LAUNCH(g, "k_relax(light)");
                st.launches++;
                st.iterations++;
                std::swap(nearq, nearq2);
                GIR_CUDA(g, cudaMemcpyAsync(hc, cnt, sizeof(unsigned long long) * S_N, cudaMemcpyDeviceToHost, g->stream));
                GIR_CUDA(g, cudaStreamSynchronize(g->stream));
                n_near = (int64_t)hc[S_NEAR];
            }
            // heavy edges of everything settled in this bucket
            const int64_t n_set = (int64_t)hc[S_SET];
            if (n_set > 0) {
                GIR_CUDA(g, cudaMemcpyAsync(qlen, cnt + S_SET, sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
                                            g->stream));
                a.near_epoch = ++near_epoch;
                a.nearq = nearq2;  // (heavy relaxations never land in this bucket)
                a.farq = farq;
                const int64_t blocks = (n_set + 31) / 32 / kWarps + 1;
                k_relax<<<(int)(blocks < grid ? blocks : grid), kBlock, 0, g->stream>>>(setq, qlen, 1, a);
                GIR_LAUNCH(g, "k_relax(heavy)");
                st.launches++;
            }
            // next non-empty bucket from the far queue
            GIR_CUDA(g, cudaMemsetAsync(cnt + S_MIN, 0xff, sizeof(unsigned long long), g->stream));
            GIR_CUDA(g, cudaMemcpyAsync(hc, cnt, sizeof(unsigned long long) * S_N, cudaMemcpyDeviceToHost, g->stream));
            GIR_CUDA(g, cudaStreamSynchronize(g->stream));
            n_far = (int64_t)hc[S_FAR];
            if (n_far == 0) break;
            k_far_min<<<grid_for(g, n_far, kBlock), kBlock, 0, g->stream>>>(farq, cnt + S_FAR, dist, a.kend, cnt);
            GIR_LAUNCH(g, "k_far_min");
            GIR_CUDA(g, cudaMemcpyAsync(hc, cnt, sizeof(unsigned long long) * S_N, cudaMemcpyDeviceToHost, g->stream));
            GIR_CUDA(g, cudaStreamSynchronize(g->stream));
            const uint64_t mind = hc[S_MIN];
            if (mind == ~0ull) break;  // only settled entries left
            k = mind / D;
            GIR_CUDA(g, cudaMemsetAsync(cnt + S_FAR2, 0, sizeof(unsigned long long), g->stream));
            a.near_epoch = ++near_epoch;
            ++far_epoch;
            k_far_split<<<grid_for(g, n_far, kBlock), kBlock, 0, g->stream>>>(farq, cnt + S_FAR, dist, k * D, (k + 1) * D,
                                                                              near_mark, near_epoch, nearq, far_mark,
                                                                              far_epoch, farq2, cnt);
            GIR_LAUNCH(g, "k_far_split");
            st.launches += 3;
            std::swap(farq, farq2);
            GIR_CUDA(g, cudaMemcpyAsync(cnt + S_FAR, cnt + S_FAR2, sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
                                        g->stream));
            GIR_CUDA(g, cudaMemcpyAsync(hc, cnt, sizeof(unsigned long long) * S_N, cudaMemcpyDeviceToHost, g->stream));
            GIR_CUDA(g, cudaStreamSynchronize(g->stream));
            n_near = (int64_t)hc[S_NEAR];
        }
        k_sssp_reached<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(dist, V, g->fw.deg, cnt);
        GIR_LAUNCH(g, "k_sssp_reached");
    }
    GIR_CUDA(g, cudaMemcpyAsync(hc, cnt, sizeof(unsigned long long) * 32, cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaEventRecord(g->ev1, g->stream));
    GIR_CUDA(g, cudaEventSynchronize(g->ev1));
    st.reached = (int64_t)hc[S_REACHED];
    st.edges = (int64_t)hc[S_EDGES];
    float ms = 0;
    GIR_CUDA(g, cudaEventElapsedTime(&ms, g->ev0, g->ev1));
    st.kernel_ms = ms;
    return GIR_OK;
}

}  // namespace gir
