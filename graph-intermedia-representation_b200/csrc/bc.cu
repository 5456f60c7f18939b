// Betweenness centrality over a set of sources (GIR::bc, gir_query.cpp:728-778): Brandes on the
// directed graph, unweighted, score(v) = sum over the sources s != v of delta_s(v). Sources
// repeat as often as they are given; ids out of range contribute nothing.
//
// Up to 64 sources run as the lanes of one traversal: the lane-parallel BFS (bfs_run) gives every
// lane's levels, which are laid out vertex-major (level[v * 64 + s]) so one warp holds all 64 lanes
// of a vertex in one 256-byte row. Then, level by level:
//  - sigma (shortest-path counts, double) is pulled over in-rows: sigma_s(w) = sum of sigma_s(x)
//    over in-neighbours x one level above w in lane s;
//  - delta is pulled over out-rows in reverse level order: delta_s(u) = sigma_s(u) * sum of
//    (1 + delta_s(w)) / sigma_s(w) over out-neighbours w one level below u in lane s.
// Pulling instead of pushing needs no floating-point atomics; the sums run in a fixed order, so
// results are deterministic (they may differ from the reference's in the last bits: its
// accumulation order across threads is not fixed either). A warp walks one row, so rows longer
// than kLongRow (hubs) are cut into chunks of kChunk entries summed by one warp each into
// per-chunk partials, which one warp per row then adds in chunk order (still a fixed order).
#include <algorithm>
#include <vector>

#include "common.cuh"

namespace gir {

namespace {

constexpr int kBlock = 256;
constexpr int kW = 64;  // lanes per group (row width of the vertex-major arrays)
constexpr int32_t kLongRow = 1024;  // rows longer than this are cut into chunks
constexpr int64_t kChunk = 512;     // entries per chunk of a long row

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

// level[s * V + v] (lanes < nl) -> lev[v * 64 + s], -1 for unused lanes; the largest level to cnt[0].
__global__ void k_bc_levels(const int32_t* level, int64_t V, int nl, int32_t* lev, unsigned long long* maxl) {
    int32_t mx = 0;
    GRID_STRIDE(i, V * kW) {
        const int64_t v = i / kW;
        const int s = (int)(i % kW);
        const int32_t l = s < nl ? level[(int64_t)s * V + v] : -1;
        lev[i] = l;
        mx = l > mx ? l : mx;
    }
    for (int o = 16; o; o >>= 1) {
        const int32_t t = __shfl_xor_sync(0xffffffffu, mx, o);
        mx = t > mx ? t : mx;
    }
    if (lane_id() == 0 && mx) atomicMax(maxl, (unsigned long long)mx);
}

__global__ void k_bc_init(const int32_t* lev, int64_t n, double* sigma, double* delta) {
    GRID_STRIDE(i, n) {
        sigma[i] = lev[i] == 0 ? 1.0 : 0.0;
        delta[i] = 0.0;
    }
}

// Sum over the entries adj[b .. e) of one row, for this warp's lanes t (s0) and t + 32 (s1) of
// the row's vertex (active where a0 / a1): sigma_s(x) over entries x at level `want` (Sigma), or
// (1 + delta_s(x)) / sigma_s(x) (delta). The warp loads 32 entries at once, then takes them 8 at a
// time with all their level loads in flight together; entries that do not count add 0.0, so the
// sums run in row order exactly as a one-entry-at-a-time loop would.
template <bool Sigma>
__device__ __forceinline__ void bc_pull(const int32_t* __restrict__ adj, int64_t b, int64_t e,
                                        const int32_t* __restrict__ lev, int32_t want, bool a0, bool a1, int t,
                                        const double* __restrict__ sigma, const double* __restrict__ delta,
                                        double& s0, double& s1) {
    constexpr int kU = 8;
    for (int64_t base = b; base < e; base += 32) {
        const int cnt = e - base < 32 ? (int)(e - base) : 32;
        const int32_t mine = t < cnt ? adj[base + t] : 0;
        for (int i0 = 0; i0 < cnt; i0 += kU) {
            int64_t x[kU];
            bool m0[kU], m1[kU];
#pragma unroll
            for (int j = 0; j < kU; ++j) {
                x[j] = (int64_t)__shfl_sync(0xffffffffu, mine, (i0 + j) & 31) * kW + t;
                const bool ok = i0 + j < cnt;
                m0[j] = ok && a0 && lev[x[j]] == want;
                m1[j] = ok && a1 && lev[x[j] + 32] == want;
            }
            double v0[kU], v1[kU];
#pragma unroll
            for (int j = 0; j < kU; ++j) {
                if (Sigma) {
                    v0[j] = m0[j] ? sigma[x[j]] : 0.0;
                    v1[j] = m1[j] ? sigma[x[j] + 32] : 0.0;
                } else {
                    v0[j] = m0[j] ? (1.0 + delta[x[j]]) / sigma[x[j]] : 0.0;
                    v1[j] = m1[j] ? (1.0 + delta[x[j] + 32]) / sigma[x[j] + 32] : 0.0;
                }
            }
#pragma unroll
            for (int j = 0; j < kU; ++j) {
                s0 += v0[j];
                s1 += v1[j];
            }
        }
    }
}

// One warp per vertex w (rows of at most kLongRow entries); lane t of the warp handles BFS
// lanes t and t + 32.
__global__ void k_bc_sigma(int64_t V, CSRView bw, const int32_t* lev, int32_t L, double* sigma) {
    const int t = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t w = warp; w < V; w += nwarps) {
        if (bw.deg[w] > kLongRow) continue;
        const bool a0 = lev[w * kW + t] == L, a1 = lev[w * kW + t + 32] == L;
        if (!__any_sync(0xffffffffu, a0 || a1)) continue;
        double s0 = 0.0, s1 = 0.0;
        bc_pull<true>(bw.adj, bw.beg[w], bw.beg[w] + bw.deg[w], lev, L - 1, a0, a1, t, sigma, nullptr, s0, s1);
        if (a0) sigma[w * kW + t] = s0;
        if (a1) sigma[w * kW + t + 32] = s1;
    }
}

__global__ void k_bc_delta(int64_t V, CSRView fw, const int32_t* lev, int32_t L, const double* sigma, double* delta) {
    const int t = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t u = warp; u < V; u += nwarps) {
        if (fw.deg[u] > kLongRow) continue;
        const bool a0 = lev[u * kW + t] == L, a1 = lev[u * kW + t + 32] == L;
        if (!__any_sync(0xffffffffu, a0 || a1)) continue;
        double c0 = 0.0, c1 = 0.0;
        bc_pull<false>(fw.adj, fw.beg[u], fw.beg[u] + fw.deg[u], lev, L + 1, a0, a1, t, sigma, delta, c0, c1);
        if (a0) delta[u * kW + t] = sigma[u * kW + t] * c0;
        if (a1) delta[u * kW + t + 32] = sigma[u * kW + t + 32] * c1;
    }
}

// Chunks of the long rows: chunk c covers entries [cfirst[c], cfirst[c] + clen[c]) of row crow[c];
// its warp writes the chunk's partial sums for the row's lanes at level L (sigma: sum of
// sigma_s(x) over in-neighbours x at level L - 1; delta: sum of (1 + delta_s(w)) / sigma_s(w)
// over out-neighbours w at level L + 1) into part[c * 64 + lane].
template <bool Sigma>
__global__ void k_bc_chunks(const int32_t* crow, const int64_t* cfirst, const int32_t* clen, int64_t n_chunks,
                            CSRView c, const int32_t* lev, int32_t L, const double* sigma, const double* delta,
                            double* part) {
    const int t = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t ch = warp; ch < n_chunks; ch += nwarps) {
        const int64_t u = crow[ch];
        const bool a0 = lev[u * kW + t] == L, a1 = lev[u * kW + t + 32] == L;
        if (!__any_sync(0xffffffffu, a0 || a1)) continue;
        double s0 = 0.0, s1 = 0.0;
        const int64_t b = c.beg[u] + cfirst[ch];
        bc_pull<Sigma>(c.adj, b, b + clen[ch], lev, Sigma ? L - 1 : L + 1, a0, a1, t, sigma, delta, s0, s1);
        part[ch * kW + t] = s0;
        part[ch * kW + t + 32] = s1;
    }
}

// One warp per long row r (its chunks are hfirst[r] .. hfirst[r + 1]): the chunk partials added
// in chunk order, into sigma (Sigma) or delta = sigma * sum.
template <bool Sigma>
__global__ void k_bc_combine(const int32_t* hrow, const int64_t* hfirst, int64_t n_rows, const int32_t* lev,
                             int32_t L, const double* part, double* sigma, double* delta) {
    const int t = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = warp; r < n_rows; r += nwarps) {
        const int64_t u = hrow[r];
        const bool a0 = lev[u * kW + t] == L, a1 = lev[u * kW + t + 32] == L;
        if (!__any_sync(0xffffffffu, a0 || a1)) continue;
        double s0 = 0.0, s1 = 0.0;
        for (int64_t ch = hfirst[r]; ch < hfirst[r + 1]; ++ch) {
            s0 += part[ch * kW + t];
            s1 += part[ch * kW + t + 32];
        }
        if (Sigma) {
            if (a0) sigma[u * kW + t] = s0;
            if (a1) sigma[u * kW + t + 32] = s1;
        } else {
            if (a0) delta[u * kW + t] = sigma[u * kW + t] * s0;
            if (a1) delta[u * kW + t + 32] = sigma[u * kW + t + 32] * s1;
        }
    }
}

// score[v] += sum over the group's lanes of delta_s(v), the lane's source excluded.
__global__ void k_bc_score(int64_t V, int nl, const int32_t* lev, const double* delta, double* score) {
    GRID_STRIDE(v, V) {
        double acc = 0.0;
        for (int s = 0; s < nl; ++s)
            if (lev[v * kW + s] > 0) acc += delta[v * kW + s];
        score[v] += acc;
    }
}

}  // namespace

namespace {

// The long rows of `c` cut into chunks (device arrays in `mem`, host counts).
struct Chunks {
    int32_t *hrow = nullptr, *crow = nullptr, *clen = nullptr;
    int64_t *hfirst = nullptr, *cfirst = nullptr;
    double* part = nullptr;
    int64_t n_rows = 0, n_chunks = 0;
};

int make_chunks(gir_dev* g, const DevCSR& c, Chunks& ch, std::vector<void*>& owned) {
    const int64_t V = g->V;
    uint8_t* flag = nullptr;
    int32_t* rows = nullptr;
    int64_t* pref = nullptr;
    GIR_TRY(dev_alloc_n(g, &flag, V + 1));
    owned.push_back(flag);
    GIR_TRY(dev_alloc_n(g, &rows, V + 1));
    owned.push_back(rows);
    GIR_TRY(dev_alloc_n(g, &pref, V + 2));
    owned.push_back(pref);
    int64_t n = 0;
    GIR_TRY(heavy_rows(g, c.deg, V, kLongRow, flag, rows, pref, &n));
    ch.n_rows = n;
    ch.hrow = rows;
    if (n == 0) return GIR_OK;
    std::vector<int32_t> hr((size_t)n);
    std::vector<int64_t> hp((size_t)n + 1);
    GIR_CUDA(g, cudaMemcpyAsync(hr.data(), rows, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaMemcpyAsync(hp.data(), pref, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    std::vector<int32_t> crow, clen;
    std::vector<int64_t> cfirst, hfirst{0};
    for (int64_t r = 0; r < n; ++r) {
        const int64_t d = hp[r + 1] - hp[r];
        for (int64_t f = 0; f < d; f += kChunk) {
            crow.push_back(hr[r]);
            cfirst.push_back(f);
            clen.push_back((int32_t)std::min<int64_t>(kChunk, d - f));
        }
        hfirst.push_back((int64_t)crow.size());
    }
    ch.n_chunks = (int64_t)crow.size();
    GIR_TRY(dev_alloc_n(g, &ch.crow, ch.n_chunks));
    owned.push_back(ch.crow);
    GIR_TRY(dev_alloc_n(g, &ch.clen, ch.n_chunks));
    owned.push_back(ch.clen);
    GIR_TRY(dev_alloc_n(g, &ch.cfirst, ch.n_chunks));
    owned.push_back(ch.cfirst);
    GIR_TRY(dev_alloc_n(g, &ch.hfirst, n + 1));
    owned.push_back(ch.hfirst);
    GIR_TRY(dev_alloc_n(g, &ch.part, (size_t)ch.n_chunks * kW));
    owned.push_back(ch.part);
    GIR_CUDA(g, cudaMemcpyAsync(ch.crow, crow.data(), sizeof(int32_t) * ch.n_chunks, cudaMemcpyHostToDevice, g->stream));
    GIR_CUDA(g, cudaMemcpyAsync(ch.clen, clen.data(), sizeof(int32_t) * ch.n_chunks, cudaMemcpyHostToDevice, g->stream));
    GIR_CUDA(g, cudaMemcpyAsync(ch.cfirst, cfirst.data(), sizeof(int64_t) * ch.n_chunks, cudaMemcpyHostToDevice, g->stream));
    GIR_CUDA(g, cudaMemcpyAsync(ch.hfirst, hfirst.data(), sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));  // (the host vectors go out of scope)
    return GIR_OK;
}

}  // namespace

int bc_run(gir_dev* g, const int32_t* srcs_d, int64_t n_src, double* score_d) {
    const int64_t V = g->V;
    GIR_CUDA(g, cudaMemsetAsync(score_d, 0, sizeof(double) * (V > 0 ? V : 1), g->stream));
    if (V == 0 || n_src <= 0) return GIR_OK;
    int32_t *level = nullptr, *lev = nullptr;
    double *sigma = nullptr, *delta = nullptr;
    unsigned long long* cnt = nullptr;
    GIR_TRY(dev_alloc_n(g, &level, (size_t)kW * V));
    GIR_TRY(dev_alloc_n(g, &lev, (size_t)kW * V));
    GIR_TRY(dev_alloc_n(g, &sigma, (size_t)kW * V));
    GIR_TRY(dev_alloc_n(g, &delta, (size_t)kW * V));
    GIR_TRY(dev_alloc_n(g, &cnt, 4));
    void* hp = nullptr;
    GIR_TRY(pinned(g, 256, &hp));
    unsigned long long* hc = static_cast<unsigned long long*>(hp);
    const QueryStats keep = g->qstats;
    const int grid = g->num_sms * 8;
    std::vector<void*> owned;
    Chunks lin, lout;  // long in-rows (sigma), long out-rows (delta)
    int rc = make_chunks(g, g->bw, lin, owned);
    if (!rc) rc = make_chunks(g, g->fw, lout, owned);
    for (int64_t g0 = 0; g0 < n_src && rc == GIR_OK; g0 += kW) {
        const int nl = (int)std::min<int64_t>(kW, n_src - g0);
        std::vector<int64_t> sb((size_t)nl + 1);
        for (int i = 0; i <= nl; ++i) sb[i] = i;
        if ((rc = bfs_run(g, sb.data(), srcs_d + g0, nl, level))) break;
        GIR_CUDA(g, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * 4, g->stream));
        k_bc_levels<<<grid_for(g, V * kW, kBlock), kBlock, 0, g->stream>>>(level, V, nl, lev, cnt);
        GIR_LAUNCH(g, "k_bc_levels");
        k_bc_init<<<grid_for(g, V * kW, kBlock), kBlock, 0, g->stream>>>(lev, V * kW, sigma, delta);
        GIR_LAUNCH(g, "k_bc_init");
        GIR_CUDA(g, cudaMemcpyAsync(hc, cnt, sizeof(unsigned long long), cudaMemcpyDeviceToHost, g->stream));
        GIR_CUDA(g, cudaStreamSynchronize(g->stream));
        const int32_t maxl = (int32_t)hc[0];
        for (int32_t L = 1; L <= maxl; ++L) {
            k_bc_sigma<<<grid, kBlock, 0, g->stream>>>(V, view(g->bw), lev, L, sigma);
            GIR_LAUNCH(g, "k_bc_sigma");
            if (lin.n_chunks) {
                k_bc_chunks<true><<<grid, kBlock, 0, g->stream>>>(lin.crow, lin.cfirst, lin.clen, lin.n_chunks, view(g->bw),
                                                                 lev, L, sigma, delta, lin.part);
                GIR_LAUNCH(g, "k_bc_chunks");
                k_bc_combine<true><<<grid, kBlock, 0, g->stream>>>(lin.hrow, lin.hfirst, lin.n_rows, lev, L, lin.part, sigma,
                                                                  delta);
                GIR_LAUNCH(g, "k_bc_combine");
            }
        }
        for (int32_t L = maxl - 1; L >= 0; --L) {
            k_bc_delta<<<grid, kBlock, 0, g->stream>>>(V, view(g->fw), lev, L, sigma, delta);
            GIR_LAUNCH(g, "k_bc_delta");
            if (lout.n_chunks) {
                k_bc_chunks<false><<<grid, kBlock, 0, g->stream>>>(lout.crow, lout.cfirst, lout.clen, lout.n_chunks,
                                                                  view(g->fw), lev, L, sigma, delta, lout.part);
                GIR_LAUNCH(g, "k_bc_chunks");
                k_bc_combine<false><<<grid, kBlock, 0, g->stream>>>(lout.hrow, lout.hfirst, lout.n_rows, lev, L, lout.part,
                                                                   sigma, delta);
                GIR_LAUNCH(g, "k_bc_combine");
            }
        }
        k_bc_score<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, nl, lev, delta, score_d);
        GIR_LAUNCH(g, "k_bc_score");
    }
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    g->qstats = keep;
    for (void* p : owned) dev_free(g, p);
    dev_free(g, cnt);
    dev_free(g, delta);
    dev_free(g, sigma);
    dev_free(g, lev);
    dev_free(g, level);
    return rc;
}

}  // namespace gir
