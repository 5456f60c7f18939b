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
// accumulation order across threads is not fixed either).
#include <algorithm>
#include <vector>

#include "common.cuh"

namespace gir {

namespace {

constexpr int kBlock = 256;
constexpr int kW = 64;  // lanes per group (row width of the vertex-major arrays)

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

// One warp per vertex w; lane t of the warp handles BFS lanes t and t + 32.
__global__ void k_bc_sigma(int64_t V, CSRView bw, const int32_t* lev, int32_t L, double* sigma) {
    const int t = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t w = warp; w < V; w += nwarps) {
        const bool a0 = lev[w * kW + t] == L, a1 = lev[w * kW + t + 32] == L;
        if (!__any_sync(0xffffffffu, a0 || a1)) continue;
        double s0 = 0.0, s1 = 0.0;
        const int64_t b = bw.beg[w], e = b + bw.deg[w];
        for (int64_t k = b; k < e; ++k) {
            const int64_t x = bw.adj[k];
            if (a0 && lev[x * kW + t] == L - 1) s0 += sigma[x * kW + t];
            if (a1 && lev[x * kW + t + 32] == L - 1) s1 += sigma[x * kW + t + 32];
        }
        if (a0) sigma[w * kW + t] = s0;
        if (a1) sigma[w * kW + t + 32] = s1;
    }
}

__global__ void k_bc_delta(int64_t V, CSRView fw, const int32_t* lev, int32_t L, const double* sigma, double* delta) {
    const int t = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t u = warp; u < V; u += nwarps) {
        const bool a0 = lev[u * kW + t] == L, a1 = lev[u * kW + t + 32] == L;
        if (!__any_sync(0xffffffffu, a0 || a1)) continue;
        double c0 = 0.0, c1 = 0.0;
        const int64_t b = fw.beg[u], e = b + fw.deg[u];
        for (int64_t k = b; k < e; ++k) {
            const int64_t w = fw.adj[k];
            if (a0 && lev[w * kW + t] == L + 1) c0 += (1.0 + delta[w * kW + t]) / sigma[w * kW + t];
            if (a1 && lev[w * kW + t + 32] == L + 1) c1 += (1.0 + delta[w * kW + t + 32]) / sigma[w * kW + t + 32];
        }
        if (a0) delta[u * kW + t] = sigma[u * kW + t] * c0;
        if (a1) delta[u * kW + t + 32] = sigma[u * kW + t + 32] * c1;
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
    int rc = GIR_OK;
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
        }
        for (int32_t L = maxl - 1; L >= 0; --L) {
            k_bc_delta<<<grid, kBlock, 0, g->stream>>>(V, view(g->fw), lev, L, sigma, delta);
            GIR_LAUNCH(g, "k_bc_delta");
        }
        k_bc_score<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, nl, lev, delta, score_d);
        GIR_LAUNCH(g, "k_bc_score");
    }
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    g->qstats = keep;
    dev_free(g, cnt);
    dev_free(g, delta);
    dev_free(g, sigma);
    dev_free(g, lev);
    dev_free(g, level);
    return rc;
}

}  // namespace gir
