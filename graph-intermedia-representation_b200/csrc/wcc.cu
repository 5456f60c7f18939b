// Weakly connected components (buildWCC, gir_constructor/gir.cpp:593-655).
//
// The reference runs a sequential union-find over the forward edges (gir.cpp:635-653). Here
// edges are linked concurrently into a lock-free union-find forest: link(u, w) finds both roots
// (with path halving) and hooks the larger root under the smaller one by compare-and-swap,
// retrying when another thread moved the root first. A root is therefore always the smallest
// vertex of its tree, and after a final pointer-jumping pass every vertex points at the smallest
// vertex id of its component -- the canonical label. The build samples the giant component first
// and links only the rows outside it (wcc_labels_sym, over the symmetric view).
#include <algorithm>

#include "common.cuh"

namespace gir {

namespace {

constexpr int kBlock = 256;

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

__device__ __forceinline__ int32_t uf_find(int32_t* parent, int32_t x) {
    int32_t p = parent[x];
    while (p != x) {
        const int32_t gp = parent[p];
        if (gp != p) parent[x] = gp;  // path halving (benign race: always an ancestor)
        x = p;
        p = parent[x];
    }
    return x;
}

// Lock-free: a failed CAS means another link moved rb first, so the retries are bounded by
// the concurrent links; the cap only turns a broken invariant into an error status.
__device__ __forceinline__ void uf_link(int32_t* parent, int32_t a, int32_t b, int32_t* err) {
    for (int iter = 0; iter < (1 << 22); ++iter) {
        int32_t ra = uf_find(parent, a), rb = uf_find(parent, b);
        if (ra == rb) return;
        if (ra > rb) { const int32_t t = ra; ra = rb; rb = t; }
        if (atomicCAS(&parent[rb], rb, ra) == rb) return;
    }
    atomicExch(err, 1);
}

__global__ void k_uf_init(int32_t* parent, int64_t V) { GRID_STRIDE(v, V) parent[v] = (int32_t)v; }

// Links the endpoints of every pair key (u << 32 | v) into the existing forest.
__global__ void k_uf_link_keys(const uint64_t* keys, int64_t n, int32_t* parent, int32_t* err) {
    GRID_STRIDE(i, n) uf_link(parent, (int32_t)(keys[i] >> 32), (int32_t)(keys[i] & 0xffffffffULL), err);
}

// Final pointer jumping. The walk only reads: with path halving, another thread could replace
// a root just stored in parent[v] by an intermediate ancestor; here every write is a final root.
__global__ void k_uf_compress(int32_t* parent, int64_t V, unsigned long long* roots) {
    unsigned long long r = 0;
    GRID_STRIDE(v, V) {
        int32_t x = (int32_t)v;
        while (parent[x] != x) x = parent[x];
        parent[v] = x;
        r += (x == (int32_t)v);
    }
    for (int o = 16; o; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    if ((threadIdx.x & 31) == 0 && r) atomicAdd(roots, r);
}

// Afforest-style sampling over the symmetric view (every pair in both rows): first every vertex
// links to its r-th neighbour, for r < kNeighbourRounds; then the forest is flattened, the most
// frequent root among sampled vertices is taken as the giant component's, and only vertices
// outside it link their remaining neighbours. An edge between a giant vertex and any other is in
// the other vertex's row too, so skipping the giant's rows loses no link. Links still hook the
// larger root under the smaller, so every root stays its component's smallest vertex.
constexpr int kNeighbourRounds = 2;
constexpr int kSamples = 1024;

__global__ void k_uf_link_nth(CSRView c, int64_t V, int r, int32_t* parent, int32_t* err) {
    GRID_STRIDE(v, V) {
        if (c.deg[v] > r) uf_link(parent, (int32_t)v, c.adj[c.beg[v] + r], err);
    }
}

// One pointer-jumping pass: every vertex to its root (reads only, then one write).
__global__ void k_uf_flatten(int32_t* parent, int64_t V) {
    GRID_STRIDE(v, V) {
        int32_t x = parent[v];
        while (parent[x] != x) x = parent[x];
        parent[v] = x;
    }
}

__global__ void k_uf_sample(const int32_t* parent, int64_t V, int32_t* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kSamples) return;
    uint64_t z = (uint64_t)(i + 1) * 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 31)) * 0xbf58476d1ce4e5b9ULL;
    out[i] = parent[(int64_t)((z >> 17) % (uint64_t)V)];
}

// Rows of the vertices outside the sampled giant root, from column `from` on, one warp per 32
// vertices as in warp_sweep_rows.
__global__ void __launch_bounds__(kBlock) k_uf_link_rest(CSRView c, int64_t V, int from, int32_t giant,
                                                         int32_t* parent, int32_t* err) {
    __shared__ int64_t s_excl[kBlock / 32][33];
    __shared__ int32_t s_u[kBlock / 32][32];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = warp * 32; base < V; base += nwarps * 32) {
        const int64_t v = base + lane;
        int64_t cnt = 0;
        if (v < V && parent[v] != giant) cnt = c.deg[v] > from ? c.deg[v] - from : 0;
        int64_t incl = cnt;
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        s_excl[wib][lane] = incl - cnt;
        if (lane == 31) s_excl[wib][32] = incl;
        s_u[wib][lane] = (int32_t)v;
        __syncwarp();
        const int64_t total = s_excl[wib][32];
        for (int64_t p0 = 0; p0 < total; p0 += 32) {
            const int64_t p = p0 + lane;
            if (p < total) {
                int lo = 0, hi = 31;
                while (lo < hi) {
                    const int m = (lo + hi + 1) >> 1;
                    if (s_excl[wib][m] <= p) lo = m; else hi = m - 1;
                }
                const int32_t u = s_u[wib][lo];
                uf_link(parent, u, c.adj[c.beg[u] + from + (p - s_excl[wib][lo])], err);
            }
        }
        __syncwarp();
    }
}

}  // namespace

// Components of the symmetric view by the sampled union-find above; labels = smallest vertex id.
static int wcc_labels_sym(gir_dev* g, int32_t* label, int64_t* n_comp) {
    const int64_t V = g->V;
    unsigned long long* roots = nullptr;
    GIR_TRY(ensure_n(g, g->scratch[14], 4 + kSamples / 2, &roots));
    int32_t* err = reinterpret_cast<int32_t*>(roots + 1);
    int32_t* sample = reinterpret_cast<int32_t*>(roots + 2);
    GIR_CUDA(g, cudaMemsetAsync(roots, 0, 2 * sizeof(unsigned long long), g->stream));
    if (V == 0) { *n_comp = 0; return GIR_OK; }
    const CSRView s = view(g->sym);
    k_uf_init<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(label, V);
    GIR_LAUNCH(g, "k_uf_init");
    for (int r = 0; r < kNeighbourRounds; ++r) {
        k_uf_link_nth<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(s, V, r, label, err);
        GIR_LAUNCH(g, "k_uf_link_nth");
    }
    k_uf_flatten<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(label, V);
    GIR_LAUNCH(g, "k_uf_flatten");
    k_uf_sample<<<(kSamples + kBlock - 1) / kBlock, kBlock, 0, g->stream>>>(label, V, sample);
    GIR_LAUNCH(g, "k_uf_sample");
    std::vector<int32_t> hs(kSamples);
    GIR_CUDA(g, cudaMemcpyAsync(hs.data(), sample, sizeof(int32_t) * kSamples, cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    std::sort(hs.begin(), hs.end());
    int32_t giant = hs[0];
    for (int i = 0, best = 0; i < kSamples;) {
        int j = i;
        while (j < kSamples && hs[j] == hs[i]) ++j;
        if (j - i > best) { best = j - i; giant = hs[i]; }
        i = j;
    }
    trace_mark(g, "wcc: neighbour rounds + sample");
    k_uf_link_rest<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(s, V, kNeighbourRounds, giant, label, err);
    GIR_LAUNCH(g, "k_uf_link_rest");
    k_uf_compress<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(label, V, roots);
    GIR_LAUNCH(g, "k_uf_compress");
    unsigned long long h[2] = {0, 0};
    GIR_CUDA(g, cudaMemcpyAsync(h, roots, sizeof(h), cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    if (h[1]) return fail(g, GIR_ERR_TIMEOUT, "wcc: union-find link exceeded its retry bound");
    *n_comp = (int64_t)h[0];
    trace_mark(g, "wcc: rest + compress");
    return GIR_OK;
}


// Inserted undirected pairs only (no pair disappeared): the current labels (smallest member,
// so every label is its own root) are a union-find forest already; linking the new pairs into
// it and flattening gives the labels a rebuild would give.
int wcc_union_pairs(gir_dev* g, const uint64_t* keys, int64_t n) {
    const int64_t V = g->V;
    int32_t* label = static_cast<int32_t*>(g->wcc.p);
    unsigned long long* roots = nullptr;
    GIR_TRY(ensure_n(g, g->scratch[14], 4, &roots));
    int32_t* err = reinterpret_cast<int32_t*>(roots + 1);
    GIR_CUDA(g, cudaMemsetAsync(roots, 0, 2 * sizeof(unsigned long long), g->stream));
    if (V == 0 || n == 0) return GIR_OK;
    k_uf_link_keys<<<grid_for(g, n, kBlock), kBlock, 0, g->stream>>>(keys, n, label, err);
    GIR_LAUNCH(g, "k_uf_link_keys");
    k_uf_compress<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(label, V, roots);
    GIR_LAUNCH(g, "k_uf_compress");
    unsigned long long h[2] = {0, 0};
    GIR_CUDA(g, cudaMemcpyAsync(h, roots, sizeof(h), cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    if (h[1]) return fail(g, GIR_ERR_TIMEOUT, "wcc: union-find link exceeded its retry bound");
    g->n_wcc = (int64_t)h[0];
    return GIR_OK;
}

int wcc_build(gir_dev* g) {
    int32_t* label = nullptr;
    GIR_TRY(ensure_n(g, g->wcc, g->V + 1, &label));
    GIR_TRY(wcc_labels_sym(g, label, &g->n_wcc));
    g->wcc_built = true;
    return GIR_OK;
}

}  // namespace gir
