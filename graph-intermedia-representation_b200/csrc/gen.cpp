// Deterministic synthetic-graph generators for the benchmark and test workloads.
//
// Every random choice is a counter-based hash of (seed, index, ...), so the output does not
// depend on the thread count and the same call gives the same graph on every machine.
// Graphs are produced as directed, self-loop-free, duplicate-free edge lists and turned into
// the reference's four-file CSR layout (fw/bw begin + adjacent, int32), which is what the
// reference loader reads (gir_constructor/graph.cpp:2-120) and what gir_dev_create takes.
//
// Host-only C++ (OpenMP). Exported through a small C ABI declared in include/gir_gen.h.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <parallel/algorithm>
#include <string>
#include <vector>

#include "gir_gen.h"

namespace {

// splitmix64 finalizer (Steele, Lea, Flood 2014): a bijective 64-bit mixer.
inline uint64_t mix64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
inline uint64_t hash3(uint64_t seed, uint64_t a, uint64_t b) {
    return mix64(mix64(seed ^ 0x5851f42d4c957f2dULL) ^ mix64(a * 0x2545f4914f6cdd1dULL + b));
}
inline double unit(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

template <class T>
void psort(std::vector<T>& v) {
    if (v.size() >= (1u << 16)) __gnu_parallel::sort(v.begin(), v.end());
    else std::sort(v.begin(), v.end());
}

struct Draw {
    uint64_t key;  // (u << 32) | v
    uint64_t idx;  // draw index (the earliest draw of a key is the one kept)
    bool operator<(const Draw& o) const { return key != o.key ? key < o.key : idx < o.idx; }
};

// One R-MAT draw: `scale` quadrant choices, most significant bit first.
inline void rmatDraw(uint64_t seed, uint64_t i, int scale, double a, double b, double c, uint64_t& u,
                     uint64_t& v) {
    u = 0; v = 0;
    const double ab = a + b, abc = a + b + c;
    for (int l = 0; l < scale; ++l) {
        const double r = unit(hash3(seed, i, (uint64_t)l));
        const uint64_t bu = r >= ab, bv = (r >= a && r < ab) || r >= abc;
        u = (u << 1) | bu;
        v = (v << 1) | bv;
    }
}

thread_local std::string g_err;

}  // namespace

extern "C" {

const char* gir_gen_last_error(void) { return g_err.c_str(); }

void gir_gen_free(void* p) { std::free(p); }

uint64_t gir_gen_hash3(uint64_t seed, uint64_t a, uint64_t b) { return hash3(seed, a, b); }

int gir_gen_rmat(int scale, int64_t V, int64_t n_draws, int64_t target_unique, double a, double b, double c,
                 uint64_t seed, int permute, int64_t* n_out, int32_t** src_out, int32_t** dst_out) {
    if (scale < 1 || scale > 31 || V < 1 || V > ((int64_t)1 << scale) || V > INT32_MAX || n_draws < 0 ||
        a < 0 || b < 0 || c < 0 || a + b + c > 1.0) {
        g_err = "gir_gen_rmat: invalid arguments";
        return 1;
    }
    // Draw, drop self-loops and ids >= V, keep the earliest draw of every distinct edge. When a
    // target count is given, keep drawing until at least that many distinct edges exist, then
    // keep the `target_unique` distinct edges whose first draw came earliest.
    std::vector<Draw> d;
    uint64_t drawn = 0;
    uint64_t want = (uint64_t)(target_unique > 0 ? (double)target_unique * 1.3 + 1024 : (double)n_draws);
    for (int attempt = 0; attempt < 8; ++attempt) {
        const uint64_t lo = drawn, hi = want;
        {  // (the new draws are released before the sort: peak memory is the sort's, not 3x)
            std::vector<Draw> add(hi - lo);
            #pragma omp parallel for schedule(static)
            for (int64_t i = (int64_t)lo; i < (int64_t)hi; ++i) {
                uint64_t u, v;
                rmatDraw(seed, (uint64_t)i, scale, a, b, c, u, v);
                add[i - lo] = (u == v || u >= (uint64_t)V || v >= (uint64_t)V) ? Draw{~0ULL, (uint64_t)i}
                                                                               : Draw{(u << 32) | v, (uint64_t)i};
            }
            d.insert(d.end(), add.begin(), add.end());
        }
        drawn = hi;
        psort(d);
        size_t m = 0;
        for (size_t i = 0; i < d.size(); ++i) {
            if (d[i].key == ~0ULL) break;
            if (m > 0 && d[m - 1].key == d[i].key) continue;
            d[m++] = d[i];
        }
        d.resize(m);
        if (target_unique <= 0 || (int64_t)m >= target_unique) break;
        want = drawn + (uint64_t)((double)(target_unique - (int64_t)m) * 2.0) + 4096;
    }
    if (target_unique > 0) {
        if ((int64_t)d.size() < target_unique) {
            g_err = "gir_gen_rmat: could not reach the target edge count (graph too dense for V)";
            return 2;
        }
        std::nth_element(d.begin(), d.begin() + target_unique, d.end(),
                         [](const Draw& x, const Draw& y) { return x.idx < y.idx; });
        d.resize(target_unique);
    }
    std::vector<int32_t> perm;
    if (permute) {
        std::vector<std::pair<uint64_t, int32_t>> r(V);
        #pragma omp parallel for schedule(static)
        for (int64_t x = 0; x < V; ++x) r[x] = {hash3(seed ^ 0x7065726dULL, (uint64_t)x, 17), (int32_t)x};
        psort(r);
        perm.resize(V);
        #pragma omp parallel for schedule(static)
        for (int64_t k = 0; k < V; ++k) perm[r[k].second] = (int32_t)k;
    }
    const int64_t n = (int64_t)d.size();
    int32_t* s = (int32_t*)std::malloc(sizeof(int32_t) * (n > 0 ? n : 1));
    int32_t* t = (int32_t*)std::malloc(sizeof(int32_t) * (n > 0 ? n : 1));
    if (!s || !t) { std::free(s); std::free(t); g_err = "gir_gen_rmat: out of host memory"; return 3; }
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        int32_t u = (int32_t)(d[i].key >> 32), v = (int32_t)(d[i].key & 0xffffffffULL);
        if (permute) { u = perm[u]; v = perm[v]; }
        s[i] = u; t[i] = v;
    }
    *n_out = n; *src_out = s; *dst_out = t;
    return 0;
}

int gir_gen_lattice(int64_t side, double remove_frac, double longrange_frac, double pareto_shape,
                    uint64_t seed, int64_t* n_out, int32_t** src_out, int32_t** dst_out, uint32_t** w_out) {
    // side x side 4-neighbour lattice, vertex id = row * side + col. Every lattice edge is kept
    // with probability 1 - remove_frac (both directions together: the result stays symmetric).
    // Then longrange_frac * (#lattice edges) extra undirected edges are added: a uniform start
    // vertex, a direction uniform on the circle and a length from a Pareto(shape, x_m = 1)
    // distribution, clamped into the lattice. Weight of {u,v} = round(100 * Euclidean length)
    // + U[0, 50], the same in both directions.
    if (side < 2 || side > 46340 || remove_frac < 0 || remove_frac > 1 || longrange_frac < 0 || pareto_shape <= 0) {
        g_err = "gir_gen_lattice: invalid arguments";
        return 1;
    }
    const int64_t V = side * side;
    const int64_t n_lat = 2 * side * (side - 1);  // undirected lattice edges
    const int64_t n_lr = (int64_t)std::llround(longrange_frac * (double)n_lat);
    struct UE { uint64_t key; uint32_t w; bool operator<(const UE& o) const { return key < o.key; } };
    std::vector<UE> und(n_lat + n_lr);
    std::vector<char> keep(n_lat + n_lr, 0);
    #pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < n_lat; ++e) {
        // e < side*(side-1): horizontal (r, c)-(r, c+1); else vertical (r, c)-(r+1, c).
        int64_t u, v;
        const int64_t h = side * (side - 1);
        if (e < h) { int64_t r = e / (side - 1), c = e % (side - 1); u = r * side + c; v = u + 1; }
        else { int64_t k = e - h, r = k / side, c = k % side; u = r * side + c; v = u + side; }
        const bool on = unit(hash3(seed, (uint64_t)e, 1)) >= remove_frac;
        const uint32_t w = 100u + (uint32_t)(hash3(seed, (uint64_t)e, 2) % 51u);
        und[e] = {((uint64_t)u << 32) | (uint64_t)v, w};
        keep[e] = on;
    }
    #pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n_lr; ++k) {
        const uint64_t id = (uint64_t)(n_lat + k);
        const int64_t u = (int64_t)(hash3(seed, id, 3) % (uint64_t)V);
        const double ang = 2.0 * M_PI * unit(hash3(seed, id, 4));
        const double len = std::pow(1.0 - unit(hash3(seed, id, 5)), -1.0 / pareto_shape);
        const int64_t r0 = u / side, c0 = u % side;
        int64_t r1 = r0 + (int64_t)std::llround(len * std::sin(ang));
        int64_t c1 = c0 + (int64_t)std::llround(len * std::cos(ang));
        r1 = std::min<int64_t>(std::max<int64_t>(r1, 0), side - 1);
        c1 = std::min<int64_t>(std::max<int64_t>(c1, 0), side - 1);
        const int64_t v = r1 * side + c1;
        const double el = std::sqrt((double)((r1 - r0) * (r1 - r0) + (c1 - c0) * (c1 - c0)));
        const uint32_t w = (uint32_t)std::llround(100.0 * el) + (uint32_t)(hash3(seed, id, 6) % 51u);
        const int64_t a = std::min(u, v), b = std::max(u, v);
        und[n_lat + k] = {((uint64_t)a << 32) | (uint64_t)b, w};
        keep[n_lat + k] = (u != v);
    }
    size_t m = 0;
    for (size_t i = 0; i < und.size(); ++i) if (keep[i]) und[m++] = und[i];
    und.resize(m);
    // Duplicate undirected pairs keep the entry that sorts first (stable: lattice entries come
    // before long-range ones with the same key).
    std::stable_sort(und.begin(), und.end());
    size_t q = 0;
    for (size_t i = 0; i < und.size(); ++i) {
        if (q > 0 && und[q - 1].key == und[i].key) continue;
        und[q++] = und[i];
    }
    und.resize(q);
    const int64_t n = 2 * (int64_t)q;
    int32_t* s = (int32_t*)std::malloc(sizeof(int32_t) * (n > 0 ? n : 1));
    int32_t* t = (int32_t*)std::malloc(sizeof(int32_t) * (n > 0 ? n : 1));
    uint32_t* w = (uint32_t*)std::malloc(sizeof(uint32_t) * (n > 0 ? n : 1));
    if (!s || !t || !w) { std::free(s); std::free(t); std::free(w); g_err = "gir_gen_lattice: out of host memory"; return 3; }
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)q; ++i) {
        const int32_t a = (int32_t)(und[i].key >> 32), b = (int32_t)(und[i].key & 0xffffffffULL);
        s[2 * i] = a; t[2 * i] = b; w[2 * i] = und[i].w;
        s[2 * i + 1] = b; t[2 * i + 1] = a; w[2 * i + 1] = und[i].w;
    }
    *n_out = n; *src_out = s; *dst_out = t; *w_out = w;
    return 0;
}

int gir_gen_csr(int64_t V, int64_t n, const int32_t* src, const int32_t* dst, const uint32_t* w_in,
                int32_t* fw_beg, int32_t* fw_adj, int32_t* bw_beg, int32_t* bw_adj, uint32_t* w_fw) {
    // Forward and backward CSR of an edge list, every row sorted by neighbour id. Duplicates and
    // self-loops are kept as given (the generators never produce them; the loader's
    // normalisation removes them). w_in / w_fw (both optional) carry one weight per edge into
    // forward-CSR order.
    if (V < 0 || V > INT32_MAX || n < 0 || n > INT32_MAX) { g_err = "gir_gen_csr: sizes exceed int32"; return 1; }
    for (int64_t i = 0; i < n; ++i)
        if (src[i] < 0 || src[i] >= V || dst[i] < 0 || dst[i] >= V) { g_err = "gir_gen_csr: vertex id out of range"; return 2; }
    std::vector<std::pair<uint64_t, uint32_t>> k(n);
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) k[i] = {((uint64_t)(uint32_t)src[i] << 32) | (uint32_t)dst[i], w_in ? w_in[i] : 0u};
    psort(k);
    std::vector<int64_t> cnt(V + 1, 0);
    for (int64_t i = 0; i < n; ++i) cnt[(k[i].first >> 32) + 1]++;
    for (int64_t x = 0; x < V; ++x) cnt[x + 1] += cnt[x];
    for (int64_t x = 0; x <= V; ++x) fw_beg[x] = (int32_t)cnt[x];
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        fw_adj[i] = (int32_t)(k[i].first & 0xffffffffULL);
        if (w_fw) w_fw[i] = k[i].second;
    }
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) k[i] = {((uint64_t)(uint32_t)dst[i] << 32) | (uint32_t)src[i], 0u};
    psort(k);
    std::fill(cnt.begin(), cnt.end(), 0);
    for (int64_t i = 0; i < n; ++i) cnt[(k[i].first >> 32) + 1]++;
    for (int64_t x = 0; x < V; ++x) cnt[x + 1] += cnt[x];
    for (int64_t x = 0; x <= V; ++x) bw_beg[x] = (int32_t)cnt[x];
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) bw_adj[i] = (int32_t)(k[i].first & 0xffffffffULL);
    return 0;
}

void gir_gen_uniform_weights(int64_t V, const int32_t* fw_beg, const int32_t* fw_adj, uint32_t lo, uint32_t hi,
                             uint64_t seed, uint32_t* w_out) {
    // w(u,v) = lo + hash(seed, u, v) mod (hi - lo + 1): a function of the edge alone, so the
    // forward and backward copies of an edge, and an edge deleted and inserted again, agree.
    const uint64_t span = (uint64_t)hi - lo + 1;
    #pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t u = 0; u < V; ++u)
        for (int64_t e = fw_beg[u]; e < fw_beg[u + 1]; ++e)
            w_out[e] = lo + (uint32_t)(hash3(seed, (uint64_t)u, (uint64_t)(uint32_t)fw_adj[e]) % span);
}

void gir_gen_sources(int64_t V, int64_t n, uint64_t seed, int32_t* out) {
    for (int64_t i = 0; i < n; ++i) out[i] = (int32_t)(hash3(seed, (uint64_t)i, 99) % (uint64_t)V);
}

void gir_gen_updates(int64_t V, const int32_t* fw_beg, const int32_t* fw_adj, int64_t n_ins, int64_t n_del,
                     uint64_t seed, int32_t* u_out, int32_t* v_out, uint8_t* ins_out) {
    // n_ins uniform random inserts (u != v) and n_del deletions of edges drawn uniformly (with
    // replacement) from the given CSR, interleaved in a hash-defined order.
    const int64_t E = fw_beg[V], n = n_ins + n_del;
    std::vector<std::pair<uint64_t, int64_t>> order(n);
    for (int64_t i = 0; i < n; ++i) order[i] = {hash3(seed, (uint64_t)i, 7), i};
    psort(order);
    #pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; ++k) {
        const int64_t i = order[k].second;
        if (i < n_ins || E == 0) {
            int64_t u = (int64_t)(hash3(seed, (uint64_t)i, 11) % (uint64_t)V);
            int64_t v = (int64_t)(hash3(seed, (uint64_t)i, 12) % (uint64_t)(V > 1 ? V - 1 : 1));
            if (V > 1 && v >= u) ++v;
            u_out[k] = (int32_t)u; v_out[k] = (int32_t)v; ins_out[k] = 1;
        } else {
            const int64_t e = (int64_t)(hash3(seed, (uint64_t)i, 13) % (uint64_t)E);
            const int32_t* p = std::upper_bound(fw_beg, fw_beg + V + 1, (int32_t)e);
            u_out[k] = (int32_t)(p - fw_beg - 1); v_out[k] = fw_adj[e]; ins_out[k] = 0;
        }
    }
}

int gir_write_four_files(const char* dir, int64_t V, const int32_t* fw_beg, const int32_t* fw_adj,
                         const int32_t* bw_beg, const int32_t* bw_adj) {
    // The reference's on-disk layout: <dir>fw_begin.bin (int32[V+1]), fw_adjacent.bin
    // (int32[E]), and the same for bw (README.md:88-96 of the reference).
    const std::string d(dir);
    const int64_t E = fw_beg[V];
    struct F { const char* name; const int32_t* p; int64_t n; } fs[4] = {
        {"fw_begin.bin", fw_beg, V + 1}, {"fw_adjacent.bin", fw_adj, E},
        {"bw_begin.bin", bw_beg, V + 1}, {"bw_adjacent.bin", bw_adj, bw_beg[V]}};
    for (auto& f : fs) {
        FILE* fp = std::fopen((d + f.name).c_str(), "wb");
        if (!fp) { g_err = "gir_write_four_files: cannot open " + d + f.name; return 1; }
        const size_t wrote = f.n ? std::fwrite(f.p, sizeof(int32_t), (size_t)f.n, fp) : 0;
        std::fclose(fp);
        if ((int64_t)wrote != f.n) { g_err = "gir_write_four_files: short write to " + d + f.name; return 2; }
    }
    return 0;
}

}  // extern "C"
