/* CPU restatement of the reference GIR hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker for the CUDA library, never part of it: only tests/, the smoke
 * check in __graft_entry__.py and bench.py's CPU-baseline leg load the library built from it.
 * Each function restates the reference's algorithm for one row of the hot path, citing the
 * reference file:line it follows (paths are relative to the reference project root). Results
 * are returned in canonical form (component label = smallest vertex id of the component;
 * blocks keyed by their two smallest vertices), the form the reference's own tests compare in
 * (gir_constructor/gir_test.cpp:365-374 normalizePartition).
 *
 * Pinning: tests/test_oracle.py checks every function here against the reference itself,
 * compiled from its own sources into oracle/_ref/ by oracle/Makefile, and against the golden
 * vectors under tests/golden/ that were generated from that build.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#define OR_OK 0
#define OR_ERR_OPEN 1       /* a file cannot be opened (graph.cpp:20-24) */
#define OR_ERR_SIZES 2      /* fw / bw files disagree in V or E (graph.cpp:104-112) */
#define OR_ERR_FW 3         /* forward CSR malformed (graph.cpp:95-103) */
#define OR_ERR_BW 4         /* backward CSR malformed */
#define OR_ERR_DEDUP 5      /* fw and bw disagree after deduplication (gir.cpp:122-126) */
#define OR_ERR_SHORT 6      /* short read */

static int64_t file_size(const char* p) {
    struct stat st;
    return stat(p, &st) == 0 ? (int64_t)st.st_size : -1;
}

/* Sizes of a four-file CSR, as the reference loader derives them: V = |fw_begin|/4 - 1,
 * E = |fw_adjacent|/4 (graph.cpp:14-15). */
int or_file_sizes(const char* dir, int64_t* V, int64_t* E, int64_t* Vb, int64_t* Eb) {
    char p[4096];
    int64_t s[4];
    const char* names[4] = {"fw_begin.bin", "fw_adjacent.bin", "bw_begin.bin", "bw_adjacent.bin"};
    for (int i = 0; i < 4; ++i) {
        snprintf(p, sizeof p, "%s%s", dir, names[i]);
        s[i] = file_size(p);
        if (s[i] < 0) return OR_ERR_OPEN;
    }
    *V = s[0] / 4 - 1; *E = s[1] / 4; *Vb = s[2] / 4 - 1; *Eb = s[3] / 4;
    return OR_OK;
}

static int read_ints(const char* dir, const char* name, int32_t* out, int64_t n) {
    char p[4096];
    snprintf(p, sizeof p, "%s%s", dir, name);
    FILE* f = fopen(p, "rb");
    if (!f) return OR_ERR_OPEN;
    int64_t got = n ? (int64_t)fread(out, sizeof(int32_t), (size_t)n, f) : 0;
    fclose(f);
    return got == n ? OR_OK : OR_ERR_SHORT;
}

static int csr_ok(int64_t V, int64_t E, const int32_t* beg, const int32_t* adj) {
    if (beg[0] != 0 || beg[V] != E) return 0;
    for (int64_t i = 0; i < V; ++i) if (beg[i] > beg[i + 1]) return 0;
    for (int64_t i = 0; i < E; ++i) if (adj[i] < 0 || adj[i] >= V) return 0;
    return 1;
}

/* graph::graph (graph.cpp:2-120): read the four int32 files and validate them. The size
 * check of the bw files comes before the per-CSR checks, as in the reference (:104-114). */
int or_load(const char* dir, int64_t V, int64_t E, int32_t* fwb, int32_t* fwa, int32_t* bwb, int32_t* bwa) {
    int64_t v0, e0, vb, eb;
    int rc = or_file_sizes(dir, &v0, &e0, &vb, &eb);
    if (rc) return rc;
    if (v0 != V || e0 != E) return OR_ERR_SIZES;
    if ((rc = read_ints(dir, "fw_begin.bin", fwb, V + 1))) return rc;
    if ((rc = read_ints(dir, "fw_adjacent.bin", fwa, E))) return rc;
    if (vb != V || eb != E) return OR_ERR_SIZES;
    if ((rc = read_ints(dir, "bw_begin.bin", bwb, V + 1))) return rc;
    if ((rc = read_ints(dir, "bw_adjacent.bin", bwa, E))) return rc;
    if (!csr_ok(V, E, fwb, fwa)) return OR_ERR_FW;
    if (!csr_ok(V, E, bwb, bwa)) return OR_ERR_BW;
    return OR_OK;
}

static int cmp_i32(const void* a, const void* b) {
    int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
    return (x > y) - (x < y);
}
static int cmp_i64(const void* a, const void* b) {
    int64_t x = *(const int64_t*)a, y = *(const int64_t*)b;
    return (x > y) - (x < y);
}

/* normalizeOneCsr (gir.cpp:95-116): sort every row, drop duplicate entries, compact. Self-loops
 * stay (only the symmetrized view drops them). beg (V+1, int64) and adj are rewritten in
 * place; returns the new edge count. */
int64_t or_normalize(int64_t V, int64_t* beg, int32_t* adj) {
    int64_t w = 0;
    for (int64_t v = 0; v < V; ++v) {
        int64_t b = beg[v], e = beg[v + 1];
        qsort(adj + b, (size_t)(e - b), sizeof(int32_t), cmp_i32);
        int64_t start = w;
        for (int64_t i = b; i < e; ++i)
            if (i == b || adj[i] != adj[i - 1]) adj[w++] = adj[i];
        beg[v] = start;
    }
    beg[V] = w;
    return w;
}

/* The symmetrized base view of buildWCC (gir.cpp:599-625): per vertex, fw list + bw list,
 * sorted, deduplicated, self removed. Call with sym_adj == NULL to get the size. */
int64_t or_sym(int64_t V, const int64_t* fwb, const int32_t* fwa, const int64_t* bwb, const int32_t* bwa,
               int64_t* sym_beg, int32_t* sym_adj) {
    int64_t maxdeg = 0;
    for (int64_t u = 0; u < V; ++u) {
        int64_t d = (fwb[u + 1] - fwb[u]) + (bwb[u + 1] - bwb[u]);
        if (d > maxdeg) maxdeg = d;
    }
    int32_t* tmp = (int32_t*)malloc(sizeof(int32_t) * (size_t)(maxdeg > 0 ? maxdeg : 1));
    int64_t w = 0;
    for (int64_t u = 0; u < V; ++u) {
        int64_t k = 0;
        for (int64_t i = fwb[u]; i < fwb[u + 1]; ++i) tmp[k++] = fwa[i];
        for (int64_t i = bwb[u]; i < bwb[u + 1]; ++i) tmp[k++] = bwa[i];
        qsort(tmp, (size_t)k, sizeof(int32_t), cmp_i32);
        if (sym_beg) sym_beg[u] = w;
        for (int64_t i = 0; i < k; ++i) {
            if (tmp[i] == (int32_t)u || (i > 0 && tmp[i] == tmp[i - 1])) continue;
            if (sym_adj) sym_adj[w] = tmp[i];
            ++w;
        }
    }
    if (sym_beg) sym_beg[V] = w;
    free(tmp);
    return w;
}

static int32_t uf_find(int32_t* p, int32_t x) {
    while (p[x] != x) { p[x] = p[p[x]]; x = p[x]; }
    return x;
}

/* buildWCC union-find over the forward edges (gir.cpp:635-653). The reference links the
 * root of u under the root of v; here the larger root goes under the smaller one, so every
 * root is its component's smallest vertex (the canonical label). Same partition. */
void or_wcc(int64_t V, const int64_t* beg, const int32_t* adj, int32_t* label) {
    for (int64_t i = 0; i < V; ++i) label[i] = (int32_t)i;
    for (int64_t u = 0; u < V; ++u)
        for (int64_t i = beg[u]; i < beg[u + 1]; ++i) {
            int32_t a = uf_find(label, (int32_t)u), b = uf_find(label, adj[i]);
            if (a < b) label[b] = a; else if (b < a) label[a] = b;
        }
    for (int64_t i = 0; i < V; ++i) label[i] = uf_find(label, (int32_t)i);
}

/* Iterative Tarjan over all vertices in id order (tarjanScc gir.cpp:494-537, run by
 * buildSCC_DAG gir.cpp:798-816). Output: label[v] = smallest vertex of v's SCC. */
void or_scc(int64_t V, const int64_t* beg, const int32_t* adj, int32_t* label) {
    int32_t* idx = (int32_t*)malloc(sizeof(int32_t) * (size_t)(V + 1));
    int32_t* low = (int32_t*)malloc(sizeof(int32_t) * (size_t)(V + 1));
    char* on = (char*)calloc((size_t)V + 1, 1);
    int32_t* stk = (int32_t*)malloc(sizeof(int32_t) * (size_t)(V + 1));
    int32_t* cs_v = (int32_t*)malloc(sizeof(int32_t) * (size_t)(V + 1));
    int64_t* cs_i = (int64_t*)malloc(sizeof(int64_t) * (size_t)(V + 1));
    for (int64_t i = 0; i < V; ++i) idx[i] = -1;
    int32_t counter = 0;
    int64_t sp = 0;
    for (int64_t r = 0; r < V; ++r) {
        if (idx[r] != -1) continue;
        int64_t cp = 0;
        idx[r] = low[r] = counter++;
        stk[sp++] = (int32_t)r; on[r] = 1;
        cs_v[cp] = (int32_t)r; cs_i[cp] = beg[r]; ++cp;
        while (cp > 0) {
            int32_t v = cs_v[cp - 1];
            if (cs_i[cp - 1] < beg[v + 1]) {
                int32_t w = adj[cs_i[cp - 1]++];
                if (idx[w] == -1) {
                    idx[w] = low[w] = counter++;
                    stk[sp++] = w; on[w] = 1;
                    cs_v[cp] = w; cs_i[cp] = beg[w]; ++cp;
                } else if (on[w] && idx[w] < low[v]) {
                    low[v] = idx[w];
                }
            } else {
                --cp;
                if (cp > 0 && low[v] < low[cs_v[cp - 1]]) low[cs_v[cp - 1]] = low[v];
                if (low[v] == idx[v]) {
                    int64_t top = sp;
                    int32_t mn = v;
                    do { --sp; if (stk[sp] < mn) mn = stk[sp]; } while (stk[sp] != v);
                    for (int64_t k = sp; k < top; ++k) { on[stk[k]] = 0; label[stk[k]] = mn; }
                }
            }
        }
    }
    free(idx); free(low); free(on); free(stk); free(cs_v); free(cs_i);
}

/* Condensation edges (buildSCC_DAG gir.cpp:825-831): every forward edge whose endpoints lie in
 * different SCCs, as the sorted distinct keys (label_u << 32 | label_v). Call with out == NULL
 * to get the count. */
int64_t or_dag(int64_t V, const int64_t* beg, const int32_t* adj, const int32_t* scc, int64_t* out) {
    int64_t n = 0;
    for (int64_t u = 0; u < V; ++u)
        for (int64_t i = beg[u]; i < beg[u + 1]; ++i)
            if (scc[u] != scc[adj[i]]) ++n;
    int64_t* k = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    n = 0;
    for (int64_t u = 0; u < V; ++u)
        for (int64_t i = beg[u]; i < beg[u + 1]; ++i)
            if (scc[u] != scc[adj[i]]) k[n++] = ((int64_t)scc[u] << 32) | (int64_t)(uint32_t)scc[adj[i]];
    qsort(k, (size_t)n, sizeof(int64_t), cmp_i64);
    int64_t m = 0;
    for (int64_t i = 0; i < n; ++i) if (i == 0 || k[i] != k[i - 1]) k[m++] = k[i];
    if (out) memcpy(out, k, sizeof(int64_t) * (size_t)m);
    free(k);
    return m;
}

typedef struct { int32_t k1, k2, v; } Triple;
static int cmp_triple(const void* a, const void* b) {
    const Triple *x = (const Triple*)a, *y = (const Triple*)b;
    if (x->k1 != y->k1) return (x->k1 > y->k1) - (x->k1 < y->k1);
    if (x->k2 != y->k2) return (x->k2 > y->k2) - (x->k2 < y->k2);
    return (x->v > y->v) - (x->v < y->v);
}

/* Per-SCC biconnected blocks of the SCC-induced undirected graph (buildBCT gir.cpp:2063-2089,
 * via the vertex-stack Hopcroft-Tarjan of gir.cpp:541-587; a vertex with no neighbour in its
 * SCC is a singleton block, gir.cpp:584). Blocks are emitted as membership triples
 * (k1, k2, v): k1 < k2 are the block's two smallest vertices (k2 = -1 for a singleton block),
 * which identify a block uniquely since two blocks share at most one vertex. Output is sorted;
 * call with out == NULL to get the count. `ap` (optional, V bytes) receives 1 for vertices in
 * two or more blocks (isArticulationPoint, gir.h:125). */
int64_t or_bicc(int64_t V, const int64_t* sb, const int32_t* sa, const int32_t* scc, int32_t* out_k1,
                int32_t* out_k2, int32_t* out_v, uint8_t* ap) {
    int32_t* disc = (int32_t*)malloc(sizeof(int32_t) * (size_t)(V + 1));
    int32_t* low = (int32_t*)malloc(sizeof(int32_t) * (size_t)(V + 1));
    int32_t* stk = (int32_t*)malloc(sizeof(int32_t) * (size_t)(V + 1));
    int32_t* cs_v = (int32_t*)malloc(sizeof(int32_t) * (size_t)(V + 1));
    int32_t* cs_p = (int32_t*)malloc(sizeof(int32_t) * (size_t)(V + 1));
    int64_t* cs_i = (int64_t*)malloc(sizeof(int64_t) * (size_t)(V + 1));
    int32_t* cnt = (int32_t*)calloc((size_t)V + 1, sizeof(int32_t));
    int32_t* blk = (int32_t*)malloc(sizeof(int32_t) * (size_t)(V + 1));
    int64_t cap = 2 * V + 16, nt = 0;
    Triple* t = (Triple*)malloc(sizeof(Triple) * (size_t)cap);
    for (int64_t i = 0; i < V; ++i) disc[i] = -1;
    int32_t tick = 0;
    int64_t sp = 0;
#define EMIT_BLOCK(ARR, N)                                                              \
    do {                                                                                \
        int32_t m1 = INT32_MAX, m2 = INT32_MAX;                                         \
        for (int64_t q = 0; q < (N); ++q) {                                             \
            int32_t x = (ARR)[q];                                                       \
            if (x < m1) { m2 = m1; m1 = x; } else if (x < m2) m2 = x;                   \
        }                                                                               \
        if ((N) == 1) m2 = -1;                                                          \
        for (int64_t q = 0; q < (N); ++q) {                                             \
            if (nt == cap) { cap *= 2; t = (Triple*)realloc(t, sizeof(Triple) * (size_t)cap); } \
            t[nt].k1 = m1; t[nt].k2 = m2; t[nt].v = (ARR)[q]; ++nt; cnt[(ARR)[q]]++;     \
        }                                                                               \
    } while (0)
    for (int64_t r = 0; r < V; ++r) {
        if (disc[r] != -1) continue;
        int64_t cp = 0;
        int root_child = 0;
        disc[r] = low[r] = tick++;
        stk[sp++] = (int32_t)r;
        cs_v[cp] = (int32_t)r; cs_p[cp] = -1; cs_i[cp] = sb[r]; ++cp;
        while (cp > 0) {
            int32_t v = cs_v[cp - 1], p = cs_p[cp - 1];
            if (cs_i[cp - 1] < sb[v + 1]) {
                int32_t w = sa[cs_i[cp - 1]++];
                if (w == v || w == p || scc[w] != scc[v]) continue;
                if (disc[w] == -1) {
                    disc[w] = low[w] = tick++;
                    stk[sp++] = w;
                    if (v == (int32_t)r) root_child = 1;
                    cs_v[cp] = w; cs_p[cp] = v; cs_i[cp] = sb[w]; ++cp;
                } else if (disc[w] < low[v]) {
                    low[v] = disc[w];
                }
            } else {
                --cp;
                if (p == -1) continue;
                if (low[v] < low[p]) low[p] = low[v];
                if (low[v] >= disc[p]) {
                    int64_t n = 0;
                    for (;;) { int32_t x = stk[--sp]; blk[n++] = x; if (x == v) break; }
                    blk[n++] = p;
                    EMIT_BLOCK(blk, n);
                }
            }
        }
        --sp;  /* r */
        if (!root_child) { blk[0] = (int32_t)r; EMIT_BLOCK(blk, 1); }
    }
#undef EMIT_BLOCK
    qsort(t, (size_t)nt, sizeof(Triple), cmp_triple);
    if (out_k1)
        for (int64_t i = 0; i < nt; ++i) { out_k1[i] = t[i].k1; out_k2[i] = t[i].k2; out_v[i] = t[i].v; }
    if (ap) for (int64_t i = 0; i < V; ++i) ap[i] = cnt[i] >= 2;
    free(disc); free(low); free(stk); free(cs_v); free(cs_p); free(cs_i); free(cnt); free(blk); free(t);
    return nt;
}

/* Breadth-first levels from a set of sources (-1 = unreachable). GIR::bfs (gir_query.cpp:108-294)
 * computes exactly these levels from one source; levels are unique, so a plain FIFO BFS
 * (sequentialBfs, gir_test.cpp:865-881) is an exact oracle for it. Several sources give the
 * multi-source levels (min over the sources). Out-of-range sources are ignored, as the
 * reference returns all -1 for them (gir_query.cpp:112). */
void or_bfs(int64_t V, const int64_t* beg, const int32_t* adj, const int32_t* srcs, int64_t n_src, int32_t* level) {
    int32_t* q = (int32_t*)malloc(sizeof(int32_t) * (size_t)(V + 1));
    int64_t qh = 0, qt = 0;
    for (int64_t i = 0; i < V; ++i) level[i] = -1;
    for (int64_t i = 0; i < n_src; ++i) {
        int32_t s = srcs[i];
        if (s < 0 || s >= V || level[s] == 0) continue;
        level[s] = 0; q[qt++] = s;
    }
    while (qh < qt) {
        int32_t u = q[qh++];
        for (int64_t i = beg[u]; i < beg[u + 1]; ++i) {
            int32_t w = adj[i];
            if (level[w] == -1) { level[w] = level[u] + 1; q[qt++] = w; }
        }
    }
    free(q);
}

/* GIR::edgeWeight (gir_query.cpp:50-54): the 64-bit finalizer of MurmurHash3 (fmix64) on
 * (u << 32 | v), mapped into [1, 100]. */
uint32_t or_edge_weight(int32_t u, int32_t v) {
    uint64_t x = ((uint64_t)(uint32_t)u << 32) | (uint32_t)v;
    x ^= x >> 33; x *= 0xff51afd7ed558ccdULL; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL; x ^= x >> 33;
    return 1 + (uint32_t)(x % 100u);
}

typedef struct { uint64_t d; int32_t v; } HeapItem;
static void heap_push(HeapItem* h, int64_t* n, HeapItem it) {
    int64_t i = (*n)++;
    while (i > 0) {
        int64_t p = (i - 1) / 2;
        if (h[p].d <= it.d) break;
        h[i] = h[p]; i = p;
    }
    h[i] = it;
}
static HeapItem heap_pop(HeapItem* h, int64_t* n) {
    HeapItem top = h[0], last = h[--(*n)];
    int64_t i = 0;
    for (;;) {
        int64_t c = 2 * i + 1;
        if (c >= *n) break;
        if (c + 1 < *n && h[c + 1].d < h[c].d) ++c;
        if (h[c].d >= last.d) break;
        h[i] = h[c]; i = c;
    }
    if (*n > 0) h[i] = last;
    return top;
}

/* Exact single/multi-source shortest distances (UINT64_MAX = unreachable), Dijkstra with a
 * binary heap, as QueryTest::dijkstra (gir_test.cpp:957-972). Shortest distances are unique,
 * so this equals GIR::sssp's Delta-stepping result (gir_query.cpp:629-703) for every Delta.
 * w == NULL: weights are or_edge_weight(u, v) (the reference's only mode); otherwise w holds
 * one uint32 weight per forward-CSR entry. */
void or_sssp(int64_t V, const int64_t* beg, const int32_t* adj, const uint32_t* w, const int32_t* srcs,
             int64_t n_src, uint64_t* dist) {
    int64_t E = beg[V];
    HeapItem* h = (HeapItem*)malloc(sizeof(HeapItem) * (size_t)(E + n_src + 1));
    int64_t n = 0;
    for (int64_t i = 0; i < V; ++i) dist[i] = UINT64_MAX;
    for (int64_t i = 0; i < n_src; ++i) {
        int32_t s = srcs[i];
        if (s < 0 || s >= V || dist[s] == 0) continue;
        dist[s] = 0;
        HeapItem it = {0, s};
        heap_push(h, &n, it);
    }
    while (n > 0) {
        HeapItem it = heap_pop(h, &n);
        if (it.d != dist[it.v]) continue;
        int32_t u = it.v;
        for (int64_t i = beg[u]; i < beg[u + 1]; ++i) {
            int32_t x = adj[i];
            uint64_t nd = it.d + (w ? w[i] : or_edge_weight(u, x));
            if (nd < dist[x]) { dist[x] = nd; HeapItem j = {nd, x}; heap_push(h, &n, j); }
        }
    }
    free(h);
}

typedef struct { int64_t key; int64_t pos; } KeyPos;
static int cmp_keypos(const void* a, const void* b) {
    const KeyPos *x = (const KeyPos*)a, *y = (const KeyPos*)b;
    if (x->key != y->key) return (x->key > y->key) - (x->key < y->key);
    return (x->pos > y->pos) - (x->pos < y->pos);
}

static int has_edge(const int64_t* beg, const int32_t* adj, int32_t u, int32_t v) {
    int64_t lo = beg[u], hi = beg[u + 1];
    while (lo < hi) {
        int64_t m = (lo + hi) / 2;
        if (adj[m] < v) lo = m + 1; else hi = m;
    }
    return lo < beg[u + 1] && adj[lo] == v;
}

/* normalizeBatch (gir.cpp:3523-3586) followed by the edge-store effect of applyBatch: per edge
 * only the last operation of the batch counts, operations with u == v or an endpoint outside
 * [0, V) are dropped, and the result is the new edge set. Input: the current graph as a
 * forward CSR with sorted rows; output: the new forward CSR (new_beg V+1, new_adj capacity
 * E + n). Returns the new edge count; *n_ins / *n_del get the number of edges that appeared /
 * disappeared. */
int64_t or_apply_batch(int64_t V, const int64_t* beg, const int32_t* adj, const int32_t* u, const int32_t* v,
                       const uint8_t* ins, int64_t n, int64_t* new_beg, int32_t* new_adj, int64_t* n_ins,
                       int64_t* n_del) {
    KeyPos* kp = (KeyPos*)malloc(sizeof(KeyPos) * (size_t)(n > 0 ? n : 1));
    int64_t m = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (u[i] == v[i] || u[i] < 0 || v[i] < 0 || u[i] >= V || v[i] >= V) continue;
        kp[m].key = ((int64_t)u[i] << 32) | (uint32_t)v[i];
        kp[m].pos = i; ++m;
    }
    qsort(kp, (size_t)m, sizeof(KeyPos), cmp_keypos);
    /* last op per key; classify against the current edge set */
    int64_t* add = (int64_t*)malloc(sizeof(int64_t) * (size_t)(m > 0 ? m : 1));
    int64_t* del = (int64_t*)malloc(sizeof(int64_t) * (size_t)(m > 0 ? m : 1));
    int64_t na = 0, nd = 0;
    for (int64_t i = 0; i < m; ++i) {
        if (i + 1 < m && kp[i + 1].key == kp[i].key) continue;
        int32_t a = (int32_t)(kp[i].key >> 32), b = (int32_t)(kp[i].key & 0xffffffff);
        int present = has_edge(beg, adj, a, b), want = ins[kp[i].pos] != 0;
        if (want && !present) add[na++] = kp[i].key;
        else if (!want && present) del[nd++] = kp[i].key;
    }
    /* merge: rows of the old CSR minus del plus add (both sorted by key) */
    int64_t ia = 0, id = 0, w = 0;
    for (int64_t x = 0; x < V; ++x) {
        new_beg[x] = w;
        int64_t i = beg[x];
        while (i < beg[x + 1] || (ia < na && (add[ia] >> 32) == x)) {
            int32_t cand_old = i < beg[x + 1] ? adj[i] : INT32_MAX;
            int32_t cand_add = (ia < na && (add[ia] >> 32) == x) ? (int32_t)(add[ia] & 0xffffffff) : INT32_MAX;
            if (cand_add < cand_old) { new_adj[w++] = cand_add; ++ia; continue; }
            while (id < nd && del[id] < (((int64_t)x << 32) | (uint32_t)cand_old)) ++id;
            if (id < nd && del[id] == (((int64_t)x << 32) | (uint32_t)cand_old)) { ++id; ++i; continue; }
            new_adj[w++] = cand_old; ++i;
        }
    }
    new_beg[V] = w;
    *n_ins = na; *n_del = nd;
    free(kp); free(add); free(del);
    return w;
}

/* Transpose of a CSR (rows of the result sorted): the backward CSR of a forward one. */
void or_transpose(int64_t V, const int64_t* beg, const int32_t* adj, int64_t* tb, int32_t* ta) {
    for (int64_t x = 0; x <= V; ++x) tb[x] = 0;
    for (int64_t i = 0; i < beg[V]; ++i) tb[adj[i] + 1]++;
    for (int64_t x = 0; x < V; ++x) tb[x + 1] += tb[x];
    int64_t* pos = (int64_t*)malloc(sizeof(int64_t) * (size_t)(V + 1));
    memcpy(pos, tb, sizeof(int64_t) * (size_t)(V + 1));
    for (int64_t u = 0; u < V; ++u)
        for (int64_t i = beg[u]; i < beg[u + 1]; ++i) ta[pos[adj[i]]++] = (int32_t)u;
    free(pos);
}
