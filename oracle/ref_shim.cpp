// extern "C" access to the reference GIR class -- TEST INFRASTRUCTURE ONLY.
//
// oracle/Makefile compiles this file together with the reference's own, unmodified sources
// (gir_constructor/gir.cpp, gir_query.cpp, graph.cpp, graph_undirected.cpp) into
// oracle/_ref/libgirref.so. Tests use it to pin the C restatement (oracle/gir_oracle.c) and
// to make golden vectors; bench.py's reference arm times the reference's own bfs / sssp /
// applyBatch through it. Every call goes to the reference's public API (gir_constructor/gir.h).
#include <cstdint>
#include <cstring>
#include <vector>

#include "block_cut_tree.h"
#include "gir.h"
#include "graph.h"

extern "C" {

// GIR(graph*) (gir.h:95) over an in-memory four-array CSR, like graph::fromEdges does.
void* ref_create(int32_t V, int64_t E, const int32_t* fwb, const int32_t* fwa, const int32_t* bwb,
                 const int32_t* bwa) {
    graph* g = new graph();
    g->vert_count = V;
    g->edge_count = (index_t)E;
    g->fw_beg_pos = new index_t[V + 1];
    g->bw_beg_pos = new index_t[V + 1];
    g->fw_csr = new vertex_t[E > 0 ? E : 1];
    g->bw_csr = new vertex_t[E > 0 ? E : 1];
    std::memcpy(g->fw_beg_pos, fwb, sizeof(int32_t) * (V + 1));
    std::memcpy(g->bw_beg_pos, bwb, sizeof(int32_t) * (V + 1));
    if (E) std::memcpy(g->fw_csr, fwa, sizeof(int32_t) * E);
    if (E) std::memcpy(g->bw_csr, bwa, sizeof(int32_t) * E);
    return new GIR(g);
}

// GIR(dir, und_dir) (gir.h:93): the four-file loader. (Malformed files end the process, as
// the reference does; tests only hand it valid files.)
void* ref_load(const char* dir) { return new GIR(std::string(dir), std::string(dir)); }

void ref_destroy(void* h) { delete static_cast<GIR*>(h); }

void ref_build(void* h, int mask) {
    GIR* g = static_cast<GIR*>(h);
    if (mask & 1) g->buildWCC();
    if (mask & 2) g->buildSCC_DAG();
    if (mask & 4) g->buildBCT();
}

int32_t ref_vertex_count(void* h) { return static_cast<GIR*>(h)->vertexCount(); }

// Current directed edge set as a forward CSR (getDirectedOutNeighbors per vertex).
int64_t ref_out_csr(void* h, int64_t* beg, int32_t* adj) {
    GIR* g = static_cast<GIR*>(h);
    int64_t w = 0;
    for (int v = 0; v < g->vertexCount(); ++v) {
        auto nb = g->getDirectedOutNeighbors(v);
        if (beg) beg[v] = w;
        for (int x : nb) { if (adj) adj[w] = x; ++w; }
    }
    if (beg) beg[g->vertexCount()] = w;
    return w;
}

// Undirected view (getUndirectedNeighborsPublic) as a CSR.
int64_t ref_und_csr(void* h, int64_t* beg, int32_t* adj) {
    GIR* g = static_cast<GIR*>(h);
    int64_t w = 0;
    for (int v = 0; v < g->vertexCount(); ++v) {
        auto nb = g->getUndirectedNeighborsPublic(v);
        if (beg) beg[v] = w;
        for (int x : nb) { if (adj) adj[w] = x; ++w; }
    }
    if (beg) beg[g->vertexCount()] = w;
    return w;
}

void ref_bfs(void* h, int32_t src, int32_t* level) {
    auto r = static_cast<GIR*>(h)->bfs(src);
    std::memcpy(level, r.data(), sizeof(int32_t) * r.size());
}

void ref_sssp(void* h, int32_t src, uint64_t delta, uint64_t* dist) {
    auto r = static_cast<GIR*>(h)->sssp(src, delta);
    std::memcpy(dist, r.data(), sizeof(uint64_t) * r.size());
}

// GIR::bfsTwoLevel / ssspTwoLevel (gir_query.cpp:604-620, 705-722): the DAG wavefront with block
// tasks inside the source SCC; same results as bfs / sssp.
void ref_bfs_two_level(void* h, int32_t src, int32_t* level) {
    auto r = static_cast<GIR*>(h)->bfsTwoLevel(src);
    std::memcpy(level, r.data(), sizeof(int32_t) * r.size());
}

void ref_sssp_two_level(void* h, int32_t src, uint64_t delta, uint64_t* dist) {
    auto r = static_cast<GIR*>(h)->ssspTwoLevel(src, delta);
    std::memcpy(dist, r.data(), sizeof(uint64_t) * r.size());
}

uint32_t ref_edge_weight(int32_t u, int32_t v) { return GIR::edgeWeight(u, v); }

void ref_apply_batch(void* h, const int32_t* u, const int32_t* v, const uint8_t* ins, int64_t n) {
    std::vector<GIR::Update> b(n);
    for (int64_t i = 0; i < n; ++i) b[i] = {u[i], v[i], ins[i] != 0};
    static_cast<GIR*>(h)->applyBatch(b);
}

// GIR::ingestBatch (gir.cpp:3588-3596): the edge store and the incremental logs only; the layers
// wait for sync().
void ref_ingest_batch(void* h, const int32_t* u, const int32_t* v, const uint8_t* ins, int64_t n) {
    std::vector<GIR::Update> b(n);
    for (int64_t i = 0; i < n; ++i) b[i] = {u[i], v[i], ins[i] != 0};
    static_cast<GIR*>(h)->ingestBatch(b);
}

// GIR::sync / synced (gir.h:115-116).
void ref_sync(void* h) { static_cast<GIR*>(h)->sync(); }
int ref_synced(void* h) { return static_cast<GIR*>(h)->synced() ? 1 : 0; }

void ref_update_edge(void* h, int32_t u, int32_t v, int insert, int undirected) {
    GIR* g = static_cast<GIR*>(h);
    if (undirected) g->updateEdgeUndirected(u, v, insert != 0);
    else g->updateEdgeDirected(u, v, insert != 0);
}

void ref_scc_raw(void* h, int32_t* out) {
    auto m = static_cast<GIR*>(h)->getNodeToScc();
    for (auto& kv : m) out[kv.first] = kv.second;
}

void ref_wcc_raw(void* h, int32_t* out) {
    auto m = static_cast<GIR*>(h)->getNodeToWcc();
    for (auto& kv : m) out[kv.first] = kv.second;
}

// getDAG (gir.h:145) flattened to (row, target) pairs in raw SCC ids.
int64_t ref_dag_raw(void* h, int32_t* a, int32_t* b) {
    auto d = static_cast<GIR*>(h)->getDAG();
    int64_t n = 0;
    for (size_t s = 0; s < d.size(); ++s)
        for (int t : d[s]) { if (a) { a[n] = (int32_t)s; b[n] = t; } ++n; }
    return n;
}

// getBCTComponents (gir.h:148) of every live SCC, flattened: block k has vertices
// verts[beg[k] .. beg[k+1]).
int64_t ref_blocks(void* h, int64_t* beg, int32_t* verts, int64_t* n_blocks) {
    GIR* g = static_cast<GIR*>(h);
    const auto& sccs = g->getSCCs();
    int64_t w = 0, k = 0;
    for (size_t s = 0; s < sccs.size(); ++s) {
        if (sccs[s].empty()) continue;
        for (auto& blk : g->getBCTComponents((int)s)) {
            if (beg) beg[k] = w;
            for (int x : blk) { if (verts) verts[w] = x; ++w; }
            ++k;
        }
    }
    if (beg) beg[k] = w;
    *n_blocks = k;
    return w;
}

void ref_ap(void* h, uint8_t* out) {
    GIR* g = static_cast<GIR*>(h);
    for (int v = 0; v < g->vertexCount(); ++v) out[v] = g->isArticulationPoint(v) ? 1 : 0;
}

// BlockCutTree (block_cut_tree.h:31) of one SCC: node count and edge count.
void ref_bct_shape(void* h, int32_t scc, int64_t* nodes, int64_t* edges) {
    BlockCutTree* t = static_cast<GIR*>(h)->getBCT(scc);
    int64_t e = 0;
    for (auto& n : t->nodes) e += (int64_t)n.neighbors.size();
    *nodes = (int64_t)t->nodes.size();
    *edges = e / 2;
    delete t;
}

// GIR::reachable (gir_query.cpp:789-825) for every (u[i], v[i]).
void ref_reachable(void* h, const int32_t* u, const int32_t* v, int64_t n, uint8_t* out) {
    GIR* g = static_cast<GIR*>(h);
    for (int64_t i = 0; i < n; ++i) out[i] = g->reachable(u[i], v[i]) ? 1 : 0;
}

// GIR::bc (gir_query.cpp:728-778) into score[V].
void ref_bc(void* h, const int32_t* src, int64_t n, double* score) {
    GIR* g = static_cast<GIR*>(h);
    auto r = g->bc(std::vector<int>(src, src + n));
    for (int v = 0; v < g->vertexCount(); ++v) score[v] = r[v];
}

// GIR::trackIncremental / updateIncremental (gir_query.cpp:867-996) and GIR::incDist (gir.h:229-232)
// for every vertex into dist[V].
void ref_inc_track(void* h, int32_t src, int weighted) { static_cast<GIR*>(h)->trackIncremental(src, weighted != 0); }

void ref_inc_update(void* h, int weighted) { static_cast<GIR*>(h)->updateIncremental(weighted != 0); }

void ref_inc_dist(void* h, int weighted, uint64_t* dist) {
    GIR* g = static_cast<GIR*>(h);
    for (int v = 0; v < g->vertexCount(); ++v) dist[v] = g->incDist(weighted != 0, v);
}

}  // extern "C"
