// The C++ GIR class (include/gir_b200.hpp) over the gir_dev_* C ABI.
#include "gir_b200.hpp"

#include <algorithm>
#include <cstdio>
#include <utility>

namespace gir_b200 {

void BlockCutTree::build(const std::vector<std::vector<int>>& blocks, const std::unordered_set<int>& aps) {
    // block_cut_tree.h:31-58: C-nodes first, then one B-node per block linked to its APs
    nodes.clear();
    std::map<int, int> ap_node;
    std::vector<int> ap_sorted(aps.begin(), aps.end());
    std::sort(ap_sorted.begin(), ap_sorted.end());
    for (int v : ap_sorted) {
        ap_node[v] = (int)nodes.size();
        nodes.push_back({C_NODE, v, {}});
    }
    for (size_t i = 0; i < blocks.size(); ++i) {
        const int b = (int)nodes.size();
        nodes.push_back({B_NODE, (int)i, {}});
        for (int x : blocks[i]) {
            auto it = ap_node.find(x);
            if (it == ap_node.end()) continue;
            nodes[b].neighbors.push_back(it->second);
            nodes[it->second].neighbors.push_back(b);
        }
    }
}

void GIR::check(int rc, const char* what) const {
    if (rc != GIR_OK) throw Error(rc, std::string(what) + ": " + gir_dev_last_error(h_));
}

GIR::GIR(gir_dev_t* h) : h_(h) {
    int64_t V = 0;
    check(gir_dev_counts(h_, &V, nullptr, nullptr, nullptr, nullptr, nullptr), "gir_dev_counts");
    V_ = (int)V;
}

GIR::GIR(const std::string& path_directed, const std::string& /*path_undirected: never read, gir.h:156-158*/) {
    gir_dev_t* h = nullptr;
    const int rc = gir_dev_load(path_directed.c_str(), &h);
    if (rc != GIR_OK) throw Error(rc, std::string("gir_dev_load: ") + gir_dev_last_error(nullptr));
    h_ = h;
    int64_t V = 0;
    check(gir_dev_counts(h_, &V, nullptr, nullptr, nullptr, nullptr, nullptr), "gir_dev_counts");
    V_ = (int)V;
}

GIR::GIR(int V, const std::vector<int>& fw_beg, const std::vector<int>& fw_adj, const std::vector<int>& bw_beg,
         const std::vector<int>& bw_adj, const std::vector<uint32_t>* weights) {
    if ((int)fw_beg.size() != V + 1 || (int)bw_beg.size() != V + 1 || fw_adj.size() != bw_adj.size() ||
        (weights && weights->size() != fw_adj.size()))
        throw Error(GIR_ERR_INVALID, "GIR: CSR arrays of inconsistent sizes");
    gir_dev_t* h = nullptr;
    const int rc = gir_dev_create(fw_beg.data(), fw_adj.data(), bw_beg.data(), bw_adj.data(), V,
                                  (int64_t)fw_adj.size(), weights ? weights->data() : nullptr, &h);
    if (rc != GIR_OK) throw Error(rc, std::string("gir_dev_create: ") + gir_dev_last_error(nullptr));
    h_ = h;
    V_ = V;
}

GIR GIR::fromEdges(int V, const std::vector<std::pair<int, int>>& edges) {
    std::vector<int> fb(V + 1, 0), bb(V + 1, 0), fa(edges.size()), ba(edges.size());
    for (auto& e : edges) { fb[e.first + 1]++; bb[e.second + 1]++; }
    for (int v = 0; v < V; ++v) { fb[v + 1] += fb[v]; bb[v + 1] += bb[v]; }
    std::vector<int> fp(fb.begin(), fb.end() - 1), bp(bb.begin(), bb.end() - 1);
    for (auto& e : edges) { fa[fp[e.first]++] = e.second; ba[bp[e.second]++] = e.first; }
    return GIR(V, fb, fa, bb, ba);
}

graph::graph(const char* fw_beg_file, const char* fw_csr_file, const char* bw_beg_file, const char* bw_csr_file) {
    auto read_all = [](const char* path, std::vector<int32_t>& out) {
        FILE* f = std::fopen(path, "rb");
        if (!f) throw Error(GIR_ERR_FILE, std::string(path) + " cannot open");
        std::fseek(f, 0, SEEK_END);
        const long bytes = std::ftell(f);
        std::fseek(f, 0, SEEK_SET);
        if (bytes < 0 || bytes % 4) {
            std::fclose(f);
            throw Error(GIR_ERR_FILE, std::string(path) + " is not an int32 array");
        }
        out.resize((size_t)bytes / 4);
        const size_t got = out.empty() ? 0 : std::fread(out.data(), 4, out.size(), f);
        std::fclose(f);
        if (got != out.size()) throw Error(GIR_ERR_FILE, std::string(path) + " is short");
    };
    std::vector<int32_t> fb, fa, bb, ba;
    read_all(fw_beg_file, fb);
    read_all(fw_csr_file, fa);
    read_all(bw_beg_file, bb);
    read_all(bw_csr_file, ba);
    // graph.cpp:95-114: sizes agree, offsets monotone from 0 to E, ids in [0, V)
    if (fb.empty() || fb.size() != bb.size() || fa.size() != ba.size())
        throw Error(GIR_ERR_MALFORMED, "graph: four-file sizes disagree");
    const int64_t V = (int64_t)fb.size() - 1, E = (int64_t)fa.size();
    auto ok = [&](const std::vector<int32_t>& beg, const std::vector<int32_t>& adj) {
        if (beg[0] != 0 || beg[V] != E) return false;
        for (int64_t i = 0; i < V; ++i)
            if (beg[i] > beg[i + 1]) return false;
        for (int32_t x : adj)
            if (x < 0 || x >= V) return false;
        return true;
    };
    if (!ok(fb, fa) || !ok(bb, ba)) throw Error(GIR_ERR_MALFORMED, "graph: malformed CSR");
    vert_count = (index_t)V;
    edge_count = (index_t)E;
    fw_beg_pos = new index_t[V + 1];
    bw_beg_pos = new index_t[V + 1];
    fw_csr = new vertex_t[E > 0 ? E : 1];
    bw_csr = new vertex_t[E > 0 ? E : 1];
    std::copy(fb.begin(), fb.end(), fw_beg_pos);
    std::copy(bb.begin(), bb.end(), bw_beg_pos);
    std::copy(fa.begin(), fa.end(), fw_csr);
    std::copy(ba.begin(), ba.end(), bw_csr);
}

graph::~graph() {
    delete[] fw_beg_pos;
    delete[] fw_csr;
    delete[] bw_beg_pos;
    delete[] bw_csr;
}

graph* graph::fromEdges(index_t V, const std::vector<std::pair<int, int>>& edges) {
    auto* g = new graph();
    const int64_t E = (int64_t)edges.size();
    g->vert_count = V;
    g->edge_count = (index_t)E;
    g->fw_beg_pos = new index_t[V + 1]();
    g->bw_beg_pos = new index_t[V + 1]();
    g->fw_csr = new vertex_t[E > 0 ? E : 1];
    g->bw_csr = new vertex_t[E > 0 ? E : 1];
    for (auto& e : edges) {
        g->fw_beg_pos[e.first + 1]++;
        g->bw_beg_pos[e.second + 1]++;
    }
    for (int v = 0; v < V; ++v) {
        g->fw_beg_pos[v + 1] += g->fw_beg_pos[v];
        g->bw_beg_pos[v + 1] += g->bw_beg_pos[v];
    }
    std::vector<index_t> fp(g->fw_beg_pos, g->fw_beg_pos + V), bp(g->bw_beg_pos, g->bw_beg_pos + V);
    for (auto& e : edges) {
        g->fw_csr[fp[e.first]++] = e.second;
        g->bw_csr[bp[e.second]++] = e.first;
    }
    return g;
}

GIR::GIR(graph* g) {
    if (!g) throw Error(GIR_ERR_INVALID, "GIR(graph*): null graph");
    std::unique_ptr<graph> own(g);
    gir_dev_t* h = nullptr;
    const int rc = gir_dev_create(g->fw_beg_pos, g->fw_csr, g->bw_beg_pos, g->bw_csr, g->vert_count, g->edge_count,
                                  nullptr, &h);
    if (rc != GIR_OK) throw Error(rc, std::string("gir_dev_create: ") + gir_dev_last_error(nullptr));
    h_ = h;
    V_ = g->vert_count;
}

GIR::GIR(GIR&& o) noexcept : h_(o.h_), V_(o.V_) { o.h_ = nullptr; }
GIR& GIR::operator=(GIR&& o) noexcept {
    if (this != &o) {
        gir_dev_destroy(h_);
        h_ = o.h_;
        V_ = o.V_;
        o.h_ = nullptr;
    }
    return *this;
}
GIR::~GIR() { gir_dev_destroy(h_); }

void GIR::buildWCC() { check(gir_dev_build(h_, GIR_LAYER_WCC), "buildWCC"); }
void GIR::buildSCC_DAG() { check(gir_dev_build(h_, GIR_LAYER_SCC), "buildSCC_DAG"); }
void GIR::buildBCT() { check(gir_dev_build(h_, GIR_LAYER_BCT), "buildBCT"); }

void GIR::applyBatch(const std::vector<Update>& batch) {
    std::vector<int32_t> u(batch.size()), v(batch.size());
    std::vector<uint8_t> ins(batch.size());
    for (size_t i = 0; i < batch.size(); ++i) {
        u[i] = batch[i].u;
        v[i] = batch[i].v;
        ins[i] = batch[i].insert ? 1 : 0;
    }
    check(gir_dev_apply_batch(h_, u.data(), v.data(), ins.data(), (int64_t)batch.size()), "applyBatch");
}
void GIR::ingestBatch(const std::vector<Update>& batch) {
    std::vector<int32_t> u(batch.size()), v(batch.size());
    std::vector<uint8_t> ins(batch.size());
    for (size_t i = 0; i < batch.size(); ++i) {
        u[i] = batch[i].u;
        v[i] = batch[i].v;
        ins[i] = batch[i].insert ? 1 : 0;
    }
    check(gir_dev_ingest_batch(h_, u.data(), v.data(), ins.data(), (int64_t)batch.size()), "ingestBatch");
}
void GIR::sync() { check(gir_dev_sync(h_), "sync"); }
bool GIR::synced() const {
    int s = 1;
    check(gir_dev_synced(h_, &s), "synced");
    return s != 0;
}
void GIR::insertEdge(int u, int v) { applyBatch({{u, v, true}}); }
void GIR::deleteEdge(int u, int v) { applyBatch({{u, v, false}}); }
void GIR::updateEdgeDirected(int u, int v, bool insert) { applyBatch({{u, v, insert}}); }
void GIR::updateEdgeUndirected(int u, int v, bool insert) { applyBatch({{u, v, insert}}); }

std::vector<int32_t> GIR::labels(int which) const {
    std::vector<int32_t> out((size_t)V_);
    check(gir_dev_get_labels(h_, which, out.data()), "get_labels");
    return out;
}

int GIR::sccOf(int v) const { return labels(GIR_LABEL_SCC).at((size_t)v); }
int GIR::wccOf(int v) const { return labels(GIR_LABEL_WCC).at((size_t)v); }
long long GIR::sccRank(int s) const { return labels(GIR_LABEL_SCC_RANK).at((size_t)s); }
bool GIR::isArticulationPoint(int v) const { return labels(GIR_LABEL_BCNT).at((size_t)v) >= 2; }

std::map<int, int> GIR::getNodeToScc() const {
    const auto l = labels(GIR_LABEL_SCC);
    std::map<int, int> m;
    for (int v = 0; v < V_; ++v) m.emplace_hint(m.end(), v, l[v]);
    return m;
}
std::map<int, int> GIR::getNodeToWcc() const {
    const auto l = labels(GIR_LABEL_WCC);
    std::map<int, int> m;
    for (int v = 0; v < V_; ++v) m.emplace_hint(m.end(), v, l[v]);
    return m;
}
std::vector<std::vector<int>> GIR::getSCCs() const {
    const auto l = labels(GIR_LABEL_SCC);
    std::vector<std::vector<int>> r((size_t)V_);
    for (int v = 0; v < V_; ++v) r[l[v]].push_back(v);
    return r;
}
std::vector<std::vector<int>> GIR::getWCCs() const {
    const auto l = labels(GIR_LABEL_WCC);
    std::vector<std::vector<int>> byid((size_t)V_), r;
    for (int v = 0; v < V_; ++v) byid[l[v]].push_back(v);
    for (auto& g : byid) if (!g.empty()) r.push_back(std::move(g));
    return r;
}
std::vector<std::vector<int>> GIR::getDAG() const {
    int64_t n = 0;
    check(gir_dev_get_dag(h_, nullptr, nullptr, 0, &n), "getDAG");
    std::vector<int32_t> a((size_t)n), b((size_t)n);
    if (n) check(gir_dev_get_dag(h_, a.data(), b.data(), n, &n), "getDAG");
    std::vector<std::vector<int>> r((size_t)V_);
    for (int64_t i = 0; i < n; ++i) r[a[i]].push_back(b[i]);
    return r;
}
std::vector<std::vector<int>> GIR::getBCTComponents(int scc_id) const {
    const auto scc = labels(GIR_LABEL_SCC);
    const auto blk = labels(GIR_LABEL_BLOCK);
    int64_t nb = 0;
    check(gir_dev_get_blocks(h_, nullptr, 0, &nb), "getBCTComponents");
    std::vector<int32_t> head((size_t)nb);
    if (nb) check(gir_dev_get_blocks(h_, head.data(), nb, &nb), "getBCTComponents");
    std::map<int, std::vector<int>> by_block;
    for (int v = 0; v < V_; ++v)
        if (scc[v] == scc_id) by_block[blk[v]].push_back(v);
    std::vector<std::vector<int>> r;
    for (auto& kv : by_block) {
        auto members = kv.second;
        if (head[kv.first] >= 0) members.push_back(head[kv.first]);
        std::sort(members.begin(), members.end());
        r.push_back(std::move(members));
    }
    return r;
}
BlockCutTree* GIR::getBCT(int scc_id) const {
    const auto comps = getBCTComponents(scc_id);
    const auto cnt = labels(GIR_LABEL_BCNT);
    std::unordered_set<int> aps;
    for (auto& c : comps)
        for (int x : c)
            if (cnt[x] >= 2) aps.insert(x);
    auto* t = new BlockCutTree();
    t->build(comps, aps);
    return t;
}

std::vector<int> GIR::row(int dir, int v) const {
    if (v < 0 || v >= V_) return {};
    int64_t n = 0;
    check(gir_dev_get_csr(h_, dir, nullptr, nullptr, 0, &n), "get_csr");
    std::vector<int64_t> beg((size_t)V_ + 1);
    std::vector<int32_t> adj((size_t)n);
    check(gir_dev_get_csr(h_, dir, beg.data(), adj.data(), n, &n), "get_csr");
    return std::vector<int>(adj.begin() + beg[v], adj.begin() + beg[v + 1]);
}
std::vector<int> GIR::getDirectedOutNeighbors(int v) const { return row(0, v); }
std::vector<int> GIR::getDirectedInNeighbors(int v) const { return row(1, v); }
std::vector<int> GIR::getUndirectedNeighborsPublic(int v) const { return row(2, v); }

bool GIR::hasDirectedEdge(int u, int v) const {
    uint8_t out = 0;
    check(gir_dev_has_edges(h_, 0, &u, &v, 1, &out), "hasDirectedEdge");
    return out != 0;
}
bool GIR::hasUndirectedEdge(int u, int v) const {
    uint8_t out = 0;
    check(gir_dev_has_edges(h_, 1, &u, &v, 1, &out), "hasUndirectedEdge");
    return out != 0;
}

QueryVec<int> GIR::bfs(int source) {
    QueryVec<int> out((size_t)V_);
    check(gir_dev_bfs(h_, &source, 1, out.data()), "bfs");
    return out;
}
QueryVec<uint64_t> GIR::sssp(int source, uint64_t delta) {
    QueryVec<uint64_t> out((size_t)V_);
    check(gir_dev_sssp(h_, &source, 1, delta, GIR_WEIGHT_HASH, out.data()), "sssp");
    return out;
}
QueryVec<double> GIR::bc(const std::vector<int>& sources) {
    QueryVec<double> out((size_t)V_);
    check(gir_dev_bc(h_, sources.data(), (int64_t)sources.size(), out.data()), "bc");
    return out;
}

bool GIR::reachable(int u, int v) { return reachableMany({u}, {v})[0] != 0; }

bool GIR::reachableNoIndex(int u, int v) {
    if (u < 0 || v < 0 || u >= V_ || v >= V_) return false;
    if (u == v) return true;
    return bfs(u)[(size_t)v] >= 0;
}

bool GIR::biconnected(int u, int v) {
    sync();
    if (u == v) return true;
    if (u < 0 || v < 0 || u >= V_ || v >= V_) return false;
    const auto scc = labels(GIR_LABEL_SCC);
    if (scc[u] != scc[v]) return false;
    const auto blk = labels(GIR_LABEL_BLOCK);
    int64_t nb = 0;
    check(gir_dev_get_blocks(h_, nullptr, 0, &nb), "biconnected");
    std::vector<int32_t> head((size_t)nb);
    if (nb) check(gir_dev_get_blocks(h_, head.data(), nb, &nb), "biconnected");
    // a vertex lies in its own block and in every block it heads
    return blk[u] == blk[v] || head[blk[v]] == u || head[blk[u]] == v;
}

bool GIR::checkBlockForestInvariants(std::string* why) const {
    auto fail = [&](const char* m) {
        if (why) *why = m;
        return false;
    };
    const auto scc = labels(GIR_LABEL_SCC);
    const auto blk = labels(GIR_LABEL_BLOCK);
    const auto cnt = labels(GIR_LABEL_BCNT);
    int64_t nb = 0;
    check(gir_dev_get_blocks(h_, nullptr, 0, &nb), "checkBlockForestInvariants");
    std::vector<int32_t> head((size_t)nb);
    if (nb) check(gir_dev_get_blocks(h_, head.data(), nb, &nb), "checkBlockForestInvariants");
    std::vector<int> members((size_t)nb, 0), headed((size_t)V_, 0), bscc((size_t)nb, -1);
    for (int v = 0; v < V_; ++v) {
        if (blk[v] < 0 || blk[v] >= nb) return fail("a vertex without a valid block");
        ++members[blk[v]];
        if (bscc[blk[v]] == -1) bscc[blk[v]] = scc[v];
        else if (bscc[blk[v]] != scc[v]) return fail("a block spans two SCCs");
    }
    for (int64_t b = 0; b < nb; ++b) {
        if (members[b] == 0) return fail("a block without members");
        if (head[b] >= 0) {
            if (scc[head[b]] != bscc[b]) return fail("a block's head lies in another SCC");
            ++headed[head[b]];
        }
    }
    for (int v = 0; v < V_; ++v)
        if (cnt[v] != 1 + headed[v]) return fail("a block count differs from 1 + the blocks the vertex heads");
    for (int64_t b = 0; b < nb; ++b)
        if (head[b] >= 0 && cnt[head[b]] < 2) return fail("a head that is not an articulation point");
    return true;
}

std::vector<uint8_t> GIR::reachableMany(const std::vector<int>& u, const std::vector<int>& v) {
    if (u.size() != v.size()) throw Error(GIR_ERR_INVALID, "reachable: u and v differ in length");
    std::vector<uint8_t> out(u.size());
    check(gir_dev_reachable(h_, u.data(), v.data(), (int64_t)u.size(), out.data()), "reachable");
    return out;
}

void GIR::trackIncremental(int source, bool weighted) {
    check(gir_dev_inc_track(h_, source, weighted ? 1 : 0), "trackIncremental");
    inc_[weighted].clear();
}

void GIR::updateIncremental(bool weighted) {
    check(gir_dev_inc_update(h_, weighted ? 1 : 0), "updateIncremental");
    inc_[weighted].clear();
}

uint64_t GIR::incDist(bool weighted, int v) const {
    std::vector<uint64_t>& c = inc_[weighted];
    if (c.empty() && V_ > 0) {
        c.resize((size_t)V_);
        check(gir_dev_inc_dist(h_, weighted ? 1 : 0, c.data()), "incDist");
    }
    if (v < 0 || v >= V_) throw Error(GIR_ERR_INVALID, "incDist: vertex out of range");
    return c[(size_t)v];
}

std::vector<int> GIR::bfsMany(const std::vector<int>& sources) {
    std::vector<int> out(sources.size() * (size_t)V_);
    check(gir_dev_bfs(h_, sources.data(), (int64_t)sources.size(), out.data()), "bfs");
    return out;
}
std::vector<uint64_t> GIR::ssspMany(const std::vector<int>& sources, uint64_t delta) {
    std::vector<uint64_t> out(sources.size() * (size_t)V_);
    check(gir_dev_sssp(h_, sources.data(), (int64_t)sources.size(), delta, GIR_WEIGHT_HASH, out.data()), "sssp");
    return out;
}

uint32_t GIR::edgeWeight(int u, int v) {
    // GIR::edgeWeight (gir_query.cpp:50-54); the device kernels compute the same function
    uint64_t x = ((uint64_t)(uint32_t)u << 32) | (uint32_t)v;
    x ^= x >> 33; x *= 0xff51afd7ed558ccdULL; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL; x ^= x >> 33;
    return 1 + (uint32_t)(x % kMaxWeight);
}

}  // namespace gir_b200
