// GIR-B200: the reference's GIR class surface (gir_constructor/gir.h:72-240) in C++, on the GPU.
//
// A drop-in for the hot path of GIR: the same method names, argument meanings and call order
// (buildWCC, then buildSCC_DAG, then buildBCT, gir.h:98). Every method forwards to the
// gir_dev_* C ABI (gir_dev.h); all computation runs in libgir_b200.so on the GPU.
//
// Differences a caller can see:
//  - component ids are canonical: an SCC or WCC is named by its smallest vertex (the reference
//    uses Tarjan emission order and union-find roots, gir.cpp:646-653, 809-816); getSCCs() has a
//    slot per vertex id, empty unless the id is an SCC's smallest vertex (the reference's list
//    also has empty slots, for retired ids);
//  - single-edge updates run as one-edge batches (same layers as the reference's
//    Scope-Prune-Update path, gir.cpp:3043-3131);
//  - malformed input throws gir_b200::Error with the GIR_ERR_* code, where the reference exits
//    (graph.cpp:95-114, gir.cpp:122-126).
#pragma once

#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <unordered_set>
#include <vector>

#include "gir_dev.h"

namespace gir_b200 {

class Error : public std::runtime_error {
public:
    Error(int code, const std::string& msg) : std::runtime_error(msg), code_(code) {}
    int code() const { return code_; }

private:
    int code_;
};

// block_cut_tree.h:15-81: B-nodes (blocks) and C-nodes (articulation points) of one SCC.
struct BlockCutTree {
    enum NodeType { B_NODE, C_NODE };
    struct Node {
        NodeType type;
        int id;  // B-node: block index; C-node: vertex id
        std::vector<int> neighbors;
    };
    std::vector<Node> nodes;
    void build(const std::vector<std::vector<int>>& blocks, const std::unordered_set<int>& aps);
};

class GIR {
public:
    struct Update {
        int u, v;
        bool insert;
    };
    static const uint32_t kMaxWeight = 100;

    // GIR(path_directed, path_undirected) (gir.h:93): the four-file CSR loader.
    GIR(const std::string& path_directed, const std::string& path_undirected);
    // GIR(graph*) (gir.h:95) / graph::fromEdges (graph.cpp:123-136): an in-memory int32 CSR
    // (forward + backward, V + 1 offsets each), optionally with uint32 forward weights.
    GIR(int V, const std::vector<int>& fw_beg, const std::vector<int>& fw_adj, const std::vector<int>& bw_beg,
        const std::vector<int>& bw_adj, const std::vector<uint32_t>* weights = nullptr);
    static GIR fromEdges(int V, const std::vector<std::pair<int, int>>& edges);
    GIR(GIR&& o) noexcept;
    GIR& operator=(GIR&& o) noexcept;
    GIR(const GIR&) = delete;
    GIR& operator=(const GIR&) = delete;
    ~GIR();

    // construction (gir.h:98-101)
    void buildWCC();
    void buildSCC_DAG();
    void buildBCT();

    // updates (gir.h:104-119)
    void insertEdge(int u, int v);
    void deleteEdge(int u, int v);
    void applyBatch(const std::vector<Update>& batch);
    void ingestBatch(const std::vector<Update>& batch) { applyBatch(batch); }
    void sync() {}
    bool synced() const { return true; }
    void updateEdgeDirected(int u, int v, bool insert);
    void updateEdgeUndirected(int u, int v, bool insert);  // routed as directed, as gir.cpp:3134 does

    // cheap per-vertex queries (gir.h:122-125)
    int sccOf(int v) const;
    int wccOf(int v) const;
    long long sccRank(int s) const;
    bool isArticulationPoint(int v) const;
    bool sameScc(int u, int v) const { return sccOf(u) == sccOf(v); }
    bool sameWcc(int u, int v) const { return wccOf(u) == wccOf(v); }
    bool articulationPoint(int v) const { return isArticulationPoint(v); }
    int vertexCount() const { return V_; }

    // materialized views (gir.h:142-153)
    std::map<int, int> getNodeToScc() const;
    std::map<int, int> getNodeToWcc() const;
    std::vector<std::vector<int>> getSCCs() const;
    std::vector<std::vector<int>> getDAG() const;
    std::vector<std::vector<int>> getWCCs() const;
    std::vector<std::vector<int>> getBCTComponents(int scc_id) const;
    BlockCutTree* getBCT(int scc_id) const;  // caller owns

    // edge store (gir.h:160-164)
    std::vector<int> getDirectedOutNeighbors(int v) const;
    std::vector<int> getDirectedInNeighbors(int v) const;
    std::vector<int> getUndirectedNeighborsPublic(int v) const;
    bool hasDirectedEdge(int u, int v) const;
    bool hasUndirectedEdge(int u, int v) const;

    // queries (gir.h:204-216)
    std::vector<int> bfs(int source);
    std::vector<uint64_t> sssp(int source, uint64_t delta = 16);
    // gir.h:128-130: u ~> v (needs buildSCC_DAG); reachableMany answers a batch of pairs.
    bool reachable(int u, int v);
    std::vector<uint8_t> reachableMany(const std::vector<int>& u, const std::vector<int>& v);
    static uint32_t edgeWeight(int u, int v);
    // gir.h:220-232 (gir_query.cpp:867-996): incremental single-source BFS (weighted false) /
    // SSSP (true). incDist reads a host copy of the tracked result, taken after each track or
    // update (the result changes only there).
    void trackIncremental(int source, bool weighted);
    void updateIncremental(bool weighted);
    uint64_t incDist(bool weighted, int v) const;
    // batched forms: one row of V per source
    std::vector<int> bfsMany(const std::vector<int>& sources);
    std::vector<uint64_t> ssspMany(const std::vector<int>& sources, uint64_t delta = 16);

    gir_dev_t* handle() const { return h_; }

private:
    explicit GIR(gir_dev_t* h);
    void check(int rc, const char* what) const;
    std::vector<int32_t> labels(int which) const;
    std::vector<int> row(int dir, int v) const;

    gir_dev_t* h_ = nullptr;
    int V_ = 0;
    mutable std::vector<uint64_t> inc_[2];  // host copies of the tracked results (empty = stale)
};

}  // namespace gir_b200
