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
//  - bfsTwoLevel / bfsTaskParallel / ssspTwoLevel return the flat device queries' results (the
//    reference's task-parallel formulations compute the same levels and distances);
//  - checkBlockForestInvariants checks the representation's structural rules (every block
//    non-empty and inside one SCC with its head, heads are articulation points, block counts
//    match the heads) and does not re-derive biconnectivity;
//  - malformed input throws gir_b200::Error with the GIR_ERR_* code, where the reference exits
//    (graph.cpp:95-114, gir.cpp:122-126).
#pragma once

#include <algorithm>
#include <cstdint>
#include <map>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <unordered_set>
#include <utility>
#include <vector>

#include "gir_dev.h"

namespace gir_b200 {

// Query results (gir.h:25-37): a std::vector whose allocator leaves elements default-initialized
// when the vector is sized, so a result row of V entries is not zeroed before the library fills
// it. Compares equal with a std::vector of the same contents.
template <class T>
struct DefaultInitAllocator : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = DefaultInitAllocator<U>;
    };
    DefaultInitAllocator() = default;
    template <class U>
    DefaultInitAllocator(const DefaultInitAllocator<U>&) noexcept {}
    template <class U>
    void construct(U* p) noexcept(std::is_nothrow_default_constructible<U>::value) {
        ::new (static_cast<void*>(p)) U;
    }
    template <class U, class... A>
    void construct(U* p, A&&... a) {
        ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
    }
};
template <class T>
using QueryVec = std::vector<T, DefaultInitAllocator<T>>;
template <class T>
bool operator==(const QueryVec<T>& a, const std::vector<T>& b) {
    return a.size() == b.size() && std::equal(a.begin(), a.end(), b.begin());
}
template <class T>
bool operator==(const std::vector<T>& a, const QueryVec<T>& b) { return b == a; }
template <class T>
bool operator!=(const QueryVec<T>& a, const std::vector<T>& b) { return !(a == b); }
template <class T>
bool operator!=(const std::vector<T>& a, const QueryVec<T>& b) { return !(b == a); }

typedef int index_t;   // util.h:17-21
typedef int vertex_t;

// The reference's loader class (graph.h:11-57): the int32 four-array CSR in host memory, read from
// the four .bin files or built from an edge list. GIR(graph*) takes ownership of it.
class graph {
public:
    index_t* fw_beg_pos = nullptr;
    vertex_t* fw_csr = nullptr;
    index_t* bw_beg_pos = nullptr;
    vertex_t* bw_csr = nullptr;
    double* weight = nullptr;  // (unused, as in the reference)
    index_t vert_count = 0;
    index_t edge_count = 0;

    graph() = default;
    // graph.cpp:2-120: reads the four files; a missing, short or malformed file throws Error.
    graph(const char* fw_beg_file, const char* fw_csr_file, const char* bw_beg_file, const char* bw_csr_file);
    ~graph();
    graph(const graph&) = delete;
    graph& operator=(const graph&) = delete;
    // graph.cpp:123-136: forward and backward CSR of an edge list (rows in edge order); caller owns.
    static graph* fromEdges(index_t V, const std::vector<std::pair<int, int>>& edges);
};

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
    // GIR(graph*) (gir.h:95): takes ownership of g (its arrays go to the GPU; g is deleted).
    explicit GIR(graph* g);
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
    // Deferred maintenance (gir.h:107-116): ingestBatch changes the edge store only; the layer
    // getters describe the last sync until sync(); updates and structure-based queries sync first.
    void ingestBatch(const std::vector<Update>& batch);
    void sync();
    bool synced() const;
    void updateEdgeDirected(int u, int v, bool insert);
    void updateEdgeUndirected(int u, int v, bool insert);  // routed as directed, as gir.cpp:3134 does

    // cheap per-vertex queries (gir.h:122-125)
    int sccOf(int v) const;
    int wccOf(int v) const;
    long long sccRank(int s) const;
    bool isArticulationPoint(int v) const;
    // gir.h:131-138: structure-based queries sync first
    bool sameScc(int u, int v) { sync(); return sccOf(u) == sccOf(v); }
    bool sameWcc(int u, int v) { sync(); return wccOf(u) == wccOf(v); }
    bool articulationPoint(int v) { sync(); return isArticulationPoint(v); }
    // u and v share a block of one SCC's undirected view
    bool biconnected(int u, int v);
    int vertexCount() const { return V_; }

    // materialized views (gir.h:142-153)
    std::map<int, int> getNodeToScc() const;
    std::map<int, int> getNodeToWcc() const;
    std::vector<std::vector<int>> getSCCs() const;
    std::vector<std::vector<int>> getDAG() const;
    std::vector<std::vector<int>> getWCCs() const;
    std::vector<std::vector<int>> getBCTComponents(int scc_id) const;
    BlockCutTree* getBCT(int scc_id) const;  // caller owns
    // gir.h:153 (gir.cpp:4159-4211): the block-cut forest's structural rules; *why gets the first
    // broken rule.
    bool checkBlockForestInvariants(std::string* why = nullptr) const;

    // edge store (gir.h:160-164)
    std::vector<int> getDirectedOutNeighbors(int v) const;
    std::vector<int> getDirectedInNeighbors(int v) const;
    std::vector<int> getUndirectedNeighborsPublic(int v) const;
    bool hasDirectedEdge(int u, int v) const;
    bool hasUndirectedEdge(int u, int v) const;

    // queries (gir.h:204-219)
    QueryVec<int> bfs(int source);
    QueryVec<int> bfsTwoLevel(int source) { return bfs(source); }
    QueryVec<int> bfsTaskParallel(int source) { return bfs(source); }
    QueryVec<uint64_t> sssp(int source, uint64_t delta = 16);
    QueryVec<uint64_t> ssspTwoLevel(int source, uint64_t delta = 16) { return sssp(source, delta); }
    // gir.h:219 (gir_query.cpp:728-778): Brandes betweenness summed over the sources
    QueryVec<double> bc(const std::vector<int>& sources);
    // gir.h:128-130: u ~> v (needs buildSCC_DAG); reachableMany answers a batch of pairs.
    bool reachable(int u, int v);
    // gir.h:138: the same answer without the index (a BFS from u on the edge store)
    bool reachableNoIndex(int u, int v);
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
