// A C++ caller of the GIR class, written the way the reference's drivers use it
// (gir_constructor/main.cpp:29-52, gir_test.cpp:704-753): load the four-file CSR, build the three
// layers, run the targeted Case 1 / 5c / 5b updates and a BFS / SSSP, and print what it sees.
// tests/test_gpu_cpp_class.py compiles it against include/gir_b200.hpp and libgir_b200.so.
#include <cstdio>
#include <memory>
#include <string>
#include <vector>

#include "gir_b200.hpp"

using GIR = gir_b200::GIR;

static int count_nonempty(const std::vector<std::vector<int>>& parts) {
    int n = 0;
    for (auto& p : parts) n += !p.empty();
    return n;
}

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <dir/>\n", argv[0]);
        return 2;
    }
    try {
        GIR g(argv[1], argv[1]);
        g.buildWCC();
        g.buildSCC_DAG();
        g.buildBCT();
        std::printf("V %d\n", g.vertexCount());
        std::printf("wcc %d scc %d\n", (int)g.getWCCs().size(), count_nonempty(g.getSCCs()));
        const int w0 = (int)g.getWCCs().size();
        g.insertEdge(3, 12);  // Case 1: joins two WCCs
        std::printf("case1 %d\n", (int)g.getWCCs().size() == w0 - 1);
        g.deleteEdge(3, 12);  // Case 5c: splits them again
        std::printf("case5c %d\n", (int)g.getWCCs().size() == w0);
        auto before = g.getNodeToScc();
        g.updateEdgeUndirected(9, 2, false);  // Case 5b: splits {0,1,2,9,10,11}
        auto after = g.getNodeToScc();
        std::printf("case5b %d\n", before[0] == before[9] && after[0] != after[9] && after[0] == after[1] &&
                                       after[9] == after[10]);
        auto comps = g.getBCTComponents(g.sccOf(0));
        std::printf("blocks_of_scc0 %d\n", (int)comps.size());
        std::unique_ptr<gir_b200::BlockCutTree> t(g.getBCT(g.sccOf(0)));
        std::printf("bct_nodes %d\n", (int)t->nodes.size());
        auto lv = g.bfs(0);
        auto d = g.sssp(0);
        std::printf("bfs_0_9 %d sssp_0_1 %llu w01 %u\n", lv[9], (unsigned long long)d[1], GIR::edgeWeight(0, 1));
        std::printf("dag_rows_with_edges %d\n", count_nonempty(g.getDAG()));
        std::printf("has %d %d %d\n", g.hasDirectedEdge(2, 9), g.hasDirectedEdge(9, 2), g.hasUndirectedEdge(9, 2));
        bool reach_ok = true;
        for (int v = 0; v < (int)lv.size(); ++v) reach_ok = reach_ok && (g.reachable(0, v) == (lv[v] >= 0));
        std::printf("reach_matches_bfs %d\n", (int)reach_ok);
        // incremental BFS / SSSP from vertex 0 (gir_test.cpp:1043-1083): cut 0's first out-edge,
        // add one, update, and compare with from-scratch results
        g.trackIncremental(0, false);
        g.trackIncremental(0, true);
        const auto out0 = g.getDirectedOutNeighbors(0);
        if (!out0.empty()) g.deleteEdge(0, out0[0]);
        g.insertEdge(g.vertexCount() - 1, 1);
        g.updateIncremental(false);
        g.updateIncremental(true);
        const auto lv2 = g.bfs(0);
        const auto d2 = g.sssp(0);
        bool inc_ok = true;
        for (int v = 0; v < (int)lv2.size(); ++v)
            inc_ok = inc_ok && g.incDist(false, v) == (lv2[v] < 0 ? UINT64_MAX : (uint64_t)lv2[v]) &&
                     g.incDist(true, v) == d2[v];
        std::printf("inc_matches_scratch %d\n", (int)inc_ok);
        // query results are QueryVec (gir.h:32-37) and compare with plain vectors
        gir_b200::QueryVec<int> q = g.bfs(0);
        std::vector<int> plain(q.begin(), q.end());
        std::printf("queryvec %d\n", (int)(q == plain && !(q != plain) && g.bfsTwoLevel(0) == plain));
        bool nidx = true;
        for (int v = 0; v < g.vertexCount(); ++v) nidx = nidx && g.reachableNoIndex(0, v) == g.reachable(0, v);
        std::printf("reach_noindex %d\n", (int)nidx);
        std::string why;
        std::printf("forest_ok %d\n", (int)g.checkBlockForestInvariants(&why));
        std::printf("bicon_self %d\n", (int)g.biconnected(5, 5));
        const auto bcv = g.bc({0, 1, 2});
        bool bc_ok = (int)bcv.size() == g.vertexCount();
        for (double x : bcv) bc_ok = bc_ok && x >= 0;
        std::printf("bc_ok %d\n", (int)bc_ok);
        // deferred maintenance (gir.h:107-116): ingestBatch changes the edge store now, the layers
        // at sync(); BFS sees the change at once
        const int w_before = (int)g.getWCCs().size();
        const int joins = g.wccOf(3) != g.wccOf(12);
        g.ingestBatch({{3, 12, true}});
        const int pending = !g.synced();
        const int w_pending = (int)g.getWCCs().size();
        const int bfs_sees = g.bfs(3)[12] == 1;
        g.sync();
        std::printf("ingest %d %d %d %d\n", pending, (int)(w_pending == w_before), bfs_sees,
                    (int)((int)g.getWCCs().size() == w_before - joins && g.synced()));
        // GIR(graph*): the reference's loader type, from graph::fromEdges and from the four files
        GIR h(gir_b200::graph::fromEdges(4, {{0, 1}, {1, 2}, {2, 0}, {2, 3}}));
        h.buildWCC();
        h.buildSCC_DAG();
        h.buildBCT();
        const std::string dir = argv[1];
        GIR f(new gir_b200::graph((dir + "fw_begin.bin").c_str(), (dir + "fw_adjacent.bin").c_str(),
                                  (dir + "bw_begin.bin").c_str(), (dir + "bw_adjacent.bin").c_str()));
        std::printf("from_graph %d %d %d\n", h.vertexCount(), count_nonempty(h.getSCCs()), f.vertexCount());
        try {
            GIR bad("/nonexistent/dir/", "/nonexistent/dir/");
            std::printf("error_missing 0\n");
        } catch (const gir_b200::Error& e) {
            std::printf("error_missing %d\n", e.code() == GIR_ERR_FILE);
        }
    } catch (const gir_b200::Error& e) {
        std::fprintf(stderr, "error %d: %s\n", e.code(), e.what());
        return 1;
    }
    return 0;
}
