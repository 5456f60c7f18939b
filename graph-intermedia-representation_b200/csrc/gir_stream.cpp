// gir_stream: the reference's streaming protocol driver (experiments/baselines/gir/gir_stream.cpp,
// DZiG's setting) over the GIR-B200 C++ class, for the GPU.
//
//   gir_stream <protocol dir> <dataset> <csv> [batch=10000] [batches=10] [mode]
//
// The protocol directory holds what the reference's `bench_gir --export` writes
// (experiments/baselines/common/protocol.h:1-10): loaded.el (the initial half of the graph, "u v"
// per line), insert.ops / delete.ops / mixed.ops ("a u v" / "d u v" per line), sources.txt and
// meta.txt ("key value" lines, V among them). For each stream (insert, delete, mixed) the graph is
// loaded fresh with its three layers built; then per batch of `batch` operations the batch is
// applied and BFS / SSSP from the first source recomputed, for `batches` batches. Modes:
//   (none)     applyBatch (every layer exact after each batch), BFS / SSSP from scratch;
//   lazy       ingestBatch (edge store only); the layers' catch-up, sync(), is timed once at the end;
//   inc        BFS / SSSP corrected incrementally (trackIncremental / updateIncremental), checked
//              against from-scratch results after the stream;
//   lazy-inc   both.
// Result rows go to the CSV in the reference's schema (dataset,system,metric,mode,value,unit,
// count,threads) with the same metric names; system is "GIR-B200" with the mode's suffixes.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

#include "gir_b200.hpp"

namespace {

using gir_b200::GIR;

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

std::string slurp(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        std::fprintf(stderr, "gir_stream: cannot open %s\n", path.c_str());
        std::exit(1);
    }
    std::ostringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

// Unsigned integers of a text file in order, skipping every other character.
std::vector<int> read_uints(const std::string& path) {
    const std::string t = slurp(path);
    std::vector<int> out;
    long long x = -1;
    for (char c : t) {
        if (c >= '0' && c <= '9') {
            x = (x < 0 ? 0 : x) * 10 + (c - '0');
        } else if (x >= 0) {
            out.push_back((int)x);
            x = -1;
        }
    }
    if (x >= 0) out.push_back((int)x);
    return out;
}

struct Op {
    bool insert;
    int u, v;
};

// "a u v" / "d u v" lines.
std::vector<Op> read_ops(const std::string& path) {
    const std::string t = slurp(path);
    std::vector<Op> out;
    size_t i = 0;
    auto number = [&](int* x) {
        while (i < t.size() && (t[i] < '0' || t[i] > '9')) {
            if (t[i] == '\n') return false;
            ++i;
        }
        if (i >= t.size()) return false;
        long long v = 0;
        while (i < t.size() && t[i] >= '0' && t[i] <= '9') v = v * 10 + (t[i++] - '0');
        *x = (int)v;
        return true;
    };
    while (i < t.size()) {
        while (i < t.size() && t[i] != 'a' && t[i] != 'd') ++i;
        if (i >= t.size()) break;
        const bool ins = t[i++] == 'a';
        int u = 0, v = 0;
        if (!number(&u) || !number(&v)) continue;
        out.push_back({ins, u, v});
    }
    return out;
}

long meta(const std::string& dir, const std::string& key) {
    std::ifstream f(dir + "/meta.txt");
    std::string k;
    long v = 0;
    while (f >> k >> v)
        if (k == key) return v;
    std::fprintf(stderr, "gir_stream: meta key %s missing\n", key.c_str());
    std::exit(1);
}

void emit(const std::string& csv, const std::string& ds, const std::string& sys, const std::string& metric,
          const std::string& mode, double value, const char* unit, long long count) {
    FILE* f = std::fopen(csv.c_str(), "a");
    if (f) {
        std::fprintf(f, "%s,%s,%s,%s,%.6g,%s,%lld,%d\n", ds.c_str(), sys.c_str(), metric.c_str(), mode.c_str(), value,
                     unit, count, 1);
        std::fclose(f);
    }
    std::printf("  %-24s %-16s %.6g %s (n=%lld)\n", metric.c_str(), mode.c_str(), value, unit, count);
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s <protocol dir> <dataset> <csv> [batch=10000] [batches=10] [lazy|inc|lazy-inc]\n",
                     argv[0]);
        return 2;
    }
    const std::string dir = argv[1], ds = argv[2], csv = argv[3];
    const size_t B = argc > 4 ? std::stoul(argv[4]) : 10000;
    const int NB = argc > 5 ? std::stoi(argv[5]) : 10;
    const std::string mode = argc > 6 ? argv[6] : "";
    const bool lazy = mode == "lazy" || mode == "lazy-inc";
    const bool incr = mode == "inc" || mode == "lazy-inc";
    const std::string sys = std::string("GIR-B200") + (lazy ? "-lazy" : "") + (incr ? "-inc" : "");
    const int V = (int)meta(dir, "V");
    const int src = read_uints(dir + "/sources.txt").at(0);
    const std::vector<int> el = read_uints(dir + "/loaded.el");
    std::vector<std::pair<int, int>> edges;
    edges.reserve(el.size() / 2);
    for (size_t i = 0; i + 1 < el.size(); i += 2) edges.push_back({el[i], el[i + 1]});
    try {
        for (const char* s : {"insert", "delete", "mixed"}) {
            GIR g(gir_b200::graph::fromEdges(V, edges));
            g.buildWCC();
            g.buildSCC_DAG();
            g.buildBCT();
            double t0 = now_s();
            if (incr) g.trackIncremental(src, false); else g.bfs(src);
            double t1 = now_s();
            if (incr) g.trackIncremental(src, true); else g.sssp(src);
            double t2 = now_s();
            if (std::string(s) == "insert") {
                emit(csv, ds, sys, "bfs_initial_ms", "from-scratch", (t1 - t0) * 1000, "ms", 1);
                emit(csv, ds, sys, "sssp_initial_ms", "from-scratch", (t2 - t1) * 1000, "ms", 1);
            }
            const std::vector<Op> ops = read_ops(dir + "/" + s + ".ops");
            double tu = 0, tb = 0, tsp = 0;
            int nb = 0;
            for (size_t i = 0; i < ops.size() && nb < NB; i += B, ++nb) {
                std::vector<GIR::Update> batch;
                for (size_t j = i; j < ops.size() && j < i + B; ++j) batch.push_back({ops[j].u, ops[j].v, ops[j].insert});
                const double a = now_s();
                if (lazy) g.ingestBatch(batch); else g.applyBatch(batch);
                const double b = now_s();
                if (incr) g.updateIncremental(false); else g.bfs(src);
                const double c = now_s();
                if (incr) g.updateIncremental(true); else g.sssp(src);
                const double d = now_s();
                tu += b - a;
                tb += c - b;
                tsp += d - c;
            }
            if (nb == 0) continue;
            if (incr) {  // the corrected results must equal from-scratch ones
                const auto lv = g.bfs(src);
                const auto dd = g.sssp(src);
                long long bad = 0;
                for (int v = 0; v < V; ++v) {
                    const uint64_t want = lv[v] < 0 ? UINT64_MAX : (uint64_t)lv[v];
                    bad += g.incDist(false, v) != want || g.incDist(true, v) != dd[v];
                }
                std::fprintf(stderr, "%s stream: incremental vs from-scratch mismatches: %lld\n", s, bad);
                emit(csv, ds, sys, std::string("inc_mismatch_") + s, "final", (double)bad, "vertices", V);
            }
            const std::string st = s;
            const std::string mm = (lazy ? "ingest_batch_" : "fmu_batch_") + std::to_string(B);
            emit(csv, ds, sys, st + "_mutation_MEPS", mm, nb * (double)B / 1e6 / tu, "MEPS", nb * (long long)B);
            emit(csv, ds, sys, "bfs_" + st + "_recompute_ms", incr ? "incremental" : "from-scratch", tb * 1000 / nb, "ms", nb);
            emit(csv, ds, sys, "bfs_" + st + "_endtoend_ms", "batch_" + std::to_string(B), (tu + tb) * 1000 / nb, "ms", nb);
            emit(csv, ds, sys, "sssp_" + st + "_recompute_ms", incr ? "incremental" : "from-scratch", tsp * 1000 / nb, "ms", nb);
            emit(csv, ds, sys, "sssp_" + st + "_endtoend_ms", "batch_" + std::to_string(B), (tu + tsp) * 1000 / nb, "ms", nb);
            if (lazy) {  // the layers' catch-up for the whole stream
                const double a = now_s();
                g.sync();
                const double b = now_s();
                emit(csv, ds, sys, "sync_" + st + "_ms", "after_" + std::to_string(nb) + "_batches", (b - a) * 1000, "ms", nb);
            }
        }
    } catch (const gir_b200::Error& e) {
        std::fprintf(stderr, "gir_stream: error %d: %s\n", e.code(), e.what());
        return 1;
    }
    return 0;
}
