// Internal declarations shared by the GIR-B200 CUDA sources: the handle, the device graph
// store, scratch buffers, error plumbing and small device helpers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "gir_dev.h"

namespace gir {

// ---------------------------------------------------------------------------------------------
// Error plumbing: every internal function returns a gir status; the first failure records its
// text in the handle.
// ---------------------------------------------------------------------------------------------
struct Status {
    int code = GIR_OK;
    std::string msg;
};

#define GIR_TRY(expr)                    \
    do {                                 \
        int _rc = (expr);                \
        if (_rc != GIR_OK) return _rc;   \
    } while (0)

// ---------------------------------------------------------------------------------------------
// Device buffers
// ---------------------------------------------------------------------------------------------
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

// ---------------------------------------------------------------------------------------------
// Slack CSR resident in HBM. Row v holds deg[v] sorted neighbour ids at adj[beg[v] ..
// beg[v] + deg[v]); the rest of [beg[v], beg[v+1]) is free room for inserts. Every row starts
// on a 16-byte boundary (beg[v] % 4 == 0) so rows can be read with 128-bit loads.
// ---------------------------------------------------------------------------------------------
struct DevCSR {
    int64_t* beg = nullptr;  // V + 1 capacity offsets
    int32_t* deg = nullptr;  // V current row lengths
    int32_t* adj = nullptr;  // beg[V] entries
    uint32_t* w = nullptr;   // optional weights aligned with adj
    int64_t cap = 0;         // beg[V]
    int64_t E = 0;           // sum of deg
};

// Device view passed to kernels by value.
struct CSRView {
    const int64_t* beg;
    const int32_t* deg;
    const int32_t* adj;
    const uint32_t* w;
};
inline CSRView view(const DevCSR& c) { return CSRView{c.beg, c.deg, c.adj, c.w}; }

struct QueryStats {
    int64_t edges = 0, reached = 0, iterations = 0, bottom_up = 0, launches = 0;
    double kernel_ms = 0, total_ms = 0, main_ms = 0;
    int64_t main_launches = 0;
    int64_t persistent_levels = 0;
};

// Times the launches issued by `launch` with CUDA events when profiling is on, adding them to
// the query statistics (the caller synchronizes the stream before reading the result).
struct MainTimer {
    gir_dev* g;
    bool on;
    template <class F>
    int run(F&& launch);
};

}  // namespace gir

// The handle. (Global namespace: the C ABI forward-declares `struct gir_dev`.)
struct gir_dev {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr, ev3 = nullptr;
    int64_t V = 0;

    gir::DevCSR fw, bw, sym;
    bool has_weights = false;
    uint64_t wrule_seed = 0;
    uint32_t wrule_lo = 0, wrule_hi = 0;  // lo > hi: use the hash weight of GIR::edgeWeight

    // Layers
    bool wcc_built = false, scc_built = false, bct_built = false;
    gir::DevBuf wcc, scc, scc_rank;  // int32[V]
    int64_t n_wcc = -1, n_scc = -1;
    gir::DevBuf dag;                 // uint64 keys (scc_u << 32 | scc_v), sorted, distinct
    gir::DevBuf dag_rows;            // int64[V + 1]: row starts of dag by source label (reachability)
    bool dag_rows_valid = false;
    gir::DevBuf reach_hub;           // uint64[2V]: hubs that reach v, then hubs v reaches (reachability)
    bool reach_hub_valid = false;
    int64_t n_dag = -1;
    gir::DevBuf blk_label, blk_head, bcnt;  // int32[V], int32[n_blocks], int32[V]
    int64_t n_blocks = -1;

    // Incremental single-source results ([0] BFS, [1] SSSP with the hash weights): per vertex
    // dist << 32 | parent (all ones = unreachable), and the edge keys (u << 32 | v) changed by
    // batches since the last update.
    bool inc_on[2] = {false, false};
    int32_t inc_src[2] = {-1, -1};
    gir::DevBuf inc_st[2], inc_pend[2];
    int64_t inc_npend[2] = {0, 0};

    // Working arrays of the single-edge checks (single.cu): generation-stamped, zeroed once.
    gir::DevBuf single_ws;
    int32_t single_gen = 1;
    int64_t single_checked = 0, single_kept = 0;  // ops that ran the checks / rebuilds they avoided

    // Weight-sorted copies of the forward CSR for SSSP ([0] hash weights, [1] stored weights).
    gir::DevCSR ws[2];
    bool ws_valid[2] = {false, false};
    // SSSP lane order, per weight mode: the distance of every vertex to the vertex of largest
    // in-degree (uint64[V], UINT64_MAX = does not reach it), from one backward single-lane run.
    // Queries place sources with close values in neighbouring lanes, so the lanes that share a
    // 32-byte sector of the distance rows tend to be active in the same bucket. It only orders
    // lanes, so it is kept across updates (a stale order costs time, never exactness).
    gir::DevBuf hub_dist[2];
    bool hub_valid[2] = {false, false};
    uint64_t hub_max[2] = {0, 0};        // largest finite value of hub_dist
    bool narrow16_failed[2] = {false, false};  // a 16-bit lane-distance run overflowed on this handle

    // Degree bins of the backward CSR (bottom-up traversal): vertex ids by in-degree class.
    gir::DevBuf bins;                // int32[V]: small | medium | large, each ascending
    int64_t bin_n[3] = {0, 0, 0};
    bool bins_valid = false;

    // Stream-ordered pool of every device buffer of the handle: allocations and frees are queued
    // on the handle's stream and the pool keeps its memory, so no call waits for the device to
    // go idle the way cudaMalloc / cudaFree do.
    cudaMemPool_t pool = nullptr;
    bool scratch_tight = false;  // the graph's working set is large against free memory (see create)

    // Scratch, grown on demand and kept across calls.
    gir::DevBuf scratch[16];
    gir::DevBuf cub_tmp;
    gir::DevBuf stage_in, stage_out;  // device staging for host pointers
    gir::DevBuf work[8];              // buffers of the create / batch pipelines (not used by store ops)
    gir::DevBuf lane_dist;            // lane-interleaved SSSP distances (V x lanes)
    gir::DevBuf qitems[5];            // per-queue-entry work items of the SSSP relaxation
    gir::DevBuf sssp_sets;            // SSSP: every set's source range and lane-order key
    gir::DevBuf sssp_lanes;           // SSSP: one lane group's source ranges and output rows
    gir::DevBuf sssp_done;            // SSSP: per vertex, the lanes whose distance is final
    void* pinned = nullptr;           // small pinned host buffer for counters
    size_t pinned_bytes = 0;

    // Deferred maintenance (GIR::ingestBatch / sync, gir.h:107-116): batches ingested since the
    // last sync are in the edge store already; the layers still describe the last sync. What the
    // pending changes can do to each layer is accumulated (flags judged against the labels of the
    // last sync, OR-ed over the ingested batches) with the undirected pairs they made present, so
    // that sync repairs the layers once for all of them.
    bool pend = false;
    bool pend_scc_split = false, pend_scc_cycle = false, pend_dag = false, pend_bct = false, pend_wcc_del = false;
    gir::DevBuf pend_pairs;          // uint64 keys of undirected pairs made present
    int64_t n_pend_pairs = 0;

    // Batch statistics
    int64_t b_ins = 0, b_del = 0, b_noop = 0, b_invalid = 0;
    double b_ms[4] = {0, 0, 0, 0};    // phases of the last batch: store, WCC, SCC, BCT
    int b_plan[3] = {2, 2, 2};        // what the last batch did per layer: 0 kept, 1 patched, 2 rebuilt

    // Schedule
    int schedule = GIR_SCHEDULE_FIXED;
    double params[GIR_PARAM_COUNT] = {15.0, 18.0, 16.0, 256.0, 32.0, 4096.0, 4.0, 0.0, -1.0, 0.0, 1.0};
    cudaEvent_t pev0 = nullptr, pev1 = nullptr;  // main-kernel timing (GIR_PARAM_PROFILE)
    gir::DevBuf sched_w;              // MLP parameters (fp32)
    gir::DevBuf sched_io;             // one decision's features and logits
    bool sched_loaded = false;
    std::vector<float> sched_host;    // host copy of the MLP parameters

    gir::QueryStats qstats;
    std::vector<float> trace_x;       // schedule features of the last query call, GIR_SCHED_IN per row
    std::vector<int32_t> trace_y;     // the class taken for each row
    double wstat[2][2] = {{0, 0}, {0, 0}};  // per weight mode: mean and max weight (set with ws)
    std::string err;
    // Phase trace on stderr (environment GIR_TRACE=1): each mark synchronizes and prints the
    // wall time since the previous one, and every scratch allocation is reported; GIR_TRACE=2
    // reports the allocations only (no synchronizing marks).
    bool trace_on = std::getenv("GIR_TRACE") != nullptr;
    bool trace_marks = trace_on && std::string(std::getenv("GIR_TRACE")) != "2";
    double trace_t = 0;
};

namespace gir {

// Records an error on the handle and returns `code`.
int fail(gir_dev* g, int code, const std::string& msg);
// The text gir_dev_last_error(NULL) returns on this thread (calls that have no handle).
void set_thread_error(const std::string& msg);
// Checks a CUDA result; on failure records it and returns GIR_ERR_CUDA (or GIR_ERR_OOM).
int cuda_check(gir_dev* g, cudaError_t e, const char* what);
#define GIR_CUDA(g, call) GIR_TRY(::gir::cuda_check((g), (call), #call))
#define GIR_LAUNCH(g, what) GIR_TRY(::gir::cuda_check((g), cudaGetLastError(), what))

// Monotonic wall clock in ms.
double now_ms();
// With tracing on: synchronizes the handle's stream, prints `what` and the ms since the last mark.
void trace_mark(gir_dev* g, const char* what);

// Device memory from the handle's pool, ordered on its stream.
int dev_alloc(gir_dev* g, void** p, size_t bytes);
template <class T>
int dev_alloc_n(gir_dev* g, T** p, size_t n) {
    return dev_alloc(g, reinterpret_cast<void**>(p), n * sizeof(T));
}
void dev_free(gir_dev* g, void* p);

// Grows a device buffer to at least `bytes` (contents not kept).
int ensure(gir_dev* g, DevBuf& b, size_t bytes);
template <class T>
int ensure_n(gir_dev* g, DevBuf& b, size_t n, T** out) {
    GIR_TRY(ensure(g, b, n * sizeof(T) + 16));
    *out = static_cast<T*>(b.p);
    return GIR_OK;
}
void release(gir_dev* g, DevBuf& b);
// When device memory is tight for the graph (scratch_tight, decided at create), returns every working buffer of at least
// `min_bytes` to the handle's pool (top-level calls do this on return: the pool hands the memory
// to the next phase that needs it, so on large graphs the phases share one working set instead of
// each keeping its own high-water mark). Otherwise the buffers are kept for the next call.
void release_scratch(gir_dev* g, size_t min_bytes);
constexpr size_t kKeepScratchBelow = 64u << 20;

// Pinned host scratch of at least `bytes`.
int pinned(gir_dev* g, size_t bytes, void** out);

bool is_device_ptr(const void* p);

// Copies `bytes` from a host or device pointer into device memory owned by the handle
// (`stage`), or returns `p` itself when it is already device memory.
int stage_input(gir_dev* g, DevBuf& stage, const void* p, size_t bytes, const void** dev);

// Grid size for a persistent/grid-stride kernel.
inline int grid_for(gir_dev* g, int64_t work, int block) {
    const int64_t blocks = (work + block - 1) / block;
    const int64_t cap = (int64_t)g->num_sms * (int64_t)g->params[GIR_PARAM_CTAS_PER_SM] * 4;
    return (int)(blocks < 1 ? 1 : (blocks < cap ? blocks : cap));
}

template <class F>
int MainTimer::run(F&& launch) {
    if (!on) return launch();
    GIR_CUDA(g, cudaEventRecord(g->pev0, g->stream));
    GIR_TRY(launch());
    GIR_CUDA(g, cudaEventRecord(g->pev1, g->stream));
    GIR_CUDA(g, cudaEventSynchronize(g->pev1));
    float ms = 0;
    GIR_CUDA(g, cudaEventElapsedTime(&ms, g->pev0, g->pev1));
    g->qstats.main_ms += ms;
    g->qstats.main_launches++;
    return GIR_OK;
}

// ---- store (store.cu) ----
int store_build_csr_from_keys(gir_dev* g, DevCSR& c, const uint64_t* keys, int64_t n, const uint32_t* w);
int store_free(gir_dev* g, DevCSR& c);
int store_build_sym(gir_dev* g);
int store_compact_csr(gir_dev* g, const DevCSR& c, int64_t* beg_out, int32_t* adj_out, int64_t cap);
int store_has_edges(gir_dev* g, const DevCSR& c, const int32_t* u, const int32_t* v, int64_t n, uint8_t* out);
int store_apply_ops(gir_dev* g, DevCSR& c, const uint64_t* ins, int64_t n_ins, const uint64_t* del, int64_t n_del,
                    bool weights);
int store_build_bins(gir_dev* g);
// One change u -> v applied in place to the fw / bw / sym rows when they have room (store.cu):
// out[0] 0 no-op, 1 applied, 2 no room (nothing changed); out[1] 1 / 2 when the undirected pair
// appeared / disappeared; out[2] layer flags (bit 0 SCC split possible, 1 cycle closed against
// the ranks, 2 a cross edge changed, 3 blocks may change); keys[0] the edge, keys[1..2] the pair.
int store_single_edit(gir_dev* g, int32_t u, int32_t v, int insert, unsigned long long* out, uint64_t* keys);

// ---- CUB wrappers (prims.cu) ----
int sort_keys_u64(gir_dev* g, uint64_t* keys, uint64_t* tmp, int64_t n, int end_bit);
int sort_pairs_u64(gir_dev* g, uint64_t* keys, uint64_t* ktmp, uint32_t* vals, uint32_t* vtmp, int64_t n, int end_bit);
int sort_pairs_u64_i64(gir_dev* g, uint64_t* keys, uint64_t* ktmp, int64_t* vals, int64_t* vtmp, int64_t n, int end_bit);
int exclusive_scan_i64(gir_dev* g, const int64_t* in, int64_t* out, int64_t n);
int sum_i64(gir_dev* g, const int64_t* in, int64_t n, int64_t* host_out);
// Compacts the entries of `in` whose flag is non-zero into `out`; *host_n = count.
int select_flagged_u64(gir_dev* g, const uint64_t* in, const uint8_t* flags, uint64_t* out, int64_t n, int64_t* host_n);
int select_flagged_i32(gir_dev* g, const int32_t* in, const uint8_t* flags, int32_t* out, int64_t n, int64_t* host_n);
// Indices i in [0, n) with flags[i] != 0, ascending.
int select_flagged_iota(gir_dev* g, const uint8_t* flags, int32_t* out, int64_t n, int64_t* host_n);
// The rows of `deg` (V entries) longer than max_deg, ascending, into rows (V entries), and the
// exclusive scan of their lengths into pref (V + 1 entries); *n = their number. flag: V bytes.
constexpr int32_t kHeavyRow = 4096;
int heavy_rows(gir_dev* g, const int32_t* deg, int64_t V, int32_t max_deg, uint8_t* flag, int32_t* rows, int64_t* pref,
               int64_t* n);

// ---- layers ----
int wcc_build(gir_dev* g);
int wcc_union_pairs(gir_dev* g, const uint64_t* keys, int64_t n);
int scc_build(gir_dev* g);
// Condensation DAG and ranks from the current SCC labels (the labels are kept).
int scc_build_dag(gir_dev* g);
// The DAG after one edge u -> v between two SCCs whose ranks respect it was inserted or deleted
// (labels unchanged): one key added or removed where that settles it (*patched), else
// scc_build_dag.
int scc_dag_patch_one(gir_dev* g, int32_t u, int32_t v, bool insert, bool* patched);
// Betweenness of every vertex over the sources (device arrays; score has V entries).
int bc_run(gir_dev* g, const int32_t* srcs_d, int64_t n_src, double* score_d);
// Reachability of every pair (u[i], v[i]) into out[i] (device arrays; the SCC layer is built).
int reach_run(gir_dev* g, const int32_t* u_d, const int32_t* v_d, int64_t n, uint8_t* out_d);
int bct_build(gir_dev* g);
// Exact checks for a batch with one effective edge change u -> v (single.cu); out[i] per check:
// 0 not run, 1 found, 2 not found, 3 over budget (unknown), 4 (wcc only) not connected, and the
// component's labels were split in place. wcc: u, v connected in sym. split:
// u reaches v inside their SCC. cycle: v reaches u within the rank window. twopath: two
// internally vertex-disjoint u-v paths in their SCC's undirected subgraph.
struct SingleChecks {
    bool wcc = false, split = false, cycle = false, twopath = false;
};
int single_op_checks(gir_dev* g, int32_t u, int32_t v, const SingleChecks& want, int32_t out[4]);
// Incremental BFS / SSSP (incr.cu): track one source, log a batch's changed edges (device keys),
// correct the tracked result for the logged changes, and write its distances (device, V entries).
int inc_track(gir_dev* g, int32_t source, int weighted);
int inc_log(gir_dev* g, const uint64_t* ins, int64_t n_ins, const uint64_t* del, int64_t n_del);
int inc_update(gir_dev* g, int weighted);
int inc_dist(gir_dev* g, int weighted, uint64_t* out_d);

// ---- queries ----
int bfs_run(gir_dev* g, const int64_t* set_beg_h, const int32_t* srcs_d, int64_t n_sets, int32_t* level_d);
int sssp_run(gir_dev* g, const int64_t* set_beg_h, const int32_t* srcs_d, int64_t n_sets, uint64_t delta,
             int weight_mode, uint64_t* dist_d);

// ---- schedule network (sched.cu) ----
int sched_choose_delta(gir_dev* g, const float* features, uint64_t* delta);
// The SCC build's forward-backward pivot rule (0..3, see GIR_PARAM_PIVOT) from the network, with
// the fixed rule 0 when its margin is small; features from sched_scc_features.
int sched_choose_pivot(gir_dev* g, const float* features, int* rule);
void sched_scc_features(const gir_dev* g, double active, double active_edges, double max_score, float* out);
// Enqueues the device decision of the next BFS level's direction: reads the frontier's pairs and
// out-edges at cnt[i_pairs] / cnt[i_medges], writes the direction (0 top-down, 1 bottom-up) to
// cnt[i_dir] and the GIR_SCHED_IN features (floats) from cnt[i_feat] on.
int sched_bfs_decide_async(gir_dev* g, unsigned long long* cnt, int i_pairs, int i_medges, int i_dir, int i_feat,
                           int lanes, double mu_prev, bool bottom_up, double alpha, double beta);
// Feature rows (GIR_SCHED_IN floats) of the two decisions. BFS level: frontier vertices and
// out-edges, unexplored out-edges, level, current direction, graph density, lanes. SSSP group:
// density, mean / max weight, size, lanes.
void sched_bfs_features(const gir_dev* g, double nf, double mf, double mu, int level, bool bottom_up, int lanes,
                        float* out);
void sched_sssp_features(const gir_dev* g, int weight_mode, int lanes, float* out);
// Class of a Delta value among the candidates (nearest in log scale).
int sched_delta_class(uint64_t delta);
void sched_trace(gir_dev* g, const float* x, int32_t y);

// ---------------------------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------------------------
#ifdef __CUDACC__
__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// GIR::edgeWeight (gir_query.cpp:50-54): MurmurHash3's fmix64 of (u << 32 | v) into [1,100].
__device__ __forceinline__ uint32_t hash_weight(int32_t u, int32_t v) {
    uint64_t x = ((uint64_t)(uint32_t)u << 32) | (uint32_t)v;
    x ^= x >> 33; x *= 0xff51afd7ed558ccdULL; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL; x ^= x >> 33;
    return 1u + (uint32_t)(x % 100ull);
}

// Lower bound of `x` in the sorted range a[lo, hi).
template <class T>
__device__ __forceinline__ int64_t lower_bound_dev(const T* a, int64_t lo, int64_t hi, T x) {
    while (lo < hi) {
        const int64_t m = (lo + hi) >> 1;
        if (a[m] < x) lo = m + 1; else hi = m;
    }
    return lo;
}

// Calls f(u, w, edge_index) for every entry of the rows of vertices [v0, v1) of `c`. Warp-
// cooperative: a warp takes 32 consecutive vertices, scans their row lengths and walks the
// concatenated rows 32 entries at a time (consecutive lanes read consecutive entries of a row),
// so a row of any length costs its warp ceil(len/32) rounds. Must be called by all threads of
// the grid (every lane of a warp takes part in every round). `scan` is per-warp shared scratch
// of 33 int64 and 32 int32.
// With max_deg >= 0, rows longer than max_deg are left out: a warp walks all of its 32 rows, so a
// hub row would keep one warp busy long after the rest of the grid is idle; sweep those rows with
// grid_sweep_heavy_rows instead (rows and offsets from heavy_rows).
template <class F>
__device__ __forceinline__ void warp_sweep_rows(const int64_t* beg, const int32_t* deg, const int32_t* adj,
                                                int64_t v0, int64_t v1, int64_t* s_excl, int32_t* s_u, F&& f,
                                                int32_t max_deg = -1) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = v0 + warp * 32; base < v1; base += nwarps * 32) {
        const int64_t v = base + lane;
        int64_t cnt = v < v1 ? deg[v] : 0;
        if (max_deg >= 0 && cnt > max_deg) cnt = 0;
        int64_t incl = cnt;
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        s_excl[lane] = incl - cnt;
        if (lane == 31) s_excl[32] = incl;
        s_u[lane] = (int32_t)v;
        __syncwarp();
        const int64_t total = s_excl[32];
        for (int64_t p0 = 0; p0 < total; p0 += 32) {
            const int64_t p = p0 + lane;
            if (p < total) {
                int lo = 0, hi = 31;
                while (lo < hi) {
                    const int m = (lo + hi + 1) >> 1;
                    if (s_excl[m] <= p) lo = m; else hi = m - 1;
                }
                const int32_t u = s_u[lo];
                const int64_t e = beg[u] + (p - s_excl[lo]);
                f(u, adj[e], e);
            }
        }
        __syncwarp();
    }
}

// Calls f(u, w, edge_index) for every entry of the rows rows[0 .. n) (pref: the exclusive scan of
// their lengths, n + 1 entries), the entries spread evenly over the whole grid: the companion of
// warp_sweep_rows(..., max_deg) for the rows it leaves out.
template <class F>
__device__ __forceinline__ void grid_sweep_heavy_rows(const int32_t* rows, const int64_t* pref, int64_t n,
                                                      const int64_t* beg, const int32_t* adj, F&& f) {
    if (n <= 0) return;
    const int64_t total = pref[n];
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        int64_t lo = 0, hi = n - 1;  // largest r with pref[r] <= e
        while (lo < hi) {
            const int64_t m = (lo + hi + 1) >> 1;
            if (pref[m] <= e) lo = m; else hi = m - 1;
        }
        const int32_t u = rows[lo];
        const int64_t k = beg[u] + (e - pref[lo]);
        f(u, adj[k], k);
    }
}

// Warp-aggregated append: every lane with `pred` gets a distinct slot in `q` (counter `cnt`).
__device__ __forceinline__ void warp_append(bool pred, int32_t value, int32_t* q, unsigned long long* cnt) {
    const unsigned m = __ballot_sync(0xffffffffu, pred);
    if (!m) return;
    const int leader = __ffs(m) - 1;
    unsigned long long base = 0;
    if (lane_id() == leader) base = atomicAdd(cnt, (unsigned long long)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (pred) q[base + __popc(m & ((1u << lane_id()) - 1))] = value;
}

// Grid-wide barrier of a cooperative launch: every CTA meets here. `bar` holds the arrival count
// at bar[0] and the generation at bar[32] (own 128-byte lines), zeroed by the host before the
// launch. The wait is bounded: after `spins` polls a CTA sets *err and leaves; every CTA also
// leaves once it sees *err set. Returns false once any CTA has flagged an error.
__device__ __forceinline__ bool grid_barrier(unsigned int* bar, unsigned long long* err, unsigned spins_max) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int* gen = bar + 32;
        const unsigned int g0 = *gen;
        __threadfence();
        if (atomicAdd(bar, 1u) == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 32, 1u);
        } else {
            unsigned int spins = 0;
            while (*gen == g0) {
                if (++spins > spins_max) {
                    atomicExch(err, 1ull);
                    break;
                }
                if ((spins & 63) == 0 && __ldcg(err) != 0ull) break;
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return __ldcg(err) == 0ull;
}

// Staged queue appends: a warp collects its entries in a shared-memory buffer of kStage slots
// and reserves queue space with one atomicAdd per buffer-full, instead of one per ballot, so
// thousands of warps appending to one queue do not serialize on its counter. Every lane of the
// warp calls stage_append (warp-uniform), and stage_flush once at the end.
constexpr int kStage = 128;
__device__ __forceinline__ void stage_flush(int32_t* s_buf, int& s_n, int32_t* q, unsigned long long* cnt) {
    if (s_n == 0) return;
    unsigned long long base = 0;
    if (lane_id() == 0) base = atomicAdd(cnt, (unsigned long long)s_n);
    base = __shfl_sync(0xffffffffu, base, 0);
    for (int i = lane_id(); i < s_n; i += 32) q[base + i] = s_buf[i];
    __syncwarp();
    s_n = 0;
}
__device__ __forceinline__ void stage_append(bool pred, int32_t value, int32_t* s_buf, int& s_n, int32_t* q,
                                             unsigned long long* cnt) {
    const unsigned m = __ballot_sync(0xffffffffu, pred);
    if (!m) return;
    const int k = __popc(m);
    if (s_n + k > kStage) stage_flush(s_buf, s_n, q, cnt);
    if (pred) s_buf[s_n + __popc(m & ((1u << lane_id()) - 1))] = value;
    __syncwarp();
    s_n += k;
}

// Slots for the CTA's flagged threads with one atomicAdd for the whole CTA (block-uniform call;
// s_w: shared int[blockDim / 32], s_base: one shared word). Returns this thread's slot.
__device__ __forceinline__ unsigned long long block_slot(bool pred, unsigned long long* cnt, int* s_w,
                                                         unsigned long long* s_base) {
    const unsigned m = __ballot_sync(0xffffffffu, pred);
    const int wib = threadIdx.x >> 5;
    if (lane_id() == 0) s_w[wib] = __popc(m);
    __syncthreads();
    if (threadIdx.x == 0) {
        int tot = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            const int c = s_w[k];
            s_w[k] = tot;
            tot += c;
        }
        *s_base = tot ? atomicAdd(cnt, (unsigned long long)tot) : 0ull;
    }
    __syncthreads();
    const unsigned long long slot = *s_base + (unsigned long long)s_w[wib] + __popc(m & ((1u << lane_id()) - 1));
    __syncthreads();  // (s_w and s_base are rewritten by the next call)
    return slot;
}

// Frontier expansion over one CSR: a warp takes 32 queue entries and walks their rows together.
// f(u, w) is called for every entry w of row u; it returns true when w joins the next queue.
template <class F>
__device__ __forceinline__ void warp_expand(const int32_t* q, int64_t n, const CSRView& c, int32_t* nq,
                                            unsigned long long* ncnt, F&& f) {
    constexpr int kW = 32;  // supports blocks of up to 1024 threads
    __shared__ int64_t s_excl[kW][33];
    __shared__ int32_t s_u[kW][32];
    __shared__ int32_t s_st[kW][kStage];
    int n_st = 0;
    const int lane = lane_id(), wib = threadIdx.x >> 5;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = warp * 32; base < n; base += nwarps * 32) {
        const int64_t i = base + lane;
        const int32_t u = i < n ? q[i] : -1;
        const int64_t cnt = u >= 0 ? c.deg[u] : 0;
        int64_t incl = cnt;
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        s_excl[wib][lane] = incl - cnt;
        if (lane == 31) s_excl[wib][32] = incl;
        s_u[wib][lane] = u;
        __syncwarp();
        const int64_t total = s_excl[wib][32];
        for (int64_t p0 = 0; p0 < total; p0 += 32) {
            const int64_t p = p0 + lane;
            bool push = false;
            int32_t w = 0;
            if (p < total) {
                int lo = 0, hi = 31;
                while (lo < hi) {
                    const int m = (lo + hi + 1) >> 1;
                    if (s_excl[wib][m] <= p) lo = m; else hi = m - 1;
                }
                const int32_t uu = s_u[wib][lo];
                w = c.adj[c.beg[uu] + (p - s_excl[wib][lo])];
                push = f(uu, w);
            }
            stage_append(push, w, s_st[wib], n_st, nq, ncnt);
        }
        __syncwarp();
    }
    stage_flush(s_st[wib], n_st, nq, ncnt);
}

#endif

}  // namespace gir
