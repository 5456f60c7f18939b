/* GIR-B200 device library: the C ABI under the GIR class surface.
 *
 * The reference has no FFI of its own: its boundary is the C++ class GIR
 * (gir_constructor/gir.h:72-671) plus the loader class graph (gir_constructor/graph.h:11-57).
 * Each entry point below replaces the reference interface named beside it; the C++ class in
 * include/gir_b200.hpp restates the GIR surface on top of these calls.
 *
 * Conventions
 *  - Every call returns an int status: GIR_OK (0) or one of the GIR_ERR_* codes; the text of
 *    the last failure on a handle is gir_dev_last_error(handle) (handle NULL: the last failure
 *    of a create / load call on this thread).
 *  - Array arguments may be host memory (pageable or pinned) or device memory of the handle's
 *    GPU; the library looks at each pointer and copies through its own staging when needed.
 *    Every call returns only once its outputs are complete.
 *  - One handle = one graph resident in HBM on the device that was current at create time,
 *    one CUDA stream. A handle is not thread-safe: one caller thread at a time (like GIR,
 *    gir_constructor/gir.h:72, which is single-caller with internal OpenMP parallelism).
 *  - Vertex ids are int32 in [0, V); edge offsets are int64 on the device.
 *  - Component labels are canonical: the label of a WCC / SCC is the smallest vertex id in it.
 */
#ifndef GIR_DEV_H
#define GIR_DEV_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gir_dev gir_dev_t;

enum {
    GIR_OK = 0,
    GIR_ERR_INVALID = 1,   /* bad argument (null handle, negative size, ...) */
    GIR_ERR_CUDA = 2,      /* a CUDA call failed (text in gir_dev_last_error) */
    GIR_ERR_OOM = 3,       /* device or host allocation failed */
    GIR_ERR_FILE = 4,      /* a graph file cannot be opened or is short */
    GIR_ERR_MALFORMED = 5, /* CSR offsets not monotone 0..E, ids outside [0,V), fw/bw sizes or
                              deduplicated edge counts disagree */
    GIR_ERR_STATE = 6,     /* call order: a layer that is needed was not built */
    GIR_ERR_TIMEOUT = 7,   /* a bounded device wait gave up (error status, context intact) */
    GIR_ERR_CAPACITY = 8,  /* a size limit of this build was exceeded */
    GIR_ERR_NODEVICE = 9   /* no CUDA device */
};

/* layers for gir_dev_build */
enum { GIR_LAYER_WCC = 1, GIR_LAYER_SCC = 2, GIR_LAYER_BCT = 4, GIR_LAYER_ALL = 7 };

/* label kinds for gir_dev_get_labels (int32[V] each) */
enum {
    GIR_LABEL_WCC = 0,   /* smallest vertex id of v's weakly connected component */
    GIR_LABEL_SCC = 1,   /* smallest vertex id of v's strongly connected component */
    GIR_LABEL_BLOCK = 2, /* id of v's parent block in the block-cut forest of its SCC (v_block,
                            gir.h:420); every vertex has one */
    GIR_LABEL_BCNT = 3,  /* number of blocks containing v (v_bcnt, gir.h:421); AP iff >= 2 */
    GIR_LABEL_SCC_RANK = 4 /* topological rank of v's SCC in the condensation DAG: rank(a) <
                              rank(b) for every DAG edge a -> b (scc_rank, gir.h:329) */
};

/* edge weights for SSSP */
enum {
    GIR_WEIGHT_HASH = 0,  /* GIR::edgeWeight(u,v) in [1,100] (gir_query.cpp:50-54) */
    GIR_WEIGHT_STORED = 1 /* the uint32 per-edge weights given to gir_dev_create */
};

/* scheduling policy for the traversal heuristics */
enum { GIR_SCHEDULE_FIXED = 0, GIR_SCHEDULE_LEARNED = 1 };

/* ---- construction: graph::graph (graph.cpp:2-120), GIR::GIR (gir.cpp:38-63) ---- */

/* Four-array int32 CSR (forward: out-neighbours; backward: in-neighbours), as graph::graph
 * holds it after loading (graph.h:14-18). w (nullable) gives one uint32 weight per forward
 * entry. Rows are sorted and de-duplicated on the device as normalizeBaseCsr does
 * (gir.cpp:95-130); malformed input gives GIR_ERR_MALFORMED, where the reference exits. */
int gir_dev_create(const int32_t* fw_beg, const int32_t* fw_adj, const int32_t* bw_beg, const int32_t* bw_adj,
                   int64_t V, int64_t E, const uint32_t* w, gir_dev_t** out);

/* GIR(path_directed, path_undirected) (gir.h:93): reads <dir>fw_begin.bin, fw_adjacent.bin,
 * bw_begin.bin, bw_adjacent.bin (int32) with the reference's checks (graph.cpp:95-114). `dir`
 * is a prefix, as in the reference (gir.cpp:40-42): give it its trailing '/'. */
int gir_dev_load(const char* dir, gir_dev_t** out);

/* ~GIR (gir.cpp:65-68). NULL is accepted. */
int gir_dev_destroy(gir_dev_t* g);

const char* gir_dev_last_error(const gir_dev_t* g);

/* Sizes of the current state. Any pointer may be NULL. V: vertices; E: directed edges; the
 * others are the number of WCCs / SCCs / condensation edges / blocks of the last build or
 * batch (-1 while that layer is not built). */
int gir_dev_counts(gir_dev_t* g, int64_t* V, int64_t* E, int64_t* n_wcc, int64_t* n_scc, int64_t* n_dag,
                   int64_t* n_blocks);

/* ---- layers: buildWCC / buildSCC_DAG / buildBCT (gir.cpp:593, 798, 2063) ---- */

/* Builds the requested layers in the reference's order (WCC, then SCC + DAG, then BCT; BCT
 * needs SCC). */
int gir_dev_build(gir_dev_t* g, unsigned layers);

/* getNodeToScc / getNodeToWcc (gir.cpp:4117-4126), sccOf / wccOf, the block-cut forest
 * per-vertex arrays and SCC ranks: int32[V] of the kind `which` (GIR_LABEL_*). */
int gir_dev_get_labels(gir_dev_t* g, int which, int32_t* out);

/* getDAG (gir.cpp:4127-4132): the distinct condensation edges (scc label of u, scc label of
 * v) over all edges u -> v between different SCCs, sorted. Writes at most `cap` pairs and
 * always sets *n to the total. */
int gir_dev_get_dag(gir_dev_t* g, int32_t* src, int32_t* dst, int64_t cap, int64_t* n);

/* getBCTComponents / getBCT (gir.cpp:4140-4157): block b consists of the vertices v with
 * label_block[v] == b plus its parent articulation point head[b] (-1 for a root block);
 * blocks are numbered 0..n_blocks-1. Writes at most `cap` heads; *n_blocks = total. */
int gir_dev_get_blocks(gir_dev_t* g, int32_t* head, int64_t cap, int64_t* n_blocks);

/* The current directed edge set (dir 0: forward, 1: backward) or its symmetrization
 * (dir 2, self-loops dropped, gir.h:50-53) as a compact CSR: beg int64[V+1], adj int32[E].
 * getDirectedOutNeighbors / getDirectedInNeighbors / getUndirectedNeighborsPublic
 * (gir.h:160-162) are rows of these. Writes at most `cap` entries of adj; *n = total. */
int gir_dev_get_csr(gir_dev_t* g, int dir, int64_t* beg, int32_t* adj, int64_t cap, int64_t* n);

/* hasDirectedEdge / hasUndirectedEdge (gir.h:163-164) for n pairs: out[i] = 1 if present. */
int gir_dev_has_edges(gir_dev_t* g, int undirected, const int32_t* u, const int32_t* v, int64_t n, uint8_t* out);

/* ---- queries: GIR::bfs (gir_query.cpp:108-294), GIR::sssp (gir_query.cpp:695-703) ---- */

/* n_src independent BFS queries; level_out is int32[n_src][V] (row i = bfs(srcs[i]):
 * levels, -1 = unreachable; an out-of-range source gives a row of -1, gir_query.cpp:112). */
int gir_dev_bfs(gir_dev_t* g, const int32_t* srcs, int64_t n_src, int32_t* level_out);

/* n_sets multi-source BFS queries: query i starts from all of
 * set_srcs[set_beg[i] .. set_beg[i+1]) at level 0; level_out is int32[n_sets][V]. */
int gir_dev_bfs_sets(gir_dev_t* g, const int64_t* set_beg, const int32_t* set_srcs, int64_t n_sets,
                     int32_t* level_out);

/* n_src independent single-source shortest-path queries by Delta-stepping with bucket width
 * `delta` (0: the schedule chooses; the reference default is 16, gir.h:215), uint64 sums,
 * UINT64_MAX = unreachable; dist_out is uint64[n_src][V]. */
int gir_dev_sssp(gir_dev_t* g, const int32_t* srcs, int64_t n_src, uint64_t delta, int weight_mode,
                 uint64_t* dist_out);

/* Multi-source SSSP (min over each set's sources), like gir_dev_bfs_sets. */
int gir_dev_sssp_sets(gir_dev_t* g, const int64_t* set_beg, const int32_t* set_srcs, int64_t n_sets,
                      uint64_t delta, int weight_mode, uint64_t* dist_out);

/* ---- updates: applyBatch (gir.cpp:3634-4111), updateEdgeDirected/Undirected (gir.cpp:3133-3134) ---- */

/* Applies a batch of edge operations (ins[i] != 0: insert u[i] -> v[i], else delete it) with
 * the reference's batch semantics (normalizeBatch, gir.cpp:3523-3586): per edge only the last
 * operation counts, operations with u == v or an endpoint outside [0, V) are dropped, no-ops
 * are skipped. Every built layer is exact again when the call returns. New edges of a graph
 * with stored weights get weight w(u,v) = lo + hash(seed,u,v) mod (hi-lo+1) with the (seed,
 * lo, hi) set by gir_dev_set_weight_rule (default: the hash weight of GIR::edgeWeight). */
int gir_dev_apply_batch(gir_dev_t* g, const int32_t* u, const int32_t* v, const uint8_t* ins, int64_t n);

/* Deferred maintenance: ingestBatch / sync / synced (gir.h:107-116, gir.cpp:3588-3632).
 * gir_dev_ingest_batch applies a batch to the edge store only (the same batch semantics as
 * apply_batch; incremental BFS / SSSP logs see it); the WCC / SCC / block layers keep describing
 * the graph as of the last sync, so the label, DAG and block getters return that state. BFS, SSSP
 * and betweenness read the edge store and see every ingested change. gir_dev_sync brings every
 * built layer up to date with all batches ingested since the last sync, in one repair.
 * gir_dev_apply_batch, gir_dev_build and gir_dev_reachable sync first, as the reference's updates
 * and structure-based queries do. *synced = 1 when nothing is pending. */
int gir_dev_ingest_batch(gir_dev_t* g, const int32_t* u, const int32_t* v, const uint8_t* ins, int64_t n);
int gir_dev_sync(gir_dev_t* g);
int gir_dev_synced(gir_dev_t* g, int* synced);

/* Wall time (ms) of the phases of the last apply_batch: [0] normalisation and the merges into the
 * edge store, [1] WCC, [2] SCC + DAG + ranks, [3] blocks. */
int gir_dev_batch_times(gir_dev_t* g, double* ms4);

/* What the last apply_batch did to each built layer ([0] WCC, [1] SCC + DAG, [2] blocks):
 * 0 kept (the batch cannot change it), 1 patched (WCC: inserted pairs unioned into the labels;
 * SCC: labels kept, DAG and ranks rebuilt), 2 rebuilt. The reference repairs per update
 * (handleInsert / deleteEdgeImpl, gir.cpp:3007-3131); here the decision is per batch, from exact
 * sufficient conditions evaluated on the device. */
int gir_dev_batch_plan(gir_dev_t* g, int32_t* plan3);

/* Autotuner (no counterpart in the reference, whose OpenMP loops take no launch shapes): times
 * gir_dev_bfs on `srcs` (1..64 sources, host or device) for every combination of
 * GIR_PARAM_CTAS_PER_SM in {2, 4, 8}, GIR_PARAM_SMALL_DEG in {8, 32, 128} and GIR_PARAM_LARGE_DEG
 * in {1024, 4096, 32768}, best of `reps` calls each, and keeps the fastest setting on the handle
 * (read it back with gir_dev_get_param). The parameters shape launches only, so results never
 * change. *best_ms (may be NULL) = the winner's device time per call. Queues need no tuning: each
 * is sized for its exact bound (V entries, or the SSSP items' bound), allocated once per handle. */
int gir_dev_autotune(gir_dev_t* g, const int32_t* srcs, int64_t n_src, int reps, double* best_ms);

/* GIR::reachable (gir_query.cpp:789-825) for a batch: out[i] = 1 iff v[i] is reachable from u[i]
 * (1 for u == v; 0 for an id out of range). Needs the SCC layer (GIR_ERR_STATE otherwise). The
 * pairs no rank or SCC test settles run 64 at a time as lanes of one search of the condensation
 * DAG. Arrays host or device. */
int gir_dev_reachable(gir_dev_t* g, const int32_t* u, const int32_t* v, int64_t n, uint8_t* out);

/* GIR::bc (gir_query.cpp:728-778): Brandes betweenness on the directed graph, unweighted,
 * score_out[v] = sum over the n_src sources s != v of delta_s(v) (V doubles; sources repeat as
 * given, ids out of range add nothing). 64 sources share one traversal. */
int gir_dev_bc(gir_dev_t* g, const int32_t* srcs, int64_t n_src, double* score_out);

/* Incremental single-source BFS (weighted = 0) / SSSP (weighted = 1, GIR::edgeWeight weights),
 * KickStarter-style: gir_dev_inc_track replaces GIR::trackIncremental (gir_query.cpp:867-892):
 * it computes the source's result and its dependence tree, and from then on every edge a batch
 * changes is logged for that mode. gir_dev_inc_update replaces GIR::updateIncremental
 * (gir_query.cpp:894-996): it corrects the result for the logged changes (nothing to do when the
 * mode is untracked, its source is negative or nothing was logged). gir_dev_inc_dist replaces
 * GIR::incDist (gir.h:229-232) for every vertex at once: dist_out[v] (V entries, host or device)
 * = the level / distance of v, UINT64_MAX = unreachable; GIR_ERR_STATE when the mode was never
 * tracked. A source out of range tracks an all-unreachable result, as GIR::bfs / sssp give one.
 * After an update, gir_dev_query_stats gives: iterations = propagation rounds, reached = vertices
 * whose tree edge was cut (and their subtrees), edges = frontier entries relaxed. An update is one
 * cooperative launch over every co-resident CTA (its phases meet at grid barriers whose waits are
 * bounded: GIR_ERR_TIMEOUT if one runs out), read back once at the end. */
int gir_dev_inc_track(gir_dev_t* g, int32_t source, int weighted);
int gir_dev_inc_update(gir_dev_t* g, int weighted);
int gir_dev_inc_dist(gir_dev_t* g, int weighted, uint64_t* dist_out);

/* Weight rule for edges inserted into a graph with stored weights (see apply_batch). */
int gir_dev_set_weight_rule(gir_dev_t* g, uint64_t seed, uint32_t lo, uint32_t hi);

/* The single-edge latency path (insertEdge / deleteEdge, gir.cpp:3043-3134, as one-op batches):
 * a batch with exactly one effective change settles what its layer flags leave open with exact
 * device searches (u, v still connected; u still reaching v inside its SCC; no cycle closed by an
 * insert against the rank order; two vertex-disjoint u-v paths left inside the SCC, so its blocks
 * stand) instead of rebuilding the layer. Counters since create: *checked = such batches that ran
 * a search, *kept = layer rebuilds the searches avoided. Either pointer may be NULL. */
int gir_dev_single_stats(gir_dev_t* g, int64_t* checked, int64_t* kept);

/* Counters of the last apply_batch: inserted / deleted edges that changed the graph, no-op and
 * invalid operations. Any pointer may be NULL. */
int gir_dev_batch_stats(gir_dev_t* g, int64_t* n_ins, int64_t* n_del, int64_t* n_noop, int64_t* n_invalid);

/* ---- schedule, tuning and measurement ---- */

/* GIR_SCHEDULE_FIXED: the reference's fixed heuristics (direction switch alpha = 15,
 * beta = 18, gir_query.cpp:161-168; Delta = 16, gir.h:215). GIR_SCHEDULE_LEARNED: the
 * per-iteration choices come from the schedule network loaded with gir_dev_sched_set_weights.
 * Results are identical under both; only the time differs. */
int gir_dev_set_schedule(gir_dev_t* g, int mode);

/* Tunable parameters (GIR_PARAM_*): read with get, changed with set. */
enum {
    GIR_PARAM_ALPHA = 0,        /* top-down -> bottom-up when frontier edges * alpha > unexplored */
    GIR_PARAM_BETA = 1,         /* bottom-up -> top-down when frontier * beta < vertices */
    GIR_PARAM_DELTA = 2,        /* default Delta of the fixed schedule */
    GIR_PARAM_BLOCK = 3,        /* reserved, no effect: every kernel's CTA size is fixed by its shared-memory
                                   layout (the launch shape the autotuner varies is CTAs per SM) */
    GIR_PARAM_SMALL_DEG = 4,    /* degree bin: thread per vertex below this in-degree */
    GIR_PARAM_LARGE_DEG = 5,    /* degree bin: CTA per vertex from this in-degree on */
    GIR_PARAM_CTAS_PER_SM = 6,  /* grid size = SMs x this */
    GIR_PARAM_PROFILE = 7,      /* 1: time every launch of the main traversal kernel with CUDA events
                                   (gir_dev_query_stats main_ms / main_launches); 0: off */
    GIR_PARAM_PIVOT = 8,        /* forward-backward pivot rule of the SCC build: -1 the schedule decides
                                   (fixed: max out x in degree; learned: the network), or forced: 0 max
                                   out x in, 1 max out + in, 2 max in-degree, 3 no forward-backward pass
                                   (colour propagation only) */
    GIR_PARAM_LANE_BITS = 9,    /* SSSP lane distances: 0 the library decides (32 bits when every finite
                                   distance fits, else 64), or 16 / 32 / 64; 16 bits run optimistically
                                   and a group that meets a longer distance is rerun wider */
    GIR_PARAM_LANE_ORDER = 10,  /* SSSP lanes: 1 ordered by the sources' distance to the largest-in-degree
                                   vertex (lanes active in the same buckets share sectors), 0 query order */
    GIR_PARAM_COUNT = 11
};
int gir_dev_set_param(gir_dev_t* g, int which, double value);
int gir_dev_get_param(gir_dev_t* g, int which, double* value);

/* Statistics of the last query call. */
typedef struct {
    int64_t edges;          /* sum over the queries of the out-degrees of their reached vertices
                               (the traversed edges of the GTEPS figure) */
    int64_t reached;        /* sum over the queries of reached vertices */
    int64_t iterations;     /* BFS levels / SSSP rounds, summed over query groups */
    int64_t bottom_up;      /* levels run bottom-up */
    int64_t launches;       /* kernels launched by the call */
    double kernel_ms;       /* device time of the traversal kernels (CUDA events) */
    double total_ms;        /* device time of the whole call including copies */
    double main_ms;         /* with GIR_PARAM_PROFILE: summed device time of the main kernel's
                               launches (BFS: expand + bottom-up kernels; SSSP: relax) */
    int64_t main_launches;  /* ... and their number */
    int64_t persistent_levels;  /* BFS levels run inside the persistent top-down launch (small
                                   frontiers of high-diameter graphs; no reference counterpart) */
} gir_dev_query_stats_t;
int gir_dev_query_stats(gir_dev_t* g, gir_dev_query_stats_t* out);

/* The CUDA stream of the handle (a cudaStream_t), for callers that time or order work on it. */
int gir_dev_stream(gir_dev_t* g, void** stream);

/* ---- BFS without allocation ----
 *
 * No counterpart in the reference: an entry point for callers that cannot allocate memory at
 * call time -- a host engine that gives all of a GPU's memory to its own arena, or a
 * latency-critical thread that cannot afford a cudaMalloc / cudaFree (they can synchronize the
 * whole device). It computes the BFS levels of GIR::bfs (gir_query.cpp:108-294) from one source
 * over the caller's compact CSR: beg int64[V+1] and adj int32[n_adj] (the allocation's length;
 * the CSR uses adj[0 .. beg[V])), and writes level_out int32[V]. All three are device memory of
 * the current device (or managed memory); `stream` is a cudaStream_t (NULL: the default stream).
 * It allocates nothing: its working memory is a static device array sized for at most
 * GIR_NOALLOC_MAX_V vertices (16 MiB, held by every GPU that loads the library until exit);
 * larger V gives GIR_ERR_CAPACITY. The CSR is validated on the device before any level runs and
 * a bad one gives GIR_ERR_MALFORMED: beg[0] != 0, beg decreasing anywhere, beg[V] > n_adj, or an
 * id outside [0, V). A source outside [0, V) gives all -1, as GIR::bfs does (gir_query.cpp:112).
 * Errors leave their text in gir_dev_last_error(NULL). Every BFS level reads one counter back
 * to the host (a copy and a stream synchronization), so the call costs about one round trip per
 * level: high-diameter graphs pay for it. The first call on a device looks up that array's
 * device address (cudaGetSymbolAddress): make that first call before any stream capture. All
 * calls share the array: calls that overlap on the GPU (other streams, other threads) race. */
#define GIR_NOALLOC_MAX_V (1 << 21)
int gir_dev_bfs_noalloc(const int64_t* beg, const int32_t* adj, int64_t n_adj, int64_t V, int32_t source,
                        int32_t* level_out, void* stream);

/* ---- learned schedule ---- */

/* Schedule network: a 2-layer MLP (GIR_SCHED_IN features -> GIR_SCHED_HID tanh -> GIR_SCHED_OUT
 * logits), fp32, trained and evaluated by this library's own CUDA kernels. */
enum { GIR_SCHED_IN = 8, GIR_SCHED_HID = 32, GIR_SCHED_OUT = 12 };
int gir_dev_sched_set_weights(gir_dev_t* g, const float* params, int64_t n_params);
int gir_dev_sched_get_weights(gir_dev_t* g, float* params, int64_t n_params);
int64_t gir_dev_sched_param_count(void);

/* One or more SGD steps of softmax cross-entropy on (features x[n][IN], target class y[n]) on
 * the device; *loss gets the mean loss before the last step. */
int gir_dev_sched_train(gir_dev_t* g, const float* x, const int32_t* y, int64_t n, int steps, float lr, float* loss);

/* Forward pass: logits[n][OUT] for features x[n][IN]. */
int gir_dev_sched_forward(gir_dev_t* g, const float* x, int64_t n, float* logits);

/* Gradient of the mean cross-entropy w.r.t. all parameters at the current weights. */
int gir_dev_sched_grad(gir_dev_t* g, const float* x, const int32_t* y, int64_t n, float* grad, float* loss);

/* The schedule decisions of the last query call: one row per BFS level or per SSSP lane group,
 * features[n][GIR_SCHED_IN] and the class taken (0/1: top-down / bottom-up; 2..7: the Delta
 * candidates of gir_dev_sched_delta_choices). Writes at most `cap` rows; *n = total. */
int gir_dev_sched_trace(gir_dev_t* g, float* features, int32_t* choice, int64_t cap, int64_t* n);

/* The six Delta candidates of classes 2..7. */
int gir_dev_sched_delta_choices(uint64_t* out6);

#ifdef __cplusplus
}
#endif

#endif /* GIR_DEV_H */
