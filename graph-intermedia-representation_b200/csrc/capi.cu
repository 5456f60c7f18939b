// The gir_dev_* C ABI (include/gir_dev.h): handle lifetime, the four-file loader, the batch
// update pipeline, getters and query entry points.
#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"

namespace gir {

namespace {

constexpr int kBlock = 256;
thread_local std::string g_create_err;  // last failure of a call without a handle

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

// graph.cpp:95-103: offsets start at 0, end at E, never decrease; neighbour ids in [0, V).
__global__ void k_validate(const int32_t* beg, const int32_t* adj, int64_t V, int64_t E, int32_t* bad) {
    GRID_STRIDE(i, V + 1) {
        if (i == 0 && beg[0] != 0) atomicExch(bad, 1);
        if (i == V && (int64_t)beg[V] != E) atomicExch(bad, 1);
        if (i < V && beg[i] > beg[i + 1]) atomicExch(bad, 1);
    }
    GRID_STRIDE(i, E) if (adj[i] < 0 || (int64_t)adj[i] >= V) atomicExch(bad, 1);
}

// Edge keys (row << 32 | col) of an int32 CSR; `unsorted` is set if some row is not strictly
// increasing (then the keys need sorting and de-duplication).
__global__ void k_csr_keys(const int32_t* beg, const int32_t* adj, int64_t V, int64_t E, uint64_t* keys,
                           int32_t* unsorted) {
    GRID_STRIDE(i, E) {
        int64_t lo = 0, hi = V - 1;  // row: largest r with beg[r] <= i
        while (lo < hi) {
            const int64_t m = (lo + hi + 1) >> 1;
            if ((int64_t)beg[m] <= i) lo = m; else hi = m - 1;
        }
        keys[i] = ((uint64_t)lo << 32) | (uint32_t)adj[i];
        if (i > beg[lo] && adj[i - 1] >= adj[i]) atomicExch(unsorted, 1);
    }
}

__global__ void k_distinct(const uint64_t* keys, int64_t n, uint8_t* flag) {
    GRID_STRIDE(i, n) flag[i] = (i == 0 || keys[i] != keys[i - 1]);
}

// Batch: key per op (invalid ops get ~0 and sort last).
__global__ void k_batch_keys(const int32_t* u, const int32_t* v, int64_t n, int64_t V, uint64_t* keys,
                             int64_t* pos, unsigned long long* n_bad) {
    unsigned long long bad = 0;
    GRID_STRIDE(i, n) {
        const int32_t a = u[i], b = v[i];
        const bool inval = a == b || a < 0 || b < 0 || a >= V || b >= V;
        keys[i] = inval ? ~0ull : (((uint64_t)a << 32) | (uint32_t)b);
        pos[i] = i;
        bad += inval;
    }
    for (int o = 16; o; o >>= 1) bad += __shfl_xor_sync(0xffffffffu, bad, o);
    if ((threadIdx.x & 31) == 0 && bad) atomicAdd(n_bad, bad);
}

__device__ __forceinline__ bool csr_has(const CSRView& c, int64_t V, int32_t a, int32_t b) {
    if (a < 0 || a >= V) return false;
    const int64_t lo = c.beg[a], hi = lo + c.deg[a];
    const int64_t p = lower_bound_dev(c.adj, lo, hi, b);
    return p < hi && c.adj[p] == b;
}

// normalizeBatch (gir.cpp:3549-3560): the last op of each key decides, classified against the
// current edge set.
__global__ void k_batch_classify(const uint64_t* keys, const int64_t* pos, int64_t n, const uint8_t* ins, CSRView fw,
                                 int64_t V, uint8_t* f_ins, uint8_t* f_del, unsigned long long* n_noop) {
    unsigned long long noop = 0;
    GRID_STRIDE(i, n) {
        const uint64_t k = keys[i];
        uint8_t fi = 0, fd = 0;
        if (k != ~0ull && (i + 1 == n || keys[i + 1] != k)) {
            const int32_t a = (int32_t)(k >> 32), b = (int32_t)(k & 0xffffffffULL);
            const bool present = csr_has(fw, V, a, b), want = ins[pos[i]] != 0;
            if (want && !present) fi = 1;
            else if (!want && present) fd = 1;
            else noop += want;  // insert of a present edge: the C4_NOOP count of gir.cpp:3638-3640
        }
        f_ins[i] = fi;
        f_del[i] = fd;
    }
    for (int o = 16; o; o >>= 1) noop += __shfl_xor_sync(0xffffffffu, noop, o);
    if ((threadIdx.x & 31) == 0 && noop) atomicAdd(n_noop, noop);
}

__global__ void k_transpose_keys(const uint64_t* in, int64_t n, uint64_t* out) {
    GRID_STRIDE(i, n) {
        const uint64_t k = in[i];
        out[i] = (k << 32) | (k >> 32);
    }
}

// Undirected pair {min, max} of every changed edge.
__global__ void k_pair_keys(const uint64_t* a, int64_t na, const uint64_t* b, int64_t nb, uint64_t* out) {
    GRID_STRIDE(i, na + nb) {
        const uint64_t k = i < na ? a[i] : b[i - na];
        const uint64_t x = k >> 32, y = k & 0xffffffffULL;
        out[i] = x < y ? ((x << 32) | y) : ((y << 32) | x);
    }
}

__global__ void k_pair_presence(const uint64_t* pairs, int64_t n, CSRView fw, int64_t V, uint8_t* pres) {
    GRID_STRIDE(i, n) {
        const int32_t x = (int32_t)(pairs[i] >> 32), y = (int32_t)(pairs[i] & 0xffffffffULL);
        pres[i] = csr_has(fw, V, x, y) || csr_has(fw, V, y, x);
    }
}

// Symmetric ops: both directions of every pair whose undirected presence changed.
__global__ void k_sym_ops(const uint64_t* pairs, int64_t n, const uint8_t* before, CSRView fw, int64_t V,
                          uint64_t* keys2, uint8_t* f_ins, uint8_t* f_del) {
    GRID_STRIDE(i, n) {
        const uint64_t p = pairs[i];
        const int32_t x = (int32_t)(p >> 32), y = (int32_t)(p & 0xffffffffULL);
        const bool after = csr_has(fw, V, x, y) || csr_has(fw, V, y, x);
        keys2[2 * i] = p;
        keys2[2 * i + 1] = ((uint64_t)(uint32_t)y << 32) | (uint32_t)x;
        const bool add = after && !before[i], rem = !after && before[i];
        f_ins[2 * i] = f_ins[2 * i + 1] = add;
        f_del[2 * i] = f_del[2 * i + 1] = rem;
    }
}

__global__ void k_dag_split(const uint64_t* keys, int64_t n, int32_t* src, int32_t* dst) {
    GRID_STRIDE(i, n) {
        src[i] = (int32_t)(keys[i] >> 32);
        dst[i] = (int32_t)(keys[i] & 0xffffffffULL);
    }
}

// Where a call writes an output: the caller's device buffer, or the handle's staging buffer
// that is copied to the caller's host buffer afterwards.
int out_target(gir_dev* g, void* user, size_t bytes, DevBuf& stage, void** dev) {
    if (is_device_ptr(user)) { *dev = user; return GIR_OK; }
    GIR_TRY(ensure(g, stage, bytes + 16));
    *dev = stage.p;
    return GIR_OK;
}

int finish_out(gir_dev* g, void* user, void* dev, size_t bytes) {
    if (user != dev && bytes > 0) GIR_CUDA(g, cudaMemcpyAsync(user, dev, bytes, cudaMemcpyDefault, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    return GIR_OK;
}

// One direction of the store from an int32 CSR (validated): keys, sort + de-duplicate when some
// row is unsorted or repeats an entry (normalizeOneCsr, gir.cpp:95-116), slack CSR. Duplicates
// keep the weight of their first occurrence (the radix sort is stable).
int build_direction(gir_dev* g, DevCSR& c, const int32_t* beg, const int32_t* adj, int64_t E, const uint32_t* w,
                    int64_t* E_out) {
    const int64_t V = g->V;
    uint64_t *keys = nullptr, *ktmp = nullptr;
    uint32_t *wv = nullptr, *wtmp = nullptr;
    uint8_t* flag = nullptr;
    int32_t* unsorted = nullptr;
    GIR_TRY(ensure_n(g, g->work[0], E + 1, &keys));
    GIR_TRY(ensure_n(g, g->work[1], E + 1, &ktmp));
    GIR_TRY(ensure_n(g, g->work[2], E + 1, &flag));
    GIR_TRY(ensure_n(g, g->work[3], 4, &unsorted));
    if (w) {
        GIR_TRY(ensure_n(g, g->work[4], E + 1, &wv));
        GIR_TRY(ensure_n(g, g->work[5], E + 1, &wtmp));
        if (E > 0) GIR_CUDA(g, cudaMemcpyAsync(wv, w, sizeof(uint32_t) * E, cudaMemcpyDeviceToDevice, g->stream));
    }
    GIR_CUDA(g, cudaMemsetAsync(unsorted, 0, sizeof(int32_t), g->stream));
    if (E > 0) {
        k_csr_keys<<<grid_for(g, E, kBlock), kBlock, 0, g->stream>>>(beg, adj, V, E, keys, unsorted);
        GIR_LAUNCH(g, "k_csr_keys");
    }
    int32_t h_unsorted = 0;
    GIR_CUDA(g, cudaMemcpyAsync(&h_unsorted, unsorted, sizeof(int32_t), cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    int64_t n = E;
    if (h_unsorted) {
        if (w) GIR_TRY(sort_pairs_u64(g, keys, ktmp, wv, wtmp, E, 64));
        else GIR_TRY(sort_keys_u64(g, keys, ktmp, E, 64));
        k_distinct<<<grid_for(g, E, kBlock), kBlock, 0, g->stream>>>(keys, E, flag);
        GIR_LAUNCH(g, "k_distinct");
        GIR_TRY(select_flagged_u64(g, keys, flag, ktmp, E, &n));
        std::swap(keys, ktmp);
        if (w) {
            int64_t m = 0;
            GIR_TRY(select_flagged_i32(g, reinterpret_cast<const int32_t*>(wv), flag, reinterpret_cast<int32_t*>(wtmp),
                                       E, &m));
            std::swap(wv, wtmp);
        }
    }
    *E_out = n;
    return store_build_csr_from_keys(g, c, keys, n, wv);
}

int create_impl(const int32_t* fw_beg, const int32_t* fw_adj, const int32_t* bw_beg, const int32_t* bw_adj, int64_t V,
                int64_t E, const uint32_t* w, gir_dev* g) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(g, GIR_ERR_NODEVICE, "no CUDA device");
    }
    GIR_CUDA(g, cudaGetDevice(&g->device));
    GIR_CUDA(g, cudaDeviceGetAttribute(&g->num_sms, cudaDevAttrMultiProcessorCount, g->device));
    GIR_CUDA(g, cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
    {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = g->device;
        GIR_CUDA(g, cudaMemPoolCreate(&g->pool, &props));
        uint64_t keep = UINT64_MAX;  // memory stays in the pool until the handle is destroyed
        GIR_CUDA(g, cudaMemPoolSetAttribute(g->pool, cudaMemPoolAttrReleaseThreshold, &keep));
    }
    GIR_CUDA(g, cudaEventCreate(&g->ev0));
    GIR_CUDA(g, cudaEventCreate(&g->ev1));
    GIR_CUDA(g, cudaEventCreate(&g->ev2));
    GIR_CUDA(g, cudaEventCreate(&g->ev3));
    GIR_CUDA(g, cudaEventCreate(&g->pev0));
    GIR_CUDA(g, cudaEventCreate(&g->pev1));
    g->V = V;
    g->wrule_lo = 1;  // lo > hi: inserted edges get the hash weight of GIR::edgeWeight
    g->wrule_hi = 0;
    // device copies of the four arrays (and weights)
    DevBuf fb, fa, bb, ba, wb;
    const void *d_fb, *d_fa, *d_bb, *d_ba, *d_w = nullptr;
    int rc = GIR_OK;
    auto cleanup = [&]() { release(g, fb); release(g, fa); release(g, bb); release(g, ba); release(g, wb); };
    if ((rc = stage_input(g, fb, fw_beg, sizeof(int32_t) * (V + 1), &d_fb)) ||
        (rc = stage_input(g, fa, fw_adj, sizeof(int32_t) * E, &d_fa)) ||
        (rc = stage_input(g, bb, bw_beg, sizeof(int32_t) * (V + 1), &d_bb)) ||
        (rc = stage_input(g, ba, bw_adj, sizeof(int32_t) * E, &d_ba)) ||
        (w && (rc = stage_input(g, wb, w, sizeof(uint32_t) * E, &d_w)))) {
        cleanup();
        return rc;
    }
    int32_t* bad = nullptr;
    if ((rc = ensure_n(g, g->scratch[15], 8, &bad))) { cleanup(); return rc; }
    cudaMemsetAsync(bad, 0, 2 * sizeof(int32_t), g->stream);
    k_validate<<<grid_for(g, V + 1 > E ? V + 1 : E, kBlock), kBlock, 0, g->stream>>>(
        (const int32_t*)d_fb, (const int32_t*)d_fa, V, E, bad);
    k_validate<<<grid_for(g, V + 1 > E ? V + 1 : E, kBlock), kBlock, 0, g->stream>>>(
        (const int32_t*)d_bb, (const int32_t*)d_ba, V, E, bad + 1);
    int32_t hb[2] = {0, 0};
    cudaMemcpyAsync(hb, bad, sizeof(hb), cudaMemcpyDeviceToHost, g->stream);
    if ((rc = cuda_check(g, cudaStreamSynchronize(g->stream), "validate"))) { cleanup(); return rc; }
    if (hb[0] || hb[1]) {
        cleanup();
        return fail(g, GIR_ERR_MALFORMED,
                    std::string(hb[0] ? "forward" : "backward") +
                        " CSR is malformed (offsets not monotone from 0 to E, or neighbour ids outside [0,V))");
    }
    int64_t e_fw = 0, e_bw = 0;
    if ((rc = build_direction(g, g->fw, (const int32_t*)d_fb, (const int32_t*)d_fa, E, (const uint32_t*)d_w, &e_fw)) ||
        (rc = build_direction(g, g->bw, (const int32_t*)d_bb, (const int32_t*)d_ba, E, nullptr, &e_bw))) {
        cleanup();
        return rc;
    }
    cleanup();
    for (auto& b : g->work) release(g, b);
    if (e_fw != e_bw)
        return fail(g, GIR_ERR_MALFORMED, "forward and backward CSR disagree after deduplication (" +
                                              std::to_string(e_fw) + " vs " + std::to_string(e_bw) + " edges)");
    g->has_weights = w != nullptr;
    GIR_TRY(store_build_sym(g));
    // Prime the pool with one block the size of the working set, so the first build, batch and
    // query do not map new memory piece by piece. At most a quarter of the free memory.
    {
        size_t free_b = 0, total_b = 0;
        GIR_CUDA(g, cudaMemGetInfo(&free_b, &total_b));
        uint64_t reserved = 0;
        GIR_CUDA(g, cudaMemPoolGetAttribute(g->pool, cudaMemPoolAttrReservedMemCurrent, &reserved));
        // the working set: build sort keys (24 bytes per symmetric slot) and the query buffers
        // (64 lanes of SSSP distances, BFS and SSSP output staging, masks and queues: ~3 KB per
        // vertex, the high-water mark measured on a 4.8M-vertex graph); calls return their large
        // buffers to the pool after use when it would take a third of free memory
        const double need = 24.0 * (double)g->sym.cap + 3072.0 * (double)V;
        g->scratch_tight = need > (double)free_b / 3.0;
        size_t want = (size_t)need;
        want = want < free_b / 4 ? want : free_b / 4;
        if (want > reserved) {
            void* p = nullptr;
            GIR_TRY(dev_alloc(g, &p, want - reserved));
            dev_free(g, p);
        }
    }
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    if (g->trace_on) {
        uint64_t r = 0;
        cudaMemPoolGetAttribute(g->pool, cudaMemPoolAttrReservedMemCurrent, &r);
        std::fprintf(stderr, "[gir] pool reserved after create: %.1f MB\n", r / 1e6);
    }
    return GIR_OK;
}

// What a batch can change in the layers, judged with the labels from before it (flags in
// cnt[F_*]); the classes are exact sufficient conditions for keeping a layer, anything else
// rebuilds it:
//  - SCC labels stay when no edge inside an SCC is deleted and every inserted edge between
//    SCCs goes forward in the rank order (rank(u) < rank(v) for u -> v: the ranks are a
//    topological order of the condensation, which such an edge keeps acyclic). The DAG then
//    changes only if a cross edge was inserted or deleted;
//  - blocks stay when the SCCs stay and every changed symmetric pair either joins two SCCs
//    (not an edge of H) or is an inserted pair whose endpoints already share a block (a
//    block's vertices are those with it as parent block plus its head).
enum { F_SCC_SPLIT = 4, F_SCC_CYCLE = 5, F_DAG = 6, F_BCT = 7, F_N = 8 };

__global__ void k_classify_directed(const uint64_t* ins, int64_t n_ins, const uint64_t* del, int64_t n_del,
                                    const int32_t* scc, const int32_t* rank, unsigned long long* cnt) {
    bool split = false, cycle = false, dag = false;
    GRID_STRIDE(i, n_ins + n_del) {
        const bool is_ins = i < n_ins;
        const uint64_t k = is_ins ? ins[i] : del[i - n_ins];
        const int32_t u = (int32_t)(k >> 32), v = (int32_t)(k & 0xffffffffULL);
        if (scc[u] == scc[v]) {
            split |= !is_ins;
        } else {
            dag = true;
            cycle |= is_ins && rank[u] >= rank[v];
        }
    }
    if (split) cnt[F_SCC_SPLIT] = 1;
    if (cycle) cnt[F_SCC_CYCLE] = 1;
    if (dag) cnt[F_DAG] = 1;
}

__global__ void k_classify_pairs(const uint64_t* ins, int64_t n_ins, const uint64_t* del, int64_t n_del,
                                 const int32_t* scc, const int32_t* blk, const int32_t* head,
                                 unsigned long long* cnt) {
    bool bct = false;
    GRID_STRIDE(i, n_ins + n_del) {
        const bool is_ins = i < n_ins;
        const uint64_t k = is_ins ? ins[i] : del[i - n_ins];
        const int32_t u = (int32_t)(k >> 32), w = (int32_t)(k & 0xffffffffULL);
        if (scc[u] != scc[w]) continue;
        if (!is_ins) {
            bct = true;
        } else {
            const int32_t bu = blk[u], bw = blk[w];
            bct |= !(bu == bw || head[bw] == u || head[bu] == w);
        }
    }
    if (bct) cnt[F_BCT] = 1;
}

int invalidate_after_update(gir_dev* g) {
    g->bins_valid = false;
    g->ws_valid[0] = g->ws_valid[1] = false;
    return GIR_OK;
}

// Per layer: keep it, patch it (WCC: union the inserted pairs; SCC: DAG and ranks only), or
// rebuild it.
enum { KEEP = 0, PATCH = 1, REBUILD = 2 };
struct RepairPlan {
    int wcc = REBUILD, scc = REBUILD, bct = REBUILD;
    const uint64_t* pairs_in = nullptr;  // newly present undirected pairs (both orientations)
    int64_t n_pairs_in = 0;
    bool one_edge = false;  // SCC PATCH for one change that respects the ranks: one DAG key
    int32_t u = 0, v = 0;
    bool insert = false;
};

// Brings every built layer up to date, timing each (phases 1..3 of gir_dev_batch_times).
int rebuild_layers(gir_dev* g, const RepairPlan& plan) {
    double t = now_ms();
    if (g->wcc_built) {
        if (plan.wcc == REBUILD) GIR_TRY(wcc_build(g));
        else if (plan.wcc == PATCH) GIR_TRY(wcc_union_pairs(g, plan.pairs_in, plan.n_pairs_in));
    }
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    g->b_ms[1] = now_ms() - t;
    t = now_ms();
    if (g->scc_built) {
        if (plan.scc == REBUILD) GIR_TRY(scc_build(g));
        else if (plan.scc == PATCH && plan.one_edge) {
            bool patched = false;
            GIR_TRY(scc_dag_patch_one(g, plan.u, plan.v, plan.insert, &patched));
            if (patched) ++g->single_kept;
        } else if (plan.scc == PATCH) {
            GIR_TRY(scc_build_dag(g));
        }
    }
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    g->b_ms[2] = now_ms() - t;
    t = now_ms();
    if (g->bct_built && (plan.bct == REBUILD || plan.scc == REBUILD)) GIR_TRY(bct_build(g));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    g->b_ms[3] = now_ms() - t;
    return GIR_OK;
}

// The repair plan of an applied batch from its flags (judged with the labels from before it),
// its symmetric-pair changes (nsi pairs made present, keys sym_ins on the device; nsd removed) and
// its directed changes; a batch of exactly one change (one_key) asks the exact searches of
// single.cu first. Then every built layer is brought up to date.
static int plan_and_repair(gir_dev* g, const unsigned long long* fl, int64_t nsi, int64_t nsd, const uint64_t* sym_ins,
                           int64_t n_ins, int64_t n_del, uint64_t one_key) {
    RepairPlan plan;
    plan.wcc = nsd > 0 ? REBUILD : (nsi > 0 ? PATCH : KEEP);
    plan.pairs_in = sym_ins;
    plan.n_pairs_in = nsi;
    plan.scc = (fl[F_SCC_SPLIT] || fl[F_SCC_CYCLE]) ? REBUILD : (fl[F_DAG] ? PATCH : KEEP);
    plan.bct = fl[F_BCT] ? REBUILD : KEEP;
    if (n_ins + n_del == 1) {
        // one change: exact searches settle what the flags leave open (single.cu)
        SingleChecks want;
        want.wcc = g->wcc_built && nsd > 0;
        want.split = g->scc_built && fl[F_SCC_SPLIT];
        want.cycle = g->scc_built && fl[F_SCC_CYCLE];
        want.twopath = g->bct_built && fl[F_BCT] && n_del == 1 && nsd > 0;
        int32_t res[4];
        GIR_TRY(single_op_checks(g, (int32_t)(one_key >> 32), (int32_t)(uint32_t)one_key, want, res));
        if (want.wcc || want.split || want.cycle || want.twopath) ++g->single_checked;
        if (want.wcc && res[0] == 1) { plan.wcc = KEEP; ++g->single_kept; }
        if (want.wcc && res[0] == 4) {  // the component split, labels already updated in place
            plan.wcc = KEEP;
            ++g->n_wcc;
            ++g->single_kept;
        }
        if (want.split && res[1] == 1) { plan.scc = fl[F_DAG] ? PATCH : KEEP; ++g->single_kept; }
        if (want.cycle && res[2] == 2) { plan.scc = PATCH; ++g->single_kept; }
        if (want.twopath && res[3] == 1 && plan.scc != REBUILD) { plan.bct = KEEP; ++g->single_kept; }
        if (plan.scc == PATCH && !fl[F_SCC_CYCLE]) {  // a cross-SCC change along the rank order
            plan.one_edge = true;
            plan.u = (int32_t)(one_key >> 32);
            plan.v = (int32_t)(uint32_t)one_key;
            plan.insert = n_ins == 1;
        }
    }
    g->b_plan[0] = plan.wcc;
    g->b_plan[1] = plan.scc;
    g->b_plan[2] = plan.scc == REBUILD ? REBUILD : plan.bct;
    GIR_TRY(rebuild_layers(g, plan));
    return GIR_OK;
}

// The single-edge latency path for a one-op batch of host arrays: the change is applied to the
// three slack rows in place by one CTA, which also judges the layer flags (store_single_edit),
// so the batch normalisation, sorts and merges are skipped. *handled = 0 sends the op through
// the batch path (device arrays, or a row without room for an insert).
static int single_fast(gir_dev* g, const int32_t* u, const int32_t* v, const uint8_t* ins, int* handled) {
    *handled = 0;
    if (is_device_ptr(u) || is_device_ptr(v) || is_device_ptr(ins)) return GIR_OK;
    const int32_t a = *u, b = *v;
    const int insert = *ins != 0;
    const double t_start = now_ms();
    if (a == b || a < 0 || b < 0 || a >= g->V || b >= g->V) {  // dropped, as normalizeBatch does
        g->b_invalid = 1;
        *handled = 1;
        return GIR_OK;
    }
    unsigned long long* dw = nullptr;
    GIR_TRY(ensure_n(g, g->work[7], 8, &dw));
    uint64_t* keys = reinterpret_cast<uint64_t*>(dw + 4);
    GIR_TRY(store_single_edit(g, a, b, insert, dw, keys));
    void* hp = nullptr;
    GIR_TRY(pinned(g, 256, &hp));
    unsigned long long* hw = static_cast<unsigned long long*>(hp);
    GIR_CUDA(g, cudaMemcpyAsync(hw, dw, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    const unsigned long long st = hw[0], symc = hw[1], bits = hw[2];
    if (st == 2) return GIR_OK;
    *handled = 1;
    if (st == 0) {
        g->b_noop = 1;
        return GIR_OK;
    }
    const int64_t d = insert ? 1 : -1;
    g->fw.E += d;
    g->bw.E += d;
    if (symc) g->sym.E += 2 * d;
    g->b_ins = insert;
    g->b_del = !insert;
    GIR_TRY(inc_log(g, keys, insert, keys, !insert));
    GIR_TRY(invalidate_after_update(g));
    g->b_ms[0] = now_ms() - t_start;
    unsigned long long fl[F_N] = {};
    fl[F_SCC_SPLIT] = bits & 1;
    fl[F_SCC_CYCLE] = (bits >> 1) & 1;
    fl[F_DAG] = (bits >> 2) & 1;
    fl[F_BCT] = (bits >> 3) & 1;
    const uint64_t one_key = ((uint64_t)(uint32_t)a << 32) | (uint32_t)b;
    // (a pair that appeared inside one weakly connected component unions nothing)
    const int64_t nsi = symc == 1 && !((bits >> 4) & 1) ? 2 : 0;
    return plan_and_repair(g, fl, nsi, symc == 2 ? 2 : 0, keys + 1, insert, !insert, one_key);
}

// sync (gir.cpp:3602-3632): the layers catch up with every batch ingested since the last sync,
// in one repair whose plan joins what each of those batches could change.
int sync_impl(gir_dev* g) {
    if (!g->pend) return GIR_OK;
    RepairPlan plan;
    plan.wcc = g->pend_wcc_del ? REBUILD : (g->n_pend_pairs > 0 ? PATCH : KEEP);
    plan.pairs_in = static_cast<const uint64_t*>(g->pend_pairs.p);
    plan.n_pairs_in = g->n_pend_pairs;
    plan.scc = (g->pend_scc_split || g->pend_scc_cycle) ? REBUILD : (g->pend_dag ? PATCH : KEEP);
    plan.bct = g->pend_bct ? REBUILD : KEEP;
    for (double& x : g->b_ms) x = 0;
    g->b_plan[0] = plan.wcc;
    g->b_plan[1] = plan.scc;
    g->b_plan[2] = plan.scc == REBUILD ? REBUILD : plan.bct;
    GIR_TRY(rebuild_layers(g, plan));
    g->pend = g->pend_scc_split = g->pend_scc_cycle = g->pend_dag = g->pend_bct = g->pend_wcc_del = false;
    g->n_pend_pairs = 0;
    return GIR_OK;
}

// Filter-Merge-Update on the device (applyBatch, gir.cpp:3634-4111): normalise the batch,
// merge it into the forward, backward and symmetrized slack CSRs, then bring every built layer
// up to date. With `deferred` (ingestBatch, gir.cpp:3588-3596) the layers are left as they are
// and what the batch can change is added to the pending plan for the next sync; otherwise
// pending batches are synced first, as the reference's applyBatch does.
int apply_batch_impl(gir_dev* g, const int32_t* u, const int32_t* v, const uint8_t* ins, int64_t n, bool deferred) {
    const int64_t V = g->V;
    if (!deferred) GIR_TRY(sync_impl(g));
    g->b_ins = g->b_del = g->b_noop = g->b_invalid = 0;
    for (double& x : g->b_ms) x = 0;
    for (int& x : g->b_plan) x = 0;  // (a batch without effective ops keeps every layer)
    const double t_start = now_ms();
    if (n <= 0) return GIR_OK;
    if (n == 1 && !deferred) {
        int handled = 0;
        GIR_TRY(single_fast(g, u, v, ins, &handled));
        if (handled) return GIR_OK;
    }
    trace_mark(g, "batch: start");
    const void *du, *dv, *dins;
    DevBuf su, sv, si;
    int rc = GIR_OK;
    auto cleanup = [&]() { release(g, su); release(g, sv); release(g, si); };
    if ((rc = stage_input(g, su, u, sizeof(int32_t) * n, &du)) || (rc = stage_input(g, sv, v, sizeof(int32_t) * n, &dv)) ||
        (rc = stage_input(g, si, ins, n, &dins))) {
        cleanup();
        return rc;
    }
    uint64_t *keys = nullptr, *ktmp = nullptr, *ins_k = nullptr, *del_k = nullptr, *tk = nullptr;
    int64_t *pos = nullptr, *ptmp = nullptr;
    uint8_t *f_ins = nullptr, *f_del = nullptr;
    unsigned long long* cnt = nullptr;
    if ((rc = ensure_n(g, g->work[0], n + 1, &keys)) || (rc = ensure_n(g, g->work[1], n + 1, &ktmp)) ||
        (rc = ensure_n(g, g->work[2], n + 1, &pos)) || (rc = ensure_n(g, g->work[3], n + 1, &ptmp)) ||
        (rc = ensure_n(g, g->work[4], 2 * n + 2, &f_ins)) || (rc = ensure_n(g, g->work[5], n + 1, &ins_k)) ||
        (rc = ensure_n(g, g->work[6], n + 1, &del_k)) || (rc = ensure_n(g, g->work[7], F_N, &cnt))) {
        cleanup();
        return rc;
    }
    f_del = f_ins + n + 1;
    cudaMemsetAsync(cnt, 0, F_N * sizeof(unsigned long long), g->stream);
    k_batch_keys<<<grid_for(g, n, kBlock), kBlock, 0, g->stream>>>((const int32_t*)du, (const int32_t*)dv, n, V, keys,
                                                                   pos, cnt);
    if ((rc = cuda_check(g, cudaGetLastError(), "k_batch_keys")) ||
        (rc = sort_pairs_u64_i64(g, keys, ktmp, pos, ptmp, n, 64))) {
        cleanup();
        return rc;
    }
    k_batch_classify<<<grid_for(g, n, kBlock), kBlock, 0, g->stream>>>(keys, pos, n, (const uint8_t*)dins, view(g->fw),
                                                                       V, f_ins, f_del, cnt + 1);
    int64_t n_ins = 0, n_del = 0;
    if ((rc = cuda_check(g, cudaGetLastError(), "k_batch_classify")) ||
        (rc = select_flagged_u64(g, keys, f_ins, ins_k, n, &n_ins)) ||
        (rc = select_flagged_u64(g, keys, f_del, del_k, n, &n_del))) {
        cleanup();
        return rc;
    }
    unsigned long long hc[2] = {0, 0};
    cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, g->stream);
    uint64_t one_key = 0;  // the change of a batch with exactly one (the single-edge latency path)
    if (n_ins + n_del == 1)
        cudaMemcpyAsync(&one_key, n_ins ? ins_k : del_k, sizeof(uint64_t), cudaMemcpyDeviceToHost, g->stream);
    if ((rc = cuda_check(g, cudaStreamSynchronize(g->stream), "batch counters"))) { cleanup(); return rc; }
    cleanup();
    g->b_invalid = (int64_t)hc[0];
    g->b_noop = (int64_t)hc[1];
    g->b_ins = n_ins;
    g->b_del = n_del;
    if (n_ins + n_del == 0) return GIR_OK;
    GIR_TRY(inc_log(g, ins_k, n_ins, del_k, n_del));
    trace_mark(g, "batch: normalize");
    if (g->scc_built) {
        k_classify_directed<<<grid_for(g, n_ins + n_del, kBlock), kBlock, 0, g->stream>>>(
            ins_k, n_ins, del_k, n_del, static_cast<const int32_t*>(g->scc.p), static_cast<const int32_t*>(g->scc_rank.p),
            cnt);
        GIR_LAUNCH(g, "k_classify_directed");
    }

    // undirected pairs touched, with their presence before the batch
    const int64_t np = n_ins + n_del;
    uint64_t *pairs = nullptr, *ptmp2 = nullptr, *sym_keys = nullptr, *sym_ins = nullptr, *sym_del = nullptr;
    uint8_t *before = nullptr, *pflag = nullptr, *fsi = nullptr, *fsd = nullptr;
    GIR_TRY(ensure_n(g, g->work[0], np + 1, &pairs));
    GIR_TRY(ensure_n(g, g->work[1], np + 1, &ptmp2));
    GIR_TRY(ensure_n(g, g->work[2], 2 * np + 2, &sym_keys));
    GIR_TRY(ensure_n(g, g->work[3], 6 * np + 6, &before));
    pflag = before + np + 1;
    fsi = pflag + np + 1;
    fsd = fsi + 2 * np + 2;
    k_pair_keys<<<grid_for(g, np, kBlock), kBlock, 0, g->stream>>>(ins_k, n_ins, del_k, n_del, pairs);
    GIR_LAUNCH(g, "k_pair_keys");
    GIR_TRY(sort_keys_u64(g, pairs, ptmp2, np, 64));
    k_distinct<<<grid_for(g, np, kBlock), kBlock, 0, g->stream>>>(pairs, np, pflag);
    GIR_LAUNCH(g, "k_distinct");
    int64_t npu = 0;
    GIR_TRY(select_flagged_u64(g, pairs, pflag, ptmp2, np, &npu));
    std::swap(pairs, ptmp2);
    k_pair_presence<<<grid_for(g, npu, kBlock), kBlock, 0, g->stream>>>(pairs, npu, view(g->fw), V, before);
    GIR_LAUNCH(g, "k_pair_presence");

    trace_mark(g, "batch: pairs");
    // forward, then backward (transposed keys, re-sorted)
    GIR_TRY(store_apply_ops(g, g->fw, ins_k, n_ins, del_k, n_del, true));
    trace_mark(g, "batch: forward ops");
    GIR_TRY(ensure_n(g, g->work[4], np + 2, &tk));
    uint64_t* tk2 = tk + n_ins + 1;
    if (n_ins) {
        k_transpose_keys<<<grid_for(g, n_ins, kBlock), kBlock, 0, g->stream>>>(ins_k, n_ins, tk);
        GIR_LAUNCH(g, "k_transpose_keys");
        GIR_TRY(sort_keys_u64(g, tk, ins_k, n_ins, 64));
    }
    if (n_del) {
        k_transpose_keys<<<grid_for(g, n_del, kBlock), kBlock, 0, g->stream>>>(del_k, n_del, tk2);
        GIR_LAUNCH(g, "k_transpose_keys");
        GIR_TRY(sort_keys_u64(g, tk2, del_k, n_del, 64));
    }
    GIR_TRY(store_apply_ops(g, g->bw, tk, n_ins, tk2, n_del, false));
    trace_mark(g, "batch: backward ops");

    // symmetrized view: pairs whose undirected presence changed
    k_sym_ops<<<grid_for(g, npu, kBlock), kBlock, 0, g->stream>>>(pairs, npu, before, view(g->fw), V, sym_keys, fsi, fsd);
    GIR_LAUNCH(g, "k_sym_ops");
    GIR_TRY(ensure_n(g, g->work[5], 2 * npu + 2, &sym_ins));
    GIR_TRY(ensure_n(g, g->work[6], 2 * npu + 2, &sym_del));
    int64_t nsi = 0, nsd = 0;
    GIR_TRY(select_flagged_u64(g, sym_keys, fsi, sym_ins, 2 * npu, &nsi));
    GIR_TRY(select_flagged_u64(g, sym_keys, fsd, sym_del, 2 * npu, &nsd));
    GIR_TRY(sort_keys_u64(g, sym_ins, sym_keys, nsi, 64));
    GIR_TRY(sort_keys_u64(g, sym_del, sym_keys, nsd, 64));
    if (g->bct_built && nsi + nsd > 0) {
        k_classify_pairs<<<grid_for(g, nsi + nsd, kBlock), kBlock, 0, g->stream>>>(
            sym_ins, nsi, sym_del, nsd, static_cast<const int32_t*>(g->scc.p), static_cast<const int32_t*>(g->blk_label.p),
            static_cast<const int32_t*>(g->blk_head.p), cnt);
        GIR_LAUNCH(g, "k_classify_pairs");
    }
    GIR_TRY(store_apply_ops(g, g->sym, sym_ins, nsi, sym_del, nsd, false));
    trace_mark(g, "batch: symmetric ops");

    GIR_TRY(invalidate_after_update(g));
    unsigned long long fl[F_N] = {};
    GIR_CUDA(g, cudaMemcpyAsync(fl, cnt, sizeof(fl), cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    g->b_ms[0] = now_ms() - t_start;
    if (deferred) {
        g->pend = true;
        g->pend_wcc_del |= nsd > 0;
        g->pend_scc_split |= fl[F_SCC_SPLIT] != 0;
        g->pend_scc_cycle |= fl[F_SCC_CYCLE] != 0;
        g->pend_dag |= fl[F_DAG] != 0;
        g->pend_bct |= fl[F_BCT] != 0;
        if (nsi > 0 && g->wcc_built) {
            uint64_t* keep = nullptr;
            const size_t need = (size_t)(g->n_pend_pairs + nsi);
            if (g->pend_pairs.bytes < need * sizeof(uint64_t) + 16) {  // grow, keeping the pairs so far
                DevBuf nb;
                GIR_TRY(ensure_n(g, nb, 2 * need, &keep));
                if (g->n_pend_pairs)
                    GIR_CUDA(g, cudaMemcpyAsync(keep, g->pend_pairs.p, sizeof(uint64_t) * g->n_pend_pairs,
                                                cudaMemcpyDeviceToDevice, g->stream));
                release(g, g->pend_pairs);
                g->pend_pairs = nb;
            }
            keep = static_cast<uint64_t*>(g->pend_pairs.p);
            GIR_CUDA(g, cudaMemcpyAsync(keep + g->n_pend_pairs, sym_ins, sizeof(uint64_t) * nsi, cudaMemcpyDeviceToDevice,
                                        g->stream));
            g->n_pend_pairs += nsi;
        }
        return GIR_OK;
    }
    return plan_and_repair(g, fl, nsi, nsd, sym_ins, n_ins, n_del, one_key);
}

int read_file_ints(const std::string& path, std::vector<int32_t>& out, int64_t n, gir_dev* g) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return fail(g, GIR_ERR_FILE, path + " cannot open");
    out.resize((size_t)(n > 0 ? n : 1));
    const size_t got = n > 0 ? std::fread(out.data(), sizeof(int32_t), (size_t)n, f) : 0;
    std::fclose(f);
    if ((int64_t)got != n) return fail(g, GIR_ERR_FILE, path + " is shorter than its size says");
    return GIR_OK;
}

int64_t file_size(const std::string& p) {
    struct stat st;
    return stat(p.c_str(), &st) == 0 ? (int64_t)st.st_size : -1;
}

int query_sets(gir_dev* g, const int64_t* set_beg_user, const int32_t* srcs, int64_t n_sets, bool bfs, uint64_t delta,
               int weight_mode, void* out_user) {
    if (!g) return GIR_ERR_INVALID;
    if (n_sets < 0 || (n_sets > 0 && (!set_beg_user || !out_user))) return fail(g, GIR_ERR_INVALID, "query: bad arguments");
    if (!bfs && weight_mode != GIR_WEIGHT_HASH && weight_mode != GIR_WEIGHT_STORED)
        return fail(g, GIR_ERR_INVALID, "sssp: unknown weight mode");
    cudaEvent_t t0 = g->ev2, t1 = g->ev3;
    GIR_CUDA(g, cudaEventRecord(t0, g->stream));
    std::vector<int64_t> sb((size_t)n_sets + 1, 0);
    if (n_sets > 0) {
        if (is_device_ptr(set_beg_user)) {
            GIR_CUDA(g, cudaMemcpy(sb.data(), set_beg_user, sizeof(int64_t) * (n_sets + 1), cudaMemcpyDeviceToHost));
        } else {
            std::memcpy(sb.data(), set_beg_user, sizeof(int64_t) * (n_sets + 1));
        }
    }
    for (int64_t i = 0; i < n_sets; ++i)
        if (sb[i + 1] < sb[i] || sb[0] < 0) return fail(g, GIR_ERR_INVALID, "query: set offsets decrease");
    const int64_t n_src = n_sets > 0 ? sb[n_sets] : 0;
    if (n_src > 0 && !srcs) return fail(g, GIR_ERR_INVALID, "query: null sources");
    const void* d_src = nullptr;
    GIR_TRY(stage_input(g, g->stage_in, srcs, sizeof(int32_t) * (n_src > 0 ? n_src : 0), &d_src));
    const size_t elem = bfs ? sizeof(int32_t) : sizeof(uint64_t);
    const size_t bytes = elem * (size_t)g->V * (size_t)n_sets;
    void* d_out = nullptr;
    GIR_TRY(out_target(g, out_user, bytes, g->stage_out, &d_out));
    if (bfs) GIR_TRY(bfs_run(g, sb.data(), (const int32_t*)d_src, n_sets, (int32_t*)d_out));
    else GIR_TRY(sssp_run(g, sb.data(), (const int32_t*)d_src, n_sets, delta, weight_mode, (uint64_t*)d_out));
    if (out_user != d_out && bytes > 0)
        GIR_CUDA(g, cudaMemcpyAsync(out_user, d_out, bytes, cudaMemcpyDefault, g->stream));
    GIR_CUDA(g, cudaEventRecord(t1, g->stream));
    GIR_CUDA(g, cudaEventSynchronize(t1));
    float ms = 0;
    GIR_CUDA(g, cudaEventElapsedTime(&ms, t0, t1));
    g->qstats.total_ms = ms;
    release_scratch(g, kKeepScratchBelow);
    return GIR_OK;
}

}  // namespace

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void trace_mark(gir_dev* g, const char* what) {
    if (!g->trace_marks) return;
    cudaStreamSynchronize(g->stream);
    const double t = now_ms();
    std::fprintf(stderr, "[gir] %-28s %9.3f ms\n", what, g->trace_t > 0 ? t - g->trace_t : 0.0);
    g->trace_t = t;
}

void set_thread_error(const std::string& msg) { g_create_err = msg; }

}  // namespace gir

using namespace gir;

extern "C" {

const char* gir_dev_last_error(const gir_dev_t* g) { return g ? g->err.c_str() : g_create_err.c_str(); }

int gir_dev_create(const int32_t* fw_beg, const int32_t* fw_adj, const int32_t* bw_beg, const int32_t* bw_adj,
                   int64_t V, int64_t E, const uint32_t* w, gir_dev_t** out) {
    g_create_err.clear();
    if (!out) { g_create_err = "gir_dev_create: null output handle"; return GIR_ERR_INVALID; }
    *out = nullptr;
    if (V < 0 || V >= INT32_MAX || E < 0 || E > INT32_MAX || !fw_beg || !bw_beg || (E > 0 && (!fw_adj || !bw_adj))) {
        g_create_err = "gir_dev_create: bad sizes or null arrays (V in [0, 2^31-1), E in [0, 2^31))";
        return GIR_ERR_INVALID;
    }
    gir_dev* g = new gir_dev();
    const int rc = create_impl(fw_beg, fw_adj, bw_beg, bw_adj, V, E, w, g);
    if (rc != GIR_OK) {
        g_create_err = g->err;
        gir_dev_destroy(g);
        return rc;
    }
    *out = g;
    return GIR_OK;
}

int gir_dev_load(const char* dir, gir_dev_t** out) {
    g_create_err.clear();
    if (!out || !dir) { g_create_err = "gir_dev_load: null argument"; return GIR_ERR_INVALID; }
    *out = nullptr;
    const std::string d(dir);
    const int64_t s_fb = file_size(d + "fw_begin.bin"), s_fa = file_size(d + "fw_adjacent.bin");
    const int64_t s_bb = file_size(d + "bw_begin.bin"), s_ba = file_size(d + "bw_adjacent.bin");
    if (s_fb < 0 || s_fa < 0 || s_bb < 0 || s_ba < 0) {
        g_create_err = d + ": one of fw_begin.bin, fw_adjacent.bin, bw_begin.bin, bw_adjacent.bin cannot open";
        return GIR_ERR_FILE;
    }
    // graph.cpp:14-15: V = |fw_begin| / 4 - 1, E = |fw_adjacent| / 4
    const int64_t V = s_fb / 4 - 1, E = s_fa / 4;
    if (V < 0) { g_create_err = d + "fw_begin.bin holds no offsets"; return GIR_ERR_MALFORMED; }
    if (s_bb / 4 - 1 != V || s_ba / 4 != E) {
        g_create_err = "forward CSR has " + std::to_string(V) + " vertices / " + std::to_string(E) +
                       " edges but backward CSR files hold " + std::to_string(s_bb / 4 - 1) + " / " +
                       std::to_string(s_ba / 4) + " entries";
        return GIR_ERR_MALFORMED;
    }
    std::vector<int32_t> fb, fa, bb, ba;
    gir_dev tmp;  // error sink for the reads
    if (read_file_ints(d + "fw_begin.bin", fb, V + 1, &tmp) || read_file_ints(d + "fw_adjacent.bin", fa, E, &tmp) ||
        read_file_ints(d + "bw_begin.bin", bb, V + 1, &tmp) || read_file_ints(d + "bw_adjacent.bin", ba, E, &tmp)) {
        g_create_err = tmp.err;
        return GIR_ERR_FILE;
    }
    return gir_dev_create(fb.data(), fa.data(), bb.data(), ba.data(), V, E, nullptr, out);
}

int gir_dev_destroy(gir_dev_t* g) {
    if (!g) return GIR_OK;
    if (g->stream && g->pool) {
        store_free(g, g->fw); store_free(g, g->bw); store_free(g, g->sym);
        store_free(g, g->ws[0]); store_free(g, g->ws[1]);
        for (DevBuf* b : {&g->wcc, &g->scc, &g->scc_rank, &g->dag, &g->dag_rows, &g->reach_hub, &g->blk_label, &g->blk_head, &g->bcnt, &g->bins,
                          &g->cub_tmp, &g->stage_in, &g->stage_out, &g->sched_w, &g->sched_io, &g->lane_dist, &g->inc_st[0], &g->inc_st[1],
                          &g->inc_pend[0], &g->inc_pend[1], &g->single_ws, &g->hub_dist[0], &g->hub_dist[1], &g->sssp_sets, &g->sssp_lanes, &g->sssp_done, &g->pend_pairs})
            release(g, *b);
        for (auto& b : g->scratch) release(g, b);
        for (auto& b : g->work) release(g, b);
        for (auto& b : g->qitems) release(g, b);
    }
    if (g->stream) cudaStreamSynchronize(g->stream);
    if (g->pool && g->trace_on) {
        uint64_t hi = 0, used_hi = 0;
        cudaMemPoolGetAttribute(g->pool, cudaMemPoolAttrReservedMemHigh, &hi);
        cudaMemPoolGetAttribute(g->pool, cudaMemPoolAttrUsedMemHigh, &used_hi);
        std::fprintf(stderr, "[gir] pool high-water: reserved %.1f MB, used %.1f MB\n", hi / 1e6, used_hi / 1e6);
    }
    if (g->pool) cudaMemPoolDestroy(g->pool);
    if (g->pinned) cudaFreeHost(g->pinned);
    for (cudaEvent_t e : {g->ev0, g->ev1, g->ev2, g->ev3, g->pev0, g->pev1}) if (e) cudaEventDestroy(e);
    if (g->stream) cudaStreamDestroy(g->stream);
    delete g;
    return GIR_OK;
}

int gir_dev_counts(gir_dev_t* g, int64_t* V, int64_t* E, int64_t* n_wcc, int64_t* n_scc, int64_t* n_dag,
                   int64_t* n_blocks) {
    if (!g) return GIR_ERR_INVALID;
    if (V) *V = g->V;
    if (E) *E = g->fw.E;
    if (n_wcc) *n_wcc = g->wcc_built ? g->n_wcc : -1;
    if (n_scc) *n_scc = g->scc_built ? g->n_scc : -1;
    if (n_dag) *n_dag = g->scc_built ? g->n_dag : -1;
    if (n_blocks) *n_blocks = g->bct_built ? g->n_blocks : -1;
    return GIR_OK;
}

int gir_dev_build(gir_dev_t* g, unsigned layers) {
    if (!g) return GIR_ERR_INVALID;
    if (layers & ~7u) return fail(g, GIR_ERR_INVALID, "gir_dev_build: unknown layer bits");
    GIR_TRY(sync_impl(g));  // (the layers built so far catch up with ingested batches first)
    if (layers & GIR_LAYER_WCC) GIR_TRY(wcc_build(g));
    if (layers & GIR_LAYER_SCC) GIR_TRY(scc_build(g));
    if (layers & GIR_LAYER_BCT) {
        if (!g->scc_built) return fail(g, GIR_ERR_STATE, "buildBCT needs buildSCC_DAG first (gir.h:98)");
        GIR_TRY(bct_build(g));
    }
    release_scratch(g, kKeepScratchBelow);
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    return GIR_OK;
}

int gir_dev_get_labels(gir_dev_t* g, int which, int32_t* out) {
    if (!g || !out) return g ? fail(g, GIR_ERR_INVALID, "get_labels: null output") : GIR_ERR_INVALID;
    const DevBuf* src = nullptr;
    switch (which) {
        case GIR_LABEL_WCC:
            if (!g->wcc_built) return fail(g, GIR_ERR_STATE, "WCC layer not built");
            src = &g->wcc; break;
        case GIR_LABEL_SCC:
            if (!g->scc_built) return fail(g, GIR_ERR_STATE, "SCC layer not built");
            src = &g->scc; break;
        case GIR_LABEL_BLOCK:
            if (!g->bct_built) return fail(g, GIR_ERR_STATE, "BCT layer not built");
            src = &g->blk_label; break;
        case GIR_LABEL_BCNT:
            if (!g->bct_built) return fail(g, GIR_ERR_STATE, "BCT layer not built");
            src = &g->bcnt; break;
        case GIR_LABEL_SCC_RANK:
            if (!g->scc_built) return fail(g, GIR_ERR_STATE, "SCC layer not built");
            src = &g->scc_rank; break;
        default: return fail(g, GIR_ERR_INVALID, "get_labels: unknown label kind");
    }
    if (g->V == 0) return GIR_OK;
    GIR_CUDA(g, cudaMemcpyAsync(out, src->p, sizeof(int32_t) * g->V, cudaMemcpyDefault, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    return GIR_OK;
}

int gir_dev_get_dag(gir_dev_t* g, int32_t* src, int32_t* dst, int64_t cap, int64_t* n) {
    if (!g || !n || cap < 0) return g ? fail(g, GIR_ERR_INVALID, "get_dag: bad arguments") : GIR_ERR_INVALID;
    if (!g->scc_built) return fail(g, GIR_ERR_STATE, "SCC layer not built");
    *n = g->n_dag;
    const int64_t m = cap < g->n_dag ? cap : g->n_dag;
    if (m == 0) return GIR_OK;
    if (!src || !dst) return fail(g, GIR_ERR_INVALID, "get_dag: null output");
    int32_t *ds = nullptr, *dd = nullptr;
    GIR_TRY(ensure_n(g, g->stage_out, 2 * m + 2, &ds));
    dd = ds + m + 1;
    k_dag_split<<<grid_for(g, m, kBlock), kBlock, 0, g->stream>>>(static_cast<const uint64_t*>(g->dag.p), m, ds, dd);
    GIR_LAUNCH(g, "k_dag_split");
    GIR_CUDA(g, cudaMemcpyAsync(src, ds, sizeof(int32_t) * m, cudaMemcpyDefault, g->stream));
    GIR_CUDA(g, cudaMemcpyAsync(dst, dd, sizeof(int32_t) * m, cudaMemcpyDefault, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    return GIR_OK;
}

int gir_dev_get_blocks(gir_dev_t* g, int32_t* head, int64_t cap, int64_t* n_blocks) {
    if (!g || !n_blocks || cap < 0) return g ? fail(g, GIR_ERR_INVALID, "get_blocks: bad arguments") : GIR_ERR_INVALID;
    if (!g->bct_built) return fail(g, GIR_ERR_STATE, "BCT layer not built");
    *n_blocks = g->n_blocks;
    const int64_t m = cap < g->n_blocks ? cap : g->n_blocks;
    if (m == 0) return GIR_OK;
    if (!head) return fail(g, GIR_ERR_INVALID, "get_blocks: null output");
    GIR_CUDA(g, cudaMemcpyAsync(head, g->blk_head.p, sizeof(int32_t) * m, cudaMemcpyDefault, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    return GIR_OK;
}

int gir_dev_get_csr(gir_dev_t* g, int dir, int64_t* beg, int32_t* adj, int64_t cap, int64_t* n) {
    if (!g || !n || cap < 0 || dir < 0 || dir > 2)
        return g ? fail(g, GIR_ERR_INVALID, "get_csr: bad arguments") : GIR_ERR_INVALID;
    const DevCSR& c = dir == 0 ? g->fw : dir == 1 ? g->bw : g->sym;
    *n = c.E;
    if (!beg) return GIR_OK;
    int64_t* db = nullptr;
    int32_t* da = nullptr;
    const int64_t m = cap < c.E ? cap : c.E;
    GIR_TRY(ensure_n(g, g->stage_in, g->V + 2, &db));
    GIR_TRY(ensure_n(g, g->stage_out, m + 2, &da));
    GIR_TRY(store_compact_csr(g, c, db, da, m));
    GIR_CUDA(g, cudaMemcpyAsync(beg, db, sizeof(int64_t) * (g->V + 1), cudaMemcpyDefault, g->stream));
    if (adj && m > 0) GIR_CUDA(g, cudaMemcpyAsync(adj, da, sizeof(int32_t) * m, cudaMemcpyDefault, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    return GIR_OK;
}

int gir_dev_has_edges(gir_dev_t* g, int undirected, const int32_t* u, const int32_t* v, int64_t n, uint8_t* out) {
    if (!g || n < 0 || (n > 0 && (!u || !v || !out))) return g ? fail(g, GIR_ERR_INVALID, "has_edges: bad arguments") : GIR_ERR_INVALID;
    if (n == 0) return GIR_OK;
    const void *du, *dv;
    DevBuf su, sv;
    int rc = stage_input(g, su, u, sizeof(int32_t) * n, &du);
    if (!rc) rc = stage_input(g, sv, v, sizeof(int32_t) * n, &dv);
    void* dout = nullptr;
    if (!rc) rc = out_target(g, out, (size_t)n, g->stage_out, &dout);
    if (!rc) rc = store_has_edges(g, undirected ? g->sym : g->fw, (const int32_t*)du, (const int32_t*)dv, n, (uint8_t*)dout);
    if (!rc) rc = finish_out(g, out, dout, (size_t)n);
    release(g, su); release(g, sv);
    return rc;
}

int gir_dev_bfs(gir_dev_t* g, const int32_t* srcs, int64_t n_src, int32_t* level_out) {
    if (!g) return GIR_ERR_INVALID;
    if (n_src < 0) return fail(g, GIR_ERR_INVALID, "bfs: negative source count");
    std::vector<int64_t> sb((size_t)n_src + 1);
    for (int64_t i = 0; i <= n_src; ++i) sb[i] = i;
    return query_sets(g, sb.data(), srcs, n_src, true, 0, 0, level_out);
}

int gir_dev_autotune(gir_dev_t* g, const int32_t* srcs, int64_t n_src, int reps, double* best_ms) {
    if (!g) return GIR_ERR_INVALID;
    if (n_src < 1 || n_src > 64 || !srcs || reps < 1)
        return fail(g, GIR_ERR_INVALID, "autotune: need 1..64 sources and reps >= 1");
    std::vector<int64_t> sb((size_t)n_src + 1);
    for (int64_t i = 0; i <= n_src; ++i) sb[i] = i;
    void* out = nullptr;
    GIR_TRY(dev_alloc(g, &out, sizeof(int32_t) * (size_t)g->V * (size_t)n_src + 16));
    const double keep[3] = {g->params[GIR_PARAM_CTAS_PER_SM], g->params[GIR_PARAM_SMALL_DEG],
                            g->params[GIR_PARAM_LARGE_DEG]};
    double best = 1e300, choice[3] = {keep[0], keep[1], keep[2]};
    int rc = GIR_OK;
    for (double ctas : {2.0, 4.0, 8.0})
        for (double small : {8.0, 32.0, 128.0})
            for (double large : {1024.0, 4096.0, 32768.0}) {
                g->params[GIR_PARAM_CTAS_PER_SM] = ctas;
                g->params[GIR_PARAM_SMALL_DEG] = small;
                g->params[GIR_PARAM_LARGE_DEG] = large;
                g->bins_valid = false;  // (the degree bins depend on the thresholds)
                rc = query_sets(g, sb.data(), srcs, n_src, true, 0, 0, out);  // untimed: builds the bins
                double t = 1e300;
                for (int r = 0; rc == GIR_OK && r < reps; ++r) {
                    rc = query_sets(g, sb.data(), srcs, n_src, true, 0, 0, out);
                    t = std::min(t, g->qstats.total_ms);
                }
                if (rc != GIR_OK) break;
                if (t < best) {
                    best = t;
                    choice[0] = ctas; choice[1] = small; choice[2] = large;
                }
            }
    dev_free(g, out);
    g->params[GIR_PARAM_CTAS_PER_SM] = rc == GIR_OK ? choice[0] : keep[0];
    g->params[GIR_PARAM_SMALL_DEG] = rc == GIR_OK ? choice[1] : keep[1];
    g->params[GIR_PARAM_LARGE_DEG] = rc == GIR_OK ? choice[2] : keep[2];
    g->bins_valid = false;
    if (rc != GIR_OK) return rc;
    if (best_ms) *best_ms = best;
    return GIR_OK;
}

int gir_dev_bc(gir_dev_t* g, const int32_t* srcs, int64_t n_src, double* score_out) {
    if (!g) return GIR_ERR_INVALID;
    if (n_src < 0 || !score_out || (n_src > 0 && !srcs)) return fail(g, GIR_ERR_INVALID, "bc: bad arguments");
    DevBuf ss;
    const void* ds = nullptr;
    void* dout = nullptr;
    int rc = GIR_OK;
    if (!(rc = stage_input(g, ss, srcs, sizeof(int32_t) * n_src, &ds)) &&
        !(rc = out_target(g, score_out, sizeof(double) * (size_t)g->V, g->stage_out, &dout)) &&
        !(rc = bc_run(g, (const int32_t*)ds, n_src, (double*)dout)))
        rc = finish_out(g, score_out, dout, sizeof(double) * (size_t)g->V);
    release(g, ss);
    release_scratch(g, kKeepScratchBelow);
    return rc;
}

int gir_dev_single_stats(gir_dev_t* g, int64_t* checked, int64_t* kept) {
    if (!g) return GIR_ERR_INVALID;
    if (checked) *checked = g->single_checked;
    if (kept) *kept = g->single_kept;
    return GIR_OK;
}

int gir_dev_inc_track(gir_dev_t* g, int32_t source, int weighted) {
    if (!g) return GIR_ERR_INVALID;
    const int rc = inc_track(g, source, weighted ? 1 : 0);
    release_scratch(g, kKeepScratchBelow);
    return rc;
}

int gir_dev_inc_update(gir_dev_t* g, int weighted) {
    if (!g) return GIR_ERR_INVALID;
    return inc_update(g, weighted ? 1 : 0);
}

int gir_dev_inc_dist(gir_dev_t* g, int weighted, uint64_t* dist_out) {
    if (!g) return GIR_ERR_INVALID;
    if (!dist_out) return fail(g, GIR_ERR_INVALID, "inc_dist: bad arguments");
    if (!g->inc_on[weighted ? 1 : 0]) return fail(g, GIR_ERR_STATE, "inc_dist: the mode is not tracked");
    void* dout = nullptr;
    const size_t bytes = sizeof(uint64_t) * (size_t)g->V;
    GIR_TRY(out_target(g, dist_out, bytes, g->stage_out, &dout));
    GIR_TRY(inc_dist(g, weighted ? 1 : 0, static_cast<uint64_t*>(dout)));
    return finish_out(g, dist_out, dout, bytes);
}

int gir_dev_reachable(gir_dev_t* g, const int32_t* u, const int32_t* v, int64_t n, uint8_t* out) {
    if (!g) return GIR_ERR_INVALID;
    if (n < 0 || (n > 0 && (!u || !v || !out))) return fail(g, GIR_ERR_INVALID, "reachable: bad arguments");
    if (!g->scc_built) return fail(g, GIR_ERR_STATE, "reachable needs buildSCC_DAG first");
    if (n == 0) return GIR_OK;
    GIR_TRY(sync_impl(g));  // a structure-based query: ingested batches are synced first (gir.h:107-113)
    DevBuf su, sv;
    const void *du = nullptr, *dv = nullptr;
    void* dout = nullptr;
    int rc = GIR_OK;
    if ((rc = stage_input(g, su, u, sizeof(int32_t) * n, &du)) || (rc = stage_input(g, sv, v, sizeof(int32_t) * n, &dv)) ||
        (rc = out_target(g, out, (size_t)n, g->stage_out, &dout)) ||
        (rc = reach_run(g, (const int32_t*)du, (const int32_t*)dv, n, (uint8_t*)dout)) ||
        (rc = finish_out(g, out, dout, (size_t)n))) {
        release(g, su);
        release(g, sv);
        return rc;
    }
    release(g, su);
    release(g, sv);
    release_scratch(g, kKeepScratchBelow);
    return GIR_OK;
}

int gir_dev_bfs_sets(gir_dev_t* g, const int64_t* set_beg, const int32_t* set_srcs, int64_t n_sets, int32_t* level_out) {
    return query_sets(g, set_beg, set_srcs, n_sets, true, 0, 0, level_out);
}

int gir_dev_sssp(gir_dev_t* g, const int32_t* srcs, int64_t n_src, uint64_t delta, int weight_mode, uint64_t* dist_out) {
    if (!g) return GIR_ERR_INVALID;
    if (n_src < 0) return fail(g, GIR_ERR_INVALID, "sssp: negative source count");
    std::vector<int64_t> sb((size_t)n_src + 1);
    for (int64_t i = 0; i <= n_src; ++i) sb[i] = i;
    return query_sets(g, sb.data(), srcs, n_src, false, delta, weight_mode, dist_out);
}

int gir_dev_sssp_sets(gir_dev_t* g, const int64_t* set_beg, const int32_t* set_srcs, int64_t n_sets, uint64_t delta,
                      int weight_mode, uint64_t* dist_out) {
    return query_sets(g, set_beg, set_srcs, n_sets, false, delta, weight_mode, dist_out);
}

int gir_dev_apply_batch(gir_dev_t* g, const int32_t* u, const int32_t* v, const uint8_t* ins, int64_t n) {
    if (!g) return GIR_ERR_INVALID;
    if (n < 0 || (n > 0 && (!u || !v || !ins))) return fail(g, GIR_ERR_INVALID, "apply_batch: bad arguments");
    const int rc = apply_batch_impl(g, u, v, ins, n, false);
    release_scratch(g, kKeepScratchBelow);
    return rc;
}

int gir_dev_ingest_batch(gir_dev_t* g, const int32_t* u, const int32_t* v, const uint8_t* ins, int64_t n) {
    if (!g) return GIR_ERR_INVALID;
    if (n < 0 || (n > 0 && (!u || !v || !ins))) return fail(g, GIR_ERR_INVALID, "ingest_batch: bad arguments");
    const int rc = apply_batch_impl(g, u, v, ins, n, true);
    release_scratch(g, kKeepScratchBelow);
    return rc;
}

int gir_dev_sync(gir_dev_t* g) {
    if (!g) return GIR_ERR_INVALID;
    const int rc = sync_impl(g);
    release_scratch(g, kKeepScratchBelow);
    return rc;
}

int gir_dev_synced(gir_dev_t* g, int* out) {
    if (!g || !out) return GIR_ERR_INVALID;
    *out = g->pend ? 0 : 1;
    return GIR_OK;
}

int gir_dev_set_weight_rule(gir_dev_t* g, uint64_t seed, uint32_t lo, uint32_t hi) {
    if (!g) return GIR_ERR_INVALID;
    g->wrule_seed = seed;
    g->wrule_lo = lo;
    g->wrule_hi = hi;
    return GIR_OK;
}

int gir_dev_batch_times(gir_dev_t* g, double* ms4) {
    if (!g || !ms4) return GIR_ERR_INVALID;
    for (int i = 0; i < 4; ++i) ms4[i] = g->b_ms[i];
    return GIR_OK;
}

int gir_dev_batch_plan(gir_dev_t* g, int32_t* plan3) {
    if (!g || !plan3) return GIR_ERR_INVALID;
    for (int i = 0; i < 3; ++i) plan3[i] = g->b_plan[i];
    return GIR_OK;
}

int gir_dev_batch_stats(gir_dev_t* g, int64_t* n_ins, int64_t* n_del, int64_t* n_noop, int64_t* n_invalid) {
    if (!g) return GIR_ERR_INVALID;
    if (n_ins) *n_ins = g->b_ins;
    if (n_del) *n_del = g->b_del;
    if (n_noop) *n_noop = g->b_noop;
    if (n_invalid) *n_invalid = g->b_invalid;
    return GIR_OK;
}

int gir_dev_set_schedule(gir_dev_t* g, int mode) {
    if (!g) return GIR_ERR_INVALID;
    if (mode != GIR_SCHEDULE_FIXED && mode != GIR_SCHEDULE_LEARNED) return fail(g, GIR_ERR_INVALID, "unknown schedule");
    g->schedule = mode;
    return GIR_OK;
}

int gir_dev_set_param(gir_dev_t* g, int which, double value) {
    if (!g) return GIR_ERR_INVALID;
    if (which < 0 || which >= GIR_PARAM_COUNT) return fail(g, GIR_ERR_INVALID, "unknown parameter");
    if (which == GIR_PARAM_PIVOT) {
        if (value != -1.0 && !(value == 0.0 || value == 1.0 || value == 2.0 || value == 3.0))
            return fail(g, GIR_ERR_INVALID, "pivot rule: -1 (the schedule decides) or 0..3");
    } else if (which == GIR_PARAM_LANE_BITS) {
        if (!(value == 0.0 || value == 16.0 || value == 32.0 || value == 64.0))
            return fail(g, GIR_ERR_INVALID, "lane bits: 0 (the library decides), 16, 32 or 64");
    } else if (which == GIR_PARAM_LANE_ORDER) {
        if (!(value == 0.0 || value == 1.0)) return fail(g, GIR_ERR_INVALID, "lane order: 0 or 1");
    } else if (!(value > 0) && which != GIR_PARAM_PROFILE) {
        return fail(g, GIR_ERR_INVALID, "parameters are positive");
    }
    if (which == GIR_PARAM_BLOCK && ((int)value % 32 != 0 || value > 1024)) return fail(g, GIR_ERR_INVALID, "block: multiple of 32, <= 1024");
    g->params[which] = value;
    if (which == GIR_PARAM_SMALL_DEG || which == GIR_PARAM_LARGE_DEG) g->bins_valid = false;
    return GIR_OK;
}

int gir_dev_get_param(gir_dev_t* g, int which, double* value) {
    if (!g || !value) return GIR_ERR_INVALID;
    if (which < 0 || which >= GIR_PARAM_COUNT) return fail(g, GIR_ERR_INVALID, "unknown parameter");
    *value = g->params[which];
    return GIR_OK;
}

int gir_dev_query_stats(gir_dev_t* g, gir_dev_query_stats_t* out) {
    if (!g || !out) return GIR_ERR_INVALID;
    out->edges = g->qstats.edges;
    out->reached = g->qstats.reached;
    out->iterations = g->qstats.iterations;
    out->bottom_up = g->qstats.bottom_up;
    out->launches = g->qstats.launches;
    out->kernel_ms = g->qstats.kernel_ms;
    out->total_ms = g->qstats.total_ms;
    out->main_ms = g->qstats.main_ms;
    out->main_launches = g->qstats.main_launches;
    out->persistent_levels = g->qstats.persistent_levels;
    return GIR_OK;
}

int gir_dev_stream(gir_dev_t* g, void** stream) {
    if (!g || !stream) return GIR_ERR_INVALID;
    *stream = (void*)g->stream;
    return GIR_OK;
}

}  // extern "C"
