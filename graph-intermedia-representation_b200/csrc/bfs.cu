// Direction-optimizing breadth-first search on the device (GIR::bfs, gir_query.cpp:108-294).
//
// Up to 64 queries run as one traversal: every vertex carries 64-bit lane masks (seen, current
// frontier, next frontier), bit i standing for query i. A query's level of v is the iteration in
// which its bit first reaches v, so every query gets exactly the levels a single-source BFS
// gives it. One source per lane is GIR::bfs; several sources in a lane are the multi-source
// query (all start at level 0).
//
// Each iteration runs in one of two directions, chosen per iteration by the schedule:
//  - top-down: the frontier queue's out-edges are cut into equal chunks (edge-balanced, as the
//    reference's 2048-edge chunks, gir_query.cpp:182-219); a lane bit newly reaching w is
//    OR-ed into next[w] and w is queued once (the atomicOr that turns next[w] non-zero queues it);
//  - bottom-up: every vertex that some lane has not reached ORs its in-neighbours' frontier
//    masks and stops once every missing lane is found (gir_query.cpp:232-279), with vertices
//    binned by in-degree: a thread, a warp or a CTA per vertex.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "sched_net.cuh"

namespace gir {

namespace {

constexpr int kBlock = 256;
constexpr int kChunk = 32 * 16;  // edge positions per warp in the top-down expand

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

// counters: [0] queue length, [1] (vertex, lane) pairs reached this iteration,
//           [2] out-edges of those pairs, [3] candidates queued by top-down
// [4] the device-decided direction of the next level and [5..8] its features (learned schedule)
enum { C_Q = 0, C_PAIRS = 1, C_MEDGES = 2, C_CAND = 3, C_DIR = 4, C_FEAT = 5, C_N = 9 };

__device__ __forceinline__ void write_levels(int32_t* level, int64_t V, int32_t v, uint64_t nb, int32_t L) {
    while (nb) {
        const int s = __ffsll((long long)nb) - 1;
        nb &= nb - 1;
        level[(int64_t)s * V + v] = L;
    }
}

__device__ __forceinline__ void warp_add_u64(unsigned long long* p, unsigned long long x) {
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane_id() == 0 && x) atomicAdd(p, x);
}

// Sources: lane s of the group starts at every vertex of set s (set_beg is device memory).
__global__ void k_init_sources(const int64_t* set_beg, int n_lanes, const int32_t* srcs, int64_t V, uint64_t* seen,
                               uint64_t* front, int32_t* q, unsigned long long* cnt, int32_t* level) {
    const int64_t lo = set_beg[0], hi = set_beg[n_lanes];
    GRID_STRIDE(i, hi - lo) {
        const int64_t e = lo + i;
        int s = 0;  // lane of entry e
        while (set_beg[s + 1] <= e) ++s;
        const int32_t v = srcs[e];
        if (v < 0 || v >= V) continue;
        const uint64_t bit = 1ull << s;
        atomicOr((unsigned long long*)&seen[v], bit);
        const unsigned long long old = atomicOr((unsigned long long*)&front[v], bit);
        level[(int64_t)s * V + v] = 0;
        if (old == 0) q[atomicAdd(&cnt[C_Q], 1ull)] = v;
    }
}

// ---- Persistent top-down levels ----------------------------------------------------------------
// A high-diameter graph (a road network, a lattice) takes thousands of levels whose frontiers are
// small: driven from the host, every level costs launches and a synchronization. While the
// frontier stays small and the schedule stays top-down, one cooperative launch runs level after
// level instead, its CTAs meeting at a grid barrier between the expand and the commit phase. It
// hands back to the host loop when the schedule turns bottom-up, when the frontier's out-edges or
// a frontier vertex's degree outgrow what warps walking whole rows balance well, or when done.
// Data that other CTAs write during the launch (masks, queues, counters) is read with ld.cg, past
// the SMs' incoherent L1; every barrier wait is bounded and sets an error flag when it runs out.
constexpr int kPersistThreads = 256;
constexpr int64_t kPersistMaxEdges = 1ll << 28;  // a frontier's out-edges (vertex level)
constexpr int kPersistMaxDeg = 4096;              // a frontier vertex's out-degree
constexpr int kPersistTrace = 8192;               // schedule decisions recorded per launch
constexpr unsigned kBarrierSpins = 1u << 25;      // bounded barrier wait (a few seconds)

// control words; counter slots (one per level, reused every third level) follow
enum { P_LEVELS = 0, P_NQ, P_REASON, P_DIR, P_EDGES, P_REACHED, P_MF, P_NF, P_MU, P_FI, P_QI, P_ERR, P_SLOTS = 16 };
enum { S_Q = 0, S_CAND, S_PAIRS, S_MEDGES, S_VEDGES, S_MAXDEG, S_W = 8 };
enum { R_DONE = 0, R_BOTTOM_UP = 1, R_BIG = 2, R_LIMIT = 3 };
// the barrier's arrival counter and generation, each on its own 128-byte line after the slots
constexpr int kCtlBarrier = 64;
constexpr int kCtlWords = kCtlBarrier + 32;

struct PersistArgs {
    CSRView fw;
    uint64_t* seen;
    uint64_t* next;
    uint64_t* front[2];       // the frontier's masks alternate between these (the other is zero)
    int32_t* q[3];            // frontier, candidates and next frontier rotate over these
    int32_t* level;
    int64_t V, nq0;
    double E, mf0, nf0, mu0, alpha, beta;
    int lanes, L0, max_levels;
    const float* net;         // schedule network parameters, or null for the fixed switch
    unsigned long long* ctl;  // P_* words and the counter slots, zeroed by the host
    unsigned int* bar;        // [0] arrivals, [32] generation (own 128-byte lines), zeroed by the host
    float* trace;             // kPersistTrace x (GIR_SCHED_IN features + decision)
};

__device__ __forceinline__ unsigned long long ldcg_u64(const unsigned long long* p) { return __ldcg(p); }

// All CTAs of the cooperative launch meet here. Returns false once any CTA has flagged an error.
__device__ __forceinline__ bool grid_sync(unsigned int* bar, unsigned long long* err) {
    return grid_barrier(bar, err, kBarrierSpins);
}

// End of a phase: the CTA's warps empty their staging buffers with one queue reservation for the
// whole CTA (block-uniform call; s_cnt holds one int per warp, s_base one word).
__device__ __forceinline__ void block_flush(int32_t* s_buf, int& s_n, int* s_cnt, unsigned long long* s_base, int32_t* q,
                                            unsigned long long* cnt) {
    const int wib = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane_id() == 0) s_cnt[wib] = s_n;
    __syncthreads();
    if (threadIdx.x == 0) {
        int total = 0;
        for (int k = 0; k < nw; ++k) total += s_cnt[k];
        *s_base = total ? atomicAdd(cnt, (unsigned long long)total) : 0ull;
    }
    __syncthreads();
    unsigned long long off = *s_base;
    for (int k = 0; k < wib; ++k) off += s_cnt[k];
    for (int i = lane_id(); i < s_n; i += 32) q[off + i] = s_buf[i];
    s_n = 0;
    __syncthreads();
}

// Sums v over the CTA (block-uniform call) and adds it to *dst with one atomic per CTA; with
// max_ set, takes the maximum instead.
__device__ __forceinline__ void block_add(unsigned long long v, unsigned long long* s_red, unsigned long long* dst,
                                          bool max_) {
    for (int o = 16; o; o >>= 1) {
        const unsigned long long t = __shfl_xor_sync(0xffffffffu, v, o);
        v = max_ ? (t > v ? t : v) : v + t;
    }
    if (lane_id() == 0) s_red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long r = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r = max_ ? (s_red[k] > r ? s_red[k] : r) : r + s_red[k];
        if (r) {
            if (max_) atomicMax(dst, r);
            else atomicAdd(dst, r);
        }
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kPersistThreads) k_bfs_persistent(PersistArgs a) {
    __shared__ int64_t s_excl[kPersistThreads / 32][33];
    __shared__ int32_t s_u[kPersistThreads / 32][32];
    __shared__ int s_dir;
    __shared__ int32_t s_stage[kPersistThreads / 32][kStage];
    __shared__ int s_cnt[kPersistThreads / 32];
    __shared__ unsigned long long s_red[kPersistThreads / 32];
    __shared__ unsigned long long s_base;
    unsigned long long* err = a.ctl + P_ERR;
    const int lane = lane_id(), wib = threadIdx.x >> 5;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    int fi = 0, qi = 0, reason = R_LIMIT, dir = 0, lev = 0, n_st = 0;
    int64_t nq = a.nq0, vedges = 0, maxdeg = 0;
    double mf = a.mf0, nf = a.nf0, mu = a.mu0;
    unsigned long long edges = 0, reached = 0;
    for (lev = 0; lev < a.max_levels; ++lev) {
        if (threadIdx.x == 0) {  // (every CTA computes the same decision from the same counters)
            float x[sched_net::IN];
            s_dir = sched_net::decide_direction(a.net, (double)a.V, a.E, nf, mf, mu, 0, a.lanes, a.alpha, a.beta, x);
            if (blockIdx.x == 0 && lev < kPersistTrace) {
                for (int i = 0; i < sched_net::IN; ++i) a.trace[lev * (sched_net::IN + 1) + i] = x[i];
                a.trace[lev * (sched_net::IN + 1) + sched_net::IN] = (float)s_dir;
            }
        }
        __syncthreads();
        dir = s_dir;
        __syncthreads();  // (s_dir is rewritten at the next level only after every thread read it)
        if (dir) { reason = R_BOTTOM_UP; break; }
        if (lev > 0 && (vedges > kPersistMaxEdges || maxdeg > kPersistMaxDeg)) { reason = R_BIG; break; }
        unsigned long long* sl = a.ctl + P_SLOTS + S_W * (lev % 3);
        unsigned long long* sl_done = a.ctl + P_SLOTS + S_W * ((lev + 2) % 3);  // last level's slot
        const int32_t* qa = a.q[qi];
        int32_t* qb = a.q[(qi + 1) % 3];
        int32_t* qc = a.q[(qi + 2) % 3];
        uint64_t* fA = a.front[fi];
        uint64_t* fB = a.front[fi ^ 1];
        // expand: a warp takes 32 frontier vertices and walks their rows together; a lane bit that
        // newly reaches w goes into next[w], and the atomicOr that turns next[w] non-zero queues w
        for (int64_t base = warp * 32; base < nq; base += nwarps * 32) {
            const int64_t i = base + lane;
            const int32_t u = i < nq ? __ldcg(qa + i) : -1;
            const int64_t cnt = u >= 0 ? a.fw.deg[u] : 0;
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
                bool fresh = false;
                int32_t w = 0;
                if (p < total) {
                    int lo = 0, hi = 31;
                    while (lo < hi) {
                        const int m = (lo + hi + 1) >> 1;
                        if (s_excl[wib][m] <= p) lo = m; else hi = m - 1;
                    }
                    const int32_t uu = s_u[wib][lo];
                    w = a.fw.adj[a.fw.beg[uu] + (p - s_excl[wib][lo])];
                    const unsigned long long bits =
                        ldcg_u64((const unsigned long long*)fA + uu) & ~ldcg_u64((const unsigned long long*)a.seen + w);
                    if (bits) fresh = atomicOr((unsigned long long*)a.next + w, bits) == 0ull;
                }
                stage_append(fresh, w, s_stage[wib], n_st, qb, &sl[S_CAND]);
            }
            __syncwarp();
        }
        block_flush(s_stage[wib], n_st, s_cnt, &s_base, qb, &sl[S_CAND]);
        if (!grid_sync(a.bar, err)) break;
        // commit: clear the old frontier's masks, then every candidate takes its new lanes
        if (blockIdx.x == 0 && threadIdx.x < S_W) sl_done[threadIdx.x] = 0;  // (read by every CTA before the barrier)
        GRID_STRIDE(i, nq) fA[__ldcg(qa + i)] = 0;
        const int64_t nc = (int64_t)ldcg_u64(&sl[S_CAND]);
        unsigned long long pairs = 0, medges = 0, ved = 0, mdeg = 0;
        for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < nc; base += (int64_t)gridDim.x * blockDim.x) {
            const int64_t i = base + threadIdx.x;
            bool on = false;
            int32_t w = 0;
            if (i < nc) {
                w = __ldcg(qb + i);
                const unsigned long long sw = ldcg_u64((const unsigned long long*)a.seen + w);
                const unsigned long long nb = ldcg_u64((const unsigned long long*)a.next + w) & ~sw;
                a.next[w] = 0;
                if (nb) {
                    a.seen[w] = sw | nb;
                    fB[w] = nb;
                    write_levels(a.level, a.V, w, nb, a.L0 + lev + 1);
                    const unsigned c = __popcll(nb);
                    const unsigned long long d = (unsigned long long)a.fw.deg[w];
                    pairs += c;
                    medges += c * d;
                    ved += d;
                    mdeg = d > mdeg ? d : mdeg;
                    on = true;
                }
            }
            stage_append(on, w, s_stage[wib], n_st, qc, &sl[S_Q]);
        }
        block_flush(s_stage[wib], n_st, s_cnt, &s_base, qc, &sl[S_Q]);
        block_add(pairs, s_red, &sl[S_PAIRS], false);
        block_add(medges, s_red, &sl[S_MEDGES], false);
        block_add(ved, s_red, &sl[S_VEDGES], false);
        block_add(mdeg, s_red, &sl[S_MAXDEG], true);
        if (!grid_sync(a.bar, err)) break;
        nq = (int64_t)ldcg_u64(&sl[S_Q]);
        const unsigned long long pr = ldcg_u64(&sl[S_PAIRS]), me = ldcg_u64(&sl[S_MEDGES]);
        vedges = (int64_t)ldcg_u64(&sl[S_VEDGES]);
        maxdeg = (int64_t)ldcg_u64(&sl[S_MAXDEG]);
        nf = (double)pr / a.lanes;
        mf = (double)me / a.lanes;
        mu -= mf;
        edges += me;
        reached += pr;
        fi ^= 1;
        qi = (qi + 2) % 3;
        if (nq == 0) {
            reason = R_DONE;
            ++lev;
            break;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.ctl[P_LEVELS] = (unsigned long long)lev;
        a.ctl[P_NQ] = (unsigned long long)nq;
        a.ctl[P_REASON] = (unsigned long long)reason;
        a.ctl[P_DIR] = (unsigned long long)dir;
        a.ctl[P_EDGES] = edges;
        a.ctl[P_REACHED] = reached;
        a.ctl[P_MF] = (unsigned long long)__double_as_longlong(mf);
        a.ctl[P_NF] = (unsigned long long)__double_as_longlong(nf);
        a.ctl[P_MU] = (unsigned long long)__double_as_longlong(mu);
        a.ctl[P_FI] = (unsigned long long)fi;
        a.ctl[P_QI] = (unsigned long long)qi;
    }
}

// Frontier out-degrees for the edge-balanced expand.
__global__ void k_frontier_degrees(const int32_t* q, int64_t nq, const int32_t* deg, int64_t* pref) {
    GRID_STRIDE(i, nq) pref[i] = deg[q[i]];
    if (blockIdx.x == 0 && threadIdx.x == 0) pref[nq] = 0;
}

// Top-down: warp w takes edge positions [w*kChunk, (w+1)*kChunk) of the frontier's out-edges
// (pref = exclusive scan of frontier degrees).
__global__ void k_td_expand(const int32_t* q, int64_t nq, const int64_t* pref, CSRView fw,
                            const uint64_t* front, const uint64_t* seen, uint64_t* next, int32_t* cand,
                            unsigned long long* cnt) {
    const int64_t total = pref[nq];  // (read here, so the host needs no copy of it)
    __shared__ int32_t s_stage[kBlock / 32][kStage];
    int n_st = 0;
    const int lane = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c0 = warp * kChunk; c0 < total; c0 += nwarps * kChunk) {
        const int64_t c1 = c0 + kChunk < total ? c0 + kChunk : total;
        // frontier index owning this lane's first position (largest i with pref[i] <= p)
        const int64_t key = c0 + lane < total ? c0 + lane : total - 1;
        int64_t lo = 0, hi = nq - 1;
        while (lo < hi) {
            const int64_t m = (lo + hi + 1) >> 1;
            if (pref[m] <= key) lo = m; else hi = m - 1;
        }
        int64_t i = lo;
        for (int64_t base = c0; base < c1; base += 32) {  // warp-uniform
            const int64_t p = base + lane;
            bool fresh = false;
            int32_t w = 0;
            if (p < c1) {
                while (pref[i + 1] <= p) ++i;
                const int32_t u = q[i];
                w = fw.adj[fw.beg[u] + (p - pref[i])];
                const uint64_t bits = front[u] & ~seen[w];
                if (bits) fresh = atomicOr((unsigned long long*)&next[w], (unsigned long long)bits) == 0ull;
            }
            stage_append(fresh, w, s_stage[threadIdx.x >> 5], n_st, cand, &cnt[C_CAND]);
        }
    }
    stage_flush(s_stage[threadIdx.x >> 5], n_st, cand, &cnt[C_CAND]);
}

__global__ void k_clear_front(const int32_t* q, int64_t nq, uint64_t* front) {
    GRID_STRIDE(i, nq) front[q[i]] = 0;
}

// Top-down commit: candidates become the new frontier with their newly reached lanes.
__global__ void k_td_commit(const unsigned long long* n_cand, const int32_t* cand, uint64_t* seen, uint64_t* front,
                            uint64_t* next, const int32_t* outdeg, int32_t* level, int64_t V, int32_t L, int32_t* q,
                            unsigned long long* cnt) {
    const int64_t nc = (int64_t)*n_cand;
    __shared__ int32_t s_stage[kBlock / 32][kStage];
    int n_st = 0;
    unsigned long long pairs = 0, medges = 0;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < nc; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = base + threadIdx.x;
        bool on = false;
        int32_t w = 0;
        if (i < nc) {
            w = cand[i];
            const uint64_t s = seen[w];
            const uint64_t nb = next[w] & ~s;
            next[w] = 0;
            if (nb) {
                seen[w] = s | nb;
                front[w] = nb;
                write_levels(level, V, w, nb, L);
                const unsigned c = __popcll(nb);
                pairs += c;
                medges += (unsigned long long)c * (unsigned long long)outdeg[w];
                on = true;
            }
        }
        stage_append(on, w, s_stage[threadIdx.x >> 5], n_st, q, &cnt[C_Q]);
    }
    stage_flush(s_stage[threadIdx.x >> 5], n_st, q, &cnt[C_Q]);
    warp_add_u64(&cnt[C_PAIRS], pairs);
    warp_add_u64(&cnt[C_MEDGES], medges);
}

// Bottom-up, thread per vertex (small in-degree bin).
__global__ void k_bu_thread(const int32_t* ids, int64_t n, CSRView bw, const uint64_t* front, uint64_t* seen,
                            uint64_t* next, uint64_t all, const int32_t* outdeg, int32_t* level, int64_t V,
                            int32_t L, int32_t* q, unsigned long long* cnt) {
    __shared__ int32_t s_stage[kBlock / 32][kStage];
    int n_st = 0;
    unsigned long long pairs = 0, medges = 0;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < n; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = base + threadIdx.x;
        bool on = false;
        int32_t v = 0;
        if (i < n) {
            v = ids[i];
            const uint64_t s = seen[v];
            const uint64_t want = all & ~s;
            uint64_t nb = 0;
            if (want) {
                // four row entries per step (rows start 16-byte aligned), their frontier masks
                // loaded together; entries read past the point where every missing lane is found
                // are in-neighbours all the same, so the lanes they add are found lanes too
                uint64_t acc = 0;
                const int64_t b = bw.beg[v], e = b + bw.deg[v];
                int64_t k = b;
                for (; k + 4 <= e; k += 4) {
                    const int4 a4 = *reinterpret_cast<const int4*>(bw.adj + k);
                    acc |= front[a4.x] | front[a4.y] | front[a4.z] | front[a4.w];
                    if ((acc & want) == want) break;
                }
                if ((acc & want) != want)
                    for (; k < e; ++k) {
                        acc |= front[bw.adj[k]];
                        if ((acc & want) == want) break;
                    }
                nb = acc & want;
            }
            next[v] = nb;
            if (nb) {
                seen[v] = s | nb;
                write_levels(level, V, v, nb, L);
                const unsigned c = __popcll(nb);
                pairs += c;
                medges += (unsigned long long)c * (unsigned long long)outdeg[v];
                on = true;
            }
        }
        stage_append(on, v, s_stage[threadIdx.x >> 5], n_st, q, &cnt[C_Q]);
    }
    stage_flush(s_stage[threadIdx.x >> 5], n_st, q, &cnt[C_Q]);
    warp_add_u64(&cnt[C_PAIRS], pairs);
    warp_add_u64(&cnt[C_MEDGES], medges);
}

__device__ __forceinline__ uint64_t warp_or_u64(uint64_t x) {
    const unsigned lo = __reduce_or_sync(0xffffffffu, (unsigned)(x & 0xffffffffu));
    const unsigned hi = __reduce_or_sync(0xffffffffu, (unsigned)(x >> 32));
    return ((uint64_t)hi << 32) | lo;
}

// Bottom-up, warp per vertex (medium bin): lanes read 32 consecutive in-neighbours per round.
__global__ void k_bu_warp(const int32_t* ids, int64_t n, CSRView bw, const uint64_t* front, uint64_t* seen,
                          uint64_t* next, uint64_t all, const int32_t* outdeg, int32_t* level, int64_t V, int32_t L,
                          int32_t* q, unsigned long long* cnt) {
    const int lane = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long pairs = 0, medges = 0;
    for (int64_t i = warp; i < n; i += nwarps) {
        const int32_t v = ids[i];
        const uint64_t s = seen[v];
        const uint64_t want = all & ~s;
        uint64_t nb = 0;
        if (want) {
            uint64_t acc = 0;
            const int64_t b = bw.beg[v], e = b + bw.deg[v];
            for (int64_t k0 = b; k0 < e; k0 += 32) {
                const int64_t k = k0 + lane;
                uint64_t a = k < e ? front[bw.adj[k]] : 0ull;
                acc |= warp_or_u64(a);
                if ((acc & want) == want) break;
            }
            nb = acc & want;
        }
        if (lane == 0) {
            next[v] = nb;
            if (nb) {
                seen[v] = s | nb;
                const unsigned c = __popcll(nb);
                pairs += c;
                medges += (unsigned long long)c * (unsigned long long)outdeg[v];
                q[atomicAdd(&cnt[C_Q], 1ull)] = v;
            }
        }
        // lanes split the level writes of this vertex
        uint64_t rest = nb;
        for (int j = 0; rest; ++j) {
            const int sbit = __ffsll((long long)rest) - 1;
            rest &= rest - 1;
            if ((j & 31) == lane) level[(int64_t)sbit * V + v] = L;
        }
    }
    if (lane == 0) {
        if (pairs) atomicAdd(&cnt[C_PAIRS], pairs);
        if (medges) atomicAdd(&cnt[C_MEDGES], medges);
    }
}

// Bottom-up, CTA per vertex (large bin).
__global__ void k_bu_cta(const int32_t* ids, int64_t n, CSRView bw, const uint64_t* front, uint64_t* seen,
                         uint64_t* next, uint64_t all, const int32_t* outdeg, int32_t* level, int64_t V, int32_t L,
                         int32_t* q, unsigned long long* cnt) {
    __shared__ unsigned long long s_acc;
    for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
        const int32_t v = ids[i];
        const uint64_t s = seen[v];
        const uint64_t want = all & ~s;
        if (threadIdx.x == 0) s_acc = 0;
        __syncthreads();
        if (want) {
            const int64_t b = bw.beg[v], e = b + bw.deg[v];
            for (int64_t k0 = b; k0 < e; k0 += blockDim.x) {
                const int64_t k = k0 + threadIdx.x;
                uint64_t a = k < e ? front[bw.adj[k]] : 0ull;
                a = warp_or_u64(a);
                if (lane_id() == 0 && (a & want)) atomicOr(&s_acc, (unsigned long long)(a & want));
                __syncthreads();
                const bool done = (s_acc & want) == want;
                __syncthreads();
                if (done) break;
            }
        }
        const uint64_t nb = s_acc & want;
        if (threadIdx.x == 0) {
            next[v] = nb;
            if (nb) {
                seen[v] = s | nb;
                const unsigned c = __popcll(nb);
                atomicAdd(&cnt[C_PAIRS], (unsigned long long)c);
                atomicAdd(&cnt[C_MEDGES], (unsigned long long)c * (unsigned long long)outdeg[v]);
                q[atomicAdd(&cnt[C_Q], 1ull)] = v;
            }
        }
        if (threadIdx.x < 64 && ((nb >> threadIdx.x) & 1ull)) level[(int64_t)threadIdx.x * V + v] = L;
        __syncthreads();
    }
}

// Out-edges of the sources' lanes, for the traversed-edge count.
__global__ void k_source_edges(const int32_t* q, int64_t nq, const uint64_t* front, const int32_t* outdeg,
                               unsigned long long* cnt) {
    unsigned long long pairs = 0, medges = 0;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < nq; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = base + threadIdx.x;
        if (i < nq) {
            const int32_t v = q[i];
            const unsigned c = __popcll(front[v]);
            pairs += c;
            medges += (unsigned long long)c * (unsigned long long)outdeg[v];
        }
    }
    warp_add_u64(&cnt[C_PAIRS], pairs);
    warp_add_u64(&cnt[C_MEDGES], medges);
}

}  // namespace

int bfs_run(gir_dev* g, const int64_t* set_beg_h, const int32_t* srcs_d, int64_t n_sets, int32_t* level_d) {
    const int64_t V = g->V;
    QueryStats& st = g->qstats;
    st = QueryStats{};
    g->trace_x.clear();
    g->trace_y.clear();
    if (n_sets <= 0) return GIR_OK;
    GIR_CUDA(g, cudaMemsetAsync(level_d, 0xff, sizeof(int32_t) * V * n_sets, g->stream));
    if (V == 0) return GIR_OK;
    if (!g->bins_valid) GIR_TRY(store_build_bins(g));

    uint64_t *seen = nullptr, *front = nullptr, *next = nullptr;
    int32_t *qa = nullptr, *qb = nullptr;
    int64_t *pref = nullptr, *sbeg = nullptr;
    unsigned long long* cnt = nullptr;
    GIR_TRY(ensure_n(g, g->scratch[0], V, &seen));
    GIR_TRY(ensure_n(g, g->scratch[1], V, &front));
    GIR_TRY(ensure_n(g, g->scratch[2], V, &next));
    GIR_TRY(ensure_n(g, g->scratch[3], V + 1, &qa));
    GIR_TRY(ensure_n(g, g->scratch[4], V + 1, &qb));
    GIR_TRY(ensure_n(g, g->scratch[5], V + 2, &pref));
    GIR_TRY(ensure_n(g, g->scratch[6], 65, &sbeg));
    GIR_TRY(ensure_n(g, g->scratch[7], C_N, &cnt));
    unsigned long long* hc = nullptr;
    {
        void* h = nullptr;
        GIR_TRY(pinned(g, 256, &h));
        hc = static_cast<unsigned long long*>(h);
    }
    const double alpha = g->params[GIR_PARAM_ALPHA], beta = g->params[GIR_PARAM_BETA];
    const int64_t E = g->fw.E;
    const int grid = g->num_sms * (int)g->params[GIR_PARAM_CTAS_PER_SM];
    // persistent top-down levels (graphs of 4096+ vertices; the device must take cooperative launches)
    uint64_t* front2 = nullptr;
    int32_t* q3 = nullptr;
    unsigned long long* pctl = nullptr;
    float* ptrace = nullptr;
    int persist_grid = 0;
    if (V >= 4096) {
        int coop = 0, per_sm = 0;
        GIR_CUDA(g, cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, g->device));
        GIR_CUDA(g, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bfs_persistent, kPersistThreads, 0));
        if (coop && per_sm > 0) {
            persist_grid = g->num_sms * per_sm;  // every co-resident CTA: the levels are latency-bound
            GIR_TRY(ensure_n(g, g->scratch[8], V, &front2));
            GIR_TRY(ensure_n(g, g->scratch[9], V + 1, &q3));
            GIR_TRY(ensure_n(g, g->scratch[10], kCtlWords, &pctl));
            GIR_TRY(ensure_n(g, g->scratch[11], (size_t)kPersistTrace * (GIR_SCHED_IN + 1), &ptrace));
        }
    }
    const float* net = nullptr;
    if (g->schedule == GIR_SCHEDULE_LEARNED && g->sched_loaded) net = static_cast<const float*>(g->sched_w.p);
    std::vector<float> trace_rows;
    MainTimer timer{g, g->params[GIR_PARAM_PROFILE] != 0.0};
    GIR_CUDA(g, cudaEventRecord(g->ev0, g->stream));

    for (int64_t g0 = 0; g0 < n_sets; g0 += 64) {
        const int nl = (int)((n_sets - g0) < 64 ? (n_sets - g0) : 64);
        const uint64_t all = nl == 64 ? ~0ull : ((1ull << nl) - 1);
        int32_t* level = level_d + g0 * V;
        GIR_CUDA(g, cudaMemsetAsync(seen, 0, sizeof(uint64_t) * V, g->stream));
        GIR_CUDA(g, cudaMemsetAsync(front, 0, sizeof(uint64_t) * V, g->stream));
        GIR_CUDA(g, cudaMemsetAsync(next, 0, sizeof(uint64_t) * V, g->stream));
        if (front2) GIR_CUDA(g, cudaMemsetAsync(front2, 0, sizeof(uint64_t) * V, g->stream));
        GIR_CUDA(g, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * C_N, g->stream));
        GIR_CUDA(g, cudaMemcpyAsync(sbeg, set_beg_h + g0, sizeof(int64_t) * (nl + 1), cudaMemcpyHostToDevice, g->stream));
        const int64_t n_entries = set_beg_h[g0 + nl] - set_beg_h[g0];
        if (n_entries > 0) {
            k_init_sources<<<grid_for(g, n_entries, kBlock), kBlock, 0, g->stream>>>(sbeg, nl, srcs_d, V, seen, front, qa,
                                                                                     cnt, level);
            GIR_LAUNCH(g, "k_init_sources");
            st.launches++;
        }
        GIR_CUDA(g, cudaMemcpyAsync(hc, cnt, sizeof(unsigned long long) * C_N, cudaMemcpyDeviceToHost, g->stream));
        GIR_CUDA(g, cudaStreamSynchronize(g->stream));
        int64_t nq = (int64_t)hc[0];
        const bool learned = g->schedule == GIR_SCHEDULE_LEARNED && g->sched_loaded && V >= 4096;
        if (nq > 0) {
            k_source_edges<<<grid_for(g, nq, kBlock), kBlock, 0, g->stream>>>(qa, nq, front, g->fw.deg, cnt);
            GIR_LAUNCH(g, "k_source_edges");
            st.launches++;
            if (learned)
                GIR_TRY(sched_bfs_decide_async(g, cnt, C_PAIRS, C_MEDGES, C_DIR, C_FEAT, nl, (double)E, false, alpha,
                                               beta));
            GIR_CUDA(g, cudaMemcpyAsync(hc, cnt, sizeof(unsigned long long) * C_N, cudaMemcpyDeviceToHost, g->stream));
            GIR_CUDA(g, cudaStreamSynchronize(g->stream));
        }
        double mf = (double)hc[C_MEDGES] / nl;       // out-edges of the frontier (per lane)
        double nf = (double)hc[C_PAIRS] / nl;        // frontier vertices (per lane)
        double mu = (double)E - mf;                  // out-edges not yet explored (per lane)
        st.edges += (int64_t)hc[C_MEDGES];
        st.reached += (int64_t)hc[C_PAIRS];
        bool bottom_up = false, next_dirty = false, handed_back = false;
        int pending = -1;  // a direction already decided (by the persistent launch) for this level
        int32_t L = 0;
        while (nq > 0) {
            // direction (the reference's switch, gir_query.cpp:159-169, or the schedule network)
            if (pending >= 0) {
                bottom_up = pending != 0;
                pending = -1;
            } else if (learned) {  // decided on the device with the counters just read
                bottom_up = hc[C_DIR] != 0;
                sched_trace(g, reinterpret_cast<const float*>(&hc[C_FEAT]), bottom_up ? 1 : 0);
            } else if (V >= 4096) {
                float feat[GIR_SCHED_IN];
                sched_bfs_features(g, nf, mf, mu, L, bottom_up, nl, feat);
                if (!bottom_up && mf * alpha > mu) bottom_up = true;
                else if (bottom_up && nf * beta < (double)V) bottom_up = false;
                sched_trace(g, feat, bottom_up ? 1 : 0);
            }
            // a small top-down frontier: levels run on the device until the launch hands back
            if (!bottom_up && persist_grid > 0 && !handed_back && mf * nl <= (double)(1 << 24)) {
                if (next_dirty) {
                    GIR_CUDA(g, cudaMemsetAsync(next, 0, sizeof(uint64_t) * V, g->stream));
                    next_dirty = false;
                }
                GIR_CUDA(g, cudaMemsetAsync(pctl, 0, sizeof(unsigned long long) * kCtlWords, g->stream));
                PersistArgs pa;
                pa.fw = view(g->fw);
                pa.seen = seen;
                pa.next = next;
                pa.front[0] = front;
                pa.front[1] = front2;
                pa.q[0] = qa;
                pa.q[1] = qb;
                pa.q[2] = q3;
                pa.level = level;
                pa.V = V;
                pa.nq0 = nq;
                pa.E = (double)E;
                pa.mf0 = mf;
                pa.nf0 = nf;
                pa.mu0 = mu;
                pa.alpha = alpha;
                pa.beta = beta;
                pa.lanes = nl;
                pa.L0 = L;
                pa.max_levels = 1 << 30;
                pa.net = learned ? net : nullptr;
                pa.ctl = pctl;
                pa.bar = reinterpret_cast<unsigned int*>(pctl + kCtlBarrier);
                pa.trace = ptrace;
                void* kargs[] = {&pa};
                GIR_TRY(timer.run([&]() -> int {
                    GIR_CUDA(g, cudaLaunchCooperativeKernel((const void*)k_bfs_persistent, persist_grid, kPersistThreads,
                                                            kargs, 0, g->stream));
                    return GIR_OK;
                }));
                st.launches++;
                unsigned long long* pc = hc + 16;
                GIR_CUDA(g, cudaMemcpyAsync(pc, pctl, sizeof(unsigned long long) * 16, cudaMemcpyDeviceToHost, g->stream));
                GIR_CUDA(g, cudaStreamSynchronize(g->stream));
                if (pc[P_ERR]) return fail(g, GIR_ERR_TIMEOUT, "bfs: the persistent level loop ran out its barrier bound");
                const int64_t lv = (int64_t)pc[P_LEVELS];
                const int64_t n_tr = std::min<int64_t>(lv + (pc[P_REASON] == R_DONE ? 0 : 1), kPersistTrace);
                if (n_tr > 0) {  // the schedule decisions taken inside the launch
                    trace_rows.resize((size_t)n_tr * (GIR_SCHED_IN + 1));
                    GIR_CUDA(g, cudaMemcpyAsync(trace_rows.data(), ptrace, sizeof(float) * trace_rows.size(),
                                                cudaMemcpyDeviceToHost, g->stream));
                    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
                    for (int64_t r = 0; r < n_tr; ++r) {
                        const float* row = trace_rows.data() + r * (GIR_SCHED_IN + 1);
                        sched_trace(g, row, (int32_t)row[GIR_SCHED_IN]);
                    }
                }
                L += (int32_t)lv;
                st.iterations += lv;
                st.persistent_levels += lv;
                st.edges += (int64_t)pc[P_EDGES];
                st.reached += (int64_t)pc[P_REACHED];
                nq = (int64_t)pc[P_NQ];
                double d3[3];
                std::memcpy(&d3[0], &pc[P_MF], sizeof(double));
                std::memcpy(&d3[1], &pc[P_NF], sizeof(double));
                std::memcpy(&d3[2], &pc[P_MU], sizeof(double));
                mf = d3[0];
                nf = d3[1];
                mu = d3[2];
                if (pc[P_FI]) std::swap(front, front2);
                int32_t* qs[3] = {qa, qb, q3};
                const int qi = (int)pc[P_QI];
                qa = qs[qi];
                qb = qs[(qi + 1) % 3];
                q3 = qs[(qi + 2) % 3];
                pending = (int)pc[P_DIR];
                handed_back = pc[P_REASON] != R_BOTTOM_UP;  // (a big frontier: one level on the host first)
                continue;
            }
            handed_back = false;
            GIR_CUDA(g, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * C_N, g->stream));
            if (!bottom_up) {
                if (next_dirty) {
                    GIR_CUDA(g, cudaMemsetAsync(next, 0, sizeof(uint64_t) * V, g->stream));
                    next_dirty = false;
                }
                k_frontier_degrees<<<grid_for(g, nq, kBlock), kBlock, 0, g->stream>>>(qa, nq, g->fw.deg, pref);
                GIR_LAUNCH(g, "k_frontier_degrees");
                GIR_TRY(exclusive_scan_i64(g, pref, pref, nq + 1));
                // The frontier's row total and the candidate count stay on the device: the
                // kernels are sized from the host's upper bound (the frontier's out-edges over
                // all lanes, counted at the end of the previous level) and read the exact ones.
                const double bound = std::min(mf * nl, (double)E) + 1.0;
                const int64_t warps_per_block = kBlock / 32;
                int64_t blocks = (int64_t)((bound / kChunk + warps_per_block) / warps_per_block) + 1;
                if (blocks > grid) blocks = grid;
                GIR_TRY(timer.run([&]() -> int {
                    k_td_expand<<<(int)blocks, kBlock, 0, g->stream>>>(qa, nq, pref, view(g->fw), front, seen, next, qb,
                                                                       cnt);
                    GIR_LAUNCH(g, "k_td_expand");
                    return GIR_OK;
                }));
                k_clear_front<<<grid_for(g, nq, kBlock), kBlock, 0, g->stream>>>(qa, nq, front);
                GIR_LAUNCH(g, "k_clear_front");
                const int64_t nc_bound = (int64_t)std::min(bound, (double)V);
                k_td_commit<<<grid_for(g, nc_bound, kBlock), kBlock, 0, g->stream>>>(
                    cnt + C_CAND, qb, seen, front, next, g->fw.deg, level, V, L + 1, qa, cnt);
                GIR_LAUNCH(g, "k_td_commit");
                st.launches += 4;
            } else {
                const int32_t* bins = static_cast<const int32_t*>(g->bins.p);
                GIR_TRY(timer.run([&]() -> int {
                    if (g->bin_n[0] > 0) {
                        k_bu_thread<<<grid_for(g, g->bin_n[0], kBlock), kBlock, 0, g->stream>>>(
                            bins, g->bin_n[0], view(g->bw), front, seen, next, all, g->fw.deg, level, V, L + 1, qa, cnt);
                        GIR_LAUNCH(g, "k_bu_thread");
                        st.launches++;
                    }
                    if (g->bin_n[1] > 0) {
                        k_bu_warp<<<grid_for(g, g->bin_n[1] * 32, kBlock), kBlock, 0, g->stream>>>(
                            bins + g->bin_n[0], g->bin_n[1], view(g->bw), front, seen, next, all, g->fw.deg, level, V,
                            L + 1, qa, cnt);
                        GIR_LAUNCH(g, "k_bu_warp");
                        st.launches++;
                    }
                    if (g->bin_n[2] > 0) {
                        const int64_t b = g->bin_n[2] < grid ? g->bin_n[2] : grid;
                        k_bu_cta<<<(int)b, kBlock, 0, g->stream>>>(bins + g->bin_n[0] + g->bin_n[1], g->bin_n[2],
                                                                   view(g->bw), front, seen, next, all, g->fw.deg, level,
                                                                   V, L + 1, qa, cnt);
                        GIR_LAUNCH(g, "k_bu_cta");
                        st.launches++;
                    }
                    return GIR_OK;
                }));
                std::swap(front, next);
                next_dirty = true;
                st.bottom_up++;
            }
            if (learned)
                GIR_TRY(sched_bfs_decide_async(g, cnt, C_PAIRS, C_MEDGES, C_DIR, C_FEAT, nl, mu, bottom_up, alpha, beta));
            GIR_CUDA(g, cudaMemcpyAsync(hc, cnt, sizeof(unsigned long long) * C_N, cudaMemcpyDeviceToHost, g->stream));
            GIR_CUDA(g, cudaStreamSynchronize(g->stream));
            nq = (int64_t)hc[C_Q];
            mf = (double)hc[C_MEDGES] / nl;
            nf = (double)hc[C_PAIRS] / nl;
            mu -= mf;
            st.edges += (int64_t)hc[C_MEDGES];
            st.reached += (int64_t)hc[C_PAIRS];
            ++L;
            st.iterations++;
        }
    }
    GIR_CUDA(g, cudaEventRecord(g->ev1, g->stream));
    GIR_CUDA(g, cudaEventSynchronize(g->ev1));
    float ms = 0;
    GIR_CUDA(g, cudaEventElapsedTime(&ms, g->ev0, g->ev1));
    st.kernel_ms = ms;
    return GIR_OK;
}

}  // namespace gir
