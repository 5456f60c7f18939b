// Delta-stepping shortest paths on the device (GIR::sssp / deltaStepping, gir_query.cpp:629-703):
// uint64 distances, UINT64_MAX = unreachable.
//
// Up to 64 queries run as one traversal (lanes), like the BFS: every vertex carries 64-bit lane
// masks for the work of the current bucket (near), for relaxations beyond it (far) and for the
// lanes settled in the bucket; distances are stored lane-interleaved (dist[v * lanes + s]) so a
// warp relaxing one edge for many lanes touches one contiguous row. All lanes step through the
// buckets together, each lane running exact Delta-stepping:
//  - bucket k = [k*Delta, (k+1)*Delta): the near vertices relax their light edges
//    (weight < Delta) round after round until no lane re-enters the bucket;
//  - then every (vertex, lane) settled in the bucket relaxes its heavy edges (weight >= Delta)
//    once -- those land in later buckets only. (The reference relaxes all edges every round and
//    has no light/heavy split, gir_query.cpp:674-688; the split changes the work, not the result.)
//  - the next bucket is the smallest live far distance; the far entries inside it become near.
// Rows are read from a weight-sorted copy of the forward CSR, so a row's light edges are its
// prefix. Shortest distances are unique, so the result is the same for every Delta, every
// schedule and every lane grouping.
#include <algorithm>

#include "common.cuh"

namespace gir {

namespace {

constexpr int kBlock = 256;
constexpr uint64_t kInf = ~0ull;

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

// counters: [0] next near queue length, [1] far queue length, [2] settled queue length,
// [3] min live far distance, [4] far queue length after a split, [5] relaxation items,
// [6] set when a 16-bit lane distance could not hold a tentative distance;
// accumulated over the call: [16] reached (vertex, lane) pairs, [17] their out-edges
enum { S_NEAR = 0, S_FAR = 1, S_SET = 2, S_MIN = 3, S_FAR2 = 4, S_ITEMS = 5, S_OVF = 6, S_REACHED = 16, S_EDGES = 17,
       S_N = 32 };

// Sort keys (row << 32 | weight) and columns of every entry of the compact copy of `c`. For the
// forward CSR the weight of entry (u, v) is that of edge u -> v. With `reverse` the rows are
// those of the backward CSR: row v holds the u of every edge u -> v, whose weight is the hash
// weight of (u, v) or the stored weight found in the forward row of u (`f`).
__global__ void k_ws_keys(int64_t V, int64_t E, const int64_t* cb, CSRView c, int hash, int reverse, CSRView f,
                          uint64_t* keys, uint32_t* cols) {
    GRID_STRIDE(i, E) {
        int64_t lo = 0, hi = V - 1;
        while (lo < hi) {
            const int64_t m = (lo + hi + 1) >> 1;
            if (cb[m] <= i) lo = m; else hi = m - 1;
        }
        const int64_t u = lo;
        const int64_t p = c.beg[u] + (i - cb[u]);
        const int32_t v = c.adj[p];
        uint32_t w;
        if (!reverse) {
            w = hash ? hash_weight((int32_t)u, v) : c.w[p];
        } else if (hash) {
            w = hash_weight(v, (int32_t)u);
        } else {
            const int64_t b = f.beg[v];
            w = f.w[lower_bound_dev(f.adj, b, b + f.deg[v], (int32_t)u)];
        }
        keys[i] = ((uint64_t)u << 32) | w;
        cols[i] = (uint32_t)v;
    }
}

__global__ void k_ws_split(int64_t E, const uint64_t* keys, const uint32_t* cols, int32_t* adj, uint32_t* w) {
    GRID_STRIDE(i, E) {
        adj[i] = (int32_t)cols[i];
        w[i] = (uint32_t)(keys[i] & 0xffffffffULL);
    }
}

// Sum and maximum of the weights (st[0], st[1]).
__global__ void k_wstat(const uint32_t* w, int64_t E, unsigned long long* st) {
    unsigned long long s = 0, m = 0;
    GRID_STRIDE(i, E) {
        s += w[i];
        m = w[i] > m ? w[i] : m;
    }
    for (int o = 16; o; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        const unsigned long long t = __shfl_xor_sync(0xffffffffu, m, o);
        m = t > m ? t : m;
    }
    if (lane_id() == 0) {
        atomicAdd(&st[0], s);
        atomicMax(&st[1], m);
    }
}

__global__ void k_deg_i64(int64_t V, const int32_t* deg, int64_t* out) {
    GRID_STRIDE(v, V) out[v] = deg[v];
    if (blockIdx.x == 0 && threadIdx.x == 0) out[V] = 0;
}

// Lane s of the group starts at every vertex of srcs[lane_rng[2s] .. lane_rng[2s + 1]) (one
// CTA row per lane: blockIdx.y = s).
template <class D>
__global__ void k_sssp_init(const int64_t* lane_rng, const int32_t* srcs, int64_t V, int nl, D* dist,
                            unsigned long long* nearmask, int32_t* nearq, unsigned long long* cnt) {
    const int s = blockIdx.y;
    const int64_t lo = lane_rng[2 * s], hi = lane_rng[2 * s + 1];
    for (int64_t e = lo + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < hi; e += (int64_t)gridDim.x * blockDim.x) {
        const int32_t v = srcs[e];
        if (v < 0 || v >= V) continue;
        dist[(int64_t)v * nl + s] = 0;
        if (atomicOr(&nearmask[v], 1ull << s) == 0ull) nearq[atomicAdd(&cnt[S_NEAR], 1ull)] = v;
    }
}

// Distances inside a lane group are uint32 when every finite distance fits ((V - 1) * max weight
// < 2^32 - 1): half the bytes, eight lanes per 32-byte sector, 32-bit atomics. Output is uint64.
template <class D>
struct DistT;
template <>
struct DistT<uint64_t> {
    static constexpr uint64_t inf = ~0ull;
    __device__ static uint64_t atomic_min(uint64_t* p, uint64_t v) {
        return atomicMin((unsigned long long*)p, (unsigned long long)v);
    }
};
template <>
struct DistT<uint32_t> {
    static constexpr uint32_t inf = ~0u;
    __device__ static uint32_t atomic_min(uint32_t* p, uint32_t v) { return atomicMin((unsigned int*)p, v); }
};
// 16-bit lane distances (64 lanes in one 128-byte line) when the distances are small: the
// minimum is taken by compare-and-swap on the aligned 32-bit word holding the lane. Every failed
// swap means the word changed, and both halves only ever decrease, so the loop ends.
template <>
struct DistT<uint16_t> {
    static constexpr uint16_t inf = 0xffffu;
    __device__ static uint16_t atomic_min(uint16_t* p, uint16_t v) {
        const uintptr_t a = reinterpret_cast<uintptr_t>(p);
        unsigned int* wp = reinterpret_cast<unsigned int*>(a & ~(uintptr_t)3);
        const int sh = (a & 2) ? 16 : 0;
        unsigned int old = *(volatile unsigned int*)wp;
        while (true) {
            const uint16_t cur = (uint16_t)(old >> sh);
            if (cur <= v) return cur;
            const unsigned int nw = (old & ~(0xffffu << sh)) | ((unsigned int)v << sh);
            const unsigned int prev = atomicCAS(wp, old, nw);
            if (prev == old) return cur;
            old = prev;
        }
    }
};

// Index of the k-th set bit of a 64-bit mask (k < popcount).
__device__ __forceinline__ int nth_bit(uint64_t m, int k) {
    const unsigned lo = (unsigned)m;
    const int cl = __popc(lo);
    if (k < cl) return __fns(lo, 0, k + 1);
    return 32 + __fns((unsigned)(m >> 32), 0, k - cl + 1);
}

struct Relax {
    const int64_t* wb;       // weight-sorted rows (compact offsets)
    const int32_t* wdeg;
    const int32_t* wadj;
    const uint32_t* ww;
    uint64_t delta, kend;    // bucket width; end of the current bucket
    int nl;                  // lanes (row stride of dist)
    void* dist;              // lane distances (uint32 or uint64, see DistT)
    unsigned long long* curmask;   // lanes of each queued vertex to process (read and cleared)
    unsigned long long* nextmask;  // lanes re-entering the bucket
    int32_t* nextq;
    unsigned long long* farmask;
    int32_t* farq;
    unsigned long long* setmask;   // lanes settled in this bucket
    int32_t* setq;
    // Lanes whose distance is final: those settled in buckets whose light phase is over (their
    // heavy pass ORs them in). k_far_split drops such lanes from the far set without reading
    // their distances. (k_relax does not test it: on R-MAT graphs the extra 8-byte load per edge
    // cost more than the distance reads and atomics it saved.)
    unsigned long long* done;
    unsigned long long* cnt;
};

// Work-balanced relaxation: k_relax_prep turns the queue into items (one per vertex with work),
// an exclusive scan of the items' work (edges x lanes) numbers all (edge, lane) pairs, and
// k_relax processes them in equal runs, so a hub with many lanes is spread over the grid.
struct Items {
    int32_t* u;
    int64_t* eb;
    unsigned long long* m;
    int64_t* pref;  // work per item, then its exclusive scan (n + 1 entries)
};

// Number of light edges (weight < delta) of every weight-sorted row, once per query group.
// Written with it, one 16-byte record per vertex for the queue bookkeeping of every pass: the
// row start (two halves), its length and its light-edge count, so a queued vertex costs one
// scattered load instead of three.
__global__ void k_light_split(int64_t V, const int64_t* wb, const int32_t* wdeg, const uint32_t* ww, uint64_t delta,
                              int4* rows) {
    GRID_STRIDE(v, V) {
        const int64_t b = wb[v];
        const int32_t d = wdeg[v];
        int64_t lo = b, hi = b + d;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if ((uint64_t)ww[mid] < delta) lo = mid + 1; else hi = mid;
        }
        rows[v] = make_int4((int32_t)(uint32_t)b, (int32_t)(b >> 32), d, (int32_t)(lo - b));
    }
}

// Takes every queued vertex's lanes (clearing them), does the settle bookkeeping and writes queue
// entry i's item (vertex, first edge, lane mask, work = edges x lanes) into slot i; cnt[S_ITEMS]
// = n and pref[n] = 0, so the scan of the n + 1 slots needs nothing cleared beforehand (and the
// near-queue counter starts the pass at zero). Items
// without work stay in place: the relaxation's searches take the largest item whose prefix is at
// most the pair's index, which is never a zero-work item (its prefix equals the next item's).
// A vertex is queued once per pass, so its setmask word is touched by one thread only.
__global__ void k_relax_prep(const int32_t* q, int64_t n, int heavy, Relax a, const int4* rows, Items it) {
    __shared__ int s_w[kBlock / 32];
    __shared__ unsigned long long s_base;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < n; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = base + threadIdx.x;
        int32_t u = 0;
        unsigned long long m = 0;
        int64_t eb = 0, work = 0;
        bool settles = false;
        if (i < n) {
            // (every load of the vertex's words is issued before any store: the stores may alias
            // them for all the compiler knows, and would otherwise serialize three DRAM latencies)
            u = q[i];
            const int4 r = rows[u];
            if (heavy) {
                m = a.setmask[u];
                const unsigned long long dn = a.done[u];
                a.setmask[u] = 0ull;
                a.done[u] = dn | m;  // (u appears once in a heavy pass)
            } else {
                m = a.curmask[u];
                const unsigned long long old = a.setmask[u];
                a.curmask[u] = 0ull;
                a.setmask[u] = old | m;
                settles = m && old == 0ull;
            }
            const int64_t b = (int64_t)(((uint64_t)(uint32_t)r.y << 32) | (uint32_t)r.x);
            const int32_t nlu = r.w;
            eb = heavy ? b + nlu : b;
            work = (int64_t)(heavy ? r.z - nlu : nlu) * __popcll(m);
            it.u[i] = u;
            it.eb[i] = eb;
            it.m[i] = m;
            it.pref[i] = work;
        }
        const unsigned long long ss = block_slot(settles, &a.cnt[S_SET], s_w, &s_base);
        if (settles) a.setq[ss] = u;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        it.pref[n] = 0;
        a.cnt[S_ITEMS] = (unsigned long long)n;
        a.cnt[S_NEAR] = 0ull;  // the pass's near appends count from zero (the host read the last count)
    }
}

constexpr int kRelaxThreads = 256;
// Pairs per thread per step, and CTAs per SM: latency-bound, so occupancy wins. Measured on the
// 4.8M-vertex R-MAT (64 lanes): 1 pair at 8 CTAs (32 registers) 71 ms per call, 7 CTAs the same,
// 6 CTAs 75 ms, 4 CTAs 83 ms; 2 pairs at 6 CTAs 74 ms, at 5 CTAs 76 ms. (With the later changes:
// 256-thread CTAs 66.3 ms, 128-thread CTAs at 16 per SM 66.8 ms.)
constexpr int kPairs = 1;
constexpr int kRelaxMinBlocks = 8;
constexpr int kDeal = 8;  // chunks of pairs per warp and launch, at least 32 pairs each (measured on
                          // the 4.8M-vertex R-MAT: 4 or 8 68.4 ms per call, 16 69.5, 32 72.0)

// Largest e in [lo, hi] with pref[e] <= key, for a non-decreasing pref with pref[lo] <= key
// (the probes at or below the key are a prefix of each round's 32). One warp, 32 probes a round:
// the window shrinks 32-fold per dependent load.
__device__ __forceinline__ int64_t warp_search(const int64_t* pref, int64_t lo, int64_t hi, int64_t key) {
    const int ln = lane_id();
    while (hi > lo) {
        const int64_t step = (hi - lo + 31) / 32;
        const int64_t p = lo + (int64_t)(ln + 1) * step;
        const bool c = p <= hi && pref[p] <= key;
        const int t = __popc(__ballot_sync(0xffffffffu, c));
        if (t > 0) lo += (int64_t)t * step;
        hi = lo + step - 1 < hi ? lo + step - 1 : hi;
    }
    return lo;
}

// Relaxes the pairs this thread holds (pair j: on[j], target w[j], lane sl[j], the source's lane
// distance du[j], edge weight wt[j]); the queue appends are staged per warp (warp-uniform call).
template <class D>
__device__ __forceinline__ void relax_held(D* dist, const Relax& a, const bool (&on)[kPairs], const int32_t (&w)[kPairs],
                                           const int32_t (&sl)[kPairs], const uint64_t (&du)[kPairs],
                                           const uint32_t (&wt)[kPairs], int32_t* s_near, int& n_near, int32_t* s_far,
                                           int& n_far) {
    uint64_t cur[kPairs];
#pragma unroll
    for (int j = 0; j < kPairs; ++j)
        cur[j] = on[j] ? *(volatile D*)&dist[(int64_t)w[j] * a.nl + sl[j]] : (D)0;
#pragma unroll
    for (int j = 0; j < kPairs; ++j) {
        bool to_near = false, to_far = false;
        if (on[j]) {
            const uint64_t nd = du[j] + (uint64_t)wt[j];
            if (sizeof(D) == 2 && nd >= (uint64_t)DistT<D>::inf) {
                // a 16-bit lane cannot hold it: the group is run again with 32-bit lanes
                if (cur[j] == (uint64_t)DistT<D>::inf) a.cnt[S_OVF] = 1ull;
            } else if (nd < cur[j]) {  // plain pre-check: most relaxations lose
                const uint64_t old = DistT<D>::atomic_min(&dist[(int64_t)w[j] * a.nl + sl[j]], (D)nd);
                if (nd < old) {
                    const unsigned long long bit = 1ull << sl[j];
                    if (nd < a.kend) to_near = atomicOr(&a.nextmask[w[j]], bit) == 0ull;
                    else to_far = atomicOr(&a.farmask[w[j]], bit) == 0ull;
                }
            }
        }
        stage_append(to_near, w[j], s_near, n_near, a.nextq, &a.cnt[S_NEAR]);
        stage_append(to_far, w[j], s_far, n_far, a.farq, &a.cnt[S_FAR]);
    }
}

// Load-balanced relaxation over all (edge, lane) pairs of the item list, numbered by the
// exclusive scan of the items' work. Every warp takes one contiguous run of pairs and finds the
// item holding its first pair with one warp search. It then walks windows of 32 consecutive
// items, one item per lane in registers: a pair finds its item by a binary search over the
// window through shuffles, so no shared memory and no block barrier is involved and warps
// proceed independently. Pairs are enumerated edge-major within an item: with many lanes
// active, consecutive threads update consecutive lanes of one distance row.
//
// Where the warp's next steps (32 * kPairs pairs each) all lie inside one item (a hub's row,
// settled in many lanes at once: a few such items hold most of the pairs of the early heavy
// passes), the warp leaves the per-pair search: each thread divides its first pair's rank once,
// then steps its (edge, lane rank) position by the constant 32 * kPairs, and takes the lane from
// a table of the item's set lanes held one per thread (two shuffles instead of a search, a divide
// and a find-n-th-bit per pair). The pairs relaxed are the same either way.
template <class D>
__global__ void __launch_bounds__(kRelaxThreads, kRelaxMinBlocks) k_relax(const unsigned long long* n_items, Items it, Relax a) {
    D* const dist = static_cast<D*>(a.dist);
    const int64_t n = (int64_t)*n_items;
    if (n == 0) return;
    const int64_t total = it.pref[n];
    __shared__ int32_t s_near[kRelaxThreads / 32][kStage], s_far[kRelaxThreads / 32][kStage];
    int32_t* const my_near = s_near[threadIdx.x >> 5];
    int32_t* const my_far = s_far[threadIdx.x >> 5];
    int n_near = 0, n_far = 0;
    const int ln = lane_id();
    const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    constexpr int kStep = 32 * kPairs;
    // The pairs are dealt in chunks, round-robin over the warps (about kDeal chunks per warp), so
    // every warp gets a mix of cheap pairs (long items, the fast path below) and costly ones
    // (short items): one contiguous run per warp left the warps inside short items running
    // 1.75x longer than the average SM in the first heavy passes.
    const int64_t chunk = (((total + nw * kDeal - 1) / (nw * kDeal)) + 31) & ~(int64_t)31;
    int64_t e_from = 0;  // (a warp's chunks ascend: each search starts at the previous chunk's item)
    for (int64_t c0 = gw * chunk; c0 < total; c0 += nw * chunk) {
        const int64_t c1 = c0 + chunk < total ? c0 + chunk : total;
        int64_t e0 = warp_search(it.pref, e_from, n - 1, c0);
        e_from = e0;
        int64_t p = c0;
        while (p < c1) {
            // window: items e0 .. e0+31, lane j holding item e0+j
            const int64_t ej = e0 + ln;
            int64_t pj = INT64_MAX, ebj = 0;
            unsigned long long mj = 0;
            int32_t uj = 0;
            if (ej < n) {
                pj = it.pref[ej];
                ebj = it.eb[ej];
                mj = it.m[ej];
                uj = it.u[ej];
            }
            const int64_t wnext = e0 + 32 < n ? it.pref[e0 + 32] : total;
            const int64_t wend = wnext < c1 ? wnext : c1;
            while (p < wend) {
                {
                    // the item holding pair p (the same for every thread) and where its run ends
                    int x = 0;
    #pragma unroll
                    for (int b = 16; b; b >>= 1) {
                        const int64_t v = __shfl_sync(0xffffffffu, pj, x + b);
                        if (v <= p) x += b;
                    }
                    const int64_t pn = __shfl_sync(0xffffffffu, pj, (x + 1) & 31);
                    const int64_t xend = x < 31 ? (pn < wend ? pn : wend) : wend;
                    if (xend - p >= 2 * kStep) {
                        const int64_t px = __shfl_sync(0xffffffffu, pj, x);
                        const int64_t ebx = __shfl_sync(0xffffffffu, ebj, x);
                        const unsigned long long mx = __shfl_sync(0xffffffffu, mj, x);
                        const int64_t urow = (int64_t)__shfl_sync(0xffffffffu, uj, x) * a.nl;
                        const int pc = __popcll(mx);
                        const int32_t sel_lo = ln < pc ? nth_bit(mx, ln) : 0;
                        const int32_t sel_hi = ln + 32 < pc ? nth_bit(mx, ln + 32) : 0;
                        const int da = kStep / pc, db = kStep % pc;
                        int64_t e[kPairs];  // the pair's entry of the weight-sorted rows (ebx + edge)
                        int r[kPairs];
    #pragma unroll
                        for (int j = 0; j < kPairs; ++j) {
                            const int64_t q2 = p + j * 32 + ln - px;
                            const int64_t ed = q2 / pc;
                            r[j] = (int)(q2 - ed * pc);
                            e[j] = ebx + ed;
                        }
                        for (; p + kStep <= xend; p += kStep) {
                            bool on[kPairs];
                            int32_t w[kPairs], sl[kPairs];
                            uint64_t du[kPairs];
                            uint32_t wt[kPairs];
    #pragma unroll
                            for (int j = 0; j < kPairs; ++j) {
                                const int32_t lo = __shfl_sync(0xffffffffu, sel_lo, r[j] & 31);
                                const int32_t hi = __shfl_sync(0xffffffffu, sel_hi, r[j] & 31);
                                sl[j] = r[j] < 32 ? lo : hi;
                                on[j] = true;
                                w[j] = __ldcs(&a.wadj[e[j]]);
                                wt[j] = __ldcs(&a.ww[e[j]]);
                                du[j] = dist[urow + sl[j]];
                                e[j] += da;
                                r[j] += db;
                                if (r[j] >= pc) {
                                    r[j] -= pc;
                                    e[j] += 1;
                                }
                            }
                            relax_held<D>(dist, a, on, w, sl, du, wt, my_near, n_near, my_far, n_far);
                        }
                        continue;  // (what is left of the item, under one step, goes the general way)
                    }
                }
                int32_t w[kPairs], sl[kPairs];
                int64_t k[kPairs];
                uint64_t du[kPairs];
                bool on[kPairs];
    #pragma unroll
                for (int j = 0; j < kPairs; ++j) {
                    const int64_t q = p + j * 32 + ln;
                    on[j] = q < wend;
                    int x = 0;  // largest x with pref(x) <= q
    #pragma unroll
                    for (int b = 16; b; b >>= 1) {
                        const int64_t v = __shfl_sync(0xffffffffu, pj, x + b);
                        if (v <= q) x += b;
                    }
                    const int64_t px = __shfl_sync(0xffffffffu, pj, x);
                    const int64_t ebx = __shfl_sync(0xffffffffu, ebj, x);
                    const unsigned long long mx = __shfl_sync(0xffffffffu, mj, x);
                    const int32_t ux = __shfl_sync(0xffffffffu, uj, x);
                    if (on[j]) {
                        const int pc = __popcll(mx);
                        const int64_t q2 = q - px;
                        // (an item of 2^31 pairs or more, a row of over 2^25 entries, takes the wide divide)
                        const int64_t ed = q2 <= INT32_MAX ? (int64_t)((uint32_t)q2 / (uint32_t)pc) : q2 / pc;
                        k[j] = ebx + ed;
                        sl[j] = nth_bit(mx, (int)(q2 - ed * pc));
                        du[j] = dist[(int64_t)ux * a.nl + sl[j]];
                    }
                }
                uint32_t wt[kPairs];
    #pragma unroll
                for (int j = 0; j < kPairs; ++j) {
                    if (on[j]) { w[j] = __ldcs(&a.wadj[k[j]]); wt[j] = __ldcs(&a.ww[k[j]]); } else { w[j] = 0; wt[j] = 0; }
                }
                relax_held<D>(dist, a, on, w, sl, du, wt, my_near, n_near, my_far, n_far);
                p += kStep;
            }
            p = wend;  // (the pairs of this window end exactly where item e0+32 begins)
            if (p >= c1) break;
            // Items without work keep their slots (their prefix equals the next item's): where the
            // whole next window is such items, jump past the run with one search instead of
            // walking it 32 items at a time (a heavy pass on a lattice can hold millions of them).
            const int64_t nx = e0 + 32;
            e0 = nx + 32 < n && it.pref[nx + 32] <= p ? warp_search(it.pref, nx, n - 1, p) : nx;
        }
    }
    stage_flush(my_near, n_near, a.nextq, &a.cnt[S_NEAR]);
    stage_flush(my_far, n_far, a.farq, &a.cnt[S_FAR]);
}

// Splits the far entries at the bucket [lo, hi): lanes inside it become near work, later lanes
// stay far (queued in farq2) and their smallest distance goes to cnt[S_MIN] (the bucket to jump
// to when this one turns out empty); settled lanes are dropped.
template <class D>
__global__ void k_far_split(const int32_t* farq, const unsigned long long* nfar, unsigned long long* farmask,
                            const D* dist, int nl, uint64_t lo, uint64_t hi, unsigned long long* nearmask,
                            int32_t* nearq, int32_t* farq2, const unsigned long long* done, unsigned long long* cnt) {
    const int64_t n = (int64_t)*nfar;
    __shared__ int32_t s_near[kBlock / 32][kStage], s_far[kBlock / 32][kStage];
    int n_near = 0, n_far = 0;
    const int ln = lane_id();
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < n; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = base + threadIdx.x;
        int32_t w = 0;
        unsigned long long m = 0;
        if (i < n) {
            w = farq[i];
            // (lanes already final were reached by a shorter path since: dropped unread)
            m = farmask[w] & ~done[w];
        }
        // The warp takes its 32 entries in turn and reads each entry's distance row once, lanes
        // ln and ln + 32 per thread (coalesced); ballots give the entry's near and kept lanes.
        unsigned long long mn = kInf, my_near = 0, my_keep = 0;
#pragma unroll 4
        for (int j = 0; j < 32; ++j) {
            const unsigned long long mj = __shfl_sync(0xffffffffu, m, j);
            if (mj == 0ull) continue;  // (warp-uniform)
            const int64_t row = (int64_t)__shfl_sync(0xffffffffu, w, j) * nl;
            bool n0 = false, n1 = false, k0 = false, k1 = false;
            if ((mj >> ln) & 1ull) {
                const uint64_t d = dist[row + ln];
                n0 = d >= lo && d < hi;
                k0 = d >= hi;
                if (k0) mn = d < mn ? d : mn;
            }
            if ((mj >> 32 >> ln) & 1ull) {
                const uint64_t d = dist[row + 32 + ln];
                n1 = d >= lo && d < hi;
                k1 = d >= hi;
                if (k1) mn = d < mn ? d : mn;
            }
            const unsigned long long nm = (unsigned long long)__ballot_sync(0xffffffffu, n0) |
                                          ((unsigned long long)__ballot_sync(0xffffffffu, n1) << 32);
            const unsigned long long kp = (unsigned long long)__ballot_sync(0xffffffffu, k0) |
                                          ((unsigned long long)__ballot_sync(0xffffffffu, k1) << 32);
            if (ln == j) {
                my_near = nm;
                my_keep = kp;
            }
        }
        bool to_near = false, to_far = false;
        if (i < n) {
            farmask[w] = my_keep;
            to_far = my_keep != 0ull;
            if (my_near) to_near = atomicOr(&nearmask[w], my_near) == 0ull;
        }
        stage_append(to_near, w, s_near[threadIdx.x >> 5], n_near, nearq, &cnt[S_NEAR]);
        stage_append(to_far, w, s_far[threadIdx.x >> 5], n_far, farq2, &cnt[S_FAR2]);
        for (int o = 16; o; o >>= 1) {
            const unsigned long long t = __shfl_xor_sync(0xffffffffu, mn, o);
            mn = t < mn ? t : mn;
        }
        if (ln == 0 && mn != kInf) atomicMin(&cnt[S_MIN], mn);
    }
    stage_flush(s_near[threadIdx.x >> 5], n_near, nearq, &cnt[S_NEAR]);
    stage_flush(s_far[threadIdx.x >> 5], n_far, farq2, &cnt[S_FAR2]);
}

// Reached (vertex, lane) pairs and their out-degrees (the traversed edges of the GTEPS figure).
template <class D>
__global__ void k_sssp_reached(const D* dist, int64_t V, int nl, const int32_t* outdeg,
                               unsigned long long* cnt) {
    unsigned long long r = 0, e = 0;
    GRID_STRIDE(v, V) {
        unsigned c = 0;
        for (int s = 0; s < nl; ++s) c += dist[v * nl + s] != DistT<D>::inf;
        r += c;
        e += (unsigned long long)c * (unsigned long long)outdeg[v];
    }
    for (int o = 16; o; o >>= 1) {
        r += __shfl_xor_sync(0xffffffffu, r, o);
        e += __shfl_xor_sync(0xffffffffu, e, o);
    }
    if (lane_id() == 0) {
        if (r) atomicAdd(&cnt[S_REACHED], r);
        if (e) atomicAdd(&cnt[S_EDGES], e);
    }
}

// dist[v * nl + s] -> out[row[s] * V + v], through 32 x 32 shared-memory tiles, a fixed grid
// striding over the tiles. On the way it counts what k_sssp_reached counts (reached (vertex, lane)
// pairs and their out-edges) from the same coalesced loads, with one atomicAdd per CTA.
template <class D>
__global__ void k_transpose(const D* dist, int64_t V, int nl, const int64_t* row, const int32_t* outdeg,
                            uint64_t* out, unsigned long long* cnt) {
    __shared__ uint64_t tile[32][33];
    __shared__ unsigned long long s_r[8], s_e[8];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
    const int64_t tiles_v = (V + 31) / 32, tiles_s = (nl + 31) / 32;
    unsigned long long r_cnt = 0, e_cnt = 0;
    for (int64_t t = blockIdx.x; t < tiles_v * tiles_s; t += gridDim.x) {
        const int64_t v0 = (t % tiles_v) * 32;
        const int s0 = (int)(t / tiles_v) * 32;
        for (int r = ty; r < 32; r += 8) {
            const int64_t v = v0 + r;
            const int s = s0 + tx;
            if (v < V && s < nl) {
                const D d = dist[v * nl + s];
                const bool fin = d != DistT<D>::inf;
                tile[r][tx] = fin ? (uint64_t)d : kInf;
                if (fin) {
                    ++r_cnt;
                    e_cnt += (unsigned long long)outdeg[v];
                }
            }
        }
        __syncthreads();
        for (int r = ty; r < 32; r += 8) {
            const int s = s0 + r;
            const int64_t v = v0 + tx;
            if (v < V && s < nl) out[row[s] * V + v] = tile[tx][r];
        }
        __syncthreads();
    }
    for (int o = 16; o; o >>= 1) {
        r_cnt += __shfl_xor_sync(0xffffffffu, r_cnt, o);
        e_cnt += __shfl_xor_sync(0xffffffffu, e_cnt, o);
    }
    if (tx == 0) {
        s_r[ty] = r_cnt;
        s_e[ty] = e_cnt;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long rr = 0, ee = 0;
        for (int k = 0; k < 8; ++k) {
            rr += s_r[k];
            ee += s_e[k];
        }
        if (rr) atomicAdd(&cnt[S_REACHED], rr);
        if (ee) atomicAdd(&cnt[S_EDGES], ee);
    }
}

// Lane-order key of every query set: the smallest distance to the hub over the set's sources
// (UINT64_MAX when none reaches it or none is in range).
__global__ void k_set_keys(const int64_t* set_beg, int64_t n_sets, const int32_t* srcs, int64_t V,
                           const uint64_t* hub_dist, uint64_t* key) {
    GRID_STRIDE(i, n_sets) {
        uint64_t k = kInf;
        for (int64_t e = set_beg[i]; e < set_beg[i + 1]; ++e) {
            const int32_t v = srcs[e];
            if (v >= 0 && v < V) k = hub_dist[v] < k ? hub_dist[v] : k;
        }
        key[i] = k;
    }
}

// The vertex of largest in-degree (smallest id among ties) as in-degree << 32 | ~id, and the
// largest finite value of a distance array: st[0], st[1] (atomicMax).
__global__ void k_argmax_deg(int64_t V, const int32_t* deg, unsigned long long* st) {
    unsigned long long best = 0;
    GRID_STRIDE(v, V) {
        const unsigned long long k = ((unsigned long long)(uint32_t)deg[v] << 32) | (uint32_t)~(uint32_t)v;
        best = k > best ? k : best;
    }
    for (int o = 16; o; o >>= 1) {
        const unsigned long long t = __shfl_xor_sync(0xffffffffu, best, o);
        best = t > best ? t : best;
    }
    if (lane_id() == 0) atomicMax(&st[0], best);
}
__global__ void k_max_finite(int64_t V, const uint64_t* d, unsigned long long* st) {
    unsigned long long m = 0;
    GRID_STRIDE(v, V) if (d[v] != kInf && d[v] > m) m = d[v];
    for (int o = 16; o; o >>= 1) {
        const unsigned long long t = __shfl_xor_sync(0xffffffffu, m, o);
        m = t > m ? t : m;
    }
    if (lane_id() == 0) atomicMax(&st[1], m);
}

}  // namespace

// Weight-sorted compact copy of the forward CSR for one weight mode; with `reverse`, of the
// backward CSR, each entry (v <- u) carrying the weight of the forward edge u -> v.
static int build_weight_sorted(gir_dev* g, int hash, int reverse, DevCSR& ws) {
    const DevCSR& c = reverse ? g->bw : g->fw;
    const int64_t V = g->V, E = c.E;
    store_free(g, ws);
    uint64_t *keys = nullptr, *ktmp = nullptr;
    uint32_t *cols = nullptr, *ctmp = nullptr;
    GIR_TRY(dev_alloc_n(g, &ws.beg, V + 1));
    GIR_TRY(dev_alloc_n(g, &ws.deg, V > 0 ? V : 1));
    GIR_TRY(dev_alloc_n(g, &ws.adj, E > 0 ? E : 1));
    GIR_TRY(dev_alloc_n(g, &ws.w, E > 0 ? E : 1));
    ws.cap = ws.E = E;
    int64_t* cb = ws.beg;
    k_deg_i64<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, c.deg, cb);
    GIR_LAUNCH(g, "k_deg_i64");
    GIR_TRY(exclusive_scan_i64(g, cb, cb, V + 1));
    GIR_CUDA(g, cudaMemcpyAsync(ws.deg, c.deg, sizeof(int32_t) * V, cudaMemcpyDeviceToDevice, g->stream));
    if (E == 0) return GIR_OK;
    GIR_TRY(ensure_n(g, g->scratch[8], E, &keys));
    GIR_TRY(ensure_n(g, g->scratch[9], E, &ktmp));
    GIR_TRY(ensure_n(g, g->scratch[10], E, &cols));
    GIR_TRY(ensure_n(g, g->scratch[11], E, &ctmp));
    k_ws_keys<<<grid_for(g, E, kBlock), kBlock, 0, g->stream>>>(V, E, cb, view(c), hash, reverse, view(g->fw), keys,
                                                                 cols);
    GIR_LAUNCH(g, "k_ws_keys");
    GIR_TRY(sort_pairs_u64(g, keys, ktmp, cols, ctmp, E, 64));
    k_ws_split<<<grid_for(g, E, kBlock), kBlock, 0, g->stream>>>(E, keys, cols, ws.adj, ws.w);
    GIR_LAUNCH(g, "k_ws_split");
    if (reverse) return GIR_OK;
    // weight statistics for the schedule's features
    unsigned long long* st = reinterpret_cast<unsigned long long*>(ktmp);
    GIR_CUDA(g, cudaMemsetAsync(st, 0, 2 * sizeof(unsigned long long), g->stream));
    k_wstat<<<grid_for(g, E, kBlock), kBlock, 0, g->stream>>>(ws.w, E, st);
    GIR_LAUNCH(g, "k_wstat");
    unsigned long long h[2] = {0, 0};
    GIR_CUDA(g, cudaMemcpyAsync(h, st, sizeof(h), cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    g->wstat[hash ? 0 : 1][0] = (double)h[0] / (double)E;
    g->wstat[hash ? 0 : 1][1] = (double)h[1];
    return GIR_OK;
}

namespace {

// Working arrays of one SSSP call, sized for V vertices and up to 64 lanes.
struct Work {
    int32_t *nearq, *nextq, *farq, *farq2, *setq;
    unsigned long long *curmask, *nextmask, *farmask, *setmask, *done, *cnt;
    int4* rows;
    Items items;
    unsigned long long* hc;  // pinned host copy of the counters
};

int sssp_work(gir_dev* g, Work& w) {
    const int64_t V = g->V;
    GIR_TRY(ensure_n(g, g->scratch[0], V + 1, &w.nearq));
    GIR_TRY(ensure_n(g, g->scratch[1], V + 1, &w.nextq));
    GIR_TRY(ensure_n(g, g->scratch[2], V + 1, &w.farq));
    GIR_TRY(ensure_n(g, g->scratch[3], V + 1, &w.farq2));
    GIR_TRY(ensure_n(g, g->scratch[4], V + 1, &w.setq));
    GIR_TRY(ensure_n(g, g->scratch[5], V + 1, &w.curmask));
    GIR_TRY(ensure_n(g, g->scratch[6], V + 1, &w.nextmask));
    GIR_TRY(ensure_n(g, g->scratch[7], V + 1, &w.farmask));
    GIR_TRY(ensure_n(g, g->scratch[12], V + 1, &w.setmask));
    GIR_TRY(ensure_n(g, g->sssp_done, V + 1, &w.done));
    GIR_TRY(ensure_n(g, g->scratch[13], S_N, &w.cnt));
    GIR_TRY(ensure_n(g, g->qitems[3], V + 1, &w.rows));
    GIR_TRY(ensure_n(g, g->qitems[0], V + 1, &w.items.u));
    GIR_TRY(ensure_n(g, g->qitems[1], V + 1, &w.items.eb));
    GIR_TRY(ensure_n(g, g->qitems[2], V + 1, &w.items.m));
    GIR_TRY(ensure_n(g, g->qitems[4], V + 2, &w.items.pref));
    void* h = nullptr;
    GIR_TRY(pinned(g, 256, &h));
    w.hc = static_cast<unsigned long long*>(h);
    return GIR_OK;
}

// One group of nl lanes (1..64) over the weight-sorted rows `ws`: lane s starts from
// srcs[lane_rng[2s] .. lane_rng[2s + 1]) (device arrays, n_entries sources in all). Lane
// distances have the type D. With nl == 1 and 64-bit lanes the result is written straight into
// `out` (V entries); otherwise lane s ends in row lane_row[s] of `out` (rows of V). A 16-bit run
// that met a distance it cannot hold sets *overflow and writes nothing.
template <class D>
int sssp_group(gir_dev* g, Work& wk, const DevCSR& ws, int nl, const int64_t* lane_rng_d, const int32_t* srcs_d,
               int64_t n_entries, const int64_t* lane_row_d, uint64_t* out, uint64_t Dw, bool* overflow) {
    const int64_t V = g->V;
    QueryStats& st = g->qstats;
    *overflow = false;
    unsigned long long* cnt = wk.cnt;
    unsigned long long* hc = wk.hc;
    auto read = [&]() -> int {
        GIR_CUDA(g, cudaMemcpyAsync(hc, cnt, sizeof(unsigned long long) * S_N, cudaMemcpyDeviceToHost, g->stream));
        GIR_CUDA(g, cudaStreamSynchronize(g->stream));
        return GIR_OK;
    };
    const bool direct = nl == 1 && sizeof(D) == sizeof(uint64_t);
    D* dist = nullptr;
    if (direct) {
        dist = reinterpret_cast<D*>(out);
    } else {
        GIR_TRY(ensure_n(g, g->lane_dist, (size_t)V * nl * sizeof(D) / sizeof(uint64_t) + 1,
                         reinterpret_cast<uint64_t**>(&dist)));
    }
    int per_sm = 0;
    GIR_CUDA(g, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_relax<D>, kRelaxThreads, 0));
    const int run_grid = g->num_sms * (per_sm > 0 ? per_sm : 1);
    MainTimer timer{g, g->params[GIR_PARAM_PROFILE] != 0.0};
    int32_t *nearq = wk.nearq, *nextq = wk.nextq, *farq = wk.farq, *farq2 = wk.farq2;
    unsigned long long *curmask = wk.curmask, *nextmask = wk.nextmask;
    // (a group that ends on settled-only far entries leaves their lane bits behind)
    GIR_CUDA(g, cudaMemsetAsync(curmask, 0, sizeof(unsigned long long) * V, g->stream));
    GIR_CUDA(g, cudaMemsetAsync(nextmask, 0, sizeof(unsigned long long) * V, g->stream));
    GIR_CUDA(g, cudaMemsetAsync(wk.farmask, 0, sizeof(unsigned long long) * V, g->stream));
    GIR_CUDA(g, cudaMemsetAsync(wk.setmask, 0, sizeof(unsigned long long) * V, g->stream));
    GIR_CUDA(g, cudaMemsetAsync(wk.done, 0, sizeof(unsigned long long) * V, g->stream));
    GIR_CUDA(g, cudaMemsetAsync(dist, 0xff, sizeof(D) * V * nl, g->stream));
    for (int k = 0; k < S_N; ++k)
        if (k != S_REACHED && k != S_EDGES) hc[k] = 0;
    GIR_CUDA(g, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * 16, g->stream));
    if (n_entries > 0) {
        const int gx = (int)((n_entries / nl + kBlock - 1) / kBlock > 0 ? (n_entries / nl + kBlock - 1) / kBlock : 1);
        k_sssp_init<D><<<dim3(gx < 1024 ? gx : 1024, nl), kBlock, 0, g->stream>>>(lane_rng_d, srcs_d, V, nl, dist,
                                                                                  curmask, nearq, cnt);
        GIR_LAUNCH(g, "k_sssp_init");
    }
    GIR_TRY(read());
    int64_t n_near = (int64_t)hc[S_NEAR], n_far = 0;
    Relax a;
    a.wb = ws.beg; a.wdeg = ws.deg; a.wadj = ws.adj; a.ww = ws.w; a.delta = Dw; a.nl = nl; a.dist = dist;
    a.farmask = wk.farmask; a.setmask = wk.setmask; a.setq = wk.setq; a.done = wk.done; a.cnt = cnt;
    uint64_t k = 0;
    int64_t trace_pairs = 0, trace_passes = 0;
    k_light_split<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, ws.beg, ws.deg, ws.w, Dw, wk.rows);
    GIR_LAUNCH(g, "k_light_split");
    Items items = wk.items;
    // one relaxation pass over queue q (n entries): prep, scan of the work, balanced run
    auto relax = [&](const int32_t* q, int64_t n, int heavy) -> int {
        k_relax_prep<<<grid_for(g, n, kBlock), kBlock, 0, g->stream>>>(q, n, heavy, a, wk.rows, items);
        GIR_LAUNCH(g, "k_relax_prep");
        GIR_TRY(exclusive_scan_i64(g, items.pref, items.pref, n + 1));
        if (g->trace_marks) {
            int64_t tot = 0;
            GIR_CUDA(g, cudaMemcpyAsync(&tot, items.pref + n, sizeof(int64_t), cudaMemcpyDeviceToHost, g->stream));
            GIR_CUDA(g, cudaStreamSynchronize(g->stream));
            trace_pairs += tot;
            ++trace_passes;
        }
        GIR_TRY(timer.run([&]() -> int {
            k_relax<D><<<run_grid, kRelaxThreads, 0, g->stream>>>(cnt + S_ITEMS, items, a);
            GIR_LAUNCH(g, "k_relax");
            return GIR_OK;
        }));
        st.launches += 4;  // prep, the scan's two kernels, the relaxation
        return GIR_OK;
    };
    while (true) {
        a.kend = (k + 1) * Dw;
        GIR_CUDA(g, cudaMemsetAsync(cnt + S_SET, 0, sizeof(unsigned long long), g->stream));
        // light rounds: nearq (lanes in curmask) -> nextq (lanes in nextmask)
        while (n_near > 0) {
            a.curmask = curmask; a.nextmask = nextmask; a.nextq = nextq; a.farq = farq;
            GIR_TRY(relax(nearq, n_near, 0));
            st.iterations++;
            std::swap(nearq, nextq);
            std::swap(curmask, nextmask);
            GIR_TRY(read());
            n_near = (int64_t)hc[S_NEAR];
        }
        // heavy edges of the (vertex, lane) pairs settled in this bucket
        const int64_t n_set = (int64_t)hc[S_SET];
        if (n_set > 0) {
            a.curmask = curmask; a.nextmask = nextmask; a.nextq = nextq; a.farq = farq;
            GIR_TRY(relax(wk.setq, n_set, 1));
        }
        // next bucket: split the far entries at bucket k + 1; when that one is empty, jump to
        // the bucket of the smallest distance still far
        GIR_TRY(read());
        n_far = (int64_t)hc[S_FAR];
        if (n_far == 0) break;
        uint64_t lo = a.kend;
        bool finished = false;
        while (true) {
            k = lo / Dw;
            GIR_CUDA(g, cudaMemsetAsync(cnt + S_MIN, 0xff, sizeof(unsigned long long), g->stream));
            GIR_CUDA(g, cudaMemsetAsync(cnt + S_FAR2, 0, sizeof(unsigned long long), g->stream));
            k_far_split<D><<<grid_for(g, n_far, kBlock), kBlock, 0, g->stream>>>(
                farq, cnt + S_FAR, wk.farmask, dist, nl, k * Dw, (k + 1) * Dw, curmask, nearq, farq2, wk.done, cnt);
            GIR_LAUNCH(g, "k_far_split");
            st.launches++;
            std::swap(farq, farq2);
            GIR_CUDA(g, cudaMemcpyAsync(cnt + S_FAR, cnt + S_FAR2, sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
                                        g->stream));
            GIR_TRY(read());
            n_near = (int64_t)hc[S_NEAR];
            n_far = (int64_t)hc[S_FAR];
            if (n_near > 0) break;
            if (hc[S_MIN] == kInf) {  // nothing live is left far
                finished = true;
                break;
            }
            lo = hc[S_MIN];
        }
        if (finished) break;
    }
    if (g->trace_marks)
        std::fprintf(stderr, "[gir] sssp group of %d lanes, %d-bit distances, delta %llu: %lld passes, %lld (edge, lane) pairs\n",
                     nl, (int)(8 * sizeof(D)), (unsigned long long)Dw, (long long)trace_passes, (long long)trace_pairs);
    if (sizeof(D) == sizeof(uint16_t)) {
        GIR_TRY(read());
        if (hc[S_OVF]) {
            *overflow = true;
            return GIR_OK;
        }
    }
    if (!direct) {  // (the transpose also counts the reached pairs and their edges)
        k_transpose<D><<<g->num_sms * 8, 256, 0, g->stream>>>(dist, V, nl, lane_row_d, g->fw.deg, out, cnt);
        GIR_LAUNCH(g, "k_transpose");
    } else {
        k_sssp_reached<D><<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(dist, V, nl, g->fw.deg, cnt);
        GIR_LAUNCH(g, "k_sssp_reached");
    }
    return GIR_OK;
}

}  // namespace

// The lane order of a weight mode (hub_dist, hub_max): one backward single-lane run from the
// vertex of largest in-degree over a temporary weight-sorted copy of the backward CSR.
static int hub_order(gir_dev* g, int hash) {
    const int mi = hash ? 0 : 1;
    if (g->hub_valid[mi]) return GIR_OK;
    const int64_t V = g->V;
    const double t0 = now_ms();
    const QueryStats saved = g->qstats;
    uint64_t* hd = nullptr;
    GIR_TRY(ensure_n(g, g->hub_dist[mi], V, &hd));
    DevCSR wsb;
    int rc = build_weight_sorted(g, hash, 1, wsb);
    Work wk;
    if (!rc) rc = sssp_work(g, wk);
    int64_t* lanes = nullptr;
    if (!rc) rc = ensure_n(g, g->sssp_lanes, 4, &lanes);
    unsigned long long st[2] = {0, 0};
    if (!rc) rc = cuda_check(g, cudaMemsetAsync(wk.cnt + 24, 0, 2 * sizeof(unsigned long long), g->stream), "memset");
    if (!rc) {
        k_argmax_deg<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, g->bw.deg, wk.cnt + 24);
        rc = cuda_check(g, cudaGetLastError(), "k_argmax_deg");
    }
    if (!rc) rc = cuda_check(g, cudaMemcpyAsync(st, wk.cnt + 24, sizeof(st), cudaMemcpyDeviceToHost, g->stream), "copy");
    if (!rc) rc = cuda_check(g, cudaStreamSynchronize(g->stream), "sync");
    if (!rc) {
        const int32_t hub = (int32_t)~(uint32_t)(st[0] & 0xffffffffull);
        const int64_t h_lane[2] = {0, 1};
        int32_t* src_d = reinterpret_cast<int32_t*>(lanes + 2);
        rc = cuda_check(g, cudaMemcpyAsync(lanes, h_lane, sizeof(h_lane), cudaMemcpyHostToDevice, g->stream), "copy");
        if (!rc) rc = cuda_check(g, cudaMemcpyAsync(src_d, &hub, sizeof(hub), cudaMemcpyHostToDevice, g->stream), "copy");
        bool ovf = false;
        if (!rc) rc = sssp_group<uint64_t>(g, wk, wsb, 1, lanes, src_d, 1, nullptr, hd, 16, &ovf);
        if (!rc) rc = cuda_check(g, cudaMemsetAsync(wk.cnt + 25, 0, sizeof(unsigned long long), g->stream), "memset");
        if (!rc) {
            k_max_finite<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, hd, wk.cnt + 24);
            rc = cuda_check(g, cudaGetLastError(), "k_max_finite");
        }
        if (!rc) rc = cuda_check(g, cudaMemcpyAsync(st, wk.cnt + 24, sizeof(st), cudaMemcpyDeviceToHost, g->stream), "copy");
        if (!rc) rc = cuda_check(g, cudaStreamSynchronize(g->stream), "sync");
        if (!rc) {
            g->hub_max[mi] = st[1];
            g->hub_valid[mi] = true;
        }
    }
    store_free(g, wsb);
    g->qstats = saved;
    if (g->trace_on)
        std::fprintf(stderr, "[gir] sssp lane order (backward run from the hub, %s weights): %.3f ms, max %llu\n",
                     hash ? "hash" : "stored", now_ms() - t0, (unsigned long long)g->hub_max[mi]);
    return rc;
}

int sssp_run(gir_dev* g, const int64_t* set_beg_h, const int32_t* srcs_d, int64_t n_sets, uint64_t delta,
             int weight_mode, uint64_t* dist_d) {
    const int64_t V = g->V;
    QueryStats& st = g->qstats;
    st = QueryStats{};
    g->trace_x.clear();
    g->trace_y.clear();
    if (n_sets <= 0) return GIR_OK;
    GIR_CUDA(g, cudaMemsetAsync(dist_d, 0xff, sizeof(uint64_t) * V * n_sets, g->stream));
    if (V == 0) return GIR_OK;
    const int hash = weight_mode == GIR_WEIGHT_HASH;
    const int mi = hash ? 0 : 1;
    if (!hash && !g->has_weights) return fail(g, GIR_ERR_STATE, "sssp: the graph has no stored weights");
    DevCSR& ws = g->ws[mi];
    if (!g->ws_valid[mi]) {
        GIR_TRY(build_weight_sorted(g, hash, 0, ws));
        g->ws_valid[mi] = true;
    }
    // Lane order: sets sorted by their distance to the hub, so that neighbouring lanes (which
    // share the 32-byte sectors of a distance row) tend to be active in the same buckets. Only
    // the placement of the queries changes, never their results.
    std::vector<int64_t> order((size_t)n_sets);
    for (int64_t i = 0; i < n_sets; ++i) order[i] = i;
    if (n_sets > 1 && g->params[GIR_PARAM_LANE_ORDER] != 0.0) {
        GIR_TRY(hub_order(g, hash));
        int64_t* sb = nullptr;
        GIR_TRY(ensure_n(g, g->sssp_sets, 2 * n_sets + 1, &sb));
        uint64_t* key_d = reinterpret_cast<uint64_t*>(sb + n_sets + 1);
        GIR_CUDA(g, cudaMemcpyAsync(sb, set_beg_h, sizeof(int64_t) * (n_sets + 1), cudaMemcpyHostToDevice, g->stream));
        k_set_keys<<<grid_for(g, n_sets, kBlock), kBlock, 0, g->stream>>>(
            sb, n_sets, srcs_d, V, static_cast<const uint64_t*>(g->hub_dist[mi].p), key_d);
        GIR_LAUNCH(g, "k_set_keys");
        std::vector<uint64_t> key((size_t)n_sets);
        GIR_CUDA(g, cudaMemcpyAsync(key.data(), key_d, sizeof(uint64_t) * n_sets, cudaMemcpyDeviceToHost, g->stream));
        GIR_CUDA(g, cudaStreamSynchronize(g->stream));
        std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) { return key[x] < key[y]; });
    }
    Work wk;
    GIR_TRY(sssp_work(g, wk));
    int64_t* lanes = nullptr;  // lane ranges (2 per lane), then output rows (1 per lane)
    GIR_TRY(ensure_n(g, g->sssp_lanes, 3 * 64, &lanes));
    // Lane distance width (GIR_PARAM_LANE_BITS): by default 32 bits when every finite distance
    // fits ((V - 1) x max weight), else 64. 16 bits are taken only when asked for, and only while
    // no 16-bit run of this handle has overflowed (an overflow reruns the group wider, so the
    // width never changes a result): their minimum is a compare-and-swap on the 32-bit word the
    // lane shares with its neighbour, and neighbouring lanes active together make those swaps
    // retry (measured slower than 32-bit atomicMin on the LJ-shape graph).
    const double wmax = g->wstat[mi][1] > 0 ? g->wstat[mi][1] : 4294967295.0;
    const int bits = (int)g->params[GIR_PARAM_LANE_BITS];
    const bool fits32 = bits != 64 && (double)V * wmax < 4294967295.0;
    const bool try16 = bits == 16 && !g->narrow16_failed[mi];
    GIR_CUDA(g, cudaEventRecord(g->ev0, g->stream));
    GIR_CUDA(g, cudaMemsetAsync(wk.cnt, 0, sizeof(unsigned long long) * S_N, g->stream));
    std::vector<int64_t> lh(3 * 64);
    for (int64_t g0 = 0; g0 < n_sets; g0 += 64) {
        const int nl = (int)((n_sets - g0) < 64 ? (n_sets - g0) : 64);
        int64_t n_entries = 0;
        for (int j = 0; j < nl; ++j) {
            const int64_t q = order[g0 + j];
            lh[2 * j] = set_beg_h[q];
            lh[2 * j + 1] = set_beg_h[q + 1];
            lh[2 * nl + j] = q;
            n_entries += set_beg_h[q + 1] - set_beg_h[q];
        }
        GIR_CUDA(g, cudaMemcpyAsync(lanes, lh.data(), sizeof(int64_t) * 3 * nl, cudaMemcpyHostToDevice, g->stream));
        uint64_t D = delta;
        float feat[GIR_SCHED_IN];
        sched_sssp_features(g, weight_mode, nl, feat);
        if (D == 0) {
            if (g->schedule == GIR_SCHEDULE_LEARNED && g->sched_loaded) {
                GIR_TRY(sched_choose_delta(g, feat, &D));
            } else {
                D = (uint64_t)g->params[GIR_PARAM_DELTA];
            }
            if (D == 0) D = 16;
        }
        sched_trace(g, feat, sched_delta_class(D));
        bool ovf = false;
        if (nl == 1) {
            GIR_TRY(sssp_group<uint64_t>(g, wk, ws, 1, lanes, srcs_d, n_entries, nullptr, dist_d + order[g0] * V, D, &ovf));
            continue;
        }
        const int64_t* rows_d = lanes + 2 * nl;
        if (try16 && !g->narrow16_failed[mi]) {
            GIR_TRY(sssp_group<uint16_t>(g, wk, ws, nl, lanes, srcs_d, n_entries, rows_d, dist_d, D, &ovf));
            if (!ovf) continue;
            g->narrow16_failed[mi] = true;
            if (g->trace_on) std::fprintf(stderr, "[gir] sssp: 16-bit lane distances overflowed, group rerun\n");
        }
        if (fits32)
            GIR_TRY(sssp_group<uint32_t>(g, wk, ws, nl, lanes, srcs_d, n_entries, rows_d, dist_d, D, &ovf));
        else
            GIR_TRY(sssp_group<uint64_t>(g, wk, ws, nl, lanes, srcs_d, n_entries, rows_d, dist_d, D, &ovf));
    }
    unsigned long long* hc = wk.hc;
    GIR_CUDA(g, cudaMemcpyAsync(hc, wk.cnt, sizeof(unsigned long long) * S_N, cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaEventRecord(g->ev1, g->stream));
    GIR_CUDA(g, cudaEventSynchronize(g->ev1));
    st.reached = (int64_t)hc[S_REACHED];
    st.edges = (int64_t)hc[S_EDGES];
    float ms = 0;
    GIR_CUDA(g, cudaEventElapsedTime(&ms, g->ev0, g->ev1));
    st.kernel_ms = ms;
    return GIR_OK;
}

}  // namespace gir
