// The edge store in HBM: forward, backward and symmetrized slack CSRs, their construction from
// sorted edge keys, and batched in-place row updates.
//
// Reference counterpart: the edge store of gir_constructor/gir.h:248-313 (immutable sorted base
// CSR + tombstone bitmaps + sorted per-vertex delta lists, with a symmetrized int64-offset
// view). Here one slack CSR per direction replaces base + tombstones + deltas: rows stay
// sorted and exact, so traversals need no per-edge tombstone test or delta-list walk.
#include "common.cuh"

namespace gir {

namespace {

constexpr int kBlock = 256;

__device__ __forceinline__ int64_t row_capacity(int64_t d) {
    // Free room per row for later inserts: an eighth of the row, at least 4 entries; the
    // capacity is rounded up to a multiple of 4 so every row starts 16-byte aligned.
    const int64_t c = d + ((d >> 3) > 4 ? (d >> 3) : 4);
    return (c + 3) & ~(int64_t)3;
}

// Row of compact position `i`, given the exclusive scan `cb` of row lengths (V+1 entries).
__device__ __forceinline__ int64_t row_of(const int64_t* cb, int64_t V, int64_t i) {
    int64_t lo = 0, hi = V - 1;  // largest r with cb[r] <= i
    while (lo < hi) {
        const int64_t m = (lo + hi + 1) >> 1;
        if (cb[m] <= i) lo = m; else hi = m - 1;
    }
    return lo;
}

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

// Stored weight of a newly inserted edge u -> x: the hash weight of GIR::edgeWeight when
// wlo > whi, else w(u,v) = lo + hash3(seed,u,v) mod span, the generator's rule (csrc/gen.cpp).
__device__ __forceinline__ uint32_t new_edge_weight(int32_t r, int32_t x, uint64_t wseed, uint32_t wlo, uint32_t whi) {
    if (wlo > whi) return hash_weight(r, x);
    uint64_t z = wseed ^ 0x5851f42d4c957f2dULL;
    auto mix = [](uint64_t s) {
        s += 0x9e3779b97f4a7c15ULL;
        s = (s ^ (s >> 30)) * 0xbf58476d1ce4e5b9ULL;
        s = (s ^ (s >> 27)) * 0x94d049bb133111ebULL;
        return s ^ (s >> 31);
    };
    const uint64_t h = mix(mix(z) ^ mix((uint64_t)(uint32_t)r * 0x2545f4914f6cdd1dULL + (uint64_t)(uint32_t)x));
    return wlo + (uint32_t)(h % ((uint64_t)whi - wlo + 1));
}

// Head and tail positions of every row's run in a sorted key array.
__global__ void k_row_runs(const uint64_t* keys, int64_t n, int64_t* first, int64_t* end) {
    GRID_STRIDE(i, n) {
        const int64_t r = (int64_t)(keys[i] >> 32);
        if (i == 0 || (int64_t)(keys[i - 1] >> 32) != r) first[r] = i;
        if (i == n - 1 || (int64_t)(keys[i + 1] >> 32) != r) end[r] = i + 1;
    }
}

__global__ void k_caps(int64_t V, const int64_t* first, const int64_t* end, int32_t* deg, int64_t* capv) {
    GRID_STRIDE(v, V) {
        const int64_t d = end[v] - first[v];
        deg[v] = (int32_t)d;
        capv[v] = row_capacity(d);
    }
}

__global__ void k_scatter_keys(const uint64_t* keys, const uint32_t* kw, int64_t n, const int64_t* first,
                               const int64_t* beg, int32_t* adj, uint32_t* w) {
    GRID_STRIDE(i, n) {
        const int64_t r = (int64_t)(keys[i] >> 32);
        const int64_t p = beg[r] + (i - first[r]);
        adj[p] = (int32_t)(keys[i] & 0xffffffffULL);
        if (w) w[p] = kw ? kw[i] : 0u;
    }
}

// Compact offsets: cb[v] = sum of deg[0..v).
__global__ void k_deg_to_i64(int64_t V, const int32_t* deg, int64_t* out) {
    GRID_STRIDE(v, V) out[v] = deg[v];
    if (blockIdx.x == 0 && threadIdx.x == 0) out[V] = 0;
}

__global__ void k_sym_keys(int64_t V, int64_t E, const int64_t* cb, CSRView c, uint64_t* keys, uint8_t* keep) {
    GRID_STRIDE(i, E) {
        const int64_t u = row_of(cb, V, i);
        const int32_t v = c.adj[c.beg[u] + (i - cb[u])];
        keys[2 * i] = ((uint64_t)u << 32) | (uint32_t)v;
        keys[2 * i + 1] = ((uint64_t)(uint32_t)v << 32) | (uint64_t)u;
        keep[2 * i] = keep[2 * i + 1] = (v != (int32_t)u);
    }
}

__global__ void k_distinct_flags(const uint64_t* keys, int64_t n, uint8_t* flag) {
    GRID_STRIDE(i, n) flag[i] = (i == 0 || keys[i] != keys[i - 1]);
}

__global__ void k_compact_copy(int64_t V, int64_t E, const int64_t* cb, CSRView c, int32_t* adj_out, int64_t cap) {
    GRID_STRIDE(i, E) {
        if (i >= cap) continue;
        const int64_t u = row_of(cb, V, i);
        adj_out[i] = c.adj[c.beg[u] + (i - cb[u])];
    }
}

__global__ void k_has_edges(CSRView c, int64_t V, const int32_t* u, const int32_t* v, int64_t n, uint8_t* out) {
    GRID_STRIDE(i, n) {
        const int32_t a = u[i], b = v[i];
        bool hit = false;
        if (a >= 0 && b >= 0 && a < V && b < V) {
            const int64_t lo = c.beg[a], hi = lo + c.deg[a];
            const int64_t p = lower_bound_dev(c.adj, lo, hi, b);
            hit = p < hi && c.adj[p] == b;
        }
        out[i] = hit;
    }
}

// ---- batched row updates -------------------------------------------------------------------
// Ops are sorted, distinct keys (row << 32 | col): `ins` are absent edges to add, `del` present
// edges to remove. For each touched row r: new length = deg - |del_r| + |ins_r|. When every
// touched row still fits its capacity the rows are rewritten in place; otherwise the whole CSR
// is re-laid-out with fresh slack.

// Per touched row (from the merged op list `rows`, sorted distinct): op ranges and new length.
__global__ void k_touched_rows(const uint64_t* ins, int64_t n_ins, const uint64_t* del, int64_t n_del,
                               const int32_t* rows, int64_t n_rows, CSRView c, int64_t* i_lo, int64_t* d_lo,
                               int32_t* newdeg, int32_t* overflow) {
    GRID_STRIDE(k, n_rows) {
        const uint64_t r = (uint64_t)(uint32_t)rows[k];
        const int64_t a = lower_bound_dev(ins, (int64_t)0, n_ins, r << 32);
        const int64_t b = lower_bound_dev(ins, a, n_ins, (r + 1) << 32);
        const int64_t x = lower_bound_dev(del, (int64_t)0, n_del, r << 32);
        const int64_t y = lower_bound_dev(del, x, n_del, (r + 1) << 32);
        i_lo[k] = a; i_lo[n_rows + k] = b;
        d_lo[k] = x; d_lo[n_rows + k] = y;
        const int64_t nd = (int64_t)c.deg[r] - (y - x) + (b - a);
        if (nd < 0) {  // more deletions than entries: the ops do not match this CSR
            atomicExch(overflow + 1, 1);
            newdeg[k] = 0;
            continue;
        }
        newdeg[k] = (int32_t)nd;
        if (c.beg[r] + nd > c.beg[r + 1]) atomicExch(overflow, 1);
    }
}

// Writes the new content of every touched row into `tmp` (at toff[k]): surviving old entries
// and inserted entries, merged in sorted order. Element-parallel: each element computes its
// output slot with two binary searches.
__global__ void k_merge_rows(const uint64_t* ins, const uint64_t* del, const int32_t* rows, int64_t n_rows,
                             const int64_t* i_lo, const int64_t* d_lo, const int64_t* eoff, int64_t n_elems,
                             const int64_t* toff, const int32_t* newdeg, CSRView c, int32_t* tmp, uint32_t* tmpw,
                             bool weights, uint64_t wseed, uint32_t wlo, uint32_t whi, int32_t* bad) {
    GRID_STRIDE(e, n_elems) {
        // row k of element e: eoff is the exclusive scan of (deg + |ins|) over touched rows
        int64_t lo = 0, hi = n_rows - 1;
        while (lo < hi) {
            const int64_t m = (lo + hi + 1) >> 1;
            if (eoff[m] <= e) lo = m; else hi = m - 1;
        }
        const int64_t k = lo, j = e - eoff[k];
        const int64_t r = rows[k];
        const int64_t ib = i_lo[k], ie = i_lo[n_rows + k], db = d_lo[k], de = d_lo[n_rows + k];
        const int64_t rb = c.beg[r], rd = c.deg[r];
        if (j < rd) {
            const int32_t x = c.adj[rb + j];
            const uint64_t key = ((uint64_t)r << 32) | (uint32_t)x;
            const int64_t pd = lower_bound_dev(del, db, de, key);
            if (pd < de && del[pd] == key) continue;  // deleted
            const int64_t pi = lower_bound_dev(ins, ib, ie, key);
            const int64_t slot = j - (pd - db) + (pi - ib);
            if (slot < 0 || slot >= newdeg[k]) { atomicExch(bad, 1); continue; }  // ops not consistent with the row
            tmp[toff[k] + slot] = x;
            if (weights) tmpw[toff[k] + slot] = c.w[rb + j];
        } else {
            const int64_t q = j - rd;  // insert index within the row
            const uint64_t key = ins[ib + q];
            const int32_t x = (int32_t)(key & 0xffffffffULL);
            const int64_t po = lower_bound_dev(c.adj, rb, rb + rd, x) - rb;
            const int64_t pd = lower_bound_dev(del, db, de, key);
            const int64_t slot = q + po - (pd - db);
            if (slot < 0 || slot >= newdeg[k]) { atomicExch(bad, 1); continue; }
            tmp[toff[k] + slot] = x;
            if (weights) tmpw[toff[k] + slot] = new_edge_weight((int32_t)r, x, wseed, wlo, whi);
        }
    }
}

// Copies touched rows back from tmp into their (unchanged) capacity slots.
__global__ void k_copy_back(const int32_t* rows, int64_t n_rows, const int32_t* newdeg, const int64_t* toff,
                            const int64_t* noff, int64_t n_new, const int32_t* tmp, const uint32_t* tmpw,
                            int64_t* beg, int32_t* deg, int32_t* adj, uint32_t* w) {
    GRID_STRIDE(e, n_new) {
        int64_t lo = 0, hi = n_rows - 1;
        while (lo < hi) {
            const int64_t m = (lo + hi + 1) >> 1;
            if (noff[m] <= e) lo = m; else hi = m - 1;
        }
        const int64_t k = lo, j = e - noff[k], r = rows[k];
        adj[beg[r] + j] = tmp[toff[k] + j];
        if (w) w[beg[r] + j] = tmpw[toff[k] + j];
    }
}

__global__ void k_set_deg(const int32_t* rows, int64_t n_rows, const int32_t* newdeg, int32_t* deg) {
    GRID_STRIDE(k, n_rows) deg[rows[k]] = newdeg[k];
}

__global__ void k_mark_rows(const uint64_t* a, int64_t na, const uint64_t* b, int64_t nb, uint8_t* flag) {
    GRID_STRIDE(i, na + nb) flag[(i < na ? a[i] : b[i - na]) >> 32] = 1;
}

__global__ void k_row_len_plus_ins(const int32_t* rows, int64_t n_rows, const int64_t* i_lo, CSRView c,
                                   int64_t* out) {
    GRID_STRIDE(k, n_rows) out[k] = (int64_t)c.deg[rows[k]] + (i_lo[n_rows + k] - i_lo[k]);
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n_rows] = 0;
}

__global__ void k_i32_to_i64(const int32_t* in, int64_t n, int64_t* out) {
    GRID_STRIDE(k, n) out[k] = in[k];
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = 0;
}

// Full re-layout: new capacities from new lengths, then every row copied (touched rows from tmp).
__global__ void k_new_caps(int64_t V, const int32_t* deg, int64_t* capv) {
    GRID_STRIDE(v, V) capv[v] = row_capacity(deg[v]);
    if (blockIdx.x == 0 && threadIdx.x == 0) capv[V] = 0;
}

__global__ void k_relayout_rows(int64_t V, const int64_t* old_beg, const int32_t* old_adj, const uint32_t* old_w,
                                const int32_t* deg, const int64_t* new_beg, int32_t* new_adj, uint32_t* new_w,
                                const int32_t* touched_slot, const int64_t* toff, const int32_t* tmp,
                                const uint32_t* tmpw) {
    // one warp per row
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t v = warp; v < V; v += nwarps) {
        const int32_t k = touched_slot[v];
        const int32_t* src = k >= 0 ? tmp + toff[k] : old_adj + old_beg[v];
        const uint32_t* srcw = k >= 0 ? tmpw + toff[k] : (old_w ? old_w + old_beg[v] : nullptr);
        const int64_t d = deg[v], nb = new_beg[v];
        for (int64_t j = lane; j < d; j += 32) {
            new_adj[nb + j] = src[j];
            if (new_w) new_w[nb + j] = srcw[j];
        }
    }
}

__global__ void k_fill_i32(int32_t* p, int64_t n, int32_t v) { GRID_STRIDE(i, n) p[i] = v; }

__global__ void k_mark_slots(const int32_t* rows, int64_t n_rows, int32_t* slot) {
    GRID_STRIDE(k, n_rows) slot[rows[k]] = (int32_t)k;
}

__global__ void k_bin_flags(int64_t V, const int32_t* deg, int32_t small, int32_t large, uint8_t* f0, uint8_t* f1,
                            uint8_t* f2, int32_t* ids) {
    GRID_STRIDE(v, V) {
        const int32_t d = deg[v];
        f0[v] = d < small;
        f1[v] = d >= small && d < large;
        f2[v] = d >= large;
        ids[v] = (int32_t)v;
    }
}

// ---- one edge, edited in place (the single-edge latency path) -------------------------------
// Block-cooperative shifts of one row's entries (and weights): all reads of a chunk happen before
// its writes, and chunks move away from the gap, so nothing is overwritten before it is read.
__device__ void row_insert_at(int32_t* adj, uint32_t* w, int64_t p, int64_t end, int32_t x, uint32_t wx) {
    for (int64_t hi = end; hi > p; hi -= blockDim.x) {
        const int64_t lo = hi - (int64_t)blockDim.x > p ? hi - (int64_t)blockDim.x : p;
        const int64_t i = lo + threadIdx.x;
        const bool act = i < hi;
        int32_t a = 0;
        uint32_t b = 0;
        if (act) { a = adj[i]; if (w) b = w[i]; }
        __syncthreads();
        if (act) { adj[i + 1] = a; if (w) w[i + 1] = b; }
        __syncthreads();
    }
    if (threadIdx.x == 0) { adj[p] = x; if (w) w[p] = wx; }
    __syncthreads();
}

__device__ void row_erase_at(int32_t* adj, uint32_t* w, int64_t p, int64_t end) {
    for (int64_t lo = p + 1; lo < end; lo += blockDim.x) {
        const int64_t i = lo + threadIdx.x;
        const bool act = i < end;
        int32_t a = 0;
        uint32_t b = 0;
        if (act) { a = adj[i]; if (w) b = w[i]; }
        __syncthreads();
        if (act) { adj[i - 1] = a; if (w) w[i - 1] = b; }
        __syncthreads();
    }
}

struct MutCSR {
    const int64_t* beg;
    int32_t* deg;
    int32_t* adj;
    uint32_t* w;
};

// One directed change u -> v on the three slack CSRs, in one CTA. out[0]: 0 no-op (the edge is
// already present / absent), 1 applied, 2 a row lacks room (nothing changed: the batch merge
// runs instead). out[1]: 1 when the undirected pair {u, v} appeared, 2 when it disappeared.
// out[2]: layer flags judged with the current labels, as the batch classification does (bit 0
// an edge inside an SCC deleted, bit 1 an inserted cross edge against the rank order, bit 2 a
// cross edge changed, bit 3 the blocks may change, bit 4 an undirected pair appeared between two
// vertices that already share a weakly connected component, so the WCC labels stand). keys:
// u << 32 | v, then the two orientations of the pair.
__global__ void __launch_bounds__(1024) k_single_edit(MutCSR fw, MutCSR bw, MutCSR sym, int32_t u, int32_t v, int insert,
                                                      int weights, uint64_t wseed, uint32_t wlo, uint32_t whi,
                                                      const int32_t* scc, const int32_t* rank, const int32_t* blk,
                                                      const int32_t* head, const int32_t* wcc, unsigned long long* out,
                                                      uint64_t* keys) {
    __shared__ int64_t s_pos[4];
    __shared__ int s_st, s_sym;
    if (threadIdx.x == 0) {
        const int64_t fb = fw.beg[u], fd = fw.deg[u];
        const int64_t pf = lower_bound_dev(fw.adj, fb, fb + fd, v);
        const bool has_uv = pf < fb + fd && fw.adj[pf] == v;
        const int64_t rb = fw.beg[v], rd = fw.deg[v];
        const int64_t pr = lower_bound_dev(fw.adj, rb, rb + rd, u);
        const bool has_vu = pr < rb + rd && fw.adj[pr] == u;
        const int64_t bb = bw.beg[v], bd = bw.deg[v];
        const int64_t pb = lower_bound_dev(bw.adj, bb, bb + bd, u);
        const int64_t su = sym.beg[u], sdu = sym.deg[u], sv = sym.beg[v], sdv = sym.deg[v];
        const int64_t psu = lower_bound_dev(sym.adj, su, su + sdu, v);
        const int64_t psv = lower_bound_dev(sym.adj, sv, sv + sdv, u);
        int st = 1, symc = 0;
        if ((insert != 0) == has_uv) {
            st = 0;
        } else if (insert) {
            symc = has_vu ? 0 : 1;
            const bool room = fb + fd + 1 <= fw.beg[u + 1] && bb + bd + 1 <= bw.beg[v + 1] &&
                              (!symc || (su + sdu + 1 <= sym.beg[u + 1] && sv + sdv + 1 <= sym.beg[v + 1]));
            if (!room) st = 2;
        } else {
            symc = has_vu ? 0 : 2;
        }
        unsigned long long fl = 0;
        if (st == 1 && scc) {
            const bool same = scc[u] == scc[v];
            if (!insert && same) fl |= 1;
            if (!same) fl |= 4;
            if (insert && !same && rank[u] >= rank[v]) fl |= 2;
            if (symc && same && blk) {
                if (symc == 2) fl |= 8;
                else {
                    const int32_t bu = blk[u], bv = blk[v];
                    if (!(bu == bv || head[bv] == u || head[bu] == v)) fl |= 8;
                }
            }
        }
        if (st == 1 && symc == 1 && wcc && wcc[u] == wcc[v]) fl |= 16;
        s_pos[0] = pf; s_pos[1] = pb; s_pos[2] = psu; s_pos[3] = psv;
        s_st = st;
        s_sym = symc;
        out[0] = (unsigned long long)st;
        out[1] = (unsigned long long)symc;
        out[2] = fl;
        keys[0] = ((uint64_t)(uint32_t)u << 32) | (uint32_t)v;
        keys[1] = keys[0];
        keys[2] = ((uint64_t)(uint32_t)v << 32) | (uint32_t)u;
    }
    __syncthreads();
    if (s_st != 1) return;
    const int64_t fend = fw.beg[u] + fw.deg[u], bend = bw.beg[v] + bw.deg[v];
    const int64_t suend = sym.beg[u] + sym.deg[u], svend = sym.beg[v] + sym.deg[v];
    if (insert) {
        row_insert_at(fw.adj, weights ? fw.w : nullptr, s_pos[0], fend, v,
                      weights ? new_edge_weight(u, v, wseed, wlo, whi) : 0u);
        row_insert_at(bw.adj, nullptr, s_pos[1], bend, u, 0u);
        if (s_sym == 1) {
            row_insert_at(sym.adj, nullptr, s_pos[2], suend, v, 0u);
            row_insert_at(sym.adj, nullptr, s_pos[3], svend, u, 0u);
        }
    } else {
        row_erase_at(fw.adj, weights ? fw.w : nullptr, s_pos[0], fend);
        row_erase_at(bw.adj, nullptr, s_pos[1], bend);
        if (s_sym == 2) {
            row_erase_at(sym.adj, nullptr, s_pos[2], suend);
            row_erase_at(sym.adj, nullptr, s_pos[3], svend);
        }
    }
    if (threadIdx.x == 0) {
        const int d = insert ? 1 : -1;
        fw.deg[u] += d;
        bw.deg[v] += d;
        if (s_sym) {
            sym.deg[u] += d;
            sym.deg[v] += d;
        }
    }
}

}  // namespace

// The single-edge latency path: u -> v inserted (insert != 0) or deleted in place (see
// k_single_edit); the result words and keys are device arrays (3 and 3 entries) the caller reads.
int store_single_edit(gir_dev* g, int32_t u, int32_t v, int insert, unsigned long long* out, uint64_t* keys) {
    auto mut = [](DevCSR& c) { return MutCSR{c.beg, c.deg, c.adj, c.w}; };
    const int32_t* scc = g->scc_built ? static_cast<const int32_t*>(g->scc.p) : nullptr;
    const int32_t* rank = g->scc_built ? static_cast<const int32_t*>(g->scc_rank.p) : nullptr;
    const int32_t* blk = g->bct_built ? static_cast<const int32_t*>(g->blk_label.p) : nullptr;
    const int32_t* head = g->bct_built ? static_cast<const int32_t*>(g->blk_head.p) : nullptr;
    const int32_t* wcc = g->wcc_built ? static_cast<const int32_t*>(g->wcc.p) : nullptr;
    k_single_edit<<<1, 1024, 0, g->stream>>>(mut(g->fw), mut(g->bw), mut(g->sym), u, v, insert,
                                             g->has_weights && g->fw.w ? 1 : 0, g->wrule_seed, g->wrule_lo, g->wrule_hi,
                                             scc, rank, blk, head, wcc, out, keys);
    GIR_LAUNCH(g, "k_single_edit");
    return GIR_OK;
}

int store_free(gir_dev* g, DevCSR& c) {
    dev_free(g, c.beg);
    dev_free(g, c.deg);
    dev_free(g, c.adj);
    dev_free(g, c.w);
    c = DevCSR{};
    return GIR_OK;
}

int store_build_csr_from_keys(gir_dev* g, DevCSR& c, const uint64_t* keys, int64_t n, const uint32_t* kw) {
    // keys: sorted, distinct (row << 32 | col). kw (nullable): weight per key.
    const int64_t V = g->V;
    store_free(g, c);
    int64_t *first = nullptr, *endp = nullptr, *capv = nullptr;
    GIR_TRY(ensure_n(g, g->scratch[10], V + 1, &first));
    GIR_TRY(ensure_n(g, g->scratch[11], V + 1, &endp));
    GIR_TRY(ensure_n(g, g->scratch[12], V + 1, &capv));
    GIR_CUDA(g, cudaMemsetAsync(first, 0, sizeof(int64_t) * (V + 1), g->stream));
    GIR_CUDA(g, cudaMemsetAsync(endp, 0, sizeof(int64_t) * (V + 1), g->stream));
    GIR_TRY(dev_alloc_n(g, &c.beg, V + 1));
    GIR_TRY(dev_alloc_n(g, &c.deg, V > 0 ? V : 1));
    if (n > 0) {
        k_row_runs<<<grid_for(g, n, kBlock), kBlock, 0, g->stream>>>(keys, n, first, endp);
        GIR_LAUNCH(g, "k_row_runs");
    }
    k_caps<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, first, endp, c.deg, capv);
    GIR_LAUNCH(g, "k_caps");
    GIR_CUDA(g, cudaMemsetAsync(capv + V, 0, sizeof(int64_t), g->stream));
    GIR_TRY(exclusive_scan_i64(g, capv, c.beg, V + 1));
    int64_t total = 0;
    GIR_CUDA(g, cudaMemcpyAsync(&total, c.beg + V, sizeof(int64_t), cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    GIR_TRY(dev_alloc_n(g, &c.adj, total > 0 ? total : 4));
    if (kw) GIR_TRY(dev_alloc_n(g, &c.w, total > 0 ? total : 4));
    c.cap = total;
    c.E = n;
    if (n > 0) {
        k_scatter_keys<<<grid_for(g, n, kBlock), kBlock, 0, g->stream>>>(keys, kw, n, first, c.beg, c.adj, c.w);
        GIR_LAUNCH(g, "k_scatter_keys");
    }
    return GIR_OK;
}

static int compact_offsets(gir_dev* g, const DevCSR& c, int64_t* cb) {
    k_deg_to_i64<<<grid_for(g, g->V, kBlock), kBlock, 0, g->stream>>>(g->V, c.deg, cb);
    GIR_LAUNCH(g, "k_deg_to_i64");
    return exclusive_scan_i64(g, cb, cb, g->V + 1);
}

int store_build_sym(gir_dev* g) {
    // Symmetrized view (buildWCC, gir.cpp:599-625): {u,v} for every u -> v with u != v, both
    // directions, sorted and distinct.
    const int64_t V = g->V, E = g->fw.E;
    int64_t* cb = nullptr;
    uint64_t *keys = nullptr, *tmp = nullptr, *out = nullptr;
    uint8_t* keep = nullptr;
    GIR_TRY(ensure_n(g, g->scratch[0], V + 1, &cb));
    GIR_TRY(ensure_n(g, g->scratch[1], 2 * E + 1, &keys));
    GIR_TRY(ensure_n(g, g->scratch[2], 2 * E + 1, &tmp));
    GIR_TRY(ensure_n(g, g->scratch[3], 2 * E + 1, &keep));
    GIR_TRY(compact_offsets(g, g->fw, cb));
    if (E > 0) {
        k_sym_keys<<<grid_for(g, E, kBlock), kBlock, 0, g->stream>>>(V, E, cb, view(g->fw), keys, keep);
        GIR_LAUNCH(g, "k_sym_keys");
    }
    int64_t n = 0;
    GIR_TRY(select_flagged_u64(g, keys, keep, tmp, 2 * E, &n));
    GIR_TRY(sort_keys_u64(g, tmp, keys, n, 64));
    if (n > 0) {
        k_distinct_flags<<<grid_for(g, n, kBlock), kBlock, 0, g->stream>>>(tmp, n, keep);
        GIR_LAUNCH(g, "k_distinct_flags");
    }
    out = keys;
    int64_t m = 0;
    GIR_TRY(select_flagged_u64(g, tmp, keep, out, n, &m));
    return store_build_csr_from_keys(g, g->sym, out, m, nullptr);
}

int store_compact_csr(gir_dev* g, const DevCSR& c, int64_t* beg_out, int32_t* adj_out, int64_t cap) {
    // beg_out / adj_out: device pointers (V+1 / cap entries)
    GIR_TRY(compact_offsets(g, c, beg_out));
    if (c.E > 0 && adj_out && cap > 0) {
        k_compact_copy<<<grid_for(g, c.E, kBlock), kBlock, 0, g->stream>>>(g->V, c.E, beg_out, view(c), adj_out, cap);
        GIR_LAUNCH(g, "k_compact_copy");
    }
    return GIR_OK;
}

int store_has_edges(gir_dev* g, const DevCSR& c, const int32_t* u, const int32_t* v, int64_t n, uint8_t* out) {
    if (n <= 0) return GIR_OK;
    k_has_edges<<<grid_for(g, n, kBlock), kBlock, 0, g->stream>>>(view(c), g->V, u, v, n, out);
    GIR_LAUNCH(g, "k_has_edges");
    return GIR_OK;
}

int store_apply_ops(gir_dev* g, DevCSR& c, const uint64_t* ins, int64_t n_ins, const uint64_t* del, int64_t n_del,
                    bool weights) {
    if (n_ins + n_del == 0) return GIR_OK;
    const int64_t V = g->V;
    const int64_t n_ops = n_ins + n_del;
    int32_t *rows = nullptr, *newdeg = nullptr, *tmp = nullptr;
    uint8_t* flag = nullptr;
    int64_t *i_lo = nullptr, *d_lo = nullptr, *eoff = nullptr, *noff = nullptr;
    uint32_t* tmpw = nullptr;
    GIR_TRY(ensure_n(g, g->scratch[4], V + 1, &flag));
    GIR_TRY(ensure_n(g, g->scratch[5], V + 1, &rows));
    // rows touched by any op, ascending and distinct
    GIR_CUDA(g, cudaMemsetAsync(flag, 0, V, g->stream));
    k_mark_rows<<<grid_for(g, n_ops, kBlock), kBlock, 0, g->stream>>>(ins, n_ins, del, n_del, flag);
    GIR_LAUNCH(g, "k_mark_rows");
    int64_t n_rows = 0;
    GIR_TRY(select_flagged_iota(g, flag, rows, V, &n_rows));

    int32_t* overflow = nullptr;
    GIR_TRY(ensure_n(g, g->scratch[9], 2 * n_rows + 2, &i_lo));
    GIR_TRY(ensure_n(g, g->scratch[13], 2 * n_rows + 2, &d_lo));
    GIR_TRY(ensure_n(g, g->scratch[14], n_rows + 1, &newdeg));
    GIR_TRY(ensure_n(g, g->scratch[10], n_rows + 1, &eoff));
    GIR_TRY(ensure_n(g, g->scratch[11], n_rows + 1, &noff));
    GIR_TRY(ensure_n(g, g->scratch[12], 4, &overflow));
    GIR_CUDA(g, cudaMemsetAsync(overflow, 0, 2 * sizeof(int32_t), g->stream));
    k_touched_rows<<<grid_for(g, n_rows, kBlock), kBlock, 0, g->stream>>>(ins, n_ins, del, n_del, rows, n_rows, view(c),
                                                                           i_lo, d_lo, newdeg, overflow);
    GIR_LAUNCH(g, "k_touched_rows");
    // element space: old entries + inserts of every touched row
    k_row_len_plus_ins<<<grid_for(g, n_rows, kBlock), kBlock, 0, g->stream>>>(rows, n_rows, i_lo, view(c), eoff);
    GIR_LAUNCH(g, "k_row_len_plus_ins");
    GIR_TRY(exclusive_scan_i64(g, eoff, eoff, n_rows + 1));
    k_i32_to_i64<<<grid_for(g, n_rows, kBlock), kBlock, 0, g->stream>>>(newdeg, n_rows, noff);
    GIR_LAUNCH(g, "k_i32_to_i64");
    GIR_TRY(exclusive_scan_i64(g, noff, noff, n_rows + 1));
    int64_t h[2] = {0, 0};
    int32_t ovf = 0;
    GIR_CUDA(g, cudaMemcpyAsync(&h[0], eoff + n_rows, sizeof(int64_t), cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaMemcpyAsync(&h[1], noff + n_rows, sizeof(int64_t), cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaMemcpyAsync(&ovf, overflow, sizeof(int32_t), cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    const int64_t n_elems = h[0], n_new = h[1];
    const bool wts = weights && c.w;
    // tmp holds each touched row's new content at noff[k] (the merged rows are written there)
    GIR_TRY(ensure_n(g, g->stage_out, n_new + 4, &tmp));
    if (wts) GIR_TRY(ensure_n(g, g->scratch[3], n_new + 4, &tmpw));
    if (n_elems > 0) {
        k_merge_rows<<<grid_for(g, n_elems, kBlock), kBlock, 0, g->stream>>>(
            ins, del, rows, n_rows, i_lo, d_lo, eoff, n_elems, noff, newdeg, view(c), tmp, tmpw, wts, g->wrule_seed,
            g->wrule_lo, g->wrule_hi, overflow + 1);
        GIR_LAUNCH(g, "k_merge_rows");
    }
    int32_t inconsistent = 0;
    GIR_CUDA(g, cudaMemcpyAsync(&inconsistent, overflow + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    if (inconsistent)
        return fail(g, GIR_ERR_MALFORMED, "edge update: the backward CSR is not the transpose of the forward CSR");
    if (!ovf) {
        if (n_new > 0) {
            k_copy_back<<<grid_for(g, n_new, kBlock), kBlock, 0, g->stream>>>(rows, n_rows, newdeg, noff, noff, n_new,
                                                                              tmp, tmpw, c.beg, c.deg, c.adj,
                                                                              wts ? c.w : nullptr);
            GIR_LAUNCH(g, "k_copy_back");
        }
        k_set_deg<<<grid_for(g, n_rows, kBlock), kBlock, 0, g->stream>>>(rows, n_rows, newdeg, c.deg);
        GIR_LAUNCH(g, "k_set_deg");
    } else {
        // Some row outgrew its slack: new layout for the whole CSR.
        trace_mark(g, "store: merge before relayout");
        int32_t* slot = nullptr;
        int64_t* capv = nullptr;
        GIR_TRY(ensure_n(g, g->scratch[0], V + 1, &slot));
        GIR_TRY(ensure_n(g, g->scratch[1], V + 1, &capv));
        k_set_deg<<<grid_for(g, n_rows, kBlock), kBlock, 0, g->stream>>>(rows, n_rows, newdeg, c.deg);
        GIR_LAUNCH(g, "k_set_deg");
        k_fill_i32<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(slot, V, -1);
        GIR_LAUNCH(g, "k_fill_i32");
        k_mark_slots<<<grid_for(g, n_rows, kBlock), kBlock, 0, g->stream>>>(rows, n_rows, slot);
        GIR_LAUNCH(g, "k_mark_slots");
        k_new_caps<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, c.deg, capv);
        GIR_LAUNCH(g, "k_new_caps");
        int64_t* nbeg = nullptr;
        GIR_TRY(dev_alloc_n(g, &nbeg, V + 1));
        GIR_TRY(exclusive_scan_i64(g, capv, nbeg, V + 1));
        int64_t total = 0;
        GIR_CUDA(g, cudaMemcpyAsync(&total, nbeg + V, sizeof(int64_t), cudaMemcpyDeviceToHost, g->stream));
        GIR_CUDA(g, cudaStreamSynchronize(g->stream));
        int32_t* nadj = nullptr;
        uint32_t* nw = nullptr;
        GIR_TRY(dev_alloc_n(g, &nadj, total > 0 ? total : 4));
        if (c.w) GIR_TRY(dev_alloc_n(g, &nw, total > 0 ? total : 4));
        k_relayout_rows<<<grid_for(g, V * 32, kBlock), kBlock, 0, g->stream>>>(V, c.beg, c.adj, c.w, c.deg, nbeg, nadj,
                                                                                 nw, slot, noff, tmp, tmpw);
        GIR_LAUNCH(g, "k_relayout_rows");
        dev_free(g, c.beg);
        dev_free(g, c.adj);
        dev_free(g, c.w);
        c.beg = nbeg; c.adj = nadj; c.w = nw; c.cap = total;
        trace_mark(g, "store: relayout");
    }
    c.E += n_ins - n_del;
    return GIR_OK;
}

int store_build_bins(gir_dev* g) {
    // Vertices by in-degree class for the bottom-up kernels: [0, small) thread per vertex,
    // [small, large) warp per vertex, [large, inf) CTA per vertex.
    const int64_t V = g->V;
    int32_t *bins = nullptr, *ids = nullptr;
    uint8_t *f0 = nullptr, *f1 = nullptr, *f2 = nullptr;
    GIR_TRY(ensure_n(g, g->bins, V + 1, &bins));
    GIR_TRY(ensure_n(g, g->scratch[4], V + 1, &ids));
    GIR_TRY(ensure_n(g, g->scratch[5], V + 1, &f0));
    GIR_TRY(ensure_n(g, g->scratch[6], V + 1, &f1));
    GIR_TRY(ensure_n(g, g->scratch[7], V + 1, &f2));
    k_bin_flags<<<grid_for(g, V, kBlock), kBlock, 0, g->stream>>>(V, g->bw.deg, (int32_t)g->params[GIR_PARAM_SMALL_DEG],
                                                                   (int32_t)g->params[GIR_PARAM_LARGE_DEG], f0, f1, f2, ids);
    GIR_LAUNCH(g, "k_bin_flags");
    int64_t n0 = 0, n1 = 0, n2 = 0;
    GIR_TRY(select_flagged_i32(g, ids, f0, bins, V, &n0));
    GIR_TRY(select_flagged_i32(g, ids, f1, bins + n0, V, &n1));
    GIR_TRY(select_flagged_i32(g, ids, f2, bins + n0 + n1, V, &n2));
    g->bin_n[0] = n0; g->bin_n[1] = n1; g->bin_n[2] = n2;
    g->bins_valid = true;
    return GIR_OK;
}

}  // namespace gir
