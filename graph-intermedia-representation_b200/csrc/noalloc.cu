// gir_dev_bfs_noalloc: breadth-first levels from one source over a caller's CSR, without any
// device or host allocation.
//
// Some callers cannot allocate device memory at call time: a host engine that hands all of a
// GPU's memory to its own arena, or a latency-critical thread for which a cudaMalloc / cudaFree
// (which can synchronize the whole device) is not acceptable. This entry point serves them: the
// caller passes the graph and the level array in device memory, and the only working memory is
// the file-scope array below -- two frontier queues for at most GIR_NOALLOC_MAX_V vertices plus
// a few counters, 16 MiB that every GPU which loads this library holds until the process exits.
//
// The array is shared by all calls: the counters are cleared by every call before use, and two
// calls that overlap on the GPU (other streams or other host threads) race on it.
#include <cuda_runtime.h>

#include <mutex>

#include "common.cuh"

namespace gir {

namespace {

constexpr int64_t kMaxV = GIR_NOALLOC_MAX_V;
constexpr int kBlock = 256;
constexpr int kCounters = 64;  // [0], [1]: lengths of the two queues (alternating by level)

static __device__ __align__(256) int32_t g_noalloc_scratch[2 * kMaxV + kCounters];

// Device address of the scratch array, set up once per device (cudaGetSymbolAddress with that
// device current; the host-side symbol is not a device address).
constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
int32_t* g_setup_ptr[kMaxDevices] = {};

int scratch_for_current_device(int32_t** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_thread_error(std::string("bfs_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
        return GIR_ERR_NODEVICE;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        set_thread_error("bfs_noalloc: device id beyond the supported range");
        return GIR_ERR_CAPACITY;
    }
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_setup_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            set_thread_error(std::string("bfs_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            return GIR_ERR_CUDA;
        }
        g_setup_ptr[dev] = static_cast<int32_t*>(p);
    }
    *out = g_setup_ptr[dev];
    return GIR_OK;
}

// The CSR is checked before it is used: beg[0] == 0, offsets never decreasing, beg[V] within the
// caller's n_adj entries of adj, ids in [0, V). A bad graph becomes an error status instead of
// out-of-bounds accesses: the id scan never reads past min(beg[V], n_adj). cnt[2] = 1 if bad.
__global__ void k_na_validate(const int64_t* beg, const int32_t* adj, int64_t n_adj, int64_t V, unsigned int* cnt) {
    const int64_t E = beg[V];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t == 0 && (beg[0] != 0 || E < 0 || E > n_adj)) atomicExch(&cnt[2], 1u);
    for (int64_t v = t; v < V; v += stride)
        if (beg[v] > beg[v + 1]) atomicExch(&cnt[2], 1u);
    const int64_t scan = E < 0 ? 0 : (E < n_adj ? E : n_adj);
    for (int64_t k = t; k < scan; k += stride)
        if (adj[k] < 0 || (int64_t)adj[k] >= V) atomicExch(&cnt[2], 1u);
}

// All levels -1 except the source's 0; the source is the first frontier.
__global__ void k_na_init(int32_t* level, int64_t V, int32_t src, int32_t* q0, unsigned int* cnt) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < V; v += (int64_t)gridDim.x * blockDim.x)
        level[v] = v == src ? 0 : -1;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const bool ok = src >= 0 && (int64_t)src < V;
        if (ok) q0[0] = src;
        cnt[0] = ok ? 1u : 0u;
        cnt[1] = 0u;
    }
}

// One level: a warp per frontier vertex, lanes striding its row; a vertex is claimed by the CAS
// that moves its level from -1 to L + 1 and queued once.
__global__ void k_na_level(const int64_t* beg, const int32_t* adj, const int32_t* q, const unsigned int* qn,
                           int32_t* level, int32_t L, int32_t* nq, unsigned int* nn) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t n = *qn;
    for (int64_t i = warp; i < n; i += nwarps) {
        const int32_t u = q[i];
        for (int64_t k = beg[u] + lane; k < beg[u + 1]; k += 32) {
            const int32_t w = adj[k];
            if (level[w] == -1 && atomicCAS(&level[w], -1, L + 1) == -1) nq[atomicAdd(nn, 1u)] = w;
        }
    }
}

}  // namespace
}  // namespace gir

using namespace gir;

// Device memory the current device can use directly: its own allocations, or managed memory.
static bool on_current_device(const void* p, int dev) {
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (a.type == cudaMemoryTypeManaged) return true;
    return a.type == cudaMemoryTypeDevice && a.device == dev;
}

extern "C" int gir_dev_bfs_noalloc(const int64_t* beg, const int32_t* adj, int64_t n_adj, int64_t V,
                                   int32_t source, int32_t* level_out, void* stream) {
    if (V < 0 || V > GIR_NOALLOC_MAX_V) {
        set_thread_error("bfs_noalloc: V exceeds GIR_NOALLOC_MAX_V (" + std::to_string((long long)GIR_NOALLOC_MAX_V) +
                         " vertices), the size of its static working memory");
        return GIR_ERR_CAPACITY;
    }
    if (n_adj < 0) {
        set_thread_error("bfs_noalloc: negative n_adj");
        return GIR_ERR_INVALID;
    }
    if (V == 0) return GIR_OK;
    int cur_dev = 0;
    if (cudaGetDevice(&cur_dev) != cudaSuccess) {
        cudaGetLastError();
        set_thread_error("bfs_noalloc: no current CUDA device");
        return GIR_ERR_NODEVICE;
    }
    if (!on_current_device(beg, cur_dev) || !on_current_device(level_out, cur_dev) ||
        (n_adj > 0 && !on_current_device(adj, cur_dev))) {
        set_thread_error("bfs_noalloc: beg, adj and level_out must be device memory of the current device");
        return GIR_ERR_INVALID;
    }
    int32_t* scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc != GIR_OK) return rc;
    int32_t* qa = scratch;
    int32_t* qb = scratch + kMaxV;
    unsigned int* cnt = reinterpret_cast<unsigned int*>(scratch + 2 * kMaxV);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int dev_sms = 148;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, cur_dev);
    const int grid = dev_sms * 4;
    auto check = [&](cudaError_t e, const char* what) {
        if (e == cudaSuccess) return GIR_OK;
        cudaGetLastError();
        set_thread_error(std::string("bfs_noalloc: ") + what + ": " + cudaGetErrorString(e));
        return GIR_ERR_CUDA;
    };
    if ((rc = check(cudaMemsetAsync(cnt, 0, sizeof(unsigned int) * kCounters, s), "counter reset"))) return rc;
    k_na_validate<<<grid, kBlock, 0, s>>>(beg, adj, n_adj, V, cnt);
    if ((rc = check(cudaGetLastError(), "k_na_validate"))) return rc;
    unsigned int bad = 0;
    if ((rc = check(cudaMemcpyAsync(&bad, cnt + 2, sizeof(bad), cudaMemcpyDeviceToHost, s), "counter read")) ||
        (rc = check(cudaStreamSynchronize(s), "synchronize")))
        return rc;
    if (bad) {
        set_thread_error("bfs_noalloc: malformed CSR (offsets not monotone from 0, beg[V] beyond n_adj, or ids outside [0,V))");
        return GIR_ERR_MALFORMED;
    }
    k_na_init<<<grid, kBlock, 0, s>>>(level_out, V, source, qa, cnt);
    if ((rc = check(cudaGetLastError(), "k_na_init"))) return rc;
    unsigned int n = 0;
    if ((rc = check(cudaMemcpyAsync(&n, cnt, sizeof(n), cudaMemcpyDeviceToHost, s), "counter read")) ||
        (rc = check(cudaStreamSynchronize(s), "synchronize")))
        return rc;
    for (int32_t L = 0; n > 0; ++L) {
        unsigned int* cur = cnt + (L & 1);
        unsigned int* nxt = cnt + ((L + 1) & 1);
        if ((rc = check(cudaMemsetAsync(nxt, 0, sizeof(unsigned int), s), "counter reset"))) return rc;
        k_na_level<<<grid, kBlock, 0, s>>>(beg, adj, (L & 1) ? qb : qa, cur, level_out, L, (L & 1) ? qa : qb, nxt);
        if ((rc = check(cudaGetLastError(), "k_na_level"))) return rc;
        if ((rc = check(cudaMemcpyAsync(&n, nxt, sizeof(n), cudaMemcpyDeviceToHost, s), "counter read")) ||
            (rc = check(cudaStreamSynchronize(s), "synchronize")))
            return rc;
    }
    return GIR_OK;
}
