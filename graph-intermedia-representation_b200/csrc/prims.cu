// Handle utilities (errors, buffers, staging) and the sort / scan / compaction primitives of
// the build and update pipelines. The primitives are CUB's device-wide algorithms (header-only
// templates from the CUDA toolkit, instantiated here for sm_100a); the traversal kernels of
// the hot path are this library's own.
#include <cub/cub.cuh>

#include "common.cuh"

namespace gir {

int fail(gir_dev* g, int code, const std::string& msg) {
    if (g) g->err = msg;
    return code;
}

int cuda_check(gir_dev* g, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return GIR_OK;
    const int code = (e == cudaErrorMemoryAllocation) ? GIR_ERR_OOM : GIR_ERR_CUDA;
    cudaGetLastError();  // clear a non-sticky error
    return fail(g, code, std::string(what) + ": " + cudaGetErrorString(e));
}

int dev_alloc(gir_dev* g, void** p, size_t bytes) {
    *p = nullptr;
    const size_t want = ((bytes < 256 ? 256 : bytes) + 255) & ~(size_t)255;
    const double t0 = g->trace_on ? now_ms() : 0.0;
    cudaError_t e = cudaMallocFromPoolAsync(p, want, g->pool, g->stream);
    if (e == cudaErrorMemoryAllocation) {
        if (g->trace_on) std::fprintf(stderr, "[gir] pool exhausted at %zu bytes: trimming\n", want);
        // The pool keeps freed blocks for reuse; when none fits, give its unused memory back to
        // the device and try once more (large graphs use most of HBM in turns).
        cudaGetLastError();
        cudaStreamSynchronize(g->stream);
        cudaMemPoolTrimTo(g->pool, 0);
        e = cudaMallocFromPoolAsync(p, want, g->pool, g->stream);
    }
    if (g->trace_on && now_ms() - t0 > 1.0)
        std::fprintf(stderr, "[gir] pool allocation of %zu bytes took %.3f ms\n", want, now_ms() - t0);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(g, GIR_ERR_OOM, "device allocation of " + std::to_string(want) + " bytes failed: " +
                                        cudaGetErrorString(e));
    }
    return GIR_OK;
}

void dev_free(gir_dev* g, void* p) {
    if (p) cudaFreeAsync(p, g->stream);
}

int ensure(gir_dev* g, DevBuf& b, size_t bytes) {
    if (b.bytes >= bytes && b.p) return GIR_OK;
    const double t0 = g->trace_on ? now_ms() : 0.0;
    // a buffer that has to grow again gets a quarter more than asked, so sizes that creep up
    // (capacities after relayouts, batch sizes) do not reallocate every call
    size_t want = b.p ? bytes + bytes / 4 : bytes;
    want = ((want < 256 ? 256 : want) + 255) & ~(size_t)255;
    release(g, b);
    GIR_TRY(dev_alloc(g, &b.p, want));
    if (g->trace_on) std::fprintf(stderr, "[gir] alloc %zu bytes: %.3f ms\n", want, now_ms() - t0);
    b.bytes = want;
    return GIR_OK;
}

void release_scratch(gir_dev* g, size_t min_bytes) {
    if (!g->scratch_tight) return;  // memory is not tight: keep the buffers for the next call
    auto drop = [&](DevBuf& b) {
        if (b.p && b.bytes >= min_bytes) release(g, b);
    };
    for (auto& b : g->scratch) drop(b);
    for (auto& b : g->work) drop(b);
    for (auto& b : g->qitems) drop(b);
    drop(g->cub_tmp);
    drop(g->stage_in);
    drop(g->stage_out);
    drop(g->lane_dist);
}

void release(gir_dev* g, DevBuf& b) {
    dev_free(g, b.p);
    b.p = nullptr;
    b.bytes = 0;
}

int pinned(gir_dev* g, size_t bytes, void** out) {
    if (g->pinned_bytes < bytes) {
        if (g->pinned) cudaFreeHost(g->pinned);
        g->pinned = nullptr;
        g->pinned_bytes = 0;
        GIR_CUDA(g, cudaMallocHost(&g->pinned, bytes));
        g->pinned_bytes = bytes;
    }
    *out = g->pinned;
    return GIR_OK;
}

bool is_device_ptr(const void* p) {
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int stage_input(gir_dev* g, DevBuf& stage, const void* p, size_t bytes, const void** dev) {
    if (bytes == 0) { *dev = p; return GIR_OK; }
    if (is_device_ptr(p)) { *dev = p; return GIR_OK; }
    GIR_TRY(ensure(g, stage, bytes));
    GIR_CUDA(g, cudaMemcpyAsync(stage.p, p, bytes, cudaMemcpyHostToDevice, g->stream));
    *dev = stage.p;
    return GIR_OK;
}

int sort_keys_u64(gir_dev* g, uint64_t* keys, uint64_t* tmp, int64_t n, int end_bit) {
    if (n <= 1) return GIR_OK;
    cub::DoubleBuffer<uint64_t> kb(keys, tmp);
    size_t bytes = 0;
    GIR_CUDA(g, cub::DeviceRadixSort::SortKeys(nullptr, bytes, kb, n, 0, end_bit, g->stream));
    GIR_TRY(ensure(g, g->cub_tmp, bytes));
    GIR_CUDA(g, cub::DeviceRadixSort::SortKeys(g->cub_tmp.p, bytes, kb, n, 0, end_bit, g->stream));
    if (kb.Current() != keys)
        GIR_CUDA(g, cudaMemcpyAsync(keys, kb.Current(), sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, g->stream));
    return GIR_OK;
}

int sort_pairs_u64(gir_dev* g, uint64_t* keys, uint64_t* ktmp, uint32_t* vals, uint32_t* vtmp, int64_t n, int end_bit) {
    if (n <= 1) return GIR_OK;
    cub::DoubleBuffer<uint64_t> kb(keys, ktmp);
    cub::DoubleBuffer<uint32_t> vb(vals, vtmp);
    size_t bytes = 0;
    GIR_CUDA(g, cub::DeviceRadixSort::SortPairs(nullptr, bytes, kb, vb, n, 0, end_bit, g->stream));
    GIR_TRY(ensure(g, g->cub_tmp, bytes));
    GIR_CUDA(g, cub::DeviceRadixSort::SortPairs(g->cub_tmp.p, bytes, kb, vb, n, 0, end_bit, g->stream));
    if (kb.Current() != keys)
        GIR_CUDA(g, cudaMemcpyAsync(keys, kb.Current(), sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, g->stream));
    if (vb.Current() != vals)
        GIR_CUDA(g, cudaMemcpyAsync(vals, vb.Current(), sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, g->stream));
    return GIR_OK;
}

int sort_pairs_u64_i64(gir_dev* g, uint64_t* keys, uint64_t* ktmp, int64_t* vals, int64_t* vtmp, int64_t n, int end_bit) {
    if (n <= 1) return GIR_OK;
    cub::DoubleBuffer<uint64_t> kb(keys, ktmp);
    cub::DoubleBuffer<int64_t> vb(vals, vtmp);
    size_t bytes = 0;
    GIR_CUDA(g, cub::DeviceRadixSort::SortPairs(nullptr, bytes, kb, vb, n, 0, end_bit, g->stream));
    GIR_TRY(ensure(g, g->cub_tmp, bytes));
    GIR_CUDA(g, cub::DeviceRadixSort::SortPairs(g->cub_tmp.p, bytes, kb, vb, n, 0, end_bit, g->stream));
    if (kb.Current() != keys)
        GIR_CUDA(g, cudaMemcpyAsync(keys, kb.Current(), sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, g->stream));
    if (vb.Current() != vals)
        GIR_CUDA(g, cudaMemcpyAsync(vals, vb.Current(), sizeof(int64_t) * n, cudaMemcpyDeviceToDevice, g->stream));
    return GIR_OK;
}

int exclusive_scan_i64(gir_dev* g, const int64_t* in, int64_t* out, int64_t n) {
    if (n <= 0) return GIR_OK;
    size_t bytes = 0;
    GIR_CUDA(g, cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, g->stream));
    GIR_TRY(ensure(g, g->cub_tmp, bytes));
    GIR_CUDA(g, cub::DeviceScan::ExclusiveSum(g->cub_tmp.p, bytes, in, out, n, g->stream));
    return GIR_OK;
}

int sum_i64(gir_dev* g, const int64_t* in, int64_t n, int64_t* host_out) {
    int64_t* d_out = nullptr;
    GIR_TRY(ensure_n(g, g->scratch[15], 1, &d_out));
    if (n <= 0) { *host_out = 0; return GIR_OK; }
    size_t bytes = 0;
    GIR_CUDA(g, cub::DeviceReduce::Sum(nullptr, bytes, in, d_out, n, g->stream));
    GIR_TRY(ensure(g, g->cub_tmp, bytes));
    GIR_CUDA(g, cub::DeviceReduce::Sum(g->cub_tmp.p, bytes, in, d_out, n, g->stream));
    void* h = nullptr;
    GIR_TRY(pinned(g, 64, &h));
    GIR_CUDA(g, cudaMemcpyAsync(h, d_out, sizeof(int64_t), cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    *host_out = *static_cast<int64_t*>(h);
    return GIR_OK;
}

template <class It, class T>
static int select_flagged(gir_dev* g, It in, const uint8_t* flags, T* out, int64_t n, int64_t* host_n) {
    int64_t* d_n = nullptr;
    GIR_TRY(ensure_n(g, g->scratch[15], 1, &d_n));
    if (n <= 0) { *host_n = 0; return GIR_OK; }
    size_t bytes = 0;
    GIR_CUDA(g, cub::DeviceSelect::Flagged(nullptr, bytes, in, flags, out, d_n, n, g->stream));
    GIR_TRY(ensure(g, g->cub_tmp, bytes));
    GIR_CUDA(g, cub::DeviceSelect::Flagged(g->cub_tmp.p, bytes, in, flags, out, d_n, n, g->stream));
    void* h = nullptr;
    GIR_TRY(pinned(g, 64, &h));
    GIR_CUDA(g, cudaMemcpyAsync(h, d_n, sizeof(int64_t), cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    *host_n = *static_cast<int64_t*>(h);
    return GIR_OK;
}

int select_flagged_u64(gir_dev* g, const uint64_t* in, const uint8_t* flags, uint64_t* out, int64_t n, int64_t* host_n) {
    return select_flagged(g, in, flags, out, n, host_n);
}
int select_flagged_i32(gir_dev* g, const int32_t* in, const uint8_t* flags, int32_t* out, int64_t n, int64_t* host_n) {
    return select_flagged(g, in, flags, out, n, host_n);
}
int select_flagged_iota(gir_dev* g, const uint8_t* flags, int32_t* out, int64_t n, int64_t* host_n) {
    return select_flagged(g, cub::CountingInputIterator<int32_t>(0), flags, out, n, host_n);
}

namespace {
__global__ void k_heavy_flags(const int32_t* deg, int64_t V, int32_t max_deg, uint8_t* flag) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < V; v += (int64_t)gridDim.x * blockDim.x)
        flag[v] = deg[v] > max_deg;
}
__global__ void k_heavy_lengths(const int32_t* deg, const int32_t* rows, int64_t n, int64_t* pref) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        pref[i] = deg[rows[i]];
    if (blockIdx.x == 0 && threadIdx.x == 0) pref[n] = 0;
}
}  // namespace

int heavy_rows(gir_dev* g, const int32_t* deg, int64_t V, int32_t max_deg, uint8_t* flag, int32_t* rows, int64_t* pref,
               int64_t* n) {
    *n = 0;
    if (V <= 0) return GIR_OK;
    k_heavy_flags<<<grid_for(g, V, 256), 256, 0, g->stream>>>(deg, V, max_deg, flag);
    GIR_LAUNCH(g, "k_heavy_flags");
    GIR_TRY(select_flagged_iota(g, flag, rows, V, n));
    k_heavy_lengths<<<grid_for(g, *n + 1, 256), 256, 0, g->stream>>>(deg, rows, *n, pref);
    GIR_LAUNCH(g, "k_heavy_lengths");
    return exclusive_scan_i64(g, pref, pref, *n + 1);
}

}  // namespace gir
