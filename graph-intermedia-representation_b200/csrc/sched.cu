// The learned schedule: a 2-layer MLP (GIR_SCHED_IN features -> GIR_SCHED_HID tanh units ->
// GIR_SCHED_OUT logits), fp32, with this library's own forward, backward and SGD kernels.
//
// It only picks schedule choices, never results: logits 0..1 choose the BFS direction of the
// next level (top-down / bottom-up), logits 2..7 the Delta-stepping bucket width (one of
// kDeltaChoices), logits 8..11 the forward-backward pivot rule of the SCC build (max out x in
// degree, max out + in, max in-degree, or no forward-backward pass). The fixed heuristics (alpha =
// 15, beta = 18, gir_query.cpp:161-168; Delta = 16, gir.h:215; the max out x in pivot of iSpan,
// gir_constructor/includes/scc_cpu/scc_common.h:98-146) are the fallback when no network is
// loaded, and for the direction and the pivot also when the network's margin is small.
//
// Feature vectors (built by the callers in bfs.cu / sssp.cu, all scaled to O(1)):
//   BFS level:  [log2(nf / V) / 8, log2(mf / mu) / 8, log2(mu / E) / 8, log2(mf / E) / 8,
//                current direction, log2(E / V + 1) / 8, lanes / 64, 0]
//               with nf / mf the frontier's vertices / out-edges and mu the out-edges not yet
//               explored (per lane). The fixed switch is a threshold on log2(mf / mu) (top-down
//               -> bottom-up) and on log2(nf / V) (back), so the log scale makes it, and any
//               better pair of thresholds, a simple function of the inputs.
//   SSSP query: [log2(E / V + 1) / 8, log2(mean weight + 1) / 16, log2(max weight + 1) / 16,
//                log2(V) / 32, lanes / 64, 0, 0, 1]
//   SCC pivot:  [log2(E / V + 1) / 8, log2(active / V) / 8, log2(active edges / active + 1) / 8,
//                log2(V) / 32, log2(max out x in + 1) / 64, 0, 0, 0.5], after trimming
// A direction is taken from the network only when its two logits differ by at least
// kDirMargin; otherwise the fixed switch decides.
// Parameter layout: W1[HID][IN], b1[HID], W2[OUT][HID], b2[OUT].
#include "common.cuh"
#include "sched_net.cuh"

namespace gir {

namespace {

using namespace sched_net;
constexpr int kBlock = 128;
constexpr uint64_t kDeltaChoices[6] = {16, 32, 64, 256, 2048, 8192};

// The next BFS level's direction, decided on the device from the level's counters (frontier
// pairs and out-edges, summed over lanes), so the network costs no extra host round trip: the
// decision and its features travel back with the counters the host reads anyway.
__global__ void k_bfs_decide(const float* params, unsigned long long* cnt, int i_pairs, int i_medges, int i_dir,
                             int i_feat, int lanes, double V, double E, double mu_prev, int bottom_up, double alpha,
                             double beta) {
    if (threadIdx.x != 0) return;
    const double nf = (double)cnt[i_pairs] / lanes, mf = (double)cnt[i_medges] / lanes;
    float x[IN];
    cnt[i_dir] = (unsigned long long)decide_direction(params, V, E, nf, mf, mu_prev - mf, bottom_up, lanes, alpha,
                                                      beta, x);
    float* f = reinterpret_cast<float*>(&cnt[i_feat]);
    for (int i = 0; i < IN; ++i) f[i] = x[i];
}

__global__ void k_mlp_forward(const float* params, const float* x, int64_t n, float* logits) {
    __shared__ float sp[NP];
    for (int i = threadIdx.x; i < NP; i += blockDim.x) sp[i] = params[i];
    __syncthreads();
    const Layout L = layout(sp);
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x) {
        float xi[IN], h[HID], o[OUT];
        for (int i = 0; i < IN; ++i) xi[i] = x[s * IN + i];
        forward_one(L, xi, h, o);
        for (int k = 0; k < OUT; ++k) logits[s * OUT + k] = o[k];
    }
}

// Gradient of the mean softmax cross-entropy; per-block partial sums in shared memory, then one
// atomicAdd per parameter per block. grad / loss must be zeroed by the caller.
__global__ void k_mlp_grad(const float* params, const float* x, const int32_t* y, int64_t n, float* grad,
                           float* loss) {
    __shared__ float sp[NP];
    __shared__ float sg[NP];
    __shared__ float sl;
    for (int i = threadIdx.x; i < NP; i += blockDim.x) { sp[i] = params[i]; sg[i] = 0.f; }
    if (threadIdx.x == 0) sl = 0.f;
    __syncthreads();
    const Layout L = layout(sp);
    float* gW1 = sg;
    float* gb1 = sg + HID * IN;
    float* gW2 = gb1 + HID;
    float* gb2 = gW2 + OUT * HID;
    const float inv_n = 1.f / (float)n;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x) {
        float xi[IN], h[HID], o[OUT];
        for (int i = 0; i < IN; ++i) xi[i] = x[s * IN + i];
        forward_one(L, xi, h, o);
        float m = o[0];
        for (int k = 1; k < OUT; ++k) m = fmaxf(m, o[k]);
        float z = 0.f;
        for (int k = 0; k < OUT; ++k) z += expf(o[k] - m);
        const int t = y[s];
        atomicAdd(&sl, (logf(z) + m - o[t]) * inv_n);
        float d[OUT];
        for (int k = 0; k < OUT; ++k) d[k] = (expf(o[k] - m) / z - (k == t ? 1.f : 0.f)) * inv_n;
        for (int k = 0; k < OUT; ++k) {
            atomicAdd(&gb2[k], d[k]);
            for (int j = 0; j < HID; ++j) atomicAdd(&gW2[k * HID + j], d[k] * h[j]);
        }
        for (int j = 0; j < HID; ++j) {
            float dh = 0.f;
            for (int k = 0; k < OUT; ++k) dh += L.W2[k * HID + j] * d[k];
            const float dz = dh * (1.f - h[j] * h[j]);
            atomicAdd(&gb1[j], dz);
            for (int i = 0; i < IN; ++i) atomicAdd(&gW1[j * IN + i], dz * xi[i]);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < NP; i += blockDim.x) atomicAdd(&grad[i], sg[i]);
    if (threadIdx.x == 0) atomicAdd(loss, sl);
}

__global__ void k_sgd(float* params, const float* grad, float lr) {
    for (int i = threadIdx.x; i < NP; i += blockDim.x) params[i] -= lr * grad[i];
}

int ensure_params(gir_dev* g, float** p) {
    GIR_TRY(ensure_n(g, g->sched_w, NP, p));
    if (!g->sched_loaded && g->sched_host.empty()) {
        // deterministic small initial weights (a hash of the index), zero biases
        std::vector<float> h(NP, 0.f);
        for (int i = 0; i < HID * IN + HID + OUT * HID; ++i) {
            if (i >= HID * IN && i < HID * IN + HID) continue;
            uint64_t z = (uint64_t)i * 0x9e3779b97f4a7c15ULL;
            z = (z ^ (z >> 31)) * 0xbf58476d1ce4e5b9ULL;
            h[i] = ((float)((z >> 40) & 0xffff) / 65535.f - 0.5f) * 0.5f;
        }
        g->sched_host = h;
        GIR_CUDA(g, cudaMemcpyAsync(*p, h.data(), sizeof(float) * NP, cudaMemcpyHostToDevice, g->stream));
    }
    return GIR_OK;
}

int run_forward(gir_dev* g, const float* x_dev, int64_t n, float* logits_dev) {
    float* p = nullptr;
    GIR_TRY(ensure_params(g, &p));
    int blocks = (int)((n + kBlock - 1) / kBlock);
    if (blocks < 1) blocks = 1;
    if (blocks > 4 * g->num_sms) blocks = 4 * g->num_sms;
    k_mlp_forward<<<blocks, kBlock, 0, g->stream>>>(p, x_dev, n, logits_dev);
    GIR_LAUNCH(g, "k_mlp_forward");
    return GIR_OK;
}

int run_grad(gir_dev* g, const float* x_dev, const int32_t* y_dev, int64_t n, float* grad_dev, float* loss_dev) {
    float* p = nullptr;
    GIR_TRY(ensure_params(g, &p));
    GIR_CUDA(g, cudaMemsetAsync(grad_dev, 0, sizeof(float) * NP, g->stream));
    GIR_CUDA(g, cudaMemsetAsync(loss_dev, 0, sizeof(float), g->stream));
    int blocks = (int)((n + kBlock - 1) / kBlock);
    if (blocks < 1) blocks = 1;
    if (blocks > 2 * g->num_sms) blocks = 2 * g->num_sms;
    k_mlp_grad<<<blocks, kBlock, 0, g->stream>>>(p, x_dev, y_dev, n, grad_dev, loss_dev);
    GIR_LAUNCH(g, "k_mlp_grad");
    return GIR_OK;
}

// One decision: logits of one feature vector, argmax over [lo, hi) and its margin over the
// runner-up.
int decide(gir_dev* g, const float* features, int lo, int hi, int* choice, float* margin) {
    float* buf = nullptr;
    GIR_TRY(ensure_n(g, g->sched_io, IN + OUT + 8, &buf));
    float tmp_in[IN];
    for (int i = 0; i < IN; ++i) tmp_in[i] = features[i];
    GIR_CUDA(g, cudaMemcpyAsync(buf, tmp_in, sizeof(float) * IN, cudaMemcpyHostToDevice, g->stream));
    GIR_TRY(run_forward(g, buf, 1, buf + IN));
    float logits[OUT];
    GIR_CUDA(g, cudaMemcpyAsync(logits, buf + IN, sizeof(float) * OUT, cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    int best = lo;
    for (int k = lo + 1; k < hi; ++k)
        if (logits[k] > logits[best]) best = k;
    float second = -3.0e38f;
    for (int k = lo; k < hi; ++k)
        if (k != best && logits[k] > second) second = logits[k];
    *choice = best;
    *margin = logits[best] - second;
    return GIR_OK;
}

}  // namespace

void sched_bfs_features(const gir_dev* g, double nf, double mf, double mu, int level, bool bottom_up, int lanes,
                        float* out) {
    (void)level;
    bfs_features((double)(g->V > 0 ? g->V : 1), (double)g->fw.E + 1.0, nf, mf, mu, bottom_up, lanes, out);
}

int sched_bfs_decide_async(gir_dev* g, unsigned long long* cnt, int i_pairs, int i_medges, int i_dir, int i_feat,
                           int lanes, double mu_prev, bool bottom_up, double alpha, double beta) {
    float* p = nullptr;
    GIR_TRY(ensure_params(g, &p));
    k_bfs_decide<<<1, 32, 0, g->stream>>>(p, cnt, i_pairs, i_medges, i_dir, i_feat, lanes,
                                          (double)(g->V > 0 ? g->V : 1), (double)g->fw.E + 1.0, mu_prev,
                                          bottom_up ? 1 : 0, alpha, beta);
    GIR_LAUNCH(g, "k_bfs_decide");
    return GIR_OK;
}

void sched_sssp_features(const gir_dev* g, int weight_mode, int lanes, float* out) {
    const double V = (double)(g->V > 0 ? g->V : 1), E = (double)g->fw.E + 1.0;
    const int m = weight_mode == GIR_WEIGHT_HASH ? 0 : 1;
    out[0] = (float)(std::log2(E / V + 1.0) / 8.0);
    out[1] = (float)(std::log2(g->wstat[m][0] + 1.0) / 16.0);
    out[2] = (float)(std::log2(g->wstat[m][1] + 1.0) / 16.0);
    out[3] = (float)(std::log2(V) / 32.0);
    out[4] = (float)(lanes / 64.0);
    out[5] = 0.f;
    out[6] = 0.f;
    out[7] = 1.f;  // task: SSSP bucket width
}

int sched_delta_class(uint64_t delta) {
    int best = 0;
    double bd = 1e300;
    for (int i = 0; i < 6; ++i) {
        const double d = std::fabs(std::log2((double)delta) - std::log2((double)kDeltaChoices[i]));
        if (d < bd) { bd = d; best = i; }
    }
    return 2 + best;
}

void sched_trace(gir_dev* g, const float* x, int32_t y) {
    if (g->trace_y.size() >= (1u << 20)) return;  // bounded
    g->trace_x.insert(g->trace_x.end(), x, x + IN);
    g->trace_y.push_back(y);
}

void sched_scc_features(const gir_dev* g, double active, double active_edges, double max_score, float* out) {
    const double V = (double)(g->V > 0 ? g->V : 1), E = (double)g->fw.E + 1.0;
    const double tiny = 1.0 / 4294967296.0;
    out[0] = (float)(std::log2(E / V + 1.0) / 8.0);
    out[1] = (float)(std::log2(active / V + tiny) / 8.0);
    out[2] = (float)(std::log2(active_edges / (active + 1.0) + 1.0) / 8.0);
    out[3] = (float)(std::log2(V) / 32.0);
    out[4] = (float)(std::log2(max_score + 1.0) / 64.0);
    out[5] = 0.f;
    out[6] = 0.f;
    out[7] = 0.5f;  // task: SCC pivot rule
}

int sched_choose_pivot(gir_dev* g, const float* features, int* rule) {
    int c = 8;
    float margin = 0.f;
    GIR_TRY(decide(g, features, 8, 12, &c, &margin));
    *rule = margin >= kPivotMargin ? c - 8 : 0;
    return GIR_OK;
}

int sched_choose_delta(gir_dev* g, const float* features, uint64_t* delta) {
    int c = 2;
    float margin = 0.f;
    GIR_TRY(decide(g, features, 2, 8, &c, &margin));
    *delta = kDeltaChoices[c - 2];
    return GIR_OK;
}

}  // namespace gir

using namespace gir;

extern "C" {

int64_t gir_dev_sched_param_count(void) { return NP; }

int gir_dev_sched_delta_choices(uint64_t* out6) {
    if (!out6) return GIR_ERR_INVALID;
    for (int i = 0; i < 6; ++i) out6[i] = kDeltaChoices[i];
    return GIR_OK;
}

int gir_dev_sched_trace(gir_dev_t* g, float* features, int32_t* choice, int64_t cap, int64_t* n) {
    if (!g || !n || cap < 0) return GIR_ERR_INVALID;
    *n = (int64_t)g->trace_y.size();
    const int64_t m = cap < *n ? cap : *n;
    if (m > 0 && (!features || !choice)) return fail(g, GIR_ERR_INVALID, "sched_trace: null output");
    for (int64_t i = 0; i < m; ++i) {
        for (int k = 0; k < IN; ++k) features[i * IN + k] = g->trace_x[(size_t)i * IN + k];
        choice[i] = g->trace_y[(size_t)i];
    }
    return GIR_OK;
}

int gir_dev_sched_set_weights(gir_dev_t* g, const float* params, int64_t n_params) {
    if (!g) return GIR_ERR_INVALID;
    if (!params || n_params != NP) return fail(g, GIR_ERR_INVALID, "sched_set_weights: need gir_dev_sched_param_count() floats");
    float* p = nullptr;
    GIR_TRY(ensure_n(g, g->sched_w, NP, &p));
    g->sched_host.assign(params, params + NP);
    GIR_CUDA(g, cudaMemcpyAsync(p, g->sched_host.data(), sizeof(float) * NP, cudaMemcpyHostToDevice, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    g->sched_loaded = true;
    return GIR_OK;
}

int gir_dev_sched_get_weights(gir_dev_t* g, float* params, int64_t n_params) {
    if (!g) return GIR_ERR_INVALID;
    if (!params || n_params != NP) return fail(g, GIR_ERR_INVALID, "sched_get_weights: need gir_dev_sched_param_count() floats");
    float* p = nullptr;
    GIR_TRY(ensure_params(g, &p));
    GIR_CUDA(g, cudaMemcpyAsync(params, p, sizeof(float) * NP, cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    return GIR_OK;
}

int gir_dev_sched_forward(gir_dev_t* g, const float* x, int64_t n, float* logits) {
    if (!g) return GIR_ERR_INVALID;
    if (n < 0 || (n > 0 && (!x || !logits))) return fail(g, GIR_ERR_INVALID, "sched_forward: bad arguments");
    if (n == 0) return GIR_OK;
    const void* dx = nullptr;
    GIR_TRY(stage_input(g, g->stage_in, x, sizeof(float) * IN * n, &dx));
    float* dl = nullptr;
    GIR_TRY(ensure_n(g, g->stage_out, OUT * n, &dl));
    GIR_TRY(run_forward(g, (const float*)dx, n, dl));
    GIR_CUDA(g, cudaMemcpyAsync(logits, dl, sizeof(float) * OUT * n, cudaMemcpyDefault, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    return GIR_OK;
}

int gir_dev_sched_grad(gir_dev_t* g, const float* x, const int32_t* y, int64_t n, float* grad, float* loss) {
    if (!g) return GIR_ERR_INVALID;
    if (n <= 0 || !x || !y || !grad || !loss) return fail(g, GIR_ERR_INVALID, "sched_grad: bad arguments");
    for (int64_t i = 0; i < n && !is_device_ptr(y); ++i)
        if (y[i] < 0 || y[i] >= OUT) return fail(g, GIR_ERR_INVALID, "sched_grad: class out of range");
    const void *dx = nullptr, *dy = nullptr;
    GIR_TRY(stage_input(g, g->stage_in, x, sizeof(float) * IN * n, &dx));
    GIR_TRY(stage_input(g, g->work[7], y, sizeof(int32_t) * n, &dy));
    float* dg = nullptr;
    GIR_TRY(ensure_n(g, g->stage_out, NP + 8, &dg));
    GIR_TRY(run_grad(g, (const float*)dx, (const int32_t*)dy, n, dg, dg + NP));
    GIR_CUDA(g, cudaMemcpyAsync(grad, dg, sizeof(float) * NP, cudaMemcpyDefault, g->stream));
    GIR_CUDA(g, cudaMemcpyAsync(loss, dg + NP, sizeof(float), cudaMemcpyDefault, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    return GIR_OK;
}

int gir_dev_sched_train(gir_dev_t* g, const float* x, const int32_t* y, int64_t n, int steps, float lr, float* loss) {
    if (!g) return GIR_ERR_INVALID;
    if (n <= 0 || steps < 1 || !x || !y || !(lr > 0.f)) return fail(g, GIR_ERR_INVALID, "sched_train: bad arguments");
    for (int64_t i = 0; i < n && !is_device_ptr(y); ++i)
        if (y[i] < 0 || y[i] >= OUT) return fail(g, GIR_ERR_INVALID, "sched_train: class out of range");
    const void *dx = nullptr, *dy = nullptr;
    GIR_TRY(stage_input(g, g->stage_in, x, sizeof(float) * IN * n, &dx));
    GIR_TRY(stage_input(g, g->work[7], y, sizeof(int32_t) * n, &dy));
    float *p = nullptr, *dg = nullptr;
    GIR_TRY(ensure_params(g, &p));
    GIR_TRY(ensure_n(g, g->stage_out, NP + 8, &dg));
    for (int s = 0; s < steps; ++s) {
        GIR_TRY(run_grad(g, (const float*)dx, (const int32_t*)dy, n, dg, dg + NP));
        k_sgd<<<1, 256, 0, g->stream>>>(p, dg, lr);
        GIR_LAUNCH(g, "k_sgd");
    }
    float hl = 0.f;
    GIR_CUDA(g, cudaMemcpyAsync(&hl, dg + NP, sizeof(float), cudaMemcpyDeviceToHost, g->stream));
    g->sched_host.resize(NP);
    GIR_CUDA(g, cudaMemcpyAsync(g->sched_host.data(), p, sizeof(float) * NP, cudaMemcpyDeviceToHost, g->stream));
    GIR_CUDA(g, cudaStreamSynchronize(g->stream));
    if (loss) *loss = hl;
    g->sched_loaded = true;
    return GIR_OK;
}

}  // extern "C"
