// The schedule network's forward pass and the BFS level features, shared by the schedule kernels
// (sched.cu) and the traversal kernels that decide on the device (bfs.cu). A 2-layer MLP:
// GIR_SCHED_IN features -> GIR_SCHED_HID tanh units -> GIR_SCHED_OUT logits, fp32; parameter
// layout W1[HID][IN], b1[HID], W2[OUT][HID], b2[OUT].
#pragma once
#include "common.cuh"

namespace gir {
namespace sched_net {

constexpr int IN = GIR_SCHED_IN, HID = GIR_SCHED_HID, OUT = GIR_SCHED_OUT;
constexpr int NP = HID * IN + HID + OUT * HID + OUT;
// A BFS direction is taken from the network only when its two logits differ by at least this;
// otherwise the fixed switch decides.
constexpr float kDirMargin = 8.0f;
// The pivot rule is taken from the network only when its best logit leads the runner-up by at
// least this; otherwise the fixed rule (max out x in degree) is used.
constexpr float kPivotMargin = 1.0f;

struct Layout {
    const float *W1, *b1, *W2, *b2;
};
__device__ __forceinline__ Layout layout(const float* p) {
    return Layout{p, p + HID * IN, p + HID * IN + HID, p + HID * IN + HID + OUT * HID};
}

__device__ __forceinline__ void forward_one(const Layout& L, const float* x, float* h, float* o) {
    for (int j = 0; j < HID; ++j) {
        float z = L.b1[j];
        for (int i = 0; i < IN; ++i) z += L.W1[j * IN + i] * x[i];
        h[j] = tanhf(z);
    }
    for (int k = 0; k < OUT; ++k) {
        float z = L.b2[k];
        for (int j = 0; j < HID; ++j) z += L.W2[k * HID + j] * h[j];
        o[k] = z;
    }
}

// BFS level features: nf / mf = the frontier's vertices / out-edges and mu = the out-edges not yet
// explored, all per lane.
__host__ __device__ inline void bfs_features(double V, double E, double nf, double mf, double mu, bool bottom_up,
                                             int lanes, float* out) {
    const double tiny = 1.0 / 4294967296.0;
    out[0] = (float)(log2(nf / V + tiny) / 8.0);
    out[1] = (float)((log2(mf + 1.0) - log2(mu + 1.0)) / 8.0);
    out[2] = (float)(log2(mu / E + tiny) / 8.0);
    out[3] = (float)(log2(mf / E + tiny) / 8.0);
    out[4] = bottom_up ? 1.f : 0.f;
    out[5] = (float)(log2(E / V + 1.0) / 8.0);
    out[6] = (float)(lanes / 64.0);
    out[7] = 0.f;  // task: BFS direction
}

// The direction of the next level: the fixed switch (alpha / beta, gir_query.cpp:159-169), or the
// network when `params` is given and its margin is large enough. x receives the features.
__device__ __forceinline__ int decide_direction(const float* params, double V, double E, double nf, double mf,
                                                double mu, int bottom_up, int lanes, double alpha, double beta,
                                                float* x) {
    int fixed = bottom_up;
    if (!bottom_up && mf * alpha > mu) fixed = 1;
    else if (bottom_up && nf * beta < V) fixed = 0;
    bfs_features(V, E, nf, mf, mu, bottom_up != 0, lanes, x);
    if (!params) return fixed;
    float h[HID], o[OUT];
    forward_one(layout(params), x, h, o);
    const int net = o[1] > o[0] ? 1 : 0;
    return fabsf(o[1] - o[0]) >= kDirMargin ? net : fixed;
}

}  // namespace sched_net
}  // namespace gir
