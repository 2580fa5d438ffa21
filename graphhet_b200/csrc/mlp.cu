// The schedule-policy network: 12 inputs -> 64 -> 64 (ReLU) -> 20 logits in
// three heads (BFS direction push/pull, top-down frontier format
// queue/bitmap, SSSP bucket-width bin of 16), 6,292 FP32 parameters.
//
// Parameter layout (row-major, x @ W): W1[12][64] b1[64] W2[64][64] b2[64]
// W3[64][20] b3[20].  Inputs are standardised first: (x - mean) * inv_std.
//
// Training is full-batch: forward, masked softmax cross-entropy per head
// (label -1 = no label), backward and Adam, each a small hand-written kernel
// (thread per output element, sums over the batch in a fixed order, so
// gradients are deterministic).  Inference for one sample runs inside the
// persistent BFS kernel (mlp_infer_block) or as a batch (ghb_mlp_forward).
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "policy.cuh"

namespace ghb {

constexpr int kIn = kPolIn, kH = kPolH, kOut = kPolOut, kParams = kPolParams;
static_assert(kParams == GHB_POLICY_PARAMS, "parameter count");

namespace {

// Z[b][o] = sum_i A[b][i] W[i][o] + bias[o] (A standardised when norm given)
__global__ void dense_fwd_kernel(const float* __restrict__ A, int in, const float* __restrict__ W,
                                 const float* __restrict__ bias, int out, int B, const float* __restrict__ norm,
                                 bool relu, float* __restrict__ Z, float* __restrict__ H) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < (int64_t)B * out;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(t / out), o = (int)(t % out);
        float z = bias[o];
        for (int i = 0; i < in; ++i) {
            float a = A[(int64_t)b * in + i];
            if (norm) a = (a - norm[i]) * norm[kIn + i];
            z += a * W[i * out + o];
        }
        Z[t] = z;
        if (H) H[t] = relu ? fmaxf(z, 0.f) : z;
    }
}

// Softmax cross-entropy per head, weighted mean over the labelled rows:
// dZ = w_b (softmax - onehot) / sum_w(head); wt NULL = weight 1.
__global__ void loss_kernel(const float* __restrict__ logits, const int32_t* __restrict__ y,
                            const float* __restrict__ wt, int B, const float* __restrict__ head_count,
                            float* __restrict__ dZ, float* __restrict__ loss) {
    const int heads[4] = {0, 2, 4, 20};
    for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < B; b += (int64_t)gridDim.x * blockDim.x) {
        float l = 0.f;
        for (int h = 0; h < 3; ++h) {
            const int s = heads[h], e = heads[h + 1];
            const int32_t lab = y[b * 3 + h];
            if (lab < 0 || lab >= e - s || head_count[h] <= 0.f) {
                for (int k = s; k < e; ++k) dZ[b * kOut + k] = 0.f;
                continue;
            }
            float mx = -INFINITY;
            for (int k = s; k < e; ++k) mx = fmaxf(mx, logits[b * kOut + k]);
            float den = 0.f;
            for (int k = s; k < e; ++k) den += expf(logits[b * kOut + k] - mx);
            const float inv_n = (wt ? wt[b] : 1.f) / head_count[h];
            for (int k = s; k < e; ++k) {
                const float p = expf(logits[b * kOut + k] - mx) / den;
                dZ[b * kOut + k] = (p - (k - s == lab ? 1.f : 0.f)) * inv_n;
            }
            l += (logf(den) + mx - logits[b * kOut + s + lab]) * inv_n;
        }
        loss[b] = l;
    }
}

// dW[i][o] = sum_b A[b][i] dZ[b][o]; db[o] = sum_b dZ[b][o] (thread per weight).
__global__ void dense_wgrad_kernel(const float* __restrict__ A, int in, const float* __restrict__ dZ, int out, int B,
                                   const float* __restrict__ norm, float* __restrict__ dW, float* __restrict__ db) {
    const int64_t total = (int64_t)(in + 1) * out;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(t / out), o = (int)(t % out);
        float s = 0.f;
        if (i < in) {
            for (int b = 0; b < B; ++b) {
                float a = A[(int64_t)b * in + i];
                if (norm) a = (a - norm[i]) * norm[kIn + i];
                s += a * dZ[(int64_t)b * out + o];
            }
            dW[i * out + o] = s;
        } else {
            for (int b = 0; b < B; ++b) s += dZ[(int64_t)b * out + o];
            db[o] = s;
        }
    }
}

// dZprev[b][i] = (sum_o dZ[b][o] W[i][o]) * relu'(Zprev[b][i]).
__global__ void dense_bgrad_kernel(const float* __restrict__ dZ, int out, const float* __restrict__ W, int in, int B,
                                   const float* __restrict__ Zprev, float* __restrict__ dZprev) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < (int64_t)B * in;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(t / in), i = (int)(t % in);
        float s = 0.f;
        for (int o = 0; o < out; ++o) s += dZ[(int64_t)b * out + o] * W[i * out + o];
        dZprev[t] = Zprev[t] > 0.f ? s : 0.f;
    }
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1,
                            float* __restrict__ m2, int count, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float a = b1 * m1[i] + (1.f - b1) * gi;
        const float v = b2 * m2[i] + (1.f - b2) * gi * gi;
        m1[i] = a;
        m2[i] = v;
        p[i] -= lr * (a / c1) / (sqrtf(v / c2) + eps);
    }
}

__global__ void sum_kernel(const float* __restrict__ x, int n, float* out) {
    __shared__ float red[32];
    float s = 0.f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += x[i];
    s = warp_sum(s);
    if (lane_id() == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
        *out = t;
    }
}

// Summed weight of the labelled rows per head (for the weighted mean).
__global__ void head_count_kernel(const int32_t* __restrict__ y, const float* __restrict__ wt, int B, float* count) {
    if (threadIdx.x < 3 && blockIdx.x == 0) {
        float c = 0.f;
        for (int b = 0; b < B; ++b) c += y[b * 3 + threadIdx.x] >= 0 ? (wt ? wt[b] : 1.f) : 0.f;
        count[threadIdx.x] = c;
    }
}

struct MlpBuffers {
    float *z1, *h1, *z2, *h2, *z3, *dz3, *dz2, *dz1, *loss, *grad, *hc, *lsum;
    static MlpBuffers carve(Carver& c, int B) {
        MlpBuffers m;
        m.z1 = c.take<float>((size_t)B * kH);
        m.h1 = c.take<float>((size_t)B * kH);
        m.z2 = c.take<float>((size_t)B * kH);
        m.h2 = c.take<float>((size_t)B * kH);
        m.z3 = c.take<float>((size_t)B * kOut);
        m.dz3 = c.take<float>((size_t)B * kOut);
        m.dz2 = c.take<float>((size_t)B * kH);
        m.dz1 = c.take<float>((size_t)B * kH);
        m.loss = c.take<float>((size_t)B);
        m.grad = c.take<float>(kParams);
        m.hc = c.take<float>(4);
        m.lsum = c.take<float>(4);
        return m;
    }
};

int mlp_forward(ghb_workspace* ws, const MlpBuffers& m, const float* P, const float* norm, const float* x, int B) {
    const unsigned g = ws->num_sms * 4;
    GHB_TRY(launch(ws, dense_fwd_kernel, dim3(grid_for((int64_t)B * kH, 256, g)), dim3(256), 0, x, kIn, P + kOffW1,
                   P + kOffB1, kH, B, norm, true, m.z1, m.h1));
    GHB_TRY(launch(ws, dense_fwd_kernel, dim3(grid_for((int64_t)B * kH, 256, g)), dim3(256), 0, (const float*)m.h1, kH,
                   P + kOffW2, P + kOffB2, kH, B, (const float*)nullptr, true, m.z2, m.h2));
    return launch(ws, dense_fwd_kernel, dim3(grid_for((int64_t)B * kOut, 256, g)), dim3(256), 0, (const float*)m.h2, kH,
                  P + kOffW3, P + kOffB3, kOut, B, (const float*)nullptr, false, m.z3, (float*)nullptr);
}

// Forward + loss + backward into m.grad; loss total into m.lsum[0].
int mlp_grad(ghb_workspace* ws, const MlpBuffers& m, const float* P, const float* norm, const float* x,
             const int32_t* y, const float* wt, int B) {
    const unsigned g = ws->num_sms * 4;
    GHB_TRY(mlp_forward(ws, m, P, norm, x, B));
    GHB_TRY(launch(ws, head_count_kernel, dim3(1), dim3(32), 0, y, wt, B, m.hc));
    GHB_TRY(launch(ws, loss_kernel, dim3(grid_for(B, 256, g)), dim3(256), 0, (const float*)m.z3, y, wt, B,
                   (const float*)m.hc, m.dz3, m.loss));
    GHB_TRY(launch(ws, sum_kernel, dim3(1), dim3(1024), 0, (const float*)m.loss, B, m.lsum));
    GHB_TRY(launch(ws, dense_wgrad_kernel, dim3(grid_for((kH + 1) * kOut, 256, g)), dim3(256), 0, (const float*)m.h2,
                   kH, (const float*)m.dz3, kOut, B, (const float*)nullptr, m.grad + kOffW3, m.grad + kOffB3));
    GHB_TRY(launch(ws, dense_bgrad_kernel, dim3(grid_for((int64_t)B * kH, 256, g)), dim3(256), 0, (const float*)m.dz3,
                   kOut, P + kOffW3, kH, B, (const float*)m.z2, m.dz2));
    GHB_TRY(launch(ws, dense_wgrad_kernel, dim3(grid_for((kH + 1) * kH, 256, g)), dim3(256), 0, (const float*)m.h1,
                   kH, (const float*)m.dz2, kH, B, (const float*)nullptr, m.grad + kOffW2, m.grad + kOffB2));
    GHB_TRY(launch(ws, dense_bgrad_kernel, dim3(grid_for((int64_t)B * kH, 256, g)), dim3(256), 0, (const float*)m.dz2,
                   kH, P + kOffW2, kH, B, (const float*)m.z1, m.dz1));
    return launch(ws, dense_wgrad_kernel, dim3(grid_for((kIn + 1) * kH, 256, g)), dim3(256), 0, x, kIn,
                  (const float*)m.dz1, kH, B, norm, m.grad + kOffW1, m.grad + kOffB1);
}

// The loaded policy, per device: parameters + normalisation, and a host copy.
struct LoadedPolicy {
    float* dev = nullptr;  // kParams + 2 * kIn floats
    bool loaded = false;
};
std::mutex g_policy_mu;
LoadedPolicy g_policy[64];
std::vector<float> g_policy_host;  // kParams + 2 * kIn

}  // namespace

const float* policy_device_params() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(g_policy_mu);
    if (!g_policy[dev].loaded) {
        if (g_policy_host.empty()) return nullptr;
        if (cudaMalloc(&g_policy[dev].dev, sizeof(float) * kPolTotal) != cudaSuccess) return nullptr;
        if (cudaMemcpy(g_policy[dev].dev, g_policy_host.data(), sizeof(float) * kPolTotal,
                       cudaMemcpyHostToDevice) != cudaSuccess)
            return nullptr;
        g_policy[dev].loaded = true;
    }
    return g_policy[dev].dev;
}

// Host-side evaluation of the loaded network for one feature row (the same
// arithmetic as the device kernels), for the host-driven level loop.
static void policy_host_logits(const float* f, float* out) {
    const float* P = g_policy_host.data();
    const float* mu = P + kParams;
    const float* is = mu + kIn;
    float x[kIn], h1[kH], h2[kH];
    for (int i = 0; i < kIn; ++i) x[i] = (f[i] - mu[i]) * is[i];
    for (int o = 0; o < kH; ++o) {
        float z = P[kOffB1 + o];
        for (int i = 0; i < kIn; ++i) z += x[i] * P[kOffW1 + i * kH + o];
        h1[o] = z > 0.f ? z : 0.f;
    }
    for (int o = 0; o < kH; ++o) {
        float z = P[kOffB2 + o];
        for (int i = 0; i < kH; ++i) z += h1[i] * P[kOffW2 + i * kH + o];
        h2[o] = z > 0.f ? z : 0.f;
    }
    for (int o = 0; o < kOut; ++o) {
        float z = P[kOffB3 + o];
        for (int i = 0; i < kH; ++i) z += h2[i] * P[kOffW3 + i * kOut + o];
        out[o] = z;
    }
}

bool policy_pick_level(const float* features, int* dir, int* fmt) {
    std::lock_guard<std::mutex> lock(g_policy_mu);
    if (g_policy_host.empty()) return false;
    float z[kOut];
    policy_host_logits(features, z);
    *dir = z[kHeadDir + 1] > z[kHeadDir] ? 1 : 0;
    *fmt = z[kHeadFmt + 1] > z[kHeadFmt] ? 1 : 0;
    return true;
}

double policy_pick_delta(const float* features, double base_delta) {
    std::lock_guard<std::mutex> lock(g_policy_mu);
    if (g_policy_host.empty()) return -1.0;
    float z[kOut];
    policy_host_logits(features, z);
    int best = 0;
    for (int k = 1; k < kDeltaBins; ++k)
        if (z[kHeadDelta + k] > z[kHeadDelta + best]) best = k;
    return base_delta * std::ldexp(1.0, best - kDeltaBinZero);
}

}  // namespace ghb

using namespace ghb;

extern "C" {

int ghb_policy_load(const float* params, const float* norm) {
    GHB_REQUIRE((params == nullptr) == (norm == nullptr), "params and norm must both be given or both NULL");
    std::lock_guard<std::mutex> lock(g_policy_mu);
    g_policy_host.clear();
    if (params) {
        g_policy_host.assign(params, params + kParams);
        g_policy_host.insert(g_policy_host.end(), norm, norm + 2 * kIn);
    }
    for (int d = 0; d < 64; ++d) {
        if (g_policy[d].dev) {
            int cur = 0;
            cudaGetDevice(&cur);
            cudaSetDevice(d);
            cudaFree(g_policy[d].dev);
            cudaSetDevice(cur);
        }
        g_policy[d] = LoadedPolicy();
    }
    return GHB_OK;
}

int ghb_policy_loaded(void) {
    std::lock_guard<std::mutex> lock(g_policy_mu);
    return g_policy_host.empty() ? 0 : 1;
}

int ghb_mlp_forward(ghb_workspace* ws, const float* params, const float* norm, const float* x, int32_t batch,
                    float* logits) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws && params && norm && x && logits, "NULL argument");
    GHB_REQUIRE(batch >= 1, "batch < 1");
    Carver sizing(nullptr);
    MlpBuffers::carve(sizing, batch);
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    MlpBuffers m = MlpBuffers::carve(c, batch);
    GHB_TRY(mlp_forward(ws, m, params, norm, x, batch));
    GHB_CUDA_TRY(cudaMemcpyAsync(logits, m.z3, sizeof(float) * batch * kOut, cudaMemcpyDeviceToDevice, ws->stream));
    return GHB_OK;
}

int ghb_mlp_grad(ghb_workspace* ws, const float* params, const float* norm, const float* x, const int32_t* y,
                 const float* sample_weight, int32_t batch, float* grad, float* loss) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws && params && norm && x && y && grad, "NULL argument");
    GHB_REQUIRE(batch >= 1, "batch < 1");
    Carver sizing(nullptr);
    MlpBuffers::carve(sizing, batch);
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    MlpBuffers m = MlpBuffers::carve(c, batch);
    GHB_TRY(mlp_grad(ws, m, params, norm, x, y, sample_weight, batch));
    GHB_CUDA_TRY(cudaMemcpyAsync(grad, m.grad, sizeof(float) * kParams, cudaMemcpyDeviceToDevice, ws->stream));
    if (loss) {
        GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, m.lsum, sizeof(float), cudaMemcpyDeviceToHost, ws->stream));
        GHB_CUDA_TRY(cudaStreamSynchronize(ws->stream));
        *loss = *reinterpret_cast<const float*>(ws->host_pinned);
    }
    return GHB_OK;
}

int ghb_mlp_train(ghb_workspace* ws, float* params, const float* norm, const float* x, const int32_t* y,
                  const float* sample_weight, int32_t batch, int32_t epochs, float lr, float* loss_history) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws && params && norm && x && y, "NULL argument");
    GHB_REQUIRE(batch >= 1 && epochs >= 0, "bad sizes");
    Carver sizing(nullptr);
    MlpBuffers::carve(sizing, batch);
    sizing.take<float>(kParams);
    sizing.take<float>(kParams);
    sizing.take<float>(epochs > 0 ? epochs : 1);
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    MlpBuffers m = MlpBuffers::carve(c, batch);
    float* m1 = c.take<float>(kParams);
    float* m2 = c.take<float>(kParams);
    float* hist = c.take<float>(epochs > 0 ? epochs : 1);
    GHB_CUDA_TRY(cudaMemsetAsync(m1, 0, sizeof(float) * kParams, ws->stream));
    GHB_CUDA_TRY(cudaMemsetAsync(m2, 0, sizeof(float) * kParams, ws->stream));
    const float b1 = 0.9f, b2 = 0.999f;
    double p1 = 1.0, p2 = 1.0;
    for (int e = 0; e < epochs; ++e) {
        GHB_TRY(mlp_grad(ws, m, params, norm, x, y, sample_weight, batch));
        GHB_CUDA_TRY(cudaMemcpyAsync(hist + e, m.lsum, sizeof(float), cudaMemcpyDeviceToDevice, ws->stream));
        p1 *= b1;
        p2 *= b2;
        GHB_TRY(launch(ws, adam_kernel, dim3(grid_for(kParams, 256, 64)), dim3(256), 0, params, (const float*)m.grad, m1,
                       m2, kParams, lr, b1, b2, 1e-8f, (float)(1.0 - p1), (float)(1.0 - p2)));
    }
    if (loss_history && epochs > 0) {
        GHB_CUDA_TRY(cudaMemcpyAsync(loss_history, hist, sizeof(float) * epochs, cudaMemcpyDeviceToHost, ws->stream));
        GHB_CUDA_TRY(cudaStreamSynchronize(ws->stream));
    }
    return GHB_OK;
}

}  // extern "C"
