// Schedule selection for the MSM: scalar-distribution features, an exhaustive
// window autotuner, and a small MLP cost model trained and evaluated by the
// kernels in this file.
//
// The model predicts log(milliseconds) of one MSM from
//   x = [log2 n / 24, log2(batch) / 8, bit-length histogram of the scalars
//        (7 bins: zero, 1-16, 17-32, 33-64, 65-128, 129-192, 193-254 bits),
//        (c - 12) / 8]
// (MLP_IN = 10 inputs), two hidden layers of 64 ReLU units, one linear
// output.  It only chooses the window width; the MSM result does not depend
// on it, so predictions never change values.
//
// There is no counterpart in the reference: its window width is the fixed
// formula of src/cuda/msm.rs:105.
#include <math.h>

#include <vector>

#include "common.cuh"
#include "kernels.h"

namespace zk {

static constexpr int MLP_IN = 10;
static constexpr int H1 = 64;
static constexpr int H2 = 64;
// parameter layout: W1[IN][H1], b1[H1], W2[H1][H2], b2[H2], W3[H2], b3
static constexpr int P_W1 = 0;
static constexpr int P_B1 = P_W1 + MLP_IN * H1;
static constexpr int P_W2 = P_B1 + H1;
static constexpr int P_B2 = P_W2 + H1 * H2;
static constexpr int P_W3 = P_B2 + H2;
static constexpr int P_B3 = P_W3 + H2;
static constexpr int P_COUNT = P_B3 + 1;

// ------------------------------------------------------------------ features

__global__ void scalar_hist_kernel(const Fr* scalars, uint32_t n, uint32_t* hist) {
    __shared__ uint32_t h[8];
    if (threadIdx.x < 8) h[threadIdx.x] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Fr k = fe_from_mont<FrCfg>(ldg_elem<FrCfg>(scalars + i));
        int bits = 0;
        for (int w = 7; w >= 0; w--)
            if (k.v[w]) {
                bits = 32 * w + 32 - __clz(k.v[w]);
                break;
            }
        const int bin = bits == 0 ? 0 : bits <= 16 ? 1 : bits <= 32 ? 2 : bits <= 64 ? 3 : bits <= 128 ? 4 : bits <= 192 ? 5 : 6;
        atomicAdd(&h[bin], 1u);
    }
    __syncthreads();
    if (threadIdx.x < 7 && h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], h[threadIdx.x]);
}

// ------------------------------------------------------------------ MLP kernels

__device__ __forceinline__ float relu(float x) { return x > 0.f ? x : 0.f; }

// one thread per sample; writes the prediction and (optionally) the hidden
// activations act[b][H1 + H2]
__global__ void mlp_forward_kernel(const float* P, const float* X, uint32_t B, float* y, float* act) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    float x[MLP_IN], h1[H1];
    for (int i = 0; i < MLP_IN; i++) x[i] = X[b * MLP_IN + i];
    for (int j = 0; j < H1; j++) {
        float s = P[P_B1 + j];
        for (int i = 0; i < MLP_IN; i++) s += x[i] * P[P_W1 + i * H1 + j];
        h1[j] = relu(s);
    }
    float out = P[P_B3];
    for (int k = 0; k < H2; k++) {
        float s = P[P_B2 + k];
        for (int j = 0; j < H1; j++) s += h1[j] * P[P_W2 + j * H2 + k];
        const float h2 = relu(s);
        if (act) act[(size_t)b * (H1 + H2) + H1 + k] = h2;
        out += h2 * P[P_W3 + k];
    }
    if (act)
        for (int j = 0; j < H1; j++) act[(size_t)b * (H1 + H2) + j] = h1[j];
    y[b] = out;
}

// per-sample output error g_b = 2 (y_b - t_b) / B and the loss sum
// weighted mean squared error: loss = sum_b w_b (y_b - t_b)^2 / B (w_b = 1
// when w is null); g_b = dloss / dy_b
__global__ void mlp_dloss_kernel(const float* y, const float* t, const float* w, uint32_t B, float* g,
                                 float* loss) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const float e = y[b] - t[b];
    const float wb = w ? w[b] : 1.f;
    g[b] = 2.f * wb * e / (float)B;
    atomicAdd(loss, wb * e * e / (float)B);
}

// per-sample backward to the hidden layers: d2[b][k] = g_b W3[k] 1(h2>0),
// d1[b][j] = sum_k d2[b][k] W2[j][k] 1(h1>0)
__global__ void mlp_backward_hidden_kernel(const float* P, const float* act, const float* g, uint32_t B, float* d) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const float* a = act + (size_t)b * (H1 + H2);
    float d2[H2];
    for (int k = 0; k < H2; k++) d2[k] = a[H1 + k] > 0.f ? g[b] * P[P_W3 + k] : 0.f;
    float* o = d + (size_t)b * (H1 + H2);
    for (int k = 0; k < H2; k++) o[H1 + k] = d2[k];
    for (int j = 0; j < H1; j++) {
        float s = 0.f;
        if (a[j] > 0.f)
            for (int k = 0; k < H2; k++) s += d2[k] * P[P_W2 + j * H2 + k];
        o[j] = s;
    }
}

// one thread per parameter: sums the per-sample contributions over the batch
// (deterministic: no float atomics)
__global__ void mlp_param_grad_kernel(const float* X, const float* act, const float* g, const float* d, uint32_t B,
                                      float* G) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P_COUNT) return;
    float s = 0.f;
    for (uint32_t b = 0; b < B; b++) {
        const float* a = act + (size_t)b * (H1 + H2);
        const float* dd = d + (size_t)b * (H1 + H2);
        if (p < P_B1) {
            const int i = p / H1, j = p % H1;
            s += X[b * MLP_IN + i] * dd[j];
        } else if (p < P_W2) {
            s += dd[p - P_B1];
        } else if (p < P_B2) {
            const int q = p - P_W2, j = q / H2, k = q % H2;
            s += a[j] * dd[H1 + k];
        } else if (p < P_W3) {
            s += dd[H1 + (p - P_B2)];
        } else if (p < P_B3) {
            s += a[H1 + (p - P_W3)] * g[b];
        } else {
            s += g[b];
        }
    }
    G[p] = s;
}

__global__ void adam_kernel(float* P, const float* G, float* m, float* v, float lr, float b1c, float b2c) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P_COUNT) return;
    const float b1 = 0.9f, b2 = 0.999f;
    m[p] = b1 * m[p] + (1.f - b1) * G[p];
    v[p] = b2 * v[p] + (1.f - b2) * G[p] * G[p];
    P[p] -= lr * (m[p] / b1c) / (sqrtf(v[p] / b2c) + 1e-8f);
}

// deterministic initialisation (He-uniform from a splitmix hash of the index)
__global__ void mlp_init_kernel(float* P, uint64_t seed) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P_COUNT) return;
    uint64_t z = seed + 0x9e3779b97f4a7c15ull * (uint64_t)(p + 1);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    const float u = (float)((z >> 11) * (1.0 / 9007199254740992.0)) * 2.f - 1.f;
    float fan_in = 1.f;
    if (p < P_B1)
        fan_in = MLP_IN;
    else if (p >= P_W2 && p < P_B2)
        fan_in = H1;
    else if (p >= P_W3 && p < P_B3)
        fan_in = H2;
    const bool bias = (p >= P_B1 && p < P_W2) || (p >= P_B2 && p < P_W3) || p == P_B3;
    P[p] = bias ? 0.f : u * sqrtf(6.f / fan_in);
}

}  // namespace zk

using namespace zk;

extern "C" {

int zkp_mlp_input_dim(void) { return MLP_IN; }
size_t zkp_mlp_param_count(void) { return P_COUNT; }

// scratch (floats) the training step needs for a batch of B samples
size_t zkp_mlp_scratch_floats(uint32_t B) { return (size_t)B * (2 * (H1 + H2) + 2) + 1 + P_COUNT; }

cudaError_t zkp_mlp_init(float* params, uint64_t seed, cudaStream_t stream) {
    if (!params) return cudaErrorInvalidValue;
    mlp_init_kernel<<<(P_COUNT + 255) / 256, 256, 0, stream>>>(params, seed);
    return cudaGetLastError();
}

cudaError_t zkp_mlp_forward(const float* params, const float* X, uint32_t B, float* y, cudaStream_t stream) {
    if (!params || !X || !y) return cudaErrorInvalidValue;
    if (B == 0) return cudaSuccess;
    mlp_forward_kernel<<<(B + 127) / 128, 128, 0, stream>>>(params, X, B, y, nullptr);
    return cudaGetLastError();
}

// gradient of the (optionally per-sample weighted) mean squared error over the
// batch; weights may be null; loss (device float) is overwritten; scratch:
// zkp_mlp_scratch_floats(B) floats
cudaError_t zkp_mlp_grad(const float* params, const float* X, const float* t, const float* weights, uint32_t B,
                         float* grads, float* loss, float* scratch, cudaStream_t stream) {
    if (!params || !X || !t || !grads || !loss || !scratch || B == 0) return cudaErrorInvalidValue;
    float* y = scratch;
    float* g = y + B;
    float* act = g + B;
    float* d = act + (size_t)B * (H1 + H2);
    ZK_CHECK(cudaMemsetAsync(loss, 0, sizeof(float), stream));
    const unsigned gb = (B + 127) / 128;
    mlp_forward_kernel<<<gb, 128, 0, stream>>>(params, X, B, y, act);
    mlp_dloss_kernel<<<gb, 128, 0, stream>>>(y, t, weights, B, g, loss);
    mlp_backward_hidden_kernel<<<gb, 128, 0, stream>>>(params, act, g, B, d);
    mlp_param_grad_kernel<<<(P_COUNT + 127) / 128, 128, 0, stream>>>(X, act, g, d, B, grads);
    return cudaGetLastError();
}

// one Adam step (step counts from 1); m and v hold the moments
cudaError_t zkp_mlp_train_step(float* params, float* grads, float* m, float* v, const float* X, const float* t,
                               const float* weights, uint32_t B, float lr, int step, float* loss, float* scratch,
                               cudaStream_t stream) {
    if (step < 1) return cudaErrorInvalidValue;
    ZK_CHECK(zkp_mlp_grad(params, X, t, weights, B, grads, loss, scratch, stream));
    const float b1c = 1.f - powf(0.9f, (float)step), b2c = 1.f - powf(0.999f, (float)step);
    adam_kernel<<<(P_COUNT + 255) / 256, 256, 0, stream>>>(params, grads, m, v, lr, b1c, b2c);
    return cudaGetLastError();
}

// bit-length histogram of n Montgomery-form scalars into hist[0..6] (device
// u32, accumulated; clear it first)
cudaError_t zkp_scalar_histogram(const void* scalars, uint32_t n, uint32_t* hist, cudaStream_t stream) {
    if (n && (!scalars || !hist)) return cudaErrorInvalidValue;
    if (n == 0) return cudaSuccess;
    unsigned g = (n + 255) / 256;
    if (g > 148 * 8) g = 148 * 8;
    scalar_hist_kernel<<<g, 256, 0, stream>>>(reinterpret_cast<const Fr*>(scalars), n, hist);
    return cudaGetLastError();
}

// Exhaustive window search: times zkp_msm for every c in [c_min, c_max] that
// fits `scratch` (reps runs each after one warm-up) and returns the fastest
// c; times_ms[c - c_min] receives the mean time or -1 when skipped.
// Synchronises `stream`.
int zkp_msm_autotune(const void* bases, const void* scalars, uint32_t n, int c_min, int c_max, int reps,
                     void* scratch, size_t scratch_bytes, float* times_ms, void* out, cudaStream_t stream) {
    if (!bases || !scalars || !scratch || !out || c_min < 4 || c_max > 22 || c_min > c_max || reps < 1 || n == 0)
        return -1;
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess) return -1;
    if (cudaEventCreate(&b) != cudaSuccess) {
        cudaEventDestroy(a);
        return -1;
    }
    int best = -1;
    float best_ms = 1e30f;
    for (int c = c_min; c <= c_max; c++) {
        float ms = -1.f;
        const MsmPlan pl = msm_make_plan(n, c);
        if (msm_scratch_bytes(pl) <= scratch_bytes && pl.NB <= 4096u * 4096u) {
            MsmScratch sc;
            msm_layout(pl, scratch, &sc);
            Jac* o = reinterpret_cast<Jac*>(out);
            bool ok = msm_run(o, reinterpret_cast<const Aff*>(bases), reinterpret_cast<const Fr*>(scalars), pl, sc,
                              stream) == cudaSuccess;
            ok = ok && cudaEventRecord(a, stream) == cudaSuccess;
            for (int r = 0; ok && r < reps; r++)
                ok = msm_run(o, reinterpret_cast<const Aff*>(bases), reinterpret_cast<const Fr*>(scalars), pl, sc,
                             stream) == cudaSuccess;
            ok = ok && cudaEventRecord(b, stream) == cudaSuccess && cudaEventSynchronize(b) == cudaSuccess;
            if (ok && cudaEventElapsedTime(&ms, a, b) == cudaSuccess) {
                ms /= reps;
                if (ms < best_ms) {
                    best_ms = ms;
                    best = c;
                }
            } else {
                ms = -1.f;
            }
        }
        if (times_ms) times_ms[c - c_min] = ms;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return best;
}

// Model-chosen window: evaluates the MLP for every candidate c in
// [c_min, c_max] (features f[0..8] = the first nine inputs, host array) and
// returns the c with the smallest predicted time.  scratch: 256 floats of
// device memory.  Synchronises `stream`.
int zkp_msm_schedule_predict(const float* params, const float* features, int c_min, int c_max, float* scratch,
                             cudaStream_t stream) {
    if (!params || !features || !scratch || c_min < 4 || c_max > 22 || c_min > c_max) return -1;
    const int k = c_max - c_min + 1;
    std::vector<float> X((size_t)k * MLP_IN);
    for (int i = 0; i < k; i++) {
        for (int j = 0; j < MLP_IN - 1; j++) X[i * MLP_IN + j] = features[j];
        X[i * MLP_IN + MLP_IN - 1] = (float)(c_min + i - 12) / 8.f;
    }
    float* dX = scratch;  // k * MLP_IN <= 19 * 10 floats
    float* dy = scratch + 19 * MLP_IN;
    if (cudaMemcpyAsync(dX, X.data(), X.size() * sizeof(float), cudaMemcpyHostToDevice, stream) != cudaSuccess)
        return -1;
    if (zkp_mlp_forward(params, dX, (uint32_t)k, dy, stream) != cudaSuccess) return -1;
    std::vector<float> y(k);
    if (cudaMemcpyAsync(y.data(), dy, k * sizeof(float), cudaMemcpyDeviceToHost, stream) != cudaSuccess) return -1;
    if (cudaStreamSynchronize(stream) != cudaSuccess) return -1;
    int best = c_min;
    for (int i = 1; i < k; i++)
        if (y[i] < y[best - c_min]) best = c_min + i;
    return best;
}

}  // extern "C"
