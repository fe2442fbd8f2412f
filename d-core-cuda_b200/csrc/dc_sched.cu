// Learned maintenance scheduler: a small BF16 MLP (16 -> 64 -> 64 -> 2,
// ReLU) that predicts, from features of an update batch and of the current
// decomposition, the log of the wall time of each maintenance method
// (output 0: local kmax / row-0 update, output 1: fused re-peel).  The
// engine runs the method with the smaller prediction; either method gives
// the exact result, so the network only changes speed, never answers.
//
// No counterpart in the reference (it picks one batching mode at compile
// time, src/common.h:18-19).
//
// Kernels are hand-written: one warp per sample, weights in shared memory
// as bf16, products accumulated in fp32.  Training keeps fp32 master
// weights, accumulates fp32 gradients and applies Adam; the bf16 copy used
// by forward and backward is refreshed after every step.
#include <atomic>
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "dc_engine.cuh"
#include "dc_internal.h"

namespace dc {

extern std::atomic<unsigned long long> g_launches;

constexpr int kIn = 16, kH = 64, kOut = 2;
constexpr int kOffW1 = 0;                   // [kH][kIn]
constexpr int kOffB1 = kOffW1 + kH * kIn;   // [kH]
constexpr int kOffW2 = kOffB1 + kH;         // [kH][kH]
constexpr int kOffB2 = kOffW2 + kH * kH;    // [kH]
constexpr int kOffW3 = kOffB2 + kH;         // [kOut][kH]
constexpr int kOffB3 = kOffW3 + kOut * kH;  // [kOut]
constexpr int kNParams = kOffB3 + kOut;     // 5378
constexpr int kSchedThreads = 256;
constexpr int kSchedBwdThreads = 128;

__device__ __forceinline__ float bf(float x) { return __bfloat162float(__float2bfloat16(x)); }

__device__ void load_params(const __nv_bfloat16* w, float* s) {
    for (int i = threadIdx.x; i < kNParams; i += blockDim.x) s[i] = __bfloat162float(w[i]);
    __syncthreads();
}

// Forward of one sample by one warp; lane j owns hidden units j and j+32.
// Activations are rounded to bf16 before they feed the next layer.
__device__ __forceinline__ void fwd_warp(const float* P, const float* x, float* h1, float* h2, float* y) {
    const int lane = threadIdx.x & 31;
    float xb[kIn];
#pragma unroll
    for (int i = 0; i < kIn; ++i) xb[i] = bf(x[i]);
    for (int r = 0; r < 2; ++r) {
        int j = lane + 32 * r;
        float a = P[kOffB1 + j];
#pragma unroll
        for (int i = 0; i < kIn; ++i) a = fmaf(P[kOffW1 + j * kIn + i], xb[i], a);
        h1[j] = bf(fmaxf(a, 0.f));
    }
    __syncwarp();
    for (int r = 0; r < 2; ++r) {
        int j = lane + 32 * r;
        float a = P[kOffB2 + j];
        for (int i = 0; i < kH; ++i) a = fmaf(P[kOffW2 + j * kH + i], h1[i], a);
        h2[j] = bf(fmaxf(a, 0.f));
    }
    __syncwarp();
    for (int o = 0; o < kOut; ++o) {
        float a = P[kOffW3 + o * kH + lane] * h2[lane] + P[kOffW3 + o * kH + lane + 32] * h2[lane + 32];
#pragma unroll
        for (int s = 16; s; s >>= 1) a += __shfl_xor_sync(0xFFFFFFFFu, a, s);
        if (lane == 0) y[o] = a + P[kOffB3 + o];
    }
    __syncwarp();
}

__global__ void k_mlp_forward(const float* X, uint32_t n, const __nv_bfloat16* w, float* Y) {
    __shared__ float P[kNParams];
    __shared__ float sh1[kSchedThreads / 32][kH], sh2[kSchedThreads / 32][kH];
    load_params(w, P);
    const int wib = threadIdx.x >> 5;
    const uint32_t nw = gridDim.x * (blockDim.x >> 5);
    for (uint32_t s = blockIdx.x * (blockDim.x >> 5) + wib; s < n; s += nw)
        fwd_warp(P, X + (uint64_t)s * kIn, sh1[wib], sh2[wib], Y + (uint64_t)s * kOut);
}

// Loss = mean over (sample, output) pairs with mask 1 of (y - t)^2.
// Gradients are summed in shared memory per block, then added to G.
__global__ void k_mlp_backward(const float* X, const float* T, const uint8_t* M, uint32_t n, float inv_count,
                               const __nv_bfloat16* w, float* G, float* loss) {
    __shared__ float P[kNParams];
    __shared__ float sG[kNParams];
    __shared__ float sh1[kSchedBwdThreads / 32][kH], sh2[kSchedBwdThreads / 32][kH];
    __shared__ float sd2[kSchedBwdThreads / 32][kH];
    load_params(w, P);
    for (int i = threadIdx.x; i < kNParams; i += blockDim.x) sG[i] = 0.f;
    __syncthreads();
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const uint32_t nw = gridDim.x * (blockDim.x >> 5);
    float my_loss = 0.f;
    for (uint32_t s = blockIdx.x * (blockDim.x >> 5) + wib; s < n; s += nw) {
        const float* x = X + (uint64_t)s * kIn;
        float* h1 = sh1[wib];
        float* h2 = sh2[wib];
        float y[kOut];
        float ys[kOut];
        fwd_warp(P, x, h1, h2, ys);
        // broadcast outputs from lane 0
        for (int o = 0; o < kOut; ++o) y[o] = __shfl_sync(0xFFFFFFFFu, ys[o], 0);
        float dy[kOut];
        for (int o = 0; o < kOut; ++o) {
            bool on = M[(uint64_t)s * kOut + o] != 0;
            float diff = on ? y[o] - T[(uint64_t)s * kOut + o] : 0.f;
            dy[o] = 2.f * diff * inv_count;
            if (lane == 0) my_loss += diff * diff * inv_count;
        }
        // layer 3
        for (int r = 0; r < 2; ++r) {
            int i = lane + 32 * r;
            float d2 = 0.f;
            for (int o = 0; o < kOut; ++o) {
                atomicAdd(&sG[kOffW3 + o * kH + i], dy[o] * h2[i]);
                d2 += P[kOffW3 + o * kH + i] * dy[o];
            }
            sd2[wib][i] = h2[i] > 0.f ? d2 : 0.f;
        }
        if (lane < kOut) atomicAdd(&sG[kOffB3 + lane], dy[lane]);
        __syncwarp();
        // layer 2: gradient of W2 rows j, and d1
        for (int r = 0; r < 2; ++r) {
            int j = lane + 32 * r;
            float d = sd2[wib][j];
            if (d != 0.f) {
                for (int i = 0; i < kH; ++i) atomicAdd(&sG[kOffW2 + j * kH + i], d * h1[i]);
                atomicAdd(&sG[kOffB2 + j], d);
            }
        }
        float d1[2];
        for (int r = 0; r < 2; ++r) {
            int i = lane + 32 * r;
            float a = 0.f;
            for (int j = 0; j < kH; ++j) a += P[kOffW2 + j * kH + i] * sd2[wib][j];
            d1[r] = h1[i] > 0.f ? a : 0.f;
        }
        // layer 1
        for (int r = 0; r < 2; ++r) {
            int j = lane + 32 * r;
            if (d1[r] != 0.f) {
                for (int i = 0; i < kIn; ++i) atomicAdd(&sG[kOffW1 + j * kIn + i], d1[r] * bf(x[i]));
                atomicAdd(&sG[kOffB1 + j], d1[r]);
            }
        }
        __syncwarp();
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kNParams; i += blockDim.x)
        if (sG[i] != 0.f) atomicAdd(&G[i], sG[i]);
    if (lane == 0 && my_loss != 0.f) atomicAdd(loss, my_loss);
}

__global__ void k_adam(float* master, const float* G, float* m, float* v, __nv_bfloat16* w, float lr, float b1,
                       float b2, float eps, float c1, float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kNParams; i += gridDim.x * blockDim.x) {
        float g = G[i];
        float mi = b1 * m[i] + (1.f - b1) * g;
        float vi = b2 * v[i] + (1.f - b2) * g * g;
        m[i] = mi;
        v[i] = vi;
        float p = master[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        master[i] = p;
        w[i] = __float2bfloat16(p);
    }
}

__global__ void k_to_bf16(const float* a, __nv_bfloat16* w) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kNParams; i += gridDim.x * blockDim.x)
        w[i] = __float2bfloat16(a[i]);
}

}  // namespace dc

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct dc_sched {
    cudaStream_t stream = nullptr;
    float* master = nullptr;  // fp32 parameters
    __nv_bfloat16* w = nullptr;
    float* g = nullptr;
    float* m = nullptr;
    float* v = nullptr;
    float* loss = nullptr;
    int step = 0;
    std::vector<float> feat_mean, feat_scale;  // input normalisation (identity by default)
    std::mutex mu;  // graphs on several threads may share one scheduler
};

using namespace dc;

#define SC_CUDA(call)                                                                       \
    do {                                                                                    \
        cudaError_t _e = (call);                                                            \
        if (_e != cudaSuccess) {                                                            \
            cudaGetLastError();                                                             \
            return set_error(DC_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(_e)); \
        }                                                                                   \
    } while (0)

extern "C" int dc_sched_free(dc_sched* s) {
    if (!s) return DC_OK;
    if (s->stream) cudaStreamSynchronize(s->stream);
    cudaFree(s->master);
    cudaFree(s->w);
    cudaFree(s->g);
    cudaFree(s->m);
    cudaFree(s->v);
    cudaFree(s->loss);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return DC_OK;
}

extern "C" int dc_sched_param_count(void) { return kNParams; }

// He-style seeded initialisation (splitmix64 -> uniform).
extern "C" int dc_sched_create(uint64_t seed, dc_sched** out) {
    if (!out) return set_error(DC_ERR_INVALID, "null output");
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return set_error(DC_ERR_NO_DEVICE, "dc_sched_create: no CUDA device (no CPU fallback)");
    }
    dc_sched* s = new dc_sched();
    s->feat_mean.assign(kIn, 0.f);
    s->feat_scale.assign(kIn, 1.f);
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&s->master, 4 * kNParams) != cudaSuccess || cudaMalloc(&s->w, 2 * kNParams) != cudaSuccess ||
        cudaMalloc(&s->g, 4 * kNParams) != cudaSuccess || cudaMalloc(&s->m, 4 * kNParams) != cudaSuccess ||
        cudaMalloc(&s->v, 4 * kNParams) != cudaSuccess || cudaMalloc(&s->loss, 4) != cudaSuccess) {
        cudaGetLastError();
        dc_sched_free(s);
        return set_error(DC_ERR_NOMEM, "dc_sched_create: allocation failed");
    }
    std::vector<float> p(kNParams, 0.f);
    uint64_t x = seed ^ 0x5CEDull;
    auto uni = [&]() {
        uint64_t z = (x += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) * 0x1.0p-53 * 2.0 - 1.0;
    };
    auto fill = [&](int off, int rows, int cols) {
        double a = std::sqrt(6.0 / cols);
        for (int i = 0; i < rows * cols; ++i) p[off + i] = (float)(a * uni());
    };
    fill(kOffW1, kH, kIn);
    fill(kOffW2, kH, kH);
    fill(kOffW3, kOut, kH);
    cudaMemcpyAsync(s->master, p.data(), 4 * kNParams, cudaMemcpyHostToDevice, s->stream);
    cudaMemsetAsync(s->m, 0, 4 * kNParams, s->stream);
    cudaMemsetAsync(s->v, 0, 4 * kNParams, s->stream);
    ++g_launches;
    k_to_bf16<<<8, 256, 0, s->stream>>>(s->master, s->w);
    if (cudaStreamSynchronize(s->stream) != cudaSuccess) {
        cudaGetLastError();
        dc_sched_free(s);
        return set_error(DC_ERR_CUDA, "dc_sched_create: init failed");
    }
    *out = s;
    return DC_OK;
}

extern "C" int dc_sched_set_params(dc_sched* s, const float* p) {
    if (!s || !p) return set_error(DC_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    SC_CUDA(cudaMemcpyAsync(s->master, p, 4 * kNParams, cudaMemcpyHostToDevice, s->stream));
    ++g_launches;
    k_to_bf16<<<8, 256, 0, s->stream>>>(s->master, s->w);
    SC_CUDA(cudaStreamSynchronize(s->stream));
    return DC_OK;
}

extern "C" int dc_sched_get_params(dc_sched* s, float* p) {
    if (!s || !p) return set_error(DC_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    SC_CUDA(cudaMemcpyAsync(p, s->master, 4 * kNParams, cudaMemcpyDeviceToHost, s->stream));
    SC_CUDA(cudaStreamSynchronize(s->stream));
    return DC_OK;
}

// Input normalisation x' = (x - mean) * scale applied before the network.
extern "C" int dc_sched_set_norm(dc_sched* s, const float* mean, const float* scale) {
    if (!s || !mean || !scale) return set_error(DC_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    s->feat_mean.assign(mean, mean + kIn);
    s->feat_scale.assign(scale, scale + kIn);
    return DC_OK;
}

static int sched_upload(dc_sched* s, const float* X, uint64_t n, float** dX) {
    std::vector<float> xn((size_t)n * kIn);
    for (uint64_t i = 0; i < n; ++i)
        for (int j = 0; j < kIn; ++j) xn[i * kIn + j] = (X[i * kIn + j] - s->feat_mean[j]) * s->feat_scale[j];
    if (cudaMallocAsync(dX, 4 * (n ? n : 1) * kIn, s->stream) != cudaSuccess) {
        cudaGetLastError();
        return set_error(DC_ERR_NOMEM, "scheduler input allocation failed");
    }
    SC_CUDA(cudaMemcpyAsync(*dX, xn.data(), 4 * n * kIn, cudaMemcpyHostToDevice, s->stream));
    SC_CUDA(cudaStreamSynchronize(s->stream));
    return DC_OK;
}

extern "C" int dc_sched_predict(dc_sched* s, const float* X, uint64_t n, float* Y) {
    if (!s || (n && (!X || !Y))) return set_error(DC_ERR_INVALID, "null argument");
    if (n == 0) return DC_OK;
    std::lock_guard<std::mutex> lk(s->mu);
    float *dX = nullptr, *dY = nullptr;
    if (int rc = sched_upload(s, X, n, &dX)) return rc;
    if (cudaMallocAsync(&dY, 4 * n * kOut, s->stream) != cudaSuccess) {
        cudaGetLastError();
        cudaFreeAsync(dX, s->stream);
        return set_error(DC_ERR_NOMEM, "scheduler output allocation failed");
    }
    int blocks = (int)std::min<uint64_t>((n + 7) / 8, 1024);
    ++g_launches;
    k_mlp_forward<<<blocks, kSchedThreads, 0, s->stream>>>(dX, (uint32_t)n, s->w, dY);
    cudaError_t e = cudaMemcpyAsync(Y, dY, 4 * n * kOut, cudaMemcpyDeviceToHost, s->stream);
    cudaFreeAsync(dX, s->stream);
    cudaFreeAsync(dY, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return set_error(DC_ERR_CUDA, "dc_sched_predict: %s", cudaGetErrorString(e));
    return DC_OK;
}

// One forward + backward pass: gradient G (fp32, kNParams) and loss,
// without changing the parameters (used to check gradients).
static int sched_grad_dev(dc_sched* s, const float* dX, const float* dT, const uint8_t* dM, uint64_t n,
                          uint64_t n_on) {
    SC_CUDA(cudaMemsetAsync(s->g, 0, 4 * kNParams, s->stream));
    SC_CUDA(cudaMemsetAsync(s->loss, 0, 4, s->stream));
    int blocks = (int)std::min<uint64_t>((n + 3) / 4, 256);
    ++g_launches;
    k_mlp_backward<<<blocks, kSchedBwdThreads, 0, s->stream>>>(dX, dT, dM, (uint32_t)n, 1.f / (float)(n_on ? n_on : 1),
                                                            s->w, s->g, s->loss);
    return DC_OK;
}

struct SchedBatch {
    cudaStream_t st;
    float* X = nullptr;
    float* T = nullptr;
    uint8_t* M = nullptr;
    uint64_t n_on = 0;
    explicit SchedBatch(cudaStream_t s) : st(s) {}
    ~SchedBatch() {
        if (X) cudaFreeAsync(X, st);
        if (T) cudaFreeAsync(T, st);
        if (M) cudaFreeAsync(M, st);
        cudaStreamSynchronize(st);
    }
};

static int sched_batch(dc_sched* s, const float* X, const float* T, const uint8_t* M, uint64_t n, SchedBatch& b) {
    if (int rc = sched_upload(s, X, n, &b.X)) return rc;
    if (cudaMallocAsync(&b.T, 4 * n * kOut, s->stream) != cudaSuccess ||
        cudaMallocAsync(&b.M, n * kOut, s->stream) != cudaSuccess) {
        cudaGetLastError();
        return set_error(DC_ERR_NOMEM, "scheduler target allocation failed");
    }
    SC_CUDA(cudaMemcpyAsync(b.T, T, 4 * n * kOut, cudaMemcpyHostToDevice, s->stream));
    SC_CUDA(cudaMemcpyAsync(b.M, M, n * kOut, cudaMemcpyHostToDevice, s->stream));
    for (uint64_t i = 0; i < n * kOut; ++i) b.n_on += M[i] != 0;
    return DC_OK;
}

extern "C" int dc_sched_grad(dc_sched* s, const float* X, const float* T, const uint8_t* M, uint64_t n, float* grad,
                             float* loss) {
    if (!s || !X || !T || !M || !grad || n == 0) return set_error(DC_ERR_INVALID, "bad argument");
    std::lock_guard<std::mutex> lk(s->mu);
    SchedBatch b(s->stream);
    if (int rc = sched_batch(s, X, T, M, n, b)) return rc;
    if (int rc = sched_grad_dev(s, b.X, b.T, b.M, n, b.n_on)) return rc;
    SC_CUDA(cudaMemcpyAsync(grad, s->g, 4 * kNParams, cudaMemcpyDeviceToHost, s->stream));
    float l = 0;
    SC_CUDA(cudaMemcpyAsync(&l, s->loss, 4, cudaMemcpyDeviceToHost, s->stream));
    SC_CUDA(cudaStreamSynchronize(s->stream));
    if (loss) *loss = l;
    return DC_OK;
}

// Full-batch Adam for `epochs` steps on (X, T, M); M marks the targets that
// exist (a logged batch may have been timed with one method only).
extern "C" int dc_sched_train(dc_sched* s, const float* X, const float* T, const uint8_t* M, uint64_t n, int epochs,
                              float lr, float* final_loss) {
    if (!s || !X || !T || !M || n == 0 || epochs < 0) return set_error(DC_ERR_INVALID, "bad argument");
    std::lock_guard<std::mutex> lk(s->mu);
    SchedBatch b(s->stream);
    if (int rc = sched_batch(s, X, T, M, n, b)) return rc;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int ep = 0; ep < epochs; ++ep) {
        if (int rc = sched_grad_dev(s, b.X, b.T, b.M, n, b.n_on)) return rc;
        ++s->step;
        float c1 = 1.f - std::pow(b1, (float)s->step), c2 = 1.f - std::pow(b2, (float)s->step);
        ++g_launches;
        k_adam<<<22, 256, 0, s->stream>>>(s->master, s->g, s->m, s->v, s->w, lr, b1, b2, eps, c1, c2);
    }
    if (final_loss) {
        if (int rc = sched_grad_dev(s, b.X, b.T, b.M, n, b.n_on)) return rc;
        SC_CUDA(cudaMemcpyAsync(final_loss, s->loss, 4, cudaMemcpyDeviceToHost, s->stream));
    }
    SC_CUDA(cudaStreamSynchronize(s->stream));
    return DC_OK;
}

// Scheduler of a graph handle (DC_MAINT_AUTO): predict with the network when
// one is attached, else the rule of thumb.
namespace dc {
int sched_choose(dc_sched* s, const float* feat) {
    float y[kOut];
    if (dc_sched_predict(s, feat, 1, y) != DC_OK) return -1;
    return y[0] <= y[1] ? DC_MAINT_LOCAL : DC_MAINT_REPEEL;
}
}  // namespace dc
