// Learned sizer: a 16 -> 64 -> 64 -> 64 -> 2 MLP (ReLU hidden layers,
// linear output) with BF16 weights and FP32 accumulation, trained on the GPU
// by the kernels below (fused forward + backward per 32-sample tile, Adam
// update of FP32 master weights that re-quantises the BF16 copy). It
// predicts (log2 group cardinality / 24, filter selectivity) from 16
// features of a query, replacing the exact count pass that sizes hash
// tables; see gpudb_batch.h.
//
// Parameter layout (9,538 floats): W1[64][16] b1[64] W2[64][64] b2[64]
// W3[64][64] b3[64] W4[2][64] b4[2] — weights out-major.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "../../../include/gpudb_batch.h"

namespace gpudb {
void setThreadError(const std::string& message);
}

namespace {

constexpr int kIn = 16, kH = 64, kOut = 2;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kH * kIn, kOffW2 = kOffB1 + kH, kOffB2 = kOffW2 + kH * kH,
              kOffW3 = kOffB2 + kH, kOffB3 = kOffW3 + kH * kH, kOffW4 = kOffB3 + kH, kOffB4 = kOffW4 + kOut * kH,
              kParams = kOffB4 + kOut;
static_assert(kParams == 9538, "parameter count");
constexpr int kTile = 32;      // samples per CTA
constexpr int kThreads = 256;  // threads per CTA

// out[s][j] = b[j] + sum_k W[j][k] * in[s][k]   (optionally ReLU)
template <int NI, int NO>
__device__ void dense(const __nv_bfloat16* W, const __nv_bfloat16* b, const float* in, float* out, int ns, bool relu) {
    for (int e = threadIdx.x; e < ns * NO; e += blockDim.x) {
        const int s = e / NO, j = e % NO;
        float acc = __bfloat162float(b[j]);
#pragma unroll 8
        for (int k = 0; k < NI; ++k) acc = fmaf(__bfloat162float(W[j * NI + k]), in[s * NI + k], acc);
        out[e] = relu ? fmaxf(acc, 0.0f) : acc;
    }
}

// dIn[s][k] = (sum_j dOut[s][j] * W[j][k]) * (act[s][k] > 0 when masked)
template <int NI, int NO>
__device__ void backIn(const __nv_bfloat16* W, const float* dOut, const float* act, float* dIn, int ns, bool mask) {
    for (int e = threadIdx.x; e < ns * NI; e += blockDim.x) {
        const int s = e / NI, k = e % NI;
        float acc = 0.0f;
#pragma unroll 8
        for (int j = 0; j < NO; ++j) acc = fmaf(dOut[s * NO + j], __bfloat162float(W[j * NI + k]), acc);
        dIn[e] = (mask && act[e] <= 0.0f) ? 0.0f : acc;
    }
}

// gW[j][k] += sum_s dOut[s][j] * in[s][k]; gb[j] += sum_s dOut[s][j]
template <int NI, int NO>
__device__ void backW(const float* dOut, const float* in, float* gW, float* gb, int ns) {
    for (int e = threadIdx.x; e < NO * NI; e += blockDim.x) {
        const int j = e / NI, k = e % NI;
        float acc = 0.0f;
        for (int s = 0; s < ns; ++s) acc = fmaf(dOut[s * NO + j], in[s * NI + k], acc);
        atomicAdd(gW + e, acc);
    }
    for (int j = threadIdx.x; j < NO; j += blockDim.x) {
        float acc = 0.0f;
        for (int s = 0; s < ns; ++s) acc += dOut[s * NO + j];
        atomicAdd(gb + j, acc);
    }
}

struct Smem {
    __nv_bfloat16 w[kParams];
    float x[kTile * kIn];
    float h1[kTile * kH], h2[kTile * kH], h3[kTile * kH];
    float y[kTile * kOut];
    float d3[kTile * kH], d2[kTile * kH];
    float dy[kTile * kOut];
};

__device__ void loadWeights(Smem& sm, const __nv_bfloat16* wbf) {
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) sm.w[i] = wbf[i];
}

__device__ void forwardTile(Smem& sm, int ns) {
    dense<kIn, kH>(sm.w + kOffW1, sm.w + kOffB1, sm.x, sm.h1, ns, true);
    __syncthreads();
    dense<kH, kH>(sm.w + kOffW2, sm.w + kOffB2, sm.h1, sm.h2, ns, true);
    __syncthreads();
    dense<kH, kH>(sm.w + kOffW3, sm.w + kOffB3, sm.h2, sm.h3, ns, true);
    __syncthreads();
    dense<kH, kOut>(sm.w + kOffW4, sm.w + kOffB4, sm.h3, sm.y, ns, false);
    __syncthreads();
}

// Forward + backward of one tile of samples; gradients of the mean squared
// error over `total` samples x 2 outputs accumulate into `grad`.
__global__ void __launch_bounds__(kThreads) mlpTrainStep(const __nv_bfloat16* __restrict__ wbf,
                                                         const float* __restrict__ X, const float* __restrict__ Y,
                                                         int n, int total, float* __restrict__ grad,
                                                         float* __restrict__ loss) {
    extern __shared__ __align__(16) unsigned char smraw[];
    Smem& sm = *reinterpret_cast<Smem*>(smraw);
    const int s0 = blockIdx.x * kTile;
    const int ns = min(kTile, n - s0);
    if (ns <= 0) return;
    loadWeights(sm, wbf);
    for (int i = threadIdx.x; i < ns * kIn; i += blockDim.x) sm.x[i] = X[(long long)s0 * kIn + i];
    __syncthreads();
    forwardTile(sm, ns);
    const float scale = 2.0f / (float)(total * kOut);
    float l = 0.0f;
    for (int e = threadIdx.x; e < ns * kOut; e += blockDim.x) {
        const float diff = sm.y[e] - Y[(long long)s0 * kOut + e];
        sm.dy[e] = diff * scale;
        l += diff * diff;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0 && l != 0.0f) atomicAdd(loss, l / (float)(total * kOut));
    __syncthreads();
    backW<kH, kOut>(sm.dy, sm.h3, grad + kOffW4, grad + kOffB4, ns);
    backIn<kH, kOut>(sm.w + kOffW4, sm.dy, sm.h3, sm.d3, ns, true);
    __syncthreads();
    backW<kH, kH>(sm.d3, sm.h2, grad + kOffW3, grad + kOffB3, ns);
    backIn<kH, kH>(sm.w + kOffW3, sm.d3, sm.h2, sm.d2, ns, true);
    __syncthreads();
    backW<kH, kH>(sm.d2, sm.h1, grad + kOffW2, grad + kOffB2, ns);
    backIn<kH, kH>(sm.w + kOffW2, sm.d2, sm.h1, sm.d3, ns, true);  // d3 now holds dH1
    __syncthreads();
    backW<kIn, kH>(sm.d3, sm.x, grad + kOffW1, grad + kOffB1, ns);
}

__global__ void __launch_bounds__(kThreads) mlpPredict(const __nv_bfloat16* __restrict__ wbf,
                                                       const float* __restrict__ X, int n, float* __restrict__ Yout) {
    extern __shared__ __align__(16) unsigned char smraw[];
    Smem& sm = *reinterpret_cast<Smem*>(smraw);
    const int s0 = blockIdx.x * kTile;
    const int ns = min(kTile, n - s0);
    if (ns <= 0) return;
    loadWeights(sm, wbf);
    for (int i = threadIdx.x; i < ns * kIn; i += blockDim.x) sm.x[i] = X[(long long)s0 * kIn + i];
    __syncthreads();
    forwardTile(sm, ns);
    for (int e = threadIdx.x; e < ns * kOut; e += blockDim.x) Yout[(long long)s0 * kOut + e] = sm.y[e];
}

// Adam on the FP32 master weights; refreshes the BF16 copy; clears grads.
__global__ void adamStep(float* __restrict__ w, __nv_bfloat16* __restrict__ wbf, float* __restrict__ m,
                         float* __restrict__ v, float* __restrict__ grad, float lr, float b1, float b2, float eps,
                         float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams) return;
    const float g = grad[i];
    const float mi = b1 * m[i] + (1.0f - b1) * g;
    const float vi = b2 * v[i] + (1.0f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    wbf[i] = __float2bfloat16_rn(wi);
    grad[i] = 0.0f;
}

__global__ void quantize(const float* __restrict__ w, __nv_bfloat16* __restrict__ wbf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kParams) wbf[i] = __float2bfloat16_rn(w[i]);
}

#define SZ_CHECK(call, code)                                                                        \
    do {                                                                                            \
        const cudaError_t _e = (call);                                                              \
        if (_e != cudaSuccess) {                                                                    \
            gpudb::setThreadError(std::string("sizer: ") + #call + ": " + cudaGetErrorString(_e)); \
            return code;                                                                            \
        }                                                                                           \
    } while (0)

}  // namespace

struct gpudb_sizer {
    int device = 0;
    cudaStream_t stream = nullptr;
    float *w = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr, *loss = nullptr;
    __nv_bfloat16* wbf = nullptr;
    float *X = nullptr, *Y = nullptr;
    int cap = 0;  // samples X/Y can hold
    long long step = 0;
};

namespace {

int ensureCapacity(gpudb_sizer* s, int n) {
    if (n <= s->cap) return GPUDB_OK;
    if (s->X) cudaFree(s->X);
    if (s->Y) cudaFree(s->Y);
    s->X = s->Y = nullptr;
    SZ_CHECK(cudaMalloc(&s->X, sizeof(float) * (size_t)n * kIn), GPUDB_E_ALLOC);
    SZ_CHECK(cudaMalloc(&s->Y, sizeof(float) * (size_t)n * kOut), GPUDB_E_ALLOC);
    s->cap = n;
    return GPUDB_OK;
}

int launchTrain(gpudb_sizer* s, const float* X, const float* Y, int n, int total) {
    const int blocks = (n + kTile - 1) / kTile;
    mlpTrainStep<<<blocks, kThreads, sizeof(Smem), s->stream>>>(s->wbf, X, Y, n, total, s->grad, s->loss);
    SZ_CHECK(cudaGetLastError(), GPUDB_E_LAUNCH);
    return GPUDB_OK;
}

}  // namespace

extern "C" {

int gpudb_sizer_create(int device, uint64_t seed, gpudb_sizer** out) {
    if (!out) return GPUDB_E_INVALID;
    *out = nullptr;
    auto s = std::make_unique<gpudb_sizer>();
    s->device = device;
    SZ_CHECK(cudaSetDevice(device), GPUDB_E_NOGPU);
    SZ_CHECK(cudaFuncSetAttribute(mlpTrainStep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem)),
             GPUDB_E_LAUNCH);
    SZ_CHECK(cudaFuncSetAttribute(mlpPredict, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem)),
             GPUDB_E_LAUNCH);
    SZ_CHECK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), GPUDB_E_CUDA);
    SZ_CHECK(cudaMalloc(&s->w, sizeof(float) * kParams), GPUDB_E_ALLOC);
    SZ_CHECK(cudaMalloc(&s->m, sizeof(float) * kParams), GPUDB_E_ALLOC);
    SZ_CHECK(cudaMalloc(&s->v, sizeof(float) * kParams), GPUDB_E_ALLOC);
    SZ_CHECK(cudaMalloc(&s->grad, sizeof(float) * kParams), GPUDB_E_ALLOC);
    SZ_CHECK(cudaMalloc(&s->loss, sizeof(float)), GPUDB_E_ALLOC);
    SZ_CHECK(cudaMalloc(&s->wbf, sizeof(__nv_bfloat16) * kParams), GPUDB_E_ALLOC);
    // He-uniform initialisation on the host (seeded), biases zero
    std::vector<float> w(kParams, 0.0f);
    std::mt19937_64 rng(seed);
    auto init = [&](int off, int fanIn, int count) {
        const float lim = std::sqrt(6.0f / (float)fanIn);
        std::uniform_real_distribution<float> u(-lim, lim);
        for (int i = 0; i < count; i++) w[off + i] = u(rng);
    };
    init(kOffW1, kIn, kH * kIn);
    init(kOffW2, kH, kH * kH);
    init(kOffW3, kH, kH * kH);
    init(kOffW4, kH, kOut * kH);
    SZ_CHECK(cudaMemcpy(s->w, w.data(), sizeof(float) * kParams, cudaMemcpyHostToDevice), GPUDB_E_CUDA);
    SZ_CHECK(cudaMemset(s->m, 0, sizeof(float) * kParams), GPUDB_E_CUDA);
    SZ_CHECK(cudaMemset(s->v, 0, sizeof(float) * kParams), GPUDB_E_CUDA);
    SZ_CHECK(cudaMemset(s->grad, 0, sizeof(float) * kParams), GPUDB_E_CUDA);
    quantize<<<(kParams + 255) / 256, 256, 0, s->stream>>>(s->w, s->wbf);
    SZ_CHECK(cudaStreamSynchronize(s->stream), GPUDB_E_CUDA);
    *out = s.release();
    return GPUDB_OK;
}

void gpudb_sizer_free(gpudb_sizer* s) {
    if (!s) return;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (void* p : {(void*)s->w, (void*)s->m, (void*)s->v, (void*)s->grad, (void*)s->loss, (void*)s->wbf, (void*)s->X,
                    (void*)s->Y})
        if (p) cudaFree(p);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

int gpudb_sizer_param_count(void) { return kParams; }

int gpudb_sizer_get_params(gpudb_sizer* s, float* out) {
    if (!s || !out) return GPUDB_E_INVALID;
    cudaSetDevice(s->device);
    SZ_CHECK(cudaMemcpyAsync(out, s->w, sizeof(float) * kParams, cudaMemcpyDeviceToHost, s->stream), GPUDB_E_CUDA);
    SZ_CHECK(cudaStreamSynchronize(s->stream), GPUDB_E_CUDA);
    return GPUDB_OK;
}

int gpudb_sizer_set_params(gpudb_sizer* s, const float* in) {
    if (!s || !in) return GPUDB_E_INVALID;
    cudaSetDevice(s->device);
    SZ_CHECK(cudaMemcpyAsync(s->w, in, sizeof(float) * kParams, cudaMemcpyHostToDevice, s->stream), GPUDB_E_CUDA);
    quantize<<<(kParams + 255) / 256, 256, 0, s->stream>>>(s->w, s->wbf);
    SZ_CHECK(cudaStreamSynchronize(s->stream), GPUDB_E_CUDA);
    return GPUDB_OK;
}

int gpudb_sizer_grads(gpudb_sizer* s, const float* X, const float* Y, int n, float* grads_out, float* loss_out) {
    if (!s || !X || !Y || n <= 0 || !grads_out) return GPUDB_E_INVALID;
    cudaSetDevice(s->device);
    if (int st = ensureCapacity(s, n)) return st;
    SZ_CHECK(cudaMemcpyAsync(s->X, X, sizeof(float) * (size_t)n * kIn, cudaMemcpyHostToDevice, s->stream), GPUDB_E_CUDA);
    SZ_CHECK(cudaMemcpyAsync(s->Y, Y, sizeof(float) * (size_t)n * kOut, cudaMemcpyHostToDevice, s->stream),
             GPUDB_E_CUDA);
    SZ_CHECK(cudaMemsetAsync(s->grad, 0, sizeof(float) * kParams, s->stream), GPUDB_E_CUDA);
    SZ_CHECK(cudaMemsetAsync(s->loss, 0, sizeof(float), s->stream), GPUDB_E_CUDA);
    if (int st = launchTrain(s, s->X, s->Y, n, n)) return st;
    SZ_CHECK(cudaMemcpyAsync(grads_out, s->grad, sizeof(float) * kParams, cudaMemcpyDeviceToHost, s->stream),
             GPUDB_E_CUDA);
    float l = 0;
    SZ_CHECK(cudaMemcpyAsync(&l, s->loss, sizeof(float), cudaMemcpyDeviceToHost, s->stream), GPUDB_E_CUDA);
    SZ_CHECK(cudaMemsetAsync(s->grad, 0, sizeof(float) * kParams, s->stream), GPUDB_E_CUDA);
    SZ_CHECK(cudaStreamSynchronize(s->stream), GPUDB_E_CUDA);
    if (loss_out) *loss_out = l;
    return GPUDB_OK;
}

int gpudb_sizer_train(gpudb_sizer* s, const float* X, const float* Y, int n, int epochs, int batch, float lr,
                      uint64_t seed, float* final_loss) {
    if (!s || !X || !Y || n <= 0 || epochs <= 0 || batch <= 0) return GPUDB_E_INVALID;
    cudaSetDevice(s->device);
    if (int st = ensureCapacity(s, n)) return st;
    // shuffle once per epoch on the host, upload the permuted set
    std::vector<int> idx(n);
    for (int i = 0; i < n; i++) idx[i] = i;
    std::mt19937_64 rng(seed);
    std::vector<float> px((size_t)n * kIn), py((size_t)n * kOut);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const long long totalSteps = (long long)epochs * ((n + batch - 1) / batch);
    long long runStep = 0;
    float last = 0.0f;
    for (int ep = 0; ep < epochs; ep++) {
        std::shuffle(idx.begin(), idx.end(), rng);
        for (int i = 0; i < n; i++) {
            std::copy(X + (size_t)idx[i] * kIn, X + (size_t)idx[i] * kIn + kIn, px.begin() + (size_t)i * kIn);
            std::copy(Y + (size_t)idx[i] * kOut, Y + (size_t)idx[i] * kOut + kOut, py.begin() + (size_t)i * kOut);
        }
        SZ_CHECK(cudaMemcpyAsync(s->X, px.data(), sizeof(float) * px.size(), cudaMemcpyHostToDevice, s->stream),
                 GPUDB_E_CUDA);
        SZ_CHECK(cudaMemcpyAsync(s->Y, py.data(), sizeof(float) * py.size(), cudaMemcpyHostToDevice, s->stream),
                 GPUDB_E_CUDA);
        SZ_CHECK(cudaMemsetAsync(s->loss, 0, sizeof(float), s->stream), GPUDB_E_CUDA);
        int nb = 0;
        for (int off = 0; off < n; off += batch, nb++) {
            const int cur = std::min(batch, n - off);
            if (int st = launchTrain(s, s->X + (size_t)off * kIn, s->Y + (size_t)off * kOut, cur, cur)) return st;
            s->step++;
            const float c1 = 1.0f - std::pow(b1, (float)s->step), c2 = 1.0f - std::pow(b2, (float)s->step);
            // cosine decay of the learning rate over this call's steps
            const float lrNow =
                totalSteps > 1 ? lr * 0.5f * (1.0f + std::cos(3.14159265358979f * (float)runStep / (float)totalSteps))
                               : lr;
            runStep++;
            adamStep<<<(kParams + 255) / 256, 256, 0, s->stream>>>(s->w, s->wbf, s->m, s->v, s->grad, lrNow, b1, b2,
                                                                    eps, c1, c2);
        }
        SZ_CHECK(cudaGetLastError(), GPUDB_E_LAUNCH);
        float l = 0;
        SZ_CHECK(cudaMemcpyAsync(&l, s->loss, sizeof(float), cudaMemcpyDeviceToHost, s->stream), GPUDB_E_CUDA);
        SZ_CHECK(cudaStreamSynchronize(s->stream), GPUDB_E_CUDA);
        last = nb ? l / (float)nb : 0.0f;  // mean of the batches' losses
    }
    if (final_loss) *final_loss = last;
    return GPUDB_OK;
}

int gpudb_sizer_predict(gpudb_sizer* s, const float* X, int n, float* Y_out) {
    if (!s || !X || n < 0 || (n && !Y_out)) return GPUDB_E_INVALID;
    if (n == 0) return GPUDB_OK;
    cudaSetDevice(s->device);
    if (int st = ensureCapacity(s, n)) return st;
    SZ_CHECK(cudaMemcpyAsync(s->X, X, sizeof(float) * (size_t)n * kIn, cudaMemcpyHostToDevice, s->stream), GPUDB_E_CUDA);
    mlpPredict<<<(n + kTile - 1) / kTile, kThreads, sizeof(Smem), s->stream>>>(s->wbf, s->X, n, s->Y);
    SZ_CHECK(cudaGetLastError(), GPUDB_E_LAUNCH);
    SZ_CHECK(cudaMemcpyAsync(Y_out, s->Y, sizeof(float) * (size_t)n * kOut, cudaMemcpyDeviceToHost, s->stream),
             GPUDB_E_CUDA);
    SZ_CHECK(cudaStreamSynchronize(s->stream), GPUDB_E_CUDA);
    return GPUDB_OK;
}

}  // extern "C"
