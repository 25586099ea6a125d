// The learned lookahead proposal: a 32 -> 64 -> 64 -> 1 MLP (ReLU, ReLU, sigmoid) with
// BF16 weights and FP32 accumulation, trained on the GPU by the kernels below.
//
// It scores a search node before its head-union-tail lookahead is issued: the
// probability that head + tail is frequent.  The engine uses the score only to decide
// which exact checks run first; every support is still counted exactly, so the MFI
// output does not depend on the network.  (The reference has no learned component.)
//
// Parameters: FP32 master copy (updated by Adam) and a BF16 copy of the weight matrices
// that the forward pass reads.  Layout of the FP32 vector (kMlpParams floats):
//   W1[64][32], b1[64], W2[64][64], b2[64], W3[64], b3[1]
// Loss: mean over the batch of w_s * BCE(sigmoid(z_s), y_s), w_s = pos_weight for y=1.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <vector>

#include <atomic>

#include "tfim_internal.h"

namespace tfim {

constexpr int kIn = 32, kH = 64;
constexpr int oW1 = 0, oB1 = oW1 + kH * kIn, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH, oB3 = oW3 + kH;
constexpr int kMlpParams = oB3 + 1;   // 6337
constexpr int kBlk = 64;              // samples per block in the backward pass

struct Mlp {
    int device = 0;
    cudaStream_t stream = nullptr;
    float* d_params = nullptr;        // FP32 master
    float* d_grads = nullptr;
    float* d_m = nullptr;
    float* d_v = nullptr;
    __nv_bfloat16* d_wbf = nullptr;   // BF16 copies of W1, W2, W3 (same offsets, biases unused)
    int64_t step = 0;
    DevBuf d_x, d_y, d_out, d_loss;
};

namespace {

__device__ __forceinline__ float bf(const __nv_bfloat16* w, int i) { return __bfloat162float(w[i]); }

// One thread per sample.
__global__ void k_mlp_forward(const float* __restrict__ X, int64_t n, const __nv_bfloat16* __restrict__ wbf,
                              const float* __restrict__ P, float* __restrict__ out) {
    __shared__ float sW1[kH * kIn], sW2[kH * kH], sW3[kH], sb1[kH], sb2[kH];
    for (int i = threadIdx.x; i < kH * kIn; i += blockDim.x) sW1[i] = bf(wbf, oW1 + i);
    for (int i = threadIdx.x; i < kH * kH; i += blockDim.x) sW2[i] = bf(wbf, oW2 + i);
    for (int i = threadIdx.x; i < kH; i += blockDim.x) {
        sW3[i] = bf(wbf, oW3 + i);
        sb1[i] = P[oB1 + i];
        sb2[i] = P[oB2 + i];
    }
    __syncthreads();
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= n) return;
    float x[kIn], h1[kH];
#pragma unroll
    for (int i = 0; i < kIn; i++) x[i] = X[s * kIn + i];
    for (int j = 0; j < kH; j++) {
        float a = sb1[j];
#pragma unroll
        for (int i = 0; i < kIn; i++) a = fmaf(sW1[j * kIn + i], x[i], a);
        h1[j] = fmaxf(a, 0.f);
    }
    float z = P[oB3];
    for (int j = 0; j < kH; j++) {
        float a = sb2[j];
#pragma unroll 8
        for (int k = 0; k < kH; k++) a = fmaf(sW2[j * kH + k], h1[k], a);
        z = fmaf(sW3[j], fmaxf(a, 0.f), z);
    }
    out[s] = 1.f / (1.f + expf(-z));
}

// Block of kBlk samples: forward, backward per sample into shared memory, then the block's
// gradient sums (dot products over its samples), added to the global gradient.
__global__ void __launch_bounds__(kBlk) k_mlp_backward(const float* __restrict__ X, const float* __restrict__ Y, int64_t n,
                                                       const __nv_bfloat16* __restrict__ wbf, const float* __restrict__ P,
                                                       float pos_weight, float inv_n, float* __restrict__ G,
                                                       float* __restrict__ loss) {
    extern __shared__ float sh[];
    float* sW1 = sh;                       // kH*kIn
    float* sW2 = sW1 + kH * kIn;           // kH*kH
    float* sW3 = sW2 + kH * kH;            // kH
    float* sx = sW3 + kH;                  // kBlk*kIn
    float* sh1 = sx + kBlk * kIn;          // kBlk*kH
    float* sh2 = sh1 + kBlk * kH;          // kBlk*kH
    float* sd2 = sh2 + kBlk * kH;          // kBlk*kH  (dL/d pre-activation 2)
    float* sd1 = sd2 + kBlk * kH;          // kBlk*kH  (dL/d pre-activation 1)
    float* sdz = sd1 + kBlk * kH;          // kBlk
    for (int i = threadIdx.x; i < kH * kIn; i += blockDim.x) sW1[i] = bf(wbf, oW1 + i);
    for (int i = threadIdx.x; i < kH * kH; i += blockDim.x) sW2[i] = bf(wbf, oW2 + i);
    for (int i = threadIdx.x; i < kH; i += blockDim.x) sW3[i] = bf(wbf, oW3 + i);
    __syncthreads();
    const int t = threadIdx.x;
    const int64_t s = blockIdx.x * (int64_t)kBlk + t;
    const bool live = s < n;
    float* x = sx + t * kIn;
    float* h1 = sh1 + t * kH;
    float* h2 = sh2 + t * kH;
    float* d2 = sd2 + t * kH;
    float* d1 = sd1 + t * kH;
    for (int i = 0; i < kIn; i++) x[i] = live ? X[s * kIn + i] : 0.f;
    for (int j = 0; j < kH; j++) {
        float a = P[oB1 + j];
        for (int i = 0; i < kIn; i++) a = fmaf(sW1[j * kIn + i], x[i], a);
        h1[j] = fmaxf(a, 0.f);
    }
    float z = P[oB3];
    for (int j = 0; j < kH; j++) {
        float a = P[oB2 + j];
        for (int k = 0; k < kH; k++) a = fmaf(sW2[j * kH + k], h1[k], a);
        h2[j] = fmaxf(a, 0.f);
        z = fmaf(sW3[j], h2[j], z);
    }
    float dz = 0.f;
    if (live) {
        const float y = Y[s];
        const float p = 1.f / (1.f + expf(-z));
        const float w = y > 0.5f ? pos_weight : 1.f;
        dz = w * (p - y) * inv_n;
        // numerically stable BCE with logits
        const float l = fmaxf(z, 0.f) - z * y + log1pf(expf(-fabsf(z)));
        atomicAdd(loss, w * l * inv_n);
    }
    sdz[t] = dz;
    for (int j = 0; j < kH; j++) d2[j] = h2[j] > 0.f ? dz * sW3[j] : 0.f;
    for (int k = 0; k < kH; k++) {
        float a = 0.f;
        for (int j = 0; j < kH; j++) a = fmaf(sW2[j * kH + k], d2[j], a);
        d1[k] = h1[k] > 0.f ? a : 0.f;
    }
    __syncthreads();
    // block sums: thread t handles parameter indices t, t+kBlk, ...
    for (int idx = t; idx < kMlpParams; idx += kBlk) {
        float g = 0.f;
        if (idx < oB1) {                       // W1[j][i] = sum_s d1[s][j] x[s][i]
            const int j = idx / kIn, i = idx % kIn;
            for (int q = 0; q < kBlk; q++) g = fmaf(sd1[q * kH + j], sx[q * kIn + i], g);
        } else if (idx < oW2) {                // b1[j]
            const int j = idx - oB1;
            for (int q = 0; q < kBlk; q++) g += sd1[q * kH + j];
        } else if (idx < oB2) {                // W2[j][k] = sum_s d2[s][j] h1[s][k]
            const int j = (idx - oW2) / kH, k = (idx - oW2) % kH;
            for (int q = 0; q < kBlk; q++) g = fmaf(sd2[q * kH + j], sh1[q * kH + k], g);
        } else if (idx < oW3) {                // b2[j]
            const int j = idx - oB2;
            for (int q = 0; q < kBlk; q++) g += sd2[q * kH + j];
        } else if (idx < oB3) {                // W3[k] = sum_s dz[s] h2[s][k]
            const int k = idx - oW3;
            for (int q = 0; q < kBlk; q++) g = fmaf(sdz[q], sh2[q * kH + k], g);
        } else {                               // b3
            for (int q = 0; q < kBlk; q++) g += sdz[q];
        }
        if (g != 0.f) atomicAdd(G + idx, g);
    }
}

__global__ void k_mlp_adam(float* __restrict__ P, const float* __restrict__ G, float* __restrict__ M, float* __restrict__ V,
                           __nv_bfloat16* __restrict__ wbf, float lr, float b1, float b2, float eps, float c1, float c2,
                           float wd) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kMlpParams) return;
    const float g = G[i];
    const float m = b1 * M[i] + (1.f - b1) * g;
    const float v = b2 * V[i] + (1.f - b2) * g * g;
    M[i] = m;
    V[i] = v;
    const bool is_w = (i < oB1) || (i >= oW2 && i < oB2) || (i >= oW3 && i < oB3);
    float p = P[i] - lr * ((m / c1) / (sqrtf(v / c2) + eps) + (is_w ? wd * P[i] : 0.f));
    P[i] = p;
    wbf[i] = __float2bfloat16(p);
}

__global__ void k_mlp_cast(const float* __restrict__ P, __nv_bfloat16* __restrict__ wbf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kMlpParams) wbf[i] = __float2bfloat16(P[i]);
}

size_t backward_smem() {
    return sizeof(float) * (size_t)(kH * kIn + kH * kH + kH + kBlk * kIn + 4 * kBlk * kH + kBlk);
}

}  // namespace

int mlp_predict_device(Mlp* m, const float* d_x, int64_t n, float* d_out, cudaStream_t s) {
    if (n <= 0) return TFIM_OK;
    k_mlp_forward<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(d_x, n, m->d_wbf, m->d_params, d_out);
    TFIM_CUDA(cudaGetLastError());
    return TFIM_OK;
}

int mlp_grad_device(Mlp* m, const float* d_x, const float* d_y, int64_t n, float pos_weight, float* d_loss,
                    cudaStream_t s) {
    TFIM_CUDA(cudaMemsetAsync(m->d_grads, 0, sizeof(float) * kMlpParams, s));
    if (n <= 0) return TFIM_OK;
    static std::atomic<bool> configured[64];   // the attribute is per device
    const size_t smem = backward_smem();
    int dev = 0;
    TFIM_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64 || !configured[dev].load()) {
        TFIM_CUDA(cudaFuncSetAttribute(k_mlp_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        if (dev >= 0 && dev < 64) configured[dev].store(true);
    }
    k_mlp_backward<<<(unsigned)((n + kBlk - 1) / kBlk), kBlk, smem, s>>>(d_x, d_y, n, m->d_wbf, m->d_params, pos_weight,
                                                                        1.0f / (float)n, m->d_grads, d_loss);
    TFIM_CUDA(cudaGetLastError());
    return TFIM_OK;
}

int mlp_device_params(tfim_mlp* h, const void** wbf, const float** params) {
    Mlp* m = (Mlp*)h;
    TFIM_CHECK(m, TFIM_E_INVALID, "null network");
    *wbf = m->d_wbf;
    *params = m->d_params;
    return TFIM_OK;
}

}  // namespace tfim

using namespace tfim;

extern "C" {

int tfim_mlp_create(int32_t device, uint64_t seed, tfim_mlp** out) {
    TFIM_CHECK(out, TFIM_E_INVALID, "null output");
    *out = nullptr;
    TFIM_CUDA(cudaSetDevice(device));
    Mlp* m = new (std::nothrow) Mlp();
    TFIM_CHECK(m, TFIM_E_NOMEM, "allocation failed");
    m->device = device;
    if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) { delete m; TFIM_CHECK(false, TFIM_E_CUDA, "stream creation failed"); }
    for (DevBuf* b : {&m->d_x, &m->d_y, &m->d_out, &m->d_loss}) b->stream = m->stream;
    int rc = TFIM_OK;
    if ((rc = dev_alloc((void**)&m->d_params, sizeof(float) * kMlpParams, m->stream)) ||
        (rc = dev_alloc((void**)&m->d_grads, sizeof(float) * kMlpParams, m->stream)) ||
        (rc = dev_alloc((void**)&m->d_m, sizeof(float) * kMlpParams, m->stream)) ||
        (rc = dev_alloc((void**)&m->d_v, sizeof(float) * kMlpParams, m->stream)) ||
        (rc = dev_alloc((void**)&m->d_wbf, sizeof(__nv_bfloat16) * kMlpParams, m->stream))) {
        tfim_mlp_free((tfim_mlp*)m);
        return rc;
    }
    // He-style initialisation from a splitmix64 stream (deterministic per seed)
    std::vector<float> p(kMlpParams, 0.f);
    uint64_t st = seed ^ 0x9E3779B97F4A7C15ull;
    auto uni = [&]() {
        st += 0x9E3779B97F4A7C15ull;
        uint64_t z = st;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) / 9007199254740992.0;   // [0, 1)
    };
    auto fill = [&](int off, int n, int fan_in) {
        const double a = std::sqrt(6.0 / fan_in);
        for (int i = 0; i < n; i++) p[off + i] = (float)((uni() * 2.0 - 1.0) * a);
    };
    fill(oW1, kH * kIn, kIn);
    fill(oW2, kH * kH, kH);
    fill(oW3, kH, kH);
    int r2 = tfim_mlp_set_params((tfim_mlp*)m, p.data());
    if (r2) { tfim_mlp_free((tfim_mlp*)m); return r2; }
    *out = (tfim_mlp*)m;
    return TFIM_OK;
}

int tfim_mlp_num_params(void) { return kMlpParams; }

int tfim_mlp_set_params(tfim_mlp* h, const float* params) {
    Mlp* m = (Mlp*)h;
    TFIM_CHECK(m && params, TFIM_E_INVALID, "null argument");
    TFIM_CUDA(cudaSetDevice(m->device));
    TFIM_CUDA(cudaMemcpyAsync(m->d_params, params, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice, m->stream));
    TFIM_CUDA(cudaMemsetAsync(m->d_m, 0, sizeof(float) * kMlpParams, m->stream));
    TFIM_CUDA(cudaMemsetAsync(m->d_v, 0, sizeof(float) * kMlpParams, m->stream));
    k_mlp_cast<<<(kMlpParams + 255) / 256, 256, 0, m->stream>>>(m->d_params, m->d_wbf);
    TFIM_CUDA(cudaGetLastError());
    TFIM_CUDA(cudaStreamSynchronize(m->stream));
    m->step = 0;
    return TFIM_OK;
}

int tfim_mlp_get_params(const tfim_mlp* h, float* params) {
    const Mlp* m = (const Mlp*)h;
    TFIM_CHECK(m && params, TFIM_E_INVALID, "null argument");
    TFIM_CUDA(cudaSetDevice(m->device));
    TFIM_CUDA(cudaMemcpyAsync(params, m->d_params, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost, m->stream));
    TFIM_CUDA(cudaStreamSynchronize(m->stream));
    return TFIM_OK;
}

int tfim_mlp_predict(tfim_mlp* h, const float* feats, int64_t n, float* probs) {
    Mlp* m = (Mlp*)h;
    TFIM_CHECK(m && (n == 0 || (feats && probs)) && n >= 0, TFIM_E_INVALID, "invalid arguments");
    if (n == 0) return TFIM_OK;
    TFIM_CUDA(cudaSetDevice(m->device));
    TFIM_TRY(m->d_x.reserve((size_t)n * kIn * 4));
    TFIM_TRY(m->d_out.reserve((size_t)n * 4));
    TFIM_CUDA(cudaMemcpyAsync(m->d_x.p, feats, (size_t)n * kIn * 4, cudaMemcpyHostToDevice, m->stream));
    TFIM_TRY(mlp_predict_device(m, m->d_x.as<float>(), n, m->d_out.as<float>(), m->stream));
    TFIM_CUDA(cudaMemcpyAsync(probs, m->d_out.p, (size_t)n * 4, cudaMemcpyDeviceToHost, m->stream));
    TFIM_CUDA(cudaStreamSynchronize(m->stream));
    return TFIM_OK;
}

int tfim_mlp_grad(tfim_mlp* h, const float* feats, const float* labels, int64_t n, float pos_weight, float* grads,
                  float* loss) {
    Mlp* m = (Mlp*)h;
    TFIM_CHECK(m && feats && labels && grads && n > 0, TFIM_E_INVALID, "invalid arguments");
    TFIM_CUDA(cudaSetDevice(m->device));
    TFIM_TRY(m->d_x.reserve((size_t)n * kIn * 4));
    TFIM_TRY(m->d_y.reserve((size_t)n * 4));
    TFIM_TRY(m->d_loss.reserve(16));
    TFIM_CUDA(cudaMemcpyAsync(m->d_x.p, feats, (size_t)n * kIn * 4, cudaMemcpyHostToDevice, m->stream));
    TFIM_CUDA(cudaMemcpyAsync(m->d_y.p, labels, (size_t)n * 4, cudaMemcpyHostToDevice, m->stream));
    TFIM_CUDA(cudaMemsetAsync(m->d_loss.p, 0, 4, m->stream));
    TFIM_TRY(mlp_grad_device(m, m->d_x.as<float>(), m->d_y.as<float>(), n, pos_weight, m->d_loss.as<float>(), m->stream));
    TFIM_CUDA(cudaMemcpyAsync(grads, m->d_grads, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost, m->stream));
    float l = 0;
    TFIM_CUDA(cudaMemcpyAsync(&l, m->d_loss.p, 4, cudaMemcpyDeviceToHost, m->stream));
    TFIM_CUDA(cudaStreamSynchronize(m->stream));
    if (loss) *loss = l;
    return TFIM_OK;
}

int tfim_mlp_train(tfim_mlp* h, const float* feats, const float* labels, int64_t n, int32_t epochs, int32_t batch,
                   float lr, float pos_weight, float weight_decay, float* final_loss) {
    Mlp* m = (Mlp*)h;
    TFIM_CHECK(m && feats && labels && n > 0 && epochs > 0 && batch > 0, TFIM_E_INVALID, "invalid arguments");
    TFIM_CUDA(cudaSetDevice(m->device));
    TFIM_TRY(m->d_x.reserve((size_t)n * kIn * 4));
    TFIM_TRY(m->d_y.reserve((size_t)n * 4));
    TFIM_TRY(m->d_loss.reserve(16));
    TFIM_CUDA(cudaMemcpyAsync(m->d_x.p, feats, (size_t)n * kIn * 4, cudaMemcpyHostToDevice, m->stream));
    TFIM_CUDA(cudaMemcpyAsync(m->d_y.p, labels, (size_t)n * 4, cudaMemcpyHostToDevice, m->stream));
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    float last = 0.f;
    for (int e = 0; e < epochs; e++) {
        TFIM_CUDA(cudaMemsetAsync(m->d_loss.p, 0, 4, m->stream));
        for (int64_t s0 = 0; s0 < n; s0 += batch) {
            const int64_t nb = std::min<int64_t>(batch, n - s0);
            TFIM_TRY(mlp_grad_device(m, m->d_x.as<float>() + s0 * kIn, m->d_y.as<float>() + s0, nb, pos_weight,
                                     m->d_loss.as<float>(), m->stream));
            m->step++;
            const float c1 = 1.f - std::pow(b1, (float)m->step), c2 = 1.f - std::pow(b2, (float)m->step);
            k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, m->stream>>>(m->d_params, m->d_grads, m->d_m, m->d_v, m->d_wbf,
                                                                      lr, b1, b2, eps, c1, c2, weight_decay);
            TFIM_CUDA(cudaGetLastError());
        }
        TFIM_CUDA(cudaMemcpyAsync(&last, m->d_loss.p, 4, cudaMemcpyDeviceToHost, m->stream));
        TFIM_CUDA(cudaStreamSynchronize(m->stream));
    }
    if (final_loss) *final_loss = last * (float)batch / (float)std::max<int64_t>(1, n);
    return TFIM_OK;
}

void tfim_mlp_free(tfim_mlp* h) {
    Mlp* m = (Mlp*)h;
    if (!m) return;
    cudaSetDevice(m->device);
    dev_free(m->d_params, m->stream);
    dev_free(m->d_grads, m->stream);
    dev_free(m->d_m, m->stream);
    dev_free(m->d_v, m->stream);
    dev_free(m->d_wbf, m->stream);
    m->d_x.release(); m->d_y.release(); m->d_out.release(); m->d_loss.release();
    if (m->stream) {
        cudaStreamSynchronize(m->stream);
        cudaStreamDestroy(m->stream);
    }
    delete m;
}

}  // extern "C"
