// Learned output-size predictor ("sizer"): a 16 -> 64 -> 64 -> 1 ReLU network with BF16 weights
// and FP32 accumulation that predicts log2(1 + output nnz) of a row from cheap per-row features.
// Training and inference run on hand-written kernels below (no library GEMM):
//   sizer_grad_kernel   one block per 128-sample tile: forward, backward, per-tile gradient sums
//   sizer_reduce_kernel per parameter: sum of the tile partials in tile order (deterministic)
//   sizer_adam_kernel   Adam step on the FP32 master weights, then the BF16 copies
//   sizer_predict_kernel one thread per sample
// Parameter order (weights and gradients): W1[64][16], b1[64], W2[64][64], b2[64], w3[64], b3.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "ptc_sizer.cuh"

namespace ptc {

constexpr int kIn = kSizerInputs;   // 16
constexpr int kHid = kSizerHidden;  // 64
constexpr int oW1 = 0, oB1 = oW1 + kHid * kIn, oW2 = oB1 + kHid, oB2 = oW2 + kHid * kHid, oW3 = oB2 + kHid,
              oB3 = oW3 + kHid;
static_assert(oB3 + 1 == kSizerParams, "parameter layout");

// Device copy of the network: weights in BF16, biases in FP32.
struct SizerDev {
    __nv_bfloat16* w = nullptr;  // W1, W2, w3 packed: [kHid*kIn + kHid*kHid + kHid]
    float* b = nullptr;          // b1, b2, b3: [2*kHid + 1]
};
constexpr int kNW = kHid * kIn + kHid * kHid + kHid;
constexpr int kNB = 2 * kHid + 1;

// Shared-memory copy of the network as FP32 values of the BF16 weights.
struct SmemNet {
    float W1[kHid][kIn];
    float W2[kHid][kHid];
    float w3[kHid];
    float b1[kHid], b2[kHid], b3;
};

__device__ __forceinline__ void load_net(SmemNet& n, const SizerDev d) {
    for (int i = threadIdx.x; i < kNW; i += blockDim.x) {
        const float v = __bfloat162float(d.w[i]);
        if (i < kHid * kIn) (&n.W1[0][0])[i] = v;
        else if (i < kHid * kIn + kHid * kHid) (&n.W2[0][0])[i - kHid * kIn] = v;
        else n.w3[i - kHid * kIn - kHid * kHid] = v;
    }
    for (int i = threadIdx.x; i < kNB; i += blockDim.x) {
        const float v = d.b[i];
        if (i < kHid) n.b1[i] = v;
        else if (i < 2 * kHid) n.b2[i - kHid] = v;
        else n.b3 = v;
    }
}

__global__ void __launch_bounds__(128) sizer_predict_kernel(SizerDev d, const float* __restrict__ x, uint64_t n,
                                                            float* __restrict__ y) {
    __shared__ SmemNet net;
    load_net(net, d);
    __syncthreads();
    const uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float xi[kIn];
#pragma unroll
    for (int k = 0; k < kIn; ++k) xi[k] = x[s * kIn + k];
    float h1[kHid];
#pragma unroll
    for (int i = 0; i < kHid; ++i) {
        float z = net.b1[i];
#pragma unroll
        for (int k = 0; k < kIn; ++k) z = fmaf(net.W1[i][k], xi[k], z);
        h1[i] = fmaxf(z, 0.f);
    }
    float out = net.b3;
    for (int j = 0; j < kHid; ++j) {
        float z = net.b2[j];
#pragma unroll
        for (int i = 0; i < kHid; ++i) z = fmaf(net.W2[j][i], h1[i], z);
        out = fmaf(net.w3[j], fmaxf(z, 0.f), out);
    }
    y[s] = out;
}

constexpr int kTile = 128;  // samples (and threads) per gradient block

__global__ void __launch_bounds__(kTile) sizer_grad_kernel(SizerDev d, const float* __restrict__ x,
                                                           const float* __restrict__ t, const uint32_t* __restrict__ idx,
                                                           uint64_t n, float inv_total, float* __restrict__ partial,
                                                           float* __restrict__ loss_partial) {
    extern __shared__ __align__(16) float sm[];
    SmemNet& net = *reinterpret_cast<SmemNet*>(sm);
    float* X = sm + (sizeof(SmemNet) + 3) / 4;          // [kTile][kIn + 1]
    float* H1 = X + kTile * (kIn + 1);                  // [kTile][kHid + 1]: z1, then dh1
    float* H2 = H1 + kTile * (kHid + 1);                // [kTile][kHid + 1]: z2, then dh2
    float* DY = H2 + kTile * (kHid + 1);                // [kTile]
    load_net(net, d);
    const int s = threadIdx.x;
    const uint64_t g = (uint64_t)blockIdx.x * kTile + s;
    const bool valid = g < n;
    const uint64_t src = valid ? (idx ? idx[g] : g) : 0;
    for (int k = 0; k < kIn; ++k) X[s * (kIn + 1) + k] = valid ? x[src * kIn + k] : 0.f;
    __syncthreads();

    // forward; z1/z2 kept for the ReLU masks
    float h1[kHid];
    for (int i = 0; i < kHid; ++i) {
        float z = net.b1[i];
#pragma unroll
        for (int k = 0; k < kIn; ++k) z = fmaf(net.W1[i][k], X[s * (kIn + 1) + k], z);
        H1[s * (kHid + 1) + i] = z;
        h1[i] = fmaxf(z, 0.f);
    }
    float y = net.b3;
    for (int j = 0; j < kHid; ++j) {
        float z = net.b2[j];
#pragma unroll
        for (int i = 0; i < kHid; ++i) z = fmaf(net.W2[j][i], h1[i], z);
        H2[s * (kHid + 1) + j] = z;
        y = fmaf(net.w3[j], fmaxf(z, 0.f), y);
    }
    const float diff = valid ? (y - t[src]) : 0.f;
    const float dy = 2.f * diff * inv_total;
    DY[s] = dy;
    __syncthreads();

    float* P = partial + (uint64_t)blockIdx.x * kSizerParams;
    // w3, b3
    if (s < kHid) {
        float acc = 0.f;
        for (int q = 0; q < kTile; ++q) acc = fmaf(DY[q], fmaxf(H2[q * (kHid + 1) + s], 0.f), acc);
        P[oW3 + s] = acc;
    }
    if (s == kHid) {
        float acc = 0.f;
        for (int q = 0; q < kTile; ++q) acc += DY[q];
        P[oB3] = acc;
    }
    if (s == kHid + 1) {
        float acc = 0.f;
        for (int q = 0; q < kTile; ++q) {
            const float e = DY[q];
            acc += e * e;
        }
        loss_partial[blockIdx.x] = acc;  // sum of dy^2; the host rescales it to the mean loss
    }
    __syncthreads();
    // dh2 = dy * w3 * [z2 > 0], in place of z2
    for (int j = 0; j < kHid; ++j) {
        const float z = H2[s * (kHid + 1) + j];
        H2[s * (kHid + 1) + j] = z > 0.f ? dy * net.w3[j] : 0.f;
    }
    __syncthreads();
    // W2, b2: entry e = (j, i)
    for (int e = s; e < kHid * kHid; e += kTile) {
        const int j = e / kHid, i = e % kHid;
        float acc = 0.f;
        for (int q = 0; q < kTile; ++q) acc = fmaf(H2[q * (kHid + 1) + j], fmaxf(H1[q * (kHid + 1) + i], 0.f), acc);
        P[oW2 + e] = acc;
    }
    if (s < kHid) {
        float acc = 0.f;
        for (int q = 0; q < kTile; ++q) acc += H2[q * (kHid + 1) + s];
        P[oB2 + s] = acc;
    }
    __syncthreads();
    // dh1 = (dh2 W2) * [z1 > 0], in place of z1
    {
        float dh1[kHid];
        for (int i = 0; i < kHid; ++i) dh1[i] = 0.f;
        for (int j = 0; j < kHid; ++j) {
            const float g2 = H2[s * (kHid + 1) + j];
#pragma unroll
            for (int i = 0; i < kHid; ++i) dh1[i] = fmaf(g2, net.W2[j][i], dh1[i]);
        }
        for (int i = 0; i < kHid; ++i) {
            const float z = H1[s * (kHid + 1) + i];
            H1[s * (kHid + 1) + i] = z > 0.f ? dh1[i] : 0.f;
        }
    }
    __syncthreads();
    // W1, b1: entry e = (i, k)
    for (int e = s; e < kHid * kIn; e += kTile) {
        const int i = e / kIn, k = e % kIn;
        float acc = 0.f;
        for (int q = 0; q < kTile; ++q) acc = fmaf(H1[q * (kHid + 1) + i], X[q * (kIn + 1) + k], acc);
        P[oW1 + e] = acc;
    }
    if (s < kHid) {
        float acc = 0.f;
        for (int q = 0; q < kTile; ++q) acc += H1[q * (kHid + 1) + s];
        P[oB1 + s] = acc;
    }
}

size_t sizer_grad_smem() {
    return ((sizeof(SmemNet) + 3) / 4 + kTile * (kIn + 1) + 2 * kTile * (kHid + 1) + kTile) * sizeof(float);
}

__global__ void sizer_reduce_kernel(const float* __restrict__ partial, uint32_t nblocks, float* __restrict__ grad) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kSizerParams) return;
    float acc = 0.f;
    for (uint32_t b = 0; b < nblocks; ++b) acc += partial[(uint64_t)b * kSizerParams + p];
    grad[p] = acc;
}

__global__ void sizer_adam_kernel(float* __restrict__ master, float* __restrict__ m, float* __restrict__ v,
                                  const float* __restrict__ grad, float lr, float beta1, float beta2, float eps,
                                  float bc1, float bc2, SizerDev d) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kSizerParams) return;
    const float g = grad[p];
    const float mm = beta1 * m[p] + (1.f - beta1) * g;
    const float vv = beta2 * v[p] + (1.f - beta2) * g * g;
    m[p] = mm;
    v[p] = vv;
    const float w = master[p] - lr * (mm / bc1) / (sqrtf(vv / bc2) + eps);
    master[p] = w;
    // device copies: weights as BF16, biases as FP32
    if (p < oB1) d.w[p] = __float2bfloat16_rn(w);
    else if (p < oW2) d.b[p - oB1] = w;
    else if (p < oB2) d.w[kHid * kIn + (p - oW2)] = __float2bfloat16_rn(w);
    else if (p < oW3) d.b[kHid + (p - oB2)] = w;
    else if (p < oB3) d.w[kHid * kIn + kHid * kHid + (p - oW3)] = __float2bfloat16_rn(w);
    else d.b[2 * kHid] = w;
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------

namespace {

void upload(const std::vector<float>& master, SizerDev d, cudaStream_t st) {
    std::vector<__nv_bfloat16> w(kNW);
    std::vector<float> b(kNB);
    for (int p = 0; p < kSizerParams; ++p) {
        const float x = master[p];
        if (p < oB1) w[p] = __float2bfloat16_rn(x);
        else if (p < oW2) b[p - oB1] = x;
        else if (p < oB2) w[kHid * kIn + (p - oW2)] = __float2bfloat16_rn(x);
        else if (p < oW3) b[kHid + (p - oB2)] = x;
        else if (p < oB3) w[kHid * kIn + kHid * kHid + (p - oW3)] = __float2bfloat16_rn(x);
        else b[2 * kHid] = x;
    }
    PTC_CUDA(cudaMemcpyAsync(d.w, w.data(), kNW * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice, st));
    PTC_CUDA(cudaMemcpyAsync(d.b, b.data(), kNB * sizeof(float), cudaMemcpyHostToDevice, st));
    PTC_CUDA(cudaStreamSynchronize(st));
}

SizerDev alloc_dev(Arena& ar) {
    SizerDev d;
    d.w = ar.alloc<__nv_bfloat16>(kNW);
    d.b = ar.alloc<float>(kNB);
    return d;
}

}  // namespace

void sizer_predict_device(const SizerHost& s, const float* d_x, uint64_t n, float* d_y, Arena& ar) {
    if (n == 0) return;
    SizerDev d = alloc_dev(ar);
    upload(s.master, d, ar.stream());
    sizer_predict_kernel<<<ceil_div_u32(n, 128), 128, 0, ar.stream()>>>(d, d_x, n, d_y);
    count_launch();
    PTC_CHECK_LAUNCH();
}

float sizer_gradients(const SizerHost& s, const float* d_x, const float* d_t, uint64_t n, float* h_grad, Arena& ar) {
    cudaStream_t st = ar.stream();
    SizerDev d = alloc_dev(ar);
    upload(s.master, d, st);
    const uint32_t nb = ceil_div_u32(n, kTile);
    float* partial = ar.alloc<float>((uint64_t)nb * kSizerParams);
    float* lossp = ar.alloc<float>(nb);
    float* grad = ar.alloc<float>(kSizerParams);
    const size_t smem = sizer_grad_smem();
    PTC_CUDA(cudaFuncSetAttribute(sizer_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    sizer_grad_kernel<<<nb, kTile, smem, st>>>(d, d_x, d_t, nullptr, n, 1.f / (float)n, partial, lossp);
    count_launch();
    PTC_CHECK_LAUNCH();
    sizer_reduce_kernel<<<ceil_div_u32(kSizerParams, 256), 256, 0, st>>>(partial, nb, grad);
    count_launch();
    PTC_CHECK_LAUNCH();
    std::vector<float> lp(nb);
    PTC_CUDA(cudaMemcpyAsync(h_grad, grad, kSizerParams * sizeof(float), cudaMemcpyDeviceToHost, st));
    PTC_CUDA(cudaMemcpyAsync(lp.data(), lossp, nb * sizeof(float), cudaMemcpyDeviceToHost, st));
    PTC_CUDA(cudaStreamSynchronize(st));
    // lossp holds sums of dy^2 = (2 diff / n)^2  ->  mean diff^2 = sum * n / 4
    double sum = 0;
    for (float v : lp) sum += v;
    return (float)(sum * (double)n / 4.0);
}

SizerTrainResult sizer_train(SizerHost& s, const float* d_x, const float* d_t, uint64_t n, uint32_t epochs,
                             uint32_t batch, float lr, uint64_t seed, Arena& ar) {
    cudaStream_t st = ar.stream();
    SizerTrainResult res;
    if (n == 0 || epochs == 0) return res;
    batch = std::max<uint32_t>(kTile, (batch / kTile) * kTile);
    SizerDev d = alloc_dev(ar);
    upload(s.master, d, st);
    float* master = ar.alloc<float>(kSizerParams);
    float* m = ar.alloc<float>(kSizerParams);
    float* v = ar.alloc<float>(kSizerParams);
    PTC_CUDA(cudaMemcpyAsync(master, s.master.data(), kSizerParams * sizeof(float), cudaMemcpyHostToDevice, st));
    PTC_CUDA(cudaMemcpyAsync(m, s.m.data(), kSizerParams * sizeof(float), cudaMemcpyHostToDevice, st));
    PTC_CUDA(cudaMemcpyAsync(v, s.v.data(), kSizerParams * sizeof(float), cudaMemcpyHostToDevice, st));
    const uint32_t nb = ceil_div_u32(batch, kTile);
    float* partial = ar.alloc<float>((uint64_t)nb * kSizerParams);
    float* lossp = ar.alloc<float>(nb * ((n + batch - 1) / batch));
    float* grad = ar.alloc<float>(kSizerParams);
    uint32_t* idx = ar.alloc<uint32_t>(n);
    const size_t smem = sizer_grad_smem();
    PTC_CUDA(cudaFuncSetAttribute(sizer_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    std::vector<uint32_t> order(n);
    for (uint64_t i = 0; i < n; ++i) order[i] = (uint32_t)i;
    std::mt19937_64 rng(seed);
    const uint64_t nbatches = (n + batch - 1) / batch;
    std::vector<float> lp(nb * nbatches);
    const float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
    for (uint32_t ep = 0; ep < epochs; ++ep) {
        std::shuffle(order.begin(), order.end(), rng);
        PTC_CUDA(cudaMemcpyAsync(idx, order.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        for (uint64_t bi = 0; bi < nbatches; ++bi) {
            const uint64_t b0 = bi * batch, bn = std::min<uint64_t>(batch, n - b0);
            const uint32_t blocks = ceil_div_u32(bn, kTile);
            sizer_grad_kernel<<<blocks, kTile, smem, st>>>(d, d_x, d_t, idx + b0, bn, 1.f / (float)bn, partial,
                                                           lossp + bi * nb);
            count_launch();
            sizer_reduce_kernel<<<ceil_div_u32(kSizerParams, 256), 256, 0, st>>>(partial, blocks, grad);
            count_launch();
            ++s.steps;
            const float bc1 = 1.f - std::pow(beta1, (float)s.steps), bc2 = 1.f - std::pow(beta2, (float)s.steps);
            sizer_adam_kernel<<<ceil_div_u32(kSizerParams, 256), 256, 0, st>>>(master, m, v, grad, lr, beta1, beta2,
                                                                              eps, bc1, bc2, d);
            count_launch();
            if (bn < batch)
                PTC_CUDA(cudaMemsetAsync(lossp + bi * nb + blocks, 0, (nb - blocks) * sizeof(float), st));
        }
        PTC_CHECK_LAUNCH();
        PTC_CUDA(cudaMemcpyAsync(lp.data(), lossp, lp.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
        PTC_CUDA(cudaStreamSynchronize(st));
        double sum = 0;
        for (uint64_t bi = 0; bi < nbatches; ++bi) {
            const uint64_t bn = std::min<uint64_t>(batch, n - bi * batch);
            double sb = 0;
            for (uint32_t q = 0; q < nb; ++q) sb += lp[bi * nb + q];
            sum += sb * (double)bn * (double)bn / 4.0;  // back to sum of diff^2
        }
        const float mean = (float)(sum / (double)n);
        if (ep == 0) res.first_loss = mean;
        res.final_loss = mean;
        res.epochs = ep + 1;
    }
    PTC_CUDA(cudaMemcpyAsync(s.master.data(), master, kSizerParams * sizeof(float), cudaMemcpyDeviceToHost, st));
    PTC_CUDA(cudaMemcpyAsync(s.m.data(), m, kSizerParams * sizeof(float), cudaMemcpyDeviceToHost, st));
    PTC_CUDA(cudaMemcpyAsync(s.v.data(), v, kSizerParams * sizeof(float), cudaMemcpyDeviceToHost, st));
    PTC_CUDA(cudaStreamSynchronize(st));
    res.steps = s.steps;
    return res;
}

void sizer_init(SizerHost& s, uint64_t seed) {
    s.master.assign(kSizerParams, 0.f);
    s.m.assign(kSizerParams, 0.f);
    s.v.assign(kSizerParams, 0.f);
    s.steps = 0;
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.f, 1.f);
    for (int p = oW1; p < oB1; ++p) s.master[p] = nd(rng) * std::sqrt(2.f / kIn);
    for (int p = oW2; p < oB2; ++p) s.master[p] = nd(rng) * std::sqrt(2.f / kHid);
    for (int p = oW3; p < oB3; ++p) s.master[p] = nd(rng) * std::sqrt(1.f / kHid);
    for (int p = oB1; p < oW2; ++p) s.master[p] = 0.01f;
    for (int p = oB2; p < oW3; ++p) s.master[p] = 0.01f;
    s.master[oB3] = 0.f;
}

}  // namespace ptc
