// Allocation-free sizer inference: ptc_sizer_predict_noalloc (include/partc.h).
//
// Some callers cannot allocate device memory when they need a prediction: a process whose device
// memory is owned by another allocator (a framework's caching allocator that holds the whole
// device), code running where an allocation would synchronize the device or is not allowed, or a
// service that budgets all device memory once at start-up.  For them this entry point does the
// work of ptc_sizer_predict without calling cudaMalloc, cudaFree or any allocating routine.  Its
// device scratch -- the network's BF16 weights and FP32 biases, the staged feature rows and the
// predictions -- lives in one file-scope __device__ array of kNoAllocScratchBytes, which every
// device that loads the library keeps until the process exits.
//
// Rules for callers:
//   * at most kNoAllocMaxRows feature rows per call; a larger call is rejected with
//     PTC_ERR_INVALID_ARGUMENT and does nothing;
//   * the first call on a device looks up the array's device address there (cudaGetSymbolAddress,
//     once per device, with that device current) and keeps it for the life of the process; make
//     that first call before capturing any stream.  The kept address does not survive a
//     cudaDeviceReset of that device: after a reset this entry point must not be called again in
//     the same process;
//   * the caller's current device is restored before the call returns;
//   * every call uses the same array and overwrites it; nothing in it needs to start at zero, since
//     each call writes every byte it later reads.  Calls whose GPU work overlaps (two host threads,
//     or two unordered streams) race on the array.  A call runs on the calling thread's per-thread
//     default stream and returns once the predictions are in `out`.
#include <cuda_bf16.h>

#include <cstring>
#include <mutex>

#include "partc.h"
#include "ptc_sizer.cuh"

namespace ptc {

namespace {

constexpr uint64_t kNoAllocMaxRows = 65536;
constexpr int kIn = kSizerInputs;
constexpr int kHid = kSizerHidden;
constexpr int kNumW = kHid * kIn + kHid * kHid + kHid;  // BF16 weights: W1, W2, w3
constexpr int kNumB = 2 * kHid + 1;                     // FP32 biases: b1, b2, b3

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffW = 0;
constexpr size_t kOffB = align256(kOffW + kNumW * sizeof(__nv_bfloat16));
constexpr size_t kOffX = align256(kOffB + kNumB * sizeof(float));
constexpr size_t kOffY = align256(kOffX + kNoAllocMaxRows * kIn * sizeof(float));
constexpr size_t kNoAllocScratchBytes = align256(kOffY + kNoAllocMaxRows * sizeof(float));  // ~4.3 MiB

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on `device` (which must be current), looked up on the
// first call there.  In host code the array's name only stands for it; the kernel needs this.
unsigned char* scratch_on(int device) {
    PTC_REQUIRE(device >= 0 && device < kMaxDevices, PTC_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            throw Error{PTC_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e)};
        g_scratch_ptr[device] = static_cast<unsigned char*>(p);
    }
    return g_scratch_ptr[device];
}

// The network's forward pass (the same arithmetic as the sizer's inference kernel), reading the
// weights and the feature rows from the scratch array and writing the predictions there.
__global__ void __launch_bounds__(128) sizer_predict_noalloc_kernel(const __nv_bfloat16* __restrict__ w,
                                                                    const float* __restrict__ b,
                                                                    const float* __restrict__ x, uint64_t n,
                                                                    float* __restrict__ y) {
    __shared__ float W1[kHid][kIn];
    __shared__ float W2[kHid][kHid];
    __shared__ float w3[kHid];
    __shared__ float b1[kHid], b2[kHid];
    __shared__ float b3;
    for (int i = threadIdx.x; i < kNumW; i += blockDim.x) {
        const float v = __bfloat162float(w[i]);
        if (i < kHid * kIn) (&W1[0][0])[i] = v;
        else if (i < kHid * kIn + kHid * kHid) (&W2[0][0])[i - kHid * kIn] = v;
        else w3[i - kHid * kIn - kHid * kHid] = v;
    }
    for (int i = threadIdx.x; i < kNumB; i += blockDim.x) {
        if (i < kHid) b1[i] = b[i];
        else if (i < 2 * kHid) b2[i - kHid] = b[i];
        else b3 = b[i];
    }
    __syncthreads();
    const uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float xi[kIn];
#pragma unroll
    for (int k = 0; k < kIn; ++k) xi[k] = x[s * kIn + k];
    float h1[kHid];
#pragma unroll
    for (int i = 0; i < kHid; ++i) {
        float z = b1[i];
#pragma unroll
        for (int k = 0; k < kIn; ++k) z = fmaf(W1[i][k], xi[k], z);
        h1[i] = fmaxf(z, 0.f);
    }
    float out = b3;
    for (int j = 0; j < kHid; ++j) {
        float z = b2[j];
#pragma unroll
        for (int i = 0; i < kHid; ++i) z = fmaf(W2[j][i], h1[i], z);
        out = fmaf(w3[j], fmaxf(z, 0.f), out);
    }
    y[s] = out;
}

}  // namespace

}  // namespace ptc

extern "C" ptc_status ptc_sizer_predict_noalloc(const ptc_sizer* s, const float* features, uint64_t n,
                                                int32_t device, float* out) {
    using namespace ptc;
    DeviceGuard keep_device;
    try {
        PTC_REQUIRE(s && features && out, PTC_ERR_INVALID_ARGUMENT, "null argument");
        PTC_REQUIRE(n <= kNoAllocMaxRows, PTC_ERR_INVALID_ARGUMENT,
                    "ptc_sizer_predict_noalloc takes at most 65536 feature rows per call");
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
            cudaGetLastError();
            throw Error{PTC_ERR_NO_DEVICE, "no usable CUDA device"};
        }
        if (device >= 0) PTC_CUDA(cudaSetDevice(device));
        else PTC_CUDA(cudaGetDevice(&device));
        unsigned char* base = scratch_on(device);
        if (n == 0) return PTC_OK;
        // the weights as the device uses them: W1, W2, w3 in BF16, biases in FP32 (host staging
        // on the stack; no allocation)
        __nv_bfloat16 hw[kNumW];
        float hb[kNumB];
        const std::vector<float>& m = s->host.master;
        int wi = 0, bi = 0;
        const int oB1 = kHid * kIn, oW2 = oB1 + kHid, oB2 = oW2 + kHid * kHid, oW3 = oB2 + kHid, oB3 = oW3 + kHid;
        for (int p = 0; p < kSizerParams; ++p) {
            const bool is_bias = (p >= oB1 && p < oW2) || (p >= oB2 && p < oW3) || p == oB3;
            if (is_bias) hb[bi++] = m[p];
            else hw[wi++] = __float2bfloat16_rn(m[p]);
        }
        cudaStream_t st = cudaStreamPerThread;
        auto* dw = reinterpret_cast<__nv_bfloat16*>(base + kOffW);
        auto* db = reinterpret_cast<float*>(base + kOffB);
        auto* dx = reinterpret_cast<float*>(base + kOffX);
        auto* dy = reinterpret_cast<float*>(base + kOffY);
        PTC_CUDA(cudaMemcpyAsync(dw, hw, sizeof(hw), cudaMemcpyHostToDevice, st));
        PTC_CUDA(cudaMemcpyAsync(db, hb, sizeof(hb), cudaMemcpyHostToDevice, st));
        PTC_CUDA(cudaMemcpyAsync(dx, features, n * kIn * sizeof(float), cudaMemcpyHostToDevice, st));
        sizer_predict_noalloc_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(dw, db, dx, n, dy);
        PTC_CUDA(cudaGetLastError());
        PTC_CUDA(cudaMemcpyAsync(out, dy, n * sizeof(float), cudaMemcpyDeviceToHost, st));
        PTC_CUDA(cudaStreamSynchronize(st));
        return PTC_OK;
    } catch (const Error& e) {
        set_last_error(e.status, e.msg);
        return e.status;
    } catch (...) {
        set_last_error(PTC_ERR_INTERNAL, "unexpected exception");
        return PTC_ERR_INTERNAL;
    }
}
