// Shared device/host helpers of the contraction engine.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "partc.h"

namespace ptc {

constexpr uint32_t kWarp = 32;
constexpr uint32_t kFullMask = 0xffffffffu;
constexpr uint64_t kEmptyKey = ~0ull;

// ---- error handling (host) ------------------------------------------------------------------

struct Error {
    ptc_status status;
    std::string msg;
};

void set_last_error(ptc_status s, const std::string& msg);

#define PTC_CUDA(call)                                                                        \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            throw ::ptc::Error{e_ == cudaErrorMemoryAllocation ? PTC_ERR_OUT_OF_MEMORY        \
                                                               : PTC_ERR_CUDA,                \
                               std::string(#call) + ": " + cudaGetErrorString(e_)};           \
        }                                                                                     \
    } while (0)

#define PTC_CHECK_LAUNCH() PTC_CUDA(cudaGetLastError())

#define PTC_REQUIRE(cond, status, message)                                                    \
    do {                                                                                      \
        if (!(cond)) throw ::ptc::Error{(status), (message)};                                 \
    } while (0)

// Restores the calling thread's current device when an entry point returns (entry points
// switch to the device named in their options).
class DeviceGuard {
  public:
    DeviceGuard() { ok_ = cudaGetDevice(&saved_) == cudaSuccess; }
    ~DeviceGuard() {
        if (ok_) cudaSetDevice(saved_);
    }
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;

  private:
    int saved_ = 0;
    bool ok_ = false;
};

// ---- stream-ordered device arena ------------------------------------------------------------

// Every device buffer of one call comes from here and is returned (stream-ordered) when the
// call ends, so repeated calls reuse the CUDA memory pool instead of cudaMalloc/cudaFree.
class Arena {
  public:
    explicit Arena(cudaStream_t s) : stream_(s) {}
    ~Arena() { release(); }
    Arena(const Arena&) = delete;
    Arena& operator=(const Arena&) = delete;

    template <typename T>
    T* alloc(size_t n) {
        void* p = nullptr;
        size_t bytes = (n ? n : 1) * sizeof(T);
        bytes = (bytes + 255) & ~size_t(255);
        PTC_CUDA(cudaMallocAsync(&p, bytes, stream_));
        ptrs_.push_back(p);
        bytes_ += bytes;
        return static_cast<T*>(p);
    }
    void release() {
        for (void* p : ptrs_) cudaFreeAsync(p, stream_);
        ptrs_.clear();
    }
    size_t bytes() const { return bytes_; }
    cudaStream_t stream() const { return stream_; }

  private:
    cudaStream_t stream_;
    std::vector<void*> ptrs_;
    size_t bytes_ = 0;
};

// Launch counter for the stats (kernels launched by this call on this thread).
extern thread_local uint64_t g_launches;
inline void count_launch() { ++g_launches; }

inline uint32_t ceil_div_u32(uint64_t a, uint64_t b) { return (uint32_t)((a + b - 1) / b); }

// ---- device helpers -------------------------------------------------------------------------

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t x) {
    // splitmix64 finalizer: a full-avalanche 64-bit bijection
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebull;
    x ^= x >> 31;
    return x;
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint32_t lanemask_lt() { return (1u << lane_id()) - 1u; }

template <typename T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T n = __shfl_up_sync(kFullMask, v, o);
        if ((int)lane_id() >= o) v += n;
    }
    return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFullMask, v, o);
    return v;
}

// Block-wide exclusive scan for NT threads (NT a multiple of 32, <= 1024).  `tmp` must hold
// NT/32 + 1 elements of shared memory.  Returns the exclusive prefix; *total gets the sum.
template <typename T, int NT>
__device__ __forceinline__ T block_exclusive_scan(T v, T* tmp, T* total) {
    constexpr int NW = NT / 32;
    const int w = threadIdx.x >> 5;
    T inc = warp_inclusive_scan(v);
    if (lane_id() == 31) tmp[w] = inc;
    __syncthreads();
    if (w == 0) {
        T s = (lane_id() < (uint32_t)NW) ? tmp[lane_id()] : T(0);
        T si = warp_inclusive_scan(s);
        if (lane_id() < (uint32_t)NW) tmp[lane_id()] = si - s;
        if (lane_id() == NW - 1) tmp[NW] = si;
    }
    __syncthreads();
    T out = tmp[w] + inc - v;
    *total = tmp[NW];
    __syncthreads();
    return out;
}

}  // namespace ptc
