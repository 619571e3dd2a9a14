// Bucketed cuckoo hash build and lookup (see ptc_cuckoo.cuh).
#include "ptc_cuckoo.cuh"

namespace ptc {

__global__ void cuckoo_clear(uint64_t* keys, uint64_t nslots) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nslots) keys[i] = kEmptyKey;
}

// One 16-lane group per key.  All control flow below is uniform within a group, so the group
// mask is valid for every shuffle and ballot.
__global__ void cuckoo_insert(const uint64_t* __restrict__ in, uint64_t n, CuckooTable t, uint32_t max_chain,
                              uint32_t* __restrict__ failed) {
    const uint64_t g = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / kBucketSlots;
    const uint32_t lane = lane_id();
    const uint32_t half = lane & 16u;
    const uint32_t sub = lane & 15u;
    const uint32_t gmask = 0xffffu << half;
    if (g >= n) return;  // whole group leaves together (n is per group)
    uint64_t key = in[g];
    uint32_t b = cuckoo_b1(t, key);
    for (uint32_t chain = 0;; ++chain) {
        uint64_t* bucket = t.keys + (uint64_t)b * kBucketSlots;
        const uint64_t cur = bucket[sub];
        uint32_t empty = (__ballot_sync(gmask, cur == kEmptyKey) >> half) & 0xffffu;
        while (empty) {
            const int s = __ffs(empty) - 1;
            uint64_t old = 0;
            if ((int)sub == s) old = atomicCAS(reinterpret_cast<unsigned long long*>(bucket + s), kEmptyKey, key);
            old = __shfl_sync(gmask, old, half + s);
            if (old == kEmptyKey) return;  // placed
            empty &= ~(1u << s);
        }
        if (chain >= max_chain) {
            if (sub == 0) atomicExch(failed, 1u);
            return;
        }
        // bucket full: swap with a pseudo-random resident, which moves to its other bucket
        const int s = (int)((mix64(key + 0x9e3779b97f4a7c15ull * (chain + 1)) >> 40) & 15u);
        uint64_t old = 0;
        if ((int)sub == s) old = atomicExch(reinterpret_cast<unsigned long long*>(bucket + s), key);
        old = __shfl_sync(gmask, old, half + s);
        if (old == kEmptyKey) return;  // the slot had been freed meanwhile; nothing evicted
        key = old;
        const uint32_t b1 = cuckoo_b1(t, key);
        const uint32_t b2 = cuckoo_b2(t, key, b1);
        b = (b == b1) ? b2 : b1;
    }
}

// Second pass: every key is now resident; record its value in its slot.  Also verifies that
// every key is found (a lost key means the build failed).
__global__ void cuckoo_set_values(const uint64_t* __restrict__ in, uint64_t n, CuckooTable t,
                                  uint32_t* __restrict__ failed) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t key = in[i];
    const uint32_t b1 = cuckoo_b1(t, key);
    const uint32_t b2 = cuckoo_b2(t, key, b1);
    for (int pass = 0; pass < 2; ++pass) {
        const uint64_t base = (uint64_t)(pass ? b2 : b1) * kBucketSlots;
        for (uint32_t s = 0; s < kBucketSlots; ++s) {
            if (t.keys[base + s] == key) {
                t.vals[base + s] = (uint32_t)i;
                return;
            }
        }
    }
    atomicExch(failed, 1u);
}

__global__ void cuckoo_lookup_kernel(CuckooTable t, const uint64_t* __restrict__ keys, uint64_t n,
                                     int32_t* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (int32_t)cuckoo_find(t, keys[i]);
}

CuckooTable cuckoo_build(const uint64_t* keys, uint64_t n, uint64_t seed, uint32_t max_chain, double max_load,
                         uint32_t max_attempts, Arena& ar, CuckooBuildInfo* info) {
    cudaStream_t st = ar.stream();
    PTC_REQUIRE(n < (1ull << 31), PTC_ERR_INVALID_ARGUMENT, "cuckoo table supports fewer than 2^31 keys");
    uint32_t log2b = 0;
    while ((double)((uint64_t)kBucketSlots << log2b) * max_load < (double)n) ++log2b;
    uint32_t* failed = ar.alloc<uint32_t>(1);
    CuckooTable t;
    for (uint32_t attempt = 0; attempt < max_attempts; ++attempt) {
        if (attempt > 0 && attempt % 2 == 0) ++log2b;  // grow after two failed seeds
        const uint64_t nslots = (uint64_t)kBucketSlots << log2b;
        t.keys = ar.alloc<uint64_t>(nslots);
        t.vals = ar.alloc<uint32_t>(nslots);
        t.log2_buckets = log2b;
        t.seed1 = mix64(seed * 2 + 1 + 0x51ed27ull * attempt);
        t.seed2 = mix64(seed * 2 + 2 + 0x6a09e667ull * attempt);
        PTC_CUDA(cudaMemsetAsync(failed, 0, sizeof(uint32_t), st));
        cuckoo_clear<<<ceil_div_u32(nslots, 256), 256, 0, st>>>(t.keys, nslots);
        count_launch();
        PTC_CHECK_LAUNCH();
        if (n > 0) {
            cuckoo_insert<<<ceil_div_u32(n * kBucketSlots, 256), 256, 0, st>>>(keys, n, t, max_chain, failed);
            count_launch();
            PTC_CHECK_LAUNCH();
            cuckoo_set_values<<<ceil_div_u32(n, 256), 256, 0, st>>>(keys, n, t, failed);
            count_launch();
            PTC_CHECK_LAUNCH();
        }
        uint32_t hf = 0;
        PTC_CUDA(cudaMemcpyAsync(&hf, failed, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        PTC_CUDA(cudaStreamSynchronize(st));
        if (info) {
            info->attempts = attempt + 1;
            info->log2_buckets = log2b;
        }
        if (!hf) return t;
    }
    throw Error{PTC_ERR_HASH_BUILD, "cuckoo table build failed for every seed and size tried"};
}

void cuckoo_lookup(const CuckooTable& t, const uint64_t* keys, uint64_t n, int32_t* out, Arena& ar) {
    if (n == 0) return;
    cuckoo_lookup_kernel<<<ceil_div_u32(n, 256), 256, 0, ar.stream()>>>(t, keys, n, out);
    count_launch();
    PTC_CHECK_LAUNCH();
}

}  // namespace ptc
