// Bucketed two-choice cuckoo hash table: distinct 64-bit keys -> 32-bit values.
//
// This replaces the reference's two-level FKS table (fksCuckoo.hpp): there, level 1 hashes a
// key to one of N buckets (get_bucket_id, :658-672) and level 2 places it in a per-bucket cuckoo
// table with two hash functions, evicting along augmenting paths (cuckooHash/augment,
// :504-597) and rehashing with new multipliers when that fails (rehash, :297-442).  Here a bucket
// is one 128-byte line of 16 key slots; a key may live in either of two buckets; a 16-lane group
// inserts a key with atomicCAS into a free slot of its bucket and, when that bucket is full,
// swaps it with a resident key (atomicExch) that then moves to its other bucket.  The eviction chain
// is bounded; when it runs out the build reports failure and the host rebuilds with fresh seeds
// (and, after repeated failures, twice the buckets) -- the analogue of the reference's rehash.
// Lookups touch at most two 128-byte lines (the reference: one bucket hash plus <= 2 slot probes,
// find_element_new, :867-978).
#pragma once

#include "ptc_common.cuh"

namespace ptc {

constexpr uint32_t kBucketSlots = 16;

struct CuckooTable {
    uint64_t* keys = nullptr;  // [nbuckets * 16], kEmptyKey = free
    uint32_t* vals = nullptr;  // [nbuckets * 16]
    uint32_t log2_buckets = 0;
    uint64_t seed1 = 0, seed2 = 0;
};

__device__ __forceinline__ uint32_t cuckoo_b1(const CuckooTable& t, uint64_t key) {
    return t.log2_buckets ? (uint32_t)(mix64(key ^ t.seed1) >> (64 - t.log2_buckets)) : 0u;
}
__device__ __forceinline__ uint32_t cuckoo_b2(const CuckooTable& t, uint64_t key, uint32_t b1) {
    if (t.log2_buckets == 0) return 0u;
    uint32_t b = (uint32_t)(mix64(key ^ t.seed2) >> (64 - t.log2_buckets));
    return b == b1 ? (b1 ^ 1u) : b;
}

// Value stored for `key`, or -1 if absent.  One thread; reads whole 128-byte buckets.
__device__ __forceinline__ int64_t cuckoo_find(const CuckooTable& t, uint64_t key) {
    const uint32_t b1 = cuckoo_b1(t, key);
    const ulonglong2* p = reinterpret_cast<const ulonglong2*>(t.keys + (uint64_t)b1 * kBucketSlots);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        ulonglong2 kk = __ldg(p + i);
        if (kk.x == key) return t.vals[(uint64_t)b1 * kBucketSlots + 2 * i];
        if (kk.y == key) return t.vals[(uint64_t)b1 * kBucketSlots + 2 * i + 1];
    }
    const uint32_t b2 = cuckoo_b2(t, key, b1);
    p = reinterpret_cast<const ulonglong2*>(t.keys + (uint64_t)b2 * kBucketSlots);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        ulonglong2 kk = __ldg(p + i);
        if (kk.x == key) return t.vals[(uint64_t)b2 * kBucketSlots + 2 * i];
        if (kk.y == key) return t.vals[(uint64_t)b2 * kBucketSlots + 2 * i + 1];
    }
    return -1;
}

struct CuckooBuildInfo {
    uint32_t attempts = 0;
    uint32_t log2_buckets = 0;
};

// Build a table over n distinct keys; vals[slot of keys[i]] = i.  Throws Error
// (PTC_ERR_HASH_BUILD) if every attempt fails.  max_chain bounds each eviction chain.
CuckooTable cuckoo_build(const uint64_t* keys, uint64_t n, uint64_t seed, uint32_t max_chain,
                         double max_load, uint32_t max_attempts, Arena& ar, CuckooBuildInfo* info);

// out[i] = value of keys[i] (or -1).
void cuckoo_lookup(const CuckooTable& t, const uint64_t* keys, uint64_t n, int32_t* out, Arena& ar);

}  // namespace ptc
