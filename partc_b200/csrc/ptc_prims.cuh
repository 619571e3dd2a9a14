// Device-wide primitives written for this engine: exclusive scan, stable LSD radix sort of
// (u64 key, u32 value) pairs, and run-head extraction over sorted keys.
#pragma once

#include "ptc_common.cuh"

namespace ptc {

// out[0..n] = exclusive prefix sums of in[0..n), out[n] = total.  `out` may alias `in` only if
// it has n+1 elements.  T is uint32_t or uint64_t.
template <typename T>
void exclusive_scan(const T* in, T* out, uint64_t n, Arena& ar);

// Stable sort of (keys, vals) by the key bits [begin_bit, end_bit); the result is written back
// into keys/vals.  n < 2^32.
void radix_sort_pairs(uint64_t* keys, uint32_t* vals, uint64_t n, int begin_bit, int end_bit, Arena& ar);

// For sorted keys: head[i] = 1 if i == 0 or keys[i] != keys[i-1] else 0; then
// run_of[i] = (number of heads in [0, i]) - 1 and, for each run r, run_start[r] = first index,
// run_key[r] = key.  run_start[nruns] = n.  Returns the number of runs (host value; syncs).
uint64_t runs_of_sorted(const uint64_t* keys, uint64_t n, uint32_t* run_of, uint32_t* run_start,
                        uint64_t* run_key, Arena& ar);

// Upper bound on the runs buffer sizes callers need: n + 1.

// Bits needed to represent values in [0, space).
inline int bits_for_space(uint64_t space) {
    int b = 0;
    while (b < 64 && ((space - 1) >> b) != 0) ++b;
    return b;
}

}  // namespace ptc
