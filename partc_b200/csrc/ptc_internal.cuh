// Internal data layout shared by the build, accumulator and host-orchestration files.
#pragma once

#include "ptc_common.cuh"
#include "ptc_cuckoo.cuh"

namespace ptc {

constexpr int kMaxOrder = 16;

// Mixed-radix linearization of a mode tuple: key = sum_j idx[mode[j]] * stride[j], first listed
// mode most significant.  Replaces the reference's per-mode key loops and fastmod bucket
// arithmetic (fksCuckoo.hpp:66-94,658-672; fastmod.h:76-85) with one 64-bit key per nonzero.
struct KeySpec {
    uint32_t n = 0;
    uint32_t mode[kMaxOrder] = {};
    uint64_t stride[kMaxOrder] = {};
    uint64_t space = 1;  // product of the mode sizes
};

struct DimSpec {
    uint32_t order = 0;
    uint32_t dim[kMaxOrder] = {};
};

// Device view of the grouped operands (all arrays in HBM).
//   A side, sorted by row (A free key), COO input order kept inside a row:
//     a_val[i], a_fib[i] (B fiber id or -1), row_start[r] (nrows+1 entries)
//   B side, sorted by (contracted key, column), so each fiber is contiguous and ordered by column:
//     b_col[j] (dense column id = rank of B's free key), b_val[j], fib_start[f] (nfib+1)
//   Output index tuples: row_tuple[r * fa + m], col_tuple[q * fb + m]
struct Operands {
    uint64_t na = 0, nb = 0, nrows = 0, ncols = 0, nfib = 0;
    uint32_t fa = 0, fb = 0;
    const double* a_val = nullptr;
    const int32_t* a_fib = nullptr;
    const uint32_t* row_start = nullptr;
    const uint32_t* b_col = nullptr;
    const double* b_val = nullptr;
    const uint32_t* fib_start = nullptr;
    const uint32_t* row_tuple = nullptr;
    const uint32_t* col_tuple = nullptr;
    // dense-panel split of every fiber: panel_off[f * (npanels + 1) + p] = first entry of fiber f
    // whose column is >= p * panel_width (null when there is a single panel)
    const uint32_t* panel_off = nullptr;
    uint32_t npanels = 1;
    uint32_t panel_log2 = 0;
    // set to nonzero by a kernel that met an impossible index (a bug guard: the access is skipped)
    uint32_t* err = nullptr;
    // batches: column ids are local to each item; row_colbase[row] is the first global column of
    // the row's item (null for a single contraction, where local and global ids coincide)
    const uint32_t* row_colbase = nullptr;
};

// A part of a row for the hash accumulator: the row's columns in fine panels [p0, p1), and
// where its output entries start.
struct PartItem {
    uint32_t row;
    uint32_t p0;
    uint32_t p1;
    uint32_t mode;  // bit 0: 1 = dense (direct-mapped by column), 0 = open-addressing table of
                    // 2^(mode >> 1) slots
    uint64_t out_off;
};

// Output destination.
// Output destination.  Work items with exact offsets write there directly.  Items whose offset is
// kClaimOffset (the learned path, where exact counts are not known in advance) claim a range
// from *cursor once their count is known; a claim that would pass `capacity`, or an item whose
// accumulator overflowed, writes nothing and is appended to fail_list for an exact rerun.
constexpr uint64_t kClaimOffset = ~0ull;

struct OutputView {
    uint32_t* idx = nullptr;        // [capacity * (fa + fb)]
    double* val = nullptr;          // [capacity]
    uint64_t* cursor = nullptr;     // next free entry (claim mode)
    uint64_t capacity = 0;          // entries available (claim mode)
    uint32_t* fail_list = nullptr;  // items to rerun exactly
    uint32_t* fail_count = nullptr;
    uint32_t* item_count = nullptr; // optional: entries written by each item
};

// Claim `n` entries at the output cursor without passing the capacity; ~0 if they do not fit.
__device__ __forceinline__ uint64_t claim_output(const OutputView& out, uint64_t n) {
    unsigned long long cur = *reinterpret_cast<volatile unsigned long long*>(out.cursor);
    for (int tries = 0; tries < (1 << 20); ++tries) {
        if (cur + n > out.capacity) return ~0ull;
        const unsigned long long prev =
            atomicCAS(reinterpret_cast<unsigned long long*>(out.cursor), cur, cur + n);
        if (prev == cur) return cur;
        cur = prev;
    }
    return ~0ull;
}

void launch_pack_keys(const uint32_t* idx, uint64_t nnz, const DimSpec& dims, const KeySpec& k1,
                      const KeySpec& k2, uint64_t* key1, uint64_t* key2, uint32_t* err, cudaStream_t st);

}  // namespace ptc
