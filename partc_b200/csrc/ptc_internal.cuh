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
    // batches (null for a single contraction): column ids are local to each item; row_item[row]
    // is the row's item and item_out[item] says where that item's output and columns start
    const uint32_t* row_item = nullptr;
    const struct ItemOut* item_out = nullptr;
    const uint32_t* item_cols = nullptr;  // columns of each item (its local column ids are below this)
};

// One item of a batch inside an output block.  Entry e of the item (e >= ent0, in the batch's entry
// numbering) has its value at val[val0 + (e - ent0)] and its fa + fb indices at
// idx[idx0 + (e - ent0) * (fa + fb)], so every item's output is one compact tensor of its own order.
struct ItemOut {
    uint64_t ent0;
    uint64_t val0;
    uint64_t idx0;
    uint32_t colbase;  // first global column (row of col_tuple) of the item
    uint32_t fa, fb;   // the item's free-mode counts (Operands::fa/fb are the batch maxima)
    uint32_t pad;
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

// Output destination.  Work items with exact offsets write there directly.  Items whose offset is
// kClaimBit (the learned path, where exact counts are not known in advance) take a range at their
// item's cursor with one atomicAdd once their count is known.  The claims of an item succeed in
// atomic order until one would pass the item's end; that claim and every later one fail, so the
// successful claims fill [start, cursor - overshoot) without gaps.  A failed item, or one whose
// accumulator overflowed, writes nothing and is appended to fail_list for an exact rerun.
constexpr uint64_t kClaimBit = 1ull << 63;

struct OutputView {
    uint32_t* idx = nullptr;            // output index tuples
    double* val = nullptr;              // output values
    uint64_t* cursor = nullptr;         // claim mode: next entry of each item
    uint64_t* overshoot = nullptr;      // claim mode: entries of each item's failed claims
    const uint64_t* cap_end = nullptr;  // claim mode: end of each item's range (null: `capacity`)
    uint64_t capacity = 0;              // claim mode, single contraction: entries available
    uint32_t* fail_list = nullptr;      // work items to rerun exactly
    uint32_t* fail_count = nullptr;
    uint32_t* item_count = nullptr;     // optional: entries written by each work item
    uint32_t* row_of = nullptr;         // optional (canonical order): row of every entry
    uint32_t* col_of = nullptr;         // optional (canonical order): column of every entry
};

// Take `n` entries at the cursor of the row's item; ~0 if they pass the item's end.  An
// atomicAdd, not a compare-and-swap loop: one L2 operation per claim however many blocks claim
// at once.
__device__ __forceinline__ uint64_t claim_output(const Operands& op, const OutputView& out, uint32_t row, uint64_t n) {
    const uint32_t item = op.row_item ? op.row_item[row] : 0u;
    const unsigned long long old =
        atomicAdd(reinterpret_cast<unsigned long long*>(out.cursor + item), (unsigned long long)n);
    const uint64_t end = out.cap_end ? out.cap_end[item] : out.capacity;
    if (old + n <= end) return (uint64_t)old;
    atomicAdd(reinterpret_cast<unsigned long long*>(out.overshoot + item), (unsigned long long)n);
    return ~0ull;
}

// Write output entry o = (row's A free tuple, column's B free tuple, value); `col` is local to
// the row's item.
__device__ __forceinline__ void write_entry(const Operands& op, const OutputView& out, uint64_t o, uint32_t row,
                                            uint32_t col, double v) {
    const uint32_t fa = op.fa, fb = op.fb;
    if (op.row_item) {
        const ItemOut io = op.item_out[op.row_item[row]];
        col += io.colbase;
        uint32_t* dst = out.idx + io.idx0 + (o - io.ent0) * (io.fa + io.fb);
        for (uint32_t m = 0; m < io.fa; ++m) dst[m] = op.row_tuple[(uint64_t)row * fa + m];
        for (uint32_t m = 0; m < io.fb; ++m) dst[io.fa + m] = op.col_tuple[(uint64_t)col * fb + m];
        out.val[io.val0 + (o - io.ent0)] = v;
        return;
    }
    const uint32_t od = fa + fb;
    uint32_t* dst = out.idx + o * od;
    if (out.row_of) {
        out.row_of[o] = row;
        out.col_of[o] = col;
    }
    if (fa == 2 && fb == 2) {
        const uint2 r = *reinterpret_cast<const uint2*>(op.row_tuple + (uint64_t)row * 2);
        const uint2 c = *reinterpret_cast<const uint2*>(op.col_tuple + (uint64_t)col * 2);
        *reinterpret_cast<uint4*>(dst) = make_uint4(r.x, r.y, c.x, c.y);
    } else if (fa == 1 && fb == 1) {
        *reinterpret_cast<uint2*>(dst) = make_uint2(op.row_tuple[row], op.col_tuple[col]);
    } else {
        for (uint32_t m = 0; m < fa; ++m) dst[m] = op.row_tuple[(uint64_t)row * fa + m];
        for (uint32_t m = 0; m < fb; ++m) dst[fa + m] = op.col_tuple[(uint64_t)col * fb + m];
    }
    out.val[o] = v;
}

void launch_pack_keys(const uint32_t* idx, uint64_t nnz, const DimSpec& dims, const KeySpec& k1,
                      const KeySpec& k2, uint64_t* key1, uint64_t* key2, uint32_t* err, cudaStream_t st);

}  // namespace ptc
