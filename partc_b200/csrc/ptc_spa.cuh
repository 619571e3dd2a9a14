// Accumulator kernels (ptc_spa.cu) and the planning kernels that feed them (ptc_plan.cu).
#pragma once

#include "ptc_internal.cuh"

namespace ptc {

// rows with at most this many products go to the one-warp-per-row kernel
uint32_t small_row_max_flops();
// largest exact output count one hash part may hold
uint32_t hash_part_capacity();
// largest column count the bitmap symbolic pass handles
uint32_t sym_bitmap_max_cols();

// small rows: symbolic (row_d[row] = output nnz) or numeric (writes at row_off[row])
void launch_small_rows(bool numeric, const Operands& op, const uint32_t* rows, uint32_t nrows, uint64_t* row_d,
                       const uint64_t* row_off, const OutputView& out, cudaStream_t st);

// other rows, symbolic: panel_cnt[i * npanels + p] = output nnz of rows[i] in fine panel p;
// row_d[rows[i]] += the row's total (row_d must start at 0 for these rows)
void launch_sym_bitmap(const Operands& op, const uint32_t* rows, uint32_t nrows, uint32_t* panel_cnt, uint64_t* row_d,
                       uint32_t* work_counter, int num_sms, cudaStream_t st);

// other rows, numeric: one block per part
void launch_hash_parts(const Operands& op, const PartItem* parts, uint32_t nparts, const OutputView& out,
                       uint32_t* work_counter, uint32_t* overflow, int num_sms, cudaStream_t st);

// ---- planning (ptc_plan.cu) ----

// class_of[r]: 0 = no products, 1 = small, 2 = other; flags for the two compactions
void launch_classify_rows(const uint64_t* row_flops, uint64_t nrows, uint64_t small_max, uint32_t* small_flag,
                          uint32_t* big_flag, cudaStream_t st);
// out[pos[i]] = i wherever flag[i] (pos = exclusive scan of flag)
void launch_compact_indices(const uint32_t* flag, const uint32_t* pos, uint64_t n, uint32_t* out, cudaStream_t st);
// key[i] = ~row_flops[rows[i]] (descending-work sort key)
void launch_work_keys(const uint32_t* rows, uint64_t n, const uint64_t* row_flops, uint64_t* key, cudaStream_t st);
// number of parts of each big row under the capacity (greedy over fine panels, in order);
// sets *oversize if one fine panel alone exceeds the capacity
void launch_count_parts(const uint32_t* panel_cnt, uint64_t nbig, uint32_t npanels, uint32_t cap, uint32_t* nparts,
                        uint32_t* oversize, cudaStream_t st);
void launch_fill_parts(const uint32_t* rows, const uint32_t* panel_cnt, uint64_t nbig, uint32_t npanels, uint32_t cap,
                       const uint32_t* part_pos, const uint64_t* row_off, PartItem* parts, cudaStream_t st);

}  // namespace ptc
