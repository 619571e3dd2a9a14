// Learned path: planning from sizer predictions and exact reruns (ptc_learned.cu, ptc_plan.cu).
#pragma once

#include "ptc_sizer.cuh"
#include "ptc_spa.cuh"

namespace ptc {

// Per-panel predicted counts of the large rows (batches: row_item/item_cols give each row's item
// and that item's column count, `is` its own panel shares; null for a single contraction).
void launch_predicted_panel_counts(const uint32_t* rows, uint64_t n, const uint64_t* row_flops, const float* pred,
                                   const float* gp, const uint32_t* row_item, const uint32_t* item_cols,
                                   const uint64_t* pbase, uint32_t P, uint32_t panel_log2, uint64_t ncols, float margin,
                                   uint32_t* cnt, Arena& ar, const ItemStats* is = nullptr);
// *out = sum of x[0..n)
void launch_sum_u32(const uint32_t* x, uint64_t n, uint64_t* out, cudaStream_t st);
void launch_gather_parts(const PartItem* parts, const uint32_t* idx, uint32_t n, PartItem* out, cudaStream_t st);
void launch_row_actual(const PartItem* parts, const uint32_t* counts, uint32_t n, uint64_t* row_actual,
                       cudaStream_t st);
void launch_log2_error(const uint32_t* rows, uint64_t n, const float* pred, const uint64_t* row_actual, double* out,
                       cudaStream_t st);

// Exact re-split of failed parts: part i covers panels [parts[i].p0, parts[i].p1) of row
// parts[i].row, whose exact panel counts are panel_cnt[ridx[i] * P ...].  nparts[i] = number of
// new parts; fill writes them with claim offsets.  total[i] = exact entries of part i.
void launch_count_parts_range(const PartItem* parts, const uint32_t* ridx, uint32_t n, const uint32_t* panel_cnt,
                              uint32_t P, SplitRule rule, uint32_t* nparts, uint32_t* total, cudaStream_t st);
void launch_fill_parts_range(const PartItem* parts, const uint32_t* ridx, uint32_t n, const uint32_t* panel_cnt,
                             uint32_t P, SplitRule rule, const uint32_t* part_pos, PartItem* out, cudaStream_t st);

// Claim budgets of the learned path: budget[big_rows[i]] = sum of the row's predicted panel counts.
void launch_claim_budgets(const uint32_t* big_rows, uint64_t n_big, const uint32_t* panel_cnt, const uint64_t* pbase,
                          uint32_t P, uint64_t* budget, cudaStream_t st);
// row_off[r] += claim_off[row_first[row_item[r]]] for every row
void launch_shift_exact(uint64_t nrows, const uint32_t* row_item, const uint32_t* row_first, const uint64_t* claim_off,
                        uint64_t* row_off, cudaStream_t st);
// key[i] = wave of part i (waves start at rows wave_row[0..nwaves)), idx[i] = i
void launch_part_wave(const PartItem* parts, uint32_t n, const uint32_t* wave_row, uint32_t nwaves, uint64_t* key,
                      uint32_t* idx, cudaStream_t st);

}  // namespace ptc
