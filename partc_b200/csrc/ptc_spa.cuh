// Accumulator kernels (ptc_spa.cu) and the planning kernels that feed them (ptc_plan.cu).
#pragma once

#include "ptc_internal.cuh"

namespace ptc {

// rows with at most this many products go to the one-warp-per-row kernel
uint32_t small_row_max_flops();
// largest exact output count one open-addressing part may hold
uint32_t hash_part_capacity();
// column width of a dense (direct-mapped) part
uint32_t dense_part_columns();
// smallest open-addressing table (log2 slots) a part uses
uint32_t hash_part_min_bits();

// small rows: symbolic (row_d[row] = output nnz) or numeric (writes at row_off[row])
void launch_small_rows(bool numeric, const Operands& op, const uint32_t* rows, uint32_t nrows, uint64_t* row_d,
                       const uint64_t* row_off, const OutputView& out, cudaStream_t st);

// other rows, symbolic: panel_cnt[pbase[i] + p] (pbase null: i * npanels + p) = output nnz of
// rows[i] in fine panel p; row_d[rows[i]] += the row's total (row_d must start at 0 for these rows)
void launch_sym_bitmap(const Operands& op, const uint32_t* rows, uint32_t nrows, uint32_t* panel_cnt,
                       const uint64_t* pbase, uint64_t* row_d, uint32_t* work_counter, int num_sms, cudaStream_t st);

// largest exact output count of a sparse warp task, and its table bounds (log2 slots)
uint32_t warp_task_capacity();
uint32_t warp_task_min_bits();
uint32_t warp_task_max_bits();
// column width of a dense warp task
uint32_t warp_task_dense_columns();
// rows whose A nonzeros number at most this go to warp tasks (they rescan the row once per task)
constexpr uint32_t kWarpTaskMaxLen = 256;

// other rows, numeric: one warp per task (a row's columns in fine panels [p0, p1))
void launch_warp_tasks(const Operands& op, const PartItem* tasks, uint32_t ntasks, const OutputView& out,
                       uint32_t* work_counter, uint32_t* overflow, int num_sms, cudaStream_t st);

// collision-free large rows (exact output count = products), numeric: each product an entry;
// alen = exclusive scan of the A nonzeros' fiber lengths, row_off the rows' exact offsets
void launch_copy_rows(const Operands& op, const uint32_t* rows, uint32_t nrows, const uint64_t* alen,
                      const uint64_t* row_off, const OutputView& out, int num_sms, cudaStream_t st);

// other rows, numeric: one block per part
void launch_hash_parts(const Operands& op, const PartItem* parts, uint32_t nparts, const OutputView& out,
                       uint32_t* work_counter, uint32_t* overflow, int num_sms, cudaStream_t st);

// ---- planning (ptc_plan.cu) ----

// Row classes: no products (skipped), small (<= small_max products: one warp), sort-based
// (fewer than esc_avg products per A nonzero on average), other (block hash).  One flag array
// per class for the compactions.
void launch_classify_rows(const uint64_t* row_flops, const uint32_t* row_start, uint64_t nrows, uint64_t small_max,
                          uint32_t esc_avg, uint32_t* small_flag, uint32_t* big_flag, uint32_t* esc_flag,
                          cudaStream_t st);
// big_flag[r] |= esc_flag[r] (sort-based rows fall back to the hash path)
void launch_merge_flags(uint32_t* big_flag, const uint32_t* esc_flag, uint64_t nrows, cudaStream_t st);

// ---- sort-based rows (ptc_esc.cu) ----
void launch_esc_index(const uint32_t* esc_rows, uint64_t n, int32_t* esc_of, cudaStream_t st);
void launch_esc_len(const uint32_t* esc_rows, uint64_t n, const uint64_t* row_flops, uint64_t* len, cudaStream_t st);
void launch_esc_expand(const Operands& op, const uint32_t* a_row, const int32_t* esc_of, const uint64_t* poff,
                       const uint64_t* esc_off, uint32_t colbits, uint64_t* key, double* val, uint32_t* perm,
                       cudaStream_t st);
void launch_esc_count(const uint64_t* run_key, uint64_t nruns, uint32_t colbits, const uint32_t* esc_rows,
                      uint64_t* row_d, uint32_t* first_run, cudaStream_t st);
// sorted[i] = val[perm[i]] for the nprod sorted products
void launch_esc_gather(const uint32_t* perm, const double* val, uint64_t nprod, double* sorted, cudaStream_t st);
// runs of at least this many products are folded by a block each (esc_fold_long_kernel)
constexpr uint32_t kEscLongMin = 16384;
// flag[r] = 1 for the runs of at least kEscLongMin products
void launch_esc_long_flags(const uint32_t* run_start, uint64_t nruns, uint32_t* flag, cudaStream_t st);
// runs [r0, r1) of the sorted products: one output entry each; long_runs[0, n_long) are the long
// runs among them (the other runs fold one per thread)
void launch_esc_fold(const Operands& op, const OutputView& out, const uint64_t* run_key, const uint32_t* run_start,
                     uint64_t r0, uint64_t r1, uint32_t colbits, const uint32_t* esc_rows, const uint32_t* first_run,
                     const uint64_t* row_off, const double* sorted, const uint32_t* long_runs, uint32_t n_long,
                     cudaStream_t st);
// out[pos[i]] = i wherever flag[i] (pos = exclusive scan of flag)
void launch_compact_indices(const uint32_t* flag, const uint32_t* pos, uint64_t n, uint32_t* out, cudaStream_t st);
// key[i] = group << 40 | ~row_flops[rows[i]] (low 40 bits), group 0 for rows of at most map_len
// A nonzeros (the row bitmap kernel), 1 up to max_len (warp tasks), 2 above (block parts):
// sorted, the groups come in that order, each largest first
void launch_work_keys(const uint32_t* rows, uint64_t n, const uint64_t* row_flops, const uint32_t* row_start,
                      uint32_t map_len, uint32_t max_len, uint64_t* key, cudaStream_t st);

// How a large row is cut into parts, from its exact output count per fine panel: windows of
// dense_panels panels holding at least dense_min entries per panel become dense parts; the
// other panels are grouped greedily into open-addressing parts of at most cap entries.
struct SplitRule {
    uint32_t cap;
    uint32_t dense_panels;  // 0 disables dense parts
    uint32_t dense_min;
    uint32_t min_bits;      // smallest open-addressing table, log2 slots
    uint32_t max_bits;      // largest open-addressing table, log2 slots
    uint32_t oversize_dense;  // 1: a single panel above cap becomes a dense part (else an error)
    uint32_t load_num, load_den;  // open-addressing tables at most load_num / load_den full
};
// number of parts of each big row; sets *oversize if one fine panel alone exceeds cap.  Row i's
// panel counts are panel_cnt[pbase[i] .. pbase[i+1]), or panel_cnt[i * npanels ..] with pbase null.
// With row_off and row_flops given (exact sizes), rows whose output count equals their products
// get no parts (the collision-free rows, written by launch_copy_rows).
void launch_count_parts(const uint32_t* rows, const uint32_t* panel_cnt, const uint64_t* pbase, uint64_t nbig,
                        uint32_t npanels, SplitRule rule, const uint64_t* row_off, const uint64_t* row_flops,
                        uint32_t* nparts, uint32_t* oversize, cudaStream_t st);
// flag[i] = 1 if rows[i]'s exact output count equals its products
void launch_copy_flags(const uint32_t* rows, uint64_t n, const uint64_t* row_off, const uint64_t* row_flops,
                       uint32_t* flag, cudaStream_t st);
void launch_fill_parts(const uint32_t* rows, const uint32_t* panel_cnt, const uint64_t* pbase, uint64_t nbig,
                       uint32_t npanels, SplitRule rule, const uint32_t* part_pos, const uint64_t* row_off,
                       const uint64_t* row_flops, PartItem* parts, cudaStream_t st);
// np[i] = panels of rows[i]'s item (a batch): ceil(item_cols[row_item[row]] / 2^log2w), at least 1
void launch_row_panel_counts(const uint32_t* rows, uint64_t n, const uint32_t* row_item, const uint32_t* item_cols,
                             uint32_t log2w, uint64_t* np, cudaStream_t st);

}  // namespace ptc
