// Large rows of a single contraction, one block per row over a bitmap of the row's columns in
// shared memory (ptc_rowmap.cu).
#pragma once

#include "ptc_internal.cuh"

namespace ptc {

enum RowmapMode {
    kRowmapCount = 0,  // row_d[rows[i]] += the row's exact output count
    kRowmapExact = 1,  // write the row's entries at row_off[rows[i]]
    kRowmapClaim = 2   // take the row's range at out.cursor once its count is known; a row that does
                       // not fit out.capacity writes nothing and lists i in out.fail_list; every
                       // row's exact count goes to out.item_count[i]
};

// largest column count (distinct B free keys) the kernel takes
uint64_t rowmap_max_cols();
// largest column count of its count mode (one bitmap: about 1.8M columns)
uint64_t row_counts_max_cols();

// The exact symbolic pass of rows `rows` by the kernel's count mode (one bitmap of the row's
// columns, no values): row_d[rows[i]] += the row's output count and, with panel_cnt given, its
// count in every fine panel at panel_cnt[pbase[i] + p] (pbase null: i * npanels + p).  Panels
// must be at least 32 columns wide.
void launch_row_counts(const Operands& op, const uint32_t* rows, uint32_t nrows, uint32_t* panel_cnt,
                       const uint64_t* pbase, uint64_t* row_d, uint32_t* work_counter, int num_sms, cudaStream_t st);

// Rows `rows` (heaviest first is best), one block each.  Entries of a row come out in column
// order; values are bit-identical to the reference's left fold in COO order.
void launch_rowmap(int mode, const Operands& op, const uint32_t* rows, uint32_t nrows, uint64_t* row_d,
                   const uint64_t* row_off, const OutputView& out, uint32_t* work_counter, int num_sms,
                   cudaStream_t st);

// flag[i] = 1 unless rows[i]'s exact output count equals its products (collision-free rows need
// no accumulator)
void launch_table_row_flags(const uint32_t* rows, uint64_t n, const uint64_t* row_off, const uint64_t* row_flops,
                            uint32_t* flag, cudaStream_t st);
// row_actual[rows[i]] = cnt[i]
void launch_scatter_counts(const uint32_t* rows, uint64_t n, const uint32_t* cnt, uint64_t* row_actual,
                           cudaStream_t st);

// key[i] = the wave (of nwaves, starting at rows wave_row[]) holding rows[i]; idx[i] = i
void launch_row_wave(const uint32_t* rows, uint32_t n, const uint32_t* wave_row, uint32_t nwaves, uint64_t* key,
                     uint32_t* idx, cudaStream_t st);

}  // namespace ptc
