// Large rows of a single contraction, one block per row over a bitmap of the row's columns in
// shared memory (ptc_rowmap.cu).
#pragma once

#include "ptc_internal.cuh"

namespace ptc {

enum RowmapMode {
    kRowmapCount = 0,  // row_d[rows[i]] = the row's exact output count
    kRowmapExact = 1,  // write the row's entries at row_off[rows[i]]
    kRowmapClaim = 2   // take the row's range at out.cursor once its count is known; a row that does
                       // not fit out.capacity writes nothing and lists i in out.fail_list; every
                       // row's exact count goes to out.item_count[i]
};

// largest column count (distinct B free keys) the kernel takes
uint64_t rowmap_max_cols();

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
