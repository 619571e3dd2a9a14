// Build-side kernel launchers (ptc_build.cu).
#pragma once

#include "ptc_internal.cuh"

namespace ptc {

void launch_iota(uint32_t* out, uint64_t n, cudaStream_t st);
void launch_scatter_u32(const uint32_t* src, const uint32_t* perm, uint64_t n, uint32_t* dst, cudaStream_t st);
template <typename T>
void launch_gather(const T* src, const uint32_t* perm, uint64_t n, T* dst, cudaStream_t st);
void launch_composite(const uint64_t* hi, const uint32_t* lo, uint64_t radix, uint64_t n, uint64_t* out,
                      cudaStream_t st);
void launch_tuples(const uint32_t* idx, uint32_t order, const uint32_t* run_start, const uint32_t* perm, uint64_t nruns,
                   const KeySpec& ks, uint32_t* tuple, cudaStream_t st);
void launch_fiber_len(const int32_t* a_fib, const uint32_t* fib_start, uint64_t n, uint64_t* len, cudaStream_t st);
void launch_row_flops(const uint64_t* poff, const uint32_t* row_start, uint64_t nrows, uint64_t* flops,
                      cudaStream_t st);
void launch_panel_offsets(const uint32_t* b_col, const uint32_t* b_fib, const uint32_t* fib_start, uint64_t nb,
                          uint32_t P, uint32_t log2w, uint32_t* off, cudaStream_t st);

}  // namespace ptc
