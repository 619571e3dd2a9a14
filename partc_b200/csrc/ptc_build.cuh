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
void launch_panel_offsets(const uint32_t* b_col, const uint32_t* fib_start, uint64_t nfib, uint32_t P, uint32_t log2w,
                          uint32_t* off, cudaStream_t st);

// key[i] = rows[i]
void launch_row_keys(const uint32_t* rows, uint64_t n, uint64_t* key, cudaStream_t st);

// ---- canonical output order ----
void launch_entry_keys(const uint32_t* row_of, const uint32_t* col_of, uint64_t n, uint32_t colbits, uint64_t* key,
                       uint32_t* perm, cudaStream_t st);
void launch_gather_tuples(const uint32_t* src, const uint32_t* perm, uint64_t n, uint32_t od, uint32_t* dst,
                          cudaStream_t st);

// ---- batches ----

// One side (A = 0, B = 1) of a batch item, as the device reads it: the item's COO arrays, its modes
// (contracted first, then free in output order), their sizes, the strides that linearize them
// (contracted key, then free key) and the base of its free-key range.
struct ItemSide {
    const uint32_t* idx;  // [nnz * order], device memory
    const double* vals;   // [nnz], device memory
    uint64_t fbase;       // free keys of this item are fbase + [0, free key space)
    uint32_t order;
    uint32_t pad;
    uint32_t mode[kMaxOrder];
    uint32_t dim[kMaxOrder];
    uint64_t stride[kMaxOrder];
};

struct ItemSpec {
    uint64_t cbase;  // contracted keys of this item are cbase + [0, contracted key space)
    uint32_t c;
    uint32_t pad;
    ItemSide side[2];
};

void launch_pack_items(const ItemSpec* specs, const uint64_t* off, uint32_t nitems, int side, uint64_t nnz,
                       uint64_t* ckey, uint64_t* fkey, double* vals, uint32_t* err, cudaStream_t st);
void launch_item_tuples(const uint32_t* run_start, const uint32_t* perm, uint64_t nruns, const ItemSpec* specs,
                        const uint64_t* off, uint32_t nitems, int side, uint32_t width, uint32_t* tuple,
                        cudaStream_t st);
void launch_key_bounds(const uint64_t* keys, uint64_t n, const uint64_t* base, uint32_t nitems, uint32_t* first,
                       cudaStream_t st);
void launch_localize(const uint32_t* global, uint64_t n, const uint64_t* off, uint32_t nitems, const uint32_t* first,
                     uint32_t* local, cudaStream_t st);
void launch_row_item(uint64_t nrows, const uint32_t* first, uint32_t nitems, uint32_t* row_item, cudaStream_t st);

}  // namespace ptc
