// Build-side kernels: key linearization, gathers, index tuples, panel split of the fibers.
#include "ptc_build.cuh"

namespace ptc {

// One thread per nonzero: range-check every index (the reference trusts its input; an index
// beyond its mode would corrupt the keys) and linearize the two mode tuples.
__global__ void pack_keys_kernel(const uint32_t* __restrict__ idx, uint64_t nnz, DimSpec dims, KeySpec k1,
                                 KeySpec k2, uint64_t* __restrict__ key1, uint64_t* __restrict__ key2,
                                 uint32_t* __restrict__ err, bool vec4) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nnz) return;
    const uint32_t d = dims.order;
    const uint32_t* row = idx + i * d;
    uint32_t v[kMaxOrder];
    bool bad = false;
    if (vec4) {
        const uint4 q = *reinterpret_cast<const uint4*>(row);
        v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
    } else {
        for (uint32_t m = 0; m < d; ++m) v[m] = row[m];
    }
    for (uint32_t m = 0; m < d; ++m) bad |= v[m] >= dims.dim[m];
    if (bad) {
        atomicOr(err, 1u);
        return;
    }
    uint64_t a = 0, b = 0;
    for (uint32_t j = 0; j < k1.n; ++j) a += (uint64_t)v[k1.mode[j]] * k1.stride[j];
    for (uint32_t j = 0; j < k2.n; ++j) b += (uint64_t)v[k2.mode[j]] * k2.stride[j];
    if (key1) key1[i] = a;
    if (key2) key2[i] = b;
}

void launch_pack_keys(const uint32_t* idx, uint64_t nnz, const DimSpec& dims, const KeySpec& k1, const KeySpec& k2,
                      uint64_t* key1, uint64_t* key2, uint32_t* err, cudaStream_t st) {
    if (nnz == 0) return;
    const bool vec4 = dims.order == 4 && (reinterpret_cast<uintptr_t>(idx) & 15u) == 0;
    pack_keys_kernel<<<ceil_div_u32(nnz, 256), 256, 0, st>>>(idx, nnz, dims, k1, k2, key1, key2, err, vec4);
    count_launch();
    PTC_CHECK_LAUNCH();
}

__global__ void iota_kernel(uint32_t* __restrict__ out, uint64_t n) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (uint32_t)i;
}

void launch_iota(uint32_t* out, uint64_t n, cudaStream_t st) {
    if (n == 0) return;
    iota_kernel<<<ceil_div_u32(n, 256), 256, 0, st>>>(out, n);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// dst[perm[i]] = src[i]
__global__ void scatter_u32_kernel(const uint32_t* __restrict__ src, const uint32_t* __restrict__ perm, uint64_t n,
                                   uint32_t* __restrict__ dst) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[perm[i]] = src[i];
}

void launch_scatter_u32(const uint32_t* src, const uint32_t* perm, uint64_t n, uint32_t* dst, cudaStream_t st) {
    if (n == 0) return;
    scatter_u32_kernel<<<ceil_div_u32(n, 256), 256, 0, st>>>(src, perm, n, dst);
    count_launch();
    PTC_CHECK_LAUNCH();
}

template <typename T>
__global__ void gather_kernel(const T* __restrict__ src, const uint32_t* __restrict__ perm, uint64_t n,
                              T* __restrict__ dst) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[perm[i]];
}

template <typename T>
void launch_gather(const T* src, const uint32_t* perm, uint64_t n, T* dst, cudaStream_t st) {
    if (n == 0) return;
    gather_kernel<T><<<ceil_div_u32(n, 256), 256, 0, st>>>(src, perm, n, dst);
    count_launch();
    PTC_CHECK_LAUNCH();
}
template void launch_gather<uint32_t>(const uint32_t*, const uint32_t*, uint64_t, uint32_t*, cudaStream_t);
template void launch_gather<uint64_t>(const uint64_t*, const uint32_t*, uint64_t, uint64_t*, cudaStream_t);
template void launch_gather<double>(const double*, const uint32_t*, uint64_t, double*, cudaStream_t);

// composite[i] = key_hi[i] * radix + lo[i]
__global__ void composite_kernel(const uint64_t* __restrict__ hi, const uint32_t* __restrict__ lo, uint64_t radix,
                                 uint64_t n, uint64_t* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = hi[i] * radix + lo[i];
}

void launch_composite(const uint64_t* hi, const uint32_t* lo, uint64_t radix, uint64_t n, uint64_t* out,
                      cudaStream_t st) {
    if (n == 0) return;
    composite_kernel<<<ceil_div_u32(n, 256), 256, 0, st>>>(hi, lo, radix, n, out);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// tuple[r * nm + j] = idx[src[r] * order + mode[j]] for every run r (src = a representative
// nonzero of the run, in original numbering).
__global__ void tuples_kernel(const uint32_t* __restrict__ idx, uint32_t order, const uint32_t* __restrict__ run_start,
                              const uint32_t* __restrict__ perm, uint64_t nruns, KeySpec ks,
                              uint32_t* __restrict__ tuple) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nruns) return;
    const uint64_t src = perm[run_start[r]];
    for (uint32_t j = 0; j < ks.n; ++j) tuple[r * ks.n + j] = idx[src * order + ks.mode[j]];
}

void launch_tuples(const uint32_t* idx, uint32_t order, const uint32_t* run_start, const uint32_t* perm, uint64_t nruns,
                   const KeySpec& ks, uint32_t* tuple, cudaStream_t st) {
    if (nruns == 0 || ks.n == 0) return;
    tuples_kernel<<<ceil_div_u32(nruns, 256), 256, 0, st>>>(idx, order, run_start, perm, nruns, ks, tuple);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// Per A nonzero (row-sorted): length of its matching fiber (0 if none).
__global__ void fiber_len_kernel(const int32_t* __restrict__ a_fib, const uint32_t* __restrict__ fib_start, uint64_t n,
                                 uint64_t* __restrict__ len) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t f = a_fib[i];
    len[i] = f >= 0 ? (uint64_t)(fib_start[f + 1] - fib_start[f]) : 0ull;
}

void launch_fiber_len(const int32_t* a_fib, const uint32_t* fib_start, uint64_t n, uint64_t* len, cudaStream_t st) {
    if (n == 0) return;
    fiber_len_kernel<<<ceil_div_u32(n, 256), 256, 0, st>>>(a_fib, fib_start, n, len);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// Per row: flops = poff[row_end] - poff[row_start].
__global__ void row_flops_kernel(const uint64_t* __restrict__ poff, const uint32_t* __restrict__ row_start,
                                 uint64_t nrows, uint64_t* __restrict__ flops) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nrows) flops[r] = poff[row_start[r + 1]] - poff[row_start[r]];
}

void launch_row_flops(const uint64_t* poff, const uint32_t* row_start, uint64_t nrows, uint64_t* flops,
                      cudaStream_t st) {
    if (nrows == 0) return;
    row_flops_kernel<<<ceil_div_u32(nrows, 256), 256, 0, st>>>(poff, row_start, nrows, flops);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// Dense-panel split of every fiber (B sorted by fiber, then column):
// off[f * (P + 1) + p] = first entry j of fiber f with b_col[j] >= p << log2w (fiber end if none).
// One thread per table entry (consecutive threads write consecutive entries): a binary search in
// the fiber, whose columns the neighbouring threads read too.
__global__ void panel_offsets_kernel(const uint32_t* __restrict__ b_col, const uint32_t* __restrict__ fib_start,
                                     uint64_t nfib, uint32_t P, uint32_t log2w, uint32_t* __restrict__ off) {
    const uint64_t n = nfib * (P + 1);
    for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t f = x / (P + 1);
        const uint32_t p = (uint32_t)(x - f * (P + 1));
        uint32_t lo = fib_start[f], hi = fib_start[f + 1];
        const uint64_t c = (uint64_t)p << log2w;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (b_col[mid] < c) lo = mid + 1; else hi = mid;
        }
        off[x] = lo;
    }
}

void launch_panel_offsets(const uint32_t* b_col, const uint32_t* fib_start, uint64_t nfib, uint32_t P, uint32_t log2w,
                          uint32_t* off, cudaStream_t st) {
    if (nfib == 0) return;
    const uint64_t n = nfib * (P + 1);
    const uint32_t grid = (uint32_t)std::min<uint64_t>((n + 255) / 256, 148ull * 64);
    panel_offsets_kernel<<<grid, 256, 0, st>>>(b_col, fib_start, nfib, P, log2w, off);
    count_launch();
    PTC_CHECK_LAUNCH();
}

}  // namespace ptc

namespace ptc {

// key[i] = rows[i] (as a 64-bit sort key)
__global__ void row_keys_kernel(const uint32_t* __restrict__ rows, uint64_t n, uint64_t* __restrict__ key) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) key[i] = rows[i];
}

void launch_row_keys(const uint32_t* rows, uint64_t n, uint64_t* key, cudaStream_t st) {
    if (n == 0) return;
    row_keys_kernel<<<ceil_div_u32(n, 256), 256, 0, st>>>(rows, n, key);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// canonical output order: key[e] = row_of[e] << colbits | col_of[e], perm[e] = e
__global__ void entry_keys_kernel(const uint32_t* __restrict__ row_of, const uint32_t* __restrict__ col_of, uint64_t n,
                                  uint32_t colbits, uint64_t* __restrict__ key, uint32_t* __restrict__ perm) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    key[e] = ((uint64_t)row_of[e] << colbits) | col_of[e];
    perm[e] = (uint32_t)e;
}

void launch_entry_keys(const uint32_t* row_of, const uint32_t* col_of, uint64_t n, uint32_t colbits, uint64_t* key,
                       uint32_t* perm, cudaStream_t st) {
    if (n == 0) return;
    entry_keys_kernel<<<ceil_div_u32(n, 256), 256, 0, st>>>(row_of, col_of, n, colbits, key, perm);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// dst tuple e = src tuple perm[e] (od u32 each)
__global__ void gather_tuples_kernel(const uint32_t* __restrict__ src, const uint32_t* __restrict__ perm, uint64_t n,
                                     uint32_t od, uint32_t* __restrict__ dst) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const uint64_t s = perm[e];
    for (uint32_t m = 0; m < od; ++m) dst[e * od + m] = src[s * od + m];
}

void launch_gather_tuples(const uint32_t* src, const uint32_t* perm, uint64_t n, uint32_t od, uint32_t* dst,
                          cudaStream_t st) {
    if (n == 0) return;
    gather_tuples_kernel<<<ceil_div_u32(n, 256), 256, 0, st>>>(src, perm, n, od, dst);
    count_launch();
    PTC_CHECK_LAUNCH();
}

}  // namespace ptc

namespace ptc {

// ---------------------------------------------------------------------------------------------
// batches: every item keeps its own mode lists and key range (ItemSpec, ptc_build.cuh)
// ---------------------------------------------------------------------------------------------

// Last item whose first element (off[item]) is <= i; off has nitems + 1 entries.
__device__ __forceinline__ uint32_t item_of(const uint64_t* __restrict__ off, uint32_t nitems, uint64_t i) {
    uint32_t lo = 0, hi = nitems;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (off[mid] <= i) lo = mid; else hi = mid;
    }
    return lo;
}

// Element i of the side's concatenation (item it, local nonzero i - off[it]): its contracted key
// cbase + sum idx[mode[j]] * stride[j] over the contracted modes, its free key fbase + the same
// over the free modes, and its value.
__global__ void pack_items_kernel(const ItemSpec* __restrict__ specs, const uint64_t* __restrict__ off,
                                  uint32_t nitems, int side, uint64_t nnz, uint64_t* __restrict__ ckey,
                                  uint64_t* __restrict__ fkey, double* __restrict__ vals, uint32_t* __restrict__ err) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nnz) return;
    const uint32_t it = item_of(off, nitems, i);
    const ItemSide& s = specs[it].side[side];
    const uint32_t d = s.order;
    const uint64_t local = i - off[it];
    const uint32_t* row = s.idx + local * d;
    uint32_t v[kMaxOrder];
    bool bad = false;
    for (uint32_t m = 0; m < d; ++m) {
        v[m] = row[m];
        bad |= v[m] >= s.dim[m];
    }
    vals[i] = s.vals[local];
    if (bad) {
        atomicOr(err, 1u);
        ckey[i] = 0;
        fkey[i] = 0;
        return;
    }
    const uint32_t c = specs[it].c;
    uint64_t a = specs[it].cbase, b = s.fbase;
    for (uint32_t j = 0; j < c; ++j) a += (uint64_t)v[s.mode[j]] * s.stride[j];
    for (uint32_t j = c; j < d; ++j) b += (uint64_t)v[s.mode[j]] * s.stride[j];
    ckey[i] = a;
    fkey[i] = b;
}

void launch_pack_items(const ItemSpec* specs, const uint64_t* off, uint32_t nitems, int side, uint64_t nnz,
                       uint64_t* ckey, uint64_t* fkey, double* vals, uint32_t* err, cudaStream_t st) {
    if (nnz == 0) return;
    pack_items_kernel<<<ceil_div_u32(nnz, 256), 256, 0, st>>>(specs, off, nitems, side, nnz, ckey, fkey, vals, err);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// tuple[r * width + m] = free index m of run r's representative element (zero past the item's
// own free-mode count)
__global__ void item_tuples_kernel(const uint32_t* __restrict__ run_start, const uint32_t* __restrict__ perm,
                                   uint64_t nruns, const ItemSpec* __restrict__ specs, const uint64_t* __restrict__ off,
                                   uint32_t nitems, int side, uint32_t width, uint32_t* __restrict__ tuple) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nruns) return;
    const uint64_t src = perm[run_start[r]];
    const uint32_t it = item_of(off, nitems, src);
    const ItemSide& s = specs[it].side[side];
    const uint32_t c = specs[it].c, nf = s.order - c;
    const uint32_t* row = s.idx + (src - off[it]) * s.order;
    for (uint32_t m = 0; m < width; ++m) tuple[r * width + m] = m < nf ? row[s.mode[c + m]] : 0u;
}

void launch_item_tuples(const uint32_t* run_start, const uint32_t* perm, uint64_t nruns, const ItemSpec* specs,
                        const uint64_t* off, uint32_t nitems, int side, uint32_t width, uint32_t* tuple,
                        cudaStream_t st) {
    if (nruns == 0 || width == 0) return;
    item_tuples_kernel<<<ceil_div_u32(nruns, 256), 256, 0, st>>>(run_start, perm, nruns, specs, off, nitems, side,
                                                                 width, tuple);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// first[i] = first index of the sorted `keys` that is >= base[i]; first[nitems] = n
__global__ void key_bounds_kernel(const uint64_t* __restrict__ keys, uint64_t n, const uint64_t* __restrict__ base,
                                  uint32_t nitems, uint32_t* __restrict__ first) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > nitems) return;
    if (i == nitems) {
        first[i] = (uint32_t)n;
        return;
    }
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (keys[mid] < base[i]) lo = mid + 1; else hi = mid;
    }
    first[i] = (uint32_t)lo;
}

void launch_key_bounds(const uint64_t* keys, uint64_t n, const uint64_t* base, uint32_t nitems, uint32_t* first,
                       cudaStream_t st) {
    key_bounds_kernel<<<ceil_div_u32((uint64_t)nitems + 1, 128), 128, 0, st>>>(keys, n, base, nitems, first);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// local[j] = global[j] - first[item of element j]
__global__ void localize_kernel(const uint32_t* __restrict__ global, uint64_t n, const uint64_t* __restrict__ off,
                                uint32_t nitems, const uint32_t* __restrict__ first, uint32_t* __restrict__ local) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) local[j] = global[j] - first[item_of(off, nitems, j)];
}

void launch_localize(const uint32_t* global, uint64_t n, const uint64_t* off, uint32_t nitems, const uint32_t* first,
                     uint32_t* local, cudaStream_t st) {
    if (n == 0) return;
    localize_kernel<<<ceil_div_u32(n, 256), 256, 0, st>>>(global, n, off, nitems, first, local);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// row_item[r] = the item whose rows [first[i], first[i + 1]) hold r
__global__ void row_item_kernel(uint64_t nrows, const uint32_t* __restrict__ first, uint32_t nitems,
                                uint32_t* __restrict__ row_item) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrows) return;
    uint32_t lo = 0, hi = nitems;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (first[mid] <= r) lo = mid; else hi = mid;
    }
    row_item[r] = lo;
}

void launch_row_item(uint64_t nrows, const uint32_t* first, uint32_t nitems, uint32_t* row_item, cudaStream_t st) {
    if (nrows == 0) return;
    row_item_kernel<<<ceil_div_u32(nrows, 256), 256, 0, st>>>(nrows, first, nitems, row_item);
    count_launch();
    PTC_CHECK_LAUNCH();
}

}  // namespace ptc
