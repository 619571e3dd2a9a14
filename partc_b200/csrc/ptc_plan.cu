// Planning kernels: row classes, work lists, and the split of large rows into hash parts.
#include "ptc_learned.cuh"
#include "ptc_spa.cuh"

namespace ptc {

__global__ void classify_rows_kernel(const uint64_t* __restrict__ row_flops, const uint32_t* __restrict__ row_start,
                                     uint64_t nrows, uint64_t small_max, uint32_t esc_avg,
                                     uint32_t* __restrict__ small_flag, uint32_t* __restrict__ big_flag,
                                     uint32_t* __restrict__ esc_flag) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrows) return;
    const uint64_t f = row_flops[r];  // rows without products are skipped (fksCuckooTC.hpp:183)
    const uint64_t len = row_start[r + 1] - row_start[r];
    const bool small = f > 0 && f <= small_max;
    const bool esc = f > small_max && f < (uint64_t)esc_avg * len;
    small_flag[r] = small ? 1u : 0u;
    esc_flag[r] = esc ? 1u : 0u;
    big_flag[r] = (f > small_max && !esc) ? 1u : 0u;
}

void launch_classify_rows(const uint64_t* row_flops, const uint32_t* row_start, uint64_t nrows, uint64_t small_max,
                          uint32_t esc_avg, uint32_t* small_flag, uint32_t* big_flag, uint32_t* esc_flag,
                          cudaStream_t st) {
    if (nrows == 0) return;
    classify_rows_kernel<<<ceil_div_u32(nrows, 256), 256, 0, st>>>(row_flops, row_start, nrows, small_max, esc_avg,
                                                                   small_flag, big_flag, esc_flag);
    count_launch();
    PTC_CHECK_LAUNCH();
}

__global__ void merge_flags_kernel(uint32_t* __restrict__ big_flag, const uint32_t* __restrict__ esc_flag, uint64_t n) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) big_flag[i] |= esc_flag[i];
}

void launch_merge_flags(uint32_t* big_flag, const uint32_t* esc_flag, uint64_t nrows, cudaStream_t st) {
    if (nrows == 0) return;
    merge_flags_kernel<<<ceil_div_u32(nrows, 256), 256, 0, st>>>(big_flag, esc_flag, nrows);
    count_launch();
    PTC_CHECK_LAUNCH();
}

__global__ void compact_indices_kernel(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ pos, uint64_t n,
                                       uint32_t* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && flag[i]) out[pos[i]] = (uint32_t)i;
}

void launch_compact_indices(const uint32_t* flag, const uint32_t* pos, uint64_t n, uint32_t* out, cudaStream_t st) {
    if (n == 0) return;
    compact_indices_kernel<<<ceil_div_u32(n, 256), 256, 0, st>>>(flag, pos, n, out);
    count_launch();
    PTC_CHECK_LAUNCH();
}

__global__ void work_keys_kernel(const uint32_t* __restrict__ rows, uint64_t n, const uint64_t* __restrict__ row_flops,
                                 const uint32_t* __restrict__ row_start, uint32_t map_len, uint32_t max_len,
                                 uint64_t* __restrict__ key) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t r = rows[i];
    const uint32_t len = row_start[r + 1] - row_start[r];
    const uint64_t group = len <= map_len ? 0ull : len <= max_len ? 1ull : 2ull;
    key[i] = (group << 40) | (~row_flops[r] & ((1ull << 40) - 1));
}

void launch_work_keys(const uint32_t* rows, uint64_t n, const uint64_t* row_flops, const uint32_t* row_start,
                      uint32_t map_len, uint32_t max_len, uint64_t* key, cudaStream_t st) {
    if (n == 0) return;
    work_keys_kernel<<<ceil_div_u32(n, 256), 256, 0, st>>>(rows, n, row_flops, row_start, map_len, max_len, key);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// Split one row's fine panels into parts (see SplitRule).  Calls emit(p0, p1, entries_before,
// mode) for each non-empty part; returns the number of parts.  The dense-window sums slide
// forward with p, so a row costs O(P).
template <typename Emit>
__device__ __forceinline__ uint32_t split_panels(const uint32_t* cnt, uint32_t P, SplitRule rule, bool* oversize,
                                                 Emit emit) {
    uint32_t parts = 0, p = 0;
    uint64_t before = 0;
    uint64_t wsum = 0;
    uint32_t wlo = 0, whi = 0;  // window [wlo, whi) with running sum wsum
    auto dense_window = [&](uint32_t q, uint32_t& w, uint64_t& sum) {
        if (rule.dense_panels == 0) return false;
        const uint32_t hi = min(q + rule.dense_panels, P);
        while (whi < hi) wsum += cnt[whi++];
        while (wlo < q) wsum -= cnt[wlo++];
        w = hi - q;
        sum = wsum;
        return sum >= (uint64_t)rule.dense_min * w;
    };
    while (p < P) {
        uint32_t w;
        uint64_t sum;
        if (dense_window(p, w, sum)) {
            emit(p, p + w, before, 1u);
            ++parts;
            before += sum;
            p += w;
            continue;
        }
        const uint32_t p0 = p;
        uint64_t acc = 0;
        while (p < P && (acc == 0 || acc + cnt[p] <= rule.cap)) {
            if (cnt[p] > rule.cap && !rule.oversize_dense) *oversize = true;
            acc += cnt[p];
            ++p;
            uint32_t w2;
            uint64_t s2;
            if (p < P && dense_window(p, w2, s2)) break;
        }
        if (acc > rule.cap && rule.oversize_dense) {
            // one panel above the table's capacity (the last one taken; those before it are
            // empty): direct-mapped over that panel alone
            emit(p - 1, p, before, 1u);
            ++parts;
            before += acc;
        } else if (acc > 0) {
            // table of at least acc * load_den / load_num slots, a power of two
            uint32_t bits = rule.min_bits;
            while (bits < rule.max_bits && ((uint64_t)rule.load_num << bits) < acc * rule.load_den) ++bits;
            emit(p0, p, before, bits << 1);
            ++parts;
            before += acc;
        }
    }
    return parts;
}

// Panels of large row i: [pbase[i], pbase[i + 1]) of panel_cnt, or i * P + [0, P) without pbase.
__device__ __forceinline__ void row_panels(const uint64_t* pbase, uint64_t i, uint32_t P, uint64_t& base, uint32_t& n) {
    base = pbase ? pbase[i] : i * P;
    n = pbase ? (uint32_t)(pbase[i + 1] - pbase[i]) : P;
}

// a large row whose exact output count equals its products: no two products share a column
__device__ __forceinline__ bool collision_free(const uint64_t* row_off, const uint64_t* row_flops, uint32_t row) {
    return row_off && row_flops && row_off[row + 1] - row_off[row] == row_flops[row];
}

__global__ void count_parts_kernel(const uint32_t* __restrict__ rows, const uint32_t* __restrict__ panel_cnt,
                                   const uint64_t* __restrict__ pbase, uint64_t nbig, uint32_t P, SplitRule rule,
                                   const uint64_t* __restrict__ row_off, const uint64_t* __restrict__ row_flops,
                                   uint32_t* __restrict__ nparts, uint32_t* __restrict__ oversize) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nbig) return;
    if (collision_free(row_off, row_flops, rows[i])) {
        nparts[i] = 0;
        return;
    }
    uint64_t b;
    uint32_t n;
    row_panels(pbase, i, P, b, n);
    bool over = false;
    nparts[i] = split_panels(panel_cnt + b, n, rule, &over, [](uint32_t, uint32_t, uint64_t, uint32_t) {});
    if (over) atomicOr(oversize, 1u);
}

void launch_count_parts(const uint32_t* rows, const uint32_t* panel_cnt, const uint64_t* pbase, uint64_t nbig,
                        uint32_t npanels, SplitRule rule, const uint64_t* row_off, const uint64_t* row_flops,
                        uint32_t* nparts, uint32_t* oversize, cudaStream_t st) {
    if (nbig == 0) return;
    count_parts_kernel<<<ceil_div_u32(nbig, 256), 256, 0, st>>>(rows, panel_cnt, pbase, nbig, npanels, rule, row_off,
                                                                row_flops, nparts, oversize);
    count_launch();
    PTC_CHECK_LAUNCH();
}

__global__ void copy_flags_kernel(const uint32_t* __restrict__ rows, uint64_t n, const uint64_t* __restrict__ row_off,
                                  const uint64_t* __restrict__ row_flops, uint32_t* __restrict__ flag) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flag[i] = collision_free(row_off, row_flops, rows[i]) ? 1u : 0u;
}

void launch_copy_flags(const uint32_t* rows, uint64_t n, const uint64_t* row_off, const uint64_t* row_flops,
                       uint32_t* flag, cudaStream_t st) {
    if (n == 0) return;
    copy_flags_kernel<<<ceil_div_u32(n, 256), 256, 0, st>>>(rows, n, row_off, row_flops, flag);
    count_launch();
    PTC_CHECK_LAUNCH();
}

__global__ void fill_parts_kernel(const uint32_t* __restrict__ rows, const uint32_t* __restrict__ panel_cnt,
                                  const uint64_t* __restrict__ pbase, uint64_t nbig, uint32_t P, SplitRule rule,
                                  const uint32_t* __restrict__ part_pos, const uint64_t* __restrict__ row_off,
                                  const uint64_t* __restrict__ row_flops, PartItem* __restrict__ parts) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nbig) return;
    const uint32_t row = rows[i];
    if (collision_free(row_off, row_flops, row)) return;
    const uint64_t base = row_off ? row_off[row] : 0;  // no offsets: the parts claim output later
    uint64_t b;
    uint32_t n;
    row_panels(pbase, i, P, b, n);
    uint32_t o = part_pos[i];
    bool over = false;
    split_panels(panel_cnt + b, n, rule, &over, [&](uint32_t p0, uint32_t p1, uint64_t before, uint32_t mode) {
        PartItem it;
        it.row = row;
        it.p0 = p0;
        it.p1 = p1;
        it.mode = mode;
        it.out_off = row_off ? base + before : kClaimBit;
        parts[o++] = it;
    });
}

void launch_fill_parts(const uint32_t* rows, const uint32_t* panel_cnt, const uint64_t* pbase, uint64_t nbig,
                       uint32_t npanels, SplitRule rule, const uint32_t* part_pos, const uint64_t* row_off,
                       const uint64_t* row_flops, PartItem* parts, cudaStream_t st) {
    if (nbig == 0) return;
    fill_parts_kernel<<<ceil_div_u32(nbig, 256), 256, 0, st>>>(rows, panel_cnt, pbase, nbig, npanels, rule, part_pos,
                                                               row_off, row_flops, parts);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// panels of every large row of a batch: its item's columns in panels of 2^log2w (at least one)
__global__ void row_panel_counts_kernel(const uint32_t* __restrict__ rows, uint64_t n,
                                        const uint32_t* __restrict__ row_item, const uint32_t* __restrict__ item_cols,
                                        uint32_t log2w, uint64_t* __restrict__ np) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t c = item_cols[row_item[rows[i]]];
    np[i] = c ? (c + (1ull << log2w) - 1) >> log2w : 1;
}

void launch_row_panel_counts(const uint32_t* rows, uint64_t n, const uint32_t* row_item, const uint32_t* item_cols,
                             uint32_t log2w, uint64_t* np, cudaStream_t st) {
    if (n == 0) return;
    row_panel_counts_kernel<<<ceil_div_u32(n, 256), 256, 0, st>>>(rows, n, row_item, item_cols, log2w, np);
    count_launch();
    PTC_CHECK_LAUNCH();
}

__global__ void count_parts_range_kernel(const PartItem* __restrict__ parts, const uint32_t* __restrict__ ridx,
                                         uint32_t n, const uint32_t* __restrict__ panel_cnt, uint32_t P, SplitRule rule,
                                         uint32_t* __restrict__ nparts, uint32_t* __restrict__ total) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const PartItem it = parts[i];
    const uint32_t* cnt = panel_cnt + (uint64_t)ridx[i] * P;
    uint64_t tot = 0;
    for (uint32_t p = it.p0; p < it.p1; ++p) tot += cnt[p];
    total[i] = (uint32_t)tot;
    bool over = false;
    nparts[i] = split_panels(cnt + it.p0, it.p1 - it.p0, rule, &over, [](uint32_t, uint32_t, uint64_t, uint32_t) {});
}

void launch_count_parts_range(const PartItem* parts, const uint32_t* ridx, uint32_t n, const uint32_t* panel_cnt,
                              uint32_t P, SplitRule rule, uint32_t* nparts, uint32_t* total, cudaStream_t st) {
    if (n == 0) return;
    count_parts_range_kernel<<<ceil_div_u32(n, 128), 128, 0, st>>>(parts, ridx, n, panel_cnt, P, rule, nparts, total);
    count_launch();
    PTC_CHECK_LAUNCH();
}

__global__ void fill_parts_range_kernel(const PartItem* __restrict__ parts, const uint32_t* __restrict__ ridx,
                                        uint32_t n, const uint32_t* __restrict__ panel_cnt, uint32_t P, SplitRule rule,
                                        const uint32_t* __restrict__ part_pos, PartItem* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const PartItem it = parts[i];
    const uint32_t* cnt = panel_cnt + (uint64_t)ridx[i] * P;
    uint32_t o = part_pos[i];
    bool over = false;
    split_panels(cnt + it.p0, it.p1 - it.p0, rule, &over, [&](uint32_t q0, uint32_t q1, uint64_t, uint32_t mode) {
        PartItem x;
        x.row = it.row;
        x.p0 = it.p0 + q0;
        x.p1 = it.p0 + q1;
        x.mode = mode;
        x.out_off = kClaimBit;
        out[o++] = x;
    });
}

void launch_fill_parts_range(const PartItem* parts, const uint32_t* ridx, uint32_t n, const uint32_t* panel_cnt,
                             uint32_t P, SplitRule rule, const uint32_t* part_pos, PartItem* out, cudaStream_t st) {
    if (n == 0) return;
    fill_parts_range_kernel<<<ceil_div_u32(n, 128), 128, 0, st>>>(parts, ridx, n, panel_cnt, P, rule, part_pos, out);
    count_launch();
    PTC_CHECK_LAUNCH();
}

}  // namespace ptc
