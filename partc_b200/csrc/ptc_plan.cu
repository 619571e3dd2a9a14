// Planning kernels: row classes, work lists, and the split of large rows into hash parts.
#include "ptc_spa.cuh"

namespace ptc {

__global__ void classify_rows_kernel(const uint64_t* __restrict__ row_flops, uint64_t nrows, uint64_t small_max,
                                     uint32_t* __restrict__ small_flag, uint32_t* __restrict__ big_flag) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrows) return;
    const uint64_t f = row_flops[r];
    small_flag[r] = (f > 0 && f <= small_max) ? 1u : 0u;  // rows without products are skipped
    big_flag[r] = (f > small_max) ? 1u : 0u;              // (fksCuckooTC.hpp:183)
}

void launch_classify_rows(const uint64_t* row_flops, uint64_t nrows, uint64_t small_max, uint32_t* small_flag,
                          uint32_t* big_flag, cudaStream_t st) {
    if (nrows == 0) return;
    classify_rows_kernel<<<ceil_div_u32(nrows, 256), 256, 0, st>>>(row_flops, nrows, small_max, small_flag, big_flag);
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
                                 uint64_t* __restrict__ key) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) key[i] = ~row_flops[rows[i]];
}

void launch_work_keys(const uint32_t* rows, uint64_t n, const uint64_t* row_flops, uint64_t* key, cudaStream_t st) {
    if (n == 0) return;
    work_keys_kernel<<<ceil_div_u32(n, 256), 256, 0, st>>>(rows, n, row_flops, key);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// Greedy split of one row's fine panels into consecutive groups holding at most `cap` entries.
// Calls emit(p0, p1, entries_before_p0) for each group; returns the number of groups.
template <typename Emit>
__device__ __forceinline__ uint32_t split_panels(const uint32_t* cnt, uint32_t P, uint32_t cap, bool* oversize,
                                                 Emit emit) {
    uint32_t groups = 0, p0 = 0, acc = 0;
    uint64_t before = 0;
    for (uint32_t p = 0; p < P; ++p) {
        const uint32_t c = cnt[p];
        if (c > cap) *oversize = true;
        if (acc > 0 && acc + c > cap) {
            emit(p0, p, before);
            ++groups;
            before += acc;
            p0 = p;
            acc = 0;
        }
        acc += c;
    }
    emit(p0, P, before);
    return groups + 1;
}

__global__ void count_parts_kernel(const uint32_t* __restrict__ panel_cnt, uint64_t nbig, uint32_t P, uint32_t cap,
                                   uint32_t* __restrict__ nparts, uint32_t* __restrict__ oversize) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nbig) return;
    bool over = false;
    nparts[i] = split_panels(panel_cnt + i * P, P, cap, &over, [](uint32_t, uint32_t, uint64_t) {});
    if (over) atomicOr(oversize, 1u);
}

void launch_count_parts(const uint32_t* panel_cnt, uint64_t nbig, uint32_t npanels, uint32_t cap, uint32_t* nparts,
                        uint32_t* oversize, cudaStream_t st) {
    if (nbig == 0) return;
    count_parts_kernel<<<ceil_div_u32(nbig, 256), 256, 0, st>>>(panel_cnt, nbig, npanels, cap, nparts, oversize);
    count_launch();
    PTC_CHECK_LAUNCH();
}

__global__ void fill_parts_kernel(const uint32_t* __restrict__ rows, const uint32_t* __restrict__ panel_cnt,
                                  uint64_t nbig, uint32_t P, uint32_t cap, const uint32_t* __restrict__ part_pos,
                                  const uint64_t* __restrict__ row_off, PartItem* __restrict__ parts) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nbig) return;
    const uint32_t row = rows[i];
    const uint64_t base = row_off[row];
    uint32_t o = part_pos[i];
    bool over = false;
    split_panels(panel_cnt + i * P, P, cap, &over, [&](uint32_t p0, uint32_t p1, uint64_t before) {
        PartItem it;
        it.row = row;
        it.p0 = p0;
        it.p1 = p1;
        it.pad = 0;
        it.out_off = base + before;
        parts[o++] = it;
    });
}

void launch_fill_parts(const uint32_t* rows, const uint32_t* panel_cnt, uint64_t nbig, uint32_t npanels, uint32_t cap,
                       const uint32_t* part_pos, const uint64_t* row_off, PartItem* parts, cudaStream_t st) {
    if (nbig == 0) return;
    fill_parts_kernel<<<ceil_div_u32(nbig, 256), 256, 0, st>>>(rows, panel_cnt, nbig, npanels, cap, part_pos, row_off,
                                                               parts);
    count_launch();
    PTC_CHECK_LAUNCH();
}

}  // namespace ptc
