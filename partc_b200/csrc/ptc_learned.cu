// Learned-path planning: predicted per-panel counts from the sizer, and the bookkeeping of the
// exact reruns of parts whose prediction was too small.
#include <cmath>

#include "ptc_learned.cuh"

namespace ptc {

// G_p(F) of the popularity table (see ptc_sizer.cuh), linear in log2 F between grid points
__device__ __forceinline__ float popularity_at(const float* __restrict__ row, float F) {
    if (F <= 1.f) return F * row[0];
    float u = fminf(log2f(F) * kGridPerOctave, (float)(kGridPoints - 1));
    const int g = (int)u;
    const float fr = u - (float)g;
    const float a = row[g], b = row[min(g + 1, kGridPoints - 1)];
    return a + fr * (b - a);
}

// cnt[i * P + p] = ceil(margin * D_pred(i) * G_p(F_i) / G(F_i)), at most the panel's width and
// the row's products; D_pred = 2^pred - 1 clamped to [1, min(F, ncols)].  In a batch
// (row_item != null) a row's columns are its item's: panels past the item's item_cols[item]
// columns get nothing and the shares are taken over the item's panels -- by its own B nonzeros
// per panel when per-item statistics are given (is.pmass), else by the batch's popularity table
// (cum = the table's prefix sums over panels).
__global__ void predicted_panel_counts_kernel(const uint32_t* __restrict__ rows, uint64_t n,
                                              const uint64_t* __restrict__ row_flops, const float* __restrict__ pred,
                                              const float* __restrict__ gp, const float* __restrict__ cum,
                                              const uint32_t* __restrict__ row_item,
                                              const uint32_t* __restrict__ item_cols,
                                              const uint64_t* __restrict__ pbase, uint32_t P, uint32_t panel_log2,
                                              uint64_t ncols, float margin, uint32_t* __restrict__ cnt, ItemStats is) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float F = (float)row_flops[rows[i]];
    const uint32_t item = row_item ? row_item[rows[i]] : 0u;
    const uint64_t nc = row_item ? item_cols[item] : ncols;
    const uint64_t base = pbase ? pbase[i] : i * P;
    const uint32_t Pi = pbase ? (uint32_t)(pbase[i + 1] - pbase[i]) : P;
    float d = exp2f(pred[i]) - 1.f;
    d = fminf(fmaxf(d, 1.f), fminf(F, (float)nc));
    const bool by_mass = row_item && is.pmass;
    const float nb_item = by_mass ? (float)(is.b_off[item + 1] - is.b_off[item]) : 0.f;
    const float tot = by_mass ? 0.f
                      : row_item ? popularity_at(cum + (uint64_t)Pi * kGridPoints, F)
                                 : popularity_at(gp + (uint64_t)P * kGridPoints, F);
    for (uint32_t p = 0; p < Pi; ++p) {
        const uint64_t lo = (uint64_t)p << panel_log2;
        if (lo >= nc) {
            cnt[base + p] = 0;
            continue;
        }
        float share;
        if (by_mass) share = nb_item > 0.f ? (float)is.pmass[is.item_pb[item] + p] / nb_item : 1.f / Pi;
        else share = tot > 0.f ? popularity_at(gp + (uint64_t)p * kGridPoints, F) / tot : 1.f / Pi;
        const uint64_t width = (nc - lo) < (1ull << panel_log2) ? (nc - lo) : (1ull << panel_log2);
        float c = ceilf(margin * d * share);
        c = fminf(fminf(c, (float)width), F);
        cnt[base + p] = (uint32_t)c;
    }
}

// cum[p * G + g] = sum over panels q < p of gp[q * G + g], p = 0..P
__global__ void popularity_prefix_kernel(const float* __restrict__ gp, uint32_t P, float* __restrict__ cum) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= kGridPoints) return;
    float acc = 0.f;
    for (uint32_t p = 0; p <= P; ++p) {
        cum[(uint64_t)p * kGridPoints + g] = acc;
        if (p < P) acc += gp[(uint64_t)p * kGridPoints + g];
    }
}

void launch_predicted_panel_counts(const uint32_t* rows, uint64_t n, const uint64_t* row_flops, const float* pred,
                                   const float* gp, const uint32_t* row_item, const uint32_t* item_cols,
                                   const uint64_t* pbase, uint32_t P, uint32_t panel_log2, uint64_t ncols, float margin,
                                   uint32_t* cnt, Arena& ar, const ItemStats* is) {
    if (n == 0) return;
    cudaStream_t st = ar.stream();
    float* cum = nullptr;
    if (row_item && !(is && is->pmass)) {
        cum = ar.alloc<float>((uint64_t)(P + 1) * kGridPoints);
        popularity_prefix_kernel<<<ceil_div_u32(kGridPoints, 128), 128, 0, st>>>(gp, P, cum);
        count_launch();
        PTC_CHECK_LAUNCH();
    }
    predicted_panel_counts_kernel<<<ceil_div_u32(n, 128), 128, 0, st>>>(
        rows, n, row_flops, pred, gp, cum, row_item, item_cols, pbase, P, panel_log2, ncols, margin, cnt,
        is ? *is : ItemStats{});
    count_launch();
    PTC_CHECK_LAUNCH();
}

__global__ void sum_u32_kernel(const uint32_t* __restrict__ x, uint64_t n, unsigned long long* __restrict__ out) {
    uint64_t acc = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        acc += x[i];
    acc = warp_sum(acc);
    if (lane_id() == 0 && acc) atomicAdd(out, (unsigned long long)acc);
}

void launch_sum_u32(const uint32_t* x, uint64_t n, uint64_t* out, cudaStream_t st) {
    PTC_CUDA(cudaMemsetAsync(out, 0, sizeof(uint64_t), st));
    if (n == 0) return;
    const uint32_t grid = std::min<uint32_t>(ceil_div_u32(n, 256), 1024);
    sum_u32_kernel<<<grid, 256, 0, st>>>(x, n, reinterpret_cast<unsigned long long*>(out));
    count_launch();
    PTC_CHECK_LAUNCH();
}

__global__ void gather_parts_kernel(const PartItem* __restrict__ parts, const uint32_t* __restrict__ idx, uint32_t n,
                                    PartItem* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = parts[idx[i]];
}

void launch_gather_parts(const PartItem* parts, const uint32_t* idx, uint32_t n, PartItem* out, cudaStream_t st) {
    if (n == 0) return;
    gather_parts_kernel<<<ceil_div_u32(n, 256), 256, 0, st>>>(parts, idx, n, out);
    count_launch();
    PTC_CHECK_LAUNCH();
}

__global__ void row_actual_kernel(const PartItem* __restrict__ parts, const uint32_t* __restrict__ counts, uint32_t n,
                                  uint64_t* __restrict__ row_actual) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && counts[i])
        atomicAdd(reinterpret_cast<unsigned long long*>(&row_actual[parts[i].row]), (unsigned long long)counts[i]);
}

void launch_row_actual(const PartItem* parts, const uint32_t* counts, uint32_t n, uint64_t* row_actual,
                       cudaStream_t st) {
    if (n == 0) return;
    row_actual_kernel<<<ceil_div_u32(n, 256), 256, 0, st>>>(parts, counts, n, row_actual);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// sum over rows of |pred_i - log2(1 + actual(row_i))|
__global__ void log2_error_kernel(const uint32_t* __restrict__ rows, uint64_t n, const float* __restrict__ pred,
                                  const uint64_t* __restrict__ row_actual, double* __restrict__ out) {
    double acc = 0.0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        acc += fabs((double)pred[i] - log2(1.0 + (double)row_actual[rows[i]]));
    acc = warp_sum(acc);
    if (lane_id() == 0) atomicAdd(out, acc);
}

void launch_log2_error(const uint32_t* rows, uint64_t n, const float* pred, const uint64_t* row_actual, double* out,
                       cudaStream_t st) {
    PTC_CUDA(cudaMemsetAsync(out, 0, sizeof(double), st));
    if (n == 0) return;
    const uint32_t grid = std::min<uint32_t>(ceil_div_u32(n, 256), 1024);
    log2_error_kernel<<<grid, 256, 0, st>>>(rows, n, pred, row_actual, out);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// ---- claim budgets and batch waves ----

// budget[rows[i]] = sum of the row's predicted panel counts (the budgets of its parts)
__global__ void big_budget_kernel(const uint32_t* __restrict__ rows, uint64_t n, const uint32_t* __restrict__ cnt,
                                  const uint64_t* __restrict__ pbase, uint32_t P, uint64_t* __restrict__ budget) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t b = pbase ? pbase[i] : i * P, e = pbase ? pbase[i + 1] : (i + 1) * P;
    uint64_t s = 0;
    for (uint64_t p = b; p < e; ++p) s += cnt[p];
    budget[rows[i]] = s;
}

void launch_claim_budgets(const uint32_t* big_rows, uint64_t n_big, const uint32_t* panel_cnt, const uint64_t* pbase,
                          uint32_t P, uint64_t* budget, cudaStream_t st) {
    if (n_big == 0) return;
    big_budget_kernel<<<ceil_div_u32(n_big, 256), 256, 0, st>>>(big_rows, n_big, panel_cnt, pbase, P, budget);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// row_off[r] += claim_off[row_first[row_item[r]]] for every row r: the exactly counted entries of
// an item go first in its range, ahead of the claimed ones
__global__ void shift_exact_kernel(uint64_t nrows, const uint32_t* __restrict__ row_item,
                                   const uint32_t* __restrict__ row_first, const uint64_t* __restrict__ claim_off,
                                   uint64_t* __restrict__ row_off) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nrows) row_off[r] += claim_off[row_first[row_item[r]]];
}

void launch_shift_exact(uint64_t nrows, const uint32_t* row_item, const uint32_t* row_first, const uint64_t* claim_off,
                        uint64_t* row_off, cudaStream_t st) {
    if (nrows == 0) return;
    shift_exact_kernel<<<ceil_div_u32(nrows, 256), 256, 0, st>>>(nrows, row_item, row_first, claim_off, row_off);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// key[i] = wave of part i: the last wave whose first row is <= the part's row
__global__ void part_wave_kernel(const PartItem* __restrict__ parts, uint32_t n, const uint32_t* __restrict__ wave_row,
                                 uint32_t nwaves, uint64_t* __restrict__ key, uint32_t* __restrict__ idx) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t r = parts[i].row;
    uint32_t lo = 0, hi = nwaves;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (wave_row[mid] <= r) lo = mid; else hi = mid;
    }
    key[i] = lo;
    idx[i] = i;
}

void launch_part_wave(const PartItem* parts, uint32_t n, const uint32_t* wave_row, uint32_t nwaves, uint64_t* key,
                      uint32_t* idx, cudaStream_t st) {
    if (n == 0) return;
    part_wave_kernel<<<ceil_div_u32(n, 256), 256, 0, st>>>(parts, n, wave_row, nwaves, key, idx);
    count_launch();
    PTC_CHECK_LAUNCH();
}

}  // namespace ptc
