// Per-row features of the learned sizer and the column-popularity table they use.
#include <cmath>

#include "ptc_sizer.cuh"

namespace ptc {

__global__ void col_degree_kernel(const uint32_t* __restrict__ b_col, uint64_t nb, uint32_t* __restrict__ deg) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < nb) atomicAdd(&deg[b_col[j]], 1u);
}

__host__ __device__ __forceinline__ float grid_flops(int g) { return exp2f((float)g / kGridPerOctave); }

// block (p, g): sum over the columns of panel p of 1 - exp(-F_g deg / nb)
__global__ void panel_popularity_kernel(const uint32_t* __restrict__ deg, uint64_t nb, uint64_t ncols,
                                        uint32_t panel_log2, float* __restrict__ gp) {
    const uint32_t p = blockIdx.x, g = blockIdx.y;
    const float scale = grid_flops((int)g) / (float)nb;
    const uint64_t lo = (uint64_t)p << panel_log2;
    const uint64_t hi = ncols < lo + (1ull << panel_log2) ? ncols : lo + (1ull << panel_log2);
    float acc = 0.f;
    for (uint64_t c = lo + threadIdx.x; c < hi; c += blockDim.x) acc += -expm1f(-scale * (float)deg[c]);
    __shared__ float red[32];
    acc = warp_sum(acc);
    if (lane_id() == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        float v = threadIdx.x < blockDim.x / 32 ? red[threadIdx.x] : 0.f;
        v = warp_sum(v);
        if (threadIdx.x == 0) gp[(uint64_t)p * kGridPoints + g] = v;
    }
}

// row npanels of gp = sum over the panels
__global__ void popularity_total_kernel(float* __restrict__ gp, uint32_t npanels) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= kGridPoints) return;
    float acc = 0.f;
    for (uint32_t p = 0; p < npanels; ++p) acc += gp[(uint64_t)p * kGridPoints + g];
    gp[(uint64_t)npanels * kGridPoints + g] = acc;
}

void launch_popularity_table(const uint32_t* b_col, uint64_t nb, uint64_t ncols, uint32_t npanels, uint32_t panel_log2,
                             float* gp, Arena& ar) {
    cudaStream_t st = ar.stream();
    uint32_t* deg = ar.alloc<uint32_t>(ncols);
    PTC_CUDA(cudaMemsetAsync(deg, 0, ncols * sizeof(uint32_t), st));
    if (nb) {
        col_degree_kernel<<<ceil_div_u32(nb, 256), 256, 0, st>>>(b_col, nb, deg);
        count_launch();
        PTC_CHECK_LAUNCH();
    }
    panel_popularity_kernel<<<dim3(npanels, kGridPoints), 256, 0, st>>>(deg, std::max<uint64_t>(nb, 1), ncols,
                                                                        panel_log2, gp);
    count_launch();
    PTC_CHECK_LAUNCH();
    popularity_total_kernel<<<ceil_div_u32(kGridPoints, 128), 128, 0, st>>>(gp, npanels);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// G(F) by linear interpolation in log2(F) on the tabulated grid
__device__ __forceinline__ float popularity(const float* __restrict__ row, float F) {
    if (F <= 1.f) return F * row[0];
    float u = log2f(F) * kGridPerOctave;
    u = fminf(u, (float)(kGridPoints - 1));
    const int g = (int)u;
    const float fr = u - (float)g;
    const float a = row[g], b = row[min(g + 1, kGridPoints - 1)];
    return a + fr * (b - a);
}

__device__ __forceinline__ float lg(float x) { return log2f(1.f + x) * (1.f / 16.f); }

// block (i, g): item i's G(F_g) = sum over its columns of 1 - exp(-F_g deg / nb_i)
__global__ void item_popularity_kernel(ItemStats is) {
    const uint32_t i = blockIdx.x, g = blockIdx.y;
    const uint64_t nb = is.b_off[i + 1] - is.b_off[i];
    const float scale = grid_flops((int)g) / (float)(nb ? nb : 1);
    float acc = 0.f;
    for (uint32_t c = is.col_first[i] + threadIdx.x; c < is.col_first[i + 1]; c += blockDim.x)
        acc += -expm1f(-scale * (float)(is.col_run[c + 1] - is.col_run[c]));
    __shared__ float red[32];
    acc = warp_sum(acc);
    if (lane_id() == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        float v = threadIdx.x < blockDim.x / 32 ? red[threadIdx.x] : 0.f;
        v = warp_sum(v);
        if (threadIdx.x == 0) is.gtot[(uint64_t)i * kGridPoints + g] = v;
    }
}

// B nonzeros of every (item, local panel): integer sums, so the shares are the same every run
__global__ void item_panel_mass_kernel(ItemStats is, uint64_t ncols, uint32_t panel_log2) {
    const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncols) return;
    uint32_t lo = 0, hi = is.nitems;  // item: the last i with col_first[i] <= c
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (is.col_first[mid] <= c) lo = mid; else hi = mid;
    }
    const uint32_t p = (uint32_t)((c - is.col_first[lo]) >> panel_log2);
    atomicAdd(&is.pmass[is.item_pb[lo] + p], is.col_run[c + 1] - is.col_run[c]);
}

void launch_item_popularity(ItemStats& is, uint64_t ncols_global, uint32_t panel_log2, Arena& ar) {
    cudaStream_t st = ar.stream();
    if (is.nitems == 0) return;
    item_popularity_kernel<<<dim3(is.nitems, kGridPoints), 128, 0, st>>>(is);
    count_launch();
    PTC_CHECK_LAUNCH();
    if (ncols_global) {
        item_panel_mass_kernel<<<ceil_div_u32(ncols_global, 256), 256, 0, st>>>(is, ncols_global, panel_log2);
        count_launch();
        PTC_CHECK_LAUNCH();
    }
}

// One warp per row: statistics over the row's A nonzeros, then the feature vector.
__global__ void row_features_kernel(Operands op, const uint32_t* __restrict__ rows, uint64_t n,
                                    const uint64_t* __restrict__ row_flops, const float* __restrict__ gtot_all,
                                    float* __restrict__ x, ItemStats is) {
    const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32;
    if (w >= n) return;
    const uint32_t lane = lane_id();
    const uint32_t row = rows[w];
    const uint32_t ka = op.row_start[row], kb = op.row_start[row + 1];
    uint32_t matched = 0, maxl = 0;
    double sum2 = 0.0;
    for (uint32_t k = ka + lane; k < kb; k += 32) {
        const int32_t f = op.a_fib[k];
        if (f >= 0) {
            const uint32_t L = op.fib_start[f + 1] - op.fib_start[f];
            ++matched;
            maxl = max(maxl, L);
            sum2 += (double)L * (double)L;
        }
    }
    matched = warp_sum(matched);
    maxl = __reduce_max_sync(kFullMask, maxl);
    sum2 = warp_sum(sum2);
    if (lane != 0) return;
    const float F = (float)row_flops[row];
    const float len = (float)(kb - ka);
    // the contraction's statistics: the whole call's, or in a batch the row's item's
    float nc = (float)op.ncols, nb = (float)op.nb, nfib = (float)op.nfib, nrows = (float)op.nrows;
    const float* gtot = gtot_all;
    if (is.gtot && op.row_item) {
        const uint32_t it = op.row_item[row];
        nc = (float)(is.col_first[it + 1] - is.col_first[it]);
        nb = (float)(is.b_off[it + 1] - is.b_off[it]);
        nfib = (float)(is.fib_first[it + 1] - is.fib_first[it]);
        nrows = (float)(is.row_first[it + 1] - is.row_first[it]);
        gtot = is.gtot + (uint64_t)it * kGridPoints;
    }
    float* o = x + w * kSizerInputs;
    o[0] = lg(F);
    o[1] = lg(len);
    o[2] = lg((float)matched);
    o[3] = lg((float)maxl);
    o[4] = lg(F / fmaxf((float)matched, 1.f));
    o[5] = lg((float)(sum2 / fmax((double)F, 1.0)));
    o[6] = lg(popularity(gtot, F));
    o[7] = lg(nc);
    o[8] = lg(fminf(F, nc));
    o[9] = lg(nc * -expm1f(-F / fmaxf(nc, 1.f)));
    o[10] = lg(nb / fmaxf(nc, 1.f));
    o[11] = (float)maxl / fmaxf(F, 1.f);
    o[12] = lg(nfib);
    o[13] = lg(nrows);
    o[14] = lg(popularity(gtot, 0.5f * F));
    o[15] = 1.f;
}

void launch_row_features(const Operands& op, const uint32_t* rows, uint64_t n, const uint64_t* row_flops,
                         const float* gp, float* x, cudaStream_t st, const ItemStats* is) {
    if (n == 0) return;
    const float* gtot = gp ? gp + (uint64_t)op.npanels * kGridPoints : nullptr;
    row_features_kernel<<<ceil_div_u32(n * 32, 256), 256, 0, st>>>(op, rows, n, row_flops, gtot, x,
                                                                   is ? *is : ItemStats{});
    count_launch();
    PTC_CHECK_LAUNCH();
}

__global__ void row_targets_kernel(const uint32_t* __restrict__ rows, uint64_t n, const uint64_t* __restrict__ row_d,
                                   float* __restrict__ t) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) t[i] = log2f(1.f + (float)row_d[rows[i]]);
}

void launch_row_targets(const uint32_t* rows, uint64_t n, const uint64_t* row_d, float* t, cudaStream_t st) {
    if (n == 0) return;
    row_targets_kernel<<<ceil_div_u32(n, 256), 256, 0, st>>>(rows, n, row_d, t);
    count_launch();
    PTC_CHECK_LAUNCH();
}

}  // namespace ptc
