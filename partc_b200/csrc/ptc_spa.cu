// Sparse accumulators of the contraction (the reference's numeric pass, fksCuckooTC.hpp:180-357,
// and its per-row SPA hash tables, fksCuckooSPA.hpp).
//
// Summation order.  The reference computes each output entry as a left fold over the row's A
// nonzeros in COO input order, each term the rounded product a*b (fksCuckooTC.hpp:294-337;
// Aux_data keeps insertion order, fksCuckoo.hpp:233-255).  Both kernels below keep exactly that
// order, so values are bit-identical to the reference:
//   * the row's products are enumerated as a stream in (A nonzero, fiber entry) order;
//   * products of one A nonzero have distinct columns (a fiber never repeats a B free key), so
//     they may be applied concurrently;
//   * products of different A nonzeros that hit the same column are applied in stream order --
//     by rank inside a warp (match_any), or by claim rounds inside a block.
// Products use __dmul_rn and sums __dadd_rn so nothing is contracted into an FMA.
#include "ptc_internal.cuh"

namespace ptc {

// ---------------------------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------------------------

__device__ __forceinline__ uint32_t hash32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

// Write output entry o = (row's A free tuple, column's B free tuple, value).
__device__ __forceinline__ void write_entry(const Operands& op, const OutputView& out, uint64_t o, uint32_t row,
                                            uint32_t col, double v) {
    const uint32_t fa = op.fa, fb = op.fb, od = fa + fb;
    uint32_t* dst = out.idx + o * od;
    if (fa == 2 && fb == 2) {
        const uint2 r = *reinterpret_cast<const uint2*>(op.row_tuple + (uint64_t)row * 2);
        const uint2 c = *reinterpret_cast<const uint2*>(op.col_tuple + (uint64_t)col * 2);
        *reinterpret_cast<uint4*>(dst) = make_uint4(r.x, r.y, c.x, c.y);
    } else if (fa == 1 && fb == 1) {
        *reinterpret_cast<uint2*>(dst) = make_uint2(op.row_tuple[row], op.col_tuple[col]);
    } else {
        for (uint32_t m = 0; m < fa; ++m) dst[m] = op.row_tuple[(uint64_t)row * fa + m];
        for (uint32_t m = 0; m < fb; ++m) dst[fa + m] = op.col_tuple[(uint64_t)col * fb + m];
    }
    out.val[o] = v;
}

// ---------------------------------------------------------------------------------------------
// small rows: one warp per row, private open-addressing table in shared memory
// ---------------------------------------------------------------------------------------------

constexpr int kSmallWarps = 8;
constexpr uint32_t kSmallSlots = 1024;       // per warp
constexpr uint32_t kSmallMaxFlops = 512;     // rows with at most this many products
constexpr uint32_t kEmptyCol = 0xffffffffu;

uint32_t small_row_max_flops() { return kSmallMaxFlops; }

template <bool NUMERIC>
__global__ void __launch_bounds__(kSmallWarps * 32) small_rows_kernel(Operands op, const WorkItem* __restrict__ items,
                                                                      uint32_t nitems, uint64_t* __restrict__ counts,
                                                                      OutputView out) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t warp = threadIdx.x >> 5, lane = lane_id();
    uint32_t* keys = reinterpret_cast<uint32_t*>(smem) + warp * kSmallSlots;
    double* vals = reinterpret_cast<double*>(smem + kSmallWarps * kSmallSlots * sizeof(uint32_t)) + warp * kSmallSlots;
    for (uint32_t i = lane; i < kSmallSlots; i += 32) keys[i] = kEmptyCol;
    __syncwarp();

    for (uint32_t item = blockIdx.x * kSmallWarps + warp; item < nitems; item += gridDim.x * kSmallWarps) {
        const WorkItem it = items[item];
        const uint32_t row = it.row;
        const uint32_t ka = op.row_start[row], kb = op.row_start[row + 1];
        uint32_t nnew = 0;
        for (uint32_t kw = ka; kw < kb; kw += 32) {
            const uint32_t k = kw + lane;
            uint32_t L = 0, s = 0;
            double a = 0.0;
            if (k < kb) {
                const int32_t f = op.a_fib[k];
                if (f >= 0) {
                    s = op.fib_start[f];
                    L = op.fib_start[f + 1] - s;
                    if (NUMERIC) a = op.a_val[k];
                }
            }
            const uint32_t incl = warp_inclusive_scan(L);
            const uint32_t excl = incl - L;
            const uint32_t total = __shfl_sync(kFullMask, incl, 31);
            for (uint32_t c0 = 0; c0 < total; c0 += 32) {
                const uint32_t p = c0 + lane;
                const bool valid = p < total;
                // source lane: number of lanes whose inclusive end is <= p
                uint32_t kk = 0;
#pragma unroll
                for (uint32_t step = 16; step > 0; step >>= 1) {
                    const uint32_t e = __shfl_sync(kFullMask, incl, kk + step - 1);
                    if (e <= p) kk += step;
                }
                kk = min(kk, 31u);
                const uint32_t sk = __shfl_sync(kFullMask, s, kk);
                const uint32_t ek = __shfl_sync(kFullMask, excl, kk);
                const double ak = __shfl_sync(kFullMask, a, kk);
                const uint32_t j = sk + (p - ek);
                const uint32_t col = valid ? op.b_col[j] : kEmptyCol;
                const uint32_t m = __match_any_sync(kFullMask, col);
                const uint32_t rank = __popc(m & lanemask_lt());
                const uint32_t leader = __ffs(m) - 1;
                int slot = -1;
                int isnew = 0;
                if (valid && rank == 0) {
                    uint32_t h = hash32(col) & (kSmallSlots - 1);
                    for (uint32_t probe = 0; probe < kSmallSlots; ++probe) {
                        const uint32_t cur = keys[h];
                        if (cur == col) { slot = (int)h; break; }
                        if (cur == kEmptyCol) {
                            const uint32_t old = atomicCAS(&keys[h], kEmptyCol, col);
                            if (old == kEmptyCol) { slot = (int)h; isnew = 1; break; }
                            if (old == col) { slot = (int)h; break; }
                        }
                        h = (h + 1) & (kSmallSlots - 1);
                    }
                }
                slot = __shfl_sync(kFullMask, slot, leader);
                isnew = __shfl_sync(kFullMask, isnew, leader);
                if (NUMERIC) {
                    const double v = valid ? __dmul_rn(ak, op.b_val[j]) : 0.0;
                    const uint32_t maxr = __reduce_max_sync(kFullMask, valid ? rank : 0u);
                    for (uint32_t r = 0; r <= maxr; ++r) {
                        if (valid && rank == r && slot >= 0) {
                            if (r == 0 && isnew) vals[slot] = v;
                            else vals[slot] = __dadd_rn(vals[slot], v);
                        }
                        __syncwarp();
                    }
                } else {
                    nnew += __popc(__ballot_sync(kFullMask, valid && rank == 0 && isnew));
                    __syncwarp();
                }
            }
        }
        // emit (numeric) or count (symbolic), resetting the table
        uint64_t o = NUMERIC ? out.item_off[it.slot] : 0;
        for (uint32_t i = 0; i < kSmallSlots; i += 32) {
            const uint32_t sidx = i + lane;
            const uint32_t kc = keys[sidx];
            const bool occ = kc != kEmptyCol;
            const uint32_t mask = __ballot_sync(kFullMask, occ);
            if (NUMERIC && occ) write_entry(op, out, o + __popc(mask & lanemask_lt()), row, kc, vals[sidx]);
            keys[sidx] = kEmptyCol;
            o += __popc(mask);
        }
        if (!NUMERIC && lane == 0) counts[it.slot] = nnew;
        __syncwarp();
    }
}

void launch_small_rows(bool numeric, const Operands& op, const WorkItem* items, uint32_t nitems, uint64_t* counts,
                       const OutputView& out, cudaStream_t st) {
    if (nitems == 0) return;
    const size_t smem = kSmallWarps * kSmallSlots * (sizeof(uint32_t) + (numeric ? sizeof(double) : 0));
    const uint32_t grid = ceil_div_u32(nitems, kSmallWarps);
    if (numeric) {
        PTC_CUDA(cudaFuncSetAttribute(small_rows_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        small_rows_kernel<true><<<grid, kSmallWarps * 32, smem, st>>>(op, items, nitems, counts, out);
    } else {
        PTC_CUDA(cudaFuncSetAttribute(small_rows_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        small_rows_kernel<false><<<grid, kSmallWarps * 32, smem, st>>>(op, items, nitems, counts, out);
    }
    count_launch();
    PTC_CHECK_LAUNCH();
}

// ---------------------------------------------------------------------------------------------
// dense panels: one block per (row, column panel), dense accumulator of panel_width columns
// ---------------------------------------------------------------------------------------------

constexpr int kPanelThreads = 256;
constexpr uint32_t kNoClaim = 0xffffffffu;

template <bool NUMERIC>
__global__ void __launch_bounds__(kPanelThreads) panel_kernel(Operands op, const WorkItem* __restrict__ items,
                                                              uint32_t nitems, uint64_t* __restrict__ counts,
                                                              OutputView out, uint32_t* __restrict__ work_counter) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t W = 1u << op.panel_log2;
    double* acc = reinterpret_cast<double*>(smem);                                   // [W]   numeric
    uint32_t* claim = reinterpret_cast<uint32_t*>(smem + (NUMERIC ? 8u * W : 0u));  // [W]   numeric
    uint8_t* flag = smem + (NUMERIC ? 12u * W : 0u);                                 // [W]
    __shared__ double wa[kPanelThreads];
    __shared__ uint32_t ws[kPanelThreads], wl[kPanelThreads], wscan[kPanelThreads];
    __shared__ uint32_t tmp[kPanelThreads / 32 + 1];
    __shared__ uint32_t s_item;
    const uint32_t t = threadIdx.x;

    for (uint32_t i = t; i < W; i += kPanelThreads) {
        flag[i] = 0;
        if (NUMERIC) claim[i] = kNoClaim;
    }
    const uint32_t P1 = op.npanels + 1;

    for (;;) {
        __syncthreads();
        if (t == 0) s_item = atomicAdd(work_counter, 1u);
        __syncthreads();
        const uint32_t item_i = s_item;
        if (item_i >= nitems) break;
        const WorkItem it = items[item_i];
        const uint32_t row = it.row, p = it.panel;
        const uint32_t base = p << op.panel_log2;
        const uint32_t ka = op.row_start[row], kb = op.row_start[row + 1];

        for (uint32_t kw = ka; kw < kb; kw += kPanelThreads) {
            const uint32_t k = kw + t;
            uint32_t L = 0, s = 0;
            double a = 0.0;
            if (k < kb) {
                const int32_t f = op.a_fib[k];
                if (f >= 0) {
                    uint32_t e;
                    if (op.panel_off) {
                        s = op.panel_off[(uint64_t)f * P1 + p];
                        e = op.panel_off[(uint64_t)f * P1 + p + 1];
                    } else {
                        s = op.fib_start[f];
                        e = op.fib_start[f + 1];
                    }
                    L = e - s;
                    if (NUMERIC) a = op.a_val[k];
                }
            }
            uint32_t total;
            const uint32_t excl = block_exclusive_scan<uint32_t, kPanelThreads>(L, tmp, &total);
            ws[t] = s;
            wl[t] = L;
            wscan[t] = excl;
            if (NUMERIC) wa[t] = a;
            __syncthreads();

            uint32_t kcur = 0;
            for (uint32_t c0 = 0; c0 < total; c0 += kPanelThreads) {
                while (kcur + 1 < kPanelThreads && wscan[kcur] + wl[kcur] <= c0) ++kcur;
                const uint32_t cend = min(c0 + kPanelThreads, total);
                const bool single = wscan[kcur] + wl[kcur] >= cend;
                const uint32_t pi = c0 + t;
                bool valid = pi < total;
                uint32_t kk = kcur;
                if (!single && valid) {
                    uint32_t lo = kcur, hi = kPanelThreads;
                    while (hi - lo > 1) {
                        const uint32_t mid = (lo + hi) >> 1;
                        if (wscan[mid] <= pi) lo = mid; else hi = mid;
                    }
                    kk = lo;
                }
                uint32_t col = 0;
                double v = 0.0;
                if (valid) {
                    const uint32_t j = ws[kk] + (pi - wscan[kk]);
                    col = op.b_col[j] - base;
                    if (col >= W) {  // impossible for a correct panel split; never touch memory
                        atomicOr(op.err, 1u);
                        valid = false;
                        col = 0;
                    }
                    if (NUMERIC) v = __dmul_rn(wa[kk], op.b_val[j]);
                }
                if (!NUMERIC) {
                    if (valid) flag[col] = 1;
                } else if (single) {
                    if (valid) {
                        if (flag[col]) acc[col] = __dadd_rn(acc[col], v);
                        else { acc[col] = v; flag[col] = 1; }
                    }
                    __syncthreads();
                } else {
                    // several A nonzeros in this chunk: apply per column in stream order
                    bool pending = valid;
                    for (;;) {
                        if (pending) atomicMin(&claim[col], t);
                        __syncthreads();
                        const bool mine = pending && claim[col] == t;
                        __syncthreads();
                        if (mine) {
                            if (flag[col]) acc[col] = __dadd_rn(acc[col], v);
                            else { acc[col] = v; flag[col] = 1; }
                            claim[col] = kNoClaim;
                            pending = false;
                        }
                        if (!__syncthreads_or(pending)) break;
                    }
                }
            }
            __syncthreads();
        }

        // count / emit the panel in column order, clearing it for the next item
        const uint32_t per = W / kPanelThreads;  // W >= 256
        const uint32_t lo = t * per;
        uint32_t cnt = 0;
        for (uint32_t i = 0; i < per; ++i) cnt += flag[lo + i];
        uint32_t total;
        const uint32_t excl = block_exclusive_scan<uint32_t, kPanelThreads>(cnt, tmp, &total);
        if (NUMERIC) {
            uint64_t o = out.item_off[it.slot] + excl;
            for (uint32_t i = 0; i < per; ++i) {
                if (flag[lo + i]) {
                    write_entry(op, out, o++, row, base + lo + i, acc[lo + i]);
                    flag[lo + i] = 0;
                }
            }
        } else {
            for (uint32_t i = 0; i < per; ++i) flag[lo + i] = 0;
            if (t == 0) counts[it.slot] = total;
        }
    }
}

void launch_panel_items(bool numeric, const Operands& op, const WorkItem* items, uint32_t nitems, uint64_t* counts,
                        const OutputView& out, uint32_t* work_counter, int num_sms, cudaStream_t st) {
    if (nitems == 0) return;
    const uint32_t W = 1u << op.panel_log2;
    const size_t smem = numeric ? (size_t)13 * W : (size_t)W;
    PTC_CUDA(cudaMemsetAsync(work_counter, 0, sizeof(uint32_t), st));
    int per_sm = 1;
    if (numeric) {
        PTC_CUDA(cudaFuncSetAttribute(panel_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        PTC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, panel_kernel<true>, kPanelThreads, smem));
    } else {
        PTC_CUDA(cudaFuncSetAttribute(panel_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        PTC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, panel_kernel<false>, kPanelThreads, smem));
    }
    per_sm = per_sm < 1 ? 1 : per_sm;
    const uint32_t grid = (uint32_t)std::min<uint64_t>(nitems, (uint64_t)num_sms * per_sm);
    if (numeric)
        panel_kernel<true><<<grid, kPanelThreads, smem, st>>>(op, items, nitems, counts, out, work_counter);
    else
        panel_kernel<false><<<grid, kPanelThreads, smem, st>>>(op, items, nitems, counts, out, work_counter);
    count_launch();
    PTC_CHECK_LAUNCH();
}

}  // namespace ptc
