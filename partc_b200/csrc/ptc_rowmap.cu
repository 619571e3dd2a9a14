// Large rows, one block per row over a bitmap of the row's columns in shared memory (the
// reference's numeric pass for rows with a hash SPA, fksCuckooTC.hpp:257-355, and its per-row
// accumulator fksCuckooSPA.hpp, without a hash table).
//
// For one row the block
//   A. sets a bit for the column of every product (any order): the distinct columns are the
//      row's output entries, and their count is the row's exact output nnz;
//   B. turns the bitmap into word prefixes: output entry of column c = set bits before c, so the
//      entries come out in column order at known positions -- no table, no probing;
//   C. applies the products to the output values at those positions, one A nonzero after the
//      other in COO input order (the reference's summation order, fksCuckooTC.hpp:294-337;
//      Aux_data keeps insertion order, fksCuckoo.hpp:233-255).  A fiber never repeats a column,
//      so the products of one A nonzero go in parallel; a block barrier separates nonzeros.  A
//      run of A nonzeros with short fibers is applied by one warp, nonzero after nonzero, between
//      two barriers.  The first product of a column assigns its value, the others add
//      (__dmul_rn / __dadd_rn: no FMA), so values are bit-identical to the reference's;
//   D. writes the index tuples in column order.
// The values are read and written in the row's own output range (it stays in L2 while the row is
// worked on); the index tuples are written once.
//
// Modes: kRowmapCount writes the row's exact count (the symbolic pass of the two-phase path);
// kRowmapExact writes at precomputed offsets; kRowmapClaim takes the row's output range with one
// atomicAdd once the count is known (the learned path, which has no symbolic pass).
#include <algorithm>

#include "ptc_rowmap.cuh"

namespace ptc {

namespace {

constexpr int kRmThreads = 256;
constexpr int kRmWarps = kRmThreads / 32;
constexpr uint32_t kShortFiber = 64;             // fibers shorter than this go to one warp
constexpr size_t kRmSmemLimit = 220 * 1024;      // dynamic shared memory of one block at most

__host__ __device__ __forceinline__ uint32_t rm_words(uint64_t ncols) {
    return (uint32_t)(((ncols + 31) / 32 + 3) & ~3ull);  // a multiple of 4 for 16-byte clears
}

// output position of column c: base + set bits of the row before c
__device__ __forceinline__ uint64_t col_pos(const uint32_t* bits, const uint32_t* pref, uint32_t c) {
    const uint32_t w = c >> 5;
    return (uint64_t)pref[w] + (uint32_t)__popc(bits[w] & ((1u << (c & 31)) - 1u));
}

constexpr int kRmUnroll = 4;  // products in flight per thread

// Products j = j0 + i * stride (i < kRmUnroll, j < L) of one fiber (entries from s), scaled by
// a, applied to the row's output values: the first product of a column assigns, later ones add
// (the block barriers between A nonzeros order them).  The columns of one fiber are distinct,
// so the loads of all kRmUnroll products are issued before any value is written.
__device__ __forceinline__ void apply_products(const Operands& op, uint32_t* wrote, const uint32_t* bits,
                                               const uint32_t* pref, double* val, uint32_t s, uint32_t L,
                                               double a, uint32_t j0, uint32_t stride) {
    uint32_t c[kRmUnroll];
    double p[kRmUnroll];
#pragma unroll
    for (int i = 0; i < kRmUnroll; ++i) {
        const uint32_t j = j0 + i * stride;
        c[i] = 0xffffffffu;
        if (j < L) {
            c[i] = __ldg(op.b_col + s + j);
            p[i] = __ldg(op.b_val + s + j);
        }
    }
    double* dst[kRmUnroll];
    bool add[kRmUnroll];
#pragma unroll
    for (int i = 0; i < kRmUnroll; ++i) {
        add[i] = false;
        dst[i] = nullptr;
        if (c[i] != 0xffffffffu) {
            const uint32_t w = c[i] >> 5, b = 1u << (c[i] & 31);
            dst[i] = val + col_pos(bits, pref, c[i]);
            add[i] = (atomicOr(&wrote[w], b) & b) != 0;
            p[i] = __dmul_rn(a, p[i]);
        }
    }
    double old[kRmUnroll];
#pragma unroll
    for (int i = 0; i < kRmUnroll; ++i)
        if (add[i]) old[i] = __ldcg(dst[i]);
#pragma unroll
    for (int i = 0; i < kRmUnroll; ++i)
        if (dst[i]) __stcg(dst[i], add[i] ? __dadd_rn(old[i], p[i]) : p[i]);
}

constexpr uint32_t kRmUnit = 1024;  // fiber entries per unit of phase A

// Fibers of A nonzeros kw .. kw + nk of a row into shared memory (thread t: nonzero kw + t):
// start and length of the matching fiber (length 0 without one) and the A value.
__device__ __forceinline__ void load_window(const Operands& op, uint32_t kw, uint32_t nk, uint32_t* ws, uint32_t* wl,
                                            double* wa) {
    const uint32_t t = threadIdx.x;
    if (t < nk) {
        const int32_t f = op.a_fib[kw + t];
        uint32_t s = 0, L = 0;
        if (f >= 0) {
            s = op.fib_start[f];
            L = op.fib_start[f + 1] - s;
        }
        ws[t] = s;
        wl[t] = L;
        wa[t] = op.a_val[kw + t];
    }
}

template <int MODE, int FA, int FB>
__global__ void __launch_bounds__(kRmThreads, 3)
    rowmap_kernel(Operands op, const uint32_t* __restrict__ rows, uint32_t nrows, uint64_t* __restrict__ row_d,
                  const uint64_t* __restrict__ row_off, OutputView out, uint32_t* __restrict__ work_counter,
                  uint32_t nwords, uint32_t* __restrict__ panel_cnt, const uint64_t* __restrict__ pbase) {
    extern __shared__ __align__(16) uint32_t sm[];
    // the count mode needs the bitmap alone
    uint32_t* bits = sm;                 // [nwords] columns of the row
    uint32_t* wrote = sm + nwords;       // [nwords] columns that hold a value already
    uint32_t* pref = sm + 2 * nwords;    // [nwords] set bits before each word
    __shared__ uint32_t ws[kRmThreads], wl[kRmThreads];  // a window of the row's A nonzeros:
    __shared__ double wa[kRmThreads];                    // fiber start, length, A value
    __shared__ uint32_t tmp[kRmWarps + 1];
    __shared__ uint32_t s_item;
    __shared__ uint64_t s_base;
    const uint32_t t = threadIdx.x, lane = lane_id(), warp = t >> 5;
    {
        uint4* b4 = reinterpret_cast<uint4*>(sm);
        const uint32_t n4 = (MODE == kRowmapCount ? nwords : 2 * nwords) / 4;  // bits (and wrote)
        for (uint32_t i = t; i < n4; i += kRmThreads) b4[i] = make_uint4(0, 0, 0, 0);
    }

    for (;;) {
        __syncthreads();
        if (t == 0) s_item = atomicAdd(work_counter, 1u);
        __syncthreads();
        const uint32_t item = s_item;
        if (item >= nrows) break;
        const uint32_t row = rows[item];
        const uint32_t ka = op.row_start[row], kb = op.row_start[row + 1];
        // the row's columns: the contraction's, or in a batch its item's (local ids)
        const uint32_t bitem = op.row_item ? op.row_item[row] : 0u;
        const uint32_t nw = (uint32_t)(((op.row_item ? (uint64_t)op.item_cols[bitem] : op.ncols) + 31) / 32);

        // A. bitmap of the row's columns.  A window of up to kRmThreads A nonzeros at a time: their
        // fibers (start, length, A value) are read in parallel into shared memory, then every
        // fiber is cut into units of kRmUnit entries that the warps take in turn (lanes over
        // entries), so one long fiber does not hold the block up.
        for (uint32_t kw = ka; kw < kb; kw += kRmThreads) {
            const uint32_t nk = min((uint32_t)kRmThreads, kb - kw);
            load_window(op, kw, nk, ws, wl, wa);
            __syncthreads();
            uint32_t unit = 0;
            for (uint32_t i = 0; i < nk; ++i) {
                const uint32_t L = wl[i], s = ws[i];
                const uint32_t nu = (L + kRmUnit - 1) / kRmUnit;
                for (uint32_t u = (warp + kRmWarps - unit % kRmWarps) % kRmWarps; u < nu; u += kRmWarps) {
                    const uint32_t e = min(L, (u + 1) * kRmUnit);
                    for (uint32_t j = u * kRmUnit + lane; j < e; j += 32 * kRmUnroll) {
                        uint32_t c[kRmUnroll];
#pragma unroll
                        for (int q = 0; q < kRmUnroll; ++q)
                            c[q] = j + q * 32 < e ? __ldg(op.b_col + s + j + q * 32) : 0xffffffffu;
#pragma unroll
                        for (int q = 0; q < kRmUnroll; ++q)
                            if (c[q] != 0xffffffffu) atomicOr(&bits[c[q] >> 5], 1u << (c[q] & 31));
                    }
                }
                unit += nu;
            }
            __syncthreads();
        }

        if (MODE == kRowmapCount) {
            // the row's output count per fine panel (panels are whole bitmap words: 2^panel_log2
            // >= 32 columns) when panel_cnt is given, and in total
            uint32_t mine = 0;
            if (panel_cnt) {
                const uint32_t wpp = (1u << op.panel_log2) >> 5;
                const uint64_t pb = pbase ? pbase[item] : (uint64_t)item * op.npanels;
                const uint32_t pn = pbase ? (uint32_t)(pbase[item + 1] - pbase[item]) : op.npanels;
                for (uint32_t p = t; p < pn; p += kRmThreads) {
                    uint32_t c = 0;
                    for (uint32_t w = p * wpp; w < min(nw, (p + 1) * wpp); ++w) c += __popc(bits[w]);
                    panel_cnt[pb + p] = c;
                    mine += c;
                }
            } else {
                for (uint32_t w = t; w < nw; w += kRmThreads) mine += __popc(bits[w]);
            }
            uint32_t count;
            block_exclusive_scan<uint32_t, kRmThreads>(mine, tmp, &count);
            if (t == 0) atomicAdd(reinterpret_cast<unsigned long long*>(&row_d[row]), (unsigned long long)count);
        } else {
            // B. word prefixes: thread t takes words [t * per, (t + 1) * per)
            const uint32_t per = (nw + kRmThreads - 1) / kRmThreads;
            const uint32_t w0 = min(nw, t * per), w1 = min(nw, w0 + per);
            uint32_t mine = 0;
            for (uint32_t w = w0; w < w1; ++w) mine += __popc(bits[w]);
            uint32_t count;
            uint32_t run = block_exclusive_scan<uint32_t, kRmThreads>(mine, tmp, &count);
            for (uint32_t w = w0; w < w1; ++w) {
                pref[w] = run;
                run += __popc(bits[w]);
            }
            if (t == 0) {
                uint64_t base = 0;
                if (MODE == kRowmapExact) {
                    base = row_off[row];
                } else {
                    base = claim_output(op, out, row, count);
                    if (out.item_count) out.item_count[item] = count;  // the row's exact count
                    if (base == ~0ull) {  // no room left: the row runs again after the output grows
                        const uint32_t f = atomicAdd(out.fail_count, 1u);
                        out.fail_list[f] = item;
                    }
                }
                s_base = base;
            }
            __syncthreads();
            const uint64_t base = s_base;
            if (base != ~0ull) {
                // where the row's entries go: entry base + i of the contraction, or of the batch's
                // block (item layout: values from val0, index tuples of the item's own order)
                uint64_t vbase = base, ibase = base * (op.fa + op.fb);
                uint32_t colbase = 0, ifa = op.fa, ifb = op.fb;
                if (op.row_item) {
                    const ItemOut io = op.item_out[bitem];
                    vbase = io.val0 + (base - io.ent0);
                    ifa = io.fa;
                    ifb = io.fb;
                    ibase = io.idx0 + (base - io.ent0) * (ifa + ifb);
                    colbase = io.colbase;
                }
                double* val = out.val + vbase;
                // C. products, one A nonzero after the other
                for (uint32_t kw = ka; kw < kb; kw += kRmThreads) {
                    const uint32_t nk = min((uint32_t)kRmThreads, kb - kw);
                    if (kb - ka > kRmThreads) {  // (a row of one window still has it from phase A)
                        load_window(op, kw, nk, ws, wl, wa);
                        __syncthreads();
                    }
                    for (uint32_t i = 0; i < nk;) {
                        const uint32_t L = wl[i];
                        if (L >= kShortFiber) {
                            const uint32_t s = ws[i];
                            const double a = wa[i];
                            for (uint32_t j = t; j < L; j += kRmThreads * kRmUnroll)
                                apply_products(op, wrote, bits, pref, val, s, L, a, j, kRmThreads);
                            ++i;
                        } else {
                            // a run of short fibers: warp 0 applies them one after the other
                            uint32_t r = i;
                            while (r < nk && wl[r] < kShortFiber) ++r;
                            if (warp == 0) {
                                for (uint32_t q = i; q < r; ++q) {
                                    const uint32_t Lq = wl[q];
                                    for (uint32_t j = lane; j < Lq; j += 32 * kRmUnroll)
                                        apply_products(op, wrote, bits, pref, val, ws[q], Lq, wa[q], j, 32);
                                    __syncwarp();
                                }
                            }
                            i = r;
                        }
                        __syncthreads();  // the next A nonzero sees this one's values
                    }
                }

                // D. index tuples in column order.  Entry o of the row holds column c.
                uint32_t rt[FA > 0 ? FA : 1];
                if (FA > 0)
                    for (int m = 0; m < FA; ++m) rt[m] = op.row_tuple[(uint64_t)row * FA + m];
                auto write_tuple = [&](uint64_t o, uint32_t c) {
                    if (FA > 0) {
                        uint32_t* dst = out.idx + ibase + o * (FA + FB);
                        if (FA == 2 && FB == 2) {
                            const uint2 ct = *reinterpret_cast<const uint2*>(op.col_tuple + (uint64_t)c * 2);
                            __stcs(reinterpret_cast<uint4*>(dst), make_uint4(rt[0], rt[1], ct.x, ct.y));
                        } else if (FA == 1 && FB == 1) {
                            __stcs(reinterpret_cast<uint2*>(dst), make_uint2(rt[0], op.col_tuple[c]));
                        } else {
                            for (int q = 0; q < FA; ++q) dst[q] = rt[q];
                            for (int q = 0; q < FB; ++q) dst[FA + q] = op.col_tuple[(uint64_t)c * FB + q];
                        }
                    } else {
                        // any order; in a batch the row and column tuples are stored with the
                        // batch's widest strides (op.fa, op.fb), the entry with the item's
                        uint32_t* dst = out.idx + ibase + o * (ifa + ifb);
                        const uint32_t cg = c + colbase;
                        for (uint32_t q = 0; q < ifa; ++q) dst[q] = op.row_tuple[(uint64_t)row * op.fa + q];
                        for (uint32_t q = 0; q < ifb; ++q) dst[ifa + q] = op.col_tuple[(uint64_t)cg * op.fb + q];
                    }
                    if (out.row_of) {
                        out.row_of[base + o] = row;
                        out.col_of[base + o] = c;
                    }
                };
                if ((uint64_t)count * 2 > (uint64_t)nw * 32) {
                    // a dense row: a warp per bitmap word, lanes over its bits, so the set lanes
                    // write consecutive entries
                    for (uint32_t w = warp; w < nw; w += kRmWarps) {
                        const uint32_t m = bits[w];
                        if ((m >> lane) & 1u) write_tuple(pref[w] + __popc(m & lanemask_lt()), (w << 5) | lane);
                    }
                } else {
                    // a sparse row: a thread per word (consecutive words per warp), its set bits in turn
                    for (uint32_t w = t; w < nw; w += kRmThreads) {
                        uint32_t m = bits[w];
                        uint64_t o = pref[w];
                        while (m) {
                            write_tuple(o++, (w << 5) | (uint32_t)(__ffs(m) - 1));
                            m &= m - 1;
                        }
                    }
                }
            }
        }
        __syncthreads();
        // clear the row's words for the next row
        for (uint32_t w = t; w < nw; w += kRmThreads) {
            bits[w] = 0;
            if (MODE != kRowmapCount) wrote[w] = 0;
        }
    }
}

template <int MODE>
void launch_mode(const Operands& op, const uint32_t* rows, uint32_t nrows, uint64_t* row_d, const uint64_t* row_off,
                 const OutputView& out, uint32_t* work_counter, int num_sms, cudaStream_t st,
                 uint32_t* panel_cnt = nullptr, const uint64_t* pbase = nullptr) {
    auto kernel = rowmap_kernel<MODE, 0, 0>;
    const bool plain = !out.row_of && !op.row_item;
    if (MODE == kRowmapCount || (plain && op.fa == 2 && op.fb == 2)) kernel = rowmap_kernel<MODE, 2, 2>;
    else if (plain && op.fa == 1 && op.fb == 1) kernel = rowmap_kernel<MODE, 1, 1>;
    else if (plain && op.fa == 1 && op.fb == 2) kernel = rowmap_kernel<MODE, 1, 2>;
    else if (plain && op.fa == 2 && op.fb == 1) kernel = rowmap_kernel<MODE, 2, 1>;
    const uint32_t nwords = rm_words(op.ncols);
    const size_t smem = (size_t)(MODE == kRowmapCount ? 1 : 3) * nwords * sizeof(uint32_t);
    PTC_CUDA(cudaMemsetAsync(work_counter, 0, sizeof(uint32_t), st));
    PTC_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 1;
    PTC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kRmThreads, smem));
    per_sm = per_sm < 1 ? 1 : per_sm;
    const uint32_t grid = (uint32_t)std::min<uint64_t>(nrows, (uint64_t)num_sms * per_sm);
    kernel<<<grid, kRmThreads, smem, st>>>(op, rows, nrows, row_d, row_off, out, work_counter, nwords, panel_cnt,
                                           pbase);
    count_launch();
    PTC_CHECK_LAUNCH();
}

}  // namespace

__global__ void table_row_flags_kernel(const uint32_t* __restrict__ rows, uint64_t n, const uint64_t* __restrict__ row_off,
                                       const uint64_t* __restrict__ row_flops, uint32_t* __restrict__ flag) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t r = rows[i];
    flag[i] = (row_off[r + 1] - row_off[r] != row_flops[r]) ? 1u : 0u;
}

__global__ void scatter_counts_kernel(const uint32_t* __restrict__ rows, uint64_t n, const uint32_t* __restrict__ cnt,
                                      uint64_t* __restrict__ row_actual) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) row_actual[rows[i]] = cnt[i];
}

void launch_table_row_flags(const uint32_t* rows, uint64_t n, const uint64_t* row_off, const uint64_t* row_flops,
                            uint32_t* flag, cudaStream_t st) {
    if (n == 0) return;
    table_row_flags_kernel<<<ceil_div_u32(n, 256), 256, 0, st>>>(rows, n, row_off, row_flops, flag);
    count_launch();
    PTC_CHECK_LAUNCH();
}

void launch_scatter_counts(const uint32_t* rows, uint64_t n, const uint32_t* cnt, uint64_t* row_actual,
                           cudaStream_t st) {
    if (n == 0) return;
    scatter_counts_kernel<<<ceil_div_u32(n, 256), 256, 0, st>>>(rows, n, cnt, row_actual);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// key[i] = the wave holding rows[i] (waves start at rows wave_row[0..nwaves)), idx[i] = i
__global__ void row_wave_kernel(const uint32_t* __restrict__ rows, uint32_t n, const uint32_t* __restrict__ wave_row,
                                uint32_t nwaves, uint64_t* __restrict__ key, uint32_t* __restrict__ idx) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t r = rows[i];
    uint32_t lo = 0, hi = nwaves;  // last wave w with wave_row[w] <= r
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (wave_row[mid] <= r) lo = mid; else hi = mid;
    }
    key[i] = lo;
    idx[i] = i;
}

void launch_row_wave(const uint32_t* rows, uint32_t n, const uint32_t* wave_row, uint32_t nwaves, uint64_t* key,
                     uint32_t* idx, cudaStream_t st) {
    if (n == 0) return;
    row_wave_kernel<<<ceil_div_u32(n, 256), 256, 0, st>>>(rows, n, wave_row, nwaves, key, idx);
    count_launch();
    PTC_CHECK_LAUNCH();
}

void launch_row_counts(const Operands& op, const uint32_t* rows, uint32_t nrows, uint32_t* panel_cnt,
                       const uint64_t* pbase, uint64_t* row_d, uint32_t* work_counter, int num_sms, cudaStream_t st) {
    if (nrows == 0) return;
    PTC_REQUIRE(op.ncols <= row_counts_max_cols() && (op.row_item == nullptr || op.item_cols != nullptr) &&
                    (!panel_cnt || op.panel_log2 >= 5),
                PTC_ERR_INTERNAL, "bitmap count: too many columns, or panels narrower than a bitmap word");
    launch_mode<kRowmapCount>(op, rows, nrows, row_d, nullptr, OutputView{}, work_counter, num_sms, st, panel_cnt,
                              pbase);
}

uint64_t row_counts_max_cols() { return (uint64_t)(kRmSmemLimit / sizeof(uint32_t)) * 32 - 128; }

uint64_t rowmap_max_cols() {
    // three bitmaps' worth of words (bits, written, prefixes) in one block's shared memory
    return (uint64_t)(kRmSmemLimit / (3 * sizeof(uint32_t))) * 32 - 128;
}

void launch_rowmap(int mode, const Operands& op, const uint32_t* rows, uint32_t nrows, uint64_t* row_d,
                   const uint64_t* row_off, const OutputView& out, uint32_t* work_counter, int num_sms,
                   cudaStream_t st) {
    if (nrows == 0) return;
    PTC_REQUIRE(op.ncols <= rowmap_max_cols() && (op.row_item == nullptr || op.item_cols != nullptr),
                PTC_ERR_INTERNAL, "row bitmap kernel: at most rowmap_max_cols() columns per contraction");
    if (mode == kRowmapCount) launch_mode<kRowmapCount>(op, rows, nrows, row_d, row_off, out, work_counter, num_sms, st);
    else if (mode == kRowmapExact) launch_mode<kRowmapExact>(op, rows, nrows, row_d, row_off, out, work_counter, num_sms, st);
    else launch_mode<kRowmapClaim>(op, rows, nrows, row_d, row_off, out, work_counter, num_sms, st);
}

}  // namespace ptc
