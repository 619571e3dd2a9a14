// Sparse accumulators of the contraction (the reference's numeric pass, fksCuckooTC.hpp:180-357,
// and its per-row SPA hash tables, fksCuckooSPA.hpp), plus the exact symbolic pass.
//
// Summation order.  The reference computes each output entry as a left fold over the row's A
// nonzeros in COO input order, each term the rounded product a*b (fksCuckooTC.hpp:294-337;
// Aux_data keeps insertion order, fksCuckoo.hpp:233-255).  The numeric kernels keep exactly that
// order, so values are bit-identical to the reference:
//   * a row's products form a stream in (A nonzero, fiber entry) order;
//   * the products of one A nonzero have distinct columns (a fiber never repeats a B free key),
//     so they are applied concurrently without any ordering;
//   * products of different A nonzeros that meet in one column are applied in stream order --
//     by rank inside a warp (match_any), or by claim rounds inside a block.
// Products use __dmul_rn and sums __dadd_rn so nothing is contracted into an FMA.
#include <algorithm>

#include "ptc_spa.cuh"

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

// "no value yet" marker of an accumulator slot: a signalling-NaN payload that no product of
// finite or NaN operands can produce (device arithmetic returns the canonical NaN)
constexpr unsigned long long kNoValue = 0x7ff4deadbeef0001ull;

// applies product p to a slot; true when the slot held no value before
__device__ __forceinline__ bool accumulate(double* slot, double p) {
    const double v = *slot;
    const bool first = __double_as_longlong(v) == (long long)kNoValue;
    *slot = first ? p : __dadd_rn(v, p);
    return first;
}

// first entry of [lo, hi) (a fiber, sorted by column) whose column is >= c
__device__ __forceinline__ uint32_t col_lower_bound(const uint32_t* __restrict__ col, uint32_t lo, uint32_t hi,
                                                   uint32_t c) {
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (col[mid] < c) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Fiber entries [s, e) of fiber f whose columns fall in fine panels [p0, p1) (the whole fiber
// when the column space is a single panel).
__device__ __forceinline__ void part_range(const Operands& op, int32_t f, uint32_t p0, uint32_t p1, uint32_t& s,
                                           uint32_t& e) {
    if (op.panel_off) {
        const uint64_t b = (uint64_t)f * (op.npanels + 1);
        s = op.panel_off[b + p0];
        e = op.panel_off[b + p1];
    } else {
        s = op.fib_start[f];
        e = op.fib_start[f + 1];
        if (op.npanels > 1) {  // no split table: search the fiber for the panels' columns
            if (p0 > 0) s = col_lower_bound(op.b_col, s, e, p0 << op.panel_log2);
            if (p1 < op.npanels) e = col_lower_bound(op.b_col, s, e, p1 << op.panel_log2);
        }
    }
}

// ---------------------------------------------------------------------------------------------
// small rows: one warp per row, private open-addressing table in shared memory
// ---------------------------------------------------------------------------------------------

constexpr int kSmallWarps = 8;
constexpr uint32_t kSmallSlots = 1024;     // per warp
constexpr uint32_t kSmallMaxFlops = 512;   // rows with at most this many products
constexpr uint32_t kEmptyCol = 0xffffffffu;

uint32_t small_row_max_flops() { return kSmallMaxFlops; }

template <bool NUMERIC>
__global__ void __launch_bounds__(kSmallWarps * 32)
    small_rows_kernel(Operands op, const uint32_t* __restrict__ rows, uint32_t nrows, uint64_t* __restrict__ row_d,
                      const uint64_t* __restrict__ row_off, OutputView out) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t warp = threadIdx.x >> 5, lane = lane_id();
    uint32_t* keys = reinterpret_cast<uint32_t*>(smem) + warp * kSmallSlots;
    double* vals = reinterpret_cast<double*>(smem + kSmallWarps * kSmallSlots * sizeof(uint32_t)) + warp * kSmallSlots;
    for (uint32_t i = lane; i < kSmallSlots; i += 32) keys[i] = kEmptyCol;
    __syncwarp();

    for (uint32_t item = blockIdx.x * kSmallWarps + warp; item < nrows; item += gridDim.x * kSmallWarps) {
        const uint32_t row = rows[item];
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
        uint64_t o = NUMERIC ? row_off[row] : 0;
        const bool write = NUMERIC;
        for (uint32_t i = 0; i < kSmallSlots; i += 32) {
            const uint32_t sidx = i + lane;
            const uint32_t kc = keys[sidx];
            const bool occ = kc != kEmptyCol;
            const uint32_t mask = __ballot_sync(kFullMask, occ);
            if (write && occ) write_entry(op, out, o + __popc(mask & lanemask_lt()), row, kc, vals[sidx]);
            keys[sidx] = kEmptyCol;
            o += __popc(mask);
        }
        if (!NUMERIC && lane == 0) row_d[row] = nnew;
        __syncwarp();
    }
}

void launch_small_rows(bool numeric, const Operands& op, const uint32_t* rows, uint32_t nrows, uint64_t* row_d,
                       const uint64_t* row_off, const OutputView& out, cudaStream_t st) {
    if (nrows == 0) return;
    const size_t smem = kSmallWarps * kSmallSlots * (sizeof(uint32_t) + (numeric ? sizeof(double) : 0));
    const uint32_t grid = ceil_div_u32(nrows, kSmallWarps);
    if (numeric) {
        PTC_CUDA(cudaFuncSetAttribute(small_rows_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        small_rows_kernel<true><<<grid, kSmallWarps * 32, smem, st>>>(op, rows, nrows, row_d, row_off, out);
    } else {
        PTC_CUDA(cudaFuncSetAttribute(small_rows_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        small_rows_kernel<false><<<grid, kSmallWarps * 32, smem, st>>>(op, rows, nrows, row_d, row_off, out);
    }
    count_launch();
    PTC_CHECK_LAUNCH();
}

// ---------------------------------------------------------------------------------------------
// exact symbolic pass for the other rows: one block per row, a bitmap over the columns in shared
// memory; the first set of a bit is a new output entry, counted per fine panel.  When the columns
// do not fit one bitmap, the row is swept in windows of whole panels (each window reads only the
// fiber entries inside it), so the column count has no limit.
// ---------------------------------------------------------------------------------------------

constexpr int kSymThreads = 512;
constexpr int kSymItems = 4;
constexpr size_t kSymSmemBytes = 200 * 1024;  // bitmap + panel counters of one window

__global__ void __launch_bounds__(kSymThreads)
    sym_bitmap_kernel(Operands op, const uint32_t* __restrict__ rows, uint32_t nrows, uint32_t* __restrict__ panel_cnt,
                      const uint64_t* __restrict__ pbase, uint64_t* __restrict__ row_d,
                      uint32_t* __restrict__ work_counter, uint32_t wpanels) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t nwords = (uint32_t)((((uint64_t)wpanels << op.panel_log2) + 31) / 32);
    uint32_t* bits = reinterpret_cast<uint32_t*>(smem);   // [nwords]: the window's columns
    uint32_t* pc = bits + nwords;                         // [wpanels]: the window's panels
    __shared__ uint32_t ws[kSymThreads], wl[kSymThreads], wscan[kSymThreads];
    __shared__ uint32_t tmp[kSymThreads / 32 + 1];
    __shared__ uint32_t s_item;
    const uint32_t t = threadIdx.x;
    const uint32_t P = op.npanels;
    for (uint32_t i = t; i < nwords; i += kSymThreads) bits[i] = 0;
    for (uint32_t i = t; i < wpanels; i += kSymThreads) pc[i] = 0;

    for (;;) {
        __syncthreads();
        if (t == 0) s_item = atomicAdd(work_counter, 1u);
        __syncthreads();
        const uint32_t item = s_item;
        if (item >= nrows) break;
        const uint32_t row = rows[item];
        const uint32_t ka = op.row_start[row], kb = op.row_start[row + 1];
        const uint64_t pb = pbase ? pbase[item] : (uint64_t)item * P;
        const uint32_t pn = pbase ? (uint32_t)(pbase[item + 1] - pbase[item]) : P;  // the row's item's panels
        uint32_t dsum = 0;
        // a row's columns lie in its item's panels: only those counters and bitmap words are set
        for (uint32_t wp0 = 0; wp0 < pn; wp0 += wpanels) {
            const uint32_t wp1 = min(pn, wp0 + wpanels);
            const bool whole = wp0 == 0 && wp1 == pn;  // one window: every fiber entry is inside it
            const uint32_t wc0 = wp0 << op.panel_log2;
            for (uint32_t kw = ka; kw < kb; kw += kSymThreads) {
                const uint32_t k = kw + t;
                uint32_t L = 0, s = 0;
                if (k < kb) {
                    const int32_t f = op.a_fib[k];
                    if (f >= 0) {
                        uint32_t e;
                        if (whole) {
                            s = op.fib_start[f];
                            e = op.fib_start[f + 1];
                        } else {
                            part_range(op, f, wp0, wp1, s, e);
                        }
                        L = e - s;
                    }
                }
                uint32_t total;
                const uint32_t excl = block_exclusive_scan<uint32_t, kSymThreads>(L, tmp, &total);
                ws[t] = s;
                wl[t] = L;
                wscan[t] = excl;
                __syncthreads();
                for (uint32_t c0 = 0; c0 < total; c0 += kSymThreads * kSymItems) {
                    // blocked: thread t takes products [c0 + t*kSymItems, ... + kSymItems)
                    const uint32_t q0 = c0 + t * kSymItems;
                    uint32_t kk = 0;
                    if (q0 < total) {
                        uint32_t hi = kSymThreads;
                        while (hi - kk > 1) {
                            const uint32_t mid = (kk + hi) >> 1;
                            if (wscan[mid] <= q0) kk = mid; else hi = mid;
                        }
                    }
#pragma unroll
                    for (int i = 0; i < kSymItems; ++i) {
                        const uint32_t q = q0 + i;
                        uint32_t panel = 0xffffffffu;
                        if (q < total) {
                            while (kk + 1 < kSymThreads && wscan[kk] + wl[kk] <= q) ++kk;
                            const uint32_t col = op.b_col[ws[kk] + (q - wscan[kk])] - wc0;
                            const uint32_t bit = 1u << (col & 31);
                            const uint32_t old = atomicOr(&bits[col >> 5], bit);
                            if (!(old & bit)) panel = col >> op.panel_log2;
                        }
                        const uint32_t m = __match_any_sync(kFullMask, panel);
                        if (panel != 0xffffffffu && (m & lanemask_lt()) == 0) atomicAdd(&pc[panel], (uint32_t)__popc(m));
                    }
                }
                __syncthreads();
            }
            for (uint32_t p = t; p < wp1 - wp0; p += kSymThreads) {
                const uint32_t v = pc[p];
                panel_cnt[pb + wp0 + p] = v;
                dsum += v;
                pc[p] = 0;
            }
            const uint32_t rw = (uint32_t)((((uint64_t)(wp1 - wp0) << op.panel_log2) + 31) / 32);
            for (uint32_t i = t; i < rw; i += kSymThreads) bits[i] = 0;
            __syncthreads();
        }
        dsum = warp_sum(dsum);
        if (lane_id() == 0 && dsum) atomicAdd(reinterpret_cast<unsigned long long*>(&row_d[row]), (unsigned long long)dsum);
    }
}

// Panels of one window: as many as fit the shared-memory budget (bitmap + counters).
uint32_t sym_window_panels(uint32_t npanels, uint32_t panel_log2) {
    const uint64_t per_panel = ((1ull << panel_log2) + 31) / 32 * 4 + 4;  // bitmap words + counter
    const uint64_t fit = std::max<uint64_t>(1, kSymSmemBytes / per_panel);
    return (uint32_t)std::min<uint64_t>(npanels, fit);
}

void launch_sym_bitmap(const Operands& op, const uint32_t* rows, uint32_t nrows, uint32_t* panel_cnt,
                       const uint64_t* pbase, uint64_t* row_d,
                       uint32_t* work_counter, int num_sms, cudaStream_t st) {
    if (nrows == 0) return;
    const uint32_t wpanels = sym_window_panels(op.npanels, op.panel_log2);
    const uint32_t nwords = (uint32_t)((((uint64_t)wpanels << op.panel_log2) + 31) / 32);
    const size_t smem = (size_t)(nwords + wpanels) * sizeof(uint32_t);
    PTC_CUDA(cudaMemsetAsync(work_counter, 0, sizeof(uint32_t), st));
    PTC_CUDA(cudaFuncSetAttribute(sym_bitmap_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 1;
    PTC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sym_bitmap_kernel, kSymThreads, smem));
    per_sm = per_sm < 1 ? 1 : per_sm;
    const uint32_t grid = (uint32_t)std::min<uint64_t>(nrows, (uint64_t)num_sms * per_sm);
    sym_bitmap_kernel<<<grid, kSymThreads, smem, st>>>(op, rows, nrows, panel_cnt, pbase, row_d, work_counter,
                                                         wpanels);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// ---------------------------------------------------------------------------------------------
// numeric pass, warp tasks: one warp per task -- a row's columns in fine panels [p0, p1) -- with
// a private table in shared memory (dense: direct-mapped by column over at most kTaskDense
// columns; sparse: open addressing, at most kTaskSlots slots).  Warps take tasks one at a time
// from a counter, with no block-wide barrier.
//
// A task walks the row's A nonzeros 32 at a time: lane j finds its nonzero's fiber entries in the
// task's panels, a warp scan packs those products into chunks of 32 in stream order, and every
// lane takes one product of a chunk.  Inside a chunk, products of one column are applied in lane
// order (= stream order) by rank (match_any); chunks run in order.  So every output value is the
// left fold of its products in stream order, as in the reference.
// ---------------------------------------------------------------------------------------------

constexpr int kTaskWarps = 4;                               // warps per block
constexpr int kTaskBlocksPerSm = 8;                         // 32 resident warps per SM
constexpr uint32_t kTaskDense = 768;                        // columns of a dense task
constexpr uint32_t kTaskSlots = 512;                        // largest sparse table
constexpr size_t kTaskBytes = kTaskDense * sizeof(double);  // a warp's table (6 KiB)
// the sparse layout keeps values in vals[0, 512) and keys in the bytes of vals[512, 768)
static_assert(kTaskSlots * (sizeof(double) + sizeof(uint32_t)) <= kTaskBytes, "sparse layout fits a warp's region");
// Behind the table, the slots a task filled, in the order they were first written: the emission
// and the claim count visit those alone instead of every slot.  A task that fills more slots
// than the list holds is emitted by scanning the table.
constexpr uint32_t kListCap = 384;
constexpr size_t kWarpBytes = kTaskBytes + kListCap * sizeof(uint16_t);  // 6912 B: 8 blocks of 4 warps per SM
static_assert(kWarpBytes % 16 == 0, "every warp's region starts 16-byte aligned");

// load factor <= 0.5: linear probes stay short, and a warp waits for its longest one
uint32_t warp_task_capacity() { return kTaskSlots / 2; }
uint32_t warp_task_dense_columns() { return kTaskDense; }
uint32_t warp_task_min_bits() { return 6; }                   // 64 slots: two per lane
uint32_t warp_task_max_bits() { return 9; }

// A sub-range of at least this many products is streamed on its own (see warp_task_kernel)
constexpr uint32_t kStreamMin = 32;
constexpr int kStreamUnroll = 2;

// Slot of column `col` in an open-addressing table of tmask + 1 = tsize slots (linear probing,
// inserted with atomicCAS if absent), or -1 when the table is full.
__device__ __forceinline__ int table_slot(uint32_t* keys, uint32_t col, uint32_t tmask, uint32_t tsize) {
    uint32_t h = hash32(col) & tmask;
    for (uint32_t probe = 0; probe < tsize; ++probe) {
        const uint32_t cv = keys[h];
        if (cv == col) return (int)h;
        if (cv == kEmptyCol) {
            const uint32_t old = atomicCAS(&keys[h], kEmptyCol, col);
            if (old == kEmptyCol || old == col) return (int)h;
        }
        h = (h + 1) & tmask;
    }
    return -1;
}

// One chunk of 32 products of a task: lane l takes product q0 + l of the packed stream.
struct Chunk {
    uint32_t kk;    // source lane (the A nonzero of this window)
    uint32_t col;   // kEmptyCol past the end
    double bval;
};

__device__ __forceinline__ Chunk load_chunk(const Operands& op, uint32_t q0, uint32_t total, uint32_t incl,
                                            uint32_t s, uint32_t excl) {
    Chunk c;
    const uint32_t q = q0 + lane_id();
    // source lane: number of lanes whose inclusive end is <= q
    uint32_t kk = 0;
#pragma unroll
    for (uint32_t step = 16; step > 0; step >>= 1) {
        const uint32_t e = __shfl_sync(kFullMask, incl, kk + step - 1);
        if (e <= q) kk += step;
    }
    kk = min(kk, 31u);
    const uint32_t sk = __shfl_sync(kFullMask, s, kk);
    const uint32_t ek = __shfl_sync(kFullMask, excl, kk);
    c.kk = kk;
    c.col = kEmptyCol;
    c.bval = 0.0;
    if (q < total) {
        const uint32_t j = sk + (q - ek);
        c.col = __ldg(op.b_col + j);
        c.bval = __ldg(op.b_val + j);
    }
    return c;
}

// 32-entry groups a warp emits at a time (their column-tuple loads are in flight together)
constexpr int kEmitGroups = 2;

// The single-contraction output layout with fa = FA, fb = FB free modes: the column's index tuple,
// and output entry e written as row tuple rt (loaded once per task), column tuple ct and value v.
template <int FA, int FB>
__device__ __forceinline__ void load_col_tuple(const Operands& op, uint32_t col, uint32_t (&ct)[FB > 0 ? FB : 1]) {
    if constexpr (FB == 2) {
        const uint2 c = *reinterpret_cast<const uint2*>(op.col_tuple + (uint64_t)col * 2);
        ct[0] = c.x;
        ct[1] = c.y;
    } else {
        for (int k = 0; k < FB; ++k) ct[k] = op.col_tuple[(uint64_t)col * FB + k];
    }
}

template <int FA, int FB>
__device__ __forceinline__ void store_entry(const OutputView& out, uint64_t e, const uint32_t (&rt)[FA > 0 ? FA : 1],
                                            const uint32_t (&ct)[FB > 0 ? FB : 1], double v) {
    uint32_t* dst = out.idx + e * (FA + FB);
    if constexpr (FA == 2 && FB == 2) {
        __stcs(reinterpret_cast<uint4*>(dst), make_uint4(rt[0], rt[1], ct[0], ct[1]));
    } else if constexpr (FA == 1 && FB == 1) {
        __stcs(reinterpret_cast<uint2*>(dst), make_uint2(rt[0], ct[0]));
    } else {
        for (int k = 0; k < FA; ++k) dst[k] = rt[k];
        for (int k = 0; k < FB; ++k) dst[FA + k] = ct[k];
    }
    __stcs(out.val + e, v);
}

// Emit n slots of the warp's table, listed in `list` (n <= kListCap), as output entries
// base .. base + n - 1 (entry i holds list[i]), resetting those slots.  Every lane writes an
// entry, so positions need no ballot; kEmitGroups 32-entry groups at a time, so their tuple loads
// are in flight together.
template <int FA, int FB>
__device__ __forceinline__ void emit_list(const Operands& op, const OutputView& out, uint64_t base, uint32_t row,
                                          uint32_t c0, bool dense, uint32_t n, const uint16_t* list, double* vals,
                                          uint32_t* keys) {
    unsigned long long* vbits = reinterpret_cast<unsigned long long*>(vals);
    const uint32_t lane = lane_id();
    uint32_t rt[FA > 0 ? FA : 1];
    if (FA > 0)
        for (int m = 0; m < FA; ++m) rt[m] = op.row_tuple[(uint64_t)row * FA + m];
    for (uint32_t i = 0; i < n; i += 32 * kEmitGroups) {
        bool occ[kEmitGroups];
        uint32_t col[kEmitGroups];
        double v[kEmitGroups];
#pragma unroll
        for (int u = 0; u < kEmitGroups; ++u) {
            const uint32_t e = i + u * 32 + lane;
            occ[u] = e < n;
            if (occ[u]) {
                const uint32_t slot = list[e];
                v[u] = vals[slot];
                col[u] = dense ? c0 + slot : keys[slot];
                vbits[slot] = kNoValue;
                if (!dense) keys[slot] = kEmptyCol;
            }
        }
        if (base == ~0ull) continue;  // rerun later: nothing written
        if (FA > 0) {
            uint32_t ct[kEmitGroups][FB > 0 ? FB : 1];
#pragma unroll
            for (int u = 0; u < kEmitGroups; ++u)
                if (occ[u]) load_col_tuple<FA, FB>(op, col[u], ct[u]);
#pragma unroll
            for (int u = 0; u < kEmitGroups; ++u)
                if (occ[u]) store_entry<FA, FB>(out, base + i + u * 32 + lane, rt, ct[u], v[u]);
        } else {
#pragma unroll
            for (int u = 0; u < kEmitGroups; ++u)
                if (occ[u]) write_entry(op, out, base + i + u * 32 + lane, row, col[u], v[u]);
        }
    }
}

// Refill the list with the next filled slots of the table, scanning from slot `scan` (a multiple
// of 32) on while a whole 32-slot group still fits; returns how many were listed.  Emission of a
// task that filled more slots than the list holds: the slots come out in slot order.
__device__ __forceinline__ uint32_t list_refill(const double* vals, uint32_t tsize, uint16_t* list, uint32_t& scan) {
    const unsigned long long* vbits = reinterpret_cast<const unsigned long long*>(vals);
    uint32_t n = 0;
    while (scan < tsize && n + 32 <= kListCap) {
        const uint32_t sidx = scan + lane_id();
        const bool occ = vbits[sidx] != kNoValue;
        const uint32_t m = __ballot_sync(kFullMask, occ);
        if (occ) list[n + __popc(m & lanemask_lt())] = (uint16_t)sidx;
        n += __popc(m);
        scan += 32;
    }
    __syncwarp();
    return n;
}

// Appends the slots that lanes with `first` wrote first to the warp's list, in lane order; n counts
// every such slot, also past the list's end.
__device__ __forceinline__ void list_append(uint16_t* list, uint32_t& n, bool first, int slot) {
    const uint32_t m = __ballot_sync(kFullMask, first);
    if (m == 0) return;
    if (first) {
        const uint32_t p = n + __popc(m & lanemask_lt());
        if (p < kListCap) list[p] = (uint16_t)slot;
    }
    n += __popc(m);
}

template <int FA, int FB>
__global__ void __launch_bounds__(kTaskWarps * 32, kTaskBlocksPerSm)
    warp_task_kernel(Operands op, const PartItem* __restrict__ tasks, uint32_t ntasks, OutputView out,
                     uint32_t* __restrict__ work_counter, uint32_t* __restrict__ overflow) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t warp = threadIdx.x >> 5, lane = lane_id();
    double* vals = reinterpret_cast<double*>(smem + warp * kWarpBytes);
    unsigned long long* vbits = reinterpret_cast<unsigned long long*>(vals);
    uint32_t* keys = reinterpret_cast<uint32_t*>(vals + kTaskSlots);
    uint16_t* list = reinterpret_cast<uint16_t*>(smem + warp * kWarpBytes + kTaskBytes);
    for (uint32_t i = lane; i < kTaskDense; i += 32) vbits[i] = kNoValue;
    bool dense_layout = true;
    __syncwarp();

    // Tasks come from a counter one ahead: lane 0 takes the index of the following task while the
    // current one starts, so the atomic's latency is off the warp's path.
    uint32_t tn = 0;
    if (lane == 0) tn = atomicAdd(work_counter, 1u);
    uint32_t t = __shfl_sync(kFullMask, tn, 0);
    for (;;) {
        if (t >= ntasks) break;
        if (lane == 0) tn = atomicAdd(work_counter, 1u);
        const PartItem it = tasks[t];
        const bool dense = (it.mode & 1u) != 0;
        const uint32_t tsize = dense ? kTaskDense : (1u << (it.mode >> 1));
        const uint32_t tmask = tsize - 1;
        if (dense != dense_layout) {  // values are all empty after an emission; only keys differ
            if (dense) {
                for (uint32_t i = kTaskSlots + lane; i < kTaskDense; i += 32) vbits[i] = kNoValue;
            } else {
                for (uint32_t i = lane; i < kTaskSlots; i += 32) keys[i] = kEmptyCol;
            }
            dense_layout = dense;
            __syncwarp();
        }
        const uint32_t row = it.row;
        const uint32_t c0 = it.p0 << op.panel_log2;  // first column of the task
        const uint32_t ka = op.row_start[row], kb = op.row_start[row + 1];
        bool bad = false;  // table overflow or a column outside a dense task (never for exact sizes)
        uint32_t filled = 0;  // slots written so far (warp-uniform); the first kListCap are listed

        for (uint32_t kw = ka; kw < kb; kw += 32) {
            const uint32_t k = kw + lane;
            uint32_t L = 0, s = 0;
            double a = 0.0;
            if (k < kb) {
                const int32_t f = op.a_fib[k];
                if (f >= 0) {
                    uint32_t e;
                    part_range(op, f, it.p0, it.p1, s, e);
                    L = e - s;
                    a = op.a_val[k];
                }
            }
            // A nonzeros with at least kStreamMin products in the task are streamed one after the
            // other, 32 lanes over the sub-range, kStreamUnroll entries in flight per lane: the
            // columns of one sub-range are distinct, so no ordering is needed inside it.  Runs of
            // shorter sub-ranges between them are packed 32 products per step, in stream order,
            // and products meeting in one column are applied by rank (match_any).
            const uint32_t longm = __ballot_sync(kFullMask, L >= kStreamMin);
            uint32_t lo = 0;
            while (lo < 32) {
                const uint32_t m = longm & ~((1u << lo) - 1u);
                const uint32_t nl = m ? (uint32_t)(__ffs(m) - 1) : 32u;
                if (nl > lo) {  // lanes [lo, nl): short sub-ranges, packed
                    const uint32_t Lp = (lane >= lo && lane < nl) ? L : 0u;
                    const uint32_t incl = warp_inclusive_scan(Lp);
                    const uint32_t excl = incl - Lp;
                    const uint32_t total = __shfl_sync(kFullMask, incl, 31);
                    // software pipeline: the next chunk's fiber entries load while this one is applied
                    Chunk nxt = total > 0 ? load_chunk(op, 0, total, incl, s, excl) : Chunk{0u, kEmptyCol, 0.0};
                    for (uint32_t q0 = 0; q0 < total; q0 += 32) {
                        const Chunk cur = nxt;
                        if (q0 + 32 < total) nxt = load_chunk(op, q0 + 32, total, incl, s, excl);
                        const bool valid = cur.col != kEmptyCol;
                        const uint32_t col = cur.col;
                        const double ak = __shfl_sync(kFullMask, a, cur.kk);
                        const double prod = valid ? __dmul_rn(ak, cur.bval) : 0.0;
                        // products of a single A nonzero have distinct columns: no ordering inside
                        const uint32_t k0 = __shfl_sync(kFullMask, cur.kk, 0);
                        const bool single = __all_sync(kFullMask, !valid || cur.kk == k0);
                        int slot = -1;
                        uint32_t rank = 0;
                        if (dense) {
                            const uint32_t d = col - c0;
                            if (valid) {
                                if (d < kTaskDense) slot = (int)d;
                                else bad = true;
                            }
                            if (!single) rank = __popc(__match_any_sync(kFullMask, slot) & lanemask_lt());
                        } else {
                            uint32_t leader = lane;
                            if (!single) {
                                const uint32_t mm = __match_any_sync(kFullMask, col);
                                rank = __popc(mm & lanemask_lt());
                                leader = __ffs(mm) - 1;
                            }
                            if (valid && rank == 0) {
                                slot = table_slot(keys, col, tmask, tsize);
                                if (slot < 0) bad = true;
                            }
                            if (!single) slot = __shfl_sync(kFullMask, slot, leader);
                        }
                        const uint32_t maxr = single ? 0u : __reduce_max_sync(kFullMask, valid ? rank : 0u);
                        bool first = false;  // only a column's rank-0 product can find its slot empty
                        for (uint32_t r = 0; r <= maxr; ++r) {
                            if (valid && rank == r && slot >= 0) first |= accumulate(&vals[slot], prod);
                            __syncwarp();
                        }
                        list_append(list, filled, first, slot);
                    }
                }
                if (nl == 32) break;
                // lane nl: a long sub-range, streamed
                const uint32_t sk = __shfl_sync(kFullMask, s, nl), Lk = __shfl_sync(kFullMask, L, nl);
                const double ak = __shfl_sync(kFullMask, a, nl);
                for (uint32_t j0 = 0; j0 < Lk; j0 += 32 * kStreamUnroll) {
                    uint32_t cc[kStreamUnroll];
                    double bv[kStreamUnroll];
#pragma unroll
                    for (int u = 0; u < kStreamUnroll; ++u) {
                        const uint32_t j = j0 + u * 32 + lane;
                        cc[u] = kEmptyCol;
                        if (j < Lk) {
                            cc[u] = __ldg(op.b_col + sk + j);
                            bv[u] = __ldg(op.b_val + sk + j);
                        }
                    }
#pragma unroll
                    for (int u = 0; u < kStreamUnroll; ++u) {
                        int slot = -1;
                        bool first = false;
                        if (cc[u] != kEmptyCol) {
                            if (dense) {
                                const uint32_t d = cc[u] - c0;
                                slot = d < kTaskDense ? (int)d : -1;
                            } else {
                                slot = table_slot(keys, cc[u], tmask, tsize);
                            }
                            if (slot < 0) bad = true;
                            else first = accumulate(&vals[slot], __dmul_rn(ak, bv[u]));
                        }
                        list_append(list, filled, first, slot);
                    }
                }
                __syncwarp();  // the next A nonzero sees this one's values
                lo = nl + 1;
            }
        }

        // output position: exact, or claimed now that the count is known
        const bool any_bad = __any_sync(kFullMask, bad);
        uint64_t base = it.out_off;
        const uint32_t cnt = filled;  // every slot written is an output entry
        if (base == kClaimBit) {
            uint64_t b = ~0ull;
            if (lane == 0) {
                b = any_bad ? ~0ull : claim_output(op, out, row, cnt);
                if (b == ~0ull) {  // rerun this task exactly
                    const uint32_t f = atomicAdd(out.fail_count, 1u);
                    out.fail_list[f] = t;
                }
            }
            base = __shfl_sync(kFullMask, b, 0);
        } else if (any_bad) {
            if (lane == 0) atomicOr(overflow, 1u);  // exact sizes cannot overflow: report an internal error
            base = ~0ull;
        }
        if (out.item_count && lane == 0) out.item_count[t] = base == ~0ull ? 0u : cnt;
        // the listed slots; a task that filled more slots than the list holds lists and emits them
        // a part of the table at a time
        const bool listed = filled <= kListCap;
        uint32_t scan = listed ? tsize : 0u, n = listed ? filled : 0u;
        for (;;) {
            if (!listed) n = list_refill(vals, tsize, list, scan);
            emit_list<FA, FB>(op, out, base, row, c0, dense, n, list, vals, keys);
            if (scan >= tsize) break;
            if (base != ~0ull) base += n;
            __syncwarp();
        }
        __syncwarp();
        t = __shfl_sync(kFullMask, tn, 0);
    }
}

void launch_warp_tasks(const Operands& op, const PartItem* tasks, uint32_t ntasks, const OutputView& out,
                       uint32_t* work_counter, uint32_t* overflow, int num_sms, cudaStream_t st) {
    if (ntasks == 0) return;
    const size_t smem = kTaskWarps * kWarpBytes;
    PTC_CUDA(cudaMemsetAsync(work_counter, 0, sizeof(uint32_t), st));
    // the single-contraction layouts of the common free-mode counts get their own emission (the
    // general one also records rows and columns for the canonical order)
    auto kernel = warp_task_kernel<0, 0>;
    const bool plain = !op.row_item && !out.row_of;
    if (plain && op.fa == 2 && op.fb == 2) kernel = warp_task_kernel<2, 2>;
    else if (plain && op.fa == 1 && op.fb == 1) kernel = warp_task_kernel<1, 1>;
    else if (plain && op.fa == 1 && op.fb == 2) kernel = warp_task_kernel<1, 2>;
    else if (plain && op.fa == 2 && op.fb == 1) kernel = warp_task_kernel<2, 1>;
    // all of the SM's unified memory as shared memory: 8 blocks of 27 KiB
    PTC_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    int per_sm = 1;
    PTC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kTaskWarps * 32, smem));
    per_sm = per_sm < 1 ? 1 : per_sm;
    const uint32_t grid = (uint32_t)std::min<uint64_t>((ntasks + kTaskWarps - 1) / kTaskWarps, (uint64_t)num_sms * per_sm);
    kernel<<<grid, kTaskWarps * 32, smem, st>>>(op, tasks, ntasks, out, work_counter, overflow);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// ---------------------------------------------------------------------------------------------
// numeric pass, collision-free rows: a large row whose exact output count equals its products has
// no two products in one column, so each product is an output entry of its own (a single term:
// no sum, no table).  Block per row, warps over its A nonzeros, lanes over each fiber: entry
// (k, j) goes to row_off[row] + (products before k in the row) + (j - fiber start).
// ---------------------------------------------------------------------------------------------

constexpr int kCopyThreads = 256;

__global__ void __launch_bounds__(kCopyThreads)
    copy_rows_kernel(Operands op, const uint32_t* __restrict__ rows, uint32_t nrows,
                     const uint64_t* __restrict__ alen, const uint64_t* __restrict__ row_off, OutputView out) {
    const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
    for (uint32_t i = blockIdx.x; i < nrows; i += gridDim.x) {
        const uint32_t row = rows[i];
        const uint32_t ka = op.row_start[row], kb = op.row_start[row + 1];
        const uint64_t base = row_off[row] - alen[ka];
        for (uint32_t k = ka + warp; k < kb; k += kCopyThreads / 32) {
            const int32_t f = op.a_fib[k];
            if (f < 0) continue;
            const uint32_t s = op.fib_start[f], e = op.fib_start[f + 1];
            const double a = op.a_val[k];
            const uint64_t o = base + alen[k];
            for (uint32_t j = s + lane; j < e; j += 32)
                write_entry(op, out, o + (j - s), row, __ldg(op.b_col + j), __dmul_rn(a, __ldg(op.b_val + j)));
        }
    }
}

void launch_copy_rows(const Operands& op, const uint32_t* rows, uint32_t nrows, const uint64_t* alen,
                      const uint64_t* row_off, const OutputView& out, int num_sms, cudaStream_t st) {
    if (nrows == 0) return;
    const uint32_t grid = std::min<uint32_t>(nrows, (uint32_t)num_sms * 8);
    copy_rows_kernel<<<grid, kCopyThreads, 0, st>>>(op, rows, nrows, alen, row_off, out);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// ---------------------------------------------------------------------------------------------
// numeric pass for the rows of many A nonzeros: one block per part (a row's columns in fine
// panels [p0, p1)).  The part's columns are dealt to the block's 16 warps (interleaved for a dense
// part, by hash for a sparse one), and every warp keeps the columns it owns in a private table:
// dense over 384 columns, or open addressing over 256 slots.
//
// The part's products are taken in stream order, 1024 per round (thread t: products pos + t and
// pos + 512 + t).  A round is split stably by owner warp into a shared buffer (a warp-level
// match_any gives each product's rank among its warp's products of the same owner; per-(item,
// warp, owner) counts give the buckets' offsets), then each warp applies its bucket -- its columns' products, still in stream
// order -- 32 at a time with match_any ranks for equal columns, as a warp task does.  So every
// column's products are applied by one warp in stream order, with three block barriers per round
// and no claim rounds.
// ---------------------------------------------------------------------------------------------

constexpr int kPartThreads = 512;
constexpr int kPartWarps = kPartThreads / 32;            // 16 owners
constexpr uint32_t kOwnDense = 384;                      // dense columns a warp owns
constexpr uint32_t kOwnSlots = 256;                      // sparse slots a warp owns
constexpr size_t kOwnBytes = kOwnDense * sizeof(double);  // a warp's table (3 KiB)
static_assert(kOwnSlots * (sizeof(double) + sizeof(uint32_t)) <= kOwnBytes, "sparse layout fits a warp's region");
constexpr uint32_t kDenseCols = kOwnDense * kPartWarps;   // 6144 columns in a dense part
constexpr uint32_t kHashSlots = kOwnSlots * kPartWarps;   // 4096 slots in a sparse part
constexpr uint32_t kPartWindow = 128;                     // A nonzeros read at a time
constexpr int kRoundItems = 2;                            // products per thread in a round
constexpr uint32_t kRound = kRoundItems * kPartThreads;   // products in a round
constexpr size_t kRegionBytes = kOwnBytes * kPartWarps;   // 48 KiB of tables
// behind the tables: a round's products by owner (value, column); 60 KiB in all, 3 blocks per SM
constexpr size_t kPartSmemBytes = kRegionBytes + kRound * (sizeof(double) + sizeof(uint32_t));

// at most 5/8 of a sparse part's slots on average, so no warp's 256 slots fill up (a single
// panel with more entries becomes a dense part over that panel)
uint32_t hash_part_capacity() { return kHashSlots * 5 / 8; }
uint32_t hash_part_min_bits() { return 12; }  // every sparse part has all 16 x 256 slots
uint32_t dense_part_columns() { return kDenseCols; }

// largest k in [lo, kPartWindow) with wscan[k] <= q (zero-length nonzeros share the next one's
// start, so this is the nonzero holding product q)
__device__ __forceinline__ uint32_t find_nonzero(const uint32_t* wscan, uint32_t lo, uint32_t q) {
    uint32_t hi = kPartWindow;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (wscan[mid] <= q) lo = mid; else hi = mid;
    }
    return lo;
}

// owner warp of a column of the part, and its slot hint: the local dense index, or the hash
// bits above the owner's for the sparse table's first probe
__device__ __forceinline__ uint32_t part_owner(uint32_t col, uint32_t lo, bool dense, uint32_t& hint) {
    if (dense) {
        const uint32_t d = col - lo;
        hint = d >> 4;
        return d & (kPartWarps - 1);
    }
    const uint32_t h = hash32(col);
    hint = h >> 4;
    return h & (kPartWarps - 1);
}

// Slot of column `col` in a warp's sparse table (linear probing from `hint`, inserted with
// atomicCAS if absent), or -1 when the table is full.
__device__ __forceinline__ int own_slot(uint32_t* keys, uint32_t col, uint32_t hint) {
    uint32_t h = hint & (kOwnSlots - 1);
    for (uint32_t probe = 0; probe < kOwnSlots; ++probe) {
        const uint32_t cv = keys[h];
        if (cv == col) return (int)h;
        if (cv == kEmptyCol) {
            const uint32_t old = atomicCAS(&keys[h], kEmptyCol, col);
            if (old == kEmptyCol || old == col) return (int)h;
        }
        h = (h + 1) & (kOwnSlots - 1);
    }
    return -1;
}

__global__ void __launch_bounds__(kPartThreads, 3)
    hash_part_kernel(Operands op, const PartItem* __restrict__ parts, uint32_t nparts, OutputView out,
                     uint32_t* __restrict__ work_counter, uint32_t* __restrict__ overflow) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t t = threadIdx.x, lane = lane_id(), warp = t >> 5;
    double* vals = reinterpret_cast<double*>(smem + warp * kOwnBytes);  // this warp's table
    unsigned long long* vbits = reinterpret_cast<unsigned long long*>(vals);
    uint32_t* keys = reinterpret_cast<uint32_t*>(vals + kOwnSlots);
    double* bval = reinterpret_cast<double*>(smem + kRegionBytes);                     // a round's products,
    uint32_t* bcol = reinterpret_cast<uint32_t*>(smem + kRegionBytes + kRound * sizeof(double));  // by owner
    __shared__ double wa[kPartWindow];
    __shared__ uint32_t ws[kPartWindow], wscan[kPartWindow];
    __shared__ __align__(16) uint32_t cnt4[kRoundItems][kPartWarps][4];  // [item][warp]: bytes per owner
    __shared__ uint16_t off[kRoundItems][kPartWarps][kPartWarps];        // [item][warp][owner]: buffer position
    __shared__ uint32_t tmp[kPartWarps + 1];
    __shared__ uint32_t wtot[kPartWarps];
    __shared__ uint32_t s_item;
    __shared__ uint64_t s_base;

    for (uint32_t i = lane; i < kOwnDense; i += 32) vbits[i] = kNoValue;
    bool dense_layout = true;
    __syncwarp();

    for (;;) {
        __syncthreads();
        if (t == 0) s_item = atomicAdd(work_counter, 1u);
        __syncthreads();
        const uint32_t item = s_item;
        if (item >= nparts) break;
        const PartItem it = parts[item];
        const bool dense = (it.mode & 1u) != 0;
        if (dense != dense_layout) {  // values are all empty after an emission; only keys differ
            if (dense) {
                for (uint32_t i = kOwnSlots + lane; i < kOwnDense; i += 32) vbits[i] = kNoValue;
            } else {
                for (uint32_t i = lane; i < kOwnSlots; i += 32) keys[i] = kEmptyCol;
            }
            dense_layout = dense;
            __syncwarp();
        }
        const uint32_t row = it.row;
        const uint32_t lo = it.p0 << op.panel_log2;  // first column of the part
        const uint32_t ka = op.row_start[row], kb = op.row_start[row + 1];
        bool bad = false;  // table overflow or a column outside a dense part (never for exact sizes)

        for (uint32_t kw = ka; kw < kb; kw += kPartWindow) {
            const uint32_t k = kw + t;
            uint32_t L = 0, s = 0;
            double a = 0.0;
            if (t < kPartWindow && k < kb) {
                const int32_t f = op.a_fib[k];
                if (f >= 0) {
                    uint32_t e;
                    part_range(op, f, it.p0, it.p1, s, e);
                    L = e - s;
                    a = op.a_val[k];
                }
            }
            uint32_t total;
            const uint32_t excl = block_exclusive_scan<uint32_t, kPartThreads>(L, tmp, &total);
            if (t < kPartWindow) {
                ws[t] = s;
                wscan[t] = excl;
                wa[t] = a;
            }
            __syncthreads();
            // Rounds of kRound products in stream order: product pos + i * 512 + t is thread t's
            // item i.  A round's fiber entries are loaded during the round before, so their loads
            // are in flight while that round's buckets are applied.
            uint32_t kk = 0;  // the window's A nonzero holding this thread's latest product
            uint32_t ncol[kRoundItems], nsrc[kRoundItems];
            double nb[kRoundItems];
            auto load_round = [&](uint32_t pos) {
#pragma unroll
                for (int i = 0; i < kRoundItems; ++i) {
                    const uint32_t q = pos + i * kPartThreads + t;
                    ncol[i] = kEmptyCol;
                    nsrc[i] = 0;
                    nb[i] = 0.0;
                    if (q < total) {
                        kk = find_nonzero(wscan, kk, q);
                        const uint32_t j = ws[kk] + (q - wscan[kk]);
                        ncol[i] = __ldg(op.b_col + j);
                        nb[i] = __ldg(op.b_val + j);
                        nsrc[i] = kk;
                    }
                }
            };
            load_round(0);
            for (uint32_t pos = 0; pos < total; pos += kRound) {
                uint32_t col[kRoundItems], owner[kRoundItems], rank[kRoundItems];
                double prod[kRoundItems];
                if (lane < kRoundItems * 4) cnt4[lane >> 2][warp][lane & 3] = 0u;
                __syncwarp();
#pragma unroll
                for (int i = 0; i < kRoundItems; ++i) {
                    col[i] = ncol[i];
                    owner[i] = kPartWarps;
                    prod[i] = 0.0;
                    if (col[i] != kEmptyCol) {
                        uint32_t hint;
                        prod[i] = __dmul_rn(wa[nsrc[i]], nb[i]);
                        if (dense && col[i] - lo >= kDenseCols) bad = true;
                        else owner[i] = part_owner(col[i], lo, dense, hint);
                    }
                    // stable split by owner: a product's rank among its warp's item-i products of
                    // its owner, and per (item, warp, owner) counts (one byte each)
                    const uint32_t same = __match_any_sync(kFullMask, owner[i]);
                    rank[i] = __popc(same & lanemask_lt());
                    if (owner[i] < kPartWarps && rank[i] == 0)
                        reinterpret_cast<uint8_t*>(&cnt4[i][warp][0])[owner[i]] = (uint8_t)__popc(same);
                }
                __syncthreads();
                // warp o: owner o's bucket starts after the buckets of owners < o; inside it the
                // products follow in (item, warp) order: lane l of the scan is item l / 16, warp l % 16
                uint32_t bstart, bcount;
                {
                    const uint32_t o = warp;
                    const uint4 c = *reinterpret_cast<const uint4*>(&cnt4[lane >> 4][lane & 15][0]);
                    const uint32_t w4[4] = {c.x, c.y, c.z, c.w};
                    uint32_t before = 0;
#pragma unroll
                    for (uint32_t k = 0; k < 4; ++k) {  // bytes of owners < o
                        const uint32_t nbytes = o > 4 * k ? min(o - 4 * k, 4u) : 0u;
                        const uint32_t mask = nbytes >= 4 ? 0xffffffffu : (1u << (8 * nbytes)) - 1u;
                        before = __dp4a(w4[k] & mask, 0x01010101u, before);
                    }
                    before = warp_sum(before);
                    const uint32_t wo = o < 4 ? c.x : o < 8 ? c.y : o < 12 ? c.z : c.w;
                    const uint32_t mine = (wo >> (8 * (o & 3))) & 0xffu;
                    const uint32_t incl = warp_inclusive_scan(mine);
                    off[lane >> 4][lane & 15][o] = (uint16_t)(before + incl - mine);
                    bstart = before;
                    bcount = __shfl_sync(kFullMask, incl, 31);
                }
                __syncthreads();
#pragma unroll
                for (int i = 0; i < kRoundItems; ++i) {
                    if (owner[i] < kPartWarps) {
                        const uint32_t d = off[i][warp][owner[i]] + rank[i];
                        bcol[d] = col[i];
                        bval[d] = prod[i];
                    }
                }
                if (pos + kRound < total) load_round(pos + kRound);
                __syncthreads();
                // this warp's bucket, in stream order, 32 products at a time; products meeting in
                // one column apply by rank
                for (uint32_t c0 = 0; c0 < bcount; c0 += 32) {
                    const bool valid = c0 + lane < bcount;
                    uint32_t cl = kEmptyCol;
                    double p = 0.0;
                    uint32_t h = 0;
                    if (valid) {
                        cl = bcol[bstart + c0 + lane];
                        p = bval[bstart + c0 + lane];
                        part_owner(cl, lo, dense, h);
                    }
                    const uint32_t mm = __match_any_sync(kFullMask, cl);
                    const uint32_t r = __popc(mm & lanemask_lt());
                    int slot = -1;
                    if (valid && r == 0) {
                        slot = dense ? (int)h : own_slot(keys, cl, h);
                        if (slot < 0) bad = true;
                    }
                    slot = __shfl_sync(kFullMask, slot, __ffs(mm) - 1);
                    const uint32_t maxr = __reduce_max_sync(kFullMask, valid ? r : 0u);
                    for (uint32_t rr = 0; rr <= maxr; ++rr) {
                        if (valid && r == rr && slot >= 0) accumulate(&vals[slot], p);
                        __syncwarp();
                    }
                }
            }
            __syncthreads();  // the window's arrays are read again next window
        }
        const bool any_bad = __syncthreads_or(bad);

        // emit: warp w writes its table's entries after those of warps < w (a dense part's column
        // of local slot l is lo + 16 l + w)
        const uint32_t tsize = dense ? kOwnDense : kOwnSlots;
        uint32_t n = 0;
        for (uint32_t i = 0; i < tsize; i += 32) n += __popc(__ballot_sync(kFullMask, vbits[i + lane] != kNoValue));
        if (lane == 0) wtot[warp] = n;
        __syncthreads();
        if (t == 0) {
            uint64_t base = it.out_off, total = 0;
            for (uint32_t w = 0; w < kPartWarps; ++w) total += wtot[w];
            if (base == kClaimBit) {
                base = any_bad ? ~0ull : claim_output(op, out, row, total);
                if (base == ~0ull) {  // rerun this part exactly
                    const uint32_t f = atomicAdd(out.fail_count, 1u);
                    out.fail_list[f] = item;
                }
            } else if (any_bad) {
                atomicOr(overflow, 1u);  // exact sizes cannot overflow: report an internal error
                base = ~0ull;
            }
            if (out.item_count) out.item_count[item] = base == ~0ull ? 0u : (uint32_t)total;
            s_base = base;
        }
        __syncthreads();
        const uint64_t base = s_base;
        uint64_t o = base;
        for (uint32_t w = 0; w < warp; ++w) o += wtot[w];
        for (uint32_t i = 0; i < tsize; i += 32) {
            const uint32_t sidx = i + lane;
            const double v = vals[sidx];
            const bool occ = __double_as_longlong(v) != (long long)kNoValue;
            const uint32_t m = __ballot_sync(kFullMask, occ);
            if (occ) {
                if (base != ~0ull) {
                    const uint32_t c = dense ? lo + (sidx << 4) + warp : keys[sidx];
                    write_entry(op, out, o + __popc(m & lanemask_lt()), row, c, v);
                }
                vbits[sidx] = kNoValue;
                if (!dense) keys[sidx] = kEmptyCol;
            }
            o += __popc(m);
        }
    }
}

void launch_hash_parts(const Operands& op, const PartItem* parts, uint32_t nparts, const OutputView& out,
                       uint32_t* work_counter, uint32_t* overflow, int num_sms, cudaStream_t st) {
    if (nparts == 0) return;
    const size_t smem = kPartSmemBytes;
    PTC_CUDA(cudaMemsetAsync(work_counter, 0, sizeof(uint32_t), st));
    PTC_CUDA(cudaFuncSetAttribute(hash_part_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    PTC_CUDA(cudaFuncSetAttribute(hash_part_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    int per_sm = 1;
    PTC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hash_part_kernel, kPartThreads, smem));
    per_sm = per_sm < 1 ? 1 : per_sm;
    const uint32_t grid = (uint32_t)std::min<uint64_t>(nparts, (uint64_t)num_sms * per_sm);
    hash_part_kernel<<<grid, kPartThreads, smem, st>>>(op, parts, nparts, out, work_counter, overflow);
    count_launch();
    PTC_CHECK_LAUNCH();
}

}  // namespace ptc
