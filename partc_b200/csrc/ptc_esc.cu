// Sort-based accumulator ("expand, sort, compress") for rows made of many short fibers.
//
// A row whose A nonzeros each meet only a few B entries (average products per A nonzero below a
// threshold) gives the block hash accumulator little to do per step and many ordering rounds.
// For those rows every product is written out in stream order, the (row, column) keys are
// sorted stably, and each run of equal keys is folded left to right -- exactly the reference's
// summation order (fksCuckooTC.hpp:294-337), since a stable sort keeps the stream order inside a
// run.  Each row's entries come out in increasing column order.
#include "ptc_spa.cuh"

namespace ptc {

// One thread per A nonzero (row-sorted numbering): products of nonzeros of sort-based rows go
// to key/val/perm at the row's base plus the nonzero's stream offset inside the row.
__global__ void esc_expand_kernel(Operands op, const uint32_t* __restrict__ a_row, const int32_t* __restrict__ esc_of,
                                  const uint64_t* __restrict__ poff, const uint64_t* __restrict__ esc_off,
                                  uint32_t colbits, uint64_t* __restrict__ key, double* __restrict__ val,
                                  uint32_t* __restrict__ perm) {
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= op.na) return;
    const uint32_t row = a_row[k];
    const int32_t e = esc_of[row];
    if (e < 0) return;
    const int32_t f = op.a_fib[k];
    if (f < 0) return;
    const uint32_t s = op.fib_start[f], L = op.fib_start[f + 1] - s;
    const uint64_t base = esc_off[e] + (poff[k] - poff[op.row_start[row]]);
    const double a = op.a_val[k];
    const uint64_t hi = (uint64_t)e << colbits;
    for (uint32_t i = 0; i < L; ++i) {
        key[base + i] = hi | op.b_col[s + i];
        val[base + i] = __dmul_rn(a, op.b_val[s + i]);
        perm[base + i] = (uint32_t)(base + i);
    }
}

void launch_esc_expand(const Operands& op, const uint32_t* a_row, const int32_t* esc_of, const uint64_t* poff,
                       const uint64_t* esc_off, uint32_t colbits, uint64_t* key, double* val, uint32_t* perm,
                       cudaStream_t st) {
    if (op.na == 0) return;
    esc_expand_kernel<<<ceil_div_u32(op.na, 256), 256, 0, st>>>(op, a_row, esc_of, poff, esc_off, colbits, key, val, perm);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// One thread per run of equal (row, column) keys: count the row's entries and remember the
// row's first run.
__global__ void esc_count_kernel(const uint64_t* __restrict__ run_key, uint64_t nruns, uint32_t colbits,
                                 const uint32_t* __restrict__ esc_rows, uint64_t* __restrict__ row_d,
                                 uint32_t* __restrict__ first_run) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nruns) return;
    const uint32_t e = (uint32_t)(run_key[r] >> colbits);
    atomicAdd(reinterpret_cast<unsigned long long*>(&row_d[esc_rows[e]]), 1ull);
    if (r == 0 || (uint32_t)(run_key[r - 1] >> colbits) != e) first_run[e] = (uint32_t)r;
}

void launch_esc_count(const uint64_t* run_key, uint64_t nruns, uint32_t colbits, const uint32_t* esc_rows,
                      uint64_t* row_d, uint32_t* first_run, cudaStream_t st) {
    if (nruns == 0) return;
    esc_count_kernel<<<ceil_div_u32(nruns, 256), 256, 0, st>>>(run_key, nruns, colbits, esc_rows, row_d, first_run);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// sorted[i] = val[perm[i]]: the products in (row, column, stream) order, so each run is
// contiguous for the fold below.
__global__ void esc_gather_kernel(const double* __restrict__ val, const uint32_t* __restrict__ perm, uint64_t n,
                                  double* __restrict__ sorted) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) sorted[i] = val[perm[i]];
}

// One thread per run of [r0, r1): left fold of the run's products in stream order, written at the row's
// output offset plus the run's rank inside the row.  Loads are issued eight at a time ahead of
// the dependent additions.
__global__ void esc_fold_kernel(Operands op, OutputView out, const uint64_t* __restrict__ run_key,
                                const uint32_t* __restrict__ run_start, uint64_t r0, uint64_t r1, uint32_t colbits,
                                const uint32_t* __restrict__ esc_rows, const uint32_t* __restrict__ first_run,
                                const uint64_t* __restrict__ row_off, const double* __restrict__ sorted,
                                uint32_t long_min) {
    const uint64_t r = r0 + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= r1) return;
    const uint32_t b = run_start[r], en = run_start[r + 1];
    if (en - b >= long_min) return;  // a long run: esc_fold_long_kernel folds it
    const uint64_t key = run_key[r];
    const uint32_t e = (uint32_t)(key >> colbits);
    const uint32_t row = esc_rows[e];
    const uint32_t col = (uint32_t)(key & ((1ull << colbits) - 1));
    double v = sorted[b];
    uint32_t i = b + 1;
    constexpr uint32_t U = 16;
    if (en - i >= U) {
        // software pipeline: the next U values load while the current U are added
        double cur[U];
#pragma unroll
        for (uint32_t u = 0; u < U; ++u) cur[u] = sorted[i + u];
        i += U;
        while (en - i >= U) {
            double nxt[U];
#pragma unroll
            for (uint32_t u = 0; u < U; ++u) nxt[u] = sorted[i + u];
#pragma unroll
            for (uint32_t u = 0; u < U; ++u) v = __dadd_rn(v, cur[u]);
#pragma unroll
            for (uint32_t u = 0; u < U; ++u) cur[u] = nxt[u];
            i += U;
        }
#pragma unroll
        for (uint32_t u = 0; u < U; ++u) v = __dadd_rn(v, cur[u]);
    }
    for (; i < en; ++i) v = __dadd_rn(v, sorted[i]);
    write_entry(op, out, row_off[row] + (r - first_run[e]), row, col, v);
}

// One block per long run (runs of at least kEscLongMin products: an output entry that many
// products meet, e.g. a popular column of a skewed tensor), folded exactly as the left fold but
// mostly in parallel.  While the running value v stays inside one binade [2^E, 2^(E+1)) (either
// sign), every double there is an integer multiple of u = 2^(E-52), so the IEEE sum
// fl(v + x) = v + u * rint(x / u) whenever x / u is not halfway between integers and the exact
// sum stays strictly inside the binade (at least one step from either end): then the rounded sum
// is the nearest multiple of u and no tie is broken.  So a tile of 8192 products becomes integer
// increments k = rint(x / u) (in parallel), a block-wide prefix of them, and the running value
// (v / u) + prefix is exact up to the first product that breaks a condition -- a tie, a value
// too large, or a prefix that reaches the binade's ends; that one is added for real
// (__dadd_rn) and the scan resumes after it with the new binade.  A tile that stops more than
// kGridMaxStops times (a sum hovering near zero crosses binades all the time), or a running value
// that is zero, subnormal or not finite, is folded by one thread, product after product.  The
// result is the sequential left fold to the bit.
constexpr int kGridThreads = 1024;
constexpr int kGridPer = 8;                             // products per thread per pass
constexpr uint32_t kGridTile = kGridThreads * kGridPer; // 8192 products (64 KiB of shared memory)
constexpr int kGridMaxStops = 8;

__global__ void __launch_bounds__(kGridThreads)
    esc_fold_long_kernel(Operands op, OutputView out, const uint64_t* __restrict__ run_key,
                         const uint32_t* __restrict__ run_start, const uint32_t* __restrict__ long_runs, uint32_t colbits,
                         const uint32_t* __restrict__ esc_rows, const uint32_t* __restrict__ first_run,
                         const uint64_t* __restrict__ row_off, const double* __restrict__ sorted) {
    extern __shared__ double tile[];  // [kGridTile]
    __shared__ unsigned long long scan_tmp[kGridThreads / 32 + 1];
    __shared__ uint32_t s_first;
    __shared__ double s_v;
    const uint32_t t = threadIdx.x;
    const uint32_t r = long_runs[blockIdx.x];
    const uint32_t b = run_start[r], n = run_start[r + 1] - b;
    if (t == 0) s_v = sorted[b];  // the first product of the entry is its value so far
    for (uint32_t t0 = 1; t0 < n; t0 += kGridTile) {
        const uint32_t len = min(kGridTile, n - t0);
        __syncthreads();  // the previous tile is done with `tile`
        for (uint32_t e = t; e < len; e += kGridThreads) tile[e] = sorted[b + t0 + e];
        __syncthreads();
        uint32_t st = 0;  // products of the tile already in s_v
        for (int stops = 0; st < len; ++stops) {
            const double v = s_v;
            const double av = fabs(v);
            if (stops > kGridMaxStops || !(av >= 2.2250738585072014e-308) || av == INFINITY || v != v) {
                if (t == 0) {  // one thread, product after product
                    double w = v;
                    for (uint32_t e = st; e < len; ++e) w = __dadd_rn(w, tile[e]);
                    s_v = w;
                }
                __syncthreads();
                break;
            }
            int E;
            frexp(av, &E);
            --E;                                                  // v in [2^E, 2^(E+1))
            const double u = ldexp(1.0, E - 52);
            const long long N = (long long)(v / u);               // exact: |N| in [2^52, 2^53)
            const long long lo = (1ll << 52), hi = (1ll << 53) - 1;
            // this thread's products st + t * kGridPer + q, q < kGridPer
            const uint32_t e0 = st + t * kGridPer;
            unsigned long long k[kGridPer];
            bool bad[kGridPer];
            unsigned long long mine = 0;
#pragma unroll
            for (int q = 0; q < kGridPer; ++q) {
                const uint32_t e = e0 + q;
                k[q] = 0;
                bad[q] = false;
                if (e < len) {
                    const double x = scalbn(tile[e], 52 - E);     // exact scaling by a power of two
                    const double ax = fabs(x);
                    if (!(ax < 9007199254740992.0) || fabs(x - trunc(x)) == 0.5) {
                        bad[q] = true;                            // too large, not finite, or a tie
                    } else {
                        k[q] = (unsigned long long)llrint(x);
                    }
                    mine += k[q];
                }
            }
            unsigned long long total;
            const unsigned long long before = block_exclusive_scan<unsigned long long, kGridThreads>(mine, scan_tmp, &total);
            // first product whose step is not on the grid
            uint32_t first = 0xffffffffu;
            unsigned long long run = (unsigned long long)N + before;
#pragma unroll
            for (int q = 0; q < kGridPer; ++q) {
                const uint32_t e = e0 + q;
                if (e < len && first == 0xffffffffu) {
                    run += k[q];
                    const long long m = (long long)run * (N > 0 ? 1 : -1);
                    if (bad[q] || !(m > lo && m < hi)) first = e;
                }
            }
            if (t == 0) s_first = 0xffffffffu;
            __syncthreads();
            if (first != 0xffffffffu) atomicMin(&s_first, first);
            __syncthreads();
            const uint32_t f = s_first;
            if (f == 0xffffffffu) {  // the whole rest of the tile is on the grid
                if (t == 0) s_v = (double)(long long)((unsigned long long)N + total) * u;
                __syncthreads();
                break;
            }
            if (first == f) {  // this thread owns product f: the value before it, then f for real
                unsigned long long p = (unsigned long long)N + before;
                for (uint32_t e = e0; e < f; ++e) p += k[e - e0];
                const double prev = f > st ? (double)(long long)p * u : v;
                s_v = __dadd_rn(prev, tile[f]);
            }
            __syncthreads();
            st = f + 1;
        }
    }
    __syncthreads();
    if (t == 0) {
        const uint64_t key = run_key[r];
        const uint32_t e = (uint32_t)(key >> colbits);
        const uint32_t row = esc_rows[e];
        write_entry(op, out, row_off[row] + (r - first_run[e]), row, (uint32_t)(key & ((1ull << colbits) - 1)), s_v);
    }
}

// flag[r] = 1 if run r has at least kEscLongMin products
__global__ void esc_long_flags_kernel(const uint32_t* __restrict__ run_start, uint64_t nruns, uint32_t* __restrict__ flag) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nruns) flag[r] = (run_start[r + 1] - run_start[r] >= kEscLongMin) ? 1u : 0u;
}

void launch_esc_long_flags(const uint32_t* run_start, uint64_t nruns, uint32_t* flag, cudaStream_t st) {
    if (nruns == 0) return;
    esc_long_flags_kernel<<<ceil_div_u32(nruns, 256), 256, 0, st>>>(run_start, nruns, flag);
    count_launch();
    PTC_CHECK_LAUNCH();
}

void launch_esc_gather(const uint32_t* perm, const double* val, uint64_t nprod, double* sorted, cudaStream_t st) {
    if (nprod == 0) return;
    esc_gather_kernel<<<ceil_div_u32(nprod, 256), 256, 0, st>>>(val, perm, nprod, sorted);
    count_launch();
    PTC_CHECK_LAUNCH();
}

void launch_esc_fold(const Operands& op, const OutputView& out, const uint64_t* run_key, const uint32_t* run_start,
                     uint64_t r0, uint64_t r1, uint32_t colbits, const uint32_t* esc_rows, const uint32_t* first_run,
                     const uint64_t* row_off, const double* sorted, const uint32_t* long_runs, uint32_t n_long,
                     cudaStream_t st) {
    if (r1 <= r0) return;
    if (n_long > 0) {  // the long runs first: each is a long chain, so they start as early as possible
        const size_t smem = kGridTile * sizeof(double);
        PTC_CUDA(cudaFuncSetAttribute(esc_fold_long_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        esc_fold_long_kernel<<<n_long, kGridThreads, smem, st>>>(op, out, run_key, run_start, long_runs, colbits,
                                                                 esc_rows, first_run, row_off, sorted);
        count_launch();
        PTC_CHECK_LAUNCH();
    }
    esc_fold_kernel<<<ceil_div_u32(r1 - r0, 128), 128, 0, st>>>(op, out, run_key, run_start, r0, r1, colbits,
                                                                esc_rows, first_run, row_off, sorted,
                                                                kEscLongMin);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// esc_of[r] = index of row r among the sort-based rows, or -1.
__global__ void esc_index_kernel(const uint32_t* __restrict__ esc_rows, uint64_t n, int32_t* __restrict__ esc_of) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) esc_of[esc_rows[i]] = (int32_t)i;
}

void launch_esc_index(const uint32_t* esc_rows, uint64_t n, int32_t* esc_of, cudaStream_t st) {
    if (n == 0) return;
    esc_index_kernel<<<ceil_div_u32(n, 256), 256, 0, st>>>(esc_rows, n, esc_of);
    count_launch();
    PTC_CHECK_LAUNCH();
}

// esc_len[i] = products of sort-based row esc_rows[i]
__global__ void esc_len_kernel(const uint32_t* __restrict__ esc_rows, uint64_t n, const uint64_t* __restrict__ row_flops,
                               uint64_t* __restrict__ len) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) len[i] = row_flops[esc_rows[i]];
}

void launch_esc_len(const uint32_t* esc_rows, uint64_t n, const uint64_t* row_flops, uint64_t* len, cudaStream_t st) {
    if (n == 0) return;
    esc_len_kernel<<<ceil_div_u32(n, 256), 256, 0, st>>>(esc_rows, n, row_flops, len);
    count_launch();
    PTC_CHECK_LAUNCH();
}

}  // namespace ptc
