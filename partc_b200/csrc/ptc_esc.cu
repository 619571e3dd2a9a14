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

// One block per long run (runs at least kEscLongMin products long: an output entry that many
// products meet, e.g. a popular column of a skewed tensor).  The left fold is a chain of
// dependent additions, so one thread does it -- from shared memory, while warps 1..7 stream the
// next stage of the run into the other buffer with coalesced loads.
constexpr int kLongThreads = 256;
constexpr uint32_t kLongStage = 2048;  // products per stage (16 KiB)

__global__ void __launch_bounds__(kLongThreads)
    esc_fold_long_kernel(Operands op, OutputView out, const uint64_t* __restrict__ run_key,
                         const uint32_t* __restrict__ run_start, const uint32_t* __restrict__ long_runs, uint32_t colbits,
                         const uint32_t* __restrict__ esc_rows, const uint32_t* __restrict__ first_run,
                         const uint64_t* __restrict__ row_off, const double* __restrict__ sorted) {
    __shared__ double buf[2][kLongStage];
    const uint32_t t = threadIdx.x;
    const uint32_t r = long_runs[blockIdx.x];
    const uint32_t b = run_start[r], n = run_start[r + 1] - b;
    const uint32_t nst = (n + kLongStage - 1) / kLongStage;
    for (uint32_t i = t; i < min(n, kLongStage); i += kLongThreads) buf[0][i] = sorted[b + i];
    __syncthreads();
    double v = 0.0;
    for (uint32_t s = 0; s < nst; ++s) {
        const uint32_t len = min(kLongStage, n - s * kLongStage);
        if (t >= 32) {  // warps 1..7 load stage s + 1
            if (s + 1 < nst) {
                const uint32_t base = (s + 1) * kLongStage, l2 = min(kLongStage, n - base);
                double* dst = buf[(s + 1) & 1];
                for (uint32_t i = t - 32; i < l2; i += kLongThreads - 32) dst[i] = sorted[b + base + i];
            }
        } else if (t == 0) {  // the fold, in stream order
            const double* src = buf[s & 1];
            uint32_t i = 0;
            if (s == 0) {
                v = src[0];
                i = 1;
            }
#pragma unroll 8
            for (; i < len; ++i) v = __dadd_rn(v, src[i]);
        }
        __syncthreads();
    }
    if (t == 0) {
        const uint64_t key = run_key[r];
        const uint32_t e = (uint32_t)(key >> colbits);
        const uint32_t row = esc_rows[e];
        write_entry(op, out, row_off[row] + (r - first_run[e]), row, (uint32_t)(key & ((1ull << colbits) - 1)), v);
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
        esc_fold_long_kernel<<<n_long, kLongThreads, 0, st>>>(op, out, run_key, run_start, long_runs, colbits,
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
