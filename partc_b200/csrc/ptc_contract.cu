// Host orchestration and the C ABI (include/partc.h).
//
// One call replaces main.cpp:112-118 of the reference: B = A (self-contraction) or a second
// tensor, the FKS/cuckoo table on B's contracted modes (buildHashTable(B), fksCuckoo.hpp:1044),
// the row grouping of A (buildHashTable(A_copy)), reorder_tensor (fksCuckooTC.hpp:31-77), the
// symbolic pass (:94-154) and the numeric pass (:180-357).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "partc.h"
#include "ptc_build.cuh"
#include "ptc_internal.cuh"
#include "ptc_prims.cuh"
#include "ptc_spa.cuh"

namespace ptc {

thread_local uint64_t g_launches = 0;
static thread_local std::string g_last_error;
static thread_local char g_last_error_buf[512];

void set_last_error(ptc_status, const std::string& msg) { g_last_error = msg; }

namespace {

KeySpec make_keyspec(const uint32_t* dims, const uint32_t* modes, uint32_t n) {
    KeySpec k;
    k.n = n;
    unsigned __int128 space = 1;
    for (int j = (int)n - 1; j >= 0; --j) {
        k.mode[j] = modes[j];
        k.stride[j] = (uint64_t)space;
        space *= (unsigned __int128)(dims[modes[j]] ? dims[modes[j]] : 1);
        PTC_REQUIRE(space <= (unsigned __int128)UINT64_MAX, PTC_ERR_KEY_OVERFLOW,
                    "the product of the key mode sizes does not fit in 64 bits");
    }
    k.space = (uint64_t)space;
    return k;
}

void validate_coo(const ptc_coo* t, const char* name) {
    PTC_REQUIRE(t != nullptr, PTC_ERR_INVALID_ARGUMENT, std::string(name) + " is null");
    PTC_REQUIRE(t->order >= 1 && t->order <= (uint32_t)kMaxOrder, PTC_ERR_INVALID_ARGUMENT,
                std::string(name) + ": order must be in [1, 16]");
    PTC_REQUIRE(t->dims != nullptr, PTC_ERR_INVALID_ARGUMENT, std::string(name) + ": dims is null");
    PTC_REQUIRE(t->nnz == 0 || (t->idx != nullptr && t->vals != nullptr), PTC_ERR_INVALID_ARGUMENT,
                std::string(name) + ": idx/vals is null");
    PTC_REQUIRE(t->nnz < (1ull << 31), PTC_ERR_INVALID_ARGUMENT, std::string(name) + ": nnz must be < 2^31");
    PTC_REQUIRE(t->location == PTC_HOST || t->location == PTC_DEVICE, PTC_ERR_INVALID_ARGUMENT,
                std::string(name) + ": bad location");
    for (uint32_t m = 0; m < t->order; ++m)
        PTC_REQUIRE(t->dims[m] >= 1, PTC_ERR_INVALID_ARGUMENT, std::string(name) + ": a mode size is 0");
}

void validate_modes(const uint32_t* modes, uint32_t order, const char* name) {
    PTC_REQUIRE(modes != nullptr, PTC_ERR_INVALID_ARGUMENT, std::string(name) + " is null");
    uint32_t seen = 0;
    for (uint32_t j = 0; j < order; ++j) {
        PTC_REQUIRE(modes[j] < order, PTC_ERR_INVALID_ARGUMENT, std::string(name) + ": mode out of range");
        PTC_REQUIRE(!(seen & (1u << modes[j])), PTC_ERR_INVALID_ARGUMENT, std::string(name) + ": repeated mode");
        seen |= 1u << modes[j];
    }
}

struct Events {
    static constexpr int kN = 8;
    cudaEvent_t ev[kN] = {};
    explicit Events() {
        for (auto& e : ev) PTC_CUDA(cudaEventCreate(&e));
    }
    ~Events() {
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
    }
    float ms(int a, int b) const {
        float x = 0.f;
        cudaEventElapsedTime(&x, ev[a], ev[b]);
        return x;
    }
};

enum { EV_START = 0, EV_H2D, EV_BSIDE, EV_ASIDE, EV_SYM, EV_NUM, EV_D2H };

cudaStream_t default_stream_for_thread(int device) {
    thread_local int dev = -1;
    thread_local cudaStream_t st = nullptr;
    if (st == nullptr || dev != device) {
        PTC_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        dev = device;
    }
    return st;
}

// Keep freed stream-ordered allocations in the device's pool (instead of returning them to the
// driver at every synchronization), so repeated calls do not remap their buffers.
void keep_pool_memory(int device) {
    static std::mutex mu;
    static uint64_t done = 0;  // bit per device
    std::lock_guard<std::mutex> lock(mu);
    if (device < 64 && (done >> device) & 1ull) return;
    cudaMemPool_t pool;
    PTC_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t threshold = UINT64_MAX;
    PTC_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
    if (device < 64) done |= 1ull << device;
}

int device_sm_count(int device) {
    int n = 0;
    PTC_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device));
    return n;
}

uint32_t floor_log2(uint64_t x) {
    uint32_t r = 0;
    while ((2ull << r) <= x) ++r;
    return r;
}

template <typename T>
T read_scalar(const T* dptr, cudaStream_t st) {
    T v{};
    PTC_CUDA(cudaMemcpyAsync(&v, dptr, sizeof(T), cudaMemcpyDeviceToHost, st));
    PTC_CUDA(cudaStreamSynchronize(st));
    return v;
}

// Stable ranks of a key array: sorted order `perm` (input order kept among equal keys), the
// rank of every element in original numbering, run starts in sorted order and run count.
struct Ranked {
    uint32_t* perm = nullptr;       // [n] original index of the i-th smallest
    uint32_t* rank_of = nullptr;    // [n] rank of original element i
    uint32_t* run_start = nullptr;  // [nruns + 1] in sorted order
    uint64_t nruns = 0;
};

Ranked rank_keys(const uint64_t* keys, uint64_t n, uint64_t space, Arena& ar) {
    cudaStream_t st = ar.stream();
    Ranked r;
    r.perm = ar.alloc<uint32_t>(n);
    uint64_t* k = ar.alloc<uint64_t>(n);
    PTC_CUDA(cudaMemcpyAsync(k, keys, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st));
    launch_iota(r.perm, n, st);
    radix_sort_pairs(k, r.perm, n, 0, bits_for_space(space), ar);
    uint32_t* run_of_sorted = ar.alloc<uint32_t>(n);
    r.run_start = ar.alloc<uint32_t>(n + 1);
    r.nruns = runs_of_sorted(k, n, run_of_sorted, r.run_start, nullptr, ar);
    r.rank_of = ar.alloc<uint32_t>(n);
    launch_scatter_u32(run_of_sorted, r.perm, n, r.rank_of, st);
    return r;
}

struct DeviceCoo {
    const uint32_t* idx = nullptr;
    const double* vals = nullptr;
    uint64_t nnz = 0;
    uint32_t order = 0;
    DimSpec dims;
};

DeviceCoo to_device(const ptc_coo* t, Arena& ar) {
    DeviceCoo d;
    d.nnz = t->nnz;
    d.order = t->order;
    d.dims.order = t->order;
    for (uint32_t m = 0; m < t->order; ++m) d.dims.dim[m] = t->dims[m];
    if (t->location == PTC_DEVICE || t->nnz == 0) {
        d.idx = t->idx;
        d.vals = t->vals;
    } else {
        uint32_t* di = ar.alloc<uint32_t>(t->nnz * t->order);
        double* dv = ar.alloc<double>(t->nnz);
        PTC_CUDA(cudaMemcpyAsync(di, t->idx, t->nnz * t->order * sizeof(uint32_t), cudaMemcpyHostToDevice, ar.stream()));
        PTC_CUDA(cudaMemcpyAsync(dv, t->vals, t->nnz * sizeof(double), cudaMemcpyHostToDevice, ar.stream()));
        d.idx = di;
        d.vals = dv;
    }
    return d;
}

void print_reference_lines(const ptc_stats& s) {
    // the reference's stdout lines (fksCuckoo.hpp:1056-1057, fksCuckooTC.hpp:161,364-365)
    printf("Number of elements inserted = %llu\n", (unsigned long long)s.b_nnz);
    printf("Total time for insertion = %g (s)\n", s.t_build_ms * 1e-3);
    printf("Number of elements inserted = %llu\n", (unsigned long long)s.a_nnz);
    printf("Total time for insertion = %g (s)\n", 0.0);
    printf("Total time for preprocessing = %g (s)\n", s.t_symbolic_ms * 1e-3);
    printf("Total time for tensor contraction = %g (s)\n", s.t_numeric_ms * 1e-3);
    printf("Total number of nonzeros in the output tensor = %llu\n", (unsigned long long)s.out_nnz);
    fflush(stdout);
}

void contract_impl(const ptc_coo* A, const ptc_coo* Bin, uint32_t c, const uint32_t* a_modes,
                   const uint32_t* b_modes_in, const ptc_options* opt_in, ptc_tensor* out, ptc_stats* stats_out) {
    ptc_options opt;
    ptc_options_init(&opt);
    if (opt_in) {
        PTC_REQUIRE(opt_in->struct_size >= offsetof(ptc_options, reserved), PTC_ERR_INVALID_ARGUMENT,
                    "ptc_options.struct_size too small (call ptc_options_init)");
        std::memcpy(&opt, opt_in, std::min<size_t>(opt_in->struct_size, sizeof(opt)));
    }
    PTC_REQUIRE(out != nullptr, PTC_ERR_INVALID_ARGUMENT, "out is null");
    std::memset(out, 0, sizeof(*out));
    ptc_stats stats;
    std::memset(&stats, 0, sizeof(stats));
    g_launches = 0;

    const bool self = (Bin == nullptr);
    const ptc_coo* B = self ? A : Bin;
    const uint32_t* b_modes = self ? a_modes : b_modes_in;
    validate_coo(A, "A");
    validate_coo(B, "B");
    PTC_REQUIRE(c >= 1 && c <= A->order && c <= B->order, PTC_ERR_INVALID_ARGUMENT,
                "need 1 <= c <= order of each tensor");
    validate_modes(a_modes, A->order, "a_modes");
    validate_modes(b_modes, B->order, "b_modes");
    for (uint32_t j = 0; j < c; ++j)
        PTC_REQUIRE(A->dims[a_modes[j]] == B->dims[b_modes[j]], PTC_ERR_INVALID_ARGUMENT,
                    "paired contracted modes have different sizes");
    const uint32_t fa = A->order - c, fb = B->order - c;
    PTC_REQUIRE(fa + fb >= 1, PTC_ERR_EMPTY_CONTRACTION, "tensor contraction not possible (no free modes)");
    if (self) PTC_REQUIRE(A->nnz > 1, PTC_ERR_TOO_FEW_NONZEROS, "Tensor B has at most one nonzeros");
    PTC_REQUIRE(opt.output_location == PTC_HOST || opt.output_location == PTC_DEVICE, PTC_ERR_INVALID_ARGUMENT,
                "bad output_location");
    PTC_REQUIRE(opt.panel_width == 0 || (opt.panel_width >= 256 && opt.panel_width <= 4096 &&
                                         (opt.panel_width & (opt.panel_width - 1)) == 0),
                PTC_ERR_INVALID_ARGUMENT, "panel_width must be 0 or a power of two in [256, 4096]");

    // device
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        throw Error{PTC_ERR_NO_DEVICE, "no usable CUDA device"};
    }
    int device = opt.device;
    if (device < 0) PTC_CUDA(cudaGetDevice(&device));
    PTC_REQUIRE(device < ndev, PTC_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    PTC_CUDA(cudaSetDevice(device));
    int major = 0;
    PTC_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
    if (major != 10) throw Error{PTC_ERR_NO_DEVICE, "this library is built for sm_100a (B200) only"};
    keep_pool_memory(device);
    cudaStream_t st = opt.stream ? static_cast<cudaStream_t>(opt.stream) : default_stream_for_thread(device);
    const int num_sms = device_sm_count(device);

    Events ev;
    Arena ar(st);
    PTC_CUDA(cudaEventRecord(ev.ev[EV_START], st));

    // ---- inputs on the device ----
    DeviceCoo dA = to_device(A, ar);
    DeviceCoo dB = self ? dA : to_device(B, ar);
    PTC_CUDA(cudaEventRecord(ev.ev[EV_H2D], st));
    stats.a_nnz = A->nnz;
    stats.b_nnz = B->nnz;

    // ---- keys ----
    const KeySpec a_con = make_keyspec(A->dims, a_modes, c);
    const KeySpec a_free = make_keyspec(A->dims, a_modes + c, fa);
    const KeySpec b_con = make_keyspec(B->dims, b_modes, c);
    const KeySpec b_free = make_keyspec(B->dims, b_modes + c, fb);
    uint32_t* err = ar.alloc<uint32_t>(1);
    PTC_CUDA(cudaMemsetAsync(err, 0, sizeof(uint32_t), st));
    uint64_t* a_ckey = ar.alloc<uint64_t>(dA.nnz);
    uint64_t* a_fkey = ar.alloc<uint64_t>(dA.nnz);
    launch_pack_keys(dA.idx, dA.nnz, dA.dims, a_con, a_free, a_ckey, a_fkey, err, st);
    uint64_t* b_ckey = a_ckey;
    uint64_t* b_fkey = a_fkey;
    if (!self) {
        b_ckey = ar.alloc<uint64_t>(dB.nnz);
        b_fkey = ar.alloc<uint64_t>(dB.nnz);
        launch_pack_keys(dB.idx, dB.nnz, dB.dims, b_con, b_free, b_ckey, b_fkey, err, st);
    }
    PTC_REQUIRE(read_scalar(err, st) == 0, PTC_ERR_INDEX_RANGE, "an index is not smaller than its mode size");

    // ---- B side: dense column ids, fibers in (contracted key, column) order, cuckoo table ----
    const uint64_t nb = dB.nnz, na = dA.nnz;
    Ranked cols = rank_keys(b_fkey, nb, b_free.space, ar);
    const uint64_t ncols = cols.nruns;
    uint32_t* col_tuple = ar.alloc<uint32_t>(ncols * std::max(fb, 1u));
    launch_tuples(dB.idx, dB.order, cols.run_start, cols.perm, ncols, b_free, col_tuple, st);

    uint32_t* fperm = ar.alloc<uint32_t>(nb);
    launch_iota(fperm, nb, st);
    const int cbits = bits_for_space(b_con.space);
    const int colbits = bits_for_space(std::max<uint64_t>(ncols, 1));
    if (cbits + colbits <= 64) {
        uint64_t* comp = ar.alloc<uint64_t>(nb);
        launch_composite(b_ckey, cols.rank_of, ncols, nb, comp, st);
        radix_sort_pairs(comp, fperm, nb, 0, cbits + colbits, ar);
    } else {
        uint64_t* k = ar.alloc<uint64_t>(nb);
        launch_composite(b_ckey, cols.rank_of, 0, nb, k, st);  // 0 * ckey + col = col
        radix_sort_pairs(k, fperm, nb, 0, colbits, ar);
        launch_gather<uint64_t>(b_ckey, fperm, nb, k, st);
        radix_sort_pairs(k, fperm, nb, 0, cbits, ar);
    }
    uint64_t* b_ckey_sorted = ar.alloc<uint64_t>(nb);
    launch_gather<uint64_t>(b_ckey, fperm, nb, b_ckey_sorted, st);
    uint32_t* b_fib = ar.alloc<uint32_t>(nb);
    uint32_t* fib_start = ar.alloc<uint32_t>(nb + 1);
    uint64_t* fib_key = ar.alloc<uint64_t>(nb);
    const uint64_t nfib = runs_of_sorted(b_ckey_sorted, nb, b_fib, fib_start, fib_key, ar);
    uint32_t* b_col = ar.alloc<uint32_t>(nb);
    double* b_val = ar.alloc<double>(nb);
    launch_gather<uint32_t>(cols.rank_of, fperm, nb, b_col, st);
    launch_gather<double>(dB.vals, fperm, nb, b_val, st);

    CuckooBuildInfo cinfo;
    const CuckooTable table = cuckoo_build(fib_key, nfib, opt.hash_seed, 64, 0.75, 8, ar, &cinfo);
    stats.hash_attempts = cinfo.attempts;
    PTC_CUDA(cudaEventRecord(ev.ev[EV_BSIDE], st));

    // ---- A side: rows (input order kept inside a row), fiber of every A nonzero ----
    Ranked rows;
    uint32_t* row_tuple = nullptr;
    if (self) {
        rows = cols;  // same tensor, same free modes
        row_tuple = col_tuple;
    } else {
        rows = rank_keys(a_fkey, na, a_free.space, ar);
        row_tuple = ar.alloc<uint32_t>(rows.nruns * std::max(fa, 1u));
        launch_tuples(dA.idx, dA.order, rows.run_start, rows.perm, rows.nruns, a_free, row_tuple, st);
    }
    const uint64_t nrows = rows.nruns;
    uint64_t* a_ckey_sorted = ar.alloc<uint64_t>(na);
    double* a_val = ar.alloc<double>(na);
    launch_gather<uint64_t>(a_ckey, rows.perm, na, a_ckey_sorted, st);
    launch_gather<double>(dA.vals, rows.perm, na, a_val, st);
    int32_t* a_fib = ar.alloc<int32_t>(na);
    cuckoo_lookup(table, a_ckey_sorted, na, a_fib, ar);
    PTC_CUDA(cudaEventRecord(ev.ev[EV_ASIDE], st));

    // ---- symbolic: flops per row, accumulator bins, exact output nnz per work item ----
    uint64_t* alen = ar.alloc<uint64_t>(na + 1);
    launch_fiber_len(a_fib, fib_start, na, alen, st);
    exclusive_scan<uint64_t>(alen, alen, na, ar);
    uint64_t* row_flops = ar.alloc<uint64_t>(nrows);
    launch_row_flops(alen, rows.run_start, nrows, row_flops, st);
    std::vector<uint64_t> h_flops(nrows);
    PTC_CUDA(cudaMemcpyAsync(h_flops.data(), row_flops, nrows * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    PTC_CUDA(cudaStreamSynchronize(st));
    uint64_t flops = 0;
    for (uint64_t f : h_flops) flops += f;
    stats.mult_adds = flops;
    stats.nrows = nrows;
    stats.ncols = ncols;
    stats.nfibers = nfib;
    PTC_REQUIRE(flops > 0, PTC_ERR_EMPTY_CONTRACTION, "tensor contraction not possible!! (no matching fibers)");

    // fine column panels: B fibers are split at multiples of W so a row can be cut into parts
    // that each fit one shared-memory table (W <= table capacity, so a part always fits)
    PTC_REQUIRE(ncols <= sym_bitmap_max_cols(), PTC_ERR_INVALID_ARGUMENT,
                "more than 1.5M distinct B free keys is not supported yet");
    uint32_t W = opt.panel_width ? opt.panel_width : 4096;
    PTC_REQUIRE(W <= hash_part_capacity(), PTC_ERR_INVALID_ARGUMENT, "panel_width larger than a hash part");
    const uint32_t log2w = floor_log2(W);
    const uint32_t P = (uint32_t)std::max<uint64_t>(1, (ncols + W - 1) / W);
    stats.panel_width = W;
    uint32_t* panel_off = nullptr;
    if (P > 1) {
        panel_off = ar.alloc<uint32_t>(nfib * (uint64_t)(P + 1));
        launch_panel_offsets(b_col, b_fib, fib_start, nb, P, log2w, panel_off, st);
    }

    Operands op;
    op.na = na; op.nb = nb; op.nrows = nrows; op.ncols = ncols; op.nfib = nfib;
    op.fa = fa; op.fb = fb;
    op.a_val = a_val; op.a_fib = a_fib; op.row_start = rows.run_start;
    op.b_col = b_col; op.b_val = b_val; op.fib_start = fib_start;
    op.row_tuple = row_tuple; op.col_tuple = col_tuple;
    op.panel_off = panel_off; op.npanels = P; op.panel_log2 = log2w;
    op.err = err;

    // row classes and work lists (largest rows first)
    uint32_t* small_flag = ar.alloc<uint32_t>(nrows + 1);
    uint32_t* big_flag = ar.alloc<uint32_t>(nrows + 1);
    launch_classify_rows(row_flops, nrows, small_row_max_flops(), small_flag, big_flag, st);
    uint32_t* small_pos = ar.alloc<uint32_t>(nrows + 1);
    uint32_t* big_pos = ar.alloc<uint32_t>(nrows + 1);
    exclusive_scan<uint32_t>(small_flag, small_pos, nrows, ar);
    exclusive_scan<uint32_t>(big_flag, big_pos, nrows, ar);
    const uint32_t n_small = read_scalar(small_pos + nrows, st);
    const uint32_t n_big = read_scalar(big_pos + nrows, st);
    uint32_t* small_rows = ar.alloc<uint32_t>(n_small);
    uint32_t* big_rows = ar.alloc<uint32_t>(n_big);
    launch_compact_indices(small_flag, small_pos, nrows, small_rows, st);
    launch_compact_indices(big_flag, big_pos, nrows, big_rows, st);
    if (n_big > 1) {
        uint64_t* wkey = ar.alloc<uint64_t>(n_big);
        launch_work_keys(big_rows, n_big, row_flops, wkey, st);
        radix_sort_pairs(wkey, big_rows, n_big, 0, 40, ar);
    }
    stats.rows_small = n_small;
    stats.rows_hash = n_big;

    // symbolic: exact output nnz per row (and per fine panel for the large rows)
    uint64_t* row_d = ar.alloc<uint64_t>(nrows + 1);
    PTC_CUDA(cudaMemsetAsync(row_d, 0, (nrows + 1) * sizeof(uint64_t), st));
    uint32_t* panel_cnt = ar.alloc<uint32_t>((uint64_t)n_big * P);
    uint32_t* work_counter = ar.alloc<uint32_t>(1);
    OutputView none;
    launch_small_rows(false, op, small_rows, n_small, row_d, nullptr, none, st);
    launch_sym_bitmap(op, big_rows, n_big, panel_cnt, row_d, work_counter, num_sms, st);
    uint64_t* row_off = ar.alloc<uint64_t>(nrows + 1);
    exclusive_scan<uint64_t>(row_d, row_off, nrows, ar);
    const uint64_t out_nnz = read_scalar(row_off + nrows, st);

    // split large rows into parts that fit a shared-memory table
    uint32_t* nparts = ar.alloc<uint32_t>((uint64_t)n_big + 1);
    launch_count_parts(panel_cnt, n_big, P, hash_part_capacity(), nparts, err, st);
    exclusive_scan<uint32_t>(nparts, nparts, n_big, ar);
    const uint32_t n_parts = read_scalar(nparts + n_big, st);
    PTC_REQUIRE(read_scalar(err, st) == 0, PTC_ERR_INTERNAL, "a fine panel exceeds the hash part capacity");
    PartItem* parts = ar.alloc<PartItem>(n_parts);
    launch_fill_parts(big_rows, panel_cnt, n_big, P, hash_part_capacity(), nparts, row_off, parts, st);
    stats.hash_parts = n_parts;
    PTC_CUDA(cudaEventRecord(ev.ev[EV_SYM], st));

    // ---- numeric ----
    const uint32_t od = fa + fb;
    OutputView ov;
    PTC_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&ov.idx), std::max<uint64_t>(out_nnz * od, 1) * sizeof(uint32_t), st));
    PTC_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&ov.val), std::max<uint64_t>(out_nnz, 1) * sizeof(double), st));
    launch_small_rows(true, op, small_rows, n_small, nullptr, row_off, ov, st);
    launch_hash_parts(op, parts, n_parts, ov, work_counter, err, num_sms, st);
    PTC_CUDA(cudaEventRecord(ev.ev[EV_NUM], st));
    if (read_scalar(err, st) != 0) {
        cudaFreeAsync(ov.idx, st);
        cudaFreeAsync(ov.val, st);
        throw Error{PTC_ERR_INTERNAL, "an accumulator table overflowed or met an out-of-range column"};
    }

    // ---- output ----
    out->order = od;
    out->nnz = out_nnz;
    if (opt.output_location == PTC_DEVICE) {
        out->location = PTC_DEVICE;
        out->idx = ov.idx;
        out->vals = ov.val;
        PTC_CUDA(cudaEventRecord(ev.ev[EV_D2H], st));
    } else {
        out->location = PTC_HOST;
        out->idx = static_cast<uint32_t*>(std::malloc(std::max<uint64_t>(out_nnz * od, 1) * sizeof(uint32_t)));
        out->vals = static_cast<double*>(std::malloc(std::max<uint64_t>(out_nnz, 1) * sizeof(double)));
        if (!out->idx || !out->vals) {
            std::free(out->idx);
            std::free(out->vals);
            cudaFreeAsync(ov.idx, st);
            cudaFreeAsync(ov.val, st);
            out->idx = nullptr;
            out->vals = nullptr;
            throw Error{PTC_ERR_OUT_OF_MEMORY, "host output allocation failed"};
        }
        PTC_CUDA(cudaMemcpyAsync(out->idx, ov.idx, out_nnz * od * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        PTC_CUDA(cudaMemcpyAsync(out->vals, ov.val, out_nnz * sizeof(double), cudaMemcpyDeviceToHost, st));
        PTC_CUDA(cudaFreeAsync(ov.idx, st));
        PTC_CUDA(cudaFreeAsync(ov.val, st));
        PTC_CUDA(cudaEventRecord(ev.ev[EV_D2H], st));
    }
    ar.release();
    PTC_CUDA(cudaStreamSynchronize(st));
    PTC_CUDA(cudaGetLastError());

    stats.out_nnz = out_nnz;
    stats.t_h2d_ms = ev.ms(EV_START, EV_H2D);
    stats.t_build_ms = ev.ms(EV_H2D, EV_ASIDE);
    stats.t_symbolic_ms = ev.ms(EV_ASIDE, EV_SYM);
    stats.t_numeric_ms = ev.ms(EV_SYM, EV_NUM);
    stats.t_d2h_ms = ev.ms(EV_NUM, EV_D2H);
    stats.t_total_ms = ev.ms(EV_START, EV_D2H);
    stats.kernel_launches = g_launches;
    if (opt.verbose) print_reference_lines(stats);
    if (stats_out) *stats_out = stats;
}

}  // namespace
}  // namespace ptc

using ptc::Error;

extern "C" {

void ptc_options_init(ptc_options* opt) {
    if (!opt) return;
    std::memset(opt, 0, sizeof(*opt));
    opt->struct_size = sizeof(ptc_options);
    opt->device = -1;
    opt->path = PTC_PATH_TWO_PHASE;
    opt->output_location = PTC_HOST;
    opt->hash_seed = 0x243f6a8885a308d3ull;
}

const char* ptc_status_string(ptc_status s) {
    switch (s) {
        case PTC_OK: return "PTC_OK";
        case PTC_ERR_INVALID_ARGUMENT: return "PTC_ERR_INVALID_ARGUMENT";
        case PTC_ERR_INDEX_RANGE: return "PTC_ERR_INDEX_RANGE";
        case PTC_ERR_KEY_OVERFLOW: return "PTC_ERR_KEY_OVERFLOW";
        case PTC_ERR_EMPTY_CONTRACTION: return "PTC_ERR_EMPTY_CONTRACTION";
        case PTC_ERR_TOO_FEW_NONZEROS: return "PTC_ERR_TOO_FEW_NONZEROS";
        case PTC_ERR_HASH_BUILD: return "PTC_ERR_HASH_BUILD";
        case PTC_ERR_OUT_OF_MEMORY: return "PTC_ERR_OUT_OF_MEMORY";
        case PTC_ERR_CUDA: return "PTC_ERR_CUDA";
        case PTC_ERR_NO_DEVICE: return "PTC_ERR_NO_DEVICE";
        case PTC_ERR_DEVICE_TIMEOUT: return "PTC_ERR_DEVICE_TIMEOUT";
        case PTC_ERR_OVERFLOW: return "PTC_ERR_OVERFLOW";
        case PTC_ERR_INTERNAL: return "PTC_ERR_INTERNAL";
    }
    return "PTC_ERR_UNKNOWN";
}

const char* ptc_last_error(void) {
    std::snprintf(ptc::g_last_error_buf, sizeof(ptc::g_last_error_buf), "%s", ptc::g_last_error.c_str());
    return ptc::g_last_error_buf;
}

ptc_status ptc_contract(const ptc_coo* A, const ptc_coo* B, uint32_t c, const uint32_t* a_modes,
                        const uint32_t* b_modes, const ptc_options* opt, ptc_tensor* out, ptc_stats* stats) {
    try {
        ptc::contract_impl(A, B, c, a_modes, b_modes, opt, out, stats);
        ptc::g_last_error.clear();
        return PTC_OK;
    } catch (const Error& e) {
        ptc::set_last_error(e.status, e.msg);
        return e.status;
    } catch (const std::bad_alloc&) {
        ptc::set_last_error(PTC_ERR_OUT_OF_MEMORY, "host allocation failed");
        return PTC_ERR_OUT_OF_MEMORY;
    } catch (...) {
        ptc::set_last_error(PTC_ERR_INTERNAL, "unexpected exception");
        return PTC_ERR_INTERNAL;
    }
}

ptc_status ptc_self_contract(const uint32_t* hedges, const double* vals, uint32_t d, uint64_t N, const uint32_t* dims,
                             uint32_t c, const uint32_t* dim_tc, const ptc_options* opt, ptc_tensor* out,
                             ptc_stats* stats) {
    ptc_coo A;
    A.order = d;
    A.location = PTC_HOST;
    A.nnz = N;
    A.idx = hedges;
    A.vals = vals;
    A.dims = dims;
    return ptc_contract(&A, nullptr, c, dim_tc, dim_tc, opt, out, stats);
}

void ptc_tensor_free(ptc_tensor* t) {
    if (!t) return;
    if (t->location == PTC_DEVICE) {
        if (t->idx) cudaFree(t->idx);
        if (t->vals) cudaFree(t->vals);
    } else {
        std::free(t->idx);
        std::free(t->vals);
    }
    t->idx = nullptr;
    t->vals = nullptr;
    t->nnz = 0;
}

int ptc_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    int usable = 0;
    for (int i = 0; i < n; ++i) {
        int major = 0;
        if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, i) == cudaSuccess && major == 10) ++usable;
    }
    return usable;
}

}  // extern "C"
