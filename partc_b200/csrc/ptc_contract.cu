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

#include <dlfcn.h>
#include <sys/mman.h>
#include <string>
#include <vector>

#include "partc.h"
#include "ptc_build.cuh"
#include "ptc_internal.cuh"
#include "ptc_prims.cuh"
#include "ptc_learned.cuh"
#include "ptc_sizer.cuh"
#include "ptc_spa.cuh"

namespace ptc {

thread_local uint64_t g_launches = 0;
static thread_local std::string g_last_error;
static thread_local char g_last_error_buf[512];

void set_last_error(ptc_status, const std::string& msg) { g_last_error = msg; }

namespace {

// rows averaging fewer products per A nonzero than this use the sort-based accumulator
constexpr uint32_t kEscMaxAvgProducts = 32;
// a window of fine panels at least 1/kDenseMinFraction full becomes a dense part
constexpr uint32_t kDenseMinFraction = 5;
// largest product count the sort-based accumulator buffers (32 bytes per product)
constexpr uint64_t kEscMaxProducts = 256ull << 20;

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
    uint32_t* run_of = nullptr;     // [n] rank of the i-th smallest
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
    r.run_of = ar.alloc<uint32_t>(n);
    r.run_start = ar.alloc<uint32_t>(n + 1);
    r.nruns = runs_of_sorted(k, n, r.run_of, r.run_start, nullptr, ar);
    r.rank_of = ar.alloc<uint32_t>(n);
    launch_scatter_u32(r.run_of, r.perm, n, r.rank_of, st);
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

// Device -> pageable host copy of a large result: chunks go by DMA into two pinned staging
// buffers while host threads copy the previous chunk out (and fault in the destination pages)
// in parallel.  A plain cudaMemcpy into fresh pageable memory runs at a small fraction of this.
class HostCopier {
  public:
    static constexpr size_t kStage = 128ull << 20;
    void copy(void* dst, const void* src, size_t bytes, cudaStream_t st) {
        if (bytes == 0) return;
        ensure();
        const size_t nchunks = (bytes + kStage - 1) / kStage;
        auto issue = [&](size_t c) {
            const size_t off = c * kStage, n = std::min(kStage, bytes - off);
            PTC_CUDA(cudaMemcpyAsync(stage_[c & 1], static_cast<const char*>(src) + off, n, cudaMemcpyDeviceToHost, st));
            PTC_CUDA(cudaEventRecord(ev_[c & 1], st));
        };
        issue(0);
        for (size_t c = 0; c < nchunks; ++c) {
            if (c + 1 < nchunks) issue(c + 1);
            PTC_CUDA(cudaEventSynchronize(ev_[c & 1]));
            const size_t off = c * kStage, n = std::min(kStage, bytes - off);
            parallel_memcpy(static_cast<char*>(dst) + off, static_cast<const char*>(stage_[c & 1]), n);
        }
    }
    ~HostCopier() {
        for (int i = 0; i < 2; ++i) {
            if (stage_[i]) cudaFreeHost(stage_[i]);
            if (ev_[i]) cudaEventDestroy(ev_[i]);
        }
    }

  private:
    void ensure() {
        if (stage_[0]) return;
        for (int i = 0; i < 2; ++i) {
            PTC_CUDA(cudaMallocHost(&stage_[i], kStage));
            PTC_CUDA(cudaEventCreateWithFlags(&ev_[i], cudaEventDisableTiming));
        }
    }
    static void parallel_memcpy(char* dst, const char* src, size_t n) {
        constexpr size_t kBlock = 1ull << 20;
        const int64_t nb = (int64_t)((n + kBlock - 1) / kBlock);
#pragma omp parallel for schedule(static)
        for (int64_t b = 0; b < nb; ++b) {
            const size_t off = (size_t)b * kBlock;
            std::memcpy(dst + off, src + off, std::min(kBlock, n - off));
        }
    }
    void* stage_[2] = {nullptr, nullptr};
    cudaEvent_t ev_[2] = {nullptr, nullptr};
};

// Host memory for a result: large blocks are 2 MiB aligned and marked for transparent huge
// pages, so filling them costs far fewer page faults.  Released with free().
void* host_result_alloc(size_t bytes) {
    constexpr size_t kHuge = 2ull << 20;
    if (bytes < (64ull << 20)) return std::malloc(bytes ? bytes : 1);
    const size_t rounded = (bytes + kHuge - 1) / kHuge * kHuge;
    void* p = std::aligned_alloc(kHuge, rounded);
    if (p) madvise(p, rounded, MADV_HUGEPAGE);
    return p;
}

HostCopier& host_copier() {
    thread_local HostCopier c;
    return c;
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

// the learned path sizes accumulators and the output for this many times the predicted count
constexpr float kSizerMargin = 1.25f;

const SizerHost* sizer_host(const ptc_sizer* s) { return s ? &s->host : nullptr; }

// The sizer shipped beside the library (sizer_default.bin in the library's directory), if any.
const SizerHost* default_sizer() {
    static std::once_flag once;
    static ptc_sizer* s = nullptr;
    std::call_once(once, [] {
        Dl_info info;
        if (!dladdr(reinterpret_cast<void*>(&default_sizer), &info) || !info.dli_fname) return;
        std::string path(info.dli_fname);
        const size_t slash = path.rfind('/');
        path = (slash == std::string::npos ? std::string(".") : path.substr(0, slash)) + "/sizer_default.bin";
        ptc_sizer* loaded = nullptr;
        if (ptc_sizer_load(path.c_str(), &loaded) == PTC_OK) s = loaded;
    });
    return s ? &s->host : nullptr;
}

// Grow the claimable output to `need` entries, keeping the first `used`.
void grow_output(OutputView& ov, uint32_t od, uint64_t used, uint64_t need, cudaStream_t st) {
    uint32_t* idx = nullptr;
    double* val = nullptr;
    PTC_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&idx), need * od * sizeof(uint32_t), st));
    PTC_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&val), need * sizeof(double), st));
    PTC_CUDA(cudaMemcpyAsync(idx, ov.idx, used * od * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    PTC_CUDA(cudaMemcpyAsync(val, ov.val, used * sizeof(double), cudaMemcpyDeviceToDevice, st));
    PTC_CUDA(cudaFreeAsync(ov.idx, st));
    PTC_CUDA(cudaFreeAsync(ov.val, st));
    ov.idx = idx;
    ov.val = val;
    ov.capacity = need;
}

// Learned path, after the first numeric pass: parts whose accumulator or output claim did not
// fit their prediction wrote nothing and are listed in ov.fail_list.  Their rows get the exact
// symbolic pass, each failed part is re-split exactly, and the new parts run (their sizes are
// exact, so they cannot fail again).  Returns the output nnz.
uint64_t learned_reruns(const Operands& op, const PartItem* parts, uint32_t n_parts, const uint32_t* big_rows,
                        uint32_t n_big, const float* pred, const SplitRule& rule, OutputView& ov,
                        uint32_t* work_counter, uint32_t* err, int num_sms, uint64_t nrows, Arena& ar,
                        ptc_stats& stats) {
    cudaStream_t st = ar.stream();
    const uint32_t P = op.npanels;
    uint64_t* row_actual = ar.alloc<uint64_t>(nrows);
    PTC_CUDA(cudaMemsetAsync(row_actual, 0, nrows * sizeof(uint64_t), st));
    launch_row_actual(parts, ov.item_count, n_parts, row_actual, st);
    const PartItem* cur = parts;
    uint64_t rerun_rows = 0;
    for (int round = 0;; ++round) {
        const uint32_t nfail = read_scalar(ov.fail_count, st);
        if (nfail == 0) break;
        PTC_REQUIRE(round < 4, PTC_ERR_INTERNAL, "exactly sized parts failed again");
        PartItem* failed = ar.alloc<PartItem>(nfail);
        launch_gather_parts(cur, ov.fail_list, nfail, failed, st);
        std::vector<PartItem> hf(nfail);
        PTC_CUDA(cudaMemcpyAsync(hf.data(), failed, nfail * sizeof(PartItem), cudaMemcpyDeviceToHost, st));
        PTC_CUDA(cudaStreamSynchronize(st));
        std::vector<uint32_t> hrows, hridx(nfail);
        std::vector<int64_t> seen;  // small: failed parts are few
        for (uint32_t i = 0; i < nfail; ++i) {
            uint32_t r = 0;
            while (r < hrows.size() && hrows[r] != hf[i].row) ++r;
            if (r == hrows.size()) hrows.push_back(hf[i].row);
            hridx[i] = r;
        }
        const uint32_t nr = (uint32_t)hrows.size();
        rerun_rows += nr;
        uint32_t* drows = ar.alloc<uint32_t>(nr);
        uint32_t* dridx = ar.alloc<uint32_t>(nfail);
        PTC_CUDA(cudaMemcpyAsync(drows, hrows.data(), nr * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        PTC_CUDA(cudaMemcpyAsync(dridx, hridx.data(), nfail * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        uint32_t* cnt = ar.alloc<uint32_t>((uint64_t)nr * P);
        uint64_t* scratch_d = ar.alloc<uint64_t>(nrows);
        PTC_CUDA(cudaMemsetAsync(scratch_d, 0, nrows * sizeof(uint64_t), st));
        launch_sym_bitmap(op, drows, nr, cnt, scratch_d, work_counter, num_sms, st);
        uint32_t* np = ar.alloc<uint32_t>((uint64_t)nfail + 1);
        uint32_t* tot = ar.alloc<uint32_t>(nfail);
        launch_count_parts_range(failed, dridx, nfail, cnt, P, rule, np, tot, st);
        exclusive_scan<uint32_t>(np, np, nfail, ar);
        const uint32_t nnew = read_scalar(np + nfail, st);
        uint64_t* need = ar.alloc<uint64_t>(1);
        launch_sum_u32(tot, nfail, need, st);
        const uint64_t used = read_scalar(ov.cursor, st);
        const uint64_t want = used + read_scalar(need, st);
        if (want > ov.capacity) grow_output(ov, op.fa + op.fb, used, want + 1024, st);
        PartItem* fresh = ar.alloc<PartItem>(nnew);
        launch_fill_parts_range(failed, dridx, nfail, cnt, P, rule, np, fresh, st);
        ov.fail_list = ar.alloc<uint32_t>(std::max<uint32_t>(nnew, 1));
        ov.item_count = ar.alloc<uint32_t>(std::max<uint32_t>(nnew, 1));
        PTC_CUDA(cudaMemsetAsync(ov.fail_count, 0, sizeof(uint32_t), st));
        launch_hash_parts(op, fresh, nnew, ov, work_counter, err, num_sms, st);
        launch_row_actual(fresh, ov.item_count, nnew, row_actual, st);
        cur = fresh;
    }
    stats.rerun_rows = rerun_rows;
    double* esum = ar.alloc<double>(1);
    launch_log2_error(big_rows, n_big, pred, row_actual, esum, st);
    stats.sizer_mean_abs_log2_err = n_big ? read_scalar(esum, st) / n_big : 0.0;
    return read_scalar(ov.cursor, st);
}

// Training samples of the learned sizer, gathered instead of running the numeric pass.
struct Collect {
    std::vector<float> x;  // n * kSizerInputs
    std::vector<float> t;  // n
};

void contract_impl(const ptc_coo* A, const ptc_coo* Bin, uint32_t c, const uint32_t* a_modes,
                   const uint32_t* b_modes_in, const ptc_options* opt_in, ptc_tensor* out, ptc_stats* stats_out,
                   Collect* collect = nullptr) {
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
    PTC_REQUIRE(opt.panel_width == 0 || (opt.panel_width >= 32 && opt.panel_width <= 4096 &&
                                         (opt.panel_width & (opt.panel_width - 1)) == 0),
                PTC_ERR_INVALID_ARGUMENT, "panel_width must be 0 or a power of two in [32, 4096]");

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
    // default: panels of 2048 columns (finer for narrow column spaces), the split table within 1 GiB
    uint32_t W = opt.panel_width;
    if (W == 0) {
        W = 32;
        while (W < 2048 && (uint64_t)W * 16 < ncols) W <<= 1;
        while (W < 4096 && nfib * ((ncols + W - 1) / W + 1) * 4 > (1ull << 30)) W <<= 1;
    }
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
    uint32_t* esc_flag = ar.alloc<uint32_t>(nrows + 1);
    launch_classify_rows(row_flops, rows.run_start, nrows, small_row_max_flops(), kEscMaxAvgProducts, small_flag,
                         big_flag, esc_flag, st);
    uint32_t* esc_pos = ar.alloc<uint32_t>(nrows + 1);
    exclusive_scan<uint32_t>(esc_flag, esc_pos, nrows, ar);
    uint32_t n_esc = read_scalar(esc_pos + nrows, st);
    uint32_t* esc_rows = ar.alloc<uint32_t>(n_esc);
    launch_compact_indices(esc_flag, esc_pos, nrows, esc_rows, st);
    uint64_t* esc_off = ar.alloc<uint64_t>((uint64_t)n_esc + 1);
    uint64_t f_esc = 0;
    if (n_esc > 0) {
        launch_esc_len(esc_rows, n_esc, row_flops, esc_off, st);
        exclusive_scan<uint64_t>(esc_off, esc_off, n_esc, ar);
        f_esc = read_scalar(esc_off + n_esc, st);
        const int ebits = bits_for_space((uint64_t)n_esc), cbits2 = bits_for_space(std::max<uint64_t>(ncols, 1));
        if (f_esc > kEscMaxProducts || ebits + cbits2 > 64) {  // too large for the sort buffers: hash path
            launch_merge_flags(big_flag, esc_flag, nrows, st);
            n_esc = 0;
            f_esc = 0;
        }
    }
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
    stats.rows_long = n_esc;

    const bool learned = opt.path == PTC_PATH_LEARNED && collect == nullptr;
    const SizerHost* sizer = nullptr;
    if (learned) {
        sizer = opt.sizer ? sizer_host(opt.sizer) : default_sizer();
        PTC_REQUIRE(sizer != nullptr, PTC_ERR_INVALID_ARGUMENT,
                    "the learned path needs a sizer: opt.sizer, or sizer_default.bin beside the library");
    }
    SplitRule rule;
    rule.cap = hash_part_capacity();
    rule.dense_panels = dense_part_columns() >> log2w;
    rule.dense_min = W / kDenseMinFraction;
    rule.min_bits = hash_part_min_bits();

    // symbolic: exact output nnz per row (and per fine panel for the large rows); the learned
    // path counts only the sort-based rows (their sort gives the counts) and predicts the rest
    uint64_t* row_d = ar.alloc<uint64_t>(nrows + 1);
    PTC_CUDA(cudaMemsetAsync(row_d, 0, (nrows + 1) * sizeof(uint64_t), st));
    uint32_t* panel_cnt = ar.alloc<uint32_t>((uint64_t)n_big * P);
    uint32_t* work_counter = ar.alloc<uint32_t>(1);
    OutputView none;
    if (!learned) {
        launch_small_rows(false, op, small_rows, n_small, row_d, nullptr, none, st);
        launch_sym_bitmap(op, big_rows, n_big, panel_cnt, row_d, work_counter, num_sms, st);
    }
    // sort-based rows: expand their products in stream order, sort stably by (row, column)
    const uint32_t esc_colbits = (uint32_t)colbits;
    uint64_t* esc_key = nullptr;
    double* esc_val = nullptr;
    uint32_t* esc_perm = nullptr;
    uint32_t* esc_run_start = nullptr;
    uint64_t* esc_run_key = nullptr;
    uint32_t* esc_first = nullptr;
    uint64_t esc_runs = 0;
    if (n_esc > 0) {
        int32_t* esc_of = ar.alloc<int32_t>(nrows);
        PTC_CUDA(cudaMemsetAsync(esc_of, 0xff, nrows * sizeof(int32_t), st));
        launch_esc_index(esc_rows, n_esc, esc_of, st);
        esc_key = ar.alloc<uint64_t>(f_esc);
        esc_val = ar.alloc<double>(f_esc);
        esc_perm = ar.alloc<uint32_t>(f_esc);
        launch_esc_expand(op, rows.run_of, esc_of, alen, esc_off, esc_colbits, esc_key, esc_val, esc_perm, st);
        radix_sort_pairs(esc_key, esc_perm, f_esc, 0, esc_colbits + bits_for_space((uint64_t)n_esc), ar);
        esc_run_start = ar.alloc<uint32_t>(f_esc + 1);
        esc_run_key = ar.alloc<uint64_t>(f_esc);
        esc_runs = runs_of_sorted(esc_key, f_esc, nullptr, esc_run_start, esc_run_key, ar);
        esc_first = ar.alloc<uint32_t>(n_esc);
        launch_esc_count(esc_run_key, esc_runs, esc_colbits, esc_rows, row_d, esc_first, st);
    }
    uint64_t* row_off = ar.alloc<uint64_t>(nrows + 1);
    exclusive_scan<uint64_t>(row_d, row_off, nrows, ar);
    const uint64_t exact_nnz = read_scalar(row_off + nrows, st);  // all rows, or sort-based rows only
    if (collect) {
        // features of the rows the learned path sizes, and log2(1 + their exact output nnz)
        float* gp = ar.alloc<float>((uint64_t)(P + 1) * kGridPoints);
        launch_popularity_table(b_col, nb, ncols, P, log2w, gp, ar);
        float* fx = ar.alloc<float>((uint64_t)n_big * kSizerInputs);
        float* ft = ar.alloc<float>(n_big);
        launch_row_features(op, big_rows, n_big, row_flops, gp, fx, st);
        launch_row_targets(big_rows, n_big, row_d, ft, st);
        collect->x.resize((uint64_t)n_big * kSizerInputs);
        collect->t.resize(n_big);
        PTC_CUDA(cudaMemcpyAsync(collect->x.data(), fx, collect->x.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
        PTC_CUDA(cudaMemcpyAsync(collect->t.data(), ft, collect->t.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
        ar.release();
        PTC_CUDA(cudaStreamSynchronize(st));
        stats.out_nnz = exact_nnz;
        if (stats_out) *stats_out = stats;
        return;
    }

    float* pred = nullptr;
    uint64_t capacity = exact_nnz;
    if (learned && n_big > 0) {
        // sizer: per-row features -> predicted log2(1 + nnz) -> per-panel counts by column popularity
        float* gp = ar.alloc<float>((uint64_t)(P + 1) * kGridPoints);
        launch_popularity_table(b_col, nb, ncols, P, log2w, gp, ar);
        float* fx = ar.alloc<float>((uint64_t)n_big * kSizerInputs);
        launch_row_features(op, big_rows, n_big, row_flops, gp, fx, st);
        pred = ar.alloc<float>(n_big);
        sizer_predict_device(*sizer, fx, n_big, pred, ar);
        launch_predicted_panel_counts(big_rows, n_big, row_flops, pred, gp, P, log2w, ncols, kSizerMargin, panel_cnt,
                                      st);
        uint64_t* psum = ar.alloc<uint64_t>(1);
        launch_sum_u32(panel_cnt, (uint64_t)n_big * P, psum, st);
        capacity += read_scalar(psum, st);
    }
    if (learned) capacity += (uint64_t)n_small * small_row_max_flops() + 1024;

    // split large rows into parts that fit a shared-memory table
    uint32_t* nparts = ar.alloc<uint32_t>((uint64_t)n_big + 1);
    launch_count_parts(panel_cnt, n_big, P, rule, nparts, err, st);
    exclusive_scan<uint32_t>(nparts, nparts, n_big, ar);
    const uint32_t n_parts = read_scalar(nparts + n_big, st);
    PTC_REQUIRE(read_scalar(err, st) == 0, PTC_ERR_INTERNAL, "a fine panel exceeds the hash part capacity");
    PartItem* parts = ar.alloc<PartItem>(n_parts);
    launch_fill_parts(big_rows, panel_cnt, n_big, P, rule, nparts, learned ? nullptr : row_off, parts, st);
    stats.hash_parts = n_parts;
    PTC_CUDA(cudaEventRecord(ev.ev[EV_SYM], st));

    // ---- numeric ----
    const uint32_t od = fa + fb;
    OutputView ov;
    PTC_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&ov.idx), std::max<uint64_t>(capacity * od, 1) * sizeof(uint32_t), st));
    PTC_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&ov.val), std::max<uint64_t>(capacity, 1) * sizeof(double), st));
    uint64_t out_nnz = exact_nnz;
    try {
        if (learned) {
            ov.capacity = capacity;
            ov.cursor = ar.alloc<uint64_t>(1);
            ov.fail_count = ar.alloc<uint32_t>(1);
            ov.fail_list = ar.alloc<uint32_t>(std::max<uint32_t>(n_parts, 1));
            ov.item_count = ar.alloc<uint32_t>(std::max<uint32_t>(n_parts, 1));
            PTC_CUDA(cudaMemcpyAsync(ov.cursor, &exact_nnz, sizeof(uint64_t), cudaMemcpyHostToDevice, st));
            PTC_CUDA(cudaMemsetAsync(ov.fail_count, 0, sizeof(uint32_t), st));
        }
        launch_small_rows(true, op, small_rows, n_small, nullptr, learned ? nullptr : row_off, ov, st);
        launch_hash_parts(op, parts, n_parts, ov, work_counter, err, num_sms, st);
        if (n_esc > 0)
            launch_esc_fold(op, ov, esc_run_key, esc_run_start, esc_runs, esc_colbits, esc_rows, esc_first, row_off,
                            esc_perm, esc_val, f_esc, reinterpret_cast<double*>(esc_key), st);
        if (learned) {
            out_nnz = learned_reruns(op, parts, n_parts, big_rows, n_big, pred, rule, ov, work_counter, err, num_sms,
                                     nrows, ar, stats);
        }
        PTC_CUDA(cudaEventRecord(ev.ev[EV_NUM], st));
        PTC_REQUIRE(read_scalar(err, st) == 0, PTC_ERR_INTERNAL,
                    "an accumulator table overflowed or met an out-of-range column");
    } catch (...) {
        cudaFreeAsync(ov.idx, st);
        cudaFreeAsync(ov.val, st);
        throw;
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
        out->idx = static_cast<uint32_t*>(host_result_alloc(out_nnz * od * sizeof(uint32_t)));
        out->vals = static_cast<double*>(host_result_alloc(out_nnz * sizeof(double)));
        if (!out->idx || !out->vals) {
            std::free(out->idx);
            std::free(out->vals);
            cudaFreeAsync(ov.idx, st);
            cudaFreeAsync(ov.val, st);
            out->idx = nullptr;
            out->vals = nullptr;
            throw Error{PTC_ERR_OUT_OF_MEMORY, "host output allocation failed"};
        }
        host_copier().copy(out->idx, ov.idx, out_nnz * od * sizeof(uint32_t), st);
        host_copier().copy(out->vals, ov.val, out_nnz * sizeof(double), st);
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

ptc_status ptc_sizer_collect(const ptc_coo* A, const ptc_coo* B, uint32_t c, const uint32_t* a_modes,
                             const uint32_t* b_modes, const ptc_options* opt, float** features, float** targets,
                             uint64_t* n) {
    try {
        PTC_REQUIRE(features && targets && n, PTC_ERR_INVALID_ARGUMENT, "null output argument");
        ptc::Collect col;
        ptc_tensor dummy;
        ptc::contract_impl(A, B, c, a_modes, b_modes, opt, &dummy, nullptr, &col);
        *n = col.t.size();
        *features = static_cast<float*>(std::malloc(std::max<size_t>(col.x.size(), 1) * sizeof(float)));
        *targets = static_cast<float*>(std::malloc(std::max<size_t>(col.t.size(), 1) * sizeof(float)));
        PTC_REQUIRE(*features && *targets, PTC_ERR_OUT_OF_MEMORY, "host allocation failed");
        std::memcpy(*features, col.x.data(), col.x.size() * sizeof(float));
        std::memcpy(*targets, col.t.data(), col.t.size() * sizeof(float));
        ptc::g_last_error.clear();
        return PTC_OK;
    } catch (const Error& e) {
        ptc::set_last_error(e.status, e.msg);
        return e.status;
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
