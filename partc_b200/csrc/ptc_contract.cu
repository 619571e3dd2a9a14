// Host orchestration and the C ABI (include/partc.h).
//
// One call replaces main.cpp:112-118 of the reference: B = A (self-contraction) or a second
// tensor, the FKS/cuckoo table on B's contracted modes (buildHashTable(B), fksCuckoo.hpp:1044),
// the row grouping of A (buildHashTable(A_copy)), reorder_tensor (fksCuckooTC.hpp:31-77), the
// symbolic pass (:94-154) and the numeric pass (:180-357).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <unistd.h>
#include <unordered_map>
#include <map>

#include <dlfcn.h>
#include <sys/mman.h>
#include <string>
#include <type_traits>
#include <vector>

#include "partc.h"
#include "ptc_build.cuh"
#include "ptc_internal.cuh"
#include "ptc_prims.cuh"
#include "ptc_learned.cuh"
#include "ptc_sizer.cuh"
#include "ptc_spa.cuh"
#include "ptc_rowmap.cuh"

namespace ptc {

thread_local uint64_t g_launches = 0;
static thread_local std::string g_last_error;
static thread_local char g_last_error_buf[512];

void set_last_error(ptc_status, const std::string& msg) { g_last_error = msg; }

namespace {

// rows averaging fewer products per A nonzero than this use the sort-based accumulator
constexpr uint32_t kEscMaxAvgProducts = 64;
// rows with at most this many products use the one-warp accumulator (its table holds 512)
constexpr uint32_t kSmallMaxProducts = 128;
// a window of fine panels at least 1/kDenseMinFraction full becomes a dense part
constexpr uint32_t kDenseMinFraction = 5;
// largest product count the sort-based accumulator buffers (32 bytes per product)
constexpr uint64_t kEscMaxProducts = 256ull << 20;
// largest per-fiber panel table (fibers x (panels + 1) offsets)
constexpr uint64_t kPanelTableBytes = 4ull << 30;
// cuckoo build of B's fibers: eviction chain bound and builds tried (ptc_options defaults)
constexpr uint32_t kCuckooMaxChain = 64;
constexpr uint32_t kCuckooMaxAttempts = 8;

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
    static constexpr int kN = 10;
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

enum { EV_START = 0, EV_H2D, EV_BSIDE, EV_ASIDE, EV_SYM, EV_NUM, EV_D2H, EV_WAVE0, EV_WAVE1 };

// Two more streams per device and host thread for kernels of one call that do not depend on each
// other (they write disjoint output ranges): fork() orders them after the call's stream so far,
// join() orders the call's stream after them.
struct AuxStreams {
    cudaStream_t s[2] = {nullptr, nullptr};
    cudaEvent_t fork_ev = nullptr, join_ev[2] = {nullptr, nullptr};
    void fork(cudaStream_t main) {
        PTC_CUDA(cudaEventRecord(fork_ev, main));
        for (cudaStream_t a : s) PTC_CUDA(cudaStreamWaitEvent(a, fork_ev, 0));
    }
    void join(cudaStream_t main) {
        for (int i = 0; i < 2; ++i) {
            PTC_CUDA(cudaEventRecord(join_ev[i], s[i]));
            PTC_CUDA(cudaStreamWaitEvent(main, join_ev[i], 0));
        }
    }
};

AuxStreams& aux_streams(int device) {
    constexpr int kMaxDevices = 64;
    PTC_REQUIRE(device >= 0 && device < kMaxDevices, PTC_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    thread_local AuxStreams aux[kMaxDevices];
    AuxStreams& a = aux[device];
    if (!a.s[0]) {
        for (int i = 0; i < 2; ++i) {
            PTC_CUDA(cudaStreamCreateWithFlags(&a.s[i], cudaStreamNonBlocking));
            PTC_CUDA(cudaEventCreateWithFlags(&a.join_ev[i], cudaEventDisableTiming));
        }
        PTC_CUDA(cudaEventCreateWithFlags(&a.fork_ev, cudaEventDisableTiming));
    }
    return a;
}

// One non-blocking stream per device and host thread, kept for the thread's lifetime.
cudaStream_t default_stream_for_thread(int device) {
    constexpr int kMaxDevices = 64;
    PTC_REQUIRE(device >= 0 && device < kMaxDevices, PTC_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    thread_local cudaStream_t streams[kMaxDevices] = {};
    if (!streams[device]) PTC_CUDA(cudaStreamCreateWithFlags(&streams[device], cudaStreamNonBlocking));
    return streams[device];
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
    uint64_t* run_key = nullptr;    // [nruns] the distinct keys, increasing
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
    r.run_key = ar.alloc<uint64_t>(std::max<uint64_t>(n, 1));
    r.nruns = runs_of_sorted(k, n, r.run_of, r.run_start, r.run_key, ar);
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

// B entries grouped into fibers: sorted by (contracted key, column) with input order kept among
// equal keys (reorder_tensor, fksCuckooTC.hpp:31-77), every fiber contiguous and ordered by column.
struct Fibers {
    uint64_t n = 0;
    uint32_t* start = nullptr;  // [n + 1]
    uint64_t* key = nullptr;    // [n] contracted key of each fiber
    uint32_t* col = nullptr;    // [nb] column id of each sorted entry
    double* val = nullptr;      // [nb]
};

// col_rank[j] = rank of entry j's free key among the ncols distinct ones; col_id (default
// col_rank) is the column id stored for it.
Fibers group_fibers(const uint64_t* ckey, const uint32_t* col_rank, uint64_t ncols, uint64_t nb, int cbits,
                    const double* vals, Arena& ar, const uint32_t* col_id = nullptr) {
    cudaStream_t st = ar.stream();
    uint32_t* fperm = ar.alloc<uint32_t>(nb);
    launch_iota(fperm, nb, st);
    const int colbits = bits_for_space(std::max<uint64_t>(ncols, 1));
    if (cbits + colbits <= 64) {
        uint64_t* comp = ar.alloc<uint64_t>(nb);
        launch_composite(ckey, col_rank, ncols, nb, comp, st);
        radix_sort_pairs(comp, fperm, nb, 0, cbits + colbits, ar);
    } else {
        uint64_t* k = ar.alloc<uint64_t>(nb);
        launch_composite(ckey, col_rank, 0, nb, k, st);  // 0 * ckey + col = col
        radix_sort_pairs(k, fperm, nb, 0, colbits, ar);
        launch_gather<uint64_t>(ckey, fperm, nb, k, st);
        radix_sort_pairs(k, fperm, nb, 0, cbits, ar);
    }
    uint64_t* ckey_sorted = ar.alloc<uint64_t>(nb);
    launch_gather<uint64_t>(ckey, fperm, nb, ckey_sorted, st);
    Fibers f;
    f.start = ar.alloc<uint32_t>(nb + 1);
    f.key = ar.alloc<uint64_t>(std::max<uint64_t>(nb, 1));
    f.n = runs_of_sorted(ckey_sorted, nb, nullptr, f.start, f.key, ar);
    f.col = ar.alloc<uint32_t>(nb);
    f.val = ar.alloc<double>(nb);
    launch_gather<uint32_t>(col_id ? col_id : col_rank, fperm, nb, f.col, st);
    launch_gather<double>(vals, fperm, nb, f.val, st);
    return f;
}

// Device -> pageable host copy of a large result: chunks go by DMA into two pinned staging
// buffers while host threads copy the previous chunk out (and fault in the destination pages)
// in parallel.  A plain cudaMemcpy into fresh pageable memory runs at a small fraction of this.
struct HostSeg {
    const void* src;
    size_t bytes;
};

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
    // Pageable host segments -> one contiguous device buffer, staged the same way.
    void gather_to_device(void* dst, const std::vector<HostSeg>& segs, cudaStream_t st) {
        size_t total = 0;
        for (const HostSeg& g : segs) total += g.bytes;
        if (total == 0) return;
        ensure();
        struct Piece {
            const char* src;
            size_t off, n;
        };
        size_t seg = 0, seg_off = 0, done = 0;
        for (size_t c = 0; done < total; ++c) {
            const size_t n = std::min(kStage, total - done);
            std::vector<Piece> pieces;
            for (size_t filled = 0; filled < n;) {
                const size_t take = std::min(segs[seg].bytes - seg_off, n - filled);
                for (size_t o = 0; o < take; o += kBlock)  // at most 1 MiB per piece
                    pieces.push_back({static_cast<const char*>(segs[seg].src) + seg_off + o, filled + o,
                                      std::min(kBlock, take - o)});
                filled += take;
                seg_off += take;
                if (seg_off == segs[seg].bytes) {
                    ++seg;
                    seg_off = 0;
                }
            }
            char* stage = static_cast<char*>(stage_[c & 1]);
            PTC_CUDA(cudaEventSynchronize(ev_[c & 1]));  // its previous copy has left the buffer
            const int64_t np = (int64_t)pieces.size();
#pragma omp parallel for schedule(dynamic, 4)
            for (int64_t i = 0; i < np; ++i) std::memcpy(stage + pieces[i].off, pieces[i].src, pieces[i].n);
            PTC_CUDA(cudaMemcpyAsync(static_cast<char*>(dst) + done, stage, n, cudaMemcpyHostToDevice, st));
            PTC_CUDA(cudaEventRecord(ev_[c & 1], st));
            done += n;
        }
        for (int i = 0; i < 2; ++i) PTC_CUDA(cudaEventSynchronize(ev_[i]));
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
    static constexpr size_t kBlock = 1ull << 20;
    static void parallel_memcpy(char* dst, const char* src, size_t n) {
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

// Pinned host blocks for results, kept between calls.  A result copied into pinned memory goes
// from HBM to the host by DMA at the link's speed, with no staging copy; pinning fresh memory for
// every call would cost more than the copy itself, so released blocks wait here for the next
// result of a similar size.  At most `cap` bytes are kept (environment variable
// PARTC_PINNED_POOL_MIB; default a quarter of the host's memory; 0 turns the pool off).
class PinnedPool {
  public:
    static PinnedPool& get() {
        static PinnedPool* p = new PinnedPool;  // never destroyed: blocks may outlive static teardown
        return *p;
    }
    // A block of at least `bytes` bytes, or nullptr (pool off, or the allocation failed).
    void* take(size_t bytes) {
        if (cap_ == 0 || bytes < kMinBytes) return nullptr;
        const size_t want = round_up(bytes);
        {
            std::lock_guard<std::mutex> lock(mu_);
            auto it = free_.lower_bound(want);
            if (it != free_.end() && it->first <= 2 * want) {
                void* p = it->second;
                kept_ -= it->first;
                free_.erase(it);
                return p;
            }
        }
        void* p = nullptr;
        if (cudaHostAlloc(&p, want, cudaHostAllocPortable) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        std::lock_guard<std::mutex> lock(mu_);
        size_[p] = want;
        return p;
    }
    // Back to the pool (the oldest kept blocks are freed while the pool holds more than cap).
    void give(void* p) {
        if (!p) return;
        std::vector<void*> drop;
        {
            std::lock_guard<std::mutex> lock(mu_);
            const size_t sz = size_.at(p);
            free_.emplace(sz, p);
            kept_ += sz;
            while (kept_ > cap_ && !free_.empty()) {
                auto it = free_.begin();
                kept_ -= it->first;
                drop.push_back(it->second);
                size_.erase(it->second);
                free_.erase(it);
            }
        }
        for (void* q : drop) cudaFreeHost(q);
    }

  private:
    static constexpr size_t kMinBytes = 64ull << 20;  // smaller results take the plain path
    static constexpr size_t kRound = 64ull << 20;
    static size_t round_up(size_t b) { return (b + kRound - 1) / kRound * kRound; }
    PinnedPool() {
        const char* env = std::getenv("PARTC_PINNED_POOL_MIB");
        if (env) {
            cap_ = (size_t)std::strtoull(env, nullptr, 10) << 20;
        } else {
            const long pages = sysconf(_SC_PHYS_PAGES), page = sysconf(_SC_PAGE_SIZE);
            cap_ = (pages > 0 && page > 0) ? (size_t)pages * (size_t)page / 4 : 0;
        }
    }
    std::mutex mu_;
    std::multimap<size_t, void*> free_;        // kept blocks by size
    std::unordered_map<void*, size_t> size_;   // size of every block the pool made
    size_t kept_ = 0;
    size_t cap_ = 0;
};

// Output block behind a ptc_tensor's arrays (ptc_tensor::opaque): one wave of a batch, shared by
// the item tensors cut from it, or a single result in pinned pool blocks.  The last
// ptc_tensor_free of its tensors releases it.
constexpr uint32_t kPinnedPoolBlock = 2;  // location of a block from the pinned pool
struct SharedBlock {
    std::atomic<uint32_t> refs{0};
    uint32_t location = PTC_HOST;  // PTC_HOST (malloc), PTC_DEVICE, or kPinnedPoolBlock
    void* idx = nullptr;
    void* val = nullptr;
};

void release_block(SharedBlock* b) {
    if (b->refs.fetch_sub(1) != 1) return;
    if (b->location == PTC_DEVICE) {
        cudaFree(b->idx);
        cudaFree(b->val);
    } else if (b->location == kPinnedPoolBlock) {
        PinnedPool::get().give(b->idx);
        PinnedPool::get().give(b->val);
    } else {
        std::free(b->idx);
        std::free(b->val);
    }
    delete b;
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
// a batch item's budget is the sum over its few large rows, whose relative errors average out
// less than over a whole contraction's: a wider margin keeps its claims from running short
constexpr float kSizerBatchMargin = 1.5f;

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

ptc_options resolve_options(const ptc_options* opt_in) {
    ptc_options opt;
    ptc_options_init(&opt);
    if (opt_in) {
        // callers built against the layout before the cuckoo fields get their defaults
        PTC_REQUIRE(opt_in->struct_size >= offsetof(ptc_options, cuckoo_max_chain), PTC_ERR_INVALID_ARGUMENT,
                    "ptc_options.struct_size too small (call ptc_options_init)");
        std::memcpy(&opt, opt_in, std::min<size_t>(opt_in->struct_size, sizeof(opt)));
    }
    PTC_REQUIRE(opt.output_location == PTC_HOST || opt.output_location == PTC_DEVICE, PTC_ERR_INVALID_ARGUMENT,
                "bad output_location");
    PTC_REQUIRE(opt.panel_width == 0 || (opt.panel_width >= 32 && opt.panel_width <= 4096 &&
                                         (opt.panel_width & (opt.panel_width - 1)) == 0),
                PTC_ERR_INVALID_ARGUMENT, "panel_width must be 0 or a power of two in [32, 4096]");
    PTC_REQUIRE(opt.large_rows <= PTC_LARGE_ROWS_PANELS, PTC_ERR_INVALID_ARGUMENT, "bad large_rows");
    PTC_REQUIRE(opt.path == PTC_PATH_TWO_PHASE || opt.path == PTC_PATH_LEARNED, PTC_ERR_INVALID_ARGUMENT,
                "bad path");
    return opt;
}

// The argument checks of one contraction (`where` prefixes the messages).
void validate_pair(const ptc_coo* A, const ptc_coo* B, uint32_t c, const uint32_t* a_modes, const uint32_t* b_modes,
                   const std::string& where) {
    validate_coo(A, (where + "A").c_str());
    validate_coo(B, (where + "B").c_str());
    PTC_REQUIRE(c >= 1 && c <= A->order && c <= B->order, PTC_ERR_INVALID_ARGUMENT,
                where + "need 1 <= c <= order of each tensor");
    validate_modes(a_modes, A->order, (where + "a_modes").c_str());
    validate_modes(b_modes, B->order, (where + "b_modes").c_str());
    for (uint32_t j = 0; j < c; ++j)
        PTC_REQUIRE(A->dims[a_modes[j]] == B->dims[b_modes[j]], PTC_ERR_INVALID_ARGUMENT,
                    where + "paired contracted modes have different sizes");
    PTC_REQUIRE(A->order - c + B->order - c >= 1, PTC_ERR_EMPTY_CONTRACTION,
                where + "tensor contraction not possible (no free modes)");
}

struct DeviceSetup {
    int device = 0;
    cudaStream_t stream = nullptr;
    int num_sms = 0;
};

DeviceSetup setup_device(const ptc_options& opt) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        throw Error{PTC_ERR_NO_DEVICE, "no usable CUDA device"};
    }
    DeviceSetup d;
    d.device = opt.device;
    if (d.device < 0) PTC_CUDA(cudaGetDevice(&d.device));
    PTC_REQUIRE(d.device < ndev, PTC_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    PTC_CUDA(cudaSetDevice(d.device));
    int major = 0;
    PTC_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, d.device));
    if (major != 10) throw Error{PTC_ERR_NO_DEVICE, "this library is built for sm_100a (B200) only"};
    keep_pool_memory(d.device);
    d.stream = opt.stream ? static_cast<cudaStream_t>(opt.stream) : default_stream_for_thread(d.device);
    d.num_sms = device_sm_count(d.device);
    return d;
}

// Grow the claimable output of a single contraction to `need` entries, keeping the first `used`.
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

// Work items of one launch on the learned path and what the launch reported about them.
struct Launched {
    int kind;                 // 0 warp tasks, 1 block parts
    const PartItem* parts;
    uint32_t n;
    uint32_t* fail_list;
    uint32_t* fail_count;
    uint32_t* item_count;
};

// Exact symbolic pass of large rows for the panel kernels: per-panel counts (panel_cnt, pbase as
// launch_sym_bitmap takes them) and row totals added to row_d.  One bitmap of each row's columns
// in shared memory when they fit (launch_row_counts), else the windowed bitmap pass.
void exact_panel_counts(const Operands& op, const uint32_t* rows, uint32_t n, uint32_t* panel_cnt,
                        const uint64_t* pbase, uint64_t* row_d, uint32_t* work_counter, int num_sms, cudaStream_t st) {
    if (op.ncols <= row_counts_max_cols() && op.panel_log2 >= 5)
        launch_row_counts(op, rows, n, panel_cnt, pbase, row_d, work_counter, num_sms, st);
    else
        launch_sym_bitmap(op, rows, n, panel_cnt, pbase, row_d, work_counter, num_sms, st);
}

// Learned path of a single contraction, after the first numeric pass: work items whose
// accumulator overflowed or whose claim did not fit wrote nothing and are listed in their launch's
// fail list.  Their rows get the exact symbolic pass, each failed item is re-split exactly into
// block parts, and those claim after the entries already written (their sizes are exact, so they
// cannot fail again).  Adds every row's entries to row_actual; returns the rows rerun.
uint64_t learned_reruns(const Operands& op, std::vector<Launched> groups, const SplitRule& rule, OutputView& ov,
                        uint32_t* work_counter, uint32_t* err, int num_sms, uint64_t nrows, uint64_t* row_actual,
                        Arena& ar) {
    cudaStream_t st = ar.stream();
    const uint32_t P = op.npanels;
    for (const Launched& g : groups) launch_row_actual(g.parts, g.item_count, g.n, row_actual, st);
    uint64_t rerun_rows = 0;
    for (int round = 0;; ++round) {
        std::vector<uint32_t> nf(groups.size());
        uint32_t nfail = 0;
        for (size_t gi = 0; gi < groups.size(); ++gi) nfail += (nf[gi] = read_scalar(groups[gi].fail_count, st));
        if (nfail == 0) break;
        PTC_REQUIRE(round < 4, PTC_ERR_INTERNAL, "exactly sized parts failed again");
        PartItem* failed = ar.alloc<PartItem>(nfail);
        for (size_t gi = 0, at = 0; gi < groups.size(); at += nf[gi], ++gi)
            launch_gather_parts(groups[gi].parts, groups[gi].fail_list, nf[gi], failed + at, st);
        std::vector<PartItem> hf(nfail);
        PTC_CUDA(cudaMemcpyAsync(hf.data(), failed, nfail * sizeof(PartItem), cudaMemcpyDeviceToHost, st));
        PTC_CUDA(cudaStreamSynchronize(st));
        std::vector<uint32_t> hrows, hridx(nfail);
        for (uint32_t i = 0; i < nfail; ++i) {  // failed items are few
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
        exact_panel_counts(op, drows, nr, cnt, nullptr, scratch_d, work_counter, num_sms, st);
        uint32_t* np = ar.alloc<uint32_t>((uint64_t)nfail + 1);
        uint32_t* tot = ar.alloc<uint32_t>(nfail);
        launch_count_parts_range(failed, dridx, nfail, cnt, P, rule, np, tot, st);
        exclusive_scan<uint32_t>(np, np, nfail, ar);
        const uint32_t nnew = read_scalar(np + nfail, st);
        uint64_t* need = ar.alloc<uint64_t>(1);
        launch_sum_u32(tot, nfail, need, st);
        // the successful claims fill [0, cursor - overshoot); later claims start there
        const uint64_t used = read_scalar(ov.cursor, st) - read_scalar(ov.overshoot, st);
        const uint64_t want = used + read_scalar(need, st);
        if (want > ov.capacity) grow_output(ov, op.fa + op.fb, used, want + 1024, st);
        PTC_CUDA(cudaMemcpyAsync(ov.cursor, &used, sizeof(uint64_t), cudaMemcpyHostToDevice, st));
        PTC_CUDA(cudaMemsetAsync(ov.overshoot, 0, sizeof(uint64_t), st));
        PartItem* fresh = ar.alloc<PartItem>(nnew);
        launch_fill_parts_range(failed, dridx, nfail, cnt, P, rule, np, fresh, st);
        Launched g{1, fresh, nnew, ar.alloc<uint32_t>(std::max<uint32_t>(nnew, 1)), groups[0].fail_count,
                   ar.alloc<uint32_t>(std::max<uint32_t>(nnew, 1))};
        for (const Launched& old : groups) PTC_CUDA(cudaMemsetAsync(old.fail_count, 0, sizeof(uint32_t), st));
        OutputView o2 = ov;
        o2.fail_list = g.fail_list;
        o2.fail_count = g.fail_count;
        o2.item_count = g.item_count;
        launch_hash_parts(op, fresh, nnew, o2, work_counter, err, num_sms, st);
        launch_row_actual(fresh, g.item_count, nnew, row_actual, st);
        groups.assign(1, g);
    }
    return rerun_rows;
}

// Learned path on the row bitmap kernel: rows whose claim did not fit the predicted output are
// listed in mo.fail_list (their exact counts in mo.item_count); the output grows to hold them
// and they run again, claiming after the entries already written (their sizes are now known, so
// they cannot fail again).  Writes every row's entries to row_actual; returns the rows rerun.
uint64_t rowmap_reruns(const Operands& op, const uint32_t* rows, uint32_t nrows, const OutputView& mo,
                       OutputView& ov, uint32_t* work_counter, int num_sms, uint64_t* row_actual, Arena& ar) {
    cudaStream_t st = ar.stream();
    const uint32_t nfail = read_scalar(mo.fail_count, st);
    launch_scatter_counts(rows, nrows, mo.item_count, row_actual, st);
    if (nfail > 0) {
        uint32_t* again = ar.alloc<uint32_t>(nfail);
        uint32_t* cnt = ar.alloc<uint32_t>(nfail);
        launch_gather<uint32_t>(rows, mo.fail_list, nfail, again, st);
        launch_gather<uint32_t>(mo.item_count, mo.fail_list, nfail, cnt, st);
        uint64_t* need = ar.alloc<uint64_t>(1);
        launch_sum_u32(cnt, nfail, need, st);
        const uint64_t used = read_scalar(ov.cursor, st) - read_scalar(ov.overshoot, st);
        const uint64_t want = used + read_scalar(need, st);
        if (want > ov.capacity) grow_output(ov, op.fa + op.fb, used, want + 1024, st);
        PTC_CUDA(cudaMemcpyAsync(ov.cursor, &used, sizeof(uint64_t), cudaMemcpyHostToDevice, st));
        PTC_CUDA(cudaMemsetAsync(ov.overshoot, 0, sizeof(uint64_t), st));
        OutputView o2 = ov;
        o2.fail_count = mo.fail_count;
        o2.fail_list = ar.alloc<uint32_t>(nfail);
        o2.item_count = nullptr;
        PTC_CUDA(cudaMemsetAsync(o2.fail_count, 0, sizeof(uint32_t), st));
        launch_rowmap(kRowmapClaim, op, again, nfail, nullptr, nullptr, o2, work_counter, num_sms, st);
        PTC_REQUIRE(read_scalar(o2.fail_count, st) == 0, PTC_ERR_INTERNAL, "exactly sized rows failed again");
    }
    return nfail;
}

// Training samples of the learned sizer, gathered instead of running the numeric pass.
struct Collect {
    std::vector<float> x;  // n * kSizerInputs
    std::vector<float> t;  // n
};

// What the build phase hands to planning: the grouped operands and, for a batch, where each
// item's rows and columns lie.
struct Front {
    Operands op;
    const uint32_t* a_row = nullptr;  // row of each sorted A element
    bool batch = false;
    uint32_t nitems = 1;
    uint32_t* row_first = nullptr;        // device [nitems + 1]: item i owns rows [row_first[i], row_first[i+1])
    std::vector<uint32_t> h_row_first;    // host copy
    std::vector<uint32_t> colbase;        // first global column of each item (nitems + 1 entries)
    ItemOut* item_out = nullptr;          // device [nitems], filled per wave
    // per-item statistics for the sizer's features (batches; device arrays)
    const uint64_t* b_off = nullptr;      // [nitems + 1] first B nonzero of each item
    const uint32_t* col_first = nullptr;  // [nitems + 1] first global column
    const uint32_t* fib_first = nullptr;  // [nitems + 1] first fiber
    const uint32_t* col_run = nullptr;    // [global columns + 1] B nonzeros before each column
    uint64_t ncols_global = 0;
};

// Tuning knobs (the autotuner's search space), resolved from the options.
struct Knobs {
    uint32_t small_max;     // products of the largest row on the one-warp accumulator
    uint32_t esc_avg;       // sort-based rows: fewer products per A nonzero than this on average
    double max_load;        // cuckoo table load factor
    uint32_t max_chain;     // cuckoo eviction chain bound
    uint32_t max_attempts;  // cuckoo builds tried
};

Knobs knobs_of(const ptc_options& opt) {
    Knobs k;
    k.small_max = std::min(opt.small_max_products ? opt.small_max_products : kSmallMaxProducts, small_row_max_flops());
    k.esc_avg = opt.sort_max_avg_products ? opt.sort_max_avg_products : kEscMaxAvgProducts;
    k.max_load = opt.hash_load_pct ? std::min(std::max(opt.hash_load_pct, 10u), 90u) / 100.0 : 0.75;
    k.max_chain = opt.cuckoo_max_chain;
    k.max_attempts = opt.cuckoo_max_attempts ? opt.cuckoo_max_attempts : kCuckooMaxAttempts;
    return k;
}

// The row classes, the sizes and the work items of one contraction or batch.
struct Plan {
    bool learned = false;
    uint64_t flops = 0;
    uint32_t W = 0, log2w = 0, P = 1;
    uint64_t* row_flops = nullptr;
    uint32_t n_small = 0, n_big = 0, n_esc = 0;
    uint32_t* small_rows = nullptr;  // in row order
    uint32_t* big_rows = nullptr;    // largest first
    uint32_t* esc_rows = nullptr;    // in row order
    uint32_t* small_pos = nullptr;   // [nrows + 1] small rows before each row
    uint32_t* esc_pos = nullptr;     // [nrows + 1] sort-based rows before each row
    // sort-based rows: runs of equal (row, column) in the sorted products
    uint64_t esc_runs = 0;
    uint32_t esc_colbits = 0;
    uint64_t* esc_run_key = nullptr;
    uint32_t* esc_run_start = nullptr;
    uint32_t* esc_first = nullptr;  // [n_esc + 1] first run of each sort-based row
    uint32_t* esc_long = nullptr;   // the runs of at least kEscLongMin products, increasing
    std::vector<uint32_t> h_esc_long;
    double* esc_sorted = nullptr;   // products in run order
    // sizes: exact offsets of the small and sort-based rows (and, on the two-phase path, of every
    // row); the learned path's large rows claim instead, within claim_off's budgets
    uint64_t* row_off = nullptr;
    uint64_t* claim_off = nullptr;
    uint64_t exact_nnz = 0, claim_total = 0;
    float* pred = nullptr;
    // work items of the large rows: [0] warp tasks (rows with at most kWarpTaskMaxLen A nonzeros,
    // big_rows[0, n_warp_rows)), [1] block parts (the others)
    uint32_t n_warp_rows = 0;
    SplitRule rule[2]{};
    PartItem* parts[2] = {nullptr, nullptr};
    uint32_t n_parts[2] = {0, 0};
    uint32_t* work_counter = nullptr;
    uint32_t* work_counter2 = nullptr;  // the block parts' counter (they can run beside the warp tasks)
    // collision-free large rows (two-phase path): written product by product, in row order
    uint64_t* alen = nullptr;        // exclusive scan of the A nonzeros' fiber lengths
    uint32_t* copy_rows = nullptr;
    uint64_t* copy_keys = nullptr;   // the same row ids as sort keys (wave slices)
    uint32_t n_copy = 0;
    bool collected = false;
    // large rows of a single contraction on the row bitmap kernel (instead of parts): the rows
    // it writes, heaviest first (the two-phase path leaves the collision-free rows to copy_rows)
    bool rowmap = false;      // every large row is on the row bitmap kernel (no panels at all)
    uint32_t n_mapped = 0;    // big_rows[0, n_mapped): the large rows on the row bitmap kernel
    uint32_t* map_rows = nullptr;
    uint32_t n_map = 0;
};

// One kind of work item and its accumulator kernel.
void launch_parts(int kind, const Operands& op, const PartItem* parts, uint32_t n, const OutputView& out,
                  uint32_t* work_counter, uint32_t* err, int num_sms, cudaStream_t st) {
    if (kind == 0) launch_warp_tasks(op, parts, n, out, work_counter, err, num_sms, st);
    else launch_hash_parts(op, parts, n, out, work_counter, err, num_sms, st);
}

Plan plan_rows(Front& F, const ptc_options& opt, const SizerHost* sizer, Collect* collect, int num_sms, Arena& ar,
               ptc_stats& stats) {
    cudaStream_t st = ar.stream();
    Operands& op = F.op;
    const uint64_t na = op.na, nb = op.nb, nrows = op.nrows, ncols = op.ncols, nfib = op.nfib;
    const Knobs kn = knobs_of(opt);
    Plan pl;
    pl.learned = sizer != nullptr;

    // flops per row
    uint64_t* alen = ar.alloc<uint64_t>(na + 1);
    launch_fiber_len(op.a_fib, op.fib_start, na, alen, st);
    exclusive_scan<uint64_t>(alen, alen, na, ar);
    pl.row_flops = ar.alloc<uint64_t>(std::max<uint64_t>(nrows, 1));
    launch_row_flops(alen, op.row_start, nrows, pl.row_flops, st);
    pl.alen = alen;
    pl.flops = read_scalar(alen + na, st);
    stats.mult_adds = pl.flops;
    stats.nrows = nrows;
    stats.nfibers = nfib;
    if (pl.flops == 0) return pl;

    // row classes and work lists (largest rows first)
    uint32_t* small_flag = ar.alloc<uint32_t>(nrows + 1);
    uint32_t* big_flag = ar.alloc<uint32_t>(nrows + 1);
    uint32_t* esc_flag = ar.alloc<uint32_t>(nrows + 1);
    launch_classify_rows(pl.row_flops, op.row_start, nrows, kn.small_max, kn.esc_avg, small_flag, big_flag, esc_flag,
                         st);
    pl.esc_pos = ar.alloc<uint32_t>(nrows + 1);
    exclusive_scan<uint32_t>(esc_flag, pl.esc_pos, nrows, ar);
    pl.n_esc = read_scalar(pl.esc_pos + nrows, st);
    pl.esc_rows = ar.alloc<uint32_t>(pl.n_esc);
    launch_compact_indices(esc_flag, pl.esc_pos, nrows, pl.esc_rows, st);
    uint64_t* esc_off = ar.alloc<uint64_t>((uint64_t)pl.n_esc + 1);
    uint64_t f_esc = 0;
    const int colbits = bits_for_space(std::max<uint64_t>(ncols, 1));
    if (pl.n_esc > 0) {
        launch_esc_len(pl.esc_rows, pl.n_esc, pl.row_flops, esc_off, st);
        exclusive_scan<uint64_t>(esc_off, esc_off, pl.n_esc, ar);
        f_esc = read_scalar(esc_off + pl.n_esc, st);
        if (f_esc > kEscMaxProducts || bits_for_space((uint64_t)pl.n_esc) + colbits > 64) {
            // too large for the sort buffers: hash path
            launch_merge_flags(big_flag, esc_flag, nrows, st);
            PTC_CUDA(cudaMemsetAsync(pl.esc_pos, 0, (nrows + 1) * sizeof(uint32_t), st));
            pl.n_esc = 0;
            f_esc = 0;
        }
    }
    pl.small_pos = ar.alloc<uint32_t>(nrows + 1);
    uint32_t* big_pos = ar.alloc<uint32_t>(nrows + 1);
    exclusive_scan<uint32_t>(small_flag, pl.small_pos, nrows, ar);
    exclusive_scan<uint32_t>(big_flag, big_pos, nrows, ar);
    pl.n_small = read_scalar(pl.small_pos + nrows, st);
    pl.n_big = read_scalar(big_pos + nrows, st);
    pl.small_rows = ar.alloc<uint32_t>(pl.n_small);
    pl.big_rows = ar.alloc<uint32_t>(pl.n_big);
    launch_compact_indices(small_flag, pl.small_pos, nrows, pl.small_rows, st);
    launch_compact_indices(big_flag, big_pos, nrows, pl.big_rows, st);
    const uint32_t n_small = pl.n_small, n_big = pl.n_big, n_esc = pl.n_esc;
    // large rows, three groups, each largest first: the row bitmap kernel takes rows of at most
    // map_len A nonzeros (its barrier rounds, one per A nonzero, stay few), when the columns fit
    // its bitmap (a batch's columns are its items' own: the widest item decides); warp tasks the
    // next rows up to warp_len A nonzeros (panels of at most a dense warp task's width); block
    // parts the others
    const bool bitmap_ok = opt.large_rows != PTC_LARGE_ROWS_PANELS && ncols <= rowmap_max_cols();
    PTC_REQUIRE(!(opt.large_rows == PTC_LARGE_ROWS_BITMAP && !bitmap_ok), PTC_ERR_INVALID_ARGUMENT,
                "large_rows = PTC_LARGE_ROWS_BITMAP: at most about 600k distinct B free keys per contraction");
    const uint32_t map_len = !bitmap_ok ? 0u
                             : opt.large_rows == PTC_LARGE_ROWS_BITMAP ? UINT32_MAX
                             : opt.bitmap_max_len;
    const uint32_t warp_len = (opt.panel_width == 0 || opt.panel_width <= warp_task_dense_columns())
                                  ? (opt.warp_task_max_len ? opt.warp_task_max_len : kWarpTaskMaxLen) : 0u;
    if (n_big > 0) {
        uint64_t* wkey = ar.alloc<uint64_t>(n_big);
        launch_work_keys(pl.big_rows, n_big, pl.row_flops, op.row_start, map_len, warp_len, wkey, st);
        if (n_big > 1) radix_sort_pairs(wkey, pl.big_rows, n_big, 0, 42, ar);
        const uint64_t split[2] = {1ull << 40, 2ull << 40};
        uint64_t* split_d = ar.alloc<uint64_t>(2);
        uint32_t* first = ar.alloc<uint32_t>(3);
        PTC_CUDA(cudaMemcpyAsync(split_d, split, 2 * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
        launch_key_bounds(wkey, n_big, split_d, 2, first, st);
        uint32_t hf[2];
        PTC_CUDA(cudaMemcpyAsync(hf, first, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        PTC_CUDA(cudaStreamSynchronize(st));
        pl.n_mapped = hf[0];
        pl.n_warp_rows = hf[1] - hf[0];
    }
    pl.rowmap = n_big > 0 && pl.n_mapped == n_big;
    stats.rows_small = n_small;
    stats.rows_hash = n_big;
    stats.rows_long = n_esc;

    // fine column panels: B fibers are split at multiples of W so a row can be cut into parts
    // that each fit one shared-memory table (W <= table capacity, so a part always fits).  The
    // per-fiber panel table is built when it fits kPanelTableBytes (else binary searches in the
    // fiber find a part's entries).
    auto table_bytes = [&](uint32_t w) { return nfib * ((ncols + w - 1) / w + 1) * 4; };
    uint32_t W = opt.panel_width;
    // a batch's large rows each have their own item's panels: per-row panel counts
    std::vector<uint32_t> item_cols_h;
    if (F.batch) {
        item_cols_h.resize(F.nitems);
        for (uint32_t i = 0; i < F.nitems; ++i) item_cols_h[i] = F.colbase[i + 1] - F.colbase[i];
    }
    auto panel_entries = [&](uint32_t w) {  // panel counters of the large rows (an upper bound for a batch)
        if (!F.batch) return (uint64_t)n_big * ((ncols + w - 1) / w);
        uint64_t e = 0;
        for (uint32_t i = 0; i < F.nitems; ++i)
            e += (uint64_t)(F.h_row_first[i + 1] - F.h_row_first[i]) * std::max<uint64_t>(1, (item_cols_h[i] + w - 1) / w);
        return e;
    };
    if (pl.rowmap) {
        // the row bitmap kernel needs no panels: one panel spans every column (the sizer's
        // popularity table then has a single panel)
        W = 1;
        while ((uint64_t)W < ncols) W <<= 1;
    } else if (W == 0) {  // at most 256 columns (a third of a dense warp task), wider for small tables
        W = 32;
        while (W < 256 && (uint64_t)W * 16 < ncols) W <<= 1;
        // wider panels for big tables, but never wider than a dense warp task (a single panel
        // above a sparse task's capacity becomes a dense task over that panel)
        while (2 * W <= warp_task_dense_columns() && panel_entries(W) * 4 > (2ull << 30)) W <<= 1;
    }
    PTC_REQUIRE(pl.rowmap || W <= dense_part_columns(), PTC_ERR_INVALID_ARGUMENT, "panel_width larger than a hash part");
    pl.W = W;
    pl.log2w = floor_log2(W);
    pl.P = (uint32_t)std::max<uint64_t>(1, (ncols + W - 1) / W);
    const uint32_t P = pl.P;
    stats.panel_width = pl.rowmap ? 0 : W;
    uint32_t* panel_off = nullptr;
    // only the panel kernels read the table: none when no large row goes to them
    if (P > 1 && n_big > pl.n_mapped && table_bytes(W) <= kPanelTableBytes) {
        panel_off = ar.alloc<uint32_t>(nfib * (uint64_t)(P + 1));
        launch_panel_offsets(op.b_col, op.fib_start, nfib, P, pl.log2w, panel_off, st);
    }
    op.panel_off = panel_off;
    op.npanels = P;
    op.panel_log2 = pl.log2w;


    SplitRule& wr = pl.rule[0];  // warp tasks
    wr.cap = warp_task_capacity();
    wr.dense_panels = warp_task_dense_columns() >> pl.log2w;
    wr.dense_min = std::max(1u, W / 6);
    wr.min_bits = warp_task_min_bits();
    wr.max_bits = warp_task_max_bits();
    wr.oversize_dense = 1;
    wr.load_num = 1;
    wr.load_den = 2;
    SplitRule& br = pl.rule[1];  // block parts
    br.cap = hash_part_capacity();
    br.dense_panels = dense_part_columns() >> pl.log2w;
    br.dense_min = W / kDenseMinFraction;
    br.min_bits = hash_part_min_bits();
    br.max_bits = 12;
    br.oversize_dense = 1;  // a panel above the capacity: a dense part over it
    br.load_num = 3;
    br.load_den = 4;
    if (pl.learned) {  // predicted sizes: every open-addressing table at its largest, for slack
        wr.min_bits = wr.max_bits;
        br.min_bits = br.max_bits;
    }

    // symbolic: exact output nnz of the small rows (both paths) and of the large rows (per fine
    // panel; two-phase path only -- the learned path predicts those)
    uint64_t* row_d = ar.alloc<uint64_t>(nrows + 1);
    PTC_CUDA(cudaMemsetAsync(row_d, 0, (nrows + 1) * sizeof(uint64_t), st));
    const uint64_t* pbase = nullptr;  // per-row panel offsets (batches; null: row i at i * P)
    const uint32_t* item_cols = nullptr;
    uint64_t n_panel_cnt = (uint64_t)n_big * P;
    if (F.batch) {
        uint32_t* ic = ar.alloc<uint32_t>(F.nitems);
        PTC_CUDA(cudaMemcpyAsync(ic, item_cols_h.data(), F.nitems * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        item_cols = ic;
        op.item_cols = ic;
        uint64_t* pb = ar.alloc<uint64_t>((uint64_t)n_big + 1);
        launch_row_panel_counts(pl.big_rows, n_big, op.row_item, item_cols, pl.log2w, pb, st);
        exclusive_scan<uint64_t>(pb, pb, n_big, ar);
        n_panel_cnt = read_scalar(pb + n_big, st);  // also orders the copy of item_cols_h
        pbase = pb;
    }
    uint32_t* panel_cnt = ar.alloc<uint32_t>(std::max<uint64_t>(n_panel_cnt, 1));
    pl.work_counter = ar.alloc<uint32_t>(1);
    pl.work_counter2 = ar.alloc<uint32_t>(1);
    OutputView none;
    launch_small_rows(false, op, pl.small_rows, n_small, row_d, nullptr, none, st);
    if (!pl.learned) {
        const uint32_t nm = pl.n_mapped;
        launch_rowmap(kRowmapCount, op, pl.big_rows, nm, row_d, nullptr, none, pl.work_counter, num_sms, st);
        exact_panel_counts(op, pl.big_rows + nm, n_big - nm, pbase ? panel_cnt : panel_cnt + (uint64_t)nm * P,
                           pbase ? pbase + nm : nullptr, row_d, pl.work_counter, num_sms, st);
    }
    // sort-based rows: expand their products in stream order, sort stably by (row, column)
    pl.esc_colbits = (uint32_t)colbits;
    if (n_esc > 0) {
        int32_t* esc_of = ar.alloc<int32_t>(nrows);
        PTC_CUDA(cudaMemsetAsync(esc_of, 0xff, nrows * sizeof(int32_t), st));
        launch_esc_index(pl.esc_rows, n_esc, esc_of, st);
        uint64_t* esc_key = ar.alloc<uint64_t>(f_esc);
        double* esc_val = ar.alloc<double>(f_esc);
        uint32_t* esc_perm = ar.alloc<uint32_t>(f_esc);
        launch_esc_expand(op, F.a_row, esc_of, alen, esc_off, pl.esc_colbits, esc_key, esc_val, esc_perm, st);
        radix_sort_pairs(esc_key, esc_perm, f_esc, 0, pl.esc_colbits + bits_for_space((uint64_t)n_esc), ar);
        pl.esc_run_start = ar.alloc<uint32_t>(f_esc + 1);
        pl.esc_run_key = ar.alloc<uint64_t>(f_esc);
        pl.esc_runs = runs_of_sorted(esc_key, f_esc, nullptr, pl.esc_run_start, pl.esc_run_key, ar);
        pl.esc_first = ar.alloc<uint32_t>((uint64_t)n_esc + 1);
        launch_esc_count(pl.esc_run_key, pl.esc_runs, pl.esc_colbits, pl.esc_rows, row_d, pl.esc_first, st);
        {  // long runs: folded a block each
            uint32_t* flag = ar.alloc<uint32_t>(pl.esc_runs + 1);
            uint32_t* pos = ar.alloc<uint32_t>(pl.esc_runs + 1);
            launch_esc_long_flags(pl.esc_run_start, pl.esc_runs, flag, st);
            exclusive_scan<uint32_t>(flag, pos, pl.esc_runs, ar);
            const uint32_t nl = read_scalar(pos + pl.esc_runs, st);
            if (nl > 0) {
                pl.esc_long = ar.alloc<uint32_t>(nl);
                launch_compact_indices(flag, pos, pl.esc_runs, pl.esc_long, st);
                pl.h_esc_long.resize(nl);
                PTC_CUDA(cudaMemcpyAsync(pl.h_esc_long.data(), pl.esc_long, nl * sizeof(uint32_t),
                                         cudaMemcpyDeviceToHost, st));
                PTC_CUDA(cudaStreamSynchronize(st));
            }
        }
        const uint32_t total_runs = (uint32_t)pl.esc_runs;
        PTC_CUDA(cudaMemcpyAsync(pl.esc_first + n_esc, &total_runs, sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        // the products in run order (the sort keys are no longer needed: their buffer takes them)
        pl.esc_sorted = reinterpret_cast<double*>(esc_key);
        launch_esc_gather(esc_perm, esc_val, f_esc, pl.esc_sorted, st);
    }
    pl.row_off = ar.alloc<uint64_t>(nrows + 1);
    exclusive_scan<uint64_t>(row_d, pl.row_off, nrows, ar);
    pl.exact_nnz = read_scalar(pl.row_off + nrows, st);

    if (collect) {
        // features of the rows the learned path sizes, and log2(1 + their exact output nnz)
        float* gp = ar.alloc<float>((uint64_t)(P + 1) * kGridPoints);
        launch_popularity_table(op.b_col, nb, ncols, P, pl.log2w, gp, ar);
        float* fx = ar.alloc<float>((uint64_t)n_big * kSizerInputs);
        float* ft = ar.alloc<float>(n_big);
        launch_row_features(op, pl.big_rows, n_big, pl.row_flops, gp, fx, st);
        launch_row_targets(pl.big_rows, n_big, row_d, ft, st);
        collect->x.resize((uint64_t)n_big * kSizerInputs);
        collect->t.resize(n_big);
        PTC_CUDA(cudaMemcpyAsync(collect->x.data(), fx, collect->x.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
        PTC_CUDA(cudaMemcpyAsync(collect->t.data(), ft, collect->t.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
        PTC_CUDA(cudaStreamSynchronize(st));
        pl.collected = true;
        return pl;
    }

    if (pl.learned) {
        pl.claim_off = ar.alloc<uint64_t>(nrows + 1);
        PTC_CUDA(cudaMemsetAsync(pl.claim_off, 0, (nrows + 1) * sizeof(uint64_t), st));
        if (n_big > 0) {
            // sizer: per-row features -> predicted log2(1 + nnz) -> per-panel counts by column popularity
            // (a batch uses its items' own tables below instead of one over the whole batch)
            float* gp = nullptr;
            if (!F.batch) {
                gp = ar.alloc<float>((uint64_t)(P + 1) * kGridPoints);
                launch_popularity_table(op.b_col, nb, ncols, P, pl.log2w, gp, ar);
            }
            // a batch row gets its own item's statistics (the features a single contraction of
            // that item gives, which the sizer was trained on)
            ItemStats is;
            if (F.batch) {
                is.nitems = F.nitems;
                is.b_off = F.b_off;
                is.col_first = F.col_first;
                is.fib_first = F.fib_first;
                is.row_first = F.row_first;
                is.col_run = F.col_run;
                is.gtot = ar.alloc<float>((uint64_t)F.nitems * kGridPoints);
                std::vector<uint64_t> ipb(F.nitems + 1, 0);
                for (uint32_t i = 0; i < F.nitems; ++i)
                    ipb[i + 1] = ipb[i] + std::max<uint64_t>(1, (item_cols_h[i] + W - 1) / W);
                uint64_t* ipb_d = ar.alloc<uint64_t>(F.nitems + 1);
                PTC_CUDA(cudaMemcpyAsync(ipb_d, ipb.data(), ipb.size() * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
                is.item_pb = ipb_d;
                is.pmass = ar.alloc<uint32_t>(std::max<uint64_t>(ipb[F.nitems], 1));
                PTC_CUDA(cudaMemsetAsync(is.pmass, 0, std::max<uint64_t>(ipb[F.nitems], 1) * sizeof(uint32_t), st));
                launch_item_popularity(is, F.ncols_global, pl.log2w, ar);
                PTC_CUDA(cudaStreamSynchronize(st));  // ipb (host) stays alive until the copy is done
            }
            float* fx = ar.alloc<float>((uint64_t)n_big * kSizerInputs);
            launch_row_features(op, pl.big_rows, n_big, pl.row_flops, gp, fx, st, F.batch ? &is : nullptr);
            pl.pred = ar.alloc<float>(n_big);
            sizer_predict_device(*sizer, fx, n_big, pl.pred, ar);
            launch_predicted_panel_counts(pl.big_rows, n_big, pl.row_flops, pl.pred, gp, op.row_item, item_cols,
                                          pbase, P, pl.log2w, ncols, F.batch ? kSizerBatchMargin : kSizerMargin,
                                          panel_cnt, ar,
                                          F.batch ? &is : nullptr);
            launch_claim_budgets(pl.big_rows, n_big, panel_cnt, pbase, P, pl.claim_off, st);
        }
        exclusive_scan<uint64_t>(pl.claim_off, pl.claim_off, nrows, ar);
        pl.claim_total = read_scalar(pl.claim_off + nrows, st);
    }

    // exact sizes: the collision-free large rows need no table (launch_copy_rows)
    const uint64_t* skip_off = pl.learned ? nullptr : pl.row_off;
    const uint64_t* skip_flops = pl.learned ? nullptr : pl.row_flops;
    if (!pl.learned && n_big > 0) {
        uint32_t* flag = ar.alloc<uint32_t>((uint64_t)n_big + 1);
        uint32_t* pos = ar.alloc<uint32_t>((uint64_t)n_big + 1);
        launch_copy_flags(pl.big_rows, n_big, pl.row_off, pl.row_flops, flag, st);
        exclusive_scan<uint32_t>(flag, pos, n_big, ar);
        pl.n_copy = read_scalar(pos + n_big, st);
        if (pl.n_copy > 0) {
            uint32_t* sel = ar.alloc<uint32_t>(pl.n_copy);
            launch_compact_indices(flag, pos, n_big, sel, st);  // positions in big_rows
            pl.copy_rows = ar.alloc<uint32_t>(pl.n_copy);
            launch_gather<uint32_t>(pl.big_rows, sel, pl.n_copy, pl.copy_rows, st);
            pl.copy_keys = ar.alloc<uint64_t>(pl.n_copy);
            launch_row_keys(pl.copy_rows, pl.n_copy, pl.copy_keys, st);
            radix_sort_pairs(pl.copy_keys, pl.copy_rows, pl.n_copy, 0, bits_for_space(nrows), ar);
        }
    }

    {
        // the rows the bitmap kernel writes: its large rows but the collision-free ones, in
        // big_rows' heaviest-first order
        const uint32_t nm = pl.n_mapped;
        pl.map_rows = pl.big_rows;
        pl.n_map = nm;
        if (skip_off && nm > 0 && pl.n_copy > 0) {
            uint32_t* flag = ar.alloc<uint32_t>((uint64_t)nm + 1);
            uint32_t* pos = ar.alloc<uint32_t>((uint64_t)nm + 1);
            launch_table_row_flags(pl.big_rows, nm, skip_off, skip_flops, flag, st);
            exclusive_scan<uint32_t>(flag, pos, nm, ar);
            pl.n_map = read_scalar(pos + nm, st);
            uint32_t* sel = ar.alloc<uint32_t>(std::max<uint32_t>(pl.n_map, 1));
            launch_compact_indices(flag, pos, nm, sel, st);
            pl.map_rows = ar.alloc<uint32_t>(std::max<uint32_t>(pl.n_map, 1));
            launch_gather<uint32_t>(pl.big_rows, sel, pl.n_map, pl.map_rows, st);
        }
    }
    if (pl.rowmap) {
        stats.hash_parts = 0;
        return pl;
    }

    // split the other large rows into tasks / parts that fit a shared-memory table
    for (int kind = 0; kind < 2; ++kind) {
        const uint64_t r0 = kind == 0 ? pl.n_mapped : pl.n_mapped + pl.n_warp_rows;
        const uint64_t nr = kind == 0 ? pl.n_warp_rows : n_big - r0;
        uint32_t* nparts = ar.alloc<uint32_t>(nr + 1);
        const uint32_t* pc = pbase ? panel_cnt : panel_cnt + r0 * P;
        const uint64_t* pb = pbase ? pbase + r0 : nullptr;
        launch_count_parts(pl.big_rows + r0, pc, pb, nr, P, pl.rule[kind], skip_off, skip_flops, nparts, op.err, st);
        exclusive_scan<uint32_t>(nparts, nparts, nr, ar);
        pl.n_parts[kind] = read_scalar(nparts + nr, st);
        PTC_REQUIRE(read_scalar(op.err, st) == 0, PTC_ERR_INTERNAL, "a fine panel exceeds the hash part capacity");
        pl.parts[kind] = ar.alloc<PartItem>(pl.n_parts[kind]);
        launch_fill_parts(pl.big_rows + r0, pc, pb, nr, P, pl.rule[kind], nparts, pl.learned ? nullptr : pl.row_off,
                          skip_flops, pl.parts[kind], st);
    }
    stats.hash_parts = pl.n_parts[0] + pl.n_parts[1];
    return pl;
}

// ---------------------------------------------------------------------------------------------
// single contraction
// ---------------------------------------------------------------------------------------------

Front front_single(const ptc_coo* A, const ptc_coo* B, bool self, uint32_t c, const uint32_t* a_modes,
                   const uint32_t* b_modes, const ptc_options& opt, const Knobs& kn, Arena& ar, Events& ev,
                   ptc_stats& stats) {
    cudaStream_t st = ar.stream();
    const uint32_t fa = A->order - c, fb = B->order - c;
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
    Fibers fib = group_fibers(b_ckey, cols.rank_of, ncols, nb, bits_for_space(b_con.space), dB.vals, ar);
    CuckooBuildInfo cinfo;
    const CuckooTable table = cuckoo_build(fib.key, fib.n, opt.hash_seed, kn.max_chain, kn.max_load, kn.max_attempts, ar, &cinfo);
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
    uint64_t* a_ckey_sorted = ar.alloc<uint64_t>(na);
    double* a_val = ar.alloc<double>(na);
    launch_gather<uint64_t>(a_ckey, rows.perm, na, a_ckey_sorted, st);
    launch_gather<double>(dA.vals, rows.perm, na, a_val, st);
    int32_t* a_fib = ar.alloc<int32_t>(na);
    cuckoo_lookup(table, a_ckey_sorted, na, a_fib, ar);
    PTC_CUDA(cudaEventRecord(ev.ev[EV_ASIDE], st));

    Front F;
    Operands& op = F.op;
    op.na = na; op.nb = nb; op.nrows = rows.nruns; op.ncols = ncols; op.nfib = fib.n;
    op.fa = fa; op.fb = fb;
    op.a_val = a_val; op.a_fib = a_fib; op.row_start = rows.run_start;
    op.b_col = fib.col; op.b_val = fib.val; op.fib_start = fib.start;
    op.row_tuple = row_tuple; op.col_tuple = col_tuple;
    op.err = err;
    F.a_row = rows.run_of;
    F.h_row_first = {0u, (uint32_t)rows.nruns};
    F.row_first = ar.alloc<uint32_t>(2);
    PTC_CUDA(cudaMemcpyAsync(F.row_first, F.h_row_first.data(), 2 * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    F.colbase = {0u, (uint32_t)ncols};
    stats.ncols = ncols;
    return F;
}

void contract_impl(const ptc_coo* A, const ptc_coo* Bin, uint32_t c, const uint32_t* a_modes,
                   const uint32_t* b_modes_in, const ptc_options* opt_in, ptc_tensor* out, ptc_stats* stats_out,
                   Collect* collect = nullptr) {
    const ptc_options opt = resolve_options(opt_in);
    PTC_REQUIRE(out != nullptr, PTC_ERR_INVALID_ARGUMENT, "out is null");
    std::memset(out, 0, sizeof(*out));
    ptc_stats stats;
    std::memset(&stats, 0, sizeof(stats));
    g_launches = 0;

    const bool self = (Bin == nullptr);
    const ptc_coo* B = self ? A : Bin;
    const uint32_t* b_modes = self ? a_modes : b_modes_in;
    validate_pair(A, B, c, a_modes, b_modes, "");
    if (self) PTC_REQUIRE(A->nnz > 1, PTC_ERR_TOO_FEW_NONZEROS, "Tensor B has at most one nonzeros");
    const uint32_t fa = A->order - c, fb = B->order - c;

    DeviceSetup dev = setup_device(opt);
    cudaStream_t st = dev.stream;
    Events ev;
    Arena ar(st);
    PTC_CUDA(cudaEventRecord(ev.ev[EV_START], st));
    const Knobs kn = knobs_of(opt);
    Front F = front_single(A, B, self, c, a_modes, b_modes, opt, kn, ar, ev, stats);

    // the canonical order (sort_rows) runs on exact offsets: the two-phase path
    const bool learned = opt.path == PTC_PATH_LEARNED && collect == nullptr && !opt.sort_rows;
    const SizerHost* sizer = nullptr;
    if (learned) {
        sizer = opt.sizer ? sizer_host(opt.sizer) : default_sizer();
        PTC_REQUIRE(sizer != nullptr, PTC_ERR_INVALID_ARGUMENT,
                    "the learned path needs a sizer: opt.sizer, or sizer_default.bin beside the library");
    }
    Plan pl = plan_rows(F, opt, sizer, collect, dev.num_sms, ar, stats);
    PTC_REQUIRE(pl.flops > 0, PTC_ERR_EMPTY_CONTRACTION, "tensor contraction not possible!! (no matching fibers)");
    if (pl.collected) {
        ar.release();
        PTC_CUDA(cudaStreamSynchronize(st));
        stats.out_nnz = pl.exact_nnz;
        if (stats_out) *stats_out = stats;
        return;
    }
    PTC_CUDA(cudaEventRecord(ev.ev[EV_SYM], st));
    const Operands& op = F.op;

    // ---- numeric ----
    const uint32_t od = fa + fb;
    const uint64_t capacity = learned ? pl.exact_nnz + pl.claim_total + 1024 : pl.exact_nnz;
    OutputView ov;
    PTC_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&ov.idx), std::max<uint64_t>(capacity * od, 1) * sizeof(uint32_t), st));
    PTC_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&ov.val), std::max<uint64_t>(capacity, 1) * sizeof(double), st));
    uint64_t out_nnz = pl.exact_nnz;
    if (opt.sort_rows) {  // canonical order: remember every entry's row and column
        ov.row_of = ar.alloc<uint32_t>(std::max<uint64_t>(capacity, 1));
        ov.col_of = ar.alloc<uint32_t>(std::max<uint64_t>(capacity, 1));
    }
    try {
        if (learned) {
            // the small and sort-based rows fill [0, exact_nnz); the large rows claim after them
            ov.capacity = capacity;
            ov.cursor = ar.alloc<uint64_t>(1);
            ov.overshoot = ar.alloc<uint64_t>(1);
            PTC_CUDA(cudaMemcpyAsync(ov.cursor, &pl.exact_nnz, sizeof(uint64_t), cudaMemcpyHostToDevice, st));
            PTC_CUDA(cudaMemsetAsync(ov.overshoot, 0, sizeof(uint64_t), st));
        }
        std::vector<Launched> groups;
        launch_small_rows(true, op, pl.small_rows, pl.n_small, nullptr, pl.row_off, ov, st);
        launch_copy_rows(op, pl.copy_rows, pl.n_copy, pl.alen, pl.row_off, ov, dev.num_sms, st);
        OutputView mo = ov;  // the row bitmap kernel's view (claim bookkeeping on the learned path)
        if (pl.n_map > 0) {
            if (learned) {
                const uint32_t n = std::max<uint32_t>(pl.n_map, 1);
                mo.fail_count = ar.alloc<uint32_t>(1);
                mo.fail_list = ar.alloc<uint32_t>(n);
                mo.item_count = ar.alloc<uint32_t>(n);
                PTC_CUDA(cudaMemsetAsync(mo.fail_count, 0, sizeof(uint32_t), st));
            }
            launch_rowmap(learned ? kRowmapClaim : kRowmapExact, op, pl.map_rows, pl.n_map, nullptr, pl.row_off, mo,
                          pl.work_counter, dev.num_sms, st);
        }
        OutputView ok[2] = {ov, ov};
        for (int kind = 0; kind < 2; ++kind) {
            if (learned) {
                const uint32_t n = std::max<uint32_t>(pl.n_parts[kind], 1);
                ok[kind].fail_count = ar.alloc<uint32_t>(1);
                ok[kind].fail_list = ar.alloc<uint32_t>(n);
                ok[kind].item_count = ar.alloc<uint32_t>(n);
                PTC_CUDA(cudaMemsetAsync(ok[kind].fail_count, 0, sizeof(uint32_t), st));
                groups.push_back({kind, pl.parts[kind], pl.n_parts[kind], ok[kind].fail_list, ok[kind].fail_count,
                                  ok[kind].item_count});
            }
        }
        // the block parts (a tail of a few heavy rows) and the sort-based folds run beside the warp
        // tasks: they write disjoint output ranges
        AuxStreams& aux = aux_streams(dev.device);
        aux.fork(st);
        launch_parts(1, op, pl.parts[1], pl.n_parts[1], ok[1], pl.work_counter2, op.err, dev.num_sms, aux.s[0]);
        launch_esc_fold(op, ov, pl.esc_run_key, pl.esc_run_start, 0, pl.esc_runs, pl.esc_colbits, pl.esc_rows,
                        pl.esc_first, pl.row_off, pl.esc_sorted, pl.esc_long,
                        (uint32_t)pl.h_esc_long.size(), aux.s[1]);
        launch_parts(0, op, pl.parts[0], pl.n_parts[0], ok[0], pl.work_counter, op.err, dev.num_sms, st);
        aux.join(st);
        if (learned) {
            // rows whose prediction fell short run again exactly (parts first, then the bitmap
            // kernel's rows; each grows the output as needed), and the sizer's error over the large
            // rows, every one of whose exact counts is known by now
            uint64_t* row_actual = ar.alloc<uint64_t>(std::max<uint64_t>(op.nrows, 1));
            PTC_CUDA(cudaMemsetAsync(row_actual, 0, std::max<uint64_t>(op.nrows, 1) * sizeof(uint64_t), st));
            stats.rerun_rows = learned_reruns(op, groups, pl.rule[1], ov, pl.work_counter, op.err, dev.num_sms,
                                              op.nrows, row_actual, ar);
            if (pl.n_map > 0)
                stats.rerun_rows += rowmap_reruns(op, pl.map_rows, pl.n_map, mo, ov, pl.work_counter, dev.num_sms,
                                                  row_actual, ar);
            double* esum = ar.alloc<double>(1);
            launch_log2_error(pl.big_rows, pl.n_big, pl.pred, row_actual, esum, st);
            stats.sizer_mean_abs_log2_err = pl.n_big ? read_scalar(esum, st) / pl.n_big : 0.0;
            out_nnz = read_scalar(ov.cursor, st) - read_scalar(ov.overshoot, st);
        }
        if (opt.sort_rows && out_nnz > 1) {
            // rows in increasing free-key order, every row in increasing column order: one sort
            // of the entries by (row, column), then the tuples and values follow the permutation
            const uint32_t colbits = (uint32_t)bits_for_space(std::max<uint64_t>(op.ncols, 1));
            const int keybits = (int)colbits + bits_for_space(std::max<uint64_t>(op.nrows, 1));
            uint64_t* key = ar.alloc<uint64_t>(out_nnz);
            uint32_t* perm = ar.alloc<uint32_t>(out_nnz);
            launch_entry_keys(ov.row_of, ov.col_of, out_nnz, colbits, key, perm, st);
            radix_sort_pairs(key, perm, out_nnz, 0, keybits, ar);
            uint32_t* idx2 = nullptr;
            double* val2 = nullptr;
            PTC_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&idx2), out_nnz * od * sizeof(uint32_t), st));
            PTC_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&val2), out_nnz * sizeof(double), st));
            launch_gather_tuples(ov.idx, perm, out_nnz, od, idx2, st);
            launch_gather<double>(ov.val, perm, out_nnz, val2, st);
            PTC_CUDA(cudaFreeAsync(ov.idx, st));
            PTC_CUDA(cudaFreeAsync(ov.val, st));
            ov.idx = idx2;
            ov.val = val2;
        }
        PTC_CUDA(cudaEventRecord(ev.ev[EV_NUM], st));
        PTC_REQUIRE(read_scalar(op.err, st) == 0, PTC_ERR_INTERNAL,
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
        const size_t ib = out_nnz * od * sizeof(uint32_t), vb = out_nnz * sizeof(double);
        void* pi = PinnedPool::get().take(ib);
        void* pv = pi ? PinnedPool::get().take(vb) : nullptr;
        if (pi && pv) {
            // pinned pool blocks: one DMA per array, no staging
            SharedBlock* blk = new SharedBlock;
            blk->refs = 1;
            blk->location = kPinnedPoolBlock;
            blk->idx = pi;
            blk->val = pv;
            out->opaque = blk;
            out->idx = static_cast<uint32_t*>(pi);
            out->vals = static_cast<double*>(pv);
            PTC_CUDA(cudaMemcpyAsync(pi, ov.idx, ib, cudaMemcpyDeviceToHost, st));
            PTC_CUDA(cudaMemcpyAsync(pv, ov.val, vb, cudaMemcpyDeviceToHost, st));
        } else {
            if (pi) PinnedPool::get().give(pi);
            out->idx = static_cast<uint32_t*>(host_result_alloc(ib));
            out->vals = static_cast<double*>(host_result_alloc(vb));
            if (!out->idx || !out->vals) {
                std::free(out->idx);
                std::free(out->vals);
                cudaFreeAsync(ov.idx, st);
                cudaFreeAsync(ov.val, st);
                out->idx = nullptr;
                out->vals = nullptr;
                throw Error{PTC_ERR_OUT_OF_MEMORY, "host output allocation failed"};
            }
            host_copier().copy(out->idx, ov.idx, ib, st);
            host_copier().copy(out->vals, ov.val, vb, st);
        }
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

// ---------------------------------------------------------------------------------------------
// batches: many contractions as one problem
// ---------------------------------------------------------------------------------------------
//
// Every item's keys are offset into a key range of its own (contracted keys by the sizes of the
// earlier items' contracted key spaces, free keys likewise), so one pass of each kernel -- keys,
// sorts, one cuckoo table, symbolic pass, accumulators -- serves the whole batch, and rows and
// columns of different items never meet.  Column ids stay local to their item (the accumulators
// index tables by them); the items' rows are contiguous in row order.  The output of the batch is
// produced in waves of consecutive items whose outputs fit a device budget; each wave's numeric
// pass is one CUDA-graph launch.

struct BatchItemHost {
    const ptc_coo* A;
    const ptc_coo* B;
    bool self;
    uint32_t c;
    const uint32_t* a_modes;
    const uint32_t* b_modes;
    uint32_t fa, fb;
};

// Where the items' outputs go: outs[id] (kept), sink(user, id, view) (streamed), or nowhere.
struct BatchTarget {
    ptc_tensor* outs = nullptr;
    ptc_batch_sink sink = nullptr;
    void* user = nullptr;
    std::vector<uint32_t> ids;  // caller's index of each item
};

void fill_side(ItemSide& s, const ptc_coo* t, const uint32_t* modes, const KeySpec& con, const KeySpec& fr,
               uint64_t fbase) {
    s.order = t->order;
    s.fbase = fbase;
    for (uint32_t j = 0; j < t->order; ++j) {
        s.mode[j] = modes[j];
        s.dim[j] = t->dims[j];
        s.stride[j] = j < con.n ? con.stride[j] : fr.stride[j - con.n];
    }
}

Front front_batch(const std::vector<BatchItemHost>& items, uint32_t location, const ptc_options& opt, const Knobs& kn,
                  Arena& ar, Events& ev, ptc_stats& stats) {
    cudaStream_t st = ar.stream();
    const uint32_t n = (uint32_t)items.size();
    std::vector<ItemSpec> spec(n);
    std::vector<uint64_t> a_off(n + 1, 0), b_off(n + 1, 0), abase(n), bbase(n);
    unsigned __int128 cb = 0, ab = 0, bb = 0;
    bool all_self = true;
    uint32_t fa_w = 0, fb_w = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const BatchItemHost& x = items[i];
        const KeySpec ac = make_keyspec(x.A->dims, x.a_modes, x.c);
        const KeySpec af = make_keyspec(x.A->dims, x.a_modes + x.c, x.fa);
        const KeySpec bc = make_keyspec(x.B->dims, x.b_modes, x.c);
        const KeySpec bf = make_keyspec(x.B->dims, x.b_modes + x.c, x.fb);
        ItemSpec& s = spec[i];
        std::memset(&s, 0, sizeof(s));
        s.cbase = (uint64_t)cb;
        s.c = x.c;
        fill_side(s.side[0], x.A, x.a_modes, ac, af, (uint64_t)ab);
        fill_side(s.side[1], x.B, x.b_modes, bc, bf, (uint64_t)bb);
        abase[i] = (uint64_t)ab;
        bbase[i] = (uint64_t)bb;
        cb += ac.space;
        ab += af.space;
        bb += bf.space;
        PTC_REQUIRE(cb <= (unsigned __int128)UINT64_MAX && ab <= (unsigned __int128)UINT64_MAX &&
                        bb <= (unsigned __int128)UINT64_MAX,
                    PTC_ERR_KEY_OVERFLOW, "the batch's key spaces together do not fit in 64 bits");
        a_off[i + 1] = a_off[i] + x.A->nnz;
        b_off[i + 1] = b_off[i] + x.B->nnz;
        all_self = all_self && x.self;
        fa_w = std::max(fa_w, x.fa);
        fb_w = std::max(fb_w, x.fb);
    }
    const uint64_t na = a_off[n], nb = all_self ? na : b_off[n];
    PTC_REQUIRE(na < (1ull << 32) && nb < (1ull << 32), PTC_ERR_INVALID_ARGUMENT,
                "a batch holds fewer than 2^32 nonzeros per side");

    // ---- inputs on the device: host items are staged into one buffer per side ----
    if (location == PTC_HOST) {
        for (int side = 0; side < 2; ++side) {
            if (side == 1 && all_self) break;
            uint64_t words = 0, vals = 0;
            for (uint32_t i = 0; i < n; ++i) {
                const ptc_coo* t = side == 0 ? items[i].A : items[i].B;
                if (side == 1 && items[i].self) continue;
                words += t->nnz * t->order;
                vals += t->nnz;
            }
            uint32_t* didx = ar.alloc<uint32_t>(words);
            double* dval = ar.alloc<double>(vals);
            std::vector<HostSeg> si, sv;
            uint64_t wo = 0, vo = 0;
            for (uint32_t i = 0; i < n; ++i) {
                const ptc_coo* t = side == 0 ? items[i].A : items[i].B;
                if (side == 1 && items[i].self) continue;
                spec[i].side[side].idx = didx + wo;
                spec[i].side[side].vals = dval + vo;
                si.push_back({t->idx, t->nnz * t->order * sizeof(uint32_t)});
                sv.push_back({t->vals, t->nnz * sizeof(double)});
                wo += t->nnz * t->order;
                vo += t->nnz;
            }
            host_copier().gather_to_device(didx, si, st);
            host_copier().gather_to_device(dval, sv, st);
        }
        for (uint32_t i = 0; i < n; ++i)
            if (items[i].self) {
                spec[i].side[1].idx = spec[i].side[0].idx;
                spec[i].side[1].vals = spec[i].side[0].vals;
            }
    } else {
        for (uint32_t i = 0; i < n; ++i) {
            spec[i].side[0].idx = items[i].A->idx;
            spec[i].side[0].vals = items[i].A->vals;
            spec[i].side[1].idx = items[i].B->idx;
            spec[i].side[1].vals = items[i].B->vals;
        }
    }
    PTC_CUDA(cudaEventRecord(ev.ev[EV_H2D], st));
    stats.a_nnz = na;
    stats.b_nnz = nb;

    auto upload = [&](const auto& v) {
        using T = typename std::decay_t<decltype(v)>::value_type;
        T* d = ar.alloc<T>(v.size());
        PTC_CUDA(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
        return d;
    };
    const ItemSpec* specs_d = upload(spec);
    const uint64_t* a_off_d = upload(a_off);
    const uint64_t* b_off_d = all_self ? a_off_d : upload(b_off);
    const uint64_t* abase_d = upload(abase);
    const uint64_t* bbase_d = all_self ? abase_d : upload(bbase);

    // ---- keys ----
    uint32_t* err = ar.alloc<uint32_t>(1);
    PTC_CUDA(cudaMemsetAsync(err, 0, sizeof(uint32_t), st));
    uint64_t* a_ckey = ar.alloc<uint64_t>(na);
    uint64_t* a_fkey = ar.alloc<uint64_t>(na);
    double* a_vals = ar.alloc<double>(na);
    launch_pack_items(specs_d, a_off_d, n, 0, na, a_ckey, a_fkey, a_vals, err, st);
    uint64_t* b_ckey = a_ckey;
    uint64_t* b_fkey = a_fkey;
    double* b_vals = a_vals;
    if (!all_self) {
        b_ckey = ar.alloc<uint64_t>(nb);
        b_fkey = ar.alloc<uint64_t>(nb);
        b_vals = ar.alloc<double>(nb);
        launch_pack_items(specs_d, b_off_d, n, 1, nb, b_ckey, b_fkey, b_vals, err, st);
    }
    PTC_REQUIRE(read_scalar(err, st) == 0, PTC_ERR_INDEX_RANGE, "an index is not smaller than its mode size");

    // ---- B side: columns (global ranks, then local to their item), fibers, cuckoo table ----
    Ranked cols = rank_keys(b_fkey, nb, (uint64_t)bb, ar);
    uint32_t* col_first = ar.alloc<uint32_t>(n + 1);
    launch_key_bounds(cols.run_key, cols.nruns, bbase_d, n, col_first, st);
    std::vector<uint32_t> h_col_first(n + 1);
    PTC_CUDA(cudaMemcpyAsync(h_col_first.data(), col_first, (n + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    uint32_t* col_local = ar.alloc<uint32_t>(nb);
    launch_localize(cols.rank_of, nb, b_off_d, n, col_first, col_local, st);
    uint32_t* col_tuple = ar.alloc<uint32_t>(cols.nruns * std::max(fb_w, 1u));
    launch_item_tuples(cols.run_start, cols.perm, cols.nruns, specs_d, b_off_d, n, 1, fb_w, col_tuple, st);
    Fibers fib = group_fibers(b_ckey, cols.rank_of, cols.nruns, nb, bits_for_space((uint64_t)cb), b_vals, ar,
                              col_local);
    // each item's fibers are contiguous (its contracted keys start at its cbase)
    std::vector<uint64_t> cbase_h(n);
    for (uint32_t i = 0; i < n; ++i) cbase_h[i] = spec[i].cbase;
    const uint64_t* cbase_d = upload(cbase_h);
    uint32_t* fib_first = ar.alloc<uint32_t>(n + 1);
    launch_key_bounds(fib.key, fib.n, cbase_d, n, fib_first, st);
    CuckooBuildInfo cinfo;
    const CuckooTable table = cuckoo_build(fib.key, fib.n, opt.hash_seed, kn.max_chain, kn.max_load, kn.max_attempts, ar, &cinfo);
    stats.hash_attempts = cinfo.attempts;
    PTC_CUDA(cudaEventRecord(ev.ev[EV_BSIDE], st));
    PTC_CUDA(cudaStreamSynchronize(st));  // h_col_first
    uint64_t ncols_local = 0;
    for (uint32_t i = 0; i < n; ++i) ncols_local = std::max<uint64_t>(ncols_local, h_col_first[i + 1] - h_col_first[i]);

    // ---- A side ----
    Ranked rows;
    uint32_t* row_first = col_first;
    uint32_t* row_tuple = col_tuple;
    if (all_self) {
        rows = cols;
    } else {
        rows = rank_keys(a_fkey, na, (uint64_t)ab, ar);
        row_first = ar.alloc<uint32_t>(n + 1);
        launch_key_bounds(rows.run_key, rows.nruns, abase_d, n, row_first, st);
        row_tuple = ar.alloc<uint32_t>(rows.nruns * std::max(fa_w, 1u));
        launch_item_tuples(rows.run_start, rows.perm, rows.nruns, specs_d, a_off_d, n, 0, fa_w, row_tuple, st);
    }
    Front F;
    F.h_row_first.resize(n + 1);
    PTC_CUDA(cudaMemcpyAsync(F.h_row_first.data(), row_first, (n + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    uint32_t* row_item = ar.alloc<uint32_t>(std::max<uint64_t>(rows.nruns, 1));
    launch_row_item(rows.nruns, row_first, n, row_item, st);
    uint64_t* a_ckey_sorted = ar.alloc<uint64_t>(na);
    double* a_val = ar.alloc<double>(na);
    launch_gather<uint64_t>(a_ckey, rows.perm, na, a_ckey_sorted, st);
    launch_gather<double>(a_vals, rows.perm, na, a_val, st);
    int32_t* a_fib = ar.alloc<int32_t>(na);
    cuckoo_lookup(table, a_ckey_sorted, na, a_fib, ar);
    PTC_CUDA(cudaEventRecord(ev.ev[EV_ASIDE], st));
    PTC_CUDA(cudaStreamSynchronize(st));  // h_row_first

    Operands& op = F.op;
    op.na = na; op.nb = nb; op.nrows = rows.nruns; op.ncols = ncols_local; op.nfib = fib.n;
    op.fa = fa_w; op.fb = fb_w;
    op.a_val = a_val; op.a_fib = a_fib; op.row_start = rows.run_start;
    op.b_col = fib.col; op.b_val = fib.val; op.fib_start = fib.start;
    op.row_tuple = row_tuple; op.col_tuple = col_tuple;
    op.err = err;
    op.row_item = row_item;
    F.item_out = ar.alloc<ItemOut>(n);
    op.item_out = F.item_out;
    F.a_row = rows.run_of;
    F.batch = true;
    F.nitems = n;
    F.row_first = row_first;
    F.colbase = h_col_first;
    F.b_off = b_off_d;
    F.col_first = col_first;
    F.fib_first = fib_first;
    F.col_run = cols.run_start;
    F.ncols_global = cols.nruns;
    stats.ncols = cols.nruns;
    return F;
}

// values of a device array at the given indices, on the host
template <typename T>
std::vector<T> read_at(const T* a, const std::vector<uint32_t>& at, Arena& ar) {
    cudaStream_t st = ar.stream();
    uint32_t* at_d = ar.alloc<uint32_t>(at.size());
    T* v_d = ar.alloc<T>(at.size());
    PTC_CUDA(cudaMemcpyAsync(at_d, at.data(), at.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    launch_gather<T>(a, at_d, at.size(), v_d, st);
    std::vector<T> v(at.size());
    PTC_CUDA(cudaMemcpyAsync(v.data(), v_d, v.size() * sizeof(T), cudaMemcpyDeviceToHost, st));
    PTC_CUDA(cudaStreamSynchronize(st));
    return v;
}

void deliver_empty(const BatchTarget& tg, uint32_t i, const BatchItemHost& x, uint32_t location) {
    ptc_tensor t;
    std::memset(&t, 0, sizeof(t));
    t.order = x.fa + x.fb;
    t.location = location;
    if (tg.outs) tg.outs[tg.ids[i]] = t;
    if (tg.sink) tg.sink(tg.user, tg.ids[i], &t);
}

void batch_impl(const std::vector<BatchItemHost>& items, uint32_t location, const ptc_options& opt, bool exact_only,
                const BatchTarget& tg, ptc_stats& stats) {
    const uint32_t n = (uint32_t)items.size();
    DeviceSetup dev = setup_device(opt);
    cudaStream_t st = dev.stream;
    Events ev;
    Arena ar(st);
    PTC_CUDA(cudaEventRecord(ev.ev[EV_START], st));
    const Knobs kn = knobs_of(opt);
    Front F = front_batch(items, location, opt, kn, ar, ev, stats);

    const bool learned = opt.path == PTC_PATH_LEARNED && !exact_only;
    const SizerHost* sizer = nullptr;
    if (learned) {
        sizer = opt.sizer ? sizer_host(opt.sizer) : default_sizer();
        PTC_REQUIRE(sizer != nullptr, PTC_ERR_INVALID_ARGUMENT,
                    "the learned path needs a sizer: opt.sizer, or sizer_default.bin beside the library");
    }
    Plan pl = plan_rows(F, opt, sizer, nullptr, dev.num_sms, ar, stats);
    const Operands& op = F.op;
    const uint64_t nrows = op.nrows;
    if (pl.flops == 0) {
        for (uint32_t i = 0; i < n; ++i) deliver_empty(tg, i, items[i], opt.output_location);
        ar.release();
        PTC_CUDA(cudaStreamSynchronize(st));
        return;
    }

    // ---- each item's range of entries: [E_i, E_i + S_i) ----
    // two-phase: exact counts; learned: the small and sort-based rows' exact entries first, then
    // the large rows' claims within their predicted budgets
    const std::vector<uint32_t>& rf = F.h_row_first;
    const std::vector<uint64_t> ex = read_at<uint64_t>(pl.row_off, rf, ar);
    std::vector<uint64_t> cl(n + 1, 0);
    if (learned) {
        cl = read_at<uint64_t>(pl.claim_off, rf, ar);
        launch_shift_exact(nrows, op.row_item, F.row_first, pl.claim_off, pl.row_off, st);
    }
    std::vector<uint64_t> E(n + 1), S(n), X(n);
    for (uint32_t i = 0; i <= n; ++i) E[i] = ex[i] + cl[i];
    for (uint32_t i = 0; i < n; ++i) {
        S[i] = E[i + 1] - E[i];
        X[i] = ex[i + 1] - ex[i];
    }
    PTC_CUDA(cudaEventRecord(ev.ev[EV_SYM], st));

    // ---- waves of consecutive items whose outputs fit the budget ----
    const bool keep_device = tg.outs && opt.output_location == PTC_DEVICE;
    uint64_t budget = (uint64_t)opt.batch_wave_mib << 20;
    if (budget == 0) {
        // free device memory, counting what the stream-ordered pool holds without using it
        size_t free_b = 0, total_b = 0;
        PTC_CUDA(cudaMemGetInfo(&free_b, &total_b));
        cudaMemPool_t pool;
        uint64_t reserved = 0, used = 0;
        PTC_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev.device));
        PTC_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved));
        PTC_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used));
        // leave room for sorting the work items by wave (item, key, index and gathered copy)
        const uint64_t sort_need = (uint64_t)(pl.n_parts[0] + pl.n_parts[1]) * (2 * sizeof(PartItem) + 24);
        const uint64_t avail = free_b + (reserved > used ? reserved - used : 0);
        budget = avail > sort_need ? (uint64_t)((avail - sort_need) * 0.6) : (64ull << 20);
    }
    if (keep_device) budget = UINT64_MAX;  // every output stays: one wave
    std::vector<uint32_t> wave_item{0};
    {
        uint64_t acc = 0;
        for (uint32_t i = 0; i < n; ++i) {
            const uint64_t b = S[i] * (8 + 4ull * (items[i].fa + items[i].fb));
            if (acc > 0 && acc + b > budget) {
                wave_item.push_back(i);
                acc = 0;
            }
            acc += b;
        }
        wave_item.push_back(n);
    }
    const uint32_t nw = (uint32_t)wave_item.size() - 1;
    stats.batch_waves = nw;

    // work of each wave: parts sorted by wave (largest first inside a wave), small rows, runs
    std::vector<uint32_t> wave_row(nw + 1);
    for (uint32_t w = 0; w <= nw; ++w) wave_row[w] = rf[wave_item[w]];
    std::vector<uint32_t> pb[2];
    PartItem* parts[2] = {pl.parts[0], pl.parts[1]};
    uint32_t* wave_row_d = ar.alloc<uint32_t>(nw + 1);
    PTC_CUDA(cudaMemcpyAsync(wave_row_d, wave_row.data(), (nw + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    std::vector<uint64_t> wid(nw);
    for (uint32_t w = 0; w < nw; ++w) wid[w] = w;
    uint64_t* wid_d = ar.alloc<uint64_t>(nw);
    PTC_CUDA(cudaMemcpyAsync(wid_d, wid.data(), nw * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    for (int kind = 0; kind < 2; ++kind) {
        const uint32_t np = pl.n_parts[kind];
        pb[kind].assign(nw + 1, 0);
        pb[kind][nw] = np;
        if (nw == 1 || np == 0) continue;
        uint64_t* key = ar.alloc<uint64_t>(np);
        uint32_t* idx = ar.alloc<uint32_t>(np);
        launch_part_wave(pl.parts[kind], np, wave_row_d, nw, key, idx, st);
        radix_sort_pairs(key, idx, np, 0, bits_for_space(nw), ar);
        parts[kind] = ar.alloc<PartItem>(np);
        launch_gather_parts(pl.parts[kind], idx, np, parts[kind], st);
        uint32_t* bounds = ar.alloc<uint32_t>(nw + 1);
        launch_key_bounds(key, np, wid_d, nw, bounds, st);
        PTC_CUDA(cudaMemcpyAsync(pb[kind].data(), bounds, (nw + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        PTC_CUDA(cudaStreamSynchronize(st));
    }
    // rows of the bitmap kernel by wave (heaviest first inside a wave: the sort is stable)
    const uint32_t* map_rows = pl.map_rows;
    std::vector<uint32_t> mb(nw + 1, 0);
    mb[nw] = pl.n_map;
    if (nw > 1 && pl.n_map > 0) {
        uint64_t* key = ar.alloc<uint64_t>(pl.n_map);
        uint32_t* idx = ar.alloc<uint32_t>(pl.n_map);
        launch_row_wave(pl.map_rows, pl.n_map, wave_row_d, nw, key, idx, st);
        radix_sort_pairs(key, idx, pl.n_map, 0, bits_for_space(nw), ar);
        uint32_t* sorted = ar.alloc<uint32_t>(pl.n_map);
        launch_gather<uint32_t>(pl.map_rows, idx, pl.n_map, sorted, st);
        map_rows = sorted;
        uint32_t* bounds = ar.alloc<uint32_t>(nw + 1);
        launch_key_bounds(key, pl.n_map, wid_d, nw, bounds, st);
        PTC_CUDA(cudaMemcpyAsync(mb.data(), bounds, (nw + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        PTC_CUDA(cudaStreamSynchronize(st));
    }
    uint32_t* map_fail_count = nullptr;
    uint32_t* map_fail_list = nullptr;
    if (learned && pl.n_map > 0) {
        map_fail_count = ar.alloc<uint32_t>(1);
        map_fail_list = ar.alloc<uint32_t>(std::max<uint32_t>(pl.n_map, 1));
    }
    const std::vector<uint32_t> sb = read_at<uint32_t>(pl.small_pos, wave_row, ar);
    std::vector<uint32_t> cb(nw + 1, 0);  // collision-free rows of each wave (sorted by row)
    if (pl.n_copy > 0) {
        std::vector<uint64_t> wr64(wave_row.begin(), wave_row.end());
        uint64_t* wr_d = ar.alloc<uint64_t>(nw + 1);
        PTC_CUDA(cudaMemcpyAsync(wr_d, wr64.data(), (nw + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
        uint32_t* cbd = ar.alloc<uint32_t>(nw + 2);
        launch_key_bounds(pl.copy_keys, pl.n_copy, wr_d, nw + 1, cbd, st);
        PTC_CUDA(cudaMemcpyAsync(cb.data(), cbd, (nw + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        PTC_CUDA(cudaStreamSynchronize(st));
    }
    std::vector<uint32_t> rb(nw + 1, 0);
    if (pl.n_esc > 0) rb = read_at<uint32_t>(pl.esc_first, read_at<uint32_t>(pl.esc_pos, wave_row, ar), ar);
    std::vector<uint32_t> lb(nw + 1, 0);  // long runs of each wave
    for (uint32_t w = 0; w <= nw; ++w)
        lb[w] = (uint32_t)(std::lower_bound(pl.h_esc_long.begin(), pl.h_esc_long.end(), rb[w]) - pl.h_esc_long.begin());

    // learned: the claim cursors of every item
    OutputView base;
    if (learned) {
        std::vector<uint64_t> cur(n), end(n);
        for (uint32_t i = 0; i < n; ++i) {
            cur[i] = E[i] + X[i];
            end[i] = E[i] + S[i];
        }
        base.cursor = ar.alloc<uint64_t>(n);
        base.overshoot = ar.alloc<uint64_t>(n);
        uint64_t* end_d = ar.alloc<uint64_t>(n);
        PTC_CUDA(cudaMemcpyAsync(base.cursor, cur.data(), n * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
        PTC_CUDA(cudaMemcpyAsync(end_d, end.data(), n * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
        PTC_CUDA(cudaMemsetAsync(base.overshoot, 0, n * sizeof(uint64_t), st));
        base.cap_end = end_d;
        PTC_CUDA(cudaStreamSynchronize(st));  // the host vectors above go out of scope
    }
    uint32_t* fail_count[2] = {nullptr, nullptr};
    uint32_t* fail_list[2] = {nullptr, nullptr};
    if (learned)
        for (int kind = 0; kind < 2; ++kind) {
            fail_count[kind] = ar.alloc<uint32_t>(1);
            fail_list[kind] = ar.alloc<uint32_t>(std::max<uint32_t>(pl.n_parts[kind], 1));
        }

    // output blocks: one per wave when the outputs are kept on the device, else one reused block
    uint64_t max_vals = 0, max_words = 0;
    std::vector<uint64_t> wave_vals(nw, 0), wave_words(nw, 0);
    for (uint32_t w = 0; w < nw; ++w) {
        for (uint32_t i = wave_item[w]; i < wave_item[w + 1]; ++i) {
            wave_vals[w] += S[i];
            wave_words[w] += S[i] * (items[i].fa + items[i].fb);
        }
        max_vals = std::max(max_vals, wave_vals[w]);
        max_words = std::max(max_words, wave_words[w]);
    }
    uint32_t* blk_idx = nullptr;
    double* blk_val = nullptr;
    void* host_blk_idx = nullptr;
    void* host_blk_val = nullptr;
    auto free_blocks = [&]() {  // blocks handed to the caller are no longer held here
        if (blk_idx) cudaFreeAsync(blk_idx, st);
        if (blk_val) cudaFreeAsync(blk_val, st);
        std::free(host_blk_idx);
        std::free(host_blk_val);
        blk_idx = nullptr;
        blk_val = nullptr;
        host_blk_idx = host_blk_val = nullptr;
    };
    std::vector<uint8_t> failed(n, 0);
    double t_numeric = 0.0, t_out = 0.0;
    try {
        if (!keep_device) {
            PTC_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&blk_idx), std::max<uint64_t>(max_words, 1) * 4, st));
            PTC_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&blk_val), std::max<uint64_t>(max_vals, 1) * 8, st));
        }
        const bool host_view = opt.output_location == PTC_HOST && tg.sink && !tg.outs;
        if (host_view) {
            host_blk_idx = host_result_alloc(std::max<uint64_t>(max_words, 1) * 4);
            host_blk_val = host_result_alloc(std::max<uint64_t>(max_vals, 1) * 8);
            PTC_REQUIRE(host_blk_idx && host_blk_val, PTC_ERR_OUT_OF_MEMORY, "host output allocation failed");
        }
        std::vector<ItemOut> io(n);
        for (uint32_t w = 0; w < nw; ++w) {
            const uint32_t i0 = wave_item[w], i1 = wave_item[w + 1];
            if (keep_device) {
                PTC_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&blk_idx), std::max<uint64_t>(wave_words[w], 1) * 4, st));
                PTC_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&blk_val), std::max<uint64_t>(wave_vals[w], 1) * 8, st));
            }
            uint64_t words = 0;
            for (uint32_t i = i0; i < i1; ++i) {
                io[i].ent0 = E[i];
                io[i].val0 = E[i] - E[i0];
                io[i].idx0 = words;
                io[i].colbase = F.colbase[i];
                io[i].fa = items[i].fa;
                io[i].fb = items[i].fb;
                io[i].pad = 0;
                words += S[i] * (items[i].fa + items[i].fb);
            }
            PTC_CUDA(cudaMemcpyAsync(F.item_out + i0, io.data() + i0, (i1 - i0) * sizeof(ItemOut),
                                     cudaMemcpyHostToDevice, st));
            OutputView ov = base;
            ov.idx = blk_idx;
            ov.val = blk_val;
            OutputView ovk[2] = {ov, ov};
            OutputView ovm = ov;
            if (learned) {
                for (int kind = 0; kind < 2; ++kind) {
                    ovk[kind].fail_count = fail_count[kind];
                    ovk[kind].fail_list = fail_list[kind];
                    PTC_CUDA(cudaMemsetAsync(fail_count[kind], 0, sizeof(uint32_t), st));
                }
                if (pl.n_map > 0) {
                    ovm.fail_count = map_fail_count;
                    ovm.fail_list = map_fail_list;
                    PTC_CUDA(cudaMemsetAsync(map_fail_count, 0, sizeof(uint32_t), st));
                }
            }
            PTC_CUDA(cudaEventRecord(ev.ev[EV_WAVE0], st));
            const bool work = sb[w + 1] > sb[w] || pb[0][w + 1] > pb[0][w] || pb[1][w + 1] > pb[1][w] ||
                              rb[w + 1] > rb[w] || cb[w + 1] > cb[w] || mb[w + 1] > mb[w];
            // the wave's numeric pass, captured and launched as one graph
            cudaGraph_t graph = nullptr;
            cudaGraphExec_t exec = nullptr;
            if (work) {
                AuxStreams& aux = aux_streams(dev.device);
                bool forked = false;
                PTC_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
                try {
                    launch_small_rows(true, op, pl.small_rows + sb[w], sb[w + 1] - sb[w], nullptr, pl.row_off, ov,
                                      st);
                    launch_copy_rows(op, pl.copy_rows + cb[w], cb[w + 1] - cb[w], pl.alen, pl.row_off, ov,
                                     dev.num_sms, st);
                    // the block parts and the sort-based folds beside the warp tasks (disjoint
                    // outputs): branches of the wave's graph
                    aux.fork(st);
                    forked = true;
                    launch_parts(1, op, parts[1] + pb[1][w], pb[1][w + 1] - pb[1][w], ovk[1], pl.work_counter2,
                                 op.err, dev.num_sms, aux.s[0]);
                    launch_esc_fold(op, ov, pl.esc_run_key, pl.esc_run_start, rb[w], rb[w + 1], pl.esc_colbits,
                                    pl.esc_rows, pl.esc_first, pl.row_off, pl.esc_sorted,
                                    pl.esc_long + lb[w], lb[w + 1] - lb[w], aux.s[1]);
                    launch_parts(0, op, parts[0] + pb[0][w], pb[0][w + 1] - pb[0][w], ovk[0], pl.work_counter,
                                 op.err, dev.num_sms, st);
                    if (pl.n_map > 0)
                        launch_rowmap(learned ? kRowmapClaim : kRowmapExact, op, map_rows + mb[w], mb[w + 1] - mb[w],
                                      nullptr, pl.row_off, ovm, pl.work_counter, dev.num_sms, st);
                    aux.join(st);
                    forked = false;
                } catch (...) {
                    if (forked)  // rejoin the branches so the capture can end
                        for (int i = 0; i < 2; ++i) {
                            cudaEventRecord(aux.join_ev[i], aux.s[i]);
                            cudaStreamWaitEvent(st, aux.join_ev[i], 0);
                        }
                    cudaStreamEndCapture(st, &graph);
                    if (graph) cudaGraphDestroy(graph);
                    throw;
                }
                PTC_CUDA(cudaStreamEndCapture(st, &graph));
                const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
                if (ie != cudaSuccess) {
                    cudaGraphDestroy(graph);
                    throw Error{PTC_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ie)};
                }
            }
            const cudaError_t le = work ? cudaGraphLaunch(exec, st) : cudaSuccess;
            PTC_CUDA(cudaEventRecord(ev.ev[EV_WAVE1], st));
            const cudaError_t se = cudaStreamSynchronize(st);
            if (exec) cudaGraphExecDestroy(exec);
            if (graph) cudaGraphDestroy(graph);
            PTC_CUDA(le);
            PTC_CUDA(se);
            t_numeric += ev.ms(EV_WAVE0, EV_WAVE1);
            PTC_REQUIRE(read_scalar(op.err, st) == 0, PTC_ERR_INTERNAL,
                        "an accumulator table overflowed or met an out-of-range column");

            // entries of each item; items with a failed claim or table are rerun exactly below
            std::vector<uint64_t> nnz(S.begin() + i0, S.begin() + i1);
            if (learned) {
                for (int kind = 0; kind < 2; ++kind) {
                    const uint32_t nfail = read_scalar(fail_count[kind], st);
                    if (nfail > 0) {
                        PartItem* fp = ar.alloc<PartItem>(nfail);
                        launch_gather_parts(parts[kind] + pb[kind][w], fail_list[kind], nfail, fp, st);
                        std::vector<PartItem> hf(nfail);
                        PTC_CUDA(cudaMemcpyAsync(hf.data(), fp, nfail * sizeof(PartItem), cudaMemcpyDeviceToHost, st));
                        PTC_CUDA(cudaStreamSynchronize(st));
                        for (const PartItem& p : hf) {
                            const uint32_t it =
                                (uint32_t)(std::upper_bound(rf.begin(), rf.end(), p.row) - rf.begin()) - 1;
                            failed[it] = 1;
                        }
                    }
                }
                if (pl.n_map > 0) {  // rows whose claim did not fit their item's budget
                    const uint32_t nfail = read_scalar(map_fail_count, st);
                    if (nfail > 0) {
                        uint32_t* fr = ar.alloc<uint32_t>(nfail);
                        launch_gather<uint32_t>(map_rows + mb[w], map_fail_list, nfail, fr, st);
                        std::vector<uint32_t> hr(nfail);
                        PTC_CUDA(cudaMemcpyAsync(hr.data(), fr, nfail * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
                        PTC_CUDA(cudaStreamSynchronize(st));
                        for (uint32_t r : hr)
                            failed[(uint32_t)(std::upper_bound(rf.begin(), rf.end(), r) - rf.begin()) - 1] = 1;
                    }
                }
                std::vector<uint64_t> cur(i1 - i0), over(i1 - i0);
                PTC_CUDA(cudaMemcpyAsync(cur.data(), ov.cursor + i0, (i1 - i0) * 8, cudaMemcpyDeviceToHost, st));
                PTC_CUDA(cudaMemcpyAsync(over.data(), ov.overshoot + i0, (i1 - i0) * 8, cudaMemcpyDeviceToHost, st));
                PTC_CUDA(cudaStreamSynchronize(st));
                for (uint32_t i = i0; i < i1; ++i) nnz[i - i0] = cur[i - i0] - over[i - i0] - E[i];
            }

            // ---- hand the wave's outputs over ----
            const auto t0 = std::chrono::steady_clock::now();
            const void* src_idx = blk_idx;
            const void* src_val = blk_val;
            uint32_t loc = opt.output_location;
            SharedBlock* shared = nullptr;
            if (tg.outs) {
                shared = new SharedBlock;
                shared->location = loc;
                if (loc == PTC_DEVICE) {
                    shared->idx = blk_idx;
                    shared->val = blk_val;
                    blk_idx = nullptr;
                    blk_val = nullptr;
                } else {
                    shared->idx = host_result_alloc(std::max<uint64_t>(wave_words[w], 1) * 4);
                    shared->val = host_result_alloc(std::max<uint64_t>(wave_vals[w], 1) * 8);
                    if (!shared->idx || !shared->val) {
                        std::free(shared->idx);
                        std::free(shared->val);
                        delete shared;
                        throw Error{PTC_ERR_OUT_OF_MEMORY, "host output allocation failed"};
                    }
                    host_copier().copy(shared->idx, blk_idx, wave_words[w] * 4, st);
                    host_copier().copy(shared->val, blk_val, wave_vals[w] * 8, st);
                }
                src_idx = shared->idx;
                src_val = shared->val;
            } else if (host_view) {
                host_copier().copy(host_blk_idx, blk_idx, wave_words[w] * 4, st);
                host_copier().copy(host_blk_val, blk_val, wave_vals[w] * 8, st);
                src_idx = host_blk_idx;
                src_val = host_blk_val;
            } else if (tg.sink) {
                loc = PTC_DEVICE;  // device views of the reused block
            }
            uint32_t refs = 0;
            for (uint32_t i = i0; i < i1; ++i) {
                if (failed[i]) continue;
                ptc_tensor t;
                std::memset(&t, 0, sizeof(t));
                t.order = items[i].fa + items[i].fb;
                t.location = loc;
                t.nnz = nnz[i - i0];
                if (t.nnz > 0) {
                    t.idx = const_cast<uint32_t*>(static_cast<const uint32_t*>(src_idx)) + io[i].idx0;
                    t.vals = const_cast<double*>(static_cast<const double*>(src_val)) + io[i].val0;
                }
                stats.out_nnz += t.nnz;
                if (tg.outs) {
                    if (t.nnz > 0) {
                        t.opaque = shared;
                        ++refs;
                    }
                    tg.outs[tg.ids[i]] = t;
                }
                if (tg.sink) tg.sink(tg.user, tg.ids[i], &t);
            }
            if (shared) {
                shared->refs = refs + 1;
                release_block(shared);  // drops the wave's own reference
            }
            t_out += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        }
    } catch (...) {
        free_blocks();
        throw;
    }
    free_blocks();
    PTC_CUDA(cudaEventRecord(ev.ev[EV_D2H], st));
    ar.release();
    PTC_CUDA(cudaStreamSynchronize(st));
    stats.t_h2d_ms += ev.ms(EV_START, EV_H2D);
    stats.t_build_ms += ev.ms(EV_H2D, EV_ASIDE);
    stats.t_symbolic_ms += ev.ms(EV_ASIDE, EV_SYM);
    stats.t_numeric_ms += t_numeric;
    stats.t_d2h_ms += t_out;
    stats.t_total_ms += ev.ms(EV_START, EV_D2H);

    // learned path: items whose prediction fell short run again, exactly
    std::vector<BatchItemHost> again;
    BatchTarget tg2;
    tg2.outs = tg.outs;
    tg2.sink = tg.sink;
    tg2.user = tg.user;
    for (uint32_t i = 0; i < n; ++i)
        if (failed[i]) {
            again.push_back(items[i]);
            tg2.ids.push_back(tg.ids[i]);
            stats.rerun_rows += rf[i + 1] - rf[i];
        }
    stats.rerun_items += again.size();
    if (!again.empty()) {
        ptc_stats s2;
        std::memset(&s2, 0, sizeof(s2));
        batch_impl(again, location, opt, true, tg2, s2);
        stats.out_nnz += s2.out_nnz;
        stats.t_total_ms += s2.t_total_ms;
        stats.t_numeric_ms += s2.t_numeric_ms;
    }
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
    opt->cuckoo_max_chain = ptc::kCuckooMaxChain;
    opt->cuckoo_max_attempts = ptc::kCuckooMaxAttempts;
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
    ptc::DeviceGuard keep_device;
    if (out) std::memset(out, 0, sizeof(*out));  // so that every error path below can release it
    try {
        ptc::contract_impl(A, B, c, a_modes, b_modes, opt, out, stats);
        ptc::g_last_error.clear();
        return PTC_OK;
    } catch (const Error& e) {
        ptc_tensor_free(out);
        ptc::set_last_error(e.status, e.msg);
        return e.status;
    } catch (const std::bad_alloc&) {
        ptc_tensor_free(out);
        ptc::set_last_error(PTC_ERR_OUT_OF_MEMORY, "host allocation failed");
        return PTC_ERR_OUT_OF_MEMORY;
    } catch (...) {
        ptc_tensor_free(out);
        ptc::set_last_error(PTC_ERR_INTERNAL, "unexpected exception");
        return PTC_ERR_INTERNAL;
    }
}

ptc_status ptc_sizer_collect(const ptc_coo* A, const ptc_coo* B, uint32_t c, const uint32_t* a_modes,
                             const uint32_t* b_modes, const ptc_options* opt, float** features, float** targets,
                             uint64_t* n) {
    ptc::DeviceGuard keep_device;
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

}  // extern "C"

namespace ptc {
namespace {

// A batch runs in chunks of consecutive items holding at most this many nonzeros (an item larger
// than that is a chunk of its own): the build and planning arrays of a chunk, and its work items,
// stay a bounded share of the device memory however long the batch is.
constexpr uint64_t kBatchChunkNnz = 32ull << 20;

void batch_chunks(const std::vector<BatchItemHost>& hi, uint32_t location, const ptc_options& opt,
                  const BatchTarget& tg, ptc_stats& stats) {
    size_t i0 = 0;
    while (i0 < hi.size()) {
        size_t i1 = i0;
        uint64_t nnz = 0;
        while (i1 < hi.size()) {
            const uint64_t k = hi[i1].A->nnz + (hi[i1].self ? 0 : hi[i1].B->nnz);
            if (i1 > i0 && nnz + k > kBatchChunkNnz) break;
            nnz += k;
            ++i1;
        }
        if (i0 == 0 && i1 == hi.size()) {
            batch_impl(hi, location, opt, false, tg, stats);
            return;
        }
        std::vector<BatchItemHost> part(hi.begin() + i0, hi.begin() + i1);
        BatchTarget t2;
        t2.outs = tg.outs;
        t2.sink = tg.sink;
        t2.user = tg.user;
        t2.ids.assign(tg.ids.begin() + i0, tg.ids.begin() + i1);
        ptc_stats s2;
        std::memset(&s2, 0, sizeof(s2));
        batch_impl(part, location, opt, false, t2, s2);
        // sums over the chunks (times, counts); the largest of the per-chunk settings
        stats.mult_adds += s2.mult_adds;
        stats.out_nnz += s2.out_nnz;
        stats.nrows += s2.nrows;
        stats.ncols += s2.ncols;
        stats.nfibers += s2.nfibers;
        stats.a_nnz += s2.a_nnz;
        stats.b_nnz += s2.b_nnz;
        stats.t_total_ms += s2.t_total_ms;
        stats.t_h2d_ms += s2.t_h2d_ms;
        stats.t_build_ms += s2.t_build_ms;
        stats.t_symbolic_ms += s2.t_symbolic_ms;
        stats.t_numeric_ms += s2.t_numeric_ms;
        stats.t_d2h_ms += s2.t_d2h_ms;
        stats.hash_attempts = std::max(stats.hash_attempts, s2.hash_attempts);
        stats.panel_width = std::max(stats.panel_width, s2.panel_width);
        stats.rows_small += s2.rows_small;
        stats.rows_hash += s2.rows_hash;
        stats.hash_parts += s2.hash_parts;
        stats.rows_long += s2.rows_long;
        stats.rerun_rows += s2.rerun_rows;
        stats.batch_waves += s2.batch_waves;
        stats.rerun_items += s2.rerun_items;
        i0 = i1;
    }
}

// The items of a batch call, checked.
std::vector<BatchItemHost> batch_host_items(const ptc_batch_item* items, uint32_t n, uint32_t& location) {
    PTC_REQUIRE(items != nullptr || n == 0, PTC_ERR_INVALID_ARGUMENT, "items is null");
    std::vector<BatchItemHost> hi(n);
    location = PTC_HOST;
    for (uint32_t i = 0; i < n; ++i) {
        const ptc_batch_item& it = items[i];
        const bool self = it.B.idx == nullptr && it.B.nnz == 0 && it.B.dims == nullptr;
        BatchItemHost& h = hi[i];
        h.A = &it.A;
        h.self = self;
        h.B = self ? &it.A : &it.B;
        h.c = it.c;
        h.a_modes = it.a_modes;
        h.b_modes = self ? it.a_modes : it.b_modes;
        const std::string where = "item " + std::to_string(i) + ": ";
        validate_pair(h.A, h.B, h.c, h.a_modes, h.b_modes, where);
        h.fa = h.A->order - h.c;
        h.fb = h.B->order - h.c;
        if (i == 0) location = it.A.location;
        PTC_REQUIRE(h.A->location == location && h.B->location == location, PTC_ERR_INVALID_ARGUMENT,
                    where + "every input of a batch must be in the same memory");
    }
    return hi;
}

// Median time (ms, the calls' own event clocks) of `repeats` discarded-output runs.
// Median time of `repeats` runs of the items under `opt`: one item runs as the single
// contraction it is (ptc_contract's kernels, output kept on the device and released), more as a
// batch (outputs discarded).
double time_batch(const std::vector<BatchItemHost>& hi, uint32_t location, const ptc_options& opt, uint32_t repeats) {
    BatchTarget tg;
    tg.ids.resize(hi.size());
    for (uint32_t i = 0; i < hi.size(); ++i) tg.ids[i] = i;
    std::vector<double> t;
    for (uint32_t r = 0; r < repeats; ++r) {
        ptc_stats st;
        std::memset(&st, 0, sizeof(st));
        if (hi.size() == 1) {
            const BatchItemHost& x = hi[0];
            ptc_options o = opt;
            o.output_location = PTC_DEVICE;
            o.verbose = 0;
            ptc_tensor out;
            contract_impl(x.A, x.self ? nullptr : x.B, x.c, x.a_modes, x.b_modes, &o, &out, &st);
            ptc_tensor_free(&out);
        } else {
            batch_chunks(hi, location, opt, tg, st);
        }
        t.push_back(st.t_total_ms);
    }
    std::sort(t.begin(), t.end());
    return t[t.size() / 2];
}

}  // namespace
}  // namespace ptc

extern "C" {

ptc_status ptc_autotune(const ptc_batch_item* items, uint32_t n, const ptc_options* opt_in, uint32_t repeats,
                        ptc_options* best_out, ptc_tune_report* report) {
    using namespace ptc;
    DeviceGuard keep_device;
    try {
        PTC_REQUIRE(best_out != nullptr && n > 0, PTC_ERR_INVALID_ARGUMENT, "need items and an output");
        ptc_options opt = resolve_options(opt_in);
        uint32_t location = PTC_HOST;
        const std::vector<BatchItemHost> hi = batch_host_items(items, n, location);
        repeats = std::max(1u, repeats);
        time_batch(hi, location, opt, 1);  // warm-up: pool memory, code loading
        ptc_tune_report rep;
        std::memset(&rep, 0, sizeof(rep));
        rep.repeats = repeats;
        double best = time_batch(hi, location, opt, repeats);
        rep.default_ms = best;
        rep.trials = 1;
        // one knob at a time, in the order of their expected effect; 0 = the default
        struct Knob {
            uint32_t ptc_options::*field;
            std::vector<uint32_t> values;
        };
        const std::vector<Knob> knobs = {
            {&ptc_options::large_rows, {PTC_LARGE_ROWS_AUTO, PTC_LARGE_ROWS_PANELS, PTC_LARGE_ROWS_BITMAP}},
            {&ptc_options::bitmap_max_len, {0, 8, 32}},
            {&ptc_options::panel_width, {0, 64, 128, 256, 512, 1024}},
            {&ptc_options::warp_task_max_len, {0, 64, 1024, 4096}},
            {&ptc_options::small_max_products, {0, 64, 256, 512}},
            {&ptc_options::sort_max_avg_products, {0, 16, 32, 128}},
            {&ptc_options::hash_load_pct, {0, 50, 90}},
        };
        const uint32_t user_panel = opt.panel_width;
        for (const Knob& k : knobs) {
            if (k.field == &ptc_options::panel_width && user_panel != 0) continue;  // the caller fixed it
            // panel knobs matter only where the panel kernels run
            // the bitmap length limit matters only when both kernels share the large rows
            if (k.field == &ptc_options::bitmap_max_len && opt.large_rows != PTC_LARGE_ROWS_AUTO) continue;
            const uint32_t start = opt.*k.field;
            for (uint32_t v : k.values) {
                if (v == start) continue;
                ptc_options cand = opt;
                cand.*k.field = v;
                const double t = time_batch(hi, location, cand, repeats);
                ++rep.trials;
                if (t < best) {
                    best = t;
                    opt = cand;
                }
            }
        }
        rep.best_ms = best;
        *best_out = opt;
        if (report) *report = rep;
        g_last_error.clear();
        return PTC_OK;
    } catch (const Error& e) {
        set_last_error(e.status, e.msg);
        return e.status;
    } catch (const std::bad_alloc&) {
        set_last_error(PTC_ERR_OUT_OF_MEMORY, "host allocation failed");
        return PTC_ERR_OUT_OF_MEMORY;
    } catch (...) {
        set_last_error(PTC_ERR_INTERNAL, "unexpected exception");
        return PTC_ERR_INTERNAL;
    }
}

ptc_status ptc_batch_contract(const ptc_batch_item* items, uint32_t n, const ptc_options* opt_in, ptc_tensor* outs,
                              ptc_batch_sink sink, void* user, ptc_stats* stats_out) {
    using namespace ptc;
    DeviceGuard keep_device;
    try {
        const ptc_options opt = resolve_options(opt_in);
        PTC_REQUIRE(!opt.sort_rows, PTC_ERR_INVALID_ARGUMENT, "sort_rows is for single contractions");
        ptc_stats stats;
        std::memset(&stats, 0, sizeof(stats));
        g_launches = 0;
        uint32_t location = PTC_HOST;
        const std::vector<BatchItemHost> hi = batch_host_items(items, n, location);
        BatchTarget tg;
        tg.outs = outs;
        tg.sink = sink;
        tg.user = user;
        tg.ids.resize(n);
        for (uint32_t i = 0; i < n; ++i) {
            tg.ids[i] = i;
            if (outs) {
                std::memset(&outs[i], 0, sizeof(ptc_tensor));
                outs[i].order = hi[i].fa + hi[i].fb;
                outs[i].location = opt.output_location;
            }
        }
        if (n > 0) {
            try {
                batch_chunks(hi, location, opt, tg, stats);
            } catch (...) {
                if (outs)
                    for (uint32_t i = 0; i < n; ++i) ptc_tensor_free(&outs[i]);
                throw;
            }
        }
        stats.kernel_launches = g_launches;
        if (stats_out) *stats_out = stats;
        g_last_error.clear();
        return PTC_OK;
    } catch (const Error& e) {
        set_last_error(e.status, e.msg);
        return e.status;
    } catch (const std::bad_alloc&) {
        set_last_error(PTC_ERR_OUT_OF_MEMORY, "host allocation failed");
        return PTC_ERR_OUT_OF_MEMORY;
    } catch (...) {
        set_last_error(PTC_ERR_INTERNAL, "unexpected exception");
        return PTC_ERR_INTERNAL;
    }
}

void ptc_tensor_free(ptc_tensor* t) {
    if (!t) return;
    if (t->opaque) {  // a slice of a batch wave's shared block
        ptc::release_block(static_cast<ptc::SharedBlock*>(t->opaque));
    } else if (t->location == PTC_DEVICE) {
        if (t->idx) cudaFree(t->idx);
        if (t->vals) cudaFree(t->vals);
    } else {
        std::free(t->idx);
        std::free(t->vals);
    }
    t->idx = nullptr;
    t->vals = nullptr;
    t->opaque = nullptr;
    t->nnz = 0;
}

ptc_status ptc_device_pool_in_use(int32_t device, uint64_t* bytes) {
    using namespace ptc;
    DeviceGuard keep_device;
    try {
        PTC_REQUIRE(bytes != nullptr, PTC_ERR_INVALID_ARGUMENT, "bytes is null");
        if (device < 0) PTC_CUDA(cudaGetDevice(&device));
        PTC_CUDA(cudaSetDevice(device));
        PTC_CUDA(cudaDeviceSynchronize());
        cudaMemPool_t pool;
        PTC_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
        uint64_t used = 0;
        PTC_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used));
        *bytes = used;
        return PTC_OK;
    } catch (const Error& e) {
        set_last_error(e.status, e.msg);
        return e.status;
    }
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
