// Exclusive scan, stable LSD radix sort and run extraction (see ptc_prims.cuh).
#include "ptc_prims.cuh"

namespace ptc {

// ---------------------------------------------------------------------------------------------
// exclusive scan: tile reduce -> scan of tile sums (recursive) -> tile scan with prefix
// ---------------------------------------------------------------------------------------------

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

template <typename T>
__global__ void __launch_bounds__(kScanThreads) scan_tile_reduce(const T* __restrict__ in, uint64_t n,
                                                                  T* __restrict__ sums) {
    __shared__ T tmp[kScanThreads / 32 + 1];
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile;
    T s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        uint64_t idx = base + (uint64_t)i * kScanThreads + threadIdx.x;
        if (idx < n) s += in[idx];
    }
    T total;
    block_exclusive_scan<T, kScanThreads>(s, tmp, &total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads) scan_tile_apply(const T* __restrict__ in, T* __restrict__ out,
                                                                 uint64_t n, const T* __restrict__ prefix) {
    __shared__ T tmp[kScanThreads / 32 + 1];
    __shared__ T stage[kScanTile];
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile;
    // coalesced load into shared memory, then each thread scans a contiguous run
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        uint64_t idx = base + (uint64_t)i * kScanThreads + threadIdx.x;
        stage[i * kScanThreads + threadIdx.x] = (idx < n) ? in[idx] : T(0);
    }
    __syncthreads();
    T v[kScanItems];
    T s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        v[i] = stage[threadIdx.x * kScanItems + i];
        s += v[i];
    }
    T total;
    T run = block_exclusive_scan<T, kScanThreads>(s, tmp, &total);
    run += prefix ? prefix[blockIdx.x] : T(0);
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        stage[threadIdx.x * kScanItems + i] = run;
        run += v[i];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        uint64_t idx = base + (uint64_t)i * kScanThreads + threadIdx.x;
        if (idx < n) out[idx] = stage[i * kScanThreads + threadIdx.x];
    }
    // the last tile writes the grand total at out[n]
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == kScanThreads - 1) out[n] = run;
}

template <typename T>
__global__ void scan_write_zero(T* out) { out[0] = 0; }

template <typename T>
void exclusive_scan(const T* in, T* out, uint64_t n, Arena& ar) {
    cudaStream_t st = ar.stream();
    if (n == 0) {
        scan_write_zero<T><<<1, 1, 0, st>>>(out);
        count_launch();
        PTC_CHECK_LAUNCH();
        return;
    }
    const uint64_t tiles = (n + kScanTile - 1) / kScanTile;
    T* prefix = nullptr;
    if (tiles > 1) {
        T* sums = ar.alloc<T>(tiles + 1);
        scan_tile_reduce<T><<<(uint32_t)tiles, kScanThreads, 0, st>>>(in, n, sums);
        count_launch();
        PTC_CHECK_LAUNCH();
        exclusive_scan<T>(sums, sums, tiles, ar);  // in place: sums has tiles+1 entries
        prefix = sums;
    }
    scan_tile_apply<T><<<(uint32_t)tiles, kScanThreads, 0, st>>>(in, out, n, prefix);
    count_launch();
    PTC_CHECK_LAUNCH();
}

template void exclusive_scan<uint32_t>(const uint32_t*, uint32_t*, uint64_t, Arena&);
template void exclusive_scan<uint64_t>(const uint64_t*, uint64_t*, uint64_t, Arena&);

// ---------------------------------------------------------------------------------------------
// stable LSD radix sort, 8-bit digits: per-tile histogram -> scan -> stable per-tile scatter
// ---------------------------------------------------------------------------------------------

constexpr int kRsThreads = 256;
constexpr int kRsWarps = kRsThreads / 32;
constexpr int kRsItems = 16;                    // per thread
constexpr int kRsTile = kRsThreads * kRsItems;  // 4096 keys per tile
constexpr int kRsWarpSpan = 32 * kRsItems;      // keys per warp, contiguous

__global__ void __launch_bounds__(kRsThreads) rs_hist(const uint64_t* __restrict__ keys, uint64_t n, int shift,
                                                      uint32_t* __restrict__ hist, uint32_t ntiles) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * kRsTile;
#pragma unroll 4
    for (int i = 0; i < kRsItems; ++i) {
        uint64_t idx = base + (uint64_t)i * kRsThreads + threadIdx.x;
        if (idx < n) atomicAdd(&h[(uint32_t)(keys[idx] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[(uint64_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(kRsThreads) rs_scatter(const uint64_t* __restrict__ kin,
                                                         const uint32_t* __restrict__ vin,
                                                         uint64_t* __restrict__ kout, uint32_t* __restrict__ vout,
                                                         uint64_t n, int shift, const uint32_t* __restrict__ offs,
                                                         uint32_t ntiles) {
    __shared__ uint32_t wcnt[kRsWarps][256];
    const uint32_t w = threadIdx.x >> 5, lane = lane_id();
    for (int i = threadIdx.x; i < kRsWarps * 256; i += kRsThreads) (&wcnt[0][0])[i] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * kRsTile + (uint64_t)w * kRsWarpSpan;
    uint64_t k[kRsItems];
    uint32_t v[kRsItems];
    uint32_t r[kRsItems];
#pragma unroll
    for (int i = 0; i < kRsItems; ++i) {
        const uint64_t idx = base + (uint64_t)i * 32 + lane;
        const bool valid = idx < n;
        uint32_t d = 256;
        if (valid) {
            k[i] = kin[idx];
            v[i] = vin[idx];
            d = (uint32_t)(k[i] >> shift) & 255u;
        }
        const uint32_t m = __match_any_sync(kFullMask, d);
        const uint32_t rank = __popc(m & lanemask_lt());
        uint32_t cnt = 0;
        if (valid) cnt = wcnt[w][d];
        __syncwarp();
        if (valid && rank == 0) wcnt[w][d] = cnt + __popc(m);
        __syncwarp();
        r[i] = cnt + rank;
    }
    __syncthreads();
    // exclusive prefix of the per-warp counts in warp order, plus the tile's global offset
    {
        const uint32_t dgt = threadIdx.x;  // kRsThreads == 256 digits
        uint32_t run = offs[(uint64_t)dgt * ntiles + blockIdx.x];
#pragma unroll
        for (int ww = 0; ww < kRsWarps; ++ww) {
            const uint32_t c = wcnt[ww][dgt];
            wcnt[ww][dgt] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kRsItems; ++i) {
        const uint64_t idx = base + (uint64_t)i * 32 + lane;
        if (idx < n) {
            const uint32_t d = (uint32_t)(k[i] >> shift) & 255u;
            const uint32_t pos = wcnt[w][d] + r[i];
            kout[pos] = k[i];
            vout[pos] = v[i];
        }
    }
}

void radix_sort_pairs(uint64_t* keys, uint32_t* vals, uint64_t n, int begin_bit, int end_bit, Arena& ar) {
    if (n < 2 || end_bit <= begin_bit) return;
    PTC_REQUIRE(n < (1ull << 32), PTC_ERR_INVALID_ARGUMENT, "radix sort supports fewer than 2^32 keys");
    cudaStream_t st = ar.stream();
    const uint32_t ntiles = (uint32_t)((n + kRsTile - 1) / kRsTile);
    uint64_t* k2 = ar.alloc<uint64_t>(n);
    uint32_t* v2 = ar.alloc<uint32_t>(n);
    uint32_t* hist = ar.alloc<uint32_t>((uint64_t)256 * ntiles + 1);
    uint64_t* ksrc = keys;
    uint32_t* vsrc = vals;
    uint64_t* kdst = k2;
    uint32_t* vdst = v2;
    int passes = 0;
    for (int shift = begin_bit; shift < end_bit; shift += 8, ++passes) {
        rs_hist<<<ntiles, kRsThreads, 0, st>>>(ksrc, n, shift, hist, ntiles);
        count_launch();
        PTC_CHECK_LAUNCH();
        exclusive_scan<uint32_t>(hist, hist, (uint64_t)256 * ntiles, ar);
        rs_scatter<<<ntiles, kRsThreads, 0, st>>>(ksrc, vsrc, kdst, vdst, n, shift, hist, ntiles);
        count_launch();
        PTC_CHECK_LAUNCH();
        std::swap(ksrc, kdst);
        std::swap(vsrc, vdst);
    }
    if (ksrc != keys) {
        PTC_CUDA(cudaMemcpyAsync(keys, ksrc, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st));
        PTC_CUDA(cudaMemcpyAsync(vals, vsrc, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    }
}

// ---------------------------------------------------------------------------------------------
// runs of equal keys in a sorted array
// ---------------------------------------------------------------------------------------------

__global__ void mark_heads(const uint64_t* __restrict__ keys, uint64_t n, uint32_t* __restrict__ head) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

__global__ void emit_runs(const uint64_t* __restrict__ keys, uint64_t n, const uint32_t* __restrict__ head_scan,
                          uint32_t* __restrict__ run_of, uint32_t* __restrict__ run_start,
                          uint64_t* __restrict__ run_key) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const uint32_t before = head_scan[i];        // heads in [0, i)
        const bool is_head = head_scan[i + 1] != before;
        const uint32_t r = is_head ? before : before - 1;
        if (run_of) run_of[i] = r;
        if (is_head) {
            if (run_start) run_start[r] = (uint32_t)i;
            if (run_key) run_key[r] = keys[i];
        }
    }
    if (i == n - 1 && run_start) run_start[head_scan[n]] = (uint32_t)n;
}

uint64_t runs_of_sorted(const uint64_t* keys, uint64_t n, uint32_t* run_of, uint32_t* run_start,
                        uint64_t* run_key, Arena& ar) {
    if (n == 0) return 0;
    cudaStream_t st = ar.stream();
    uint32_t* head = ar.alloc<uint32_t>(n + 1);
    const uint32_t grid = ceil_div_u32(n, 256);
    mark_heads<<<grid, 256, 0, st>>>(keys, n, head);
    count_launch();
    PTC_CHECK_LAUNCH();
    exclusive_scan<uint32_t>(head, head, n, ar);
    emit_runs<<<grid, 256, 0, st>>>(keys, n, head, run_of, run_start, run_key);
    count_launch();
    PTC_CHECK_LAUNCH();
    uint32_t nruns = 0;
    PTC_CUDA(cudaMemcpyAsync(&nruns, head + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    PTC_CUDA(cudaStreamSynchronize(st));
    return nruns;
}

}  // namespace ptc
