// FROSTT .tns input on the GPU (ptc_read_tns, include/partc.h) and .tns output (ptc_write_tns).
//
// The reference reads a tensor with pigo (readTensor, mtxTnsIO.cpp:30-65): one nonzero per line,
// d 1-based labels then the value; d is the number of labels on a line, each mode's size its
// largest label.  Here the file's bytes go to the device once, and kernels
//   1. count the line breaks of every 64 KiB chunk, scan the counts and list the line starts;
//   2. parse one line per thread: the labels as integers, the value with pigo's own arithmetic
//      (read_fp, extern/pigo/pigo.hpp:2587-2627: integer part res = res*10 + digit, fraction
//      likewise, res += fraction / 10^count, then res *= 10^exponent), with the powers of ten
//      computed by the host's std::pow -- the same function the reference calls -- so values are
//      bit-identical to the reference reader's;
//   3. compact the data lines (comments '#'/'%' and blank lines dropped) and take each mode's
//      largest label.
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "partc.h"
#include "ptc_build.cuh"
#include "ptc_prims.cuh"
#include "ptc_learned.cuh"

namespace ptc {

void set_last_error(ptc_status, const std::string& msg);

namespace {

constexpr uint64_t kChunk = 64 * 1024;
constexpr int kPow10Min = -340, kPow10Max = 340;  // table of std::pow(10., n) for the parser

__global__ void count_breaks_kernel(const char* __restrict__ buf, uint64_t n, uint32_t* __restrict__ cnt) {
    const uint64_t c = blockIdx.x;
    const uint64_t lo = c * kChunk, hi = min(lo + kChunk, n);
    __shared__ uint32_t total;
    if (threadIdx.x == 0) total = 0;
    __syncthreads();
    uint32_t k = 0;
    for (uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) k += buf[i] == '\n';
    k = warp_sum(k);
    if ((threadIdx.x & 31) == 0) atomicAdd(&total, k);
    __syncthreads();
    if (threadIdx.x == 0) cnt[c] = total;
}

// line r (r >= 1) starts after the r-th line break; line 0 at byte 0
__global__ void line_starts_kernel(const char* __restrict__ buf, uint64_t n, const uint32_t* __restrict__ off,
                                   uint64_t* __restrict__ start) {
    const uint64_t c = blockIdx.x;
    const uint64_t lo = c * kChunk, hi = min(lo + kChunk, n);
    __shared__ uint32_t base;
    if (threadIdx.x == 0) base = off[c];
    __syncthreads();
    // warps walk the chunk in order, 32 bytes at a time
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (warp != 0) return;
    uint32_t b = base;
    for (uint64_t i = lo; i < hi; i += 32) {
        const uint64_t j = i + lane;
        const bool br = j < hi && buf[j] == '\n';
        const uint32_t m = __ballot_sync(0xffffffffu, br);
        if (br) start[b + __popc(m & ((1u << lane) - 1u)) + 1] = j + 1;
        b += __popc(m);
    }
    if (c == 0 && lane == 0) start[0] = 0;
}

__device__ __forceinline__ bool is_digit(char ch) { return ch >= '0' && ch <= '9'; }
__device__ __forceinline__ bool is_fp_char(char ch) {
    return is_digit(ch) || ch == 'e' || ch == 'E' || ch == '-' || ch == '+' || ch == '.';
}

// pigo's read_fp on [p, e): returns the value and advances p (see the file comment).  pigo
// raises the value to 10^exponent with std::pow for any exponent it reads, itself parsed by
// read_fp (so "2e0.5" and "3e1e1" are numbers to it).  The table covers every integral exponent;
// a line whose exponent is not an integer, or holds an exponent of its own, gets `host` set and
// its value is computed again on the host with std::pow, as pigo does.
__device__ double parse_fp(const char*& p, const char* e, const double* __restrict__ pow10, int depth,
                           uint32_t& host) {
    double res = 0.0;
    while (p < e && !is_fp_char(*p)) ++p;
    bool positive = true;
    if (p < e && *p == '-') {
        positive = false;
        ++p;
    } else if (p < e && *p == '+') {
        ++p;
    }
    while (p < e && is_digit(*p)) {
        res = __dadd_rn(__dmul_rn(res, 10.0), (double)(*p - '0'));
        ++p;
    }
    if (p < e && *p == '.') {
        ++p;
        double fraction = 0.0;
        int count = 0;
        while (p < e && is_digit(*p)) {
            fraction = __dadd_rn(__dmul_rn(fraction, 10.0), (double)(*p - '0'));
            ++p;
            ++count;
        }
        const double scale = count <= kPow10Max ? pow10[count - kPow10Min] : INFINITY;
        res = __dadd_rn(res, __ddiv_rn(fraction, scale));
    }
    if (p < e && (*p == 'e' || *p == 'E')) {
        if (depth > 0) {  // an exponent with an exponent of its own: pigo recurses; the host does it
            host = 1;
            return positive ? res : -res;
        }
        ++p;
        const double ex = parse_fp(p, e, pow10, 1, host);
        if (ex != floor(ex)) {
            host = 1;  // non-integral (or NaN) exponent: std::pow on the host
        } else {
            const double k = fmin(fmax(ex, (double)kPow10Min), (double)kPow10Max);
            // beyond the table, 10^ex is inf or 0 in double, as std::pow gives
            res = __dmul_rn(res, k == ex ? pow10[(int)k - kPow10Min] : (ex > 0 ? INFINITY : 0.0));
        }
    }
    return positive ? res : -res;
}

// One thread per line: d labels and a value, or nothing for a comment or blank line.
__global__ void parse_lines_kernel(const char* __restrict__ buf, uint64_t n, const uint64_t* __restrict__ start,
                                   uint64_t nlines, uint32_t d, const double* __restrict__ pow10,
                                   uint32_t* __restrict__ idx, double* __restrict__ val, uint32_t* __restrict__ keep,
                                   uint32_t* __restrict__ host_line, uint32_t* __restrict__ err) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nlines) return;
    const char* p = buf + start[r];
    const char* e = buf + (r + 1 < nlines ? start[r + 1] : n);
    const char* q = p;
    while (q < e && (*q == ' ' || *q == '\t' || *q == '\r')) ++q;
    if (q >= e || *q == '\n' || *q == '#' || *q == '%') {
        keep[r] = 0;
        return;
    }
    keep[r] = 1;
    {  // a data line holds d labels and one value
        uint32_t tokens = 0;
        bool in = false;
        for (const char* x = q; x < e && *x != '\n'; ++x) {
            const bool sp = *x == ' ' || *x == '\t' || *x == '\r';
            if (!sp && !in) ++tokens;
            in = !sp;
        }
        if (tokens != d + 1) {
            atomicOr(err, 1u);
            return;
        }
    }
    for (uint32_t m = 0; m < d; ++m) {
        while (q < e && !is_digit(*q) && *q != '\n') ++q;
        if (q >= e || !is_digit(*q)) {
            atomicOr(err, 1u);  // a label that is not a number
            return;
        }
        uint64_t v = 0;
        while (q < e && is_digit(*q)) {
            v = v * 10 + (uint64_t)(*q - '0');
            ++q;
        }
        if (v == 0 || v > 0xffffffffull) atomicOr(err, 2u);  // labels are 1-based and fit 32 bits
        idx[r * d + m] = (uint32_t)(v - 1);
    }
    uint32_t host = 0;
    val[r] = parse_fp(q, e, pow10, 0, host);
    if (host) host_line[r] = 1;
}

// val[line[i]] = v[i]
__global__ void patch_values_kernel(const uint64_t* __restrict__ line, const double* __restrict__ v, uint32_t n,
                                    double* __restrict__ val) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) val[line[i]] = v[i];
}

bool host_fp_char(char ch) {
    return (ch >= '0' && ch <= '9') || ch == 'e' || ch == 'E' || ch == '-' || ch == '+' || ch == '.';
}

// pigo's read_fp on the host (extern/pigo/pigo.hpp:2587-2627): integer and fraction parts
// accumulated in double, res += fraction / std::pow(10, digits), then res *= std::pow(10, exp)
// with the exponent read by the same routine.
double host_read_fp(const char*& p, const char* e) {
    double res = 0.0;
    while (p < e && !host_fp_char(*p)) ++p;
    bool positive = true;
    if (p < e && *p == '-') {
        positive = false;
        ++p;
    } else if (p < e && *p == '+') {
        ++p;
    }
    while (p < e && *p >= '0' && *p <= '9') res = res * 10. + (double)(*p++ - '0');
    if (p < e && *p == '.') {
        ++p;
        double fraction = 0.;
        size_t count = 0;
        while (p < e && *p >= '0' && *p <= '9') {
            fraction = fraction * 10. + (double)(*p++ - '0');
            ++count;
        }
        res += fraction / std::pow(10., (double)count);
    }
    if (p < e && (*p == 'e' || *p == 'E')) {
        ++p;
        const double ex = host_read_fp(p, e);
        res *= std::pow(10., ex);
    }
    if (!positive) res *= -1;
    return res;
}

// The value of data line [p, e) with d labels, by host_read_fp.
double host_line_value(const char* p, const char* e, uint32_t d) {
    for (uint32_t m = 0; m < d; ++m) {
        while (p < e && !(*p >= '0' && *p <= '9')) ++p;
        while (p < e && *p >= '0' && *p <= '9') ++p;
    }
    return host_read_fp(p, e);
}

__global__ void compact_lines_kernel(const uint32_t* __restrict__ idx, const double* __restrict__ val,
                                     const uint32_t* __restrict__ keep, const uint32_t* __restrict__ pos,
                                     uint64_t nlines, uint32_t d, uint32_t* __restrict__ out_idx,
                                     double* __restrict__ out_val, uint32_t* __restrict__ dims) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nlines || !keep[r]) return;
    const uint64_t o = pos[r];
    for (uint32_t m = 0; m < d; ++m) {
        const uint32_t v = idx[r * d + m];
        out_idx[o * d + m] = v;
        atomicMax(&dims[m], v + 1);  // the mode's size is its largest label
    }
    out_val[o] = val[r];
}

// number of labels on the first data line (labels, then one value)
uint32_t first_line_order(const char* buf, size_t n) {
    size_t i = 0;
    while (i < n) {
        size_t e = i;
        while (e < n && buf[e] != '\n') ++e;
        size_t q = i;
        while (q < e && (buf[q] == ' ' || buf[q] == '\t' || buf[q] == '\r')) ++q;
        if (q < e && buf[q] != '#' && buf[q] != '%') {
            uint32_t tokens = 0;
            bool in = false;
            for (size_t k = q; k < e; ++k) {
                const bool sp = buf[k] == ' ' || buf[k] == '\t' || buf[k] == '\r';
                if (!sp && !in) ++tokens;
                in = !sp;
            }
            return tokens >= 2 ? tokens - 1 : 0;
        }
        i = e + 1;
    }
    return 0;
}

}  // namespace
}  // namespace ptc

extern "C" ptc_status ptc_read_tns(const char* path, const ptc_options* opt_in, ptc_tensor* out, uint32_t* dims_out) {
    using namespace ptc;
    DeviceGuard keep_device;
    std::vector<char> host;
    try {
        PTC_REQUIRE(path && out && dims_out, PTC_ERR_INVALID_ARGUMENT, "null argument");
        std::memset(out, 0, sizeof(*out));
        ptc_options opt;
        ptc_options_init(&opt);
        if (opt_in) std::memcpy(&opt, opt_in, std::min<size_t>(opt_in->struct_size, sizeof(opt)));
        const int fd = open(path, O_RDONLY);
        PTC_REQUIRE(fd >= 0, PTC_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path);
        struct stat sb;
        fstat(fd, &sb);
        host.resize((size_t)sb.st_size + 1);
        size_t got = 0;
        while (got < (size_t)sb.st_size) {
            const ssize_t k = read(fd, host.data() + got, (size_t)sb.st_size - got);
            if (k <= 0) break;
            got += (size_t)k;
        }
        close(fd);
        PTC_REQUIRE(got == (size_t)sb.st_size, PTC_ERR_INVALID_ARGUMENT, std::string("cannot read ") + path);
        const uint64_t n = got;
        const uint32_t d = first_line_order(host.data(), n);
        PTC_REQUIRE(d >= 1 && d <= 16, PTC_ERR_INVALID_ARGUMENT, "no data line with 1..16 labels and a value");

        int device = opt.device;
        if (device < 0) PTC_CUDA(cudaGetDevice(&device));
        PTC_CUDA(cudaSetDevice(device));
        cudaStream_t st = opt.stream ? static_cast<cudaStream_t>(opt.stream) : cudaStreamPerThread;
        Arena ar(st);
        char* dbuf = ar.alloc<char>(n + 1);
        PTC_CUDA(cudaMemcpyAsync(dbuf, host.data(), n, cudaMemcpyHostToDevice, st));
        std::vector<double> hp(kPow10Max - kPow10Min + 1);
        for (int k = kPow10Min; k <= kPow10Max; ++k) hp[k - kPow10Min] = std::pow(10., (double)k);
        double* pow10 = ar.alloc<double>(hp.size());
        PTC_CUDA(cudaMemcpyAsync(pow10, hp.data(), hp.size() * sizeof(double), cudaMemcpyHostToDevice, st));

        // 1. line starts
        const uint64_t nchunks = (n + kChunk - 1) / kChunk;
        uint32_t* cnt = ar.alloc<uint32_t>(nchunks + 1);
        count_breaks_kernel<<<(unsigned)nchunks, 256, 0, st>>>(dbuf, n, cnt);
        PTC_CUDA(cudaGetLastError());
        // the line positions below are 32-bit: count the breaks in 64 bits first and refuse files
        // with 2^32 - 1 lines or more instead of wrapping
        uint64_t* nbreaks64 = ar.alloc<uint64_t>(1);
        launch_sum_u32(cnt, nchunks, nbreaks64, st);
        uint64_t total_breaks = 0;
        PTC_CUDA(cudaMemcpyAsync(&total_breaks, nbreaks64, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
        PTC_CUDA(cudaStreamSynchronize(st));
        PTC_REQUIRE(total_breaks + 1 < (uint64_t)UINT32_MAX, PTC_ERR_INVALID_ARGUMENT,
                    "the file has 2^32 - 1 lines or more");
        exclusive_scan<uint32_t>(cnt, cnt, nchunks, ar);
        const uint32_t nbreaks = (uint32_t)total_breaks;
        const uint64_t nlines = (uint64_t)nbreaks + 1;  // the text after the last break is a line too
        uint64_t* start = ar.alloc<uint64_t>(nlines + 1);
        line_starts_kernel<<<(unsigned)nchunks, 32, 0, st>>>(dbuf, n, cnt, start);
        PTC_CUDA(cudaGetLastError());

        // 2. parse
        uint32_t* tidx = ar.alloc<uint32_t>(nlines * d);
        double* tval = ar.alloc<double>(nlines);
        uint32_t* keep = ar.alloc<uint32_t>(nlines + 1);
        uint32_t* err = ar.alloc<uint32_t>(1);
        PTC_CUDA(cudaMemsetAsync(err, 0, sizeof(uint32_t), st));
        uint32_t* host_line = ar.alloc<uint32_t>(nlines);
        PTC_CUDA(cudaMemsetAsync(host_line, 0, nlines * sizeof(uint32_t), st));
        const unsigned grid = (unsigned)((nlines + 255) / 256);
        parse_lines_kernel<<<grid, 256, 0, st>>>(dbuf, n, start, nlines, d, pow10, tidx, tval, keep, host_line, err);
        PTC_CUDA(cudaGetLastError());
        uint32_t herr = 0;
        PTC_CUDA(cudaMemcpyAsync(&herr, err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        // lines whose exponent needs std::pow (non-integral or nested exponents; normally none)
        uint64_t* nhost_d = ar.alloc<uint64_t>(1);
        launch_sum_u32(host_line, nlines, nhost_d, st);
        uint64_t nhost = 0;
        PTC_CUDA(cudaMemcpyAsync(&nhost, nhost_d, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
        PTC_CUDA(cudaStreamSynchronize(st));
        if (nhost > 0) {
            std::vector<uint32_t> hl(nlines);
            std::vector<uint64_t> hs(nlines + 1);
            PTC_CUDA(cudaMemcpyAsync(hl.data(), host_line, nlines * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
            PTC_CUDA(cudaMemcpyAsync(hs.data(), start, nlines * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
            PTC_CUDA(cudaStreamSynchronize(st));
            std::vector<uint64_t> lines;
            std::vector<double> vals;
            for (uint64_t r = 0; r < nlines; ++r) {
                if (!hl[r]) continue;
                const uint64_t e = r + 1 < nlines ? hs[r + 1] : n;
                lines.push_back(r);
                vals.push_back(host_line_value(host.data() + hs[r], host.data() + e, d));
            }
            uint64_t* dl = ar.alloc<uint64_t>(lines.size());
            double* dvv = ar.alloc<double>(vals.size());
            PTC_CUDA(cudaMemcpyAsync(dl, lines.data(), lines.size() * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
            PTC_CUDA(cudaMemcpyAsync(dvv, vals.data(), vals.size() * sizeof(double), cudaMemcpyHostToDevice, st));
            patch_values_kernel<<<ceil_div_u32(lines.size(), 256), 256, 0, st>>>(dl, dvv, (uint32_t)lines.size(), tval);
            PTC_CUDA(cudaGetLastError());
            PTC_CUDA(cudaStreamSynchronize(st));  // the host vectors stay alive until the copies are done
        }

        // 3. compact and mode sizes
        uint32_t* pos = ar.alloc<uint32_t>(nlines + 1);
        exclusive_scan<uint32_t>(keep, pos, nlines, ar);
        uint32_t nnz = 0;
        PTC_CUDA(cudaMemcpyAsync(&nnz, pos + nlines, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        PTC_CUDA(cudaStreamSynchronize(st));
        PTC_REQUIRE((herr & 1u) == 0, PTC_ERR_INVALID_ARGUMENT,
                    "a data line does not hold as many labels as the first one, plus a value");
        PTC_REQUIRE((herr & 2u) == 0, PTC_ERR_INDEX_RANGE, "a label is 0 or does not fit 32 bits (labels are 1-based)");
        uint32_t* dims = ar.alloc<uint32_t>(16);
        PTC_CUDA(cudaMemsetAsync(dims, 0, 16 * sizeof(uint32_t), st));
        uint32_t* oidx = nullptr;
        double* oval = nullptr;
        PTC_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&oidx), std::max<uint64_t>((uint64_t)nnz * d, 1) * 4, st));
        PTC_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&oval), std::max<uint64_t>(nnz, 1) * 8, st));
        // `out` owns the device arrays from here on, so every error path below releases them
        out->location = PTC_DEVICE;
        out->idx = oidx;
        out->vals = oval;
        out->order = d;
        compact_lines_kernel<<<grid, 256, 0, st>>>(tidx, tval, keep, pos, nlines, d, oidx, oval, dims);
        PTC_CUDA(cudaGetLastError());
        PTC_CUDA(cudaMemcpyAsync(dims_out, dims, d * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        if (opt.output_location != PTC_DEVICE) {
            uint32_t* hidx = static_cast<uint32_t*>(std::malloc(std::max<uint64_t>((uint64_t)nnz * d, 1) * 4));
            double* hval = static_cast<double*>(std::malloc(std::max<uint64_t>(nnz, 1) * 8));
            if (!hidx || !hval) {
                std::free(hidx);
                std::free(hval);
                throw Error{PTC_ERR_OUT_OF_MEMORY, "host allocation failed"};
            }
            const cudaError_t e1 = cudaMemcpyAsync(hidx, oidx, (uint64_t)nnz * d * 4, cudaMemcpyDeviceToHost, st);
            const cudaError_t e2 = cudaMemcpyAsync(hval, oval, (uint64_t)nnz * 8, cudaMemcpyDeviceToHost, st);
            const cudaError_t e3 = cudaStreamSynchronize(st);
            if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
                std::free(hidx);
                std::free(hval);
                PTC_CUDA(e1 != cudaSuccess ? e1 : e2 != cudaSuccess ? e2 : e3);
            }
            cudaFreeAsync(oidx, st);
            cudaFreeAsync(oval, st);
            out->location = PTC_HOST;
            out->idx = hidx;
            out->vals = hval;
        }
        ar.release();
        PTC_CUDA(cudaStreamSynchronize(st));
        out->nnz = nnz;
        return PTC_OK;
    } catch (const Error& e) {
        ptc_tensor_free(out);
        set_last_error(e.status, e.msg);
        return e.status;
    } catch (const std::bad_alloc&) {
        ptc_tensor_free(out);
        set_last_error(PTC_ERR_OUT_OF_MEMORY, "host allocation failed");
        return PTC_ERR_OUT_OF_MEMORY;
    } catch (...) {
        ptc_tensor_free(out);
        set_last_error(PTC_ERR_INTERNAL, "unexpected exception");
        return PTC_ERR_INTERNAL;
    }
}

extern "C" ptc_status ptc_write_tns(const char* path, const ptc_tensor* t) {
    using namespace ptc;
    try {
        PTC_REQUIRE(path && t, PTC_ERR_INVALID_ARGUMENT, "null argument");
        PTC_REQUIRE(t->nnz == 0 || (t->idx && t->vals), PTC_ERR_INVALID_ARGUMENT, "tensor without arrays");
        std::vector<uint32_t> idx;
        std::vector<double> val;
        const uint32_t* ip = t->idx;
        const double* vp = t->vals;
        if (t->location == PTC_DEVICE && t->nnz > 0) {
            idx.resize(t->nnz * t->order);
            val.resize(t->nnz);
            PTC_CUDA(cudaMemcpy(idx.data(), t->idx, idx.size() * 4, cudaMemcpyDeviceToHost));
            PTC_CUDA(cudaMemcpy(val.data(), t->vals, val.size() * 8, cudaMemcpyDeviceToHost));
            ip = idx.data();
            vp = val.data();
        }
        FILE* f = std::fopen(path, "w");
        PTC_REQUIRE(f != nullptr, PTC_ERR_INVALID_ARGUMENT, std::string("cannot write ") + path);
        std::vector<char> line(32 * (t->order + 2));
        for (uint64_t e = 0; e < t->nnz; ++e) {
            int k = 0;
            for (uint32_t m = 0; m < t->order; ++m)
                k += std::snprintf(line.data() + k, line.size() - k, "%u ", ip[e * t->order + m] + 1);
            k += std::snprintf(line.data() + k, line.size() - k, "%.17g\n", vp[e]);
            std::fwrite(line.data(), 1, (size_t)k, f);
        }
        const bool ok = std::fclose(f) == 0;
        PTC_REQUIRE(ok, PTC_ERR_INVALID_ARGUMENT, std::string("write failed: ") + path);
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
