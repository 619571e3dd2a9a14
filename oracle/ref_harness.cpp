// Harness around the reference's own, unmodified fksCuckooTC path (test infrastructure only).
//
// It is compiled by oracle/Makefile directly from the reference's headers, where they lie, into
// oracle/_ref/ (git-ignored): a shared library for the tests and a command-line program for the
// CPU baseline.  It replays main.cpp:59-118 of the reference on arrays instead of a .tns file:
//   A           <- the caller's COO arrays plus the meta information (tensor.hpp:151-173)
//   A_copy      <- A with the free modes first in dim_tc (main.cpp:68-109)
//   B           <- get_sparse_tensor(A)                 (main.cpp:112)
//   HT_B, HT_A  <- buildHashTable(B), buildHashTable(A_copy)  (main.cpp:115-116)
//   O           <- tc_fksCuckoo(HT_A, HT_B, A_copy, B)  (main.cpp:118)
// Optionally A_copy keeps only some of A's nonzeros (a row sample for a bounded CPU baseline);
// B is always the whole tensor, so every kept row is computed in full.
// The reference prints its phase timings to stdout; the harness captures and parses them.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <sstream>
#include <string>
#include <vector>

#include "tensor.hpp"
#include "fksCuckoo.hpp"
#include "fksCuckooTC.hpp"
#include "sparse_tensor_generator.hpp"

extern "C" {

struct ref_result {
    uint32_t out_order;
    uint64_t out_nnz;
    uint32_t* out_idx;   // [out_nnz * out_order], the reference's own malloc'd array
    double* out_val;     // [out_nnz]
    double t_insert_b;   // "Total time for insertion" of HT_B (s)
    double t_insert_a;   // "Total time for insertion" of HT_A (s)
    double t_preprocess; // "Total time for preprocessing" (s)
    double t_contract;   // "Total time for tensor contraction" (s)
    double t_wall;       // wall time of the three calls above (s)
};

static void parse_times(const std::string& text, ref_result* r) {
    std::istringstream in(text);
    std::string line;
    int ins = 0;
    auto value_of = [](const std::string& l) {
        size_t eq = l.find('=');
        return eq == std::string::npos ? 0.0 : atof(l.c_str() + eq + 1);
    };
    while (std::getline(in, line)) {
        if (line.find("Total time for insertion") != std::string::npos) {
            if (ins++ == 0) r->t_insert_b = value_of(line); else r->t_insert_a = value_of(line);
        } else if (line.find("Total time for preprocessing") != std::string::npos) {
            r->t_preprocess = value_of(line);
        } else if (line.find("Total time for tensor contraction") != std::string::npos) {
            r->t_contract = value_of(line);
        }
    }
}

// Self-contraction of one COO tensor, exactly as main.cpp does it.  `keep` (nullable, one byte
// per nonzero) selects the nonzeros of A_copy.  Returns 0 on success.  The reference calls exit()
// on an empty contraction and on N <= 1; callers must not pass such inputs.
int ref_self_contract(const uint32_t* idx, const double* vals, uint32_t d, uint32_t N,
                      const uint32_t* dims, uint32_t c, const uint32_t* dim_tc,
                      const uint8_t* keep, int quiet, ref_result* res) {
    Tensor A;
    A.d = d;
    A.N = N;
    A.hedges_array = (unsigned*)malloc(sizeof(unsigned) * (size_t)N * d);
    A.val_array = (double*)malloc(sizeof(double) * (size_t)N);
    A.dimensions_array = (unsigned*)malloc(sizeof(unsigned) * d);
    A.dim_tc = (unsigned*)malloc(sizeof(unsigned) * d);
    for (size_t i = 0; i < (size_t)N * d; ++i) A.hedges_array[i] = idx[i];
    for (size_t i = 0; i < N; ++i) A.val_array[i] = vals[i];
    for (uint32_t j = 0; j < d; ++j) { A.dimensions_array[j] = dims[j]; A.dim_tc[j] = dim_tc[j]; }
    A.num_key_dimensions = c;

    // main.cpp:68-109, with an optional subset of nonzeros kept
    Tensor A_copy;
    A_copy.d = A.d;
    A_copy.num_key_dimensions = A.d - A.num_key_dimensions;
    A_copy.dim_tc = (unsigned*)malloc(sizeof(unsigned) * A_copy.d);
    for (unsigned i = A.num_key_dimensions; i < A.d; ++i) A_copy.dim_tc[i - A.num_key_dimensions] = A.dim_tc[i];
    for (unsigned i = 0; i < A.num_key_dimensions; ++i) A_copy.dim_tc[A.d - A.num_key_dimensions + i] = A.dim_tc[i];
    unsigned kept = 0;
    for (unsigned i = 0; i < A.N; ++i) kept += (keep == nullptr || keep[i]) ? 1u : 0u;
    A_copy.N = kept;
    A_copy.hedges_array = (unsigned*)malloc(sizeof(unsigned) * (size_t)kept * A_copy.d);
    A_copy.val_array = (double*)malloc(sizeof(double) * (size_t)kept);
    for (unsigned i = 0, o = 0; i < A.N; ++i) {
        if (keep != nullptr && !keep[i]) continue;
        for (unsigned xy = 0; xy < A_copy.d; ++xy) A_copy.hedges_array[o * A_copy.d + xy] = A.hedges_array[i * A.d + xy];
        A_copy.val_array[o] = A.val_array[i];
        ++o;
    }
    A_copy.dimensions_array = (unsigned*)malloc(sizeof(unsigned) * A_copy.d);
    for (unsigned j = 0; j < A_copy.d; ++j) A_copy.dimensions_array[j] = A.dimensions_array[j];

    Tensor B = get_sparse_tensor(A);

    std::ostringstream captured;
    std::streambuf* saved = std::cout.rdbuf(captured.rdbuf());
    auto t0 = std::chrono::high_resolution_clock::now();
    Hash_Table* HT_B = buildHashTable(B);
    Hash_Table* HT_A = buildHashTable(A_copy);
    Tensor O = tc_fksCuckoo(HT_A, HT_B, A_copy, B);
    auto t1 = std::chrono::high_resolution_clock::now();
    std::cout.rdbuf(saved);
    if (!quiet) std::cout << captured.str() << std::flush;

    parse_times(captured.str(), res);
    res->t_wall = std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count() * 1e-9;
    res->out_order = O.d;
    res->out_nnz = O.N;
    res->out_idx = O.hedges_array;
    res->out_val = O.val_array;
    // The reference never frees its tensors or hash tables; the harness frees what it made.
    free(A.hedges_array); free(A.val_array); free(A.dimensions_array); free(A.dim_tc);
    free(A_copy.hedges_array); free(A_copy.val_array); free(A_copy.dimensions_array); free(A_copy.dim_tc);
    free(B.hedges_array); free(B.val_array); free(B.dimensions_array); free(B.dim_tc);
    return 0;
}

void ref_free(ref_result* r) {
    free(r->out_idx);
    free(r->out_val);
    r->out_idx = nullptr;
    r->out_val = nullptr;
}

}  // extern "C"

#ifdef PTC_REF_MAIN
// Command-line form used for the CPU baseline:
//   ref_tc <input.bin> [keep.bin] [out.bin]
// input.bin: u32 d, u32 N, u32 c, u32 dims[d], u32 dim_tc[d], u32 idx[N*d], f64 vals[N]
// keep.bin (or "-"): u8 keep[N].  Prints one JSON line with the parsed timings.
static std::vector<char> slurp(const char* path) {
    FILE* f = fopen(path, "rb");
    if (!f) { fprintf(stderr, "cannot open %s\n", path); exit(2); }
    fseek(f, 0, SEEK_END);
    long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    std::vector<char> buf((size_t)n);
    if (n > 0 && fread(buf.data(), 1, (size_t)n, f) != (size_t)n) { fprintf(stderr, "short read\n"); exit(2); }
    fclose(f);
    return buf;
}

int main(int argc, char** argv) {
    if (argc < 2) { fprintf(stderr, "usage: %s input.bin [keep.bin|-] [out.bin]\n", argv[0]); return 2; }
    std::vector<char> in = slurp(argv[1]);
    const uint32_t* h = (const uint32_t*)in.data();
    uint32_t d = h[0], N = h[1], c = h[2];
    const uint32_t* dims = h + 3;
    const uint32_t* dim_tc = dims + d;
    const uint32_t* idx = dim_tc + d;
    const double* vals = (const double*)(idx + (size_t)N * d);
    std::vector<char> keep;
    if (argc >= 3 && std::string(argv[2]) != "-") keep = slurp(argv[2]);
    ref_result r{};
    ref_self_contract(idx, vals, d, N, dims, c, dim_tc, keep.empty() ? nullptr : (const uint8_t*)keep.data(), 1, &r);
    if (argc >= 4) {
        FILE* f = fopen(argv[3], "wb");
        fwrite(&r.out_order, sizeof(uint32_t), 1, f);
        fwrite(&r.out_nnz, sizeof(uint64_t), 1, f);
        fwrite(r.out_idx, sizeof(uint32_t), (size_t)r.out_nnz * r.out_order, f);
        fwrite(r.out_val, sizeof(double), (size_t)r.out_nnz, f);
        fclose(f);
    }
    printf("{\"out_nnz\": %llu, \"t_insert_b\": %.9g, \"t_insert_a\": %.9g, \"t_preprocess\": %.9g, "
           "\"t_contract\": %.9g, \"t_wall\": %.9g}\n",
           (unsigned long long)r.out_nnz, r.t_insert_b, r.t_insert_a, r.t_preprocess, r.t_contract, r.t_wall);
    ref_free(&r);
    return 0;
}
#endif
