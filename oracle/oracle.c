/*
 * CPU restatement of parTC's fksCuckooTC contraction -- TEST INFRASTRUCTURE, the checker.
 *
 * Only the tests, the smoke check and the CPU-baseline leg of the benchmark may load this file's
 * library.  The product (partc_b200) never links, imports or calls it.
 *
 * What it restates (reference files, by path within the parTC project):
 *   - tc_fksCuckoo, fksCuckooTC.hpp:80-371: row-wise Gustavson contraction
 *       O[f_A, f_B] = sum_c A[f_A, c] * B[c, f_B]
 *     where a "row" is the set of A nonzeros sharing A's free-mode tuple (HT_A, main.cpp:116)
 *     and a "fiber" is the set of B nonzeros sharing B's contracted-mode tuple (HT_B,
 *     main.cpp:115).
 *   - the symbolic pass, fksCuckooTC.hpp:94-154: flops(row) = sum of |fiber| over the row.
 *   - the numeric pass, fksCuckooTC.hpp:180-357: for each row with flops > 0, a sparse
 *     accumulator keyed by B's free-mode tuple; the row's A nonzeros are visited in COO input
 *     order (Aux_data keeps insertion order, fksCuckoo.hpp:233-255) and each fiber in B's input
 *     order (reorder_tensor, fksCuckooTC.hpp:31-77); the value of an output entry is the left
 *     fold  ((a1*b1) + a2*b2) + ...  in that order, the product rounded first (no FMA, as the
 *     reference's x86-64 build without -march has none).  New keys are appended in
 *     first-appearance order (ele_count_SPA, fksCuckooTC.hpp:283,326-330).
 *   - output tuple = A's free modes in meta order, then B's free modes in meta order
 *     (fksCuckooTC.hpp:216-218,241,349-352).
 * The reference's FKS/cuckoo tables only decide WHERE entries live; they never change which
 * entries exist or the order of any sum, so the restatement groups by sorting instead of
 * hashing.  Rows are emitted in increasing linearized free-key order (the reference's row order
 * is hash order, so comparisons are made on sorted outputs).
 *
 * Parity of this restatement is pinned against the reference itself (oracle/_ref, built from the
 * reference's own sources) by tests/test_oracle_pin.py and by golden fixtures.
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>

static void set_err(oracle_result* r, const char* m) {
    size_t n = strlen(m);
    if (n >= sizeof(r->err)) n = sizeof(r->err) - 1;
    memcpy(r->err, m, n);
    r->err[n] = 0;
}

/* Stable LSD radix sort of (key, payload) pairs on the low `bits` bits of the key. */
static int radix_sort_pairs(uint64_t* keys, uint64_t* pay, uint64_t n, int bits) {
    if (n < 2 || bits <= 0) return 0;
    uint64_t* k2 = (uint64_t*)malloc(sizeof(uint64_t) * n);
    uint64_t* p2 = (uint64_t*)malloc(sizeof(uint64_t) * n);
    size_t* cnt = (size_t*)malloc(sizeof(size_t) * 65536);
    if (!k2 || !p2 || !cnt) { free(k2); free(p2); free(cnt); return -1; }
    uint64_t *sk = keys, *sp = pay, *dk = k2, *dp = p2;
    for (int shift = 0; shift < bits; shift += 16) {
        memset(cnt, 0, sizeof(size_t) * 65536);
        for (uint64_t i = 0; i < n; ++i) cnt[(sk[i] >> shift) & 0xFFFF]++;
        size_t run = 0;
        for (int b = 0; b < 65536; ++b) { size_t t = cnt[b]; cnt[b] = run; run += t; }
        for (uint64_t i = 0; i < n; ++i) {
            size_t o = cnt[(sk[i] >> shift) & 0xFFFF]++;
            dk[o] = sk[i];
            dp[o] = sp[i];
        }
        uint64_t* t;
        t = sk; sk = dk; dk = t;
        t = sp; sp = dp; dp = t;
    }
    if (sk != keys) {
        memcpy(keys, sk, sizeof(uint64_t) * n);
        memcpy(pay, sp, sizeof(uint64_t) * n);
    }
    free(k2); free(p2); free(cnt);
    return 0;
}

static int bits_for(uint64_t space) {
    int b = 0;
    while (b < 64 && (space - 1) >> b) ++b;
    return b;
}

/* Mixed-radix linearization of the tuple (idx[modes[0]], idx[modes[1]], ...), first mode most
 * significant.  Returns 0 and sets *space, or -1 if the key space does not fit in 64 bits. */
static int key_space(const uint32_t* dims, const uint32_t* modes, uint32_t nm, uint64_t* space) {
    unsigned __int128 s = 1;
    for (uint32_t j = 0; j < nm; ++j) {
        s *= (unsigned __int128)(dims[modes[j]] ? dims[modes[j]] : 1);
        if (s > (unsigned __int128)UINT64_MAX) return -1;
    }
    *space = (uint64_t)s;
    return 0;
}

static inline uint64_t lin_key(const uint32_t* row, const uint32_t* dims, const uint32_t* modes, uint32_t nm) {
    uint64_t k = 0;
    for (uint32_t j = 0; j < nm; ++j) k = k * (uint64_t)dims[modes[j]] + (uint64_t)row[modes[j]];
    return k;
}

/* Open-addressing map from a 64-bit key to a dense position, used as the row accumulator. */
typedef struct {
    uint64_t* keys;
    uint32_t* pos;
    uint64_t cap;   /* power of two */
} spa_map;

static inline uint64_t mix64(uint64_t x) {
    x ^= x >> 33; x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return x;
}

int oracle_contract(const oracle_coo* A, const oracle_coo* B, uint32_t c,
                    const uint32_t* a_modes, const uint32_t* b_modes, int mode, oracle_result* r) {
    memset(r, 0, sizeof(*r));
    if (!A || !B || !a_modes || !b_modes) { set_err(r, "null argument"); return ORACLE_EINVAL; }
    if (c == 0 || c >= A->order || c >= B->order) { set_err(r, "need 0 < c < order"); return ORACLE_EINVAL; }
    const uint32_t da = A->order, db = B->order;
    const uint32_t fa = da - c, fb = db - c;
    for (uint32_t j = 0; j < c; ++j)
        if (A->dims[a_modes[j]] != B->dims[b_modes[j]]) { set_err(r, "contracted mode sizes differ"); return ORACLE_EINVAL; }

    uint64_t cspace, faspace, fbspace;
    if (key_space(B->dims, b_modes, c, &cspace) || key_space(A->dims, a_modes + c, fa, &faspace) ||
        key_space(B->dims, b_modes + c, fb, &fbspace)) {
        set_err(r, "key space exceeds 64 bits");
        return ORACLE_EINVAL;
    }
    for (uint64_t i = 0; i < A->nnz; ++i)
        for (uint32_t m = 0; m < da; ++m)
            if (A->idx[i * da + m] >= A->dims[m]) { set_err(r, "A index out of range"); return ORACLE_EINVAL; }
    for (uint64_t i = 0; i < B->nnz; ++i)
        for (uint32_t m = 0; m < db; ++m)
            if (B->idx[i * db + m] >= B->dims[m]) { set_err(r, "B index out of range"); return ORACLE_EINVAL; }

    /* --- B: fibers by contracted key (HT_B + reorder_tensor) --- */
    uint64_t nb = B->nnz, na = A->nnz;
    uint64_t* bkey = (uint64_t*)malloc(sizeof(uint64_t) * (nb ? nb : 1));
    uint64_t* bperm = (uint64_t*)malloc(sizeof(uint64_t) * (nb ? nb : 1));
    uint64_t* bfree = (uint64_t*)malloc(sizeof(uint64_t) * (nb ? nb : 1));
    uint64_t* akey = (uint64_t*)malloc(sizeof(uint64_t) * (na ? na : 1));
    uint64_t* aperm = (uint64_t*)malloc(sizeof(uint64_t) * (na ? na : 1));
    if (!bkey || !bperm || !bfree || !akey || !aperm) { set_err(r, "out of memory"); return ORACLE_ENOMEM; }
    for (uint64_t i = 0; i < nb; ++i) {
        bkey[i] = lin_key(B->idx + i * db, B->dims, b_modes, c);
        bfree[i] = lin_key(B->idx + i * db, B->dims, b_modes + c, fb);
        bperm[i] = i;
    }
    radix_sort_pairs(bkey, bperm, nb, bits_for(cspace));
    uint64_t nfib = 0;
    for (uint64_t i = 0; i < nb; ++i) if (i == 0 || bkey[i] != bkey[i - 1]) ++nfib;
    uint64_t* fkey = (uint64_t*)malloc(sizeof(uint64_t) * (nfib + 1));
    uint64_t* fstart = (uint64_t*)malloc(sizeof(uint64_t) * (nfib + 1));
    for (uint64_t i = 0, f = 0; i < nb; ++i)
        if (i == 0 || bkey[i] != bkey[i - 1]) { fkey[f] = bkey[i]; fstart[f] = i; ++f; }
    fstart[nfib] = nb;

    /* --- A: rows by free key (HT_A on A_copy, main.cpp:68-116) --- */
    for (uint64_t i = 0; i < na; ++i) {
        akey[i] = lin_key(A->idx + i * da, A->dims, a_modes + c, fa);
        aperm[i] = i;
    }
    radix_sort_pairs(akey, aperm, na, bits_for(faspace));
    uint64_t nrows = 0;
    for (uint64_t i = 0; i < na; ++i) if (i == 0 || akey[i] != akey[i - 1]) ++nrows;
    r->nrows = nrows;
    r->row_key = (uint64_t*)malloc(sizeof(uint64_t) * (nrows + 1));
    r->row_flops = (uint64_t*)malloc(sizeof(uint64_t) * (nrows + 1));
    r->row_nnz = (uint64_t*)malloc(sizeof(uint64_t) * (nrows + 1));
    r->row_len = (uint32_t*)malloc(sizeof(uint32_t) * (nrows + 1));
    uint64_t* rstart = (uint64_t*)malloc(sizeof(uint64_t) * (nrows + 1));
    /* fiber of each A nonzero, by binary search on the sorted fiber keys (HT_B->find_element_new) */
    int64_t* afib = (int64_t*)malloc(sizeof(int64_t) * (na ? na : 1));
    for (uint64_t i = 0, q = 0; i < na; ++i) {
        if (i == 0 || akey[i] != akey[i - 1]) { r->row_key[q] = akey[i]; rstart[q] = i; ++q; }
    }
    rstart[nrows] = na;
    for (uint64_t s = 0; s < na; ++s) {
        uint64_t i = aperm[s];
        uint64_t k = lin_key(A->idx + i * da, A->dims, a_modes, c);
        uint64_t lo = 0, hi = nfib;
        while (lo < hi) { uint64_t mid = (lo + hi) >> 1; if (fkey[mid] < k) lo = mid + 1; else hi = mid; }
        afib[s] = (lo < nfib && fkey[lo] == k) ? (int64_t)lo : -1;
    }
    /* symbolic pass (fksCuckooTC.hpp:94-154) */
    uint64_t flops = 0;
    for (uint64_t q = 0; q < nrows; ++q) {
        uint64_t f = 0;
        for (uint64_t s = rstart[q]; s < rstart[q + 1]; ++s)
            if (afib[s] >= 0) f += fstart[afib[s] + 1] - fstart[afib[s]];
        r->row_flops[q] = f;
        r->row_len[q] = (uint32_t)(rstart[q + 1] - rstart[q]);
        r->row_nnz[q] = 0;
        flops += f;
    }
    r->flops = flops;
    r->out_order = fa + fb;
    r->nfibers = nfib;

    if (mode != ORACLE_FLOPS_ONLY) {
        /* numeric pass (fksCuckooTC.hpp:180-357), one sparse accumulator per row */
        uint64_t maxf = 0;
        for (uint64_t q = 0; q < nrows; ++q) if (r->row_flops[q] > maxf) maxf = r->row_flops[q];
        uint64_t cap = 16;
        while (cap < 2 * maxf) cap <<= 1;
        spa_map m;
        m.cap = cap;
        m.keys = (uint64_t*)malloc(sizeof(uint64_t) * cap);
        m.pos = (uint32_t*)malloc(sizeof(uint32_t) * cap);
        uint64_t* dkey = (uint64_t*)malloc(sizeof(uint64_t) * (maxf + 1));
        uint64_t* dsrc = (uint64_t*)malloc(sizeof(uint64_t) * (maxf + 1));
        double* dval = (double*)malloc(sizeof(double) * (maxf + 1));
        uint64_t out_cap = 0, out_n = 0;
        uint32_t* oidx = NULL;
        double* oval = NULL;
        if (!m.keys || !m.pos || !dkey || !dsrc || !dval) { set_err(r, "out of memory"); return ORACLE_ENOMEM; }
        memset(m.keys, 0xFF, sizeof(uint64_t) * cap);
        for (uint64_t q = 0; q < nrows; ++q) {
            if (r->row_flops[q] == 0) continue;       /* rows without flops are skipped, fksCuckooTC.hpp:183 */
            uint64_t mask = 1;
            while (mask < 2 * r->row_flops[q]) mask <<= 1;
            mask -= 1;
            uint64_t n = 0;
            for (uint64_t s = rstart[q]; s < rstart[q + 1]; ++s) {
                if (afib[s] < 0) continue;
                const double av = A->vals[aperm[s]];
                for (uint64_t t = fstart[afib[s]]; t < fstart[afib[s] + 1]; ++t) {
                    const uint64_t bi = bperm[t];
                    const uint64_t k = bfree[bi];
                    const double p = av * B->vals[bi];
                    uint64_t h = mix64(k) & mask;
                    for (;;) {
                        if (m.keys[h] == UINT64_MAX) {
                            m.keys[h] = k; m.pos[h] = (uint32_t)n;
                            dkey[n] = k; dsrc[n] = bi; dval[n] = p; ++n;
                            break;
                        }
                        if (m.keys[h] == k) { dval[m.pos[h]] += p; break; }
                        h = (h + 1) & mask;
                    }
                }
            }
            r->row_nnz[q] = n;
            if (mode == ORACLE_VALUES) {
                if (out_n + n > out_cap) {
                    uint64_t nc = out_cap ? out_cap : 1024;
                    while (nc < out_n + n) nc *= 2;
                    uint32_t* ni = (uint32_t*)realloc(oidx, sizeof(uint32_t) * nc * (fa + fb));
                    double* nv = (double*)realloc(oval, sizeof(double) * nc);
                    if (!ni || !nv) { set_err(r, "out of memory (output)"); return ORACLE_ENOMEM; }
                    oidx = ni; oval = nv; out_cap = nc;
                }
                const uint64_t a0 = aperm[rstart[q]];
                for (uint64_t e = 0; e < n; ++e) {
                    uint32_t* o = oidx + (out_n + e) * (uint64_t)(fa + fb);
                    for (uint32_t j = 0; j < fa; ++j) o[j] = A->idx[a0 * da + a_modes[c + j]];
                    for (uint32_t j = 0; j < fb; ++j) o[fa + j] = B->idx[dsrc[e] * db + b_modes[c + j]];
                    oval[out_n + e] = dval[e];
                }
            }
            out_n += n;
            /* clear the touched clusters */
            for (uint64_t e = 0; e < n; ++e) {
                uint64_t h = mix64(dkey[e]) & mask;
                while (m.keys[h] != UINT64_MAX) { m.keys[h] = UINT64_MAX; h = (h + 1) & mask; }
            }
        }
        r->out_nnz = out_n;
        r->out_idx = oidx;
        r->out_val = oval;
        free(m.keys); free(m.pos); free(dkey); free(dsrc); free(dval);
    }
    free(bkey); free(bperm); free(bfree); free(akey); free(aperm);
    free(fkey); free(fstart); free(rstart); free(afib);
    return ORACLE_OK;
}

void oracle_free(oracle_result* r) {
    free(r->out_idx); free(r->out_val);
    free(r->row_key); free(r->row_flops); free(r->row_nnz); free(r->row_len);
    memset(r, 0, sizeof(*r));
}
