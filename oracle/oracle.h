/* CPU restatement of parTC's fksCuckooTC contraction -- test infrastructure (the checker). */
#ifndef PTC_ORACLE_H
#define PTC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORACLE_OK = 0, ORACLE_EINVAL = 1, ORACLE_ENOMEM = 2 };

/* what oracle_contract computes */
enum {
    ORACLE_FLOPS_ONLY = 0, /* grouping + symbolic flop count per row (fksCuckooTC.hpp:94-154) */
    ORACLE_COUNTS = 1,     /* + exact output nnz per row, no output arrays */
    ORACLE_VALUES = 2      /* + the output tensor */
};

typedef struct {
    uint32_t order;
    uint64_t nnz;
    const uint32_t* idx;  /* [nnz*order], 0-based */
    const double* vals;   /* [nnz] */
    const uint32_t* dims; /* [order] */
} oracle_coo;

typedef struct {
    uint32_t out_order;
    uint64_t out_nnz;
    uint32_t* out_idx;    /* [out_nnz*out_order] */
    double* out_val;      /* [out_nnz] */
    uint64_t flops;       /* mult-adds */
    uint64_t nrows;       /* distinct A free keys */
    uint64_t nfibers;     /* distinct B contracted keys */
    uint64_t* row_key;    /* [nrows] linearized A free key, increasing */
    uint64_t* row_flops;  /* [nrows] */
    uint64_t* row_nnz;    /* [nrows] exact output nnz (ORACLE_COUNTS / ORACLE_VALUES) */
    uint32_t* row_len;    /* [nrows] A nonzeros in the row */
    char err[128];
} oracle_result;

/* O = A x B over the c modes a_modes[0..c) of A and b_modes[0..c) of B; a_modes[c..) and
 * b_modes[c..) list the free modes in output order. */
int oracle_contract(const oracle_coo* A, const oracle_coo* B, uint32_t c, const uint32_t* a_modes,
                    const uint32_t* b_modes, int mode, oracle_result* r);
void oracle_free(oracle_result* r);

#ifdef __cplusplus
}
#endif
#endif
