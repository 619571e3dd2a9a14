/*
 * partc.h -- C ABI of the B200 sparse tensor contraction engine (parTC's fksCuckooTC path).
 *
 * parTC's driver (main.cpp:115-118) builds two FKS/cuckoo hash tables and calls
 *     Tensor tc_fksCuckoo(Hash_Table* HT_A, Hash_Table* HT_B, Tensor& A_copy, Tensor& B);
 * (fksCuckooTC.hpp:80).  This header replaces those three calls with one entry point that takes
 * the same COO arrays (tensor.hpp:19-27: hedges_array = 0-based u32 indices, AoS, N x d;
 * val_array = f64; dimensions_array; dim_tc = contracted modes first) and returns the same
 * output tensor (u32 AoS indices, A's free modes then B's free modes, and f64 values).
 *
 * Differences in error behaviour: where the reference calls exit(), these functions return a
 * status code (see ptc_status); ptc_last_error() gives the message.  Functions are thread-safe;
 * the last error is kept per host thread.
 */
#ifndef PARTC_H
#define PARTC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PTC_API_VERSION 1

typedef enum ptc_status {
    PTC_OK = 0,
    PTC_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad order / mode list / sizes */
    PTC_ERR_INDEX_RANGE = 2,      /* an index is >= its mode size */
    PTC_ERR_KEY_OVERFLOW = 3,     /* product of the contracted (or free) mode sizes >= 2^64 */
    PTC_ERR_EMPTY_CONTRACTION = 4,/* no A nonzero meets a B fiber; the reference exits with
                                     "tensor contraction not possible!!" (tensor.hpp:116-119) */
    PTC_ERR_TOO_FEW_NONZEROS = 5, /* self-contraction of a tensor with <= 1 nonzero; the reference
                                     exits with "Tensor B has at most one nonzeros!!"
                                     (sparse_tensor_generator.hpp:18-21) */
    PTC_ERR_HASH_BUILD = 6,       /* cuckoo build failed after every reseed/growth; the reference
                                     exits with "None of the keys in kDict worked"
                                     (fksCuckoo.hpp:439-441) */
    PTC_ERR_OUT_OF_MEMORY = 7,    /* device or host allocation failed (reference: exit(1),
                                     fksCuckoo.hpp:244-247) */
    PTC_ERR_CUDA = 8,             /* a CUDA runtime call failed */
    PTC_ERR_NO_DEVICE = 9,        /* no usable sm_100 device */
                                  /* 10 is not used (no device-side wait exists to time out) */
    PTC_ERR_OVERFLOW = 11,        /* a result does not fit the caller-provided capacity */
    PTC_ERR_INTERNAL = 12
} ptc_status;

/* where a buffer lives */
enum { PTC_HOST = 0, PTC_DEVICE = 1 };

/* which numeric path to run */
enum {
    PTC_PATH_TWO_PHASE = 0, /* exact symbolic pass (per-row output nnz), then numeric pass */
    PTC_PATH_LEARNED = 1    /* learned sizer replaces the symbolic pass; rows that overflow
                               their predicted accumulator rerun exactly */
};

/* COO input tensor (the reference's Tensor, tensor.hpp:19-27). */
typedef struct ptc_coo {
    uint32_t order;        /* d */
    uint32_t location;     /* PTC_HOST or PTC_DEVICE, for idx and vals */
    uint64_t nnz;          /* N */
    const uint32_t* idx;   /* [nnz * order], 0-based, AoS (hedges_array) */
    const double* vals;    /* [nnz] (val_array) */
    const uint32_t* dims;  /* [order] mode sizes, host memory (dimensions_array) */
} ptc_coo;

/* Output tensor (the Tensor returned by tc_fksCuckoo, fksCuckooTC.hpp:156,360). */
typedef struct ptc_tensor {
    uint32_t order;        /* (A free modes) + (B free modes) */
    uint32_t location;     /* PTC_HOST or PTC_DEVICE */
    uint64_t nnz;          /* O.N */
    uint32_t* idx;         /* [nnz * order] */
    double* vals;          /* [nnz] */
    void* opaque;          /* owned by the library; release with ptc_tensor_free */
} ptc_tensor;

typedef struct ptc_sizer ptc_sizer; /* learned output-size predictor (opaque) */

typedef struct ptc_options {
    uint32_t struct_size;      /* sizeof(ptc_options) */
    int32_t device;            /* CUDA device ordinal; -1 = current device */
    void* stream;              /* cudaStream_t to run on; NULL = the library's own stream */
    uint32_t path;             /* PTC_PATH_TWO_PHASE (default) or PTC_PATH_LEARNED */
    uint32_t output_location;  /* PTC_HOST (default, like the reference) or PTC_DEVICE */
    uint32_t verbose;          /* 1: print the reference's stdout lines (timings, nnz) */
    uint32_t panel_width;      /* columns per fine panel (power of two in [32, 4096]); large
                                  rows are cut at panel boundaries into work items (a warp's or a
                                  block's range of panels); above 512 only block parts are used;
                                  0 = automatic (at most 256 unless the counters grow too big) */
    uint64_t hash_seed;        /* seed of the cuckoo hash family */
    const ptc_sizer* sizer;    /* PTC_PATH_LEARNED: trained sizer (NULL = built-in weights) */
    uint32_t sort_rows;        /* 1: rows of the output in increasing free-key order and every
                                  row in increasing column order (canonical COO); runs the
                                  two-phase path and one sort of the entries (about 24 extra bytes
                                  of device memory per output entry); single contractions only */
    /* tuning knobs (0 = default) */
    uint32_t small_max_products;    /* rows with at most this many products use the one-warp
                                       accumulator (<= 512; default 128) */
    uint32_t sort_max_avg_products; /* rows averaging fewer products per A nonzero use the
                                       sort-based accumulator (default 64) */
    uint32_t hash_load_pct;         /* cuckoo table load factor in percent, 10-90 (default 75) */
    uint32_t batch_wave_mib;        /* ptc_batch_contract: device memory for one wave's outputs,
                                       MiB (default: 60% of the free memory) */
    uint32_t warp_task_max_len;     /* large rows with at most this many A nonzeros use one warp per
                                       column range, longer ones one block per part (default 256) */
    /* cuckoo build of B's fiber table (the reference's buildHashTable, fksCuckoo.hpp:1044-1060) */
    uint32_t cuckoo_max_chain;      /* evictions one insertion may cause before the build attempt
                                       fails (default 64; 0 = no eviction at all) -- set it small to
                                       exercise the rebuild path */
    uint32_t cuckoo_max_attempts;   /* builds tried, each with new hash seeds and, after every two
                                       failures, twice the buckets (the reference's rehash with new
                                       kDict pairs and a larger table, fksCuckoo.hpp:297-442), before
                                       the call returns PTC_ERR_HASH_BUILD (default 8) */
    uint32_t large_rows;            /* accumulator of the large rows: PTC_LARGE_ROWS_AUTO (0,
                                       default: rows of at most bitmap_max_len A nonzeros on the
                                       row bitmap kernel when the columns fit it, the others on the
                                       panel kernels), PTC_LARGE_ROWS_BITMAP (every large row on the
                                       row bitmap kernel -- one block per row, a bitmap of its
                                       columns in shared memory, up to about 600k distinct B free
                                       keys) or PTC_LARGE_ROWS_PANELS (warp tasks and block parts
                                       over column panels, any size).  Results are identical; the
                                       panel kernels are the faster on the 4-D 3.1M Zipf workload */
    uint32_t bitmap_max_len;        /* PTC_LARGE_ROWS_AUTO: A nonzeros of the longest row on the
                                       row bitmap kernel (default 0: none) */
    uint32_t reserved[2];
} ptc_options;

enum { PTC_LARGE_ROWS_AUTO = 0, PTC_LARGE_ROWS_BITMAP = 1, PTC_LARGE_ROWS_PANELS = 2 };

/* Per-call statistics; every time is measured with CUDA events on the call's stream. */
typedef struct ptc_stats {
    uint64_t mult_adds;        /* sum over A nonzeros of the matching B fiber's length */
    uint64_t out_nnz;
    uint64_t nrows;            /* distinct A free keys (rows of HT_A) */
    uint64_t ncols;            /* distinct B free keys */
    uint64_t nfibers;          /* distinct B contracted keys (fibers of HT_B) */
    uint64_t a_nnz, b_nnz;
    double t_total_ms;         /* whole call */
    double t_h2d_ms;           /* host-to-device input copies */
    double t_build_ms;         /* keys, sorts, cuckoo build, probes (HT_B + HT_A + reorder) */
    double t_symbolic_ms;      /* exact symbolic pass, or sizer features + inference */
    double t_numeric_ms;       /* numeric pass incl. output writes (the reference's
                                  "Total time for tensor contraction") */
    double t_d2h_ms;           /* device-to-host output copies */
    uint32_t hash_attempts;    /* cuckoo builds tried (1 = first seed worked) */
    uint32_t panel_width;      /* fine panel width used */
    uint64_t rows_small;       /* rows on the one-warp accumulator */
    uint64_t rows_hash;        /* rows on the block hash accumulator */
    uint64_t hash_parts;       /* parts those rows were cut into */
    uint64_t rows_long;        /* rows on the sort-based accumulator */
    uint64_t rerun_rows;       /* learned path: rows rerun exactly after an overflow */
    double sizer_mean_abs_log2_err; /* learned path: mean |log2(pred/actual)| over rows */
    uint64_t kernel_launches;  /* kernels this call launched */
    uint64_t batch_waves;      /* ptc_batch_contract: output waves */
    uint64_t rerun_items;      /* ptc_batch_contract, learned path: items rerun exactly */
    double reserved[2];
} ptc_stats;

/* Fill *opt with defaults. */
void ptc_options_init(ptc_options* opt);

/* Human-readable message of the last failing call on this host thread. */
const char* ptc_last_error(void);

/* Status code name. */
const char* ptc_status_string(ptc_status s);

/*
 * O = A x B over c contracted modes.  a_modes[0..c) and b_modes[0..c) are the contracted modes
 * (paired in order); a_modes[c..order_A) and b_modes[c..order_B) are the free modes in output
 * order -- the dim_tc arrays of the reference (meta file line 2).  B == NULL means B = A with
 * b_modes = a_modes: the reference's self-contraction (main.cpp:112,
 * sparse_tensor_generator.hpp:4-88).  Replaces main.cpp:115-118.
 * The output is allocated by the library (host malloc or device memory per
 * opt->output_location) and must be released with ptc_tensor_free.
 */
ptc_status ptc_contract(const ptc_coo* A, const ptc_coo* B, uint32_t c, const uint32_t* a_modes,
                        const uint32_t* b_modes, const ptc_options* opt, ptc_tensor* out,
                        ptc_stats* stats);

/*
 * The self-contraction exactly as main.cpp calls it: the tensor's arrays as read by readTensor
 * (mtxTnsIO.cpp:30-65), c and dim_tc as read by Tensor::populate_meta_info (tensor.hpp:151-173).
 * Equivalent to ptc_contract(&A, NULL, c, dim_tc, dim_tc, ...).  Replaces main.cpp:112-118.
 */
ptc_status ptc_self_contract(const uint32_t* hedges, const double* vals, uint32_t d, uint64_t N,
                             const uint32_t* dims, uint32_t c, const uint32_t* dim_tc,
                             const ptc_options* opt, ptc_tensor* out, ptc_stats* stats);

/* Release an output tensor made by this library. */
void ptc_tensor_free(ptc_tensor* t);

/* One contraction of a batch (no counterpart in the reference, which contracts one tensor per
 * run).  A zeroed B (idx, dims NULL and nnz 0) means B = A with b_modes = a_modes: the
 * self-contraction. */
typedef struct ptc_batch_item {
    ptc_coo A;
    ptc_coo B;
    uint32_t c;
    uint32_t a_modes[16];
    uint32_t b_modes[16];
} ptc_batch_item;

/* Receives item `item`'s output; the arrays are valid only during the call (the library reuses
 * them) and must not be freed. */
typedef void (*ptc_batch_sink)(void* user, uint32_t item, const ptc_tensor* out);

/*
 * Contract n independent items as one problem: every key of item i is offset into a key range of
 * its own, so one pass of each kernel (keys, sorts, one cuckoo table, symbolic pass) serves the
 * whole batch (items are taken in chunks of at most 32M nonzeros, so the working arrays stay a
 * bounded share of the device).  Outputs are produced in waves of consecutive items that fit
 * opt->batch_wave_mib; each wave's numeric pass is one CUDA-graph launch.  Results of every item equal ptc_contract's
 * (same entries; values bit-identical).
 *   outs != NULL: outs[i] receives item i's output (release each with ptc_tensor_free; items of a
 *                 wave share one block, freed with the last of them).  With PTC_DEVICE outputs
 *                 every output stays on the device: one wave.
 *   sink != NULL: sink(user, i, &view) is called for every item as its wave completes (views in
 *                 opt->output_location memory, valid during the call only).
 *   both NULL:    outputs are computed and discarded (for timing).
 * Every input must be in the same memory.  Unlike ptc_contract, an item with no matching fiber or
 * with at most one nonzero is not an error: its output is empty.  opt->path = PTC_PATH_LEARNED
 * sizes the large rows with the sizer; an item whose prediction falls short runs again exactly.
 * Replaces a loop of main.cpp:115-118 over many tensors.
 */
ptc_status ptc_batch_contract(const ptc_batch_item* items, uint32_t n, const ptc_options* opt,
                              ptc_tensor* outs, ptc_batch_sink sink, void* user, ptc_stats* stats);

/*
 * Read a FROSTT .tns file (one nonzero per line: d 1-based labels, then the value; '#' / '%'
 * comment lines) on the GPU, as readTensor does with pigo (mtxTnsIO.cpp:30-65): same labels
 * (minus one), same values (pigo's decimal arithmetic, bit for bit), each mode's size its largest
 * label.  *out gets the tensor (order d, in opt->output_location memory; release with
 * ptc_tensor_free) and dims[0..d) the mode sizes (dims must hold 16 entries).
 */
ptc_status ptc_read_tns(const char* path, const ptc_options* opt, ptc_tensor* out, uint32_t* dims);

/* Write a tensor (host or device arrays) as .tns text: 1-based labels, values with 17
 * significant digits (which read back to the same double). */
ptc_status ptc_write_tns(const char* path, const ptc_tensor* t);

/* What ptc_autotune measured. */
typedef struct ptc_tune_report {
    uint32_t trials;     /* settings timed */
    uint32_t repeats;    /* runs per setting (the median is kept) */
    double default_ms;   /* median time of one run with the default knobs */
    double best_ms;      /* median time of one run with the chosen knobs */
    double reserved[4];
} ptc_tune_report;

/*
 * Autotuner (no counterpart in the reference): picks the tuning knobs of ptc_options --
 * large_rows (row bitmap or panel kernels), panel_width (shared-table column ranges),
 * small_max_products / warp_task_max_len /
 * sort_max_avg_products (which accumulator, and so how many threads, each row gets) and
 * hash_load_pct (cuckoo table load factor) -- for the given items by timing
 * ptc_batch_contract on them (outputs discarded) under candidate settings, one knob at a time from
 * the defaults, `repeats` runs per setting (median).  *best = *opt with the chosen knobs; results
 * are identical under every setting, only the time changes.
 */
ptc_status ptc_autotune(const ptc_batch_item* items, uint32_t n, const ptc_options* opt, uint32_t repeats,
                        ptc_options* best, ptc_tune_report* report);

/* Number of CUDA devices the library can use (sm_100 class). */
int ptc_device_count(void);

/* Bytes of the device's stream-ordered memory pool (the pool every call allocates its working
 * arrays and device outputs from) that are allocated and not yet freed, after the device has
 * finished the work queued so far.  Device outputs a caller still holds count; with none held,
 * a finished call -- successful or failed -- leaves 0 behind. */
ptc_status ptc_device_pool_in_use(int32_t device, uint64_t* bytes);

/* ---- learned sizer (no counterpart in the reference: it replaces the symbolic pass) ----
 * A 16 -> 64 -> 64 -> 1 ReLU network with BF16 weights and FP32 accumulation that predicts
 * log2(1 + output nnz) of a row from per-row features computed on the device.  It is trained
 * and evaluated by the library's own CUDA kernels. */
#define PTC_SIZER_FEATURES 16
#define PTC_SIZER_PARAMS 5313 /* W1[64][16], b1[64], W2[64][64], b2[64], w3[64], b3 */

typedef struct ptc_train_options {
    uint32_t struct_size;  /* sizeof(ptc_train_options) */
    uint32_t epochs;       /* passes over the samples (default 20) */
    uint32_t batch;        /* samples per Adam step (default 8192) */
    float lr;              /* Adam learning rate (default 2e-3) */
    uint64_t seed;         /* minibatch shuffling seed */
    int32_t device;        /* -1 = current device */
    uint32_t reserved[5];
} ptc_train_options;

typedef struct ptc_train_stats {
    float first_epoch_loss;  /* mean squared error (log2 units) over the first epoch */
    float final_epoch_loss;  /* ... over the last epoch */
    uint32_t epochs;
    uint64_t steps;          /* Adam steps taken by this sizer so far */
    double ms;               /* wall time of the training call */
} ptc_train_stats;

void ptc_train_options_init(ptc_train_options* opt);
/* New sizer with seeded He-normal weights. */
ptc_status ptc_sizer_create(uint64_t seed, ptc_sizer** out);
ptc_status ptc_sizer_load(const char* path, ptc_sizer** out);
ptc_status ptc_sizer_save(const ptc_sizer* s, const char* path);
void ptc_sizer_free(ptc_sizer* s);
/* FP32 master weights in the PTC_SIZER_PARAMS order (the device computes with BF16 copies). */
ptc_status ptc_sizer_get_params(const ptc_sizer* s, float* params);
ptc_status ptc_sizer_set_params(ptc_sizer* s, const float* params);
/* Training samples of one contraction: the features and log2(1 + exact output nnz) of every
 * row the learned path sizes.  *features (n x PTC_SIZER_FEATURES) and *targets (n) are
 * allocated by the library; release them with ptc_buffer_free. */
ptc_status ptc_sizer_collect(const ptc_coo* A, const ptc_coo* B, uint32_t c, const uint32_t* a_modes,
                             const uint32_t* b_modes, const ptc_options* opt, float** features,
                             float** targets, uint64_t* n);
/* Adam on the mean squared error, minibatches shuffled per epoch; all math on the device. */
ptc_status ptc_sizer_train(ptc_sizer* s, const float* features, const float* targets, uint64_t n,
                           const ptc_train_options* opt, ptc_train_stats* stats);
/* out[i] = predicted log2(1 + output nnz) for n feature rows (host arrays). */
ptc_status ptc_sizer_predict(const ptc_sizer* s, const float* features, uint64_t n, int32_t device,
                             float* out);
/* ptc_sizer_predict without any device allocation.  No counterpart in the reference: it is for
 * callers that cannot allocate device memory where they need a prediction (another allocator
 * owns the device, or an allocation would synchronize the device or is not allowed there).  Its
 * device scratch -- the BF16 weights, up to 65536 staged feature rows and their predictions -- is
 * one static device array of about 4.3 MiB that every device loading the library keeps until the
 * process exits.  n > 65536 is rejected with PTC_ERR_INVALID_ARGUMENT.  The first call on a device
 * looks up that array's address there and keeps it; make that call before capturing any stream
 * (the kept address does not survive a cudaDeviceReset of the device).  All calls share the array:
 * calls whose GPU work overlaps race on it.  Runs on the calling thread's per-thread default
 * stream, restores the caller's current device and returns when out holds the predictions (host
 * arrays in and out). */
ptc_status ptc_sizer_predict_noalloc(const ptc_sizer* s, const float* features, uint64_t n,
                                     int32_t device, float* out);
/* Gradient of the mean squared error over n samples (host arrays; grads has PTC_SIZER_PARAMS). */
ptc_status ptc_sizer_gradients(const ptc_sizer* s, const float* features, const float* targets,
                               uint64_t n, int32_t device, float* grads, float* loss);
void ptc_buffer_free(void* p);

#ifdef __cplusplus
}
#endif
#endif /* PARTC_H */
