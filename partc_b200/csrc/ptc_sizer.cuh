// Learned output-size predictor: network, training and features (ptc_sizer.cu, ptc_features.cu).
#pragma once

#include <vector>

#include "ptc_internal.cuh"

namespace ptc {

constexpr int kSizerInputs = 16;
constexpr int kSizerHidden = 64;
constexpr int kSizerParams = kSizerHidden * kSizerInputs + kSizerHidden + kSizerHidden * kSizerHidden + kSizerHidden +
                             kSizerHidden + 1;  // 5313

// Host state of a sizer: FP32 master weights (the device uses BF16 copies) and Adam moments.
struct SizerHost {
    std::vector<float> master, m, v;
    uint64_t steps = 0;
};

struct SizerTrainResult {
    float first_loss = 0.f, final_loss = 0.f;
    uint32_t epochs = 0;
    uint64_t steps = 0;
};

void sizer_init(SizerHost& s, uint64_t seed);
// y[i] = network(x[i]) for n samples of kSizerInputs features (device arrays)
void sizer_predict_device(const SizerHost& s, const float* d_x, uint64_t n, float* d_y, Arena& ar);
// gradient of the mean squared error over all n samples; returns the loss
float sizer_gradients(const SizerHost& s, const float* d_x, const float* d_t, uint64_t n, float* h_grad, Arena& ar);
// Adam over shuffled minibatches; updates s in place
SizerTrainResult sizer_train(SizerHost& s, const float* d_x, const float* d_t, uint64_t n, uint32_t epochs,
                             uint32_t batch, float lr, uint64_t seed, Arena& ar);

// ---- features (ptc_features.cu) ----

// Column-popularity model: for a row of F products, the expected number of distinct columns if
// each product picks a column with probability deg(col) / nb is
//     G(F) = sum_col 1 - exp(-F deg(col) / nb),
// tabulated per fine panel at F = 2^(g / kGridPerOctave), g = 0 .. kGridPoints-1.
constexpr int kGridPerOctave = 4;
constexpr int kGridPoints = 41 * kGridPerOctave;

// gp[p * kGridPoints + g] = G restricted to the columns of panel p (device, npanels * kGridPoints)
void launch_popularity_table(const uint32_t* b_col, uint64_t nb, uint64_t ncols, uint32_t npanels, uint32_t panel_log2,
                             float* gp, Arena& ar);
// Per-item statistics of a batch (device arrays indexed by item).  With them every row of a batch
// gets the features a single contraction of its own item would give it: its item's column,
// nonzero, fiber and row counts and its item's column popularity, not the whole batch's.
struct ItemStats {
    uint32_t nitems = 0;
    const uint64_t* b_off = nullptr;      // [nitems + 1] first B nonzero of each item
    const uint32_t* col_first = nullptr;  // [nitems + 1] first (global) column of each item
    const uint32_t* fib_first = nullptr;  // [nitems + 1] first fiber of each item
    const uint32_t* row_first = nullptr;  // [nitems + 1] first row of each item
    const uint32_t* col_run = nullptr;    // [ncols + 1] B nonzeros before each global column (degrees)
    float* gtot = nullptr;                // [nitems * kGridPoints] each item's G(F) table
    uint32_t* pmass = nullptr;            // [item_pb[i] + p] B nonzeros in local panel p of item i
    const uint64_t* item_pb = nullptr;    // [nitems + 1] first panel of each item in pmass
};

// Fill is.gtot and is.pmass (panels of 2^panel_log2 columns); is.item_pb must be set.
void launch_item_popularity(ItemStats& is, uint64_t ncols_global, uint32_t panel_log2, Arena& ar);

// Per-row features of `rows` (device): x[i * kSizerInputs + f].  `is` (batches) gives each row
// its item's statistics; null for a single contraction.
void launch_row_features(const Operands& op, const uint32_t* rows, uint64_t n, const uint64_t* row_flops,
                         const float* gp, float* x, cudaStream_t st, const ItemStats* is = nullptr);
// t[i] = log2(1 + row_d[rows[i]])
void launch_row_targets(const uint32_t* rows, uint64_t n, const uint64_t* row_d, float* t, cudaStream_t st);

}  // namespace ptc

// The opaque handle of include/partc.h.
struct ptc_sizer {
    ptc::SizerHost host;
};
