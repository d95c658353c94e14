// The surrogate network on the device: a fused inference kernel (all five layers per 128-row
// tile, activations kept in registers between layers), a tiled BF16 matrix product for training
// (forward, backward and weight gradients), and Adam. Built as its own translation unit
// (qm_mlp.cu); the painter's host code calls the functions below.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace qm {

constexpr int MLP_IN = 32, MLP_HID = 256, MLP_OUT = 8, MLP_LAYERS = 5;
constexpr size_t MLP_WEIGHTS = 256 * 32 + 256 + 3 * (256 * 256 + 256) + 8 * 256 + 8;
constexpr size_t MLP_W16 = 256 * 32 + 3 * 256 * 256 + 8 * 256;

// Width of layer boundary l (0: the features, 5: the outputs).
__host__ __device__ constexpr int mlp_dim(int l) { return l == 0 ? MLP_IN : (l == MLP_LAYERS ? MLP_OUT : MLP_HID); }
// Offsets of layer l's weight matrix [out][in] and bias in the packed FP32 parameter vector.
__host__ __device__ constexpr size_t mlp_w_offset(int l) {
    size_t o = 0;
    for (int k = 0; k < l; ++k) o += (size_t)mlp_dim(k + 1) * mlp_dim(k) + mlp_dim(k + 1);
    return o;
}
__host__ __device__ constexpr size_t mlp_b_offset(int l) { return mlp_w_offset(l) + (size_t)mlp_dim(l + 1) * mlp_dim(l); }
// Offset of layer l's matrix in the packed BF16 copy (matrices only; every offset is a multiple
// of 8 elements, so 16-byte aligned).
__host__ __device__ constexpr size_t mlp_w16_offset(int l) {
    size_t o = 0;
    for (int k = 0; k < l; ++k) o += (size_t)mlp_dim(k + 1) * mlp_dim(k);
    return o;
}
static_assert(mlp_w_offset(MLP_LAYERS) == MLP_WEIGHTS, "parameter count");
static_assert(mlp_w16_offset(MLP_LAYERS) == MLP_W16, "matrix count");

// Normalisation and the ranges the network was trained on.
struct MlpScales {
    float in_shift[MLP_IN], in_scale[MLP_IN];
    float out_shift[MLP_OUT], out_scale[MLP_OUT];
    float feat_lo[MLP_IN], feat_hi[MLP_IN];
    float lab_lo[MLP_OUT], lab_hi[MLP_OUT];
    float feature_set;  // 0 flat, 1 terrain
};

struct MlpDev {
    float *master = nullptr;          // [MLP_WEIGHTS] FP32 weights and biases
    __nv_bfloat16 *w16 = nullptr;     // [MLP_W16] BF16 matrices
    __nv_bfloat16 *wpack = nullptr;   // [mlp_packed_bytes()] the matrices in the tcgen05 operand layout
    unsigned *error = nullptr;        // set by an inference kernel whose bounded wait gave up
    int kernel = 0;                   // inference: 0 tcgen05 (tensor memory), 1 mma.sync
    float *adam_m = nullptr, *adam_v = nullptr;  // Adam moments (allocated by training)
    MlpScales scales;
};

// Bytes of the packed tcgen05 operand copy of the matrices.
size_t mlp_packed_bytes();

// Refreshes the BF16 matrices (and their packed copy, when allocated) from the FP32 master weights.
cudaError_t mlp_cast(const MlpDev &net, cudaStream_t stream);

// Normalised BF16 feature rows from raw FP32 rows: x' = (x - shift) * scale.
cudaError_t mlp_normalise(const MlpScales &s, const float *raw, size_t n, __nv_bfloat16 *out, cudaStream_t stream);

// Inference on normalised rows x[n][32]: A_boundary (dB) per row, out[n][8].
cudaError_t mlp_forward(const MlpDev &net, const __nv_bfloat16 *x, size_t n, float *out, cudaStream_t stream);

// The painter's use: rows are (cell, source) paths, `rows_per_cell` (a multiple of 128) per
// cell; a row's coefficients (coef[row][16]: 8 for the day bands, 8 for the Lden sum) turn the
// predicted A_boundary into energies, summed per 128-row tile into partial[tile of cell][cell][9]
// (added). Eligible rows whose prediction leaves the label range join the re-run list instead.
struct MlpPaintArgs {
    const __nv_bfloat16 *x;
    const float *coef;
    const uint8_t *eligible;
    size_t rows;
    uint32_t rows_per_cell;
    uint32_t rows_per_path;  // 1, or 2 (homogeneous and favourable rows of one path, adjacent)
    int cells;
    float *partial;  // [rows_per_cell / 128][cells][9]
    uint32_t source_begin, n_sources;
    uint2 *retry;
    uint32_t retry_cap;
    unsigned int *retry_count;
    unsigned long long *taken;  // eligible rows the network answered
};
cudaError_t mlp_paint(const MlpDev &net, const MlpPaintArgs &a, cudaStream_t stream);

// Mean squared error on normalised labels y[n][8] and the gradient of every weight and bias
// (grads[MLP_WEIGHTS], zeroed here); loss (device double) gets the mean.
struct MlpWork;  // activations of one batch
MlpWork *mlp_work_create(size_t max_rows);
void mlp_work_free(MlpWork *w);
cudaError_t mlp_gradients(const MlpDev &net, MlpWork *w, const __nv_bfloat16 *x, const float *y, size_t n,
                          float *grads, double *loss, cudaStream_t stream);

// One Adam step on the master weights from grads, then the BF16 refresh.
cudaError_t mlp_adam(MlpDev &net, const float *grads, float lr, int step, cudaStream_t stream);

// Rows `index[i]` of x and y gathered into contiguous batch buffers.
cudaError_t mlp_gather(const __nv_bfloat16 *x, const float *y, const uint32_t *index, size_t n, __nv_bfloat16 *bx,
                       float *by, cudaStream_t stream);

// Column statistics of raw rows (width w, n rows; rows with keep[i] == 0 skipped when keep is
// given): sum, sum of squares (double), min and max.
cudaError_t mlp_column_stats(const float *rows, const uint8_t *keep, size_t n, int w, double *sum, double *sumsq,
                             float *lo, float *hi, cudaStream_t stream);

}  // namespace qm
