/*
 * qm_surrogate.h — the learned ground/diffraction surrogate of the B200 painter.
 *
 * The reference has no counterpart: its painter always runs the exact CNOSSOS path
 * (physics/src/cnossos/{mean_plane,ground,rubber_band,diffraction}.rs). This part replaces, for
 * eligible paths, the boundary attenuation A_boundary = A_ground + A_dif per octave band (what
 * `boundary_for_candidates`, physics/src/cnossos/diffraction.rs:64-197, returns) by a small
 * BF16 network:
 *
 *   32 features -> 4 x (256, GELU) -> 8 outputs (A_boundary per band, dB)
 *
 * with BF16 weights and activations in the matrix products and FP32 accumulation. The network
 * is trained on the GPU by this library's own forward and backward kernels, on labels the exact
 * path code computes. A network serves one feature set, fixed by the scene it was trained on.
 *
 * Flat feature set (scenes without a DEM, homogeneous conditions), path from source S to
 * receiver R (horizontal length L metres):
 *   f0 L / 1000; f1 source height above the ground at S / 10; f2 receiver height above the
 *   ground at R / 10; f3 (ground at R - ground at S) / 10; f4 condition (0 homogeneous);
 *   f5, f6, f7 ground factor at S (the source's own G when it has one), at the middle and at R;
 *   f8 .. f31 up to 8 roofs crossed (the vertical path's roof spans after clipping, in their
 *   closing order), each as (x0 / L, x1 / L, height above the ground / 10); absent roofs are
 *   zeros (a present roof has x1 > x0 > 0, which is its mask).
 * Terrain feature set (scenes with a DEM; both conditions, one row per state): f0 .. f3 and
 *   f5 .. f7 as above (f6 the mean ground factor of the samples below), f4 the state (0
 *   homogeneous, 1 favourable); f8 .. f19 over 12 stretches of the path (ends at 0, 2, 5, 10,
 *   20, 35, 50, 65, 80, 90, 95, 98 and 100 % of L), the largest rise of the terrain above the
 *   straight source-receiver line among 3 DEM samples each (metres / 10); f20 .. f31 over the
 *   same stretches, the largest rise of the obstacle tops the path
 *   crosses above that line (-10 where it crosses none).
 * A flat path is eligible when all its obstacle tops pair into roofs and it crosses at most 8
 * roofs, a terrain path when its crossing list fits; both need their features inside the
 * training ranges. Other paths, and paths whose predicted levels fall outside the training
 * labels' range, are evaluated by the exact path code.
 */
#ifndef QM_SURROGATE_H
#define QM_SURROGATE_H

#include "qm_batch.h"

#ifdef __cplusplus
extern "C" {
#endif

#define QM_SURR_FEATURES 32
#define QM_SURR_HIDDEN 256
#define QM_SURR_LAYERS 4      /* hidden layers */
#define QM_SURR_OUTPUTS 8
#define QM_SURR_MAX_ROOFS 8
/* Parameters, in this order (FP32): W1[256][32], b1[256], W2..W4[256][256], b2..b4[256],
 * W5[8][256], b5[8], then the input shift[32] and scale[32] (x' = (x - shift) * scale), the
 * output shift[8] and scale[8] (A = y * scale + shift), the eligible feature range lo[32],
 * hi[32], the label range lo[8], hi[8], and the feature set (0 flat, 1 terrain). */
#define QM_SURR_WEIGHTS (256 * 32 + 256 + 3 * (256 * 256 + 256) + 8 * 256 + 8)
#define QM_SURR_PARAMS (QM_SURR_WEIGHTS + 32 + 32 + 8 + 8 + 32 + 32 + 8 + 8 + 1)

typedef struct qm_surrogate qm_surrogate;

/* A network on the context's device from `params` (QM_SURR_PARAMS floats). */
qm_status qm_surrogate_create(qm_ctx *ctx, const float *params, qm_surrogate **out);
void qm_surrogate_free(qm_surrogate *net);
/* Selects the inference kernel: 0 (the default) accumulates on the fifth-generation tensor cores
 * in tensor memory (tcgen05, operands staged by TMA bulk copies); 1 uses warp-level mma.sync with
 * register accumulators. Both compute the same network; the choice exists to compare them. */
qm_status qm_surrogate_set_kernel(qm_surrogate *net, int kernel);

/* Its current parameters (QM_SURR_PARAMS floats; the FP32 master copy). */
qm_status qm_surrogate_params(const qm_surrogate *net, float *params);

/* Training samples from the exact path code: for every path (cell, source) of the grid, its raw
 * features (features[rows][32]), its exact A_boundary per band (labels[rows][8], dB) and whether
 * its geometry is eligible (eligible[rows], 0/1; the feature range test is not applied). Flat
 * scenes: one row per path, row cell * n_sources + (source - source_begin), the homogeneous
 * state. Terrain scenes: two rows per path (2 * that + state), homogeneous then favourable. */
qm_status qm_surrogate_samples(qm_scene *scene, const qm_grid_desc *grid, float *features,
                               float *labels, uint8_t *eligible);

/* Forward pass on raw feature rows (features[n][32]) -> outputs[n][8] (A_boundary, dB). */
qm_status qm_surrogate_forward(qm_surrogate *net, const float *features, size_t n, float *outputs);

/* One backward pass of the mean squared error over n rows of normalised labels (the loss the
 * training minimises, on (A - out_shift) / out_scale): the gradient of every weight and bias
 * (grads[QM_SURR_WEIGHTS], the first QM_SURR_WEIGHTS parameters' order) and the loss. */
qm_status qm_surrogate_gradients(qm_surrogate *net, const float *features, const float *labels,
                                 size_t n, float *grads, double *loss);

typedef struct {
    uint32_t epochs;
    uint32_t batch;          /* rows per step */
    float learning_rate;     /* Adam, cosine decay to 5 % over the run */
    uint32_t seed;           /* shuffling */
    uint32_t max_samples;    /* 0: every eligible path of the grids */
    float exact_within_m;    /* paths shorter than this (horizontal metres) are left to the exact
                                path: not trained on, and below the eligible range of f0, so the
                                painter evaluates them exactly; 0 for none */
} qm_train_config;

/* Trains the network in place on the device: samples from every path of each grid (exact
 * labels, eligible paths at least exact_within_m long), the normalisation and eligible ranges
 * set from them, then Adam over shuffled batches. loss_history[epochs] (nullable) gets each
 * epoch's mean loss; n_samples (nullable) the number of samples used. */
qm_status qm_surrogate_train(qm_surrogate *net, qm_scene *scene, const qm_grid_desc *grids,
                             size_t n_grids, const qm_train_config *config, double *loss_history,
                             uint64_t *n_samples);

/* The grid painter with the surrogate: `qm_paint_grid`'s outputs, where eligible paths take
 * A_boundary from the network and the others (and out-of-range predictions) run the exact
 * path. stats->paths counts every path; surrogate_paths (nullable) those the network took. The
 * scene must be of the network's feature set (flat scenes: homogeneous conditions only). */
qm_status qm_paint_grid_surrogate(qm_scene *scene, const qm_grid_desc *grid, qm_surrogate *net,
                                  float *cell_bands, float *cell_dba, float *cell_lden,
                                  uint32_t *histogram, qm_paint_stats *stats,
                                  uint64_t *surrogate_paths);

#ifdef __cplusplus
}
#endif

#endif /* QM_SURROGATE_H */
