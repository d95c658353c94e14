/*
 * qm_tiles.h — many receiver tiles of uneven sizes painted as one batch.
 *
 * The reference paints a square block by block and fills its card with launches of at most
 * ~2 M pairs, admitting 2–3 squares at once by candidate count (paint-gpu/src/card.rs:50-101,
 * eval_slot.rs:55-63). Here a batch of tiles (each a regular receiver grid with its own source
 * range over one uploaded scene) becomes a list of work items — (tile, receiver block, source
 * chunk) — that persistent CTAs take from a device queue, largest first. The launches of a batch
 * are captured once in a CUDA graph and replayed. Block shape, threads per CTA and source-chunk
 * size are chosen per tile-size bucket by `qm_batch_autotune`, which times the candidates on the
 * device.
 *
 * Outputs are per cell, tile after tile: cell k of tile t is output cell `tiles[t].cell_offset
 * + k` (cells in row order j * nx + i), with `qm_paint_grid`'s levels: 8 day band levels,
 * dBA and Lden.
 */
#ifndef QM_TILES_H
#define QM_TILES_H

#include "qm_batch.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int32_t origin[2];       /* first receiver, lattice steps */
    int32_t spacing;         /* receiver spacing, lattice steps */
    int32_t nx, ny;
    float height_m;          /* receiver height above the ground */
    uint32_t source_begin;   /* this tile's sources: [source_begin, source_end) */
    uint32_t source_end;
    uint64_t cell_offset;    /* first output cell of the tile */
} qm_tile_desc;

/* One launch shape: receivers per work item (block_w x block_h, each a multiple of 8 and at
 * most 64), threads per CTA (128 or 256; a thread takes block_w * block_h / threads receivers)
 * and sources per work item (128 .. 2048). */
typedef struct {
    uint32_t block_w, block_h;
    uint32_t threads;
    uint32_t chunk;
} qm_tile_config;

/* Tile-size buckets by the longer side of a tile: < 64, < 128, < 256, and >= 256 receivers. */
#define QM_TILE_BUCKETS 4
typedef struct {
    qm_tile_config bucket[QM_TILE_BUCKETS];
} qm_tune_table;

/* The candidates the autotuner times, in this order (QM_TILE_CANDIDATES of them):
 * block 16x8 / 16x16 / 32x16 / 32x32 / 64x64 with 128, 256, 128, 256 and 256 threads, each with
 * chunks of 128, 256, 512, 1024 and 2048 sources. */
#define QM_TILE_CANDIDATES 25

/* The bucket of a tile (0 .. QM_TILE_BUCKETS - 1). */
uint32_t qm_tile_bucket(const qm_tile_desc *tile);

/* A fixed table: 16x8 blocks of 128 threads and 512-source chunks in every bucket. */
void qm_tune_default(qm_tune_table *table);

/* Times every candidate on the given sample tiles of each bucket (each sample clipped to its
 * first 64 x 64 receivers and 4,096 sources) and keeps the fastest per bucket; buckets without
 * a sample keep the default. timings (nullable) gets ms per candidate, [bucket][candidate]
 * (-1 where not timed). */
qm_status qm_batch_autotune(qm_scene *scene, const qm_tile_desc *sample, size_t n_sample, qm_tune_table *table,
                            float *timings);

typedef struct qm_batch_plan qm_batch_plan;

/* Plans a batch: validates the tiles (inside the scene, cell ranges disjoint and within
 * `n_cells`), sets up every receiver, builds the work queue per launch shape and (with
 * QM_BATCH_GRAPH) captures the batch's launches in a CUDA graph. */
#define QM_BATCH_GRAPH 1u
qm_status qm_batch_plan_create(qm_scene *scene, const qm_tile_desc *tiles, size_t n_tiles, uint64_t n_cells,
                               const qm_tune_table *table, uint32_t flags, qm_batch_plan **out);
void qm_batch_plan_free(qm_batch_plan *plan);

/* Paints every tile of the plan (one graph replay, or the same launches one by one without
 * QM_BATCH_GRAPH), then re-runs over-capacity paths and reduces the cells. stats (nullable): path
 * counts of the batch and kernel_ms, the device time of the whole run; paint_ms the persistent
 * launches alone. */
qm_status qm_batch_plan_run(qm_batch_plan *plan, qm_paint_stats *stats);

/* The last run's cell levels: cell_bands[n_cells][8], cell_dba[n_cells], cell_lden[n_cells]
 * (each nullable; cells no tile covers read -inf). */
qm_status qm_batch_plan_read(qm_batch_plan *plan, float *cell_bands, float *cell_dba, float *cell_lden);

#ifdef __cplusplus
}
#endif

#endif /* QM_TILES_H */
