/*
 * qm_batch.h — C ABI of the B200 noise-map painter hot path.
 *
 * This library replaces what sits behind the painter's exact-evaluation trait
 * `paint::exact::Batch` (paint/src/exact.rs:163-183) and its CUDA implementor
 * `paint_gpu::GpuBatch` (paint-gpu/src/batch.rs:247-373). Plain C types only:
 * host pointers and sizes in, caller-owned host buffers out, a status code back and
 * `qm_last_error` for the message. Every entry point validates its arguments before
 * touching the device and names the offending argument in the error text, as
 * `Gpu::evaluate_pairs` does (paint-gpu/src/device.rs:450-473).
 *
 * Frame: positions are lattice steps of `qm_scene_desc.step_m` metres, x east, y north.
 * Obstacle vertices, sources and receivers all sit on that lattice, so every
 * segment–edge cross product is an exact integer and crossing lists are reproducible
 * bit for bit (the reference stores obstacle vertices as exact integers of its own
 * int16 lattice too: popup/src/obstacles/mod.rs:5-8).
 */
#ifndef QM_BATCH_H
#define QM_BATCH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QM_ABI_VERSION 3

#define QM_BANDS 8      /* octave bands 63 Hz .. 8 kHz (physics/src/bands.rs:4) */
#define QM_PERIODS 3    /* day, evening, night (physics/src/bands.rs:14) */
#define QM_SECTORS 16   /* favourable-probability sectors (physics/src/weather.rs:16) */
#define QM_LAYERS 6     /* source layers of a point's bands (paint/src/exact.rs:19) */
#define QM_THIRDS 28    /* third-octave bands 25 Hz .. 12.5 kHz (physics/src/loudness.rs:12) */
#define QM_NPD_DISTANCES 10 /* (physics/src/doc29/npd.rs:20) */
#define QM_PAIR_SUMS 9  /* mixed, calm, downwind per period (paint-gpu/src/device.rs:92) */
#define QM_POINT_BANDS (QM_LAYERS * QM_PERIODS * QM_BANDS)

typedef enum {
    QM_OK = 0,
    QM_ERR_ARGUMENT = 1,    /* an argument is invalid; the message names it */
    QM_ERR_CUDA = 2,        /* a CUDA call failed; the message starts with "cuda: " */
    QM_ERR_CAPACITY = 3,    /* a device buffer or per-path capacity was exceeded */
    QM_ERR_TIMEOUT = 4,     /* a bounded device wait gave up */
    QM_ERR_UNSUPPORTED = 5  /* no sm_100 device, or a feature this build leaves out */
} qm_status;

/* Per-pair failure bits, with the reference's meanings (paint-gpu/kernels/common.cuh:27-31). */
#define QM_FAILED_NOT_READ 1u
#define QM_FAILED_NO_TERRAIN 2u
#define QM_FAILED_CAPACITY 4u
#define QM_FAILED_LINE_CUTOFF 8u
#define QM_FAILED_TIMEOUT 16u

/* One obstacle outline: a closed ring (its last vertex repeats its first) or an open
 * wall polyline. Ring vertices are `vertices[first_vertex .. first_vertex + vertex_count)`.
 * Mirrors the qmobs2 outline record the crossing walk reads
 * (popup/src/obstacles/crossings.rs:136-149). */
typedef struct {
    uint32_t first_vertex;
    uint32_t vertex_count;
    uint64_t footprint_id;  /* two walls of one building share it; 0 is reserved */
    float height_m;         /* above the local ground */
    uint32_t building;      /* 1 building ring (bounds roofs), 0 barrier/wall */
} qm_outline;

/* One point source (a 1 m road/rail piece, or any point emitter). Mirrors the
 * candidate + attribute the pair oracle reads (popup/src/evaluate.rs:47-57, 193-214). */
typedef struct {
    int32_t x, y;                 /* lattice steps */
    float height_m;               /* above its ground */
    float ground_factor;          /* Gs of (2.5.14); negative: the terrain's under it */
    float exclusion_radius_m;     /* minimum horizontal distance of the divergence */
    float platform_half_width_m;  /* terrain clamp near the source (0 for points) */
    uint64_t footprint_id;        /* the source's own building, 0 none */
    uint32_t layer;               /* 0 .. QM_LAYERS-1 */
    uint32_t pad_;
    float energy[QM_PERIODS][QM_BANDS]; /* A-weighted linear sound power per band */
} qm_source;

/* A scene: obstacles, terrain, sources and weather, uploaded once and shared by calls. */
typedef struct {
    double step_m;                 /* metres per lattice step */
    int32_t cell_steps;            /* obstacle grid cell side in steps (>= 16) */
    int32_t extent_steps[2];       /* scene covers [0, extent) steps on each axis */
    uint32_t n_vertices;
    const int32_t *vertices;       /* [n_vertices][2] */
    uint32_t n_outlines;
    const qm_outline *outlines;
    /* Terrain: dem_nx == 0 is flat ground at flat_altitude_m with flat_ground_factor.
     * Otherwise nodes (i, j) at (dem_origin + i*dem_spacing, dem_origin + j*dem_spacing)
     * steps, row-major [j][i]; altitude and ground factor linear along lattice lines
     * (physics/src/profile.rs:1-6, popup/src/scene.rs:236-296). */
    int32_t dem_nx, dem_ny;
    int32_t dem_origin[2];
    int32_t dem_spacing;
    const float *dem_altitude_m;
    const float *dem_ground_factor;
    float flat_altitude_m;
    float flat_ground_factor;
    uint32_t n_sources;
    const qm_source *sources;
    /* Weather of the place (physics/src/weather.rs:46-70): p per period and sector,
     * sector s centred on bearing 22.5 s degrees clockwise from north; air absorption. */
    float favourable[QM_PERIODS][QM_SECTORS];
    float alpha_db_per_km[QM_BANDS];
} qm_scene_desc;

/* A regular receiver grid for the fused painter: nx*ny receivers at origin + (i, j)*spacing
 * steps, `height_m` above the ground, in cell order j*nx + i. */
typedef struct {
    int32_t origin[2];
    int32_t spacing;
    int32_t nx, ny;
    float height_m;
    /* Sources [source_begin, source_end) are painted; an empty range means all. */
    uint32_t source_begin, source_end;
    /* Histogram of per-cell day dBA levels: bin k holds levels rounding to
     * level_min_db + k*bin_db (popup/src/distribution.rs:69-72). */
    double level_min_db;
    double bin_db;
    uint32_t n_bins;
} qm_grid_desc;

typedef struct {
    uint64_t paths;          /* receiver x source paths evaluated */
    uint64_t failed_paths;   /* paths re-run by the high-capacity pass */
    uint64_t crossings;      /* obstacle crossings found */
    uint64_t edge_tests;     /* exact segment-edge tests of the crossing walk */
    uint64_t vertices;       /* vertical-profile vertices streamed (terrain and roofs) */
    uint64_t candidates;     /* diffraction candidates fed to the rubber bands */
    double kernel_ms;        /* device time of the painting kernels (paint, re-run, reduce) */
    double paint_ms;         /* device time of the main painting kernel alone */
} qm_paint_stats;

typedef struct qm_ctx qm_ctx;
typedef struct qm_scene qm_scene;

/* Library ABI version; a binding checks it before the first call. */
int qm_abi_version(void);

/* Opens device `device_ordinal` (an sm_100 GPU). Replaces `Gpu::new`
 * (paint-gpu/src/device.rs:270): kernels are linked in as sm_100a cubins, no NVRTC. */
qm_status qm_open(int device_ordinal, qm_ctx **out);
/* Closes a context. Scenes and surrogate networks made on it stay usable: the context is
 * released when the last of them is freed. */
void qm_close(qm_ctx *ctx);
/* The last error of this context's calls on the calling thread ("" if none). */
const char *qm_last_error(const qm_ctx *ctx);

/* Uploads a scene: obstacles with their grid cell lists, terrain, sources, weather.
 * Replaces `DeviceSquare::upload` (paint-gpu/src/square_upload.rs:18). */
qm_status qm_scene_upload(qm_ctx *ctx, const qm_scene_desc *desc, qm_scene **out);
/* Frees a scene; batch plans made on it stay usable, and it is released with the last of them. */
void qm_scene_free(qm_scene *scene);

/* A line piece candidate (a road or rail piece, popup/src/evaluate.rs:171-267 `source_rays` with
 * physics/src/line.rs): its ends in lattice steps (fractional positions allowed) and its source
 * properties as a point source has them, `energy` per metre of the piece; source.x and .y are not
 * read. */
typedef struct {
    double a[2], b[2];
    qm_source source;
} qm_line_source;

/* Sets a scene's line pieces: candidate k of qm_evaluate_pairs is point source k below the
 * scene's n_sources and piece k - n_sources from there on. Builds the receivers' skyline index of
 * the scene's outlines (popup/src/obstacles/skyline.rs, qm_skyline_build) on the device beside
 * them. Replaces any pieces set before. */
qm_status qm_scene_line_pieces(qm_scene *scene, const qm_line_source *pieces, size_t n_pieces);

/* Batch::evaluate and Batch::pair_spectra (paint/src/exact.rs:164-170; GPU
 * `Gpu::evaluate_pairs`, paint-gpu/src/device.rs:440). Receivers at `receiver_xy`
 * (metres, snapped to the scene lattice), `receiver_height_m` above their ground,
 * standing in building `own_footprint` (0 none) and adding into point
 * `point_of_receiver`. Each pair names a source and a receiver; `band_weight` (nullable:
 * all 1) weighs its spectrum into the point's bands.
 * Outputs: pair_sums[n_pairs][9] = mixed[3], calm[3], downwind[3] (PairEnergy,
 * exact.rs:128-132); pair_bands (nullable) [n_pairs][3][8] each pair's unweighted bands
 * (pair_spectra); point_bands[n_points][6][3][8] += weighted bands by source layer
 * (add_bands, exact.rs:208-215); pair_status[n_pairs] failure bits. A candidate at or past the
 * scene's n_sources is a line piece (qm_scene_line_pieces): its pair sums its quadrature nodes'
 * rays (each from its point along the piece, by the f64 walks, with the skyline's mask), as
 * Point::line evaluation does (popup/src/evaluate.rs:171-267, paint-gpu/kernels/line.cuh). */
qm_status qm_evaluate_pairs(qm_scene *scene,
                            const double *receiver_xy, const float *receiver_height_m,
                            const uint64_t *own_footprint, const uint32_t *point_of_receiver,
                            size_t n_receivers,
                            const uint32_t *source_of_pair, const uint32_t *receiver_of_pair,
                            const float *band_weight, size_t n_pairs,
                            float *pair_sums, float *pair_bands, uint32_t *pair_status,
                            float *point_bands, size_t n_points);

/* The fused grid painter: every receiver of `grid` against the source range, with
 * per-cell compensated energetic sums. Outputs (each nullable): cell_bands[nx*ny][8] day
 * band levels (dB), cell_dba[nx*ny] day dBA, cell_lden[nx*ny] Lden (dBA), histogram[n_bins]
 * counts of cell_dba. This is `evaluate_all` over a regular grid (paint/src/exact.rs:218-254)
 * with `add_bands` folded into the kernel. */
qm_status qm_paint_grid(qm_scene *scene, const qm_grid_desc *grid,
                        float *cell_bands, float *cell_dba, float *cell_lden,
                        uint32_t *histogram, qm_paint_stats *stats);

/* ISO 532-1 stationary Zwicker loudness of n spectra of 28 third-octave levels (dB;
 * -inf silent): sone[n]. The per-pixel core of `Batch::loudness`
 * (physics/src/loudness.rs:148; GPU `loud_zwicker`, paint-gpu/kernels/loudness.cuh:85). */
qm_status qm_zwicker(qm_ctx *ctx, const float *thirds_db, size_t n, float *sone);

/* The bounded wait's own check. Every wait on a bulk copy's mbarrier gives up after about a second
 * and becomes QM_ERR_TIMEOUT (or a failed path's QM_FAILED_TIMEOUT) instead of a hang; here one
 * kernel waits `limit_ms` (at most 2,000) on an mbarrier that nothing completes. QM_OK when the wait
 * gave up no sooner than its limit and the kernel returned; waited_ms (nullable) is the device time
 * it waited. The context stays usable. */
qm_status qm_check_bounded_wait(qm_ctx *ctx, double limit_ms, double *waited_ms);

/* Level histogram of n levels (dB): counts[n_bins] of round((L - level_min)/bin), clamped
 * into the grid (popup/src/distribution.rs:69-72). Counts are exact. */
qm_status qm_level_histogram(qm_ctx *ctx, const float *levels_db, size_t n,
                             double level_min_db, double bin_db, uint32_t n_bins,
                             uint32_t *counts);

/* Map cells of n pixels, one byte per layer and one for the total (last), as
 * `PaintedCells::from_painted` makes them (paint/src/levels.rs:55-68, called by the painter at
 * paint/src/paint.rs:497):
 * - Lden cells (lden_cells[n][QM_LAYERS + 1]) from the linear Lden energy of each layer
 *   (lden_energy[n][QM_LAYERS]): round(2 Lden dB), at most 253, QM_CELL_SILENCE below energy 1
 *   (`lden_cell`, levels.rs:87-98); the total sums the layers' energies before the logarithm
 *   (`lden_cells`, levels.rs:100-111);
 * - loudness cells (nden_cells[n][QM_LAYERS + 1], wanted only with sone[n][QM_LAYERS + 1]):
 *   round(80 + 20 log2 sone), twice the loudness level in phon, at most 253, QM_CELL_SILENCE
 *   under 0 phon or for NaN (`cell`, levels.rs:25-33).
 * Pixels with assessed[p] == 0 (assessed may be null: every pixel assessed) are QM_CELL_NO_LEVEL
 * in every byte. An assessed pixel with a negative or non-finite Lden energy, or whose layers sum
 * to a non-finite total, fails the call with QM_ERR_ARGUMENT and a message naming the lowest such
 * pixel and its first bad layer ("pixel P, layer L: ..." or "pixel P, total: ..."), the outputs
 * left unwritten. Arithmetic is f64 rounded as the reference rounds it; a byte can differ from
 * the reference's only where CUDA's and the host's log10/log2 differ in the last bit at a half
 * step. */
#define QM_CELL_NO_LEVEL 255
#define QM_CELL_SILENCE 254
qm_status qm_quantize_cells(qm_ctx *ctx, const double *lden_energy, const double *sone,
                            const uint8_t *assessed, size_t n, uint8_t *lden_cells,
                            uint8_t *nden_cells);

/* HM3 / HMD tile streams up to their Brotli stage (`encode_metric_tile`, paint/src/hm3.rs:95-109):
 * per tile, the 5-byte header ("HM3 \x07" for loudness cells, metric 0; "HMD \x01" for Lden cells,
 * metric 1; hm3.rs:22-27), the layer byte, then the 512 x 512 cells (row-major from the
 * north-west) as PNG Paeth residuals, cell - prediction mod 256 (filter 4 with its left, above,
 * upper-left tie order and zeros outside the tile; `paeth_prediction`, hm3.rs:68-93).
 * cells[n_tiles][512 * 512], layers[n_tiles] (each at most QM_LAYERS: the total), streams
 * [n_tiles][QM_HM3_STREAM_BYTES]. The reference then compresses each stream with Google's Brotli
 * encoder (quality 10 for loudness, 9 for Lden, window 2^19); that stage is the caller's. */
#define QM_HM3_TILE_PX 512
#define QM_HM3_STREAM_BYTES (6 + 512 * 512)
qm_status qm_hm3_predict(qm_ctx *ctx, const uint8_t *cells, const uint8_t *layers, size_t n_tiles,
                         int metric, uint8_t *streams);

/* The inverse, on the host (`decode_metric_tile` after its Brotli stage, paint/src/hm3.rs:127-169):
 * a decompressed stream of QM_HM3_STREAM_BYTES whose header must be the metric's and whose layer
 * byte must be `layer` ("not this layer's HM3 tile" otherwise; "unknown HM3 layer" for a layer
 * above QM_LAYERS), back to its 512 x 512 cells (cells[512 * 512]). Needs no device. */
qm_status qm_hm3_unpredict(const uint8_t *stream, size_t n_bytes, uint32_t layer, int metric,
                           uint8_t *cells);

/* How a line of moving emitters' level varies in time (Kurze 1971; physics/src/percentile.rs):
 * a line with `lambda` emitters per distance of its closest point stays below
 * out[k] = its intensity relative to the mean with probability p[k] (0 < p < 1), for n pairs
 * (lambda[k], p[k]), computed on the device in FP64. Dense lines (lambda >= 10) are normal;
 * below that the 41 x 100 quantile table is read log-linearly between rows and in log(1 - p)
 * between quantiles, with the nearest emitter's passing above the last quantile; lambda 0 is
 * silence, an infinite lambda a steady source (1). The table is the reference's simulation
 * (physics/src/percentile_tests.rs:1-102) run by this library on its first use (a few seconds). */
qm_status qm_line_level_quantiles(qm_ctx *ctx, const double *lambda, const double *p, size_t n,
                                  double *out);

/* That table, 41 rows (lambda = 1e-4 * 10^(row / 8)) of 100 quantiles (probabilities
 * (k + 0.5) / 100) of the intensity relative to the mean, as floats: table[41 * 100]. Host only. */
qm_status qm_line_level_table(float *table);

/* The obstacle crossings of n rays from (from_xy) to (to_xy), lattice steps: per ray its count
 * (counts[n]) and, up to `cap` per ray, the crossed edges (the edge's first vertex index),
 * chainages t (f64) and flags (bit 0 building, bit 1 bounds_roof), sorted and deduplicated as
 * `Scene::crossings` returns them (popup/src/obstacles/crossings.rs:163-226). A ray with more
 * than `cap` crossings reports its count and QM_FAILED_CAPACITY in status[n]. */
qm_status qm_list_crossings(qm_scene *scene, const int32_t *from_xy, const int32_t *to_xy, size_t n,
                            uint32_t cap, uint32_t *counts, uint32_t *edges, double *t,
                            uint32_t *flags, uint32_t *status);

/* The grid painter for callers that cannot allocate device memory while they paint (an engine
 * that owns every device allocation and cannot let a cudaMalloc synchronise its device, or a thread
 * that may not allocate after set-up). It has no counterpart in the reference: it is
 * `qm_paint_grid` with every intermediate buffer carved out of one static device array of
 * QM_STATIC_SCRATCH_BYTES (64 MiB) that each GPU loading this library holds until exit, so its
 * success path calls no cudaMalloc, cudaFree or other allocating routine. Limits: at most
 * QM_STATIC_MAX_CELLS (65,536) cells and QM_STATIC_MAX_BINS (4,096) histogram bins, and the grid's
 * partial sums must fit the array (rejected with QM_ERR_CAPACITY otherwise); paths over the
 * per-path capacities are not re-run (QM_ERR_CAPACITY: use qm_paint_grid). cell_bands, cell_dba
 * and cell_lden are required host outputs; stats->kernel_ms is -1 (not timed). The first call on a
 * device looks up the array's device address and loads the kernels this entry point launches, with
 * that device current, so make the first call before any stream capture; the no-allocation promise
 * holds from the first call's launches on. Receivers are set up on the device by the host set-up's
 * rules (ground altitude in double, the lowest containing footprint id). Every call reuses the one
 * array: calls that overlap on the GPU (from two contexts on one device) race. */
#define QM_STATIC_SCRATCH_BYTES (64u << 20)
#define QM_STATIC_MAX_CELLS 65536
#define QM_STATIC_MAX_BINS 4096
qm_status qm_paint_grid_static(qm_scene *scene, const qm_grid_desc *grid,
                               float *cell_bands, float *cell_dba, float *cell_lden,
                               uint32_t *histogram, qm_paint_stats *stats);

#ifdef __cplusplus
}
#endif

#endif /* QM_BATCH_H */
