/*
 * qm_obstacles.h — reading the reference's `obstacles` tiles (format "qmobs2") into scene outlines.
 *
 * A tile (tiles/src/obstacles.rs:1-24) stores every building ring and wall that crosses one of its
 * 128 x 128 cells of 256 lattice steps, whole, in the tile's int16 frame (0 at the tile's centre,
 * y growing south), with an index of the runs of consecutive edges passing through each cell. The
 * functions below check a tile as the reference's reader does (tiles/src/obstacles/parse.rs:23-128)
 * and turn its outlines into `qm_outline` records and int32 vertices for `qm_scene_desc`. They
 * run on the host only and need no device.
 *
 * Errors are QM_ERR_ARGUMENT with the reference's own message ("obstacles: bad magic",
 * "obstacles: run out of range", ...); `qm_last_error(NULL)` returns it.
 */
#ifndef QM_OBSTACLES_H
#define QM_OBSTACLES_H

#include "qm_batch.h"

#ifdef __cplusplus
extern "C" {
#endif

#define QM_OBSTACLES_CELLS_PER_SIDE 128
#define QM_OBSTACLES_CELL_STEPS 256

/* The header's counts (tiles/src/obstacles.rs:15). */
typedef struct {
    uint32_t outlines;
    uint32_t vertices;
    uint32_t runs;
    uint32_t occupied_cells;
    uint32_t footprint_squares;
    uint32_t pad_;
} qm_obstacles_counts;

/* Checks a tile of n_bytes: the magic, the header, the section lengths against the counts, the
 * occupied-cell counts, the cells' run ranges, the footprint squares' order, every outline (kind,
 * envelope, non-zero height, its square, its vertex range, footprint ids in order, closed rings
 * of four or more vertices, walls of two or more) and every run (its outline, a non-empty range
 * below the outline's last vertex). counts (nullable) gets the header's counts. */
qm_status qm_obstacles_check(const uint8_t *bytes, size_t n_bytes, qm_obstacles_counts *counts);

/* The tile's outlines in their stored order (sorted by footprint id): outlines[counts.outlines]
 * and vertices_xy[counts.vertices][2]. A vertex is the stored int16 pair plus (offset_x, offset_y),
 * the tile centre's position in the scene's lattice steps; outline i gets first_vertex (plus
 * first_vertex_base, for tiles appended to one vertex array), vertex_count, footprint_id (its
 * square's high half and its ordinal), height_m (decimetres / 10) and building (1 for exterior
 * rings and holes, 0 for walls). envelope (nullable) gets each outline's envelope class code
 * (0 outdoor, 1 residential, 2 commercial, 3 industrial, 4 historic, 5 default; walls outdoor).
 * The tile is checked first. */
qm_status qm_obstacles_outlines(const uint8_t *bytes, size_t n_bytes, int32_t offset_x,
                                int32_t offset_y, uint32_t first_vertex_base, qm_outline *outlines,
                                int32_t *vertices_xy, uint8_t *envelope);

/* The outlines of several tiles as one scene's: tile k (bytes[k], n_bytes[k]) with its centre at
 * offsets_xy[k] in the scene's steps. An outline crossing several tiles is stored whole in each,
 * with bit-identical global vertices under the same footprint id (tiles/src/obstacles.rs:5-6), so
 * it is kept once: the first occurrence, tiles in the given order, each tile's outlines in stored
 * order, of every (footprint id, kind, vertices) it meets. With null outlines and vertices_xy the
 * call only counts: *n_outlines and *n_vertices get the merged counts. Otherwise they hold the
 * arrays' capacities on entry (QM_ERR_CAPACITY when short) and the counts written on return;
 * envelope (nullable) gets the envelope class codes. Every tile is checked first. */
qm_status qm_obstacles_merge(const uint8_t *const *bytes, const size_t *n_bytes, const int32_t *offsets_xy,
                             size_t n_tiles, qm_outline *outlines, uint32_t *n_outlines,
                             int32_t *vertices_xy, uint32_t *n_vertices, uint8_t *envelope);

/* The runs of cell (column, row) of a checked tile (`cell_runs`, parse.rs:190-207): up to cap
 * runs as runs[k][3] = (outline, first edge, edge count); count gets the cell's number of runs
 * (which may exceed cap). */
qm_status qm_obstacles_cell_runs(const uint8_t *bytes, size_t n_bytes, uint32_t column, uint32_t row,
                                 uint32_t *runs, uint32_t cap, uint32_t *count);

#ifdef __cplusplus
}
#endif

#endif /* QM_OBSTACLES_H */
