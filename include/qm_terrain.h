/*
 * qm_terrain.h — decoding the reference's `terrain` tiles ("qmterr2").
 *
 * A tile (tiles/src/terrain.rs:1-30, 180-214) is the one-arc-second node window of a z12 tile —
 * rows from north_node southwards, columns from west_node eastwards, latitude = node / 3600
 * degrees — as a 24-byte header and one zstd frame of five planes: the height residual's low and
 * high bytes (zigzag-coded, after a planar prediction from the west, north and north-west nodes in
 * the u16 ring), imperviousness (%), forest cover (%) and canopy height (m). Heights are codes:
 * metres = -500 + code / 5, 65535 missing. Host only; zstd comes from the system's libzstd.so.1,
 * loaded on first use (QM_ERR_UNSUPPORTED without it).
 *
 * Errors are QM_ERR_ARGUMENT with the reference's messages ("terrain: bad magic", "terrain: a
 * window no tile has", "terrain: the frame does not decode", "terrain: the frame does not match
 * the window"); `qm_last_error(NULL)` returns them.
 */
#ifndef QM_TERRAIN_H
#define QM_TERRAIN_H

#include "qm_batch.h"

#ifdef __cplusplus
extern "C" {
#endif

#define QM_TERRAIN_HEIGHT_MISSING 65535
#define QM_TERRAIN_MAX_WINDOW_NODES 1024

typedef struct {
    int32_t north_node;  /* global node index of row 0 (latitude north_node / 3600) */
    int32_t west_node;   /* global node index of column 0 (longitude west_node / 3600) */
    uint32_t rows, columns;
} qm_terrain_window;

/* `Terrain::parse` (tiles/src/terrain.rs:232-272): the window, then, when height_codes is given,
 * every node row-major: height_codes[rows * columns] and, each nullable, impervious, forest and
 * canopy (one byte a node). With height_codes null only the header is read. */
qm_status qm_terrain_decode(const uint8_t *bytes, size_t n_bytes, qm_terrain_window *window,
                            uint16_t *height_codes, uint8_t *impervious, uint8_t *forest,
                            uint8_t *canopy);

/* `terrain-fine` tiles ("qmtfin2", tiles/src/terrain_fine.rs:1-11, 70-110): a national model's
 * detail on the 1/6 arc-second lattice over the `terrain` tile's window (six fine intervals to
 * each; rows and columns at most 6 * 1023 + 1), in signed 0.2 m codes, stored as a directory of
 * frame ends and one zstd frame per block of 128 x 128 cells (each block also holds the node row
 * and column closing its last cells), each the planar residual as in `terrain`. The window,
 * then, when details is given, every node row-major (`FineTerrain::parse` and `codes`,
 * terrain_fine.rs:128-172, 266-281): details[rows * columns]. Errors: "terrain-fine: bad magic",
 * "... a window no tile has", "... the directory is cut", "... a frame outside the tile",
 * "... a block does not decode". */
qm_status qm_terrain_fine_decode(const uint8_t *bytes, size_t n_bytes, qm_terrain_window *window,
                                 int16_t *details);

/* The ground at one point, as `Terrain::sample` gives it (tiles/src/terrain.rs:115-127). */
typedef struct {
    double height_m;       /* bilinear over the cell's four nodes */
    double ground_factor;  /* 1 - bilinear imperviousness / 100 */
    double forest_cover;   /* the nearest node's, in [0, 1] */
    double canopy_m;       /* the nearest node's */
} qm_ground_sample;

/* Web Mercator in z12 tile units (x east, y south, both in [0, 4096)) of a latitude and longitude
 * in degrees, latitude clamped to the Mercator limit, longitude wrapped (tiles/src/geo.rs:28-40). */
void qm_mercator_from_degrees(double lat_deg, double lon_deg, double *x, double *y);

/* The node window of z12 tile (tile_x, tile_y): floor and ceiling nodes bracketing the tile
 * (`Window::of_tile`, terrain.rs:66-88), what its `terrain` file holds. */
qm_status qm_terrain_window_of_tile(uint32_t tile_x, uint32_t tile_y, qm_terrain_window *window);

/* The fractional column (0 at west_node) of Mercator x, across the antimeridian the same meridian
 * a world away, the column nearest the window (`Window::column_of`, terrain.rs:55-64). */
double qm_terrain_column_of(const qm_terrain_window *window, double mercator_x);

/* `Terrain::locate` and `sample_at` (terrain.rs:289-387) at n Mercator points (mercator_xy[n][2])
 * over a decoded window (`qm_terrain_decode`'s arrays): found[k] 1 with out[k] filled, 0 where
 * the point is outside the window or a node it needs has no data (a missing height or an
 * imperviousness or forest cover above 100 %). */
qm_status qm_terrain_sample(const qm_terrain_window *window, const uint16_t *height_codes,
                            const uint8_t *impervious, const uint8_t *forest, const uint8_t *canopy,
                            const double *mercator_xy, size_t n, qm_ground_sample *out,
                            uint8_t *found);

#ifdef __cplusplus
}
#endif

#endif /* QM_TERRAIN_H */
