/*
 * qm_weather.h — the weather of a place from the reference's global weather table ("qmwthr2").
 *
 * The table (physics/src/weather.rs:1-27) holds 361 x 720 nodes on a 0.5 degree grid, rows from
 * 90 N to 90 S and columns from 0 E eastwards; a node is 3 x 16 percentages (the probability of
 * favourable propagation per period and direction sector, sector s centred on the bearing
 * 22.5 s degrees clockwise from north) and 8 air absorptions in 0.01 dB/km (u16 LE). A place's
 * weather is the bilinear mix of its four nodes, longitude wrapping (weather.rs:170-214). The
 * results fill a `qm_scene_desc`'s `favourable` and `alpha_db_per_km` (cast to float). Host only.
 *
 * Errors are QM_ERR_ARGUMENT with the reference's messages ("weather table: bad magic or
 * length", "weather table: a percentage above 100"; the file form prefixes the path);
 * `qm_last_error(NULL)` returns them.
 */
#ifndef QM_WEATHER_H
#define QM_WEATHER_H

#include "qm_batch.h"

#ifdef __cplusplus
extern "C" {
#endif

#define QM_WEATHER_ROWS 361
#define QM_WEATHER_COLUMNS 720
#define QM_WEATHER_NODE_BYTES (QM_PERIODS * QM_SECTORS + 2 * QM_BANDS)
#define QM_WEATHER_TABLE_BYTES (8 + QM_WEATHER_ROWS * QM_WEATHER_COLUMNS * QM_WEATHER_NODE_BYTES)

/* From the whole table in memory (`WeatherTable::parse` and `place`, weather.rs:102-131): the
 * table is checked (length, magic, every percentage at most 100), then favourable[3][16] gets p
 * in [0, 1] and alpha_db_per_km[8] the absorption (dB/km) at (lat, lon) degrees. */
qm_status qm_weather_place(const uint8_t *table, size_t n_bytes, double lat, double lon,
                           double *favourable, double *alpha_db_per_km);

/* The same from the table's file, reading its magic and the place's four nodes alone
 * (`read_place`, weather.rs:137-166: the file's length and magic, those nodes' percentages). */
qm_status qm_weather_read_place(const char *path, double lat, double lon, double *favourable,
                                double *alpha_db_per_km);

#ifdef __cplusplus
}
#endif

#endif /* QM_WEATHER_H */
