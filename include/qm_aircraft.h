/*
 * qm_aircraft.h — Doc 29 aircraft noise on a receiver grid, with ISO 532-1 loudness of the
 * resulting third-octave spectra. The device counterpart of the reference's segment SEL
 * (physics/src/doc29/segment.rs:284-345 `segment_sel_at_receiver` / `screened_segment_sel`, with
 * its NPD reading physics/src/doc29/npd.rs:115-277 and corrections
 * physics/src/doc29/corrections.rs:21-85), summed over flights as `Batch::flight_sums` sums boxes
 * (paint/src/exact.rs:177-182; paint-gpu/kernels/aircraft.cuh:260-311), and fed to Zwicker
 * (physics/src/loudness.rs:148).
 */
#ifndef QM_AIRCRAFT_H
#define QM_AIRCRAFT_H

#include "qm_batch.h"

#ifdef __cplusplus
extern "C" {
#endif

#define QM_NPD_POWERS 10

/* One aircraft type: NPD curves per operation (0 approach, 1 departure), power row and NPD
 * distance (200 .. 25,000 ft, npd.rs:21-23), its NPD reference speed, its engine installation
 * (0 wing, 1 fuselage, 2 propeller: corrections.rs:69-74) and its relative third-octave spectrum
 * (unweighted dB, 25 Hz .. 12.5 kHz). */
typedef struct {
    float sel_db[2][QM_NPD_POWERS][QM_NPD_DISTANCES];
    float lamax_db[2][QM_NPD_POWERS][QM_NPD_DISTANCES];
    float v_ref_kt;
    uint32_t installation;
    float spectrum_db[QM_THIRDS];
    uint32_t pad_[2];
} qm_aircraft_type;

/* One flight segment: ends in metres (x east, y north, z above the receivers' ground plane),
 * the power setting as a fractional row index in [0, 9], ground speed, type, operation and the
 * flight it belongs to. 48 bytes. */
typedef struct {
    float start[3];
    float end[3];
    float power;
    float speed_mps;
    uint32_t type;
    uint32_t departure;
    uint32_t flight;
    uint32_t pad_;
} qm_flight_segment;

/* Receivers on a regular grid at origin + (i, j) * spacing metres, height_m above the ground
 * plane. A segment is heard at a receiver when the receiver lies within `reach_m` (horizontal)
 * of its flight's bounding box (reach_m <= 0: every segment everywhere). */
typedef struct {
    double origin_m[2];
    double spacing_m;
    int32_t nx, ny;
    float receiver_height_m;
    float pad_;
    double reach_m;
    double duration_s;  /* averaging time of the levels (86,400 s: a day's Leq) */
} qm_flight_grid_desc;

/* Work and device time of one qm_flight_grid call. */
typedef struct {
    uint64_t pairs;          /* cells x segments */
    uint64_t pairs_in_reach; /* of which evaluated (the others were culled with their flight) */
    double kernel_ms;        /* device time of the flight kernel */
    double loudness_ms;      /* device time of the Zwicker kernel (0 without sone) */
} qm_flight_stats;

/* Per cell: the total A-weighted sound exposure level (lae_db), the day-average third-octave
 * levels (thirds_db[cells][28]) of the summed flights and their Zwicker loudness (sone). Each
 * output is nullable. Segments must be grouped by flight (flight ids non-decreasing); 1 to 48
 * aircraft types (their NPD rows are held in shared memory). stats is nullable. */
qm_status qm_flight_grid(qm_ctx *ctx, const qm_aircraft_type *types, uint32_t n_types,
                         const qm_flight_segment *segments, size_t n_segments,
                         const qm_flight_grid_desc *grid, float *lae_db, float *thirds_db,
                         float *sone, qm_flight_stats *stats);

#ifdef __cplusplus
}
#endif

#endif /* QM_AIRCRAFT_H */
