/*
 * qm_flights.h — a square's aircraft boxes summed at the painter's lattice points on the device:
 * the drop-in for `Batch::flight_sums` (paint/src/exact.rs:177-182, paint/src/flight_boxes.rs:185-200),
 * whose GPU form is paint-gpu/src/aircraft.rs:145-230 `DeviceFlightBoxes::upload` and :235-340
 * `Gpu::flight_sums` over the kernel paint-gpu/kernels/aircraft.cuh:260-311.
 *
 * Per request and band of boxes: the boxes' energy per period (Leq, linear) and their passes in
 * 3 dB classes (popup/src/aircraft.rs:47-95 FlightPasses::add_pass), each box read by the
 * click-time equation (physics/src/doc29/boxes.rs:156-280 box_sel_at_receiver, two average
 * pieces at the gradient less and plus its spread) through the receiver's horizons
 * (popup/src/aircraft/horizons.rs:84-112 SectorEdges::loss_db), weighed by the lattice's
 * FlightWeight (paint/src/flight_boxes.rs:14-33) and heard within the aircraft reach
 * (popup/src/aircraft/boxes.rs:272-316 tile_flight_passes). Everything is computed in FP64, as
 * the cores compute it, so the 16 km reach, the horizon sectors and the 3 dB class edges take the
 * cores' branches.
 */
#ifndef QM_FLIGHTS_H
#define QM_FLIGHTS_H

#include "qm_batch.h"

#ifdef __cplusplus
extern "C" {
#endif

#define QM_PASS_CLASSES 48        /* popup/src/aircraft.rs:51 */
#define QM_PASS_CLASS_DB 3.0      /* popup/src/aircraft.rs:52 */
#define QM_PASS_LOWEST_DB (-30.0) /* popup/src/aircraft.rs:53 */
/* Doubles of one request band's sums: the energy per period, then per period the classes'
 * energies, then per period the classes' passing shares (paint-gpu/src/aircraft.rs:35-38). */
#define QM_FLIGHT_SUMS (QM_PERIODS + 2 * QM_PERIODS * QM_PASS_CLASSES)
#define QM_TERRAIN_SECTORS 32   /* popup/src/aircraft/horizons.rs:14 */
#define QM_BUILDING_SECTORS 256 /* popup/src/aircraft/horizons.rs:21 */
#define QM_HORIZON_BANDS 6      /* popup/src/aircraft/horizons.rs:23 */
/* Floats of one point's horizons (popup/src/aircraft/horizons.rs:24-29 and 196-201 write_f32):
 * the terrain's steepest tangent of all, then per sector its steepest and per band the edge's
 * range and tangent (NaN range: an empty band); then the buildings' alike. */
#define QM_TERRAIN_HORIZON_FLOATS (1 + QM_TERRAIN_SECTORS * (1 + 2 * QM_HORIZON_BANDS))
#define QM_HORIZON_FLOATS \
    (QM_TERRAIN_HORIZON_FLOATS + 1 + QM_BUILDING_SECTORS * (1 + 2 * QM_HORIZON_BANDS))
#define QM_AIRCRAFT_REACH_M 16000.0 /* popup/src/aircraft/boxes.rs:22 */

/* One aircraft box (tiles::aircraft::AircraftBox) at the square's frame, as box_at reads it
 * (popup/src/aircraft/boxes.rs:187-223). 600 bytes. */
typedef struct {
    double east_m, north_m;      /* the centroid in the square's metres */
    double centroid_altitude_m;  /* the centroid's altitude (m) */
    double ground_m;             /* the terrain under the box (m, the place's ground) */
    double axis_rad;             /* the horizontal axis, radians anticlockwise from east */
    double gradient;             /* climb along the axis */
    double gradient_spread;      /* the pieces' gradients' spread about it */
    double piece_length_m[QM_PERIODS];
    double levels_db[QM_PERIODS][QM_NPD_DISTANCES]; /* summed SEL at the NPD distances, -inf silent */
    double tail_levels_db[QM_PERIODS];              /* at the tail anchor (16 km), -inf silent */
    double lg_scaled_distance[QM_NPD_DISTANCES];    /* lg d_lambda at the NPD distances */
    double installation_shares[QM_PERIODS][2][3];   /* wing, fuselage, propeller at 1,000 ft and 16 km */
    double passing[QM_PERIODS];  /* the share of each period its flights are in it (box_passing) */
    uint32_t helicopter;         /* 1: a helicopter box, no impedance gain */
    uint32_t pad_;
} qm_flight_box;

/* One lattice point (paint-gpu/kernels/aircraft.cuh FlightPoint): where it stands in the
 * square's metres, its altitude, where its QM_HORIZON_FLOATS horizons begin in `horizons`, and
 * the impedance gain of the NPD levels at its altitude (the energy of receiver_impedance_db). */
typedef struct {
    double x, y;
    double altitude_m;
    uint64_t horizons;
    double impedance_gain;
} qm_flight_point;

#define QM_FLIGHT_WEIGHT_ONE 0u
#define QM_FLIGHT_WEIGHT_FAR 1u
#define QM_FLIGHT_WEIGHT_NEAR 2u

/* One point's boxes of one tile, file and band (paint-gpu/kernels/aircraft.cuh FlightSegment):
 * `count` boxes from `first`, heard within min(within_m, 16 km) of the point, each weighted by
 * `weight` (QM_FLIGHT_WEIGHT_*) at its distance with the hum's spacing `coarse_m`, added to the
 * QM_FLIGHT_SUMS doubles of request band `sum`. */
typedef struct {
    double within_m;
    double coarse_m;
    uint32_t point;
    uint32_t sum;
    uint32_t first;
    uint32_t count;
    uint32_t weight;
    uint32_t pad_;
} qm_box_segment;

/* Work and device time of one qm_flight_sums call. */
typedef struct {
    uint64_t box_reads;    /* (segment, box) pairs read */
    uint64_t boxes_heard;  /* of which within reach with a positive weight */
    double kernel_ms;      /* device time of the sums kernel */
} qm_flight_sums_stats;

typedef struct qm_flight_boxes qm_flight_boxes;

/* Decodes a square's boxes once onto the device (DeviceFlightBoxes::upload): each box with what
 * box_sel_at_receiver derives from it alone (the axis's sine and cosine, the average piece's
 * length, which periods are silent, whether it is low enough to be screened). */
qm_status qm_flight_boxes_upload(qm_ctx *ctx, const qm_flight_box *boxes, size_t n_boxes,
                                 qm_flight_boxes **out);
void qm_flight_boxes_free(qm_flight_boxes *boxes);

/* The sums of every request band (Gpu::flight_sums): `sums` holds n_sums x QM_FLIGHT_SUMS doubles,
 * written whole (bands no segment names read zero). Every segment's boxes must lie in `boxes`, its
 * point in `points`, the point's horizons in `horizons` (n_horizon_floats floats) and its sum
 * below n_sums; QM_ERR_ARGUMENT names the first that does not. stats is nullable. */
qm_status qm_flight_sums(qm_ctx *ctx, const qm_flight_boxes *boxes, const qm_flight_point *points,
                         size_t n_points, const float *horizons, size_t n_horizon_floats,
                         const qm_box_segment *segments, size_t n_segments, double *sums,
                         size_t n_sums, qm_flight_sums_stats *stats);

/* The points' horizons for aircraft screening, built on the device from a scene's terrain and
 * buildings (popup/src/aircraft/horizons.rs:145-198 Horizons::build, which the reference runs on the
 * host for every request): per point its position in the scene's lattice steps (x, y; fractional
 * allowed), its altitude (m) and the footprint it stands in (0 none, its walls are no horizon),
 * QM_HORIZON_FLOATS floats into `horizons` (n_points x QM_HORIZON_FLOATS) as qm_flight_sums reads
 * them. Terrain: 32 sectors x 48 samples from 30 m to 8 km growing geometrically, a sample outside
 * the scene's DEM is no terrain; buildings: 256 sectors, a 512 m ray each, the crossings within
 * 1 cm left out. QM_ERR_CAPACITY when a ray crosses more than 256 edges. kernel_ms (nullable): the
 * kernel's device time. */
qm_status qm_scene_flight_horizons(qm_scene *scene, const double *xy_steps, const double *altitude_m,
                                   const uint64_t *own_footprint, size_t n_points, float *horizons,
                                   double *kernel_ms);

/* qm_flight_sums with the points' horizons built on the device from the scene (as
 * qm_scene_flight_horizons builds them) and read there, nothing of them crossing to the host. The
 * points' positions are in the square's metres, the scene's lattice steps being step_m metres from
 * the same origin; their `horizons` fields are ignored; own_footprint (nullable) names the footprint
 * each stands in. The boxes must belong to the scene's context. */
qm_status qm_flight_sums_on_scene(qm_scene *scene, const qm_flight_boxes *boxes, const qm_flight_point *points,
                                  const uint64_t *own_footprint, size_t n_points, const qm_box_segment *segments,
                                  size_t n_segments, double *sums, size_t n_sums, qm_flight_sums_stats *stats);

#ifdef __cplusplus
}
#endif

#endif /* QM_FLIGHTS_H */
