/* Line source pieces: the quadrature nodes of a straight piece and the receiver skyline that
 * places them (physics/src/line.rs, popup/src/obstacles/skyline.rs).
 *
 * The node placement and the skyline query are one __host__ __device__ source
 * (quietmap_b200/csrc/qm_line.cuh, qm_skyline.cuh) that a device thread runs per receiver and
 * piece; these entry points run it on the calling host thread, for a caller planning pieces
 * and for checking it against the reference's own tests without a GPU. They need no device and
 * allocate no device memory. Errors go to qm_last_error like every other entry point. */
#ifndef QM_LINE_H
#define QM_LINE_H

#include <stddef.h>
#include <stdint.h>

#include "qm_batch.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One quadrature node (physics/src/line.rs:64-71 LineQuadratureNode): where along the piece its
 * ray starts (metres from the piece's start), its weight (the in-plane angle it stands for) and
 * whether obstacles can stand on its ray (0 inside a clear gap of a wide bucket's mask). */
typedef struct {
    double along_m;
    double weight_rad;
    uint32_t obstacles_on_ray;
    uint32_t reserved;
} qm_line_node;

/* A piece's figures (physics/src/line.rs:120-134): its length, the in-plane angle it subtends,
 * the divergence factor that multiplies each node's weight times the power per metre
 * (hypot(ux, uy) / (10^1.1 d_perp)), and the in-plane angle of its start. */
typedef struct {
    double length_m;
    double subtended_angle_rad;
    double divergence_factor;
    double start_angle_rad;
} qm_line_piece_info;

/* A skyline query (physics/src/line.rs:82-84 SkylineQuery): hand `visit` every obstacle edge
 * within `radius_m` of the receiver whose azimuth arc may meet the wedge [wedge_lo_rad,
 * wedge_hi_rad] (radians, atan2(north, east)), as (arc lo, arc hi, nearest horizontal range). */
typedef void (*qm_skyline_visit_fn)(double lo_rad, double hi_rad, double nearest_m, void *visit_ctx);
typedef void (*qm_skyline_query_fn)(double wedge_lo_rad, double wedge_hi_rad, double radius_m,
                                    qm_skyline_visit_fn visit, void *visit_ctx, void *user);

/* LinePieceGeometry::new and line_quadrature_nodes (physics/src/line.rs:88-118, 178-206) for a
 * piece from `start` to `end` (metres relative to the receiver: x east, y north, z up). The
 * query `skyline` (NULL: no obstacles) is asked once per bucket wide enough in azimuth. Writes
 * the nodes in order and, when `info` is not NULL, the piece's figures. A piece shorter than a
 * millimetre radiates nothing: QM_OK with no nodes. More nodes than `cap`: the first `cap` are
 * written, *n_nodes holds the count and the call returns QM_ERR_CAPACITY. At most
 * QM_LINE_MAX_NODES nodes per piece. */
#define QM_LINE_MAX_NODES 705
qm_status qm_line_quadrature_nodes(const double start[3], const double end[3], qm_skyline_query_fn skyline,
                                   void *user, qm_line_node *nodes, size_t cap, size_t *n_nodes,
                                   qm_line_piece_info *info);

/* The receiver skyline over a scene's outlines (popup/src/obstacles/skyline.rs:22-110), indexed
 * as the reference's tiles index theirs: 256-step cells in the reference's south-growing frame
 * (a scene point (x, y) is (x, -y) there), each edge listed in the cells its supercover walk
 * passes through (tiles/src/obstacles/cells.rs:13-47), consecutive edges of an outline in one
 * run, and per cell its tallest outline (popup/src/obstacles/tile.rs:93-104). The index keeps
 * its own copy of the vertices and outlines. */
typedef struct qm_skyline qm_skyline;

/* Builds the index over `outlines` whose vertices are `vertices[n_vertices][2]` (scene steps,
 * y north) on a lattice of `step_m` metres. QM_ERR_ARGUMENT names an outline whose vertices lie
 * outside the array, or a step that is not positive and finite. */
qm_status qm_skyline_build(const int32_t *vertices, size_t n_vertices, const qm_outline *outlines,
                           size_t n_outlines, double step_m, qm_skyline **out);

/* The occupied cells and the runs listed in them. */
qm_status qm_skyline_counts(const qm_skyline *skyline, size_t *n_cells, size_t *n_runs);

/* Every arc the receiver at scene steps (x, y) gets for the wedge [lo_rad, hi_rad] within
 * radius_m above floor_m (the sight line's height: cells whose tallest outline, and walls whose
 * own height, stay at or under it hand over nothing), as arcs[n][3] = (lo, hi, nearest) in the
 * order the reference's query visits them, once per cell an edge is listed in
 * (popup/src/obstacles/skyline.rs:39-110). More than `cap`: the first `cap` are written,
 * *n_arcs holds the count and the call returns QM_ERR_CAPACITY. */
qm_status qm_skyline_arcs(const qm_skyline *skyline, int64_t x, int64_t y, double lo_rad, double hi_rad,
                          double radius_m, double floor_m, double *arcs, size_t cap, size_t *n_arcs);

void qm_skyline_free(qm_skyline *skyline);

/* A receiver's view of an index, for qm_skyline_query. The line evaluation queries with the
 * source's height, never under the ground, as the floor (popup/src/evaluate.rs:225-242). */
typedef struct {
    const qm_skyline *skyline;
    int64_t x, y;
    double floor_m;
} qm_skyline_receiver;

/* A qm_skyline_query_fn over an index: pass it with `user` pointing at a qm_skyline_receiver. */
void qm_skyline_query(double wedge_lo_rad, double wedge_hi_rad, double radius_m, qm_skyline_visit_fn visit,
                      void *visit_ctx, void *user);

#ifdef __cplusplus
}
#endif

#endif /* QM_LINE_H */
