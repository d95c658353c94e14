// Line source pieces on the host side of the library: the skyline index builder and the C entry
// points that run the shared __host__ __device__ quadrature and skyline query (qm_line.cuh,
// qm_skyline.cuh) on the calling thread. The index's arrays are laid out as a device copy will
// hold them, so a device upload is a plain copy of each.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <map>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/qm_line.h"
#include "qm_host.h"
#include "qm_line.cuh"
#include "qm_skyline.cuh"

static_assert(QM_LINE_MAX_NODES == qm::line::MAX_NODES, "the header's node bound is the quadrature's");
static_assert(sizeof(qm_line_node) == 24, "qm_line_node is 24 bytes");

struct qm_skyline {
    std::vector<int32_t> vertices;
    std::vector<qm_outline> outlines;
    std::vector<uint64_t> keys;
    std::vector<uint32_t> run_start;
    std::vector<float> tallest;
    std::vector<qm::skyline::Run> runs;
    double step_m = 0.0;

    qm::skyline::Index view() const {
        qm::skyline::Index ix;
        ix.keys = keys.data();
        ix.run_start = run_start.data();
        ix.tallest = tallest.data();
        ix.runs = runs.data();
        ix.vertices = vertices.data();
        ix.outlines = outlines.data();
        ix.n_cells = (uint32_t)keys.size();
        ix.step_m = step_m;
        return ix;
    }
};

namespace {

// A C visit callback as the functor the shared query and quadrature call.
struct VisitThunk {
    qm_skyline_visit_fn visit;
    void *ctx;
    void operator()(double lo, double hi, double nearest) const { visit(lo, hi, nearest, ctx); }
};

// A C skyline query as the functor the shared quadrature calls; a NULL query hands over nothing.
struct QueryThunk {
    qm_skyline_query_fn query;
    void *user;
    template <class Visit>
    void operator()(double lo, double hi, double radius, Visit &visit) const {
        if (query == nullptr) return;
        query(lo, hi, radius, [](double a, double b, double nearest, void *ctx) { (*static_cast<Visit *>(ctx))(a, b, nearest); },
              &visit, user);
    }
};

}  // namespace

extern "C" {

qm_status qm_line_quadrature_nodes(const double start[3], const double end[3], qm_skyline_query_fn skyline,
                                   void *user, qm_line_node *nodes, size_t cap, size_t *n_nodes,
                                   qm_line_piece_info *info) {
    if (start == nullptr || end == nullptr || n_nodes == nullptr || (cap > 0 && nodes == nullptr))
        return qm::set_error(QM_ERR_ARGUMENT, "qm_line_quadrature_nodes: null start, end, n_nodes or nodes");
    for (int k = 0; k < 3; ++k)
        if (!std::isfinite(start[k]) || !std::isfinite(end[k]))
            return qm::set_error(QM_ERR_ARGUMENT, "qm_line_quadrature_nodes: a coordinate is not finite");
    *n_nodes = 0;
    qm::line::Piece g;
    if (!g.make(start, end)) {
        if (info != nullptr) {
            std::memset(info, 0, sizeof(*info));
            info->length_m = std::sqrt((end[0] - start[0]) * (end[0] - start[0]) + (end[1] - start[1]) * (end[1] - start[1]) +
                                       (end[2] - start[2]) * (end[2] - start[2]));
        }
        return QM_OK;
    }
    if (info != nullptr) {
        info->length_m = g.length;
        info->subtended_angle_rad = g.span();
        info->divergence_factor = g.divergence();
        info->start_angle_rad = g.angle0;
    }
    size_t count = 0;
    auto emit = [&](double along, double weight, bool on_ray) {
        if (count < cap) nodes[count] = qm_line_node{along, weight, on_ray ? 1u : 0u, 0u};
        ++count;
    };
    QueryThunk query{skyline, user};
    qm::line::quadrature_nodes(g, query, emit);
    *n_nodes = count;
    if (count > cap)
        return qm::set_error(QM_ERR_CAPACITY, "qm_line_quadrature_nodes: " + std::to_string(count) +
                                                  " nodes, room for " + std::to_string(cap));
    return QM_OK;
}

qm_status qm_skyline_build(const int32_t *vertices, size_t n_vertices, const qm_outline *outlines,
                           size_t n_outlines, double step_m, qm_skyline **out) {
    if (out == nullptr) return qm::set_error(QM_ERR_ARGUMENT, "qm_skyline_build: null out");
    *out = nullptr;
    if (!(step_m > 0.0) || !std::isfinite(step_m))
        return qm::set_error(QM_ERR_ARGUMENT, "qm_skyline_build: step_m must be positive and finite");
    if ((n_vertices > 0 && vertices == nullptr) || (n_outlines > 0 && outlines == nullptr))
        return qm::set_error(QM_ERR_ARGUMENT, "qm_skyline_build: null vertices or outlines");
    for (size_t o = 0; o < n_outlines; ++o)
        if ((uint64_t)outlines[o].first_vertex + outlines[o].vertex_count > n_vertices)
            return qm::set_error(QM_ERR_ARGUMENT, "qm_skyline_build: outline " + std::to_string(o) +
                                                      " lists vertices past the end of the array");
    if (n_outlines > UINT32_MAX) return qm::set_error(QM_ERR_ARGUMENT, "qm_skyline_build: too many outlines");
    qm_skyline *sky = new (std::nothrow) qm_skyline;
    if (sky == nullptr) return qm::set_error(QM_ERR_CAPACITY, "qm_skyline_build: out of host memory");
    try {
        sky->vertices.assign(vertices, vertices + 2 * n_vertices);
        sky->outlines.assign(outlines, outlines + n_outlines);
        sky->step_m = step_m;
        // Each cell's runs in the order its edges were listed, and its tallest outline.
        std::map<uint64_t, std::pair<std::vector<qm::skyline::Run>, float>> cells;
        for (uint32_t o = 0; o < (uint32_t)n_outlines; ++o) {
            const qm_outline &rec = outlines[o];
            for (uint32_t k = 0; k + 1 < rec.vertex_count; ++k) {
                const size_t e = (size_t)rec.first_vertex + k;
                auto list = [&](int64_t column, int64_t row) {
                    auto found = cells.find(qm::skyline::cell_key(column, row));
                    if (found == cells.end())
                        found = cells.emplace(qm::skyline::cell_key(column, row),
                                              std::make_pair(std::vector<qm::skyline::Run>(), -INFINITY))
                                    .first;
                    std::vector<qm::skyline::Run> &runs = found->second.first;
                    if (!runs.empty() && runs.back().outline == o && runs.back().first_edge + runs.back().count == k)
                        ++runs.back().count;
                    else
                        runs.push_back(qm::skyline::Run{o, k, 1});
                    found->second.second = std::fmax(found->second.second, rec.height_m);
                };
                qm::skyline::edge_cells(vertices[2 * e], -(int64_t)vertices[2 * e + 1], vertices[2 * e + 2],
                                        -(int64_t)vertices[2 * e + 3], list);
            }
        }
        if (cells.size() >= UINT32_MAX) throw std::length_error("cells");
        sky->keys.reserve(cells.size());
        sky->tallest.reserve(cells.size());
        sky->run_start.reserve(cells.size() + 1);
        sky->run_start.push_back(0);
        for (const auto &cell : cells) {
            sky->keys.push_back(cell.first);
            sky->tallest.push_back(cell.second.second);
            sky->runs.insert(sky->runs.end(), cell.second.first.begin(), cell.second.first.end());
            if (sky->runs.size() >= UINT32_MAX) throw std::length_error("runs");
            sky->run_start.push_back((uint32_t)sky->runs.size());
        }
    } catch (const std::exception &) {
        delete sky;
        return qm::set_error(QM_ERR_CAPACITY, "qm_skyline_build: out of host memory or index space");
    }
    *out = sky;
    return QM_OK;
}

qm_status qm_skyline_counts(const qm_skyline *skyline, size_t *n_cells, size_t *n_runs) {
    if (skyline == nullptr || n_cells == nullptr || n_runs == nullptr)
        return qm::set_error(QM_ERR_ARGUMENT, "qm_skyline_counts: null argument");
    *n_cells = skyline->keys.size();
    *n_runs = skyline->runs.size();
    return QM_OK;
}

qm_status qm_skyline_arcs(const qm_skyline *skyline, int64_t x, int64_t y, double lo_rad, double hi_rad,
                          double radius_m, double floor_m, double *arcs, size_t cap, size_t *n_arcs) {
    if (skyline == nullptr || n_arcs == nullptr || (cap > 0 && arcs == nullptr))
        return qm::set_error(QM_ERR_ARGUMENT, "qm_skyline_arcs: null skyline, n_arcs or arcs");
    if (!std::isfinite(lo_rad) || !std::isfinite(hi_rad) || std::isnan(radius_m) || std::isnan(floor_m))
        return qm::set_error(QM_ERR_ARGUMENT, "qm_skyline_arcs: a wedge edge is not finite or a bound is NaN");
    size_t count = 0;
    auto visit = [&](double lo, double hi, double nearest) {
        if (count < cap) {
            arcs[3 * count] = lo;
            arcs[3 * count + 1] = hi;
            arcs[3 * count + 2] = nearest;
        }
        ++count;
    };
    qm::skyline::arcs(skyline->view(), x, y, lo_rad, hi_rad, radius_m, floor_m, visit);
    *n_arcs = count;
    if (count > cap)
        return qm::set_error(QM_ERR_CAPACITY,
                             "qm_skyline_arcs: " + std::to_string(count) + " arcs, room for " + std::to_string(cap));
    return QM_OK;
}

void qm_skyline_free(qm_skyline *skyline) { delete skyline; }

void qm_skyline_query(double wedge_lo_rad, double wedge_hi_rad, double radius_m, qm_skyline_visit_fn visit,
                      void *visit_ctx, void *user) {
    const qm_skyline_receiver *r = static_cast<const qm_skyline_receiver *>(user);
    if (r == nullptr || r->skyline == nullptr || visit == nullptr) return;
    VisitThunk thunk{visit, visit_ctx};
    qm::skyline::arcs(r->skyline->view(), r->x, r->y, wedge_lo_rad, wedge_hi_rad, radius_m, r->floor_m, thunk);
}

}  // extern "C"

namespace qm {
// The index's host arrays (the library uploads them for the device's line pairs); the run count is
// run_start[n_cells].
skyline::Index skyline_view(const qm_skyline *s) { return s->view(); }
}  // namespace qm
