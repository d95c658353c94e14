// The C ABI of include/qm_batch.h: context, scene upload (obstacle grid cell lists, dense footprint
// ids, DEM), the grid painter, the pair evaluator, Zwicker loudness and level histograms.
//
// Host conventions follow the reference's card host (paint-gpu/src/device.rs): arguments are
// validated before any device work and the error names the argument (device.rs:450-473); CUDA
// failures read "cuda: ..." (device.rs:249-251). There is no CPU fallback: a pair the device cannot
// finish is retried on the device with larger per-path capacities, and a call that still cannot
// finish returns QM_ERR_CAPACITY.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cerrno>
#include <dlfcn.h>
#include <cstring>
#include <memory>
#include <mutex>
#include <random>
#include <string>
#include <unordered_map>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/qm_batch.h"
#include "../../include/qm_surrogate.h"
#include "../../include/qm_terrain.h"
#include "../../include/qm_obstacles.h"
#include "../../include/qm_tiles.h"
#include "../../include/qm_weather.h"
#include "qm_aircraft.cuh"
#include "qm_flights.cuh"
#include "qm_horizons.cuh"
#include "qm_kernels.cuh"
#include "qm_linepairs.cuh"
#include "qm_host.h"
#include "../../include/qm_line.h"

namespace qm {
skyline::Index skyline_view(const qm_skyline *s);
}
#include "qm_mlp.h"
#include "qm_percentile.cuh"
#include "qm_pixel.cuh"
#include "../../include/qm_distribution.h"
#include "qm_surrogate.cuh"
#include "qm_tiles.cuh"

#include <climits>

namespace qm {
void launch_zwicker(const float *thirds, size_t n, float *sone, cudaStream_t stream);
}  // namespace qm

using namespace qm;

static thread_local std::string g_last_error;

qm_status qm::set_error(qm_status status, const std::string &message) {
    g_last_error = message;
    return status;
}

const std::string &qm::last_error() { return g_last_error; }

struct qm_ctx {
    int device;
    int sm_count;
    cudaStream_t stream;
    std::mutex lock;
    // Scenes and networks made on the context hold it: qm_close releases it once they are freed.
    int children = 0;
    bool closed = false;
    float *line_table = nullptr;  // the line-level quantile table on the device, on first use
};

struct DeviceBuffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer &) = delete;
    DeviceBuffer &operator=(const DeviceBuffer &) = delete;
    ~DeviceBuffer() {
        if (ptr) cudaFree(ptr);
    }
};

// A device buffer that grows to the largest size asked of it and is kept between calls.
struct GrowBuffer {
    void *p = nullptr;
    size_t bytes = 0;
    GrowBuffer() = default;
    GrowBuffer(const GrowBuffer &) = delete;
    GrowBuffer &operator=(const GrowBuffer &) = delete;
    ~GrowBuffer() {
        if (p) cudaFree(p);
    }
    cudaError_t reserve(size_t want) {
        want = std::max<size_t>(want, 16);
        if (want <= bytes) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) bytes = want;
        return e;
    }
};

// A pinned host buffer that grows to the largest size asked of it and is kept between calls.
struct PinnedBuffer {
    void *p = nullptr;
    size_t bytes = 0;
    PinnedBuffer() = default;
    PinnedBuffer(const PinnedBuffer &) = delete;
    PinnedBuffer &operator=(const PinnedBuffer &) = delete;
    ~PinnedBuffer() {
        if (p) cudaFreeHost(p);
    }
    cudaError_t reserve(size_t want) {
        want = std::max<size_t>(want, 16);
        if (want <= bytes) return cudaSuccess;
        if (p) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaHostAlloc(&p, want, cudaHostAllocDefault);
        if (e == cudaSuccess) bytes = want;
        return e;
    }
};

struct qm_scene {
    qm_ctx *ctx;
    SceneDev dev;
    std::vector<DeviceBuffer *> buffers;
    // Host copies for receiver preparation.
    double step_m;
    int extent[2];
    std::vector<int32_t> vertices;
    std::vector<qm_outline> outlines;
    std::vector<uint64_t> fp_sorted;  // dense id = index + 1
    int dem_nx, dem_ny, dem_ox, dem_oy, dem_sp;
    std::vector<float> dem_z, dem_g;
    float flat_z, flat_g;
    uint32_t n_sources;
    std::vector<uint32_t> source_layer;
    bool any_favourable;
    size_t n_edges_listed;
    // Line pieces (qm_scene_line_pieces): candidates n_sources .. n_sources + n_pieces - 1, and the
    // receivers' skyline index on the device; replaced whole when set again.
    uint32_t n_pieces = 0;
    std::vector<uint32_t> piece_layer;
    const qm::PieceDev *pieces = nullptr;
    qm::skyline::Index sky{};
    std::vector<DeviceBuffer *> piece_buffers;
    // qm_paint_grid's device buffers, kept between calls and grown as a call needs (the call holds
    // the context's lock throughout, so calls on the scene never share them at once).
    struct GridScratch {
        GrowBuffer alt, own, partial, failed, counters, dba, retry, rcount, bands, dbaout, lden, hist;
    } grid_scratch;
    // Batch plans made on the scene hold it: qm_scene_free releases it once they are freed.
    int plans = 0;
    bool freed = false;
    ~qm_scene() {
        for (auto *b : buffers) delete b;
        for (auto *b : piece_buffers) delete b;
    }
};

namespace {

qm_status fail(qm_status status, const std::string &message) {
    g_last_error = message;
    return status;
}

void ctx_destroy(qm_ctx *ctx) {
    cudaSetDevice(ctx->device);
    if (ctx->line_table) cudaFree(ctx->line_table);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
}

// One holder of the context gone: the context goes too once it is closed and holds nothing.
void ctx_release(qm_ctx *ctx) {
    bool last;
    {
        std::lock_guard<std::mutex> guard(ctx->lock);
        last = --ctx->children == 0 && ctx->closed;
    }
    if (last) ctx_destroy(ctx);
}

#define QM_CUDA(call)                                                                  \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) return fail(QM_ERR_CUDA, std::string("cuda: ") + cudaGetErrorString(e_) + " (" #call ")"); \
    } while (0)

template <class T>
qm_status upload(qm_scene *s, const T *host, size_t count, const T **out) {
    auto *b = new DeviceBuffer();
    s->buffers.push_back(b);
    b->bytes = std::max<size_t>(count * sizeof(T), 16);
    QM_CUDA(cudaMalloc(&b->ptr, b->bytes));
    if (count) QM_CUDA(cudaMemcpy(b->ptr, host, count * sizeof(T), cudaMemcpyHostToDevice));
    *out = static_cast<const T *>(b->ptr);
    return QM_OK;
}

// A device allocation freed when the holder leaves scope.
// A device buffer freed when its owner leaves scope. Move-only: a copy would free the buffer
// twice (and leave the other copy pointing at freed memory), e.g. when a vector of structs that
// hold one grows.
struct Scratch {
    void *p = nullptr;
    Scratch() = default;
    Scratch(const Scratch &) = delete;
    Scratch &operator=(const Scratch &) = delete;
    Scratch(Scratch &&o) noexcept : p(o.p) { o.p = nullptr; }
    ~Scratch() {
        if (p) cudaFree(p);
    }
};

// Timing events destroyed when the holder leaves scope (not copyable, for the same reason).
// A named NVTX range over an entry point's host and device work (a profiler's timeline shows each
// call; without a tool attached a range costs a test of a null pointer).
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

struct Events {
    Events() = default;
    Events(const Events &) = delete;
    Events &operator=(const Events &) = delete;
    cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr;
    cudaError_t create() {
        cudaError_t e = cudaEventCreate(&e0);
        if (e == cudaSuccess) e = cudaEventCreate(&e1);
        return e != cudaSuccess ? e : cudaEventCreate(&e2);
    }
    ~Events() {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (e2) cudaEventDestroy(e2);
    }
};

bool segment_meets_box(int64_t ax, int64_t ay, int64_t bx, int64_t by, int64_t x0, int64_t y0, int64_t x1, int64_t y1) {
    if (std::max(ax, bx) < x0 || std::min(ax, bx) > x1 || std::max(ay, by) < y0 || std::min(ay, by) > y1) return false;
    int64_t dx = bx - ax, dy = by - ay;
    int pos = 0, neg = 0;
    const int64_t cx[4] = {x0, x1, x0, x1}, cy[4] = {y0, y0, y1, y1};
    for (int k = 0; k < 4; ++k) {
        int64_t c = dx * (cy[k] - ay) - dy * (cx[k] - ax);
        pos += c > 0;
        neg += c < 0;
    }
    return !(pos == 4 || neg == 4);
}

uint32_t dense_fp(const qm_scene *s, uint64_t fp) {
    if (fp == 0) return 0;
    auto it = std::lower_bound(s->fp_sorted.begin(), s->fp_sorted.end(), fp);
    if (it == s->fp_sorted.end() || *it != fp) return 0xFFFFFFFFu;  // matches no outline
    return (uint32_t)(it - s->fp_sorted.begin()) + 1;
}

bool point_in_ring(const qm_scene *s, const qm_outline &o, int64_t x, int64_t y) {
    bool inside = false;
    for (uint32_t k = 0; k + 1 < o.vertex_count; ++k) {
        uint32_t e = o.first_vertex + k;
        int64_t ax = s->vertices[2 * e], ay = s->vertices[2 * e + 1];
        int64_t bx = s->vertices[2 * e + 2], by = s->vertices[2 * e + 3];
        if ((ay > y) != (by > y)) {
            int64_t lhs = (x - ax) * (by - ay), rhs = (y - ay) * (bx - ax);
            if (by - ay > 0 ? lhs < rhs : lhs > rhs) inside = !inside;
        }
    }
    return inside;
}

// Ground altitude and G at a lattice point: bilinear between the DEM nodes around it.
double terrain_altitude(const qm_scene *s, int64_t x, int64_t y) {
    if (s->dem_nx == 0) return s->flat_z;
    double fx = (double)(x - s->dem_ox) / s->dem_sp, fy = (double)(y - s->dem_oy) / s->dem_sp;
    fx = std::min(std::max(fx, 0.0), (double)(s->dem_nx - 1));
    fy = std::min(std::max(fy, 0.0), (double)(s->dem_ny - 1));
    int64_t i0 = std::min<int64_t>((int64_t)std::floor(fx), s->dem_nx - 2);
    int64_t j0 = std::min<int64_t>((int64_t)std::floor(fy), s->dem_ny - 2);
    double ax = fx - i0, ay = fy - j0;
    auto node = [&](int64_t i, int64_t j) { return (double)s->dem_z[j * s->dem_nx + i]; };
    double lo = node(i0, j0) + ax * (node(i0 + 1, j0) - node(i0, j0));
    double hi = node(i0, j0 + 1) + ax * (node(i0 + 1, j0 + 1) - node(i0, j0 + 1));
    return lo + ay * (hi - lo);
}

void band_constants(BandConstants &bc) {
    const double f[8] = {63.0, 125.0, 250.0, 500.0, 1000.0, 2000.0, 4000.0, 8000.0};
    const double pi = 3.141592653589793116;
    for (int b = 0; b < 8; ++b) {
        bc.f25[b] = (float)std::pow(f[b], 2.5);
        bc.f15[b] = (float)std::pow(f[b], 1.5);
        bc.f075[b] = (float)std::pow(f[b], 0.75);
        bc.k[b] = (float)(2.0 * pi * f[b] / 340.0);
        bc.lambda[b] = (float)(340.0 / f[b]);
        bc.inv_lambda[b] = (float)(f[b] / 340.0);
        bc.lambda_d[b] = 340.0 / f[b];
        bc.lambda_over_20_d[b] = bc.lambda_d[b] / 20.0;
        bc.lambda_over_4_d[b] = bc.lambda_d[b] / 4.0;
    }
}

const double LDEN_W[3] = {12.0 / 24.0, 4.0 / 24.0 * 3.1622776601683795, 8.0 / 24.0 * 10.0};

}  // namespace

extern "C" {

int qm_abi_version(void) { return QM_ABI_VERSION; }

const char *qm_last_error(const qm_ctx *) { return g_last_error.c_str(); }

qm_status qm_open(int device_ordinal, qm_ctx **out) {
    if (!out) return fail(QM_ERR_ARGUMENT, "qm_open: out is null");
    *out = nullptr;
    int count = 0;
    QM_CUDA(cudaGetDeviceCount(&count));
    if (device_ordinal < 0 || device_ordinal >= count)
        return fail(QM_ERR_ARGUMENT, "qm_open: device_ordinal outside the visible devices");
    cudaDeviceProp prop;
    QM_CUDA(cudaGetDeviceProperties(&prop, device_ordinal));
    if (prop.major != 10)
        return fail(QM_ERR_UNSUPPORTED, "qm_open: this library is built for sm_100 (B200); the device is sm_" +
                                            std::to_string(prop.major * 10 + prop.minor));
    QM_CUDA(cudaSetDevice(device_ordinal));
    BandConstants bc;
    band_constants(bc);
    QM_CUDA(cudaMemcpyToSymbol(c_band, &bc, sizeof(bc)));
    auto *ctx = new qm_ctx();
    ctx->device = device_ordinal;
    ctx->sm_count = prop.multiProcessorCount;
    cudaError_t e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete ctx;
        return fail(QM_ERR_CUDA, std::string("cuda: ") + cudaGetErrorString(e));
    }
    *out = ctx;
    g_last_error.clear();
    return QM_OK;
}

void qm_close(qm_ctx *ctx) {
    if (!ctx) return;
    bool now;
    {
        std::lock_guard<std::mutex> guard(ctx->lock);
        ctx->closed = true;
        now = ctx->children == 0;
    }
    if (now) ctx_destroy(ctx);
}

qm_status qm_scene_upload(qm_ctx *ctx, const qm_scene_desc *d, qm_scene **out) {
    NvtxRange nvtx_range("qm_scene_upload");
    if (!ctx || !d || !out) return fail(QM_ERR_ARGUMENT, "qm_scene_upload: null ctx, desc or out");
    *out = nullptr;
    if (!(d->step_m > 0.0) || !std::isfinite(d->step_m)) return fail(QM_ERR_ARGUMENT, "qm_scene_upload: step_m");
    if (d->cell_steps < 16) return fail(QM_ERR_ARGUMENT, "qm_scene_upload: cell_steps below 16");
    const int64_t LIM = int64_t(1) << 27;  // coordinates within 2^27 steps keep every product exact
    if (d->extent_steps[0] <= 0 || d->extent_steps[1] <= 0 || d->extent_steps[0] > LIM || d->extent_steps[1] > LIM)
        return fail(QM_ERR_ARGUMENT, "qm_scene_upload: extent_steps");
    if (d->n_vertices && !d->vertices) return fail(QM_ERR_ARGUMENT, "qm_scene_upload: vertices is null");
    if (d->n_outlines && !d->outlines) return fail(QM_ERR_ARGUMENT, "qm_scene_upload: outlines is null");
    if (d->n_sources && !d->sources) return fail(QM_ERR_ARGUMENT, "qm_scene_upload: sources is null");
    for (uint32_t i = 0; i < 2 * d->n_vertices; ++i)
        if (d->vertices[i] < -LIM || d->vertices[i] > LIM)
            return fail(QM_ERR_ARGUMENT, "qm_scene_upload: a vertex beyond 2^27 steps");
    for (uint32_t o = 0; o < d->n_outlines; ++o) {
        const qm_outline &ol = d->outlines[o];
        if (ol.vertex_count < 2 || (uint64_t)ol.first_vertex + ol.vertex_count > d->n_vertices)
            return fail(QM_ERR_ARGUMENT, "qm_scene_upload: outline " + std::to_string(o) + " vertices out of range");
        if (ol.footprint_id == 0) return fail(QM_ERR_ARGUMENT, "qm_scene_upload: outline footprint_id 0");
        if (ol.building) {
            const int32_t *a = d->vertices + 2 * (size_t)ol.first_vertex;
            const int32_t *b = d->vertices + 2 * ((size_t)ol.first_vertex + ol.vertex_count - 1);
            if (ol.vertex_count < 4 || a[0] != b[0] || a[1] != b[1])
                return fail(QM_ERR_ARGUMENT, "qm_scene_upload: building outline " + std::to_string(o) + " is not a closed ring");
        }
        if (!std::isfinite(ol.height_m)) return fail(QM_ERR_ARGUMENT, "qm_scene_upload: outline height_m");
    }
    if (d->dem_nx != 0) {
        if (d->dem_nx < 2 || d->dem_ny < 2 || d->dem_spacing <= 0 || !d->dem_altitude_m || !d->dem_ground_factor)
            return fail(QM_ERR_ARGUMENT, "qm_scene_upload: dem dimensions, spacing or arrays");
    }
    for (uint32_t i = 0; i < d->n_sources; ++i) {
        const qm_source &s = d->sources[i];
        if (s.x < 0 || s.y < 0 || s.x >= d->extent_steps[0] || s.y >= d->extent_steps[1])
            return fail(QM_ERR_ARGUMENT, "qm_scene_upload: source " + std::to_string(i) + " outside the extent");
        if (s.layer >= QM_LAYERS) return fail(QM_ERR_ARGUMENT, "qm_scene_upload: source layer");
    }
    QM_CUDA(cudaSetDevice(ctx->device));
    auto *s = new qm_scene();
    s->ctx = ctx;
    s->step_m = d->step_m;
    s->extent[0] = d->extent_steps[0];
    s->extent[1] = d->extent_steps[1];
    s->vertices.assign(d->vertices, d->vertices + 2 * (size_t)d->n_vertices);
    s->outlines.assign(d->outlines, d->outlines + d->n_outlines);
    for (auto &o : s->outlines) s->fp_sorted.push_back(o.footprint_id);
    std::sort(s->fp_sorted.begin(), s->fp_sorted.end());
    s->fp_sorted.erase(std::unique(s->fp_sorted.begin(), s->fp_sorted.end()), s->fp_sorted.end());
    if (s->fp_sorted.size() >= 0xFFFFFFFEu) {
        delete s;
        return fail(QM_ERR_ARGUMENT, "qm_scene_upload: too many footprints");
    }
    // Obstacle grid: every edge in every cell whose closed box it meets.
    const int64_t C = d->cell_steps;
    const int cells_x = (int)((d->extent_steps[0] + C - 1) / C), cells_y = (int)((d->extent_steps[1] + C - 1) / C);
    std::vector<uint32_t> counts((size_t)cells_x * cells_y + 1, 0);
    struct Entry {
        uint32_t cell, edge, outline;
    };
    std::vector<Entry> entries;
    for (uint32_t o = 0; o < d->n_outlines; ++o) {
        const qm_outline &ol = d->outlines[o];
        for (uint32_t k = 0; k + 1 < ol.vertex_count; ++k) {
            uint32_t e = ol.first_vertex + k;
            int64_t ax = d->vertices[2 * e], ay = d->vertices[2 * e + 1];
            int64_t bx = d->vertices[2 * e + 2], by = d->vertices[2 * e + 3];
            auto fl = [&](int64_t v) { return (int64_t)std::floor((double)v / (double)C); };
            int64_t cx0 = std::max<int64_t>(0, fl(std::min(ax, bx)) - 1), cx1 = std::min<int64_t>(cells_x - 1, fl(std::max(ax, bx)) + 1);
            int64_t cy0 = std::max<int64_t>(0, fl(std::min(ay, by)) - 1), cy1 = std::min<int64_t>(cells_y - 1, fl(std::max(ay, by)) + 1);
            for (int64_t cy = cy0; cy <= cy1; ++cy)
                for (int64_t cx = cx0; cx <= cx1; ++cx)
                    if (segment_meets_box(ax, ay, bx, by, cx * C, cy * C, (cx + 1) * C, (cy + 1) * C))
                        entries.push_back(Entry{(uint32_t)(cy * cells_x + cx), e, o});
        }
    }
    std::stable_sort(entries.begin(), entries.end(), [](const Entry &a, const Entry &b) { return a.cell < b.cell; });
    std::vector<uint32_t> cell_start((size_t)cells_x * cells_y + 1, 0);
    std::vector<int4> cell_seg(entries.size());
    std::vector<uint2> cell_ref(entries.size());
    for (size_t i = 0; i < entries.size(); ++i) {
        const Entry &en = entries[i];
        cell_start[en.cell + 1]++;
        cell_seg[i] = make_int4(d->vertices[2 * en.edge], d->vertices[2 * en.edge + 1], d->vertices[2 * en.edge + 2],
                                d->vertices[2 * en.edge + 3]);
        cell_ref[i] = make_uint2(en.edge, en.outline);
    }
    for (size_t c = 1; c < cell_start.size(); ++c) cell_start[c] += cell_start[c - 1];
    std::vector<uint2> cell_range((size_t)cells_x * cells_y);
    for (size_t c = 0; c < cell_range.size(); ++c) cell_range[c] = make_uint2(cell_start[c], cell_start[c + 1]);
    // The same entries column by column (cell (cx, cy) at cx * cells_y + cy), each cell's entries
    // in the row-ordered copy's order.
    std::vector<uint32_t> col_order(entries.size());
    for (size_t i = 0; i < col_order.size(); ++i) col_order[i] = (uint32_t)i;
    auto col_key = [&](uint32_t i) {
        const uint32_t c = entries[i].cell;
        return (uint64_t)(c % (uint32_t)cells_x) * (uint64_t)cells_y + c / (uint32_t)cells_x;
    };
    std::stable_sort(col_order.begin(), col_order.end(), [&](uint32_t a, uint32_t b) { return col_key(a) < col_key(b); });
    std::vector<int4> col_seg(entries.size());
    std::vector<uint2> col_ref(entries.size());
    std::vector<uint2> col_range((size_t)cells_x * cells_y, make_uint2(0u, 0u));
    for (size_t k = 0; k < col_order.size(); ++k) {
        const uint32_t i = col_order[k];
        col_seg[k] = cell_seg[i];
        col_ref[k] = cell_ref[i];
    }
    {
        // Each column-ordered cell's range; empty cells start where the next entries do.
        size_t k = 0;
        for (uint64_t key = 0; key < (uint64_t)cells_x * cells_y; ++key) {
            const size_t b = k;
            while (k < col_order.size() && col_key(col_order[k]) == key) ++k;
            col_range[key] = make_uint2((uint32_t)b, (uint32_t)k);
        }
    }
    s->n_edges_listed = entries.size();
    std::vector<OutlineDev> outl(d->n_outlines);
    for (uint32_t o = 0; o < d->n_outlines; ++o) {
        const qm_outline &ol = d->outlines[o];
        outl[o] = OutlineDev{ol.first_vertex, ol.vertex_count, dense_fp(s, ol.footprint_id), ol.building ? 1u : 0u,
                             ol.height_m, {0, 0, 0}};
    }
    std::vector<SourceDev> src(d->n_sources);
    s->source_layer.resize(d->n_sources);
    for (uint32_t i = 0; i < d->n_sources; ++i) {
        const qm_source &q = d->sources[i];
        SourceDev &v = src[i];
        v.x = q.x;
        v.y = q.y;
        v.height = q.height_m;
        v.gf = q.ground_factor;
        v.excl = q.exclusion_radius_m;
        v.platform = q.platform_half_width_m;
        v.fp = dense_fp(s, q.footprint_id);
        v.layer = q.layer;
        for (int p = 0; p < 3; ++p)
            for (int b = 0; b < 8; ++b) v.energy[p * 8 + b] = q.energy[p][b];
        s->source_layer[i] = q.layer;
    }
    s->n_sources = d->n_sources;
    s->dem_nx = d->dem_nx;
    s->dem_ny = d->dem_ny;
    s->dem_ox = d->dem_origin[0];
    s->dem_oy = d->dem_origin[1];
    s->dem_sp = d->dem_spacing;
    s->flat_z = d->flat_altitude_m;
    s->flat_g = d->flat_ground_factor;
    std::vector<float2> dem;
    if (d->dem_nx) {
        size_t n = (size_t)d->dem_nx * d->dem_ny;
        s->dem_z.assign(d->dem_altitude_m, d->dem_altitude_m + n);
        s->dem_g.assign(d->dem_ground_factor, d->dem_ground_factor + n);
        dem.resize(n);
        for (size_t i = 0; i < n; ++i) dem[i] = make_float2(d->dem_altitude_m[i], d->dem_ground_factor[i]);
    }
    s->any_favourable = false;
    for (int p = 0; p < 3; ++p)
        for (int k = 0; k < 16; ++k)
            if (d->favourable[p][k] != 0.0f) s->any_favourable = true;
    SceneDev &dv = s->dev;
    std::memset(&dv, 0, sizeof(dv));
    dv.step_m = (float)d->step_m;
    dv.cell_steps = d->cell_steps;
    dv.cells_x = cells_x;
    dv.cells_y = cells_y;
    qm_status st;
    if ((st = upload(s, cell_range.data(), cell_range.size(), &dv.cell_range)) != QM_OK ||
        (st = upload(s, col_range.data(), col_range.size(), &dv.col_range)) != QM_OK ||
        (st = upload(s, col_seg.data(), col_seg.size(), &dv.col_seg)) != QM_OK ||
        (st = upload(s, col_ref.data(), col_ref.size(), &dv.col_ref)) != QM_OK ||
        (st = upload(s, cell_seg.data(), cell_seg.size(), &dv.cell_seg)) != QM_OK ||
        (st = upload(s, cell_ref.data(), cell_ref.size(), &dv.cell_ref)) != QM_OK ||
        (st = upload(s, reinterpret_cast<const int2 *>(d->vertices), (size_t)d->n_vertices, &dv.vertices)) != QM_OK ||
        (st = upload(s, outl.data(), outl.size(), &dv.outlines)) != QM_OK ||
        (st = upload(s, src.data(), src.size(), &dv.sources)) != QM_OK ||
        (st = upload(s, dem.data(), dem.size(), &dv.dem)) != QM_OK) {
        delete s;
        return st;
    }
    dv.dem_nx = d->dem_nx;
    dv.dem_ny = d->dem_ny;
    dv.dem_ox = d->dem_origin[0];
    dv.dem_oy = d->dem_origin[1];
    dv.dem_sp = d->dem_spacing;
    dv.flat_z = d->flat_altitude_m;
    dv.flat_g = d->flat_ground_factor;
    dv.n_sources = d->n_sources;
    std::memcpy(dv.fav, d->favourable, sizeof(dv.fav));
    std::memcpy(dv.alpha, d->alpha_db_per_km, sizeof(dv.alpha));
    for (int b = 0; b < 8; ++b) dv.air_per_m[b] = (float)((double)d->alpha_db_per_km[b] * (2.302585092994046 / 10.0 / 1000.0));
    {
        std::lock_guard<std::mutex> guard(ctx->lock);
        ++ctx->children;
    }
    *out = s;
    return QM_OK;
}

void qm_scene_free(qm_scene *scene) {
    if (!scene) return;
    qm_ctx *ctx = scene->ctx;
    bool now;
    {
        std::lock_guard<std::mutex> guard(ctx->lock);
        scene->freed = true;
        now = scene->plans == 0;
    }
    if (!now) return;  // its last plan's qm_batch_plan_free deletes it
    cudaSetDevice(ctx->device);
    delete scene;
    ctx_release(ctx);
}

}  // extern "C"

namespace {

// Receiver altitude (ground + height) and dense own footprint of each grid cell.
void grid_receivers(const qm_scene *s, const qm_grid_desc *g, std::vector<float> &alt, std::vector<uint32_t> &own) {
    size_t cells = (size_t)g->nx * g->ny;
    alt.resize(cells);
    own.assign(cells, 0);
    std::vector<uint64_t> own64(cells, 0);
    for (size_t c = 0; c < cells; ++c) {
        int64_t x = g->origin[0] + (int64_t)(c % g->nx) * g->spacing, y = g->origin[1] + (int64_t)(c / g->nx) * g->spacing;
        alt[c] = (float)(terrain_altitude(s, x, y) + g->height_m);
    }
    // The building a receiver stands in: the lowest footprint id among the rings containing it (a
    // ring without a footprint id, 0, names no building).
    for (const qm_outline &o : s->outlines) {
        if (!o.building || o.vertex_count < 4 || o.footprint_id == 0) continue;
        int64_t x0 = INT64_MAX, x1 = INT64_MIN, y0 = INT64_MAX, y1 = INT64_MIN;
        for (uint32_t k = 0; k < o.vertex_count; ++k) {
            int64_t vx = s->vertices[2 * (o.first_vertex + k)], vy = s->vertices[2 * (o.first_vertex + k) + 1];
            x0 = std::min(x0, vx);
            x1 = std::max(x1, vx);
            y0 = std::min(y0, vy);
            y1 = std::max(y1, vy);
        }
        auto lo = [&](int64_t v, int32_t origin) {
            int64_t k = (int64_t)std::ceil((double)(v - origin) / g->spacing);
            return std::max<int64_t>(k, 0);
        };
        auto hi = [&](int64_t v, int32_t origin, int n) {
            int64_t k = (int64_t)std::floor((double)(v - origin) / g->spacing);
            return std::min<int64_t>(k, n - 1);
        };
        for (int64_t j = lo(y0, g->origin[1]); j <= hi(y1, g->origin[1], g->ny); ++j)
            for (int64_t i = lo(x0, g->origin[0]); i <= hi(x1, g->origin[0], g->nx); ++i) {
                int64_t x = g->origin[0] + i * g->spacing, y = g->origin[1] + j * g->spacing;
                if (point_in_ring(s, o, x, y)) {
                    uint64_t &cur = own64[j * g->nx + i];
                    if (cur == 0 || o.footprint_id < cur) cur = o.footprint_id;
                }
            }
    }
    for (size_t c = 0; c < cells; ++c) own[c] = dense_fp(s, own64[c]);
}

// The larger per-path capacities: terrain scenes, and flat scenes whose rays may run longer than
// 1.5 km (more crossings than the flat capacities hold).
bool terrain_caps(const qm_scene *s) {
    double diagonal_m = std::hypot((double)s->extent[0], (double)s->extent[1]) * s->step_m;
    return s->dem_nx != 0 || diagonal_m > 1500.0;
}

// Re-runs a grid call's failed paths in (cell, source) order with large per-path capacities and
// sums them into the partial slice `slice`.
qm_status rerun_failed(qm_scene *scene, const GridArgs &A, const uint2 *d_retry, unsigned int n_retry, uint32_t slice,
                       int cells, cudaStream_t stream) {
    Scratch d_sorted, d_cids, d_cstart, d_works, d_results, d_rstatus;
    // Re-run the failed paths in (cell, source) order with large capacities.
    std::vector<uint2> list(n_retry);
    QM_CUDA(cudaMemcpy(list.data(), d_retry, n_retry * sizeof(uint2), cudaMemcpyDeviceToHost));
    std::sort(list.begin(), list.end(), [](uint2 a, uint2 b) { return a.x != b.x ? a.x < b.x : a.y < b.y; });
    std::vector<uint32_t> cids, cstart;
    for (uint32_t i = 0; i < n_retry; ++i)
        if (cids.empty() || cids.back() != list[i].x) {
            cids.push_back(list[i].x);
            cstart.push_back(i);
        }
    cstart.push_back(n_retry);
    const uint32_t threads = std::min<uint32_t>(((n_retry + 63) / 64) * 64, 8192);
    using Large = PathWork<CapsLarge::C, CapsLarge::K, CapsLarge::H>;
    QM_CUDA(cudaMalloc(&d_sorted.p, n_retry * sizeof(uint2)));
    QM_CUDA(cudaMalloc(&d_cids.p, cids.size() * sizeof(uint32_t)));
    QM_CUDA(cudaMalloc(&d_cstart.p, cstart.size() * sizeof(uint32_t)));
    QM_CUDA(cudaMalloc(&d_works.p, (size_t)threads * sizeof(Large)));
    QM_CUDA(cudaMalloc(&d_results.p, (size_t)n_retry * GRID_SLOTS * sizeof(float)));
    QM_CUDA(cudaMalloc(&d_rstatus.p, (size_t)n_retry * sizeof(uint32_t)));
    QM_CUDA(cudaMemcpyAsync(d_sorted.p, list.data(), n_retry * sizeof(uint2), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(d_cids.p, cids.data(), cids.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(d_cstart.p, cstart.data(), cstart.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    retry_paths_kernel<<<threads / 64, 64, 0, stream>>>(scene->dev, A, static_cast<uint2 *>(d_sorted.p), n_retry,
                                                        static_cast<Large *>(d_works.p),
                                                        static_cast<float *>(d_results.p),
                                                        static_cast<uint32_t *>(d_rstatus.p));
    QM_CUDA(cudaGetLastError());
    fold_retry_kernel<<<(unsigned)((cids.size() + 127) / 128), 128, 0, stream>>>(
        static_cast<uint32_t *>(d_cids.p), static_cast<uint32_t *>(d_cstart.p), (uint32_t)cids.size(),
        static_cast<float *>(d_results.p), A.partial, slice, cells);
    QM_CUDA(cudaGetLastError());
    std::vector<uint32_t> rstatus(n_retry);
    QM_CUDA(cudaMemcpyAsync(rstatus.data(), d_rstatus.p, n_retry * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaStreamSynchronize(stream));
    size_t still = 0;
    for (uint32_t v : rstatus) still += v != 0;
    if (still)
        return fail(QM_ERR_CAPACITY, "qm_paint_grid: " + std::to_string(still) +
                                         " paths exceed even the large per-path capacities");
    return QM_OK;
}


}  // namespace

extern "C" {

qm_status qm_paint_grid(qm_scene *scene, const qm_grid_desc *grid, float *cell_bands, float *cell_dba,
                        float *cell_lden, uint32_t *histogram, qm_paint_stats *stats) {
    NvtxRange nvtx_range("qm_paint_grid");
    if (!scene || !grid) return fail(QM_ERR_ARGUMENT, "qm_paint_grid: null scene or grid");
    const qm_grid_desc &g = *grid;
    if (g.nx <= 0 || g.ny <= 0 || g.spacing <= 0 || (int64_t)g.nx * g.ny > (int64_t(1) << 30))
        return fail(QM_ERR_ARGUMENT, "qm_paint_grid: grid nx, ny or spacing");
    int64_t last_x = g.origin[0] + (int64_t)(g.nx - 1) * g.spacing, last_y = g.origin[1] + (int64_t)(g.ny - 1) * g.spacing;
    if (g.origin[0] < 0 || g.origin[1] < 0 || last_x >= scene->extent[0] || last_y >= scene->extent[1])
        return fail(QM_ERR_ARGUMENT, "qm_paint_grid: grid receivers outside the scene extent");
    if (histogram && (g.n_bins == 0 || g.n_bins > 51200 || !(g.bin_db > 0.0)))
        return fail(QM_ERR_ARGUMENT, "qm_paint_grid: histogram needs 0 < n_bins <= 51200 and bin_db > 0");
    uint32_t sb = g.source_begin, se = g.source_end;
    if (se <= sb) {
        sb = 0;
        se = scene->n_sources;
    }
    if (se > scene->n_sources) return fail(QM_ERR_ARGUMENT, "qm_paint_grid: source range beyond the scene's sources");
    qm_ctx *ctx = scene->ctx;
    std::lock_guard<std::mutex> guard(ctx->lock);
    QM_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t stream = ctx->stream;
    const int cells = g.nx * g.ny;
    std::vector<float> alt;
    std::vector<uint32_t> own;
    grid_receivers(scene, grid, alt, own);
    GridArgs A{};
    A.origin_x = g.origin[0];
    A.origin_y = g.origin[1];
    A.spacing = g.spacing;
    A.nx = g.nx;
    A.ny = g.ny;
    A.height_m = g.height_m;
    A.source_begin = sb;
    A.source_end = se;
    A.tile_w = 16;
    A.tile_h = 8;
    A.want_fav = scene->any_favourable;
    for (int p = 0; p < 3; ++p) A.lden_w[p] = (float)LDEN_W[p];
    const int tiles = ((g.nx + A.tile_w - 1) / A.tile_w) * ((g.ny + A.tile_h - 1) / A.tile_h);
    const uint32_t n_src = se - sb;
    // Source chunks: about 16 CTAs per SM, several waves so that uneven chunk times even out. On
    // a 1 km terrain tile (80 k sources) 9 per SM took 834 ms, 16 took 745, 24 took 747 and 48
    // took 740; the road tile is flat from 16 up.
    uint32_t want_ctas = (uint32_t)ctx->sm_count * 16;
    uint32_t n_chunks = std::max<uint32_t>(1, (want_ctas + tiles - 1) / tiles);
    n_chunks = std::min<uint32_t>(n_chunks, std::max<uint32_t>(1, n_src / 32));
    n_chunks = std::min<uint32_t>(n_chunks, 65535);
    A.chunk = std::max<uint32_t>(1, (n_src + n_chunks - 1) / n_chunks);
    A.n_chunks = n_src == 0 ? 1 : (n_src + A.chunk - 1) / A.chunk;
    const uint32_t slices = A.n_chunks + 1;  // the last slice holds the re-run paths
    // The re-run list holds up to 1 path in 16 (at least 1 M, at most 2^27): over-capacity paths are
    // rare, but tiles in dense quarters with kilometre-long rays reach a few per cent.
    A.retry_cap = (uint32_t)std::min<int64_t>(std::max<int64_t>((int64_t)cells * n_src / 16, 1 << 20), 1 << 27);
    qm_scene::GridScratch &G = scene->grid_scratch;
    GrowBuffer &d_alt = G.alt, &d_own = G.own, &d_partial = G.partial, &d_failed = G.failed, &d_counters = G.counters,
               &d_dba = G.dba, &d_hist = G.hist, &d_bands = G.bands, &d_dbaout = G.dbaout, &d_lden = G.lden,
               &d_retry = G.retry, &d_rcount = G.rcount;
    size_t partial_bytes = (size_t)slices * cells * GRID_SLOTS * sizeof(float);
    QM_CUDA(d_alt.reserve(cells * sizeof(float)));
    QM_CUDA(d_own.reserve(cells * sizeof(uint32_t)));
    QM_CUDA(d_partial.reserve(partial_bytes));
    QM_CUDA(d_failed.reserve(cells * sizeof(uint32_t)));
    QM_CUDA(d_counters.reserve(6 * sizeof(unsigned long long)));
    QM_CUDA(d_dba.reserve(cells * sizeof(float)));
    QM_CUDA(d_retry.reserve((size_t)A.retry_cap * sizeof(uint2)));
    QM_CUDA(d_rcount.reserve(sizeof(unsigned int)));
    QM_CUDA(cudaMemcpyAsync(d_alt.p, alt.data(), cells * sizeof(float), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(d_own.p, own.data(), cells * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemsetAsync(d_partial.p, 0, partial_bytes, stream));
    QM_CUDA(cudaMemsetAsync(d_failed.p, 0, cells * sizeof(uint32_t), stream));
    QM_CUDA(cudaMemsetAsync(d_counters.p, 0, 6 * sizeof(unsigned long long), stream));
    QM_CUDA(cudaMemsetAsync(d_rcount.p, 0, sizeof(unsigned int), stream));
    A.rcv_alt = static_cast<float *>(d_alt.p);
    A.rcv_own = static_cast<uint32_t *>(d_own.p);
    A.partial = static_cast<float *>(d_partial.p);
    A.failed = static_cast<uint32_t *>(d_failed.p);
    A.counters = static_cast<unsigned long long *>(d_counters.p);
    A.retry = static_cast<uint2 *>(d_retry.p);
    A.retry_count = static_cast<unsigned int *>(d_rcount.p);
    // The terrain painter's three resident CTAs need 28 KB of shared memory (8.3 KB each plus the
    // 1 KB the device reserves); a 32 KB carveout (14 % of 228 KB) leaves the rest of the SM's
    // 256 KB to L1, which caches the threads' local work areas. Left to itself the driver takes
    // 64 KB.
    if (terrain_caps(scene))
        QM_CUDA(cudaFuncSetAttribute(paint_grid_kernel<CapsTerrain>, cudaFuncAttributePreferredSharedMemoryCarveout, 14));
    else
        QM_CUDA(cudaFuncSetAttribute(paint_grid_kernel<CapsFlat>, cudaFuncAttributePreferredSharedMemoryCarveout, 14));
    Events ev;
    QM_CUDA(ev.create());
    QM_CUDA(cudaEventRecord(ev.e0, stream));
    if (n_src > 0) {
        dim3 grid_dim(tiles, A.n_chunks);
        if (terrain_caps(scene)) {
            paint_grid_kernel<CapsTerrain><<<grid_dim, 128, 0, stream>>>(scene->dev, A);
        } else {
            paint_grid_kernel<CapsFlat><<<grid_dim, 128, 0, stream>>>(scene->dev, A);
        }
        QM_CUDA(cudaGetLastError());
    }
    QM_CUDA(cudaEventRecord(ev.e2, stream));
    unsigned int n_retry = 0;
    QM_CUDA(cudaMemcpyAsync(&n_retry, d_rcount.p, sizeof(n_retry), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaStreamSynchronize(stream));
    if (n_retry > A.retry_cap)
        return fail(QM_ERR_CAPACITY, "qm_paint_grid: " + std::to_string(n_retry) +
                                         " paths exceeded the per-path capacities, more than the retry list holds");
    if (n_retry > 0) {
        qm_status st = rerun_failed(scene, A, static_cast<uint2 *>(d_retry.p), n_retry, A.n_chunks, cells, stream);
        if (st != QM_OK) return st;
    }
    ReduceArgs R{};
    R.cells = cells;
    R.n_chunks = slices;
    R.partial = A.partial;
    R.level_min = g.level_min_db;
    R.bin_db = g.bin_db;
    R.n_bins = histogram ? g.n_bins : 0;
    R.dba_scratch = static_cast<float *>(d_dba.p);
    if (cell_bands) QM_CUDA(d_bands.reserve((size_t)cells * 8 * sizeof(float)));
    if (cell_dba) QM_CUDA(d_dbaout.reserve((size_t)cells * sizeof(float)));
    if (cell_lden) QM_CUDA(d_lden.reserve((size_t)cells * sizeof(float)));
    if (histogram) {
        QM_CUDA(d_hist.reserve(g.n_bins * sizeof(uint32_t)));
        QM_CUDA(cudaMemsetAsync(d_hist.p, 0, g.n_bins * sizeof(uint32_t), stream));
    }
    // Outputs the caller did not ask for stay null (the kept buffers may hold an earlier call's).
    R.cell_bands = cell_bands ? static_cast<float *>(d_bands.p) : nullptr;
    R.cell_dba = cell_dba ? static_cast<float *>(d_dbaout.p) : nullptr;
    R.cell_lden = cell_lden ? static_cast<float *>(d_lden.p) : nullptr;
    R.histogram = histogram ? static_cast<uint32_t *>(d_hist.p) : nullptr;
    size_t smem = histogram ? g.n_bins * sizeof(uint32_t) : 0;
    if (smem > 48 * 1024) QM_CUDA(cudaFuncSetAttribute(reduce_cells_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    reduce_cells_kernel<<<(cells + 255) / 256, 256, smem, stream>>>(R);
    QM_CUDA(cudaGetLastError());
    QM_CUDA(cudaEventRecord(ev.e1, stream));
    unsigned long long counters[6];
    QM_CUDA(cudaMemcpyAsync(counters, d_counters.p, sizeof(counters), cudaMemcpyDeviceToHost, stream));
    if (cell_bands) QM_CUDA(cudaMemcpyAsync(cell_bands, d_bands.p, (size_t)cells * 8 * sizeof(float), cudaMemcpyDeviceToHost, stream));
    if (cell_dba) QM_CUDA(cudaMemcpyAsync(cell_dba, d_dbaout.p, (size_t)cells * sizeof(float), cudaMemcpyDeviceToHost, stream));
    if (cell_lden) QM_CUDA(cudaMemcpyAsync(cell_lden, d_lden.p, (size_t)cells * sizeof(float), cudaMemcpyDeviceToHost, stream));
    if (histogram) QM_CUDA(cudaMemcpyAsync(histogram, d_hist.p, g.n_bins * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaStreamSynchronize(stream));
    float ms = 0.f, paint_ms = 0.f;
    QM_CUDA(cudaEventElapsedTime(&ms, ev.e0, ev.e1));
    QM_CUDA(cudaEventElapsedTime(&paint_ms, ev.e0, ev.e2));
    if (stats) {
        stats->paths = counters[0];
        stats->crossings = counters[1];
        stats->failed_paths = counters[3];
        stats->edge_tests = counters[2];
        stats->vertices = counters[4];
        stats->candidates = counters[5];
        stats->kernel_ms = ms;
        stats->paint_ms = paint_ms;
    }
    return QM_OK;
}

qm_status qm_scene_line_pieces(qm_scene *scene, const qm_line_source *pieces, size_t n_pieces) {
    NvtxRange nvtx_range("qm_scene_line_pieces");
    if (!scene) return fail(QM_ERR_ARGUMENT, "qm_scene_line_pieces: null scene");
    if (n_pieces && !pieces) return fail(QM_ERR_ARGUMENT, "qm_scene_line_pieces: null pieces");
    if ((uint64_t)scene->n_sources + n_pieces > 0xFFFFFFFFull)
        return fail(QM_ERR_ARGUMENT, "qm_scene_line_pieces: too many candidates");
    std::vector<PieceDev> dev(n_pieces);
    std::vector<uint32_t> layers(n_pieces);
    for (size_t k = 0; k < n_pieces; ++k) {
        const qm_line_source &p = pieces[k];
        for (int e = 0; e < 2; ++e)
            if (!std::isfinite(p.a[e]) || !std::isfinite(p.b[e]) || p.a[e] < 0.0 || p.b[e] < 0.0 ||
                p.a[e] >= scene->extent[e] || p.b[e] >= scene->extent[e])
                return fail(QM_ERR_ARGUMENT, "qm_scene_line_pieces: piece " + std::to_string(k) +
                                                 " has an end outside the scene extent");
        if (p.source.layer >= QM_LAYERS)
            return fail(QM_ERR_ARGUMENT, "qm_scene_line_pieces: piece " + std::to_string(k) + " names layer " +
                                             std::to_string(p.source.layer));
        PieceDev &d = dev[k];
        d.ax = p.a[0];
        d.ay = p.a[1];
        d.bx = p.b[0];
        d.by = p.b[1];
        d.src.x = (int32_t)std::llround(p.a[0]);
        d.src.y = (int32_t)std::llround(p.a[1]);
        d.src.height = p.source.height_m;
        d.src.gf = p.source.ground_factor;
        d.src.excl = p.source.exclusion_radius_m;
        d.src.platform = p.source.platform_half_width_m;
        d.src.fp = dense_fp(scene, p.source.footprint_id);
        d.src.layer = p.source.layer;
        for (int q = 0; q < 3; ++q)
            for (int b = 0; b < 8; ++b) d.src.energy[q * 8 + b] = p.source.energy[q][b];
        layers[k] = p.source.layer;
    }
    // The receivers' skyline index of the scene's outlines, built on the host and copied as is.
    qm_skyline *sky = nullptr;
    qm_status st = qm_skyline_build(scene->vertices.data(), scene->vertices.size() / 2, scene->outlines.data(),
                                    scene->outlines.size(), scene->step_m, &sky);
    if (st != QM_OK) return fail(st, std::string("qm_scene_line_pieces: ") + qm::last_error());
    const qm::skyline::Index host = qm::skyline_view(sky);
    std::lock_guard<std::mutex> guard(scene->ctx->lock);
    QM_CUDA(cudaSetDevice(scene->ctx->device));
    for (auto *b : scene->piece_buffers) delete b;
    scene->piece_buffers.clear();
    scene->n_pieces = 0;
    auto put = [&](const void *data, size_t bytes, const void **out) -> qm_status {
        auto *b = new DeviceBuffer();
        scene->piece_buffers.push_back(b);
        b->bytes = std::max<size_t>(bytes, 16);
        QM_CUDA(cudaMalloc(&b->ptr, b->bytes));
        if (bytes) QM_CUDA(cudaMemcpy(b->ptr, data, bytes, cudaMemcpyHostToDevice));
        *out = b->ptr;
        return QM_OK;
    };
    const size_t n_cells = host.n_cells, n_runs = n_cells ? host.run_start[n_cells] : 0;
    qm::skyline::Index d = host;
    const void *p_keys, *p_start, *p_tall, *p_runs, *p_outl, *p_pieces;
    std::vector<uint32_t> start_copy(n_cells + 1, 0u);
    if (n_cells) std::copy(host.run_start, host.run_start + n_cells + 1, start_copy.begin());
    if ((st = put(host.keys, n_cells * sizeof(uint64_t), &p_keys)) != QM_OK ||
        (st = put(start_copy.data(), start_copy.size() * sizeof(uint32_t), &p_start)) != QM_OK ||
        (st = put(host.tallest, n_cells * sizeof(float), &p_tall)) != QM_OK ||
        (st = put(host.runs, n_runs * sizeof(qm::skyline::Run), &p_runs)) != QM_OK ||
        (st = put(scene->outlines.data(), scene->outlines.size() * sizeof(qm_outline), &p_outl)) != QM_OK ||
        (st = put(dev.data(), dev.size() * sizeof(PieceDev), &p_pieces)) != QM_OK) {
        qm_skyline_free(sky);
        return st;
    }
    qm_skyline_free(sky);
    d.keys = static_cast<const uint64_t *>(p_keys);
    d.run_start = static_cast<const uint32_t *>(p_start);
    d.tallest = static_cast<const float *>(p_tall);
    d.runs = static_cast<const qm::skyline::Run *>(p_runs);
    d.outlines = static_cast<const qm_outline *>(p_outl);
    d.vertices = reinterpret_cast<const int32_t *>(scene->dev.vertices);
    scene->sky = d;
    scene->pieces = static_cast<const PieceDev *>(p_pieces);
    scene->piece_layer = layers;
    scene->n_pieces = (uint32_t)n_pieces;
    return QM_OK;
}

qm_status qm_evaluate_pairs(qm_scene *scene, const double *receiver_xy, const float *receiver_height_m,
                            const uint64_t *own_footprint, const uint32_t *point_of_receiver, size_t n_receivers,
                            const uint32_t *source_of_pair, const uint32_t *receiver_of_pair, const float *band_weight,
                            size_t n_pairs, float *pair_sums, float *pair_bands, uint32_t *pair_status,
                            float *point_bands, size_t n_points) {
    NvtxRange nvtx_range("qm_evaluate_pairs");
    if (!scene) return fail(QM_ERR_ARGUMENT, "qm_evaluate_pairs: null scene");
    if (n_pairs && (!source_of_pair || !receiver_of_pair || !pair_sums || !pair_status))
        return fail(QM_ERR_ARGUMENT, "qm_evaluate_pairs: a source and receiver per pair, sums and status outputs");
    if (n_receivers && (!receiver_xy || !receiver_height_m || !own_footprint || !point_of_receiver))
        return fail(QM_ERR_ARGUMENT, "qm_evaluate_pairs: an owner, height and point a receiver");
    if (n_pairs && !point_bands) return fail(QM_ERR_ARGUMENT, "qm_evaluate_pairs: point_bands is null");
    std::vector<int2> rxy(n_receivers);
    std::vector<float> ralt(n_receivers);
    std::vector<uint32_t> rown(n_receivers);
    for (size_t r = 0; r < n_receivers; ++r) {
        double x = receiver_xy[2 * r] / scene->step_m, y = receiver_xy[2 * r + 1] / scene->step_m;
        if (!std::isfinite(x) || !std::isfinite(y) || x < 0 || y < 0 || x >= scene->extent[0] || y >= scene->extent[1])
            return fail(QM_ERR_ARGUMENT, "qm_evaluate_pairs: receiver " + std::to_string(r) + " outside the scene extent");
        if (point_of_receiver[r] >= n_points)
            return fail(QM_ERR_ARGUMENT, "qm_evaluate_pairs: a point outside the bands");
        rxy[r] = make_int2((int)std::llround(x), (int)std::llround(y));
        ralt[r] = (float)(terrain_altitude(scene, rxy[r].x, rxy[r].y) + receiver_height_m[r]);
        rown[r] = dense_fp(scene, own_footprint[r]);
    }
    for (size_t i = 0; i < n_pairs; ++i)
        if ((uint64_t)source_of_pair[i] >= (uint64_t)scene->n_sources + scene->n_pieces || receiver_of_pair[i] >= n_receivers)
            return fail(QM_ERR_ARGUMENT,
                        "qm_evaluate_pairs: a candidate outside the square, a receiver outside the receivers");
    if (n_pairs == 0) return QM_OK;
    qm_ctx *ctx = scene->ctx;
    std::lock_guard<std::mutex> guard(ctx->lock);
    QM_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t stream = ctx->stream;
    // Pairs grouped by point, stable (the order point bands are summed in).
    std::vector<uint32_t> order(n_pairs), layer(n_pairs);
    for (size_t i = 0; i < n_pairs; ++i) {
        order[i] = (uint32_t)i;
        const uint32_t c = source_of_pair[i];
        layer[i] = c < scene->n_sources ? scene->source_layer[c] : scene->piece_layer[c - scene->n_sources];
    }
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
        return point_of_receiver[receiver_of_pair[a]] < point_of_receiver[receiver_of_pair[b]];
    });
    std::vector<uint32_t> group_start, group_point;
    for (size_t k = 0; k < n_pairs; ++k) {
        uint32_t pt = point_of_receiver[receiver_of_pair[order[k]]];
        if (group_point.empty() || group_point.back() != pt) {
            group_start.push_back((uint32_t)k);
            group_point.push_back(pt);
        }
    }
    group_start.push_back((uint32_t)n_pairs);
    Scratch d_rxy, d_ralt, d_rown, d_sop, d_rop, d_sums, d_bands, d_status, d_order, d_gs, d_gp, d_w, d_layer, d_points;
    QM_CUDA(cudaMalloc(&d_rxy.p, n_receivers * sizeof(int2)));
    QM_CUDA(cudaMalloc(&d_ralt.p, n_receivers * sizeof(float)));
    QM_CUDA(cudaMalloc(&d_rown.p, n_receivers * sizeof(uint32_t)));
    QM_CUDA(cudaMalloc(&d_sop.p, n_pairs * sizeof(uint32_t)));
    QM_CUDA(cudaMalloc(&d_rop.p, n_pairs * sizeof(uint32_t)));
    QM_CUDA(cudaMalloc(&d_sums.p, n_pairs * 9 * sizeof(float)));
    QM_CUDA(cudaMalloc(&d_bands.p, n_pairs * 24 * sizeof(float)));
    QM_CUDA(cudaMalloc(&d_status.p, n_pairs * sizeof(uint32_t)));
    QM_CUDA(cudaMalloc(&d_order.p, n_pairs * sizeof(uint32_t)));
    QM_CUDA(cudaMalloc(&d_gs.p, group_start.size() * sizeof(uint32_t)));
    QM_CUDA(cudaMalloc(&d_gp.p, group_point.size() * sizeof(uint32_t)));
    QM_CUDA(cudaMalloc(&d_layer.p, n_pairs * sizeof(uint32_t)));
    QM_CUDA(cudaMalloc(&d_points.p, n_points * QM_POINT_BANDS * sizeof(float)));
    if (band_weight) QM_CUDA(cudaMalloc(&d_w.p, n_pairs * sizeof(float)));
    QM_CUDA(cudaMemcpyAsync(d_rxy.p, rxy.data(), n_receivers * sizeof(int2), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(d_ralt.p, ralt.data(), n_receivers * sizeof(float), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(d_rown.p, rown.data(), n_receivers * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(d_sop.p, source_of_pair, n_pairs * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(d_rop.p, receiver_of_pair, n_pairs * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(d_order.p, order.data(), n_pairs * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(d_gs.p, group_start.data(), group_start.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(d_gp.p, group_point.data(), group_point.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(d_layer.p, layer.data(), n_pairs * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(d_points.p, point_bands, n_points * QM_POINT_BANDS * sizeof(float), cudaMemcpyHostToDevice, stream));
    if (band_weight) QM_CUDA(cudaMemcpyAsync(d_w.p, band_weight, n_pairs * sizeof(float), cudaMemcpyHostToDevice, stream));
    PairArgs A{};
    A.rcv_xy = static_cast<int2 *>(d_rxy.p);
    A.rcv_alt = static_cast<float *>(d_ralt.p);
    A.rcv_own = static_cast<uint32_t *>(d_rown.p);
    A.source_of_pair = static_cast<uint32_t *>(d_sop.p);
    A.receiver_of_pair = static_cast<uint32_t *>(d_rop.p);
    A.n_pairs = n_pairs;
    A.pair_sums = static_cast<float *>(d_sums.p);
    A.pair_bands = static_cast<float *>(d_bands.p);
    A.status = static_cast<uint32_t *>(d_status.p);
    unsigned blocks = (unsigned)((n_pairs + 127) / 128);
    if (terrain_caps(scene))
        evaluate_pairs_kernel<CapsTerrain><<<blocks, 128, 0, stream>>>(scene->dev, A);
    else
        evaluate_pairs_kernel<CapsFlat><<<blocks, 128, 0, stream>>>(scene->dev, A);
    QM_CUDA(cudaGetLastError());
    // Line pieces: one thread a (receiver, piece) pair over the piece's quadrature nodes.
    std::vector<uint32_t> line_pairs;
    for (size_t i = 0; i < n_pairs; ++i)
        if (source_of_pair[i] >= scene->n_sources) line_pairs.push_back((uint32_t)i);
    Scratch d_lines;
    LinePairArgs LA{};
    LA.pieces = scene->pieces;
    LA.sky = scene->sky;
    if (!line_pairs.empty()) {
        QM_CUDA(cudaMalloc(&d_lines.p, line_pairs.size() * sizeof(uint32_t)));
        QM_CUDA(cudaMemcpyAsync(d_lines.p, line_pairs.data(), line_pairs.size() * sizeof(uint32_t),
                                cudaMemcpyHostToDevice, stream));
        LA.line_pairs = static_cast<uint32_t *>(d_lines.p);
        LA.n_line_pairs = (uint32_t)line_pairs.size();
        const unsigned line_blocks = (unsigned)((line_pairs.size() + 127) / 128);
        if (terrain_caps(scene))
            evaluate_line_pairs_kernel<CapsTerrain><<<line_blocks, 128, 0, stream>>>(scene->dev, A, LA);
        else
            evaluate_line_pairs_kernel<CapsFlat><<<line_blocks, 128, 0, stream>>>(scene->dev, A, LA);
        QM_CUDA(cudaGetLastError());
    }
    // Pairs over the per-path capacities again with large ones (global scratch work areas).
    std::vector<uint32_t> status_host(n_pairs);
    QM_CUDA(cudaMemcpyAsync(status_host.data(), d_status.p, n_pairs * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaStreamSynchronize(stream));
    std::vector<uint32_t> again, again_lines;
    for (size_t i = 0; i < n_pairs; ++i)
        if (status_host[i] & QM_FAILED_CAPACITY)
            (source_of_pair[i] < scene->n_sources ? again : again_lines).push_back((uint32_t)i);
    Scratch d_again, d_works, d_again_lines, d_line_works;
    if (!again_lines.empty()) {
        using Large = PathWork<CapsLarge::C, CapsLarge::K, CapsLarge::H>;
        const uint32_t threads = std::min<uint32_t>(((uint32_t)again_lines.size() + 63) / 64 * 64, 4096);
        QM_CUDA(cudaMalloc(&d_again_lines.p, again_lines.size() * sizeof(uint32_t)));
        QM_CUDA(cudaMalloc(&d_line_works.p, (size_t)threads * sizeof(Large)));
        QM_CUDA(cudaMemcpyAsync(d_again_lines.p, again_lines.data(), again_lines.size() * sizeof(uint32_t),
                                cudaMemcpyHostToDevice, stream));
        retry_line_pairs_kernel<<<threads / 64, 64, 0, stream>>>(scene->dev, A, LA, static_cast<uint32_t *>(d_again_lines.p),
                                                                 (uint32_t)again_lines.size(),
                                                                 static_cast<Large *>(d_line_works.p));
        QM_CUDA(cudaGetLastError());
    }
    if (!again.empty()) {
        using Large = PathWork<CapsLarge::C, CapsLarge::K, CapsLarge::H>;
        const uint32_t threads = std::min<uint32_t>(((uint32_t)again.size() + 63) / 64 * 64, 8192);
        QM_CUDA(cudaMalloc(&d_again.p, again.size() * sizeof(uint32_t)));
        QM_CUDA(cudaMalloc(&d_works.p, (size_t)threads * sizeof(Large)));
        QM_CUDA(cudaMemcpyAsync(d_again.p, again.data(), again.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        retry_pairs_kernel<<<threads / 64, 64, 0, stream>>>(scene->dev, A, static_cast<uint32_t *>(d_again.p),
                                                            (uint32_t)again.size(), static_cast<Large *>(d_works.p));
        QM_CUDA(cudaGetLastError());
    }
    point_bands_kernel<<<(unsigned)group_point.size(), 160, 0, stream>>>(
        static_cast<uint32_t *>(d_order.p), static_cast<uint32_t *>(d_gs.p), static_cast<uint32_t *>(d_gp.p),
        (uint32_t)group_point.size(), A.pair_bands, static_cast<float *>(d_w.p), static_cast<uint32_t *>(d_layer.p),
        static_cast<float *>(d_points.p));
    QM_CUDA(cudaGetLastError());
    QM_CUDA(cudaMemcpyAsync(pair_sums, d_sums.p, n_pairs * 9 * sizeof(float), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaMemcpyAsync(pair_status, d_status.p, n_pairs * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    if (pair_bands) QM_CUDA(cudaMemcpyAsync(pair_bands, d_bands.p, n_pairs * 24 * sizeof(float), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaMemcpyAsync(point_bands, d_points.p, n_points * QM_POINT_BANDS * sizeof(float), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaStreamSynchronize(stream));
    return QM_OK;
}

qm_status qm_zwicker(qm_ctx *ctx, const float *thirds_db, size_t n, float *sone) {
    NvtxRange nvtx_range("qm_zwicker");
    if (!ctx) return fail(QM_ERR_ARGUMENT, "qm_zwicker: null ctx");
    if (n && (!thirds_db || !sone)) return fail(QM_ERR_ARGUMENT, "qm_zwicker: null thirds_db or sone");
    if (n == 0) return QM_OK;
    std::lock_guard<std::mutex> guard(ctx->lock);
    QM_CUDA(cudaSetDevice(ctx->device));
    Scratch d_in, d_out;
    QM_CUDA(cudaMalloc(&d_in.p, n * 28 * sizeof(float)));
    QM_CUDA(cudaMalloc(&d_out.p, n * sizeof(float)));
    QM_CUDA(cudaMemcpyAsync(d_in.p, thirds_db, n * 28 * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    launch_zwicker(static_cast<float *>(d_in.p), n, static_cast<float *>(d_out.p), ctx->stream);
    QM_CUDA(cudaGetLastError());
    QM_CUDA(cudaMemcpyAsync(sone, d_out.p, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    QM_CUDA(cudaStreamSynchronize(ctx->stream));
    return QM_OK;
}

qm_status qm_level_histogram(qm_ctx *ctx, const float *levels_db, size_t n, double level_min_db, double bin_db,
                             uint32_t n_bins, uint32_t *counts) {
    if (!ctx) return fail(QM_ERR_ARGUMENT, "qm_level_histogram: null ctx");
    if (!counts || n_bins == 0 || n_bins > 51200 || !(bin_db > 0.0))
        return fail(QM_ERR_ARGUMENT, "qm_level_histogram: counts, n_bins (1..51200) or bin_db");
    if (n && !levels_db) return fail(QM_ERR_ARGUMENT, "qm_level_histogram: levels_db is null");
    std::lock_guard<std::mutex> guard(ctx->lock);
    QM_CUDA(cudaSetDevice(ctx->device));
    Scratch d_in, d_out;
    QM_CUDA(cudaMalloc(&d_out.p, n_bins * sizeof(uint32_t)));
    QM_CUDA(cudaMemsetAsync(d_out.p, 0, n_bins * sizeof(uint32_t), ctx->stream));
    if (n) {
        QM_CUDA(cudaMalloc(&d_in.p, n * sizeof(float)));
        QM_CUDA(cudaMemcpyAsync(d_in.p, levels_db, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
        size_t smem = n_bins * sizeof(uint32_t);
        if (smem > 48 * 1024)
            QM_CUDA(cudaFuncSetAttribute(histogram_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)ctx->sm_count * 8);
        histogram_kernel<<<blocks, 256, smem, ctx->stream>>>(static_cast<float *>(d_in.p), n, level_min_db, bin_db,
                                                             n_bins, static_cast<uint32_t *>(d_out.p));
        QM_CUDA(cudaGetLastError());
    }
    QM_CUDA(cudaMemcpyAsync(counts, d_out.p, n_bins * sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
    QM_CUDA(cudaStreamSynchronize(ctx->stream));
    return QM_OK;
}

qm_status qm_quantize_cells(qm_ctx *ctx, const double *lden_energy, const double *sone, const uint8_t *assessed,
                            size_t n, uint8_t *lden_cells, uint8_t *nden_cells) {
    NvtxRange nvtx_range("qm_quantize_cells");
    if (!ctx) return fail(QM_ERR_ARGUMENT, "qm_quantize_cells: null ctx");
    if ((sone == nullptr) != (nden_cells == nullptr))
        return fail(QM_ERR_ARGUMENT, "qm_quantize_cells: sone and nden_cells are given together or not at all");
    if (n == 0) return QM_OK;
    if (!lden_energy || !lden_cells) return fail(QM_ERR_ARGUMENT, "qm_quantize_cells: null lden_energy or lden_cells");
    if (n > (size_t(1) << 40)) return fail(QM_ERR_ARGUMENT, "qm_quantize_cells: more than 2^40 pixels");
    constexpr size_t W = QM_LAYERS + 1;
    std::lock_guard<std::mutex> guard(ctx->lock);
    QM_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t stream = ctx->stream;
    Scratch d_energy, d_sone, d_assessed, d_lc, d_nc, d_bad;
    QM_CUDA(cudaMalloc(&d_energy.p, n * QM_LAYERS * sizeof(double)));
    QM_CUDA(cudaMalloc(&d_lc.p, n * W));
    QM_CUDA(cudaMalloc(&d_bad.p, sizeof(unsigned long long)));
    QM_CUDA(cudaMemcpyAsync(d_energy.p, lden_energy, n * QM_LAYERS * sizeof(double), cudaMemcpyHostToDevice, stream));
    if (sone) {
        QM_CUDA(cudaMalloc(&d_sone.p, n * W * sizeof(double)));
        QM_CUDA(cudaMalloc(&d_nc.p, n * W));
        QM_CUDA(cudaMemcpyAsync(d_sone.p, sone, n * W * sizeof(double), cudaMemcpyHostToDevice, stream));
    }
    if (assessed) {
        QM_CUDA(cudaMalloc(&d_assessed.p, n));
        QM_CUDA(cudaMemcpyAsync(d_assessed.p, assessed, n, cudaMemcpyHostToDevice, stream));
    }
    QM_CUDA(cudaMemsetAsync(d_bad.p, 0xff, sizeof(unsigned long long), stream));
    const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)ctx->sm_count * 16);
    quantize_cells_kernel<<<blocks, 256, 0, stream>>>(
        static_cast<const double *>(d_energy.p), static_cast<const double *>(d_sone.p),
        static_cast<const uint8_t *>(d_assessed.p), n, static_cast<uint8_t *>(d_lc.p), static_cast<uint8_t *>(d_nc.p),
        static_cast<unsigned long long *>(d_bad.p));
    QM_CUDA(cudaGetLastError());
    unsigned long long bad = 0;
    QM_CUDA(cudaMemcpyAsync(&bad, d_bad.p, sizeof(bad), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaStreamSynchronize(stream));
    if (bad != ~0ull) {
        // The reference's message (levels.rs:100-111), with the offending value from the input.
        const size_t pixel = (size_t)(bad / 8);
        const int layer = (int)(bad % 8);
        double value = 0.0;
        if (layer < QM_LAYERS) {
            value = lden_energy[pixel * QM_LAYERS + layer];
        } else {
            for (int l = 0; l < QM_LAYERS; ++l) value += lden_energy[pixel * QM_LAYERS + l];
        }
        char text[64];
        if (std::isnan(value))
            std::snprintf(text, sizeof text, "NaN");
        else if (std::isinf(value))
            std::snprintf(text, sizeof text, value > 0 ? "inf" : "-inf");
        else
            std::snprintf(text, sizeof text, "%.17g", value);
        const std::string where = layer < QM_LAYERS ? "layer " + std::to_string(layer) : std::string("total");
        return fail(QM_ERR_ARGUMENT, "qm_quantize_cells: pixel " + std::to_string(pixel) + ", " + where +
                                         ": invalid Lden energy " + text);
    }
    QM_CUDA(cudaMemcpyAsync(lden_cells, d_lc.p, n * W, cudaMemcpyDeviceToHost, stream));
    if (sone) QM_CUDA(cudaMemcpyAsync(nden_cells, d_nc.p, n * W, cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaStreamSynchronize(stream));
    return QM_OK;
}

qm_status qm_hm3_unpredict(const uint8_t *stream, size_t n_bytes, uint32_t layer, int metric, uint8_t *cells) {
    if (layer > QM_LAYERS) return fail(QM_ERR_ARGUMENT, "unknown HM3 layer");
    if (metric != 0 && metric != 1) return fail(QM_ERR_ARGUMENT, "qm_hm3_unpredict: metric is 0 (loudness) or 1 (Lden)");
    if (!cells) return fail(QM_ERR_ARGUMENT, "qm_hm3_unpredict: null cells");
    const uint8_t header[2][5] = {{'H', 'M', '3', ' ', 0x07}, {'H', 'M', 'D', ' ', 0x01}};
    if (!stream || n_bytes != (size_t)QM_HM3_STREAM_BYTES || std::memcmp(stream, header[metric], 5) != 0 ||
        stream[5] != layer)
        return fail(QM_ERR_ARGUMENT, "not this layer's HM3 tile");
    // In order, each cell is its residual plus the Paeth prediction from the cells already restored
    // (hm3.rs:165-167): left, above, upper-left, zeros outside the tile, ties to left then above.
    constexpr size_t P = QM_HM3_TILE_PX;
    for (size_t at = 0; at < P * P; ++at) {
        const bool has_left = at % P != 0, has_above = at >= P;
        const int left = has_left ? cells[at - 1] : 0, above = has_above ? cells[at - P] : 0;
        const int corner = has_left && has_above ? cells[at - P - 1] : 0;
        const int estimate = left + above - corner;
        const int dl = std::abs(estimate - left), da = std::abs(estimate - above), dc = std::abs(estimate - corner);
        const int predicted = (dl <= da && dl <= dc) ? left : (da <= dc ? above : corner);
        cells[at] = (uint8_t)(stream[6 + at] + predicted);
    }
    return QM_OK;
}

qm_status qm_hm3_predict(qm_ctx *ctx, const uint8_t *cells, const uint8_t *layers, size_t n_tiles, int metric,
                         uint8_t *streams) {
    NvtxRange nvtx_range("qm_hm3_predict");
    if (!ctx) return fail(QM_ERR_ARGUMENT, "qm_hm3_predict: null ctx");
    if (metric != 0 && metric != 1) return fail(QM_ERR_ARGUMENT, "qm_hm3_predict: metric is 0 (loudness) or 1 (Lden)");
    if (n_tiles == 0) return QM_OK;
    if (!cells || !layers || !streams) return fail(QM_ERR_ARGUMENT, "qm_hm3_predict: null cells, layers or streams");
    if (n_tiles > (size_t(1) << 16)) return fail(QM_ERR_ARGUMENT, "qm_hm3_predict: more than 65,536 tiles in one call");
    for (size_t t = 0; t < n_tiles; ++t)
        if (layers[t] > QM_LAYERS)
            return fail(QM_ERR_ARGUMENT, "qm_hm3_predict: tile " + std::to_string(t) + ": unknown layer " +
                                             std::to_string(layers[t]));
    constexpr size_t PIX = (size_t)QM_HM3_TILE_PX * QM_HM3_TILE_PX;
    // "HM3 \x07" (loudness) or "HMD \x01" (Lden): the first four bytes little-endian, then the fifth.
    const uint8_t header[2][5] = {{'H', 'M', '3', ' ', 0x07}, {'H', 'M', 'D', ' ', 0x01}};
    const uint8_t *h = header[metric];
    const uint32_t word = (uint32_t)h[0] | ((uint32_t)h[1] << 8) | ((uint32_t)h[2] << 16) | ((uint32_t)h[3] << 24);
    std::lock_guard<std::mutex> guard(ctx->lock);
    QM_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t stream = ctx->stream;
    Scratch d_cells, d_layers, d_streams;
    QM_CUDA(cudaMalloc(&d_cells.p, n_tiles * PIX));
    QM_CUDA(cudaMalloc(&d_layers.p, n_tiles));
    QM_CUDA(cudaMalloc(&d_streams.p, n_tiles * (size_t)QM_HM3_STREAM_BYTES));
    QM_CUDA(cudaMemcpyAsync(d_cells.p, cells, n_tiles * PIX, cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(d_layers.p, layers, n_tiles, cudaMemcpyHostToDevice, stream));
    const unsigned blocks = (unsigned)std::min<size_t>((n_tiles * PIX + 255) / 256, (size_t)ctx->sm_count * 16);
    hm3_predict_kernel<<<blocks, 256, 0, stream>>>(static_cast<const uint8_t *>(d_cells.p),
                                                   static_cast<const uint8_t *>(d_layers.p), n_tiles, word, h[4],
                                                   static_cast<uint8_t *>(d_streams.p));
    QM_CUDA(cudaGetLastError());
    QM_CUDA(cudaMemcpyAsync(streams, d_streams.p, n_tiles * (size_t)QM_HM3_STREAM_BYTES, cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaStreamSynchronize(stream));
    return QM_OK;
}

qm_status qm_list_crossings(qm_scene *scene, const int32_t *from_xy, const int32_t *to_xy, size_t n, uint32_t cap,
                            uint32_t *counts, uint32_t *edges, double *t, uint32_t *flags, uint32_t *status) {
    if (!scene) return fail(QM_ERR_ARGUMENT, "qm_list_crossings: null scene");
    if (n && (!from_xy || !to_xy || !counts || !status)) return fail(QM_ERR_ARGUMENT, "qm_list_crossings: null ray or output");
    if (n && cap && (!edges || !t || !flags)) return fail(QM_ERR_ARGUMENT, "qm_list_crossings: null list output");
    if (cap > 256) return fail(QM_ERR_ARGUMENT, "qm_list_crossings: cap above 256");
    for (size_t i = 0; i < 2 * n; ++i) {
        const int64_t LIM = int64_t(1) << 27;
        if (from_xy[i] < -LIM || from_xy[i] > LIM || to_xy[i] < -LIM || to_xy[i] > LIM)
            return fail(QM_ERR_ARGUMENT, "qm_list_crossings: a ray end beyond 2^27 steps");
    }
    if (n == 0) return QM_OK;
    qm_ctx *ctx = scene->ctx;
    std::lock_guard<std::mutex> guard(ctx->lock);
    QM_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t stream = ctx->stream;
    size_t m = n * (size_t)std::max<uint32_t>(cap, 1);
    Scratch d_from, d_to, d_counts, d_edges, d_t, d_flags, d_status;
    QM_CUDA(cudaMalloc(&d_from.p, n * sizeof(int2)));
    QM_CUDA(cudaMalloc(&d_to.p, n * sizeof(int2)));
    QM_CUDA(cudaMalloc(&d_counts.p, n * sizeof(uint32_t)));
    QM_CUDA(cudaMalloc(&d_status.p, n * sizeof(uint32_t)));
    QM_CUDA(cudaMalloc(&d_edges.p, m * sizeof(uint32_t)));
    QM_CUDA(cudaMalloc(&d_t.p, m * sizeof(double)));
    QM_CUDA(cudaMalloc(&d_flags.p, m * sizeof(uint32_t)));
    QM_CUDA(cudaMemcpyAsync(d_from.p, from_xy, n * sizeof(int2), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(d_to.p, to_xy, n * sizeof(int2), cudaMemcpyHostToDevice, stream));
    list_crossings_kernel<256><<<(unsigned)((n + 127) / 128), 128, 0, stream>>>(
        scene->dev, static_cast<int2 *>(d_from.p), static_cast<int2 *>(d_to.p), n, cap,
        static_cast<uint32_t *>(d_counts.p), static_cast<uint32_t *>(d_edges.p), static_cast<double *>(d_t.p),
        static_cast<uint32_t *>(d_flags.p), static_cast<uint32_t *>(d_status.p));
    QM_CUDA(cudaGetLastError());
    QM_CUDA(cudaMemcpyAsync(counts, d_counts.p, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaMemcpyAsync(status, d_status.p, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    if (cap) {
        QM_CUDA(cudaMemcpyAsync(edges, d_edges.p, m * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        QM_CUDA(cudaMemcpyAsync(t, d_t.p, m * sizeof(double), cudaMemcpyDeviceToHost, stream));
        QM_CUDA(cudaMemcpyAsync(flags, d_flags.p, m * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    }
    QM_CUDA(cudaStreamSynchronize(stream));
    return QM_OK;
}

}  // extern "C"

// =============================================================================================
// The grid painter for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc while they paint: an engine that hands the
// GPU to this library between its own stream-ordered work and owns every device allocation (a
// cudaMalloc there would synchronise the device and stall its other streams), or a host thread that
// is not allowed to allocate once its set-up is over. For them `qm_paint_grid_static` paints a grid
// with every intermediate buffer carved out of one file-scope device array of QM_STATIC_SCRATCH_BYTES,
// which each GPU that loads this library holds until the process exits. Its success path calls no
// cudaMalloc, cudaFree or other allocating routine, on the device or the host; the scene must have
// been uploaded before (qm_scene_upload allocates).

static __device__ __align__(256) unsigned char g_static_scratch[QM_STATIC_SCRATCH_BYTES];

namespace {

// The device address of g_static_scratch per device, taken once with that device current. In host
// code the array's name is only a host-side stand-in, never a device address.
std::mutex g_static_lock;
void *g_static_ptr[64] = {nullptr};

qm_status static_scratch(int device, unsigned char **out) {
    if (device < 0 || device >= 64) return fail(QM_ERR_UNSUPPORTED, "qm_paint_grid_static: device ordinal above 63");
    std::lock_guard<std::mutex> guard(g_static_lock);
    if (!g_static_ptr[device]) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_scratch);
        if (e != cudaSuccess || !ptr)
            return fail(QM_ERR_CUDA, std::string("cuda: cudaGetSymbolAddress of the static scratch: ") +
                                         cudaGetErrorString(e));
        g_static_ptr[device] = ptr;
    }
    *out = static_cast<unsigned char *>(g_static_ptr[device]);
    return QM_OK;
}

// The ground's altitude at a lattice point in double, by the host's `terrain_altitude` rule and
// operation for operation (each product and sum rounded on its own, no contraction), so that a
// receiver set up on the device stands exactly where qm_paint_grid's host set-up puts it.
__device__ double static_terrain_altitude(const SceneDev &S, long long x, long long y) {
    if (S.dem_nx == 0) return (double)S.flat_z;
    double fx = (double)(x - S.dem_ox) / (double)S.dem_sp, fy = (double)(y - S.dem_oy) / (double)S.dem_sp;
    fx = fmin(fmax(fx, 0.0), (double)(S.dem_nx - 1));
    fy = fmin(fmax(fy, 0.0), (double)(S.dem_ny - 1));
    long long i0 = min((long long)floor(fx), (long long)S.dem_nx - 2);
    long long j0 = min((long long)floor(fy), (long long)S.dem_ny - 2);
    double ax = __dsub_rn(fx, (double)i0), ay = __dsub_rn(fy, (double)j0);
    auto node = [&](long long i, long long j) { return (double)S.dem[j * S.dem_nx + i].x; };
    double lo = __dadd_rn(node(i0, j0), __dmul_rn(ax, __dsub_rn(node(i0 + 1, j0), node(i0, j0))));
    double hi = __dadd_rn(node(i0, j0 + 1), __dmul_rn(ax, __dsub_rn(node(i0 + 1, j0 + 1), node(i0, j0 + 1))));
    return __dadd_rn(lo, __dmul_rn(ay, __dsub_rn(hi, lo)));
}

// Receiver altitude (ground + height) of every grid cell, and UINT_MAX as "no building yet".
__global__ void static_receivers_kernel(SceneDev S, int ox, int oy, int spacing, int nx, int ny, float height,
                                        float *alt, uint32_t *own) {
    int cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= nx * ny) return;
    double z = static_terrain_altitude(S, ox + (long long)(cell % nx) * spacing, oy + (long long)(cell / nx) * spacing);
    alt[cell] = (float)__dadd_rn(z, (double)height);
    own[cell] = 0xFFFFFFFFu;
}

// The building each grid receiver stands in: every closed ring tests the receivers in its box
// (exact even-odd rule on lattice integers) and keeps the lowest dense footprint id, which is the
// lowest footprint id (dense ids keep their order).
__global__ void static_own_kernel(SceneDev S, uint32_t n_outlines, int ox, int oy, int spacing, int nx, int ny,
                                  uint32_t *own) {
    uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n_outlines) return;
    OutlineDev ol = S.outlines[o];
    // A ring without a footprint id (dense id 0) names no building, as in the host set-up.
    if (!ol.building || ol.count < 4 || ol.fp == 0) return;
    long long x0 = LLONG_MAX, x1 = LLONG_MIN, y0 = LLONG_MAX, y1 = LLONG_MIN;
    for (uint32_t k = 0; k < ol.count; ++k) {
        int2 v = S.vertices[ol.first + k];
        x0 = min(x0, (long long)v.x);
        x1 = max(x1, (long long)v.x);
        y0 = min(y0, (long long)v.y);
        y1 = max(y1, (long long)v.y);
    }
    long long i_lo = max(0LL, -floor_div64(-(x0 - ox), spacing)), i_hi = min((long long)nx - 1, floor_div64(x1 - ox, spacing));
    long long j_lo = max(0LL, -floor_div64(-(y0 - oy), spacing)), j_hi = min((long long)ny - 1, floor_div64(y1 - oy, spacing));
    for (long long j = j_lo; j <= j_hi; ++j)
        for (long long i = i_lo; i <= i_hi; ++i) {
            long long x = ox + i * spacing, y = oy + j * spacing;
            bool inside = false;
            for (uint32_t k = 0; k + 1 < ol.count; ++k) {
                int2 a = S.vertices[ol.first + k], b = S.vertices[ol.first + k + 1];
                if (((long long)a.y > y) != ((long long)b.y > y)) {
                    long long lhs = (x - a.x) * ((long long)b.y - a.y), rhs = (y - a.y) * ((long long)b.x - a.x);
                    if (b.y - a.y > 0 ? lhs < rhs : lhs > rhs) inside = !inside;
                }
            }
            if (inside) atomicMin(own + j * nx + i, ol.fp);
        }
}

__global__ void static_own_finish_kernel(uint32_t *own, int cells) {
    int cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell < cells && own[cell] == 0xFFFFFFFFu) own[cell] = 0;
}

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// Loads every kernel the static painter launches, once per device, with that device current. Under
// CUDA's lazy module loading a kernel's first launch would otherwise load its code then, which can
// allocate device memory inside the caller's first paint; loading them here, in the first call's
// set-up beside the array's address, keeps every later launch free of it.
bool g_static_loaded[64] = {false};
qm_status static_load_kernels(int device) {
    std::lock_guard<std::mutex> guard(g_static_lock);
    if (g_static_loaded[device]) return QM_OK;
    cudaFuncAttributes attr;
    const void *kernels[] = {
        reinterpret_cast<const void *>(&static_receivers_kernel),
        reinterpret_cast<const void *>(&static_own_kernel),
        reinterpret_cast<const void *>(&static_own_finish_kernel),
        reinterpret_cast<const void *>(&paint_grid_kernel<CapsTerrain>),
        reinterpret_cast<const void *>(&paint_grid_kernel<CapsFlat>),
        reinterpret_cast<const void *>(&reduce_cells_kernel),
    };
    for (const void *k : kernels) {
        cudaError_t e = cudaFuncGetAttributes(&attr, k);
        if (e != cudaSuccess)
            return fail(QM_ERR_CUDA, std::string("cuda: loading the static painter's kernels: ") + cudaGetErrorString(e));
    }
    g_static_loaded[device] = true;
    return QM_OK;
}

}  // namespace

extern "C" {

qm_status qm_paint_grid_static(qm_scene *scene, const qm_grid_desc *grid, float *cell_bands, float *cell_dba,
                               float *cell_lden, uint32_t *histogram, qm_paint_stats *stats) {
    NvtxRange nvtx_range("qm_paint_grid_static");
    if (!scene || !grid) return fail(QM_ERR_ARGUMENT, "qm_paint_grid_static: null scene or grid");
    const qm_grid_desc &g = *grid;
    if (g.nx <= 0 || g.ny <= 0 || g.spacing <= 0)
        return fail(QM_ERR_ARGUMENT, "qm_paint_grid_static: grid nx, ny or spacing");
    if ((int64_t)g.nx * g.ny > QM_STATIC_MAX_CELLS)
        return fail(QM_ERR_CAPACITY, "qm_paint_grid_static: more than 65536 cells do not fit the static scratch");
    int64_t last_x = g.origin[0] + (int64_t)(g.nx - 1) * g.spacing, last_y = g.origin[1] + (int64_t)(g.ny - 1) * g.spacing;
    if (g.origin[0] < 0 || g.origin[1] < 0 || last_x >= scene->extent[0] || last_y >= scene->extent[1])
        return fail(QM_ERR_ARGUMENT, "qm_paint_grid_static: grid receivers outside the scene extent");
    if (histogram && (g.n_bins == 0 || g.n_bins > QM_STATIC_MAX_BINS || !(g.bin_db > 0.0)))
        return fail(QM_ERR_ARGUMENT, "qm_paint_grid_static: histogram needs 0 < n_bins <= 4096 and bin_db > 0");
    if (!cell_bands || !cell_dba || !cell_lden)
        return fail(QM_ERR_ARGUMENT, "qm_paint_grid_static: cell_bands, cell_dba and cell_lden are required");
    uint32_t sb = g.source_begin, se = g.source_end;
    if (se <= sb) {
        sb = 0;
        se = scene->n_sources;
    }
    if (se > scene->n_sources) return fail(QM_ERR_ARGUMENT, "qm_paint_grid_static: source range beyond the scene's sources");
    qm_ctx *ctx = scene->ctx;
    std::lock_guard<std::mutex> guard(ctx->lock);
    QM_CUDA(cudaSetDevice(ctx->device));
    unsigned char *base = nullptr;
    qm_status st = static_scratch(ctx->device, &base);
    if (st != QM_OK) return st;
    st = static_load_kernels(ctx->device);
    if (st != QM_OK) return st;
    cudaStream_t stream = ctx->stream;
    const int cells = g.nx * g.ny;
    const uint32_t n_src = se - sb;
    // Fixed part of the scratch, then as many partial slices as fit (at most one per 16 CTAs a SM).
    size_t off = 0;
    auto carve = [&](size_t bytes) {
        size_t at = off;
        off = align256(off + bytes);
        return base + at;
    };
    float *d_alt = reinterpret_cast<float *>(carve((size_t)cells * 4));
    uint32_t *d_own = reinterpret_cast<uint32_t *>(carve((size_t)cells * 4));
    uint32_t *d_failed = reinterpret_cast<uint32_t *>(carve((size_t)cells * 4));
    float *d_dba = reinterpret_cast<float *>(carve((size_t)cells * 4));
    float *d_bands = reinterpret_cast<float *>(carve((size_t)cells * 32));
    float *d_dbaout = reinterpret_cast<float *>(carve((size_t)cells * 4));
    float *d_lden = reinterpret_cast<float *>(carve((size_t)cells * 4));
    uint32_t *d_hist = reinterpret_cast<uint32_t *>(carve((size_t)QM_STATIC_MAX_BINS * 4));
    unsigned long long *d_counters = reinterpret_cast<unsigned long long *>(carve(6 * 8));
    unsigned int *d_rcount = reinterpret_cast<unsigned int *>(carve(4));
    uint2 *d_retry = reinterpret_cast<uint2 *>(carve(256 * sizeof(uint2)));
    const size_t slice_bytes = (size_t)cells * GRID_SLOTS * sizeof(float);
    if (off + 2 * slice_bytes > (size_t)QM_STATIC_SCRATCH_BYTES)
        return fail(QM_ERR_CAPACITY, "qm_paint_grid_static: the grid does not fit the static scratch");
    GridArgs A{};
    A.origin_x = g.origin[0];
    A.origin_y = g.origin[1];
    A.spacing = g.spacing;
    A.nx = g.nx;
    A.ny = g.ny;
    A.height_m = g.height_m;
    A.source_begin = sb;
    A.source_end = se;
    A.tile_w = 16;
    A.tile_h = 8;
    A.want_fav = scene->any_favourable;
    for (int p = 0; p < 3; ++p) A.lden_w[p] = (float)LDEN_W[p];
    const int tiles = ((g.nx + A.tile_w - 1) / A.tile_w) * ((g.ny + A.tile_h - 1) / A.tile_h);
    const uint32_t fit_chunks = (uint32_t)((QM_STATIC_SCRATCH_BYTES - off) / slice_bytes) - 1;
    uint32_t n_chunks = std::max<uint32_t>(1, ((uint32_t)ctx->sm_count * 16 + tiles - 1) / tiles);
    n_chunks = std::min<uint32_t>(n_chunks, std::max<uint32_t>(1, n_src / 32));
    n_chunks = std::min<uint32_t>(n_chunks, fit_chunks);
    A.chunk = std::max<uint32_t>(1, (n_src + n_chunks - 1) / n_chunks);
    A.n_chunks = n_src == 0 ? 1 : (n_src + A.chunk - 1) / A.chunk;
    const uint32_t slices = A.n_chunks + 1;
    float *d_partial = reinterpret_cast<float *>(carve((size_t)slices * slice_bytes));
    // The array keeps the last call's contents: clear what must start at zero.
    QM_CUDA(cudaMemsetAsync(d_partial, 0, (size_t)slices * slice_bytes, stream));
    QM_CUDA(cudaMemsetAsync(d_failed, 0, (size_t)cells * 4, stream));
    QM_CUDA(cudaMemsetAsync(d_counters, 0, 6 * 8, stream));
    QM_CUDA(cudaMemsetAsync(d_rcount, 0, 4, stream));
    QM_CUDA(cudaMemsetAsync(d_hist, 0, (size_t)QM_STATIC_MAX_BINS * 4, stream));
    static_receivers_kernel<<<(cells + 127) / 128, 128, 0, stream>>>(scene->dev, g.origin[0], g.origin[1], g.spacing,
                                                                      g.nx, g.ny, g.height_m, d_alt, d_own);
    const uint32_t n_outlines = (uint32_t)scene->outlines.size();
    if (n_outlines)
        static_own_kernel<<<(n_outlines + 127) / 128, 128, 0, stream>>>(scene->dev, n_outlines, g.origin[0],
                                                                        g.origin[1], g.spacing, g.nx, g.ny, d_own);
    static_own_finish_kernel<<<(cells + 127) / 128, 128, 0, stream>>>(d_own, cells);
    QM_CUDA(cudaGetLastError());
    A.rcv_alt = d_alt;
    A.rcv_own = d_own;
    A.partial = d_partial;
    A.failed = d_failed;
    A.counters = d_counters;
    A.retry = d_retry;
    A.retry_cap = 256;
    A.retry_count = d_rcount;
    if (n_src > 0) {
        dim3 grid_dim(tiles, A.n_chunks);
        if (terrain_caps(scene))
            paint_grid_kernel<CapsTerrain><<<grid_dim, 128, 0, stream>>>(scene->dev, A);
        else
            paint_grid_kernel<CapsFlat><<<grid_dim, 128, 0, stream>>>(scene->dev, A);
        QM_CUDA(cudaGetLastError());
    }
    ReduceArgs R{};
    R.cells = cells;
    R.n_chunks = slices;
    R.partial = d_partial;
    R.level_min = g.level_min_db;
    R.bin_db = g.bin_db;
    R.n_bins = histogram ? g.n_bins : 0;
    R.dba_scratch = d_dba;
    R.cell_bands = d_bands;
    R.cell_dba = d_dbaout;
    R.cell_lden = d_lden;
    R.histogram = histogram ? d_hist : nullptr;
    size_t smem = histogram ? g.n_bins * sizeof(uint32_t) : 0;
    reduce_cells_kernel<<<(cells + 255) / 256, 256, smem, stream>>>(R);
    QM_CUDA(cudaGetLastError());
    unsigned long long counters[6];
    QM_CUDA(cudaMemcpyAsync(counters, d_counters, sizeof(counters), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaMemcpyAsync(cell_bands, d_bands, (size_t)cells * 32, cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaMemcpyAsync(cell_dba, d_dbaout, (size_t)cells * 4, cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaMemcpyAsync(cell_lden, d_lden, (size_t)cells * 4, cudaMemcpyDeviceToHost, stream));
    if (histogram) QM_CUDA(cudaMemcpyAsync(histogram, d_hist, (size_t)g.n_bins * 4, cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaStreamSynchronize(stream));
    if (stats) {
        stats->paths = counters[0];
        stats->crossings = counters[1];
        stats->failed_paths = counters[3];
        stats->edge_tests = counters[2];
        stats->vertices = counters[4];
        stats->candidates = counters[5];
        stats->kernel_ms = -1.0;  // not timed: timing events are left out of this entry point
        stats->paint_ms = -1.0;
    }
    if (counters[3] != 0)
        return fail(QM_ERR_CAPACITY, "qm_paint_grid_static: paths exceeded the per-path capacities; their re-run "
                                     "needs device allocations, use qm_paint_grid");
    return QM_OK;
}

}  // extern "C"

// =============================================================================================
// Doc 29 aircraft on a receiver grid (qm_aircraft.h).

namespace {

const double NPD_FT[10] = {200.0, 400.0, 630.0, 1000.0, 2000.0, 4000.0, 6300.0, 10000.0, 16000.0, 25000.0};
const double A_THIRDS[28] = {-44.7, -39.4, -34.6, -30.2, -26.2, -22.5, -19.1, -16.1, -13.4, -10.9, -8.6, -6.6, -4.8, -3.2,
                             -1.9,  -0.8,  0.0,   0.6,   1.0,   1.2,   1.3,   1.2,   1.0,   0.5,   -0.1, -1.1, -2.5, -4.3};

// The tail's absorption of a SEL curve (npd.rs:169-186), in double on the host.
double tail_alpha_of(const float *sel) {
    double sx = 0, sy = 0, sxx = 0, sxy = 0;
    for (int i = 0; i < 3; ++i) {
        int k = 7 + i;
        double d = NPD_FT[k] * 0.3048;
        double y = sel[k] + 20.0 * std::log10(d / (25000.0 * 0.3048));
        sx += d;
        sy += y;
        sxx += d * d;
        sxy += d * y;
    }
    return std::max(-(3.0 * sxy - sx * sy) / (3.0 * sxx - sx * sx), 0.0);
}

}  // namespace

extern "C" qm_status qm_flight_grid(qm_ctx *ctx, const qm_aircraft_type *types, uint32_t n_types,
                                    const qm_flight_segment *segments, size_t n_segments,
                                    const qm_flight_grid_desc *grid, float *lae_db, float *thirds_db, float *sone,
                                    qm_flight_stats *stats) {
    NvtxRange nvtx_range("qm_flight_grid");
    if (!ctx || !grid) return fail(QM_ERR_ARGUMENT, "qm_flight_grid: null ctx or grid");
    if (n_types == 0 || n_types > 48 || !types) return fail(QM_ERR_ARGUMENT, "qm_flight_grid: 1 to 48 aircraft types");
    if (n_segments && !segments) return fail(QM_ERR_ARGUMENT, "qm_flight_grid: segments is null");
    if (n_segments >= (1ull << 31)) return fail(QM_ERR_ARGUMENT, "qm_flight_grid: too many segments");
    const qm_flight_grid_desc &g = *grid;
    if (g.nx <= 0 || g.ny <= 0 || !(g.spacing_m > 0.0) || (int64_t)g.nx * g.ny > (int64_t(1) << 28) || !(g.duration_s > 0.0))
        return fail(QM_ERR_ARGUMENT, "qm_flight_grid: grid nx, ny, spacing_m or duration_s");
    uint32_t n_flights = 0, last_flight = 0;
    for (size_t i = 0; i < n_segments; ++i) {
        const qm_flight_segment &q = segments[i];
        if (q.type >= n_types) return fail(QM_ERR_ARGUMENT, "qm_flight_grid: segment " + std::to_string(i) + " type");
        if (!(q.power >= 0.0f && q.power <= 9.0f))
            return fail(QM_ERR_ARGUMENT, "qm_flight_grid: segment " + std::to_string(i) + " power outside [0, 9]");
        for (int k = 0; k < 3; ++k)
            if (!std::isfinite(q.start[k]) || !std::isfinite(q.end[k]))
                return fail(QM_ERR_ARGUMENT, "qm_flight_grid: segment " + std::to_string(i) + " ends");
        if (i > 0 && q.flight < last_flight)
            return fail(QM_ERR_ARGUMENT, "qm_flight_grid: segments not grouped by flight");
        last_flight = q.flight;
        n_flights = std::max(n_flights, q.flight + 1);
    }
    std::vector<AcRow> rows((size_t)n_types * 20);
    std::vector<AcType> tv(n_types);
    for (uint32_t t = 0; t < n_types; ++t) {
        const qm_aircraft_type &a = types[t];
        if (!(a.v_ref_kt > 0.0f) || a.installation > 2)
            return fail(QM_ERR_ARGUMENT, "qm_flight_grid: type " + std::to_string(t) + " v_ref_kt or installation");
        for (int op = 0; op < 2; ++op)
            for (int r = 0; r < 10; ++r) {
                AcRow &R = rows[(size_t)t * 20 + op * 10 + r];
                bool placeholder = true;
                for (int k = 0; k < 10; ++k) {
                    R.sel[k] = a.sel_db[op][r][k];
                    double sml = (double)a.sel_db[op][r][k] - (double)a.lamax_db[op][r][k];
                    R.sml[k] = (float)sml;
                    if (std::fabs(sml - 12.0) >= 1e-9) placeholder = false;
                }
                R.tail_alpha = (float)tail_alpha_of(a.sel_db[op][r]);
                R.d0 = (float)(2.0 / 3.141592653589793 * a.v_ref_kt * 1852.0 / 3600.0);
                R.dipole = placeholder ? 1u : 0u;
                R.pad = 0;
            }
        tv[t].v_ref_kt = a.v_ref_kt;
        tv[t].installation = a.installation;
        double weighted = 0.0;
        for (int b = 0; b < 28; ++b) weighted += std::pow(10.0, (a.spectrum_db[b] + A_THIRDS[b]) / 10.0);
        for (int b = 0; b < 28; ++b) tv[t].share[b] = (float)(std::pow(10.0, a.spectrum_db[b] / 10.0) / weighted);
    }
    std::vector<float4> boxes(std::max<uint32_t>(n_flights, 1), make_float4(1e30f, 1e30f, -1e30f, -1e30f));
    for (size_t i = 0; i < n_segments; ++i) {
        const qm_flight_segment &q = segments[i];
        float4 &b = boxes[q.flight];
        b.x = std::min({b.x, q.start[0], q.end[0]});
        b.y = std::min({b.y, q.start[1], q.end[1]});
        b.z = std::max({b.z, q.start[0], q.end[0]});
        b.w = std::max({b.w, q.start[1], q.end[1]});
    }
    std::lock_guard<std::mutex> guard(ctx->lock);
    QM_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t stream = ctx->stream;
    const size_t cells = (size_t)g.nx * g.ny;
    Scratch d_segs, d_boxes, d_rows, d_types, d_lae, d_thirds, d_sone, d_error, d_pairs;
    QM_CUDA(cudaMalloc(&d_segs.p, std::max<size_t>(n_segments, 1) * sizeof(qm_flight_segment)));
    QM_CUDA(cudaMalloc(&d_boxes.p, boxes.size() * sizeof(float4)));
    QM_CUDA(cudaMalloc(&d_rows.p, rows.size() * sizeof(AcRow)));
    QM_CUDA(cudaMalloc(&d_types.p, tv.size() * sizeof(AcType)));
    QM_CUDA(cudaMalloc(&d_lae.p, cells * sizeof(float)));
    QM_CUDA(cudaMalloc(&d_thirds.p, cells * 28 * sizeof(float)));
    QM_CUDA(cudaMalloc(&d_error.p, sizeof(unsigned)));
    QM_CUDA(cudaMalloc(&d_pairs.p, sizeof(unsigned long long)));
    QM_CUDA(cudaMemsetAsync(d_pairs.p, 0, sizeof(unsigned long long), stream));
    if (sone) QM_CUDA(cudaMalloc(&d_sone.p, cells * sizeof(float)));
    if (n_segments)
        QM_CUDA(cudaMemcpyAsync(d_segs.p, segments, n_segments * sizeof(qm_flight_segment), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(d_boxes.p, boxes.data(), boxes.size() * sizeof(float4), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(d_rows.p, rows.data(), rows.size() * sizeof(AcRow), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(d_types.p, tv.data(), tv.size() * sizeof(AcType), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemsetAsync(d_error.p, 0, sizeof(unsigned), stream));
    FlightGridArgs A{};
    A.segs = static_cast<qm_flight_segment *>(d_segs.p);
    A.n_segs = (uint32_t)n_segments;
    A.boxes = static_cast<float4 *>(d_boxes.p);
    A.rows = static_cast<AcRow *>(d_rows.p);
    A.types = static_cast<AcType *>(d_types.p);
    A.n_types = n_types;
    A.ox = g.origin_m[0];
    A.oy = g.origin_m[1];
    A.spacing = g.spacing_m;
    A.nx = g.nx;
    A.ny = g.ny;
    A.height = g.receiver_height_m;
    A.reach2 = g.reach_m > 0.0 ? g.reach_m * g.reach_m : 0.0;
    A.inv_duration = (float)(1.0 / g.duration_s);
    A.lae = static_cast<float *>(d_lae.p);
    A.thirds = static_cast<float *>(d_thirds.p);
    A.error = static_cast<unsigned *>(d_error.p);
    A.pairs = static_cast<unsigned long long *>(d_pairs.p);
    const size_t smem = 2 * AC_TILE * sizeof(qm_flight_segment) + 16 + (size_t)n_types * 20 * sizeof(AcRow) +
                        n_types * sizeof(AcType) + (size_t)n_types * 2 * AC_THREADS * sizeof(float) +
                        AC_TILE * sizeof(SegPre);
    if (smem > 227 * 1024)
        return fail(QM_ERR_UNSUPPORTED, "qm_flight_grid: " + std::to_string(n_types) + " types exceed shared memory");
    QM_CUDA(cudaFuncSetAttribute(flight_grid_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const unsigned blocks = (unsigned)(((g.nx + 15) / 16) * ((g.ny + 15) / 16));
    Events ev;
    QM_CUDA(ev.create());
    QM_CUDA(cudaEventRecord(ev.e0, stream));
    flight_grid_kernel<<<blocks, AC_THREADS, smem, stream>>>(A);
    QM_CUDA(cudaGetLastError());
    QM_CUDA(cudaEventRecord(ev.e1, stream));
    if (sone) {
        launch_zwicker(A.thirds, cells, static_cast<float *>(d_sone.p), stream);
        QM_CUDA(cudaGetLastError());
    }
    QM_CUDA(cudaEventRecord(ev.e2, stream));
    unsigned long long pairs_in_reach = 0;
    QM_CUDA(cudaMemcpyAsync(&pairs_in_reach, d_pairs.p, sizeof(pairs_in_reach), cudaMemcpyDeviceToHost, stream));
    unsigned error = 0;
    QM_CUDA(cudaMemcpyAsync(&error, d_error.p, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
    if (lae_db) QM_CUDA(cudaMemcpyAsync(lae_db, d_lae.p, cells * sizeof(float), cudaMemcpyDeviceToHost, stream));
    if (thirds_db) QM_CUDA(cudaMemcpyAsync(thirds_db, d_thirds.p, cells * 28 * sizeof(float), cudaMemcpyDeviceToHost, stream));
    if (sone) QM_CUDA(cudaMemcpyAsync(sone, d_sone.p, cells * sizeof(float), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaStreamSynchronize(stream));
    if (error) return fail(QM_ERR_TIMEOUT, "qm_flight_grid: a segment tile's copy did not arrive in time");
    if (stats) {
        float k_ms = 0.f, z_ms = 0.f;
        QM_CUDA(cudaEventElapsedTime(&k_ms, ev.e0, ev.e1));
        QM_CUDA(cudaEventElapsedTime(&z_ms, ev.e1, ev.e2));
        stats->pairs = (uint64_t)cells * n_segments;
        stats->pairs_in_reach = pairs_in_reach;
        stats->kernel_ms = k_ms;
        stats->loudness_ms = sone ? z_ms : 0.0;
    }
    return QM_OK;
}

// ---------------------------------------------------------------------------------------------
// The points' horizons for aircraft screening (include/qm_flights.h).

extern "C" qm_status qm_scene_flight_horizons(qm_scene *scene, const double *xy_steps, const double *altitude_m,
                                              const uint64_t *own_footprint, size_t n_points, float *horizons,
                                              double *kernel_ms) {
    NvtxRange nvtx_range("qm_scene_flight_horizons");
    if (kernel_ms) *kernel_ms = 0.0;
    if (!scene) return fail(QM_ERR_ARGUMENT, "qm_scene_flight_horizons: null scene");
    if (n_points == 0) return QM_OK;
    if (!xy_steps || !altitude_m || !own_footprint || !horizons)
        return fail(QM_ERR_ARGUMENT, "qm_scene_flight_horizons: null points, altitudes, footprints or horizons");
    if (n_points >= (1ull << 31)) return fail(QM_ERR_ARGUMENT, "qm_scene_flight_horizons: too many points");
    std::vector<uint32_t> own(n_points);
    for (size_t i = 0; i < n_points; ++i) {
        if (!std::isfinite(xy_steps[2 * i]) || !std::isfinite(xy_steps[2 * i + 1]) || !std::isfinite(altitude_m[i]))
            return fail(QM_ERR_ARGUMENT, "qm_scene_flight_horizons: point " + std::to_string(i) + " position or altitude");
        own[i] = dense_fp(scene, own_footprint[i]);
    }
    qm_ctx *ctx = scene->ctx;
    std::lock_guard<std::mutex> guard(ctx->lock);
    QM_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t stream = ctx->stream;
    const size_t out_bytes = n_points * QM_HORIZON_FLOATS * sizeof(float);
    Scratch d_xy, d_alt, d_own, d_out, d_failed;
    QM_CUDA(cudaMalloc(&d_xy.p, n_points * 2 * sizeof(double)));
    QM_CUDA(cudaMalloc(&d_alt.p, n_points * sizeof(double)));
    QM_CUDA(cudaMalloc(&d_own.p, n_points * sizeof(uint32_t)));
    QM_CUDA(cudaMalloc(&d_out.p, out_bytes));
    QM_CUDA(cudaMalloc(&d_failed.p, n_points * sizeof(unsigned)));
    QM_CUDA(cudaMemcpyAsync(d_xy.p, xy_steps, n_points * 2 * sizeof(double), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(d_alt.p, altitude_m, n_points * sizeof(double), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(d_own.p, own.data(), n_points * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemsetAsync(d_failed.p, 0, n_points * sizeof(unsigned), stream));
    qm::hz::Args H{};
    H.xy = static_cast<const double *>(d_xy.p);
    H.altitude_m = static_cast<const double *>(d_alt.p);
    H.own = static_cast<const uint32_t *>(d_own.p);
    H.n = (uint32_t)n_points;
    H.growth = std::pow(8000.0 / 30.0, 1.0 / (double)(qm::hz::SAMPLES - 1));  // horizons.rs:155-156
    H.out = static_cast<float *>(d_out.p);
    H.failed = static_cast<unsigned *>(d_failed.p);
    Events ev;
    QM_CUDA(ev.create());
    QM_CUDA(cudaEventRecord(ev.e0, stream));
    qm::hz::flight_horizons_kernel<<<(unsigned)n_points, qm::hz::THREADS, 0, stream>>>(scene->dev, H);
    QM_CUDA(cudaGetLastError());
    QM_CUDA(cudaEventRecord(ev.e1, stream));
    std::vector<unsigned> failed(n_points);
    QM_CUDA(cudaMemcpyAsync(horizons, d_out.p, out_bytes, cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaMemcpyAsync(failed.data(), d_failed.p, n_points * sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaStreamSynchronize(stream));
    if (kernel_ms) {
        float ms = 0.f;
        QM_CUDA(cudaEventElapsedTime(&ms, ev.e0, ev.e1));
        *kernel_ms = ms;
    }
    for (size_t i = 0; i < n_points; ++i)
        if (failed[i])
            return fail(QM_ERR_CAPACITY, "qm_scene_flight_horizons: a ray from point " + std::to_string(i) +
                                             " crosses more than 256 edges");
    return QM_OK;
}

// ---------------------------------------------------------------------------------------------
// The bounded wait's own check (include/qm_batch.h).

namespace qm {

// One thread waits on a barrier that nothing completes, so the wait gives up after `limit_ns`; the
// kernel records that it did and how long it waited, and returns. No copy is in flight, so
// returning is safe.
__global__ void bounded_wait_check_kernel(uint64_t limit_ns, unsigned *gave_up, unsigned long long *waited_ns) {
    __shared__ uint64_t bar;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    const uint64_t t0 = global_ns();
    const bool landed = mbar_wait(&bar, 0, limit_ns);
    *waited_ns = global_ns() - t0;
    *gave_up = landed ? 0u : 1u;
}

}  // namespace qm

extern "C" qm_status qm_check_bounded_wait(qm_ctx *ctx, double limit_ms, double *waited_ms) {
    if (!ctx) return fail(QM_ERR_ARGUMENT, "qm_check_bounded_wait: null ctx");
    if (!(limit_ms > 0.0 && limit_ms <= 2000.0)) return fail(QM_ERR_ARGUMENT, "qm_check_bounded_wait: limit_ms in (0, 2000]");
    std::lock_guard<std::mutex> guard(ctx->lock);
    QM_CUDA(cudaSetDevice(ctx->device));
    Scratch d_flag, d_ns;
    QM_CUDA(cudaMalloc(&d_flag.p, sizeof(unsigned)));
    QM_CUDA(cudaMalloc(&d_ns.p, sizeof(unsigned long long)));
    QM_CUDA(cudaMemsetAsync(d_flag.p, 0, sizeof(unsigned), ctx->stream));
    qm::bounded_wait_check_kernel<<<1, 32, 0, ctx->stream>>>((uint64_t)(limit_ms * 1e6), static_cast<unsigned *>(d_flag.p),
                                                             static_cast<unsigned long long *>(d_ns.p));
    QM_CUDA(cudaGetLastError());
    unsigned gave_up = 0;
    unsigned long long ns = 0;
    QM_CUDA(cudaMemcpyAsync(&gave_up, d_flag.p, sizeof(gave_up), cudaMemcpyDeviceToHost, ctx->stream));
    QM_CUDA(cudaMemcpyAsync(&ns, d_ns.p, sizeof(ns), cudaMemcpyDeviceToHost, ctx->stream));
    QM_CUDA(cudaStreamSynchronize(ctx->stream));
    if (waited_ms) *waited_ms = (double)ns / 1e6;
    if (!gave_up) return fail(QM_ERR_CUDA, "qm_check_bounded_wait: a barrier that nothing completes was seen complete");
    if ((double)ns < limit_ms * 1e6) return fail(QM_ERR_CUDA, "qm_check_bounded_wait: the wait gave up before its limit");
    return QM_OK;
}

// ---------------------------------------------------------------------------------------------
// A square's aircraft boxes at lattice points (include/qm_flights.h).

namespace {


bool finite_or_silent(double level) { return !std::isnan(level) && level != INFINITY; }

}  // namespace

struct qm_flight_boxes {
    qm_ctx *ctx = nullptr;
    qm::fl::BoxDev *boxes = nullptr;
    size_t n = 0;
    qm::fl::NpdLogs logs{};
    // The per-call buffers of qm_flight_sums, kept between calls: on the device, and pinned on the
    // host for the horizons going up and the sums coming down while batches compute.
    GrowBuffer points, horizons, segments, order, read_start, slices, sums, heard;
    PinnedBuffer pinned_horizons, pinned_sums;
    cudaStream_t copies = nullptr;  // the copies' stream, beside the context's
    ~qm_flight_boxes() {
        if (boxes) cudaFree(boxes);
        if (copies) cudaStreamDestroy(copies);
    }
};

extern "C" qm_status qm_flight_boxes_upload(qm_ctx *ctx, const qm_flight_box *boxes, size_t n_boxes,
                                            qm_flight_boxes **out) {
    NvtxRange nvtx_range("qm_flight_boxes_upload");
    if (!ctx || !out) return fail(QM_ERR_ARGUMENT, "qm_flight_boxes_upload: null ctx or out");
    *out = nullptr;
    if (n_boxes && !boxes) return fail(QM_ERR_ARGUMENT, "qm_flight_boxes_upload: boxes is null");
    if (n_boxes >= (1ull << 32)) return fail(QM_ERR_ARGUMENT, "qm_flight_boxes_upload: more than 2^32 - 1 boxes");
    for (size_t i = 0; i < n_boxes; ++i) {
        const qm_flight_box &b = boxes[i];
        auto bad = [&](const char *what) {
            return fail(QM_ERR_ARGUMENT, "qm_flight_boxes_upload: box " + std::to_string(i) + " " + what);
        };
        if (!std::isfinite(b.east_m) || !std::isfinite(b.north_m) || !std::isfinite(b.centroid_altitude_m) ||
            !std::isfinite(b.ground_m))
            return bad("position");
        if (!std::isfinite(b.axis_rad) || !std::isfinite(b.gradient) || !(b.gradient_spread >= 0.0) ||
            !std::isfinite(b.gradient_spread))
            return bad("axis, gradient or spread");
        if (b.helicopter > 1) return bad("helicopter flag");
        for (int p = 0; p < QM_PERIODS; ++p) {
            if (!(b.piece_length_m[p] >= 0.0) || !std::isfinite(b.piece_length_m[p])) return bad("piece length");
            if (!(b.passing[p] >= 0.0) || !std::isfinite(b.passing[p])) return bad("passing share");
            if (!finite_or_silent(b.tail_levels_db[p])) return bad("tail level");
            for (int k = 0; k < QM_NPD_DISTANCES; ++k)
                if (!finite_or_silent(b.levels_db[p][k])) return bad("level");
            for (int s = 0; s < 2; ++s)
                for (int k = 0; k < 3; ++k)
                    if (!std::isfinite(b.installation_shares[p][s][k])) return bad("installation share");
        }
        for (int k = 0; k < QM_NPD_DISTANCES; ++k)
            if (!std::isfinite(b.lg_scaled_distance[k])) return bad("scaled distance");
    }
    std::unique_ptr<qm_flight_boxes> h(new qm_flight_boxes);
    h->ctx = ctx;
    h->n = n_boxes;
    const double feet[QM_NPD_DISTANCES] = {200.0, 400.0, 630.0, 1000.0, 2000.0, 4000.0, 6300.0, 10000.0, 16000.0, 25000.0};
    for (int k = 0; k < QM_NPD_DISTANCES; ++k) h->logs.lg[k] = std::log10(feet[k]);  // npd.rs:21-23
    // box_sums.rs:14 and boxes.rs:137-149, as the cores take them
    h->logs.lg_share_span = std::log10(qm::fl::SHARE_FAR_M / qm::fl::SHARE_NEAR_M);
    h->logs.tail_anchor_db = 20.0 * std::log10(qm::fl::TAIL_ANCHOR_M / qm::fl::NPD_LAST_DISTANCE_M);
    {
        std::lock_guard<std::mutex> guard(ctx->lock);
        QM_CUDA(cudaSetDevice(ctx->device));
        QM_CUDA(cudaMalloc(&h->boxes, std::max<size_t>(n_boxes, 1) * sizeof(qm::fl::BoxDev)));
        if (n_boxes) {
            Scratch staged;
            QM_CUDA(cudaMalloc(&staged.p, n_boxes * sizeof(qm_flight_box)));
            QM_CUDA(cudaMemcpyAsync(staged.p, boxes, n_boxes * sizeof(qm_flight_box), cudaMemcpyHostToDevice, ctx->stream));
            qm::fl::derive_boxes_kernel<<<(unsigned)((n_boxes + 127) / 128), 128, 0, ctx->stream>>>(
                static_cast<const qm_flight_box *>(staged.p), (uint32_t)n_boxes, h->boxes);
            QM_CUDA(cudaGetLastError());
            QM_CUDA(cudaStreamSynchronize(ctx->stream));
        }
        ++ctx->children;
    }
    *out = h.release();
    return QM_OK;
}

extern "C" void qm_flight_boxes_free(qm_flight_boxes *boxes) {
    if (!boxes) return;
    qm_ctx *ctx = boxes->ctx;
    cudaSetDevice(ctx->device);
    delete boxes;
    ctx_release(ctx);
}

// qm_flight_sums, and with a scene qm_flight_sums_on_scene: the points' horizons then come from the
// horizons kernel into the handle's device buffer (each point's at its own row) and go nowhere else.
static qm_status flight_sums_impl(qm_ctx *ctx, const qm_flight_boxes *boxes, qm_scene *scene,
                                  const uint64_t *own_footprint, const qm_flight_point *points_in, size_t n_points,
                                  const float *horizons, size_t n_horizon_floats, const qm_box_segment *segments,
                                  size_t n_segments, double *sums, size_t n_sums, qm_flight_sums_stats *stats) {
    // On a scene every point reads its own row of the horizons built on the device.
    std::vector<qm_flight_point> own_rows;
    const qm_flight_point *points = points_in;
    if (scene && points_in) {
        own_rows.assign(points_in, points_in + n_points);
        for (size_t i = 0; i < n_points; ++i) own_rows[i].horizons = (uint64_t)i * QM_HORIZON_FLOATS;
        points = own_rows.data();
        n_horizon_floats = n_points * QM_HORIZON_FLOATS;
    }
    using qm::fl::Slice;
    if (!ctx || !boxes || boxes->ctx != ctx) return fail(QM_ERR_ARGUMENT, "qm_flight_sums: null ctx, or boxes of another context");
    if (n_sums && !sums) return fail(QM_ERR_ARGUMENT, "qm_flight_sums: sums is null");
    if ((n_segments && !segments) || (n_points && !points))
        return fail(QM_ERR_ARGUMENT, "qm_flight_sums: segments or points is null");
    if (n_points >= (1ull << 31) || n_sums >= (1ull << 32) || n_segments >= (1ull << 32))
        return fail(QM_ERR_ARGUMENT, "qm_flight_sums: too many points, sums or segments");
    for (size_t i = 0; i < n_points; ++i) {
        const qm_flight_point &p = points[i];
        if (!std::isfinite(p.x) || !std::isfinite(p.y) || !std::isfinite(p.altitude_m) ||
            !(p.impedance_gain >= 0.0) || !std::isfinite(p.impedance_gain))
            return fail(QM_ERR_ARGUMENT, "qm_flight_sums: point " + std::to_string(i) + " position or impedance gain");
        if ((horizons || scene) && (p.horizons > n_horizon_floats || n_horizon_floats - p.horizons < QM_HORIZON_FLOATS))
            return fail(QM_ERR_ARGUMENT, "qm_flight_sums: point " + std::to_string(i) + " horizons outside the horizon floats");
    }
    // The segments grouped by sum (a counting sort keeps each group in the caller's order).
    std::vector<uint32_t> group_start(n_sums + 1, 0);
    uint64_t total_reads = 0;
    for (size_t i = 0; i < n_segments; ++i) {
        const qm_box_segment &s = segments[i];
        auto bad = [&](const char *what) {
            return fail(QM_ERR_ARGUMENT, "qm_flight_sums: segment " + std::to_string(i) + " " + what);
        };
        if (s.point >= n_points) return bad("point");
        if (s.sum >= n_sums) return bad("sum");
        if ((uint64_t)s.first + s.count > boxes->n) return bad("boxes outside the uploaded boxes");
        if (s.weight > QM_FLIGHT_WEIGHT_NEAR) return bad("weight");
        if (std::isnan(s.within_m)) return bad("within_m");
        if (s.weight != QM_FLIGHT_WEIGHT_ONE && !(s.coarse_m > 0.0 && std::isfinite(s.coarse_m))) return bad("coarse_m");
        if (s.count) ++group_start[s.sum + 1];
        total_reads += s.count;
    }
    for (size_t k = 0; k < n_sums; ++k) group_start[k + 1] += group_start[k];
    const uint32_t n_ordered = n_sums ? group_start[n_sums] : 0;
    std::vector<uint32_t> order(std::max<uint32_t>(n_ordered, 1));
    {
        std::vector<uint32_t> next(group_start.begin(), group_start.end() - (n_sums ? 1 : 0));
        for (size_t i = 0; i < n_segments; ++i)
            if (segments[i].count) order[next[segments[i].sum]++] = (uint32_t)i;
    }
    std::vector<uint64_t> read_start(std::max<uint32_t>(n_ordered, 1), 0);
    std::vector<Slice> slices;
    uint64_t at = 0;
    for (size_t k = 0; k < n_sums; ++k) {
        const uint32_t g0 = group_start[k], g1 = group_start[k + 1];
        if (g0 == g1) continue;
        const uint64_t begin = at;
        int32_t point = (int32_t)segments[order[g0]].point;
        for (uint32_t j = g0; j < g1; ++j) {
            read_start[j] = at;
            at += segments[order[j]].count;
            if ((int32_t)segments[order[j]].point != point) point = -1;
        }
        for (uint64_t r = begin; r < at; r += qm::fl::SLICE_READS)
            slices.push_back(Slice{r, std::min(at, r + qm::fl::SLICE_READS), g0, g1, (uint32_t)k, point});
    }
    if (slices.size() >= (1ull << 31)) return fail(QM_ERR_ARGUMENT, "qm_flight_sums: too many box reads");
    qm_flight_boxes *h = const_cast<qm_flight_boxes *>(boxes);
    std::lock_guard<std::mutex> guard(ctx->lock);
    QM_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t stream = ctx->stream;
    GrowBuffer d_failed;
    if (scene && n_points) {
        // The horizons on the device (qm_scene_flight_horizons' kernel), positions in the scene's steps.
        std::vector<double> xy(2 * n_points), alt(n_points);
        std::vector<uint32_t> own(n_points);
        for (size_t i = 0; i < n_points; ++i) {
            xy[2 * i] = points[i].x / scene->step_m;
            xy[2 * i + 1] = points[i].y / scene->step_m;
            alt[i] = points[i].altitude_m;
            own[i] = own_footprint ? dense_fp(scene, own_footprint[i]) : 0u;
        }
        GrowBuffer d_xy, d_alt, d_own;
        QM_CUDA(d_xy.reserve(xy.size() * sizeof(double)));
        QM_CUDA(d_alt.reserve(alt.size() * sizeof(double)));
        QM_CUDA(d_own.reserve(own.size() * sizeof(uint32_t)));
        QM_CUDA(d_failed.reserve(n_points * sizeof(unsigned)));
        QM_CUDA(h->horizons.reserve(n_horizon_floats * sizeof(float)));
        QM_CUDA(cudaMemcpyAsync(d_xy.p, xy.data(), xy.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
        QM_CUDA(cudaMemcpyAsync(d_alt.p, alt.data(), alt.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
        QM_CUDA(cudaMemcpyAsync(d_own.p, own.data(), own.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        QM_CUDA(cudaMemsetAsync(d_failed.p, 0, n_points * sizeof(unsigned), stream));
        qm::hz::Args H{};
        H.xy = static_cast<const double *>(d_xy.p);
        H.altitude_m = static_cast<const double *>(d_alt.p);
        H.own = static_cast<const uint32_t *>(d_own.p);
        H.n = (uint32_t)n_points;
        H.growth = std::pow(8000.0 / 30.0, 1.0 / (double)(qm::hz::SAMPLES - 1));  // horizons.rs:155-156
        H.out = static_cast<float *>(h->horizons.p);
        H.failed = static_cast<unsigned *>(d_failed.p);
        qm::hz::flight_horizons_kernel<<<(unsigned)n_points, qm::hz::THREADS, 0, stream>>>(scene->dev, H);
        QM_CUDA(cudaGetLastError());
        std::vector<unsigned> failed(n_points);
        QM_CUDA(cudaMemcpyAsync(failed.data(), d_failed.p, n_points * sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
        QM_CUDA(cudaStreamSynchronize(stream));
        for (size_t i = 0; i < n_points; ++i)
            if (failed[i])
                return fail(QM_ERR_CAPACITY, "qm_flight_sums_on_scene: a horizon ray from point " + std::to_string(i) +
                                                 " crosses more than 256 edges");
    }
    const bool resident = scene != nullptr;  // the horizons are on the device already
    const size_t sum_bytes = n_sums * QM_FLIGHT_SUMS * sizeof(double);
    QM_CUDA(h->sums.reserve(sum_bytes));
    QM_CUDA(h->heard.reserve(sizeof(unsigned long long)));
    QM_CUDA(h->points.reserve(n_points * sizeof(qm_flight_point)));
    if (!resident) QM_CUDA(h->horizons.reserve(horizons ? n_horizon_floats * sizeof(float) : 0));
    QM_CUDA(h->segments.reserve(n_segments * sizeof(qm_box_segment)));
    QM_CUDA(h->order.reserve(order.size() * sizeof(uint32_t)));
    QM_CUDA(h->read_start.reserve(read_start.size() * sizeof(uint64_t)));
    QM_CUDA(h->slices.reserve(slices.size() * sizeof(Slice)));
    if (sum_bytes) QM_CUDA(cudaMemsetAsync(h->sums.p, 0, sum_bytes, stream));
    QM_CUDA(cudaMemsetAsync(h->heard.p, 0, sizeof(unsigned long long), stream));
    unsigned long long heard = 0;
    double kernel_ms = 0.0;
    if (slices.empty()) {
        if (sum_bytes) QM_CUDA(cudaMemcpyAsync(sums, h->sums.p, sum_bytes, cudaMemcpyDeviceToHost, stream));
        QM_CUDA(cudaStreamSynchronize(stream));
    } else {
        QM_CUDA(cudaMemcpyAsync(h->points.p, points, n_points * sizeof(qm_flight_point), cudaMemcpyHostToDevice, stream));
        QM_CUDA(cudaMemcpyAsync(h->segments.p, segments, n_segments * sizeof(qm_box_segment), cudaMemcpyHostToDevice, stream));
        QM_CUDA(cudaMemcpyAsync(h->order.p, order.data(), order.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        QM_CUDA(cudaMemcpyAsync(h->read_start.p, read_start.data(), read_start.size() * sizeof(uint64_t),
                                cudaMemcpyHostToDevice, stream));
        QM_CUDA(cudaMemcpyAsync(h->slices.p, slices.data(), slices.size() * sizeof(Slice), cudaMemcpyHostToDevice, stream));
        if (!h->copies) QM_CUDA(cudaStreamCreateWithFlags(&h->copies, cudaStreamNonBlocking));
        QM_CUDA(h->pinned_sums.reserve(sum_bytes));
        if (horizons && !resident) QM_CUDA(h->pinned_horizons.reserve(n_horizon_floats * sizeof(float)));
        // Batches of whole request bands, each with the prefix of the horizons its points read: a
        // batch's horizons go up (through pinned memory, on the copies' stream) while the batch before
        // it computes, and its sums come down while the batches after it compute.
        // A batch of at least five full waves of CTAs (four an SM), so that the launches' partly
        // filled last waves stay a small part of the time; small calls are one batch.
        const size_t wave = (size_t)ctx->sm_count * 4;
        const size_t n_batches = std::max<size_t>(1, std::min<size_t>(8, slices.size() / (5 * wave)));
        std::vector<size_t> cut(1, 0);  // slice boundaries
        for (size_t k = 1; k < n_batches; ++k) {
            size_t at = std::max(cut.back() + 1, slices.size() * k / n_batches);
            while (at < slices.size() && slices[at].sum == slices[at - 1].sum) ++at;
            if (at < slices.size()) cut.push_back(at);
        }
        cut.push_back(slices.size());
        const size_t batches = cut.size() - 1;
        struct BatchEvents {
            cudaEvent_t up = nullptr, start = nullptr, end = nullptr, down = nullptr;
        };
        std::vector<BatchEvents> bev(batches);
        struct EventsGuard {
            std::vector<BatchEvents> &v;
            ~EventsGuard() {
                for (auto &e : v)
                    for (cudaEvent_t x : {e.up, e.start, e.end, e.down})
                        if (x) cudaEventDestroy(x);
            }
        } guard_events{bev};
        for (auto &e : bev) {
            QM_CUDA(cudaEventCreateWithFlags(&e.up, cudaEventDisableTiming));
            QM_CUDA(cudaEventCreate(&e.start));
            QM_CUDA(cudaEventCreate(&e.end));
            QM_CUDA(cudaEventCreateWithFlags(&e.down, cudaEventDisableTiming));
        }
        qm::fl::SumsArgs A{};
        A.boxes = h->boxes;
        A.points = static_cast<const qm_flight_point *>(h->points.p);
        A.horizons = (horizons || resident) ? static_cast<const float *>(h->horizons.p) : nullptr;
        A.segments = static_cast<const qm_box_segment *>(h->segments.p);
        A.order = static_cast<const uint32_t *>(h->order.p);
        A.read_start = static_cast<const uint64_t *>(h->read_start.p);
        A.sums = static_cast<double *>(h->sums.p);
        A.heard = static_cast<unsigned long long *>(h->heard.p);
        A.logs = h->logs;
        // The sums' memset precedes every batch's read-back.
        cudaEvent_t zeroed = nullptr;
        QM_CUDA(cudaEventCreateWithFlags(&zeroed, cudaEventDisableTiming));
        std::unique_ptr<CUevent_st, cudaError_t (*)(cudaEvent_t)> zeroed_guard(zeroed, cudaEventDestroy);
        QM_CUDA(cudaEventRecord(zeroed, stream));
        QM_CUDA(cudaStreamWaitEvent(h->copies, zeroed, 0));
        unsigned char *pin_hz = static_cast<unsigned char *>(h->pinned_horizons.p);
        double *pin_sums = static_cast<double *>(h->pinned_sums.p);
        size_t have = 0;  // horizon floats already sent
        for (size_t bi = 0; bi < batches; ++bi) {
            const Slice &first = slices[cut[bi]], &last = slices[cut[bi + 1] - 1];
            if (horizons && !resident) {
                size_t need = have;
                for (uint32_t j = first.seg_begin; j < last.seg_end; ++j)
                    need = std::max<size_t>(need, points[segments[order[j]].point].horizons + QM_HORIZON_FLOATS);
                if (need > have) {
                    const size_t off = have * sizeof(float), bytes = (need - have) * sizeof(float);
                    std::memcpy(pin_hz + off, reinterpret_cast<const unsigned char *>(horizons) + off, bytes);
                    QM_CUDA(cudaMemcpyAsync(static_cast<unsigned char *>(h->horizons.p) + off, pin_hz + off, bytes,
                                            cudaMemcpyHostToDevice, h->copies));
                    have = need;
                }
            }
            QM_CUDA(cudaEventRecord(bev[bi].up, h->copies));
            QM_CUDA(cudaStreamWaitEvent(stream, bev[bi].up, 0));
            A.slices = static_cast<const Slice *>(h->slices.p) + cut[bi];
            QM_CUDA(cudaEventRecord(bev[bi].start, stream));
            qm::fl::flight_sums_kernel<<<(unsigned)(cut[bi + 1] - cut[bi]), qm::fl::THREADS, 0, stream>>>(A);
            QM_CUDA(cudaGetLastError());
            QM_CUDA(cudaEventRecord(bev[bi].end, stream));
            // The batch's bands: the sums from its first slice's to its last slice's.
            QM_CUDA(cudaStreamWaitEvent(h->copies, bev[bi].end, 0));
            const size_t k0 = first.sum, k1 = (size_t)last.sum + 1;
            QM_CUDA(cudaMemcpyAsync(pin_sums + k0 * QM_FLIGHT_SUMS, static_cast<double *>(h->sums.p) + k0 * QM_FLIGHT_SUMS,
                                    (k1 - k0) * QM_FLIGHT_SUMS * sizeof(double), cudaMemcpyDeviceToHost, h->copies));
            QM_CUDA(cudaEventRecord(bev[bi].down, h->copies));
        }
        // Bands no segment names stay zero; each batch's bands are copied out as they arrive.
        if (sum_bytes) std::memset(sums, 0, sum_bytes);
        for (size_t bi = 0; bi < batches; ++bi) {
            QM_CUDA(cudaEventSynchronize(bev[bi].down));
            const size_t k0 = slices[cut[bi]].sum, k1 = (size_t)slices[cut[bi + 1] - 1].sum + 1;
            std::memcpy(sums + k0 * QM_FLIGHT_SUMS, pin_sums + k0 * QM_FLIGHT_SUMS, (k1 - k0) * QM_FLIGHT_SUMS * sizeof(double));
            float ms = 0.f;
            QM_CUDA(cudaEventElapsedTime(&ms, bev[bi].start, bev[bi].end));
            kernel_ms += ms;
        }
        QM_CUDA(cudaMemcpyAsync(&heard, h->heard.p, sizeof(heard), cudaMemcpyDeviceToHost, stream));
        QM_CUDA(cudaStreamSynchronize(stream));
    }
    if (stats) {
        stats->box_reads = total_reads;
        stats->boxes_heard = heard;
        stats->kernel_ms = kernel_ms;
    }
    return QM_OK;
}

extern "C" qm_status qm_flight_sums(qm_ctx *ctx, const qm_flight_boxes *boxes, const qm_flight_point *points,
                                    size_t n_points, const float *horizons, size_t n_horizon_floats,
                                    const qm_box_segment *segments, size_t n_segments, double *sums, size_t n_sums,
                                    qm_flight_sums_stats *stats) {
    NvtxRange nvtx_range("qm_flight_sums");
    return flight_sums_impl(ctx, boxes, nullptr, nullptr, points, n_points, horizons, n_horizon_floats, segments,
                            n_segments, sums, n_sums, stats);
}

extern "C" qm_status qm_flight_sums_on_scene(qm_scene *scene, const qm_flight_boxes *boxes,
                                             const qm_flight_point *points, const uint64_t *own_footprint,
                                             size_t n_points, const qm_box_segment *segments, size_t n_segments,
                                             double *sums, size_t n_sums, qm_flight_sums_stats *stats) {
    NvtxRange nvtx_range("qm_flight_sums_on_scene");
    if (!scene) return fail(QM_ERR_ARGUMENT, "qm_flight_sums_on_scene: null scene");
    for (size_t i = 0; points && i < n_points; ++i)
        if (!std::isfinite(points[i].x) || !std::isfinite(points[i].y))
            return fail(QM_ERR_ARGUMENT, "qm_flight_sums_on_scene: point " + std::to_string(i) + " position");
    return flight_sums_impl(scene->ctx, boxes, scene, own_footprint, points, n_points, nullptr, 0, segments, n_segments,
                            sums, n_sums, stats);
}

// ---------------------------------------------------------------------------------------------
// The learned surrogate (include/qm_surrogate.h).

struct qm_surrogate {
    qm_ctx *ctx = nullptr;
    qm::MlpDev net;
    ~qm_surrogate() {
        cudaFree(net.master);
        cudaFree(net.w16);
        cudaFree(net.wpack);
        cudaFree(net.error);
        cudaFree(net.adam_m);
        cudaFree(net.adam_v);
    }
};

namespace {

static_assert(QM_SURR_WEIGHTS == MLP_WEIGHTS, "surrogate parameter layout");
static_assert(QM_SURR_FEATURES == MLP_IN && QM_SURR_OUTPUTS == MLP_OUT, "surrogate widths");

void scales_from_params(const float *p, MlpScales &s) {
    const float *q = p + QM_SURR_WEIGHTS;
    auto take = [&](float *dst, int n) {
        std::memcpy(dst, q, n * sizeof(float));
        q += n;
    };
    take(s.in_shift, MLP_IN);
    take(s.in_scale, MLP_IN);
    take(s.out_shift, MLP_OUT);
    take(s.out_scale, MLP_OUT);
    take(s.feat_lo, MLP_IN);
    take(s.feat_hi, MLP_IN);
    take(s.lab_lo, MLP_OUT);
    take(s.lab_hi, MLP_OUT);
    take(&s.feature_set, 1);
}

void scales_to_params(const MlpScales &s, float *p) {
    float *q = p + QM_SURR_WEIGHTS;
    auto put = [&](const float *src, int n) {
        std::memcpy(q, src, n * sizeof(float));
        q += n;
    };
    put(s.in_shift, MLP_IN);
    put(s.in_scale, MLP_IN);
    put(s.out_shift, MLP_OUT);
    put(s.out_scale, MLP_OUT);
    put(s.feat_lo, MLP_IN);
    put(s.feat_hi, MLP_IN);
    put(s.lab_lo, MLP_OUT);
    put(s.lab_hi, MLP_OUT);
    put(&s.feature_set, 1);
}

// The grid checks qm_paint_grid makes.
qm_status check_grid(const qm_scene *scene, const qm_grid_desc &g, const char *name) {
    if (g.nx <= 0 || g.ny <= 0 || g.spacing <= 0 || (int64_t)g.nx * g.ny > (int64_t(1) << 30))
        return fail(QM_ERR_ARGUMENT, std::string(name) + ": grid nx, ny or spacing");
    int64_t last_x = g.origin[0] + (int64_t)(g.nx - 1) * g.spacing, last_y = g.origin[1] + (int64_t)(g.ny - 1) * g.spacing;
    if (g.origin[0] < 0 || g.origin[1] < 0 || last_x >= scene->extent[0] || last_y >= scene->extent[1])
        return fail(QM_ERR_ARGUMENT, std::string(name) + ": grid receivers outside the scene extent");
    uint32_t sb = g.source_begin, se = g.source_end;
    if (se > sb && se > scene->n_sources)
        return fail(QM_ERR_ARGUMENT, std::string(name) + ": source range beyond the scene's sources");
    return QM_OK;
}

// Receivers of a grid on the device and its (tile, source chunk) launch shape.
struct GridSetup {
    Scratch alt, own;
    GridArgs A{};
    int cells = 0, tiles = 0;
};

qm_status setup_grid(qm_scene *scene, const qm_grid_desc &g, uint32_t sb, uint32_t se, GridSetup &G,
                     cudaStream_t stream) {
    qm_ctx *ctx = scene->ctx;
    G.cells = g.nx * g.ny;
    std::vector<float> alt;
    std::vector<uint32_t> own;
    grid_receivers(scene, &g, alt, own);
    GridArgs &A = G.A;
    A.origin_x = g.origin[0];
    A.origin_y = g.origin[1];
    A.spacing = g.spacing;
    A.nx = g.nx;
    A.ny = g.ny;
    A.height_m = g.height_m;
    A.source_begin = sb;
    A.source_end = se;
    A.tile_w = 16;
    A.tile_h = 8;
    A.want_fav = scene->any_favourable;
    for (int p = 0; p < 3; ++p) A.lden_w[p] = (float)LDEN_W[p];
    G.tiles = ((g.nx + A.tile_w - 1) / A.tile_w) * ((g.ny + A.tile_h - 1) / A.tile_h);
    const uint32_t n_src = se - sb;
    uint32_t want_ctas = (uint32_t)ctx->sm_count * 16;
    uint32_t n_chunks = std::max<uint32_t>(1, (want_ctas + G.tiles - 1) / G.tiles);
    n_chunks = std::min<uint32_t>(n_chunks, std::max<uint32_t>(1, n_src / 32));
    n_chunks = std::min<uint32_t>(n_chunks, 65535);
    A.chunk = std::max<uint32_t>(1, (n_src + n_chunks - 1) / n_chunks);
    A.n_chunks = n_src == 0 ? 1 : (n_src + A.chunk - 1) / A.chunk;
    QM_CUDA(cudaMalloc(&G.alt.p, G.cells * sizeof(float)));
    QM_CUDA(cudaMalloc(&G.own.p, G.cells * sizeof(uint32_t)));
    QM_CUDA(cudaMemcpyAsync(G.alt.p, alt.data(), G.cells * sizeof(float), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(G.own.p, own.data(), G.cells * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    A.rcv_alt = static_cast<float *>(G.alt.p);
    A.rcv_own = static_cast<uint32_t *>(G.own.p);
    return QM_OK;
}

// Launch shape of a source sub-range [b0, b1) of a set-up grid.
void chunk_range(const qm_ctx *ctx, GridArgs &A, int tiles, uint32_t b0, uint32_t b1) {
    A.source_begin = b0;
    A.source_end = b1;
    const uint32_t n_src = b1 - b0;
    uint32_t want_ctas = (uint32_t)ctx->sm_count * 16;
    uint32_t n_chunks = std::max<uint32_t>(1, (want_ctas + tiles - 1) / tiles);
    n_chunks = std::min<uint32_t>(n_chunks, std::max<uint32_t>(1, n_src / 32));
    n_chunks = std::min<uint32_t>(n_chunks, 65535);
    A.chunk = std::max<uint32_t>(1, (n_src + n_chunks - 1) / n_chunks);
    A.n_chunks = n_src == 0 ? 1 : (n_src + A.chunk - 1) / A.chunk;
}

// Rows whose first feature (L / 1000) is below `f0_min` lose their eligible flag.
__global__ void floor_rows_kernel(const float *features, uint8_t *eligible, size_t rows, float f0_min) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < rows && features[i * MLP_IN] < f0_min) eligible[i] = 0;
}

__global__ void gather_rows_kernel(const float *src, const uint32_t *index, size_t n, int w, float *dst) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n * w) return;
    size_t r = i / w;
    dst[i] = src[(size_t)index[r] * w + (i - r * w)];
}

__global__ void affine_rows_kernel(float *rows, size_t n, int w, const float *shift, const float *inv_scale) {
    __shared__ float sh[64], sc[64];
    if (threadIdx.x < w) {
        sh[threadIdx.x] = shift[threadIdx.x];
        sc[threadIdx.x] = inv_scale[threadIdx.x];
    }
    __syncthreads();
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n * w) return;
    int c = (int)(i % w);
    rows[i] = (rows[i] - sh[c]) * sc[c];
}

// Exact training samples of one grid: every path's raw features, label and eligibility on the device.
qm_status grid_samples(qm_scene *scene, const qm_grid_desc &g, Scratch &feat, Scratch &lab, Scratch &elig,
                       size_t &rows, cudaStream_t stream) {
    uint32_t sb = g.source_begin, se = g.source_end;
    if (se <= sb) {
        sb = 0;
        se = scene->n_sources;
    }
    GridSetup G;
    qm_status st = setup_grid(scene, g, sb, se, G, stream);
    if (st != QM_OK) return st;
    const size_t per_path = scene->dem_nx != 0 ? 2 : 1;
    rows = (size_t)G.cells * (se - sb) * per_path;
    if (rows == 0) return QM_OK;
    QM_CUDA(cudaMalloc(&feat.p, rows * MLP_IN * sizeof(float)));
    QM_CUDA(cudaMalloc(&lab.p, rows * MLP_OUT * sizeof(float)));
    QM_CUDA(cudaMalloc(&elig.p, rows));
    SampleArgs P{};
    P.g = G.A;
    P.features = static_cast<float *>(feat.p);
    P.labels = static_cast<float *>(lab.p);
    P.eligible = static_cast<uint8_t *>(elig.p);
    if (per_path == 2)
        surrogate_samples_terrain_kernel<<<dim3(G.tiles, G.A.n_chunks), 128, 0, stream>>>(scene->dev, P);
    else
        surrogate_samples_kernel<<<dim3(G.tiles, G.A.n_chunks), 128, 0, stream>>>(scene->dev, P);
    QM_CUDA(cudaGetLastError());
    QM_CUDA(cudaStreamSynchronize(stream));
    return QM_OK;
}

}  // namespace

extern "C" {

qm_status qm_surrogate_create(qm_ctx *ctx, const float *params, qm_surrogate **out) {
    if (!ctx || !params || !out) return fail(QM_ERR_ARGUMENT, "qm_surrogate_create: null ctx, params or out");
    for (size_t i = 0; i < QM_SURR_PARAMS; ++i)
        if (!std::isfinite(params[i])) return fail(QM_ERR_ARGUMENT, "qm_surrogate_create: params[" + std::to_string(i) + "] is not finite");
    std::lock_guard<std::mutex> guard(ctx->lock);
    QM_CUDA(cudaSetDevice(ctx->device));
    auto *s = new qm_surrogate;
    s->ctx = ctx;
    scales_from_params(params, s->net.scales);
    cudaError_t e = cudaMalloc(&s->net.master, MLP_WEIGHTS * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&s->net.w16, MLP_W16 * sizeof(__nv_bfloat16));
    if (e == cudaSuccess) e = cudaMalloc(&s->net.wpack, mlp_packed_bytes());
    if (e == cudaSuccess) e = cudaMalloc(&s->net.error, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemsetAsync(s->net.error, 0, sizeof(unsigned), ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->net.master, params, MLP_WEIGHTS * sizeof(float), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = mlp_cast(s->net, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        delete s;
        return fail(QM_ERR_CUDA, std::string("cuda: ") + cudaGetErrorString(e));
    }
    ++ctx->children;
    *out = s;
    return QM_OK;
}

void qm_surrogate_free(qm_surrogate *net) {
    if (!net) return;
    qm_ctx *ctx = net->ctx;
    {
        std::lock_guard<std::mutex> guard(ctx->lock);
        cudaSetDevice(ctx->device);
        delete net;
    }
    ctx_release(ctx);
}

qm_status qm_surrogate_set_kernel(qm_surrogate *net, int kernel) {
    if (!net || (kernel != 0 && kernel != 1)) return fail(QM_ERR_ARGUMENT, "qm_surrogate_set_kernel: kernel is 0 or 1");
    std::lock_guard<std::mutex> guard(net->ctx->lock);
    net->net.kernel = kernel;
    return QM_OK;
}

qm_status qm_surrogate_params(const qm_surrogate *net, float *params) {
    if (!net || !params) return fail(QM_ERR_ARGUMENT, "qm_surrogate_params: null net or params");
    std::lock_guard<std::mutex> guard(net->ctx->lock);
    QM_CUDA(cudaSetDevice(net->ctx->device));
    QM_CUDA(cudaMemcpyAsync(params, net->net.master, MLP_WEIGHTS * sizeof(float), cudaMemcpyDeviceToHost, net->ctx->stream));
    QM_CUDA(cudaStreamSynchronize(net->ctx->stream));
    scales_to_params(net->net.scales, params);
    return QM_OK;
}

qm_status qm_surrogate_samples(qm_scene *scene, const qm_grid_desc *grid, float *features, float *labels,
                               uint8_t *eligible) {
    NvtxRange nvtx_range("qm_surrogate_samples");
    if (!scene || !grid || !features || !labels || !eligible)
        return fail(QM_ERR_ARGUMENT, "qm_surrogate_samples: null scene, grid or output");
    qm_status st = check_grid(scene, *grid, "qm_surrogate_samples");
    if (st != QM_OK) return st;
    std::lock_guard<std::mutex> guard(scene->ctx->lock);
    QM_CUDA(cudaSetDevice(scene->ctx->device));
    cudaStream_t stream = scene->ctx->stream;
    Scratch f, l, e;
    size_t rows = 0;
    st = grid_samples(scene, *grid, f, l, e, rows, stream);
    if (st != QM_OK) return st;
    if (rows == 0) return QM_OK;
    QM_CUDA(cudaMemcpy(features, f.p, rows * MLP_IN * sizeof(float), cudaMemcpyDeviceToHost));
    QM_CUDA(cudaMemcpy(labels, l.p, rows * MLP_OUT * sizeof(float), cudaMemcpyDeviceToHost));
    QM_CUDA(cudaMemcpy(eligible, e.p, rows, cudaMemcpyDeviceToHost));
    return QM_OK;
}

qm_status qm_surrogate_forward(qm_surrogate *net, const float *features, size_t n, float *outputs) {
    NvtxRange nvtx_range("qm_surrogate_forward");
    if (!net || (n && (!features || !outputs))) return fail(QM_ERR_ARGUMENT, "qm_surrogate_forward: null net, features or outputs");
    if (n == 0) return QM_OK;
    std::lock_guard<std::mutex> guard(net->ctx->lock);
    QM_CUDA(cudaSetDevice(net->ctx->device));
    cudaStream_t stream = net->ctx->stream;
    Scratch raw, x, out;
    QM_CUDA(cudaMalloc(&raw.p, n * MLP_IN * sizeof(float)));
    QM_CUDA(cudaMalloc(&x.p, n * MLP_IN * sizeof(__nv_bfloat16)));
    QM_CUDA(cudaMalloc(&out.p, n * MLP_OUT * sizeof(float)));
    QM_CUDA(cudaMemcpyAsync(raw.p, features, n * MLP_IN * sizeof(float), cudaMemcpyHostToDevice, stream));
    QM_CUDA(mlp_normalise(net->net.scales, static_cast<float *>(raw.p), n, static_cast<__nv_bfloat16 *>(x.p), stream));
    QM_CUDA(mlp_forward(net->net, static_cast<__nv_bfloat16 *>(x.p), n, static_cast<float *>(out.p), stream));
    QM_CUDA(cudaMemcpyAsync(outputs, out.p, n * MLP_OUT * sizeof(float), cudaMemcpyDeviceToHost, stream));
    unsigned err = 0;
    QM_CUDA(cudaMemcpyAsync(&err, net->net.error, sizeof(err), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaStreamSynchronize(stream));
    if (err) return fail(QM_ERR_TIMEOUT, "qm_surrogate_forward: a bounded wait of the inference kernel gave up");
    return QM_OK;
}

qm_status qm_surrogate_gradients(qm_surrogate *net, const float *features, const float *labels, size_t n,
                                 float *grads, double *loss) {
    if (!net || !features || !labels || !grads || !loss)
        return fail(QM_ERR_ARGUMENT, "qm_surrogate_gradients: null net, features, labels, grads or loss");
    if (n == 0 || n % 8 != 0 || n > (1u << 24))
        return fail(QM_ERR_ARGUMENT, "qm_surrogate_gradients: n must be a positive multiple of 8 up to 2^24");
    std::lock_guard<std::mutex> guard(net->ctx->lock);
    QM_CUDA(cudaSetDevice(net->ctx->device));
    cudaStream_t stream = net->ctx->stream;
    std::vector<float> y(n * MLP_OUT);
    for (size_t i = 0; i < n; ++i)
        for (int o = 0; o < MLP_OUT; ++o)
            y[i * MLP_OUT + o] = (labels[i * MLP_OUT + o] - net->net.scales.out_shift[o]) / net->net.scales.out_scale[o];
    Scratch raw, x, dy, dg, dl;
    QM_CUDA(cudaMalloc(&raw.p, n * MLP_IN * sizeof(float)));
    QM_CUDA(cudaMalloc(&x.p, n * MLP_IN * sizeof(__nv_bfloat16)));
    QM_CUDA(cudaMalloc(&dy.p, n * MLP_OUT * sizeof(float)));
    QM_CUDA(cudaMalloc(&dg.p, MLP_WEIGHTS * sizeof(float)));
    QM_CUDA(cudaMalloc(&dl.p, sizeof(double)));
    QM_CUDA(cudaMemcpyAsync(raw.p, features, n * MLP_IN * sizeof(float), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(dy.p, y.data(), n * MLP_OUT * sizeof(float), cudaMemcpyHostToDevice, stream));
    QM_CUDA(mlp_normalise(net->net.scales, static_cast<float *>(raw.p), n, static_cast<__nv_bfloat16 *>(x.p), stream));
    MlpWork *w = mlp_work_create(n);
    if (!w) return fail(QM_ERR_CUDA, "cuda: out of memory for the activations");
    cudaError_t e = mlp_gradients(net->net, w, static_cast<__nv_bfloat16 *>(x.p), static_cast<float *>(dy.p), n,
                                  static_cast<float *>(dg.p), static_cast<double *>(dl.p), stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    mlp_work_free(w);
    if (e != cudaSuccess) return fail(QM_ERR_CUDA, std::string("cuda: ") + cudaGetErrorString(e));
    QM_CUDA(cudaMemcpy(grads, dg.p, MLP_WEIGHTS * sizeof(float), cudaMemcpyDeviceToHost));
    QM_CUDA(cudaMemcpy(loss, dl.p, sizeof(double), cudaMemcpyDeviceToHost));
    return QM_OK;
}

qm_status qm_surrogate_train(qm_surrogate *net, qm_scene *scene, const qm_grid_desc *grids, size_t n_grids,
                             const qm_train_config *config, double *loss_history, uint64_t *n_samples) {
    NvtxRange nvtx_range("qm_surrogate_train");
    if (!net || !scene || !grids || !config || n_grids == 0)
        return fail(QM_ERR_ARGUMENT, "qm_surrogate_train: null net, scene, grids or config");
    if (scene->ctx != net->ctx) return fail(QM_ERR_ARGUMENT, "qm_surrogate_train: net and scene on different contexts");
    const qm_train_config &c = *config;
    if (c.epochs == 0 || c.batch < 256 || c.batch % 128 != 0 || c.batch > (1u << 20) || !(c.learning_rate > 0.0f))
        return fail(QM_ERR_ARGUMENT, "qm_surrogate_train: epochs >= 1, batch a multiple of 128 in [256, 2^20], learning_rate > 0");
    if (!(c.exact_within_m >= 0.0f) || !std::isfinite(c.exact_within_m))
        return fail(QM_ERR_ARGUMENT, "qm_surrogate_train: exact_within_m must be finite and >= 0");
    for (size_t k = 0; k < n_grids; ++k) {
        qm_status st = check_grid(scene, grids[k], "qm_surrogate_train");
        if (st != QM_OK) return st;
    }
    std::lock_guard<std::mutex> guard(net->ctx->lock);
    QM_CUDA(cudaSetDevice(net->ctx->device));
    cudaStream_t stream = net->ctx->stream;
    // Samples: every path of each grid, eligible ones gathered in row order.
    size_t upper = 0;
    for (size_t k = 0; k < n_grids; ++k) {
        const qm_grid_desc &g = grids[k];
        uint32_t n_src = g.source_end > g.source_begin ? g.source_end - g.source_begin : scene->n_sources;
        upper += (size_t)g.nx * g.ny * n_src * (scene->dem_nx != 0 ? 2 : 1);
    }
    if (upper == 0) return fail(QM_ERR_ARGUMENT, "qm_surrogate_train: the grids hold no paths");
    Scratch all_f, all_l;
    QM_CUDA(cudaMalloc(&all_f.p, upper * MLP_IN * sizeof(float)));
    QM_CUDA(cudaMalloc(&all_l.p, upper * MLP_OUT * sizeof(float)));
    size_t total = 0;
    for (size_t k = 0; k < n_grids; ++k) {
        Scratch f, l, e, idx;
        size_t rows = 0;
        qm_status st = grid_samples(scene, grids[k], f, l, e, rows, stream);
        if (st != QM_OK) return st;
        if (rows == 0) continue;
        if (c.exact_within_m > 0.0f) {
            floor_rows_kernel<<<(unsigned)((rows + 255) / 256), 256, 0, stream>>>(
                static_cast<const float *>(f.p), static_cast<uint8_t *>(e.p), rows, c.exact_within_m * 1e-3f);
            QM_CUDA(cudaGetLastError());
        }
        std::vector<uint8_t> flags(rows);
        QM_CUDA(cudaMemcpy(flags.data(), e.p, rows, cudaMemcpyDeviceToHost));
        std::vector<uint32_t> keep;
        keep.reserve(rows);
        for (size_t i = 0; i < rows; ++i)
            if (flags[i]) keep.push_back((uint32_t)i);
        if (keep.empty()) continue;
        QM_CUDA(cudaMalloc(&idx.p, keep.size() * sizeof(uint32_t)));
        QM_CUDA(cudaMemcpyAsync(idx.p, keep.data(), keep.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        size_t nf = keep.size() * MLP_IN, nl = keep.size() * MLP_OUT;
        gather_rows_kernel<<<(unsigned)((nf + 255) / 256), 256, 0, stream>>>(
            static_cast<float *>(f.p), static_cast<uint32_t *>(idx.p), keep.size(), MLP_IN,
            static_cast<float *>(all_f.p) + total * MLP_IN);
        gather_rows_kernel<<<(unsigned)((nl + 255) / 256), 256, 0, stream>>>(
            static_cast<float *>(l.p), static_cast<uint32_t *>(idx.p), keep.size(), MLP_OUT,
            static_cast<float *>(all_l.p) + total * MLP_OUT);
        QM_CUDA(cudaGetLastError());
        QM_CUDA(cudaStreamSynchronize(stream));
        total += keep.size();
    }
    std::mt19937_64 rng(c.seed);
    if (c.max_samples && total > c.max_samples) {
        // A seeded subset, kept in row order.
        std::vector<uint32_t> pick(total);
        for (size_t i = 0; i < total; ++i) pick[i] = (uint32_t)i;
        std::shuffle(pick.begin(), pick.end(), rng);
        pick.resize(c.max_samples);
        std::sort(pick.begin(), pick.end());
        Scratch idx, f2, l2;
        QM_CUDA(cudaMalloc(&idx.p, pick.size() * sizeof(uint32_t)));
        QM_CUDA(cudaMalloc(&f2.p, pick.size() * MLP_IN * sizeof(float)));
        QM_CUDA(cudaMalloc(&l2.p, pick.size() * MLP_OUT * sizeof(float)));
        QM_CUDA(cudaMemcpyAsync(idx.p, pick.data(), pick.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        size_t nf = pick.size() * MLP_IN, nl = pick.size() * MLP_OUT;
        gather_rows_kernel<<<(unsigned)((nf + 255) / 256), 256, 0, stream>>>(
            static_cast<float *>(all_f.p), static_cast<uint32_t *>(idx.p), pick.size(), MLP_IN, static_cast<float *>(f2.p));
        gather_rows_kernel<<<(unsigned)((nl + 255) / 256), 256, 0, stream>>>(
            static_cast<float *>(all_l.p), static_cast<uint32_t *>(idx.p), pick.size(), MLP_OUT, static_cast<float *>(l2.p));
        QM_CUDA(cudaGetLastError());
        QM_CUDA(cudaStreamSynchronize(stream));
        std::swap(all_f.p, f2.p);
        std::swap(all_l.p, l2.p);
        total = pick.size();
    }
    if (total < c.batch) return fail(QM_ERR_ARGUMENT, "qm_surrogate_train: fewer eligible samples than one batch");
    if (n_samples) *n_samples = total;
    // Normalisation and ranges from the samples.
    Scratch stats;
    const size_t stats_bytes = (MLP_IN + MLP_OUT) * (2 * sizeof(double) + 2 * sizeof(float));
    QM_CUDA(cudaMalloc(&stats.p, stats_bytes));
    double *d_sum = static_cast<double *>(stats.p), *d_sq = d_sum + MLP_IN + MLP_OUT;
    float *d_lo = reinterpret_cast<float *>(d_sq + MLP_IN + MLP_OUT), *d_hi = d_lo + MLP_IN + MLP_OUT;
    {
        std::vector<double> zeros(2 * (MLP_IN + MLP_OUT), 0.0);
        std::vector<float> lo(MLP_IN + MLP_OUT, INFINITY), hi(MLP_IN + MLP_OUT, -INFINITY);
        QM_CUDA(cudaMemcpyAsync(d_sum, zeros.data(), zeros.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
        QM_CUDA(cudaMemcpyAsync(d_lo, lo.data(), lo.size() * sizeof(float), cudaMemcpyHostToDevice, stream));
        QM_CUDA(cudaMemcpyAsync(d_hi, hi.data(), hi.size() * sizeof(float), cudaMemcpyHostToDevice, stream));
    }
    QM_CUDA(mlp_column_stats(static_cast<float *>(all_f.p), nullptr, total, MLP_IN, d_sum, d_sq, d_lo, d_hi, stream));
    QM_CUDA(mlp_column_stats(static_cast<float *>(all_l.p), nullptr, total, MLP_OUT, d_sum + MLP_IN, d_sq + MLP_IN,
                             d_lo + MLP_IN, d_hi + MLP_IN, stream));
    std::vector<double> sum(MLP_IN + MLP_OUT), sq(MLP_IN + MLP_OUT);
    std::vector<float> lo(MLP_IN + MLP_OUT), hi(MLP_IN + MLP_OUT);
    QM_CUDA(cudaMemcpyAsync(sum.data(), d_sum, sum.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaMemcpyAsync(sq.data(), d_sq, sq.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaMemcpyAsync(lo.data(), d_lo, lo.size() * sizeof(float), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaMemcpyAsync(hi.data(), d_hi, hi.size() * sizeof(float), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaStreamSynchronize(stream));
    MlpScales &S = net->net.scales;
    S.feature_set = scene->dem_nx != 0 ? 1.0f : 0.0f;
    for (int k = 0; k < MLP_IN + MLP_OUT; ++k) {
        double mean = sum[k] / (double)total;
        double var = std::max(sq[k] / (double)total - mean * mean, 0.0);
        double sd = std::sqrt(var);
        if (k < MLP_IN) {
            S.in_shift[k] = (float)mean;
            S.in_scale[k] = sd > 1e-6 ? (float)(1.0 / sd) : 1.0f;
            S.feat_lo[k] = lo[k];
            S.feat_hi[k] = hi[k];
        } else {
            int o = k - MLP_IN;
            S.out_shift[o] = (float)mean;
            S.out_scale[o] = sd > 1e-6 ? (float)sd : 1.0f;
            S.lab_lo[o] = lo[k];
            S.lab_hi[o] = hi[k];
        }
    }
    // Normalised training set: BF16 features, FP32 labels.
    Scratch X, shift_scale;
    QM_CUDA(cudaMalloc(&X.p, total * MLP_IN * sizeof(__nv_bfloat16)));
    QM_CUDA(mlp_normalise(S, static_cast<float *>(all_f.p), total, static_cast<__nv_bfloat16 *>(X.p), stream));
    {
        std::vector<float> ss(2 * MLP_OUT);
        for (int o = 0; o < MLP_OUT; ++o) {
            ss[o] = S.out_shift[o];
            ss[MLP_OUT + o] = 1.0f / S.out_scale[o];
        }
        QM_CUDA(cudaMalloc(&shift_scale.p, ss.size() * sizeof(float)));
        QM_CUDA(cudaMemcpyAsync(shift_scale.p, ss.data(), ss.size() * sizeof(float), cudaMemcpyHostToDevice, stream));
        size_t nl = total * MLP_OUT;
        affine_rows_kernel<<<(unsigned)((nl + 255) / 256), 256, 0, stream>>>(
            static_cast<float *>(all_l.p), total, MLP_OUT, static_cast<float *>(shift_scale.p),
            static_cast<float *>(shift_scale.p) + MLP_OUT);
        QM_CUDA(cudaGetLastError());
    }
    QM_CUDA(cudaStreamSynchronize(stream));
    cudaFree(all_f.p);
    all_f.p = nullptr;
    // Adam state.
    if (!net->net.adam_m) QM_CUDA(cudaMalloc(&net->net.adam_m, MLP_WEIGHTS * sizeof(float)));
    if (!net->net.adam_v) QM_CUDA(cudaMalloc(&net->net.adam_v, MLP_WEIGHTS * sizeof(float)));
    QM_CUDA(cudaMemsetAsync(net->net.adam_m, 0, MLP_WEIGHTS * sizeof(float), stream));
    QM_CUDA(cudaMemsetAsync(net->net.adam_v, 0, MLP_WEIGHTS * sizeof(float), stream));
    // Shuffled order, batches in a fresh order each epoch.
    std::vector<uint32_t> perm(total);
    for (size_t i = 0; i < total; ++i) perm[i] = (uint32_t)i;
    std::shuffle(perm.begin(), perm.end(), rng);
    Scratch d_perm, bx, by, grads, losses;
    const size_t B = c.batch, steps = total / B;
    QM_CUDA(cudaMalloc(&d_perm.p, total * sizeof(uint32_t)));
    QM_CUDA(cudaMemcpyAsync(d_perm.p, perm.data(), total * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMalloc(&bx.p, B * MLP_IN * sizeof(__nv_bfloat16)));
    QM_CUDA(cudaMalloc(&by.p, B * MLP_OUT * sizeof(float)));
    QM_CUDA(cudaMalloc(&grads.p, MLP_WEIGHTS * sizeof(float)));
    QM_CUDA(cudaMalloc(&losses.p, steps * sizeof(double)));
    MlpWork *work = mlp_work_create(B);
    if (!work) return fail(QM_ERR_CUDA, "cuda: out of memory for the activations");
    std::vector<size_t> order(steps);
    std::vector<double> step_loss(steps);
    const double total_steps = (double)steps * c.epochs;
    int t = 0;
    cudaError_t e = cudaSuccess;
    for (uint32_t epoch = 0; epoch < c.epochs && e == cudaSuccess; ++epoch) {
        for (size_t k = 0; k < steps; ++k) order[k] = k;
        std::shuffle(order.begin(), order.end(), rng);
        for (size_t k = 0; k < steps && e == cudaSuccess; ++k) {
            e = mlp_gather(static_cast<__nv_bfloat16 *>(X.p), static_cast<float *>(all_l.p),
                           static_cast<uint32_t *>(d_perm.p) + order[k] * B, B, static_cast<__nv_bfloat16 *>(bx.p),
                           static_cast<float *>(by.p), stream);
            if (e == cudaSuccess)
                e = mlp_gradients(net->net, work, static_cast<__nv_bfloat16 *>(bx.p), static_cast<float *>(by.p), B,
                                  static_cast<float *>(grads.p), static_cast<double *>(losses.p) + k, stream);
            ++t;
            double frac = t / total_steps;
            float lr = c.learning_rate * (float)(0.05 + 0.95 * 0.5 * (1.0 + std::cos(3.141592653589793 * frac)));
            if (e == cudaSuccess) e = mlp_adam(net->net, static_cast<float *>(grads.p), lr, t, stream);
        }
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(step_loss.data(), losses.p, steps * sizeof(double), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e == cudaSuccess && loss_history) {
            double m = 0.0;
            for (double v : step_loss) m += v;
            loss_history[epoch] = m / (double)steps;
        }
    }
    mlp_work_free(work);
    if (e != cudaSuccess) return fail(QM_ERR_CUDA, std::string("cuda: ") + cudaGetErrorString(e));
    return QM_OK;
}

qm_status qm_paint_grid_surrogate(qm_scene *scene, const qm_grid_desc *grid, qm_surrogate *net, float *cell_bands,
                                  float *cell_dba, float *cell_lden, uint32_t *histogram, qm_paint_stats *stats,
                                  uint64_t *surrogate_paths) {
    NvtxRange nvtx_range("qm_paint_grid_surrogate");
    if (!scene || !grid || !net) return fail(QM_ERR_ARGUMENT, "qm_paint_grid_surrogate: null scene, grid or net");
    if (scene->ctx != net->ctx) return fail(QM_ERR_ARGUMENT, "qm_paint_grid_surrogate: net and scene on different contexts");
    const bool terrain = scene->dem_nx != 0;
    if (!terrain && scene->any_favourable)
        return fail(QM_ERR_UNSUPPORTED, "qm_paint_grid_surrogate: flat scenes in homogeneous conditions only");
    if ((net->net.scales.feature_set != 0.0f) != terrain)
        return fail(QM_ERR_ARGUMENT, std::string("qm_paint_grid_surrogate: the network was trained for ") +
                                         (terrain ? "flat" : "terrain") + " scenes");
    const uint32_t per_path = terrain ? 2 : 1;
    const qm_grid_desc &g = *grid;
    qm_status st = check_grid(scene, g, "qm_paint_grid_surrogate");
    if (st != QM_OK) return st;
    if (histogram && (g.n_bins == 0 || g.n_bins > 51200 || !(g.bin_db > 0.0)))
        return fail(QM_ERR_ARGUMENT, "qm_paint_grid_surrogate: histogram needs 0 < n_bins <= 51200 and bin_db > 0");
    uint32_t sb = g.source_begin, se = g.source_end;
    if (se <= sb) {
        sb = 0;
        se = scene->n_sources;
    }
    qm_ctx *ctx = scene->ctx;
    std::lock_guard<std::mutex> guard(ctx->lock);
    QM_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t stream = ctx->stream;
    GridSetup G;
    st = setup_grid(scene, g, sb, se, G, stream);
    if (st != QM_OK) return st;
    const int cells = G.cells;
    const uint32_t n_src = se - sb;
    // Sources in batches of whole 128-row tiles per cell, at most 2^25 rows a batch.
    const size_t max_rows = size_t(1) << 25;
    uint32_t batch = (uint32_t)std::max<size_t>(128, (max_rows / (size_t)cells / per_path) / 128 * 128);
    batch = std::min<uint32_t>(batch, ((n_src + 127) / 128) * 128);
    uint32_t max_chunks = 1;
    for (uint32_t b0 = sb; b0 < se; b0 += batch) {
        GridArgs tmp = G.A;
        chunk_range(ctx, tmp, G.tiles, b0, std::min(se, b0 + batch));
        max_chunks = std::max(max_chunks, tmp.n_chunks);
    }
    const uint32_t mlp_slices = std::max<uint32_t>(1, batch * per_path / 128);
    const uint32_t slices = max_chunks + 1 + mlp_slices;
    const size_t rows_cap = (size_t)cells * std::max<uint32_t>(batch, 128) * per_path;
    GridArgs A = G.A;
    A.retry_cap = (uint32_t)std::min<int64_t>(std::max<int64_t>((int64_t)cells * n_src / 16, 1 << 20), 1 << 27);
    Scratch d_partial, d_failed, d_counters, d_retry, d_rcount, d_x, d_coef, d_elig, d_taken, d_dba, d_hist, d_bands,
        d_dbaout, d_lden;
    const size_t partial_bytes = (size_t)slices * cells * GRID_SLOTS * sizeof(float);
    QM_CUDA(cudaMalloc(&d_partial.p, partial_bytes));
    QM_CUDA(cudaMalloc(&d_failed.p, cells * sizeof(uint32_t)));
    QM_CUDA(cudaMalloc(&d_counters.p, 6 * sizeof(unsigned long long)));
    QM_CUDA(cudaMalloc(&d_retry.p, (size_t)A.retry_cap * sizeof(uint2)));
    QM_CUDA(cudaMalloc(&d_rcount.p, sizeof(unsigned int)));
    QM_CUDA(cudaMalloc(&d_x.p, rows_cap * MLP_IN * sizeof(__nv_bfloat16)));
    QM_CUDA(cudaMalloc(&d_coef.p, rows_cap * 16 * sizeof(float)));
    QM_CUDA(cudaMalloc(&d_elig.p, rows_cap));
    QM_CUDA(cudaMalloc(&d_taken.p, sizeof(unsigned long long)));
    QM_CUDA(cudaMalloc(&d_dba.p, cells * sizeof(float)));
    QM_CUDA(cudaMemsetAsync(d_partial.p, 0, partial_bytes, stream));
    QM_CUDA(cudaMemsetAsync(d_failed.p, 0, cells * sizeof(uint32_t), stream));
    QM_CUDA(cudaMemsetAsync(d_counters.p, 0, 6 * sizeof(unsigned long long), stream));
    QM_CUDA(cudaMemsetAsync(d_rcount.p, 0, sizeof(unsigned int), stream));
    QM_CUDA(cudaMemsetAsync(d_taken.p, 0, sizeof(unsigned long long), stream));
    A.partial = static_cast<float *>(d_partial.p);
    A.failed = static_cast<uint32_t *>(d_failed.p);
    A.counters = static_cast<unsigned long long *>(d_counters.p);
    A.retry = static_cast<uint2 *>(d_retry.p);
    A.retry_count = static_cast<unsigned int *>(d_rcount.p);
    const MlpScales &S = net->net.scales;
    Events ev;
    QM_CUDA(ev.create());
    QM_CUDA(cudaEventRecord(ev.e0, stream));
    for (uint32_t b0 = sb; b0 < se; b0 += batch) {
        const uint32_t b1 = std::min(se, b0 + batch);
        const uint32_t rpc = ((per_path * (b1 - b0) + 127) / 128) * 128;
        const size_t rows = (size_t)cells * rpc;
        SurrPaintArgs P{};
        P.g = A;
        chunk_range(ctx, P.g, G.tiles, b0, b1);
        P.x = static_cast<__nv_bfloat16 *>(d_x.p);
        P.coef = static_cast<float *>(d_coef.p);
        P.eligible = static_cast<uint8_t *>(d_elig.p);
        P.rows_per_cell = rpc;
        for (int k = 0; k < MLP_IN; ++k) {
            P.in_shift[k] = S.in_shift[k];
            P.in_scale[k] = S.in_scale[k];
            P.lo[k] = S.feat_lo[k];
            P.hi[k] = S.feat_hi[k];
        }
        QM_CUDA(cudaMemsetAsync(d_elig.p, 0, rows, stream));
        if (terrain)
            surrogate_front_terrain_kernel<<<dim3(G.tiles, P.g.n_chunks), 128, 0, stream>>>(scene->dev, P);
        else
            surrogate_front_kernel<<<dim3(G.tiles, P.g.n_chunks), 128, 0, stream>>>(scene->dev, P);
        QM_CUDA(cudaGetLastError());
        MlpPaintArgs M{};
        M.x = P.x;
        M.coef = P.coef;
        M.eligible = P.eligible;
        M.rows = rows;
        M.rows_per_cell = rpc;
        M.cells = cells;
        M.partial = A.partial + (size_t)(max_chunks + 1) * cells * GRID_SLOTS;
        M.source_begin = b0;
        M.n_sources = b1 - b0;
        M.rows_per_path = per_path;
        M.retry = A.retry;
        M.retry_cap = A.retry_cap;
        M.retry_count = A.retry_count;
        M.taken = static_cast<unsigned long long *>(d_taken.p);
        QM_CUDA(mlp_paint(net->net, M, stream));
    }
    QM_CUDA(cudaEventRecord(ev.e2, stream));
    unsigned int n_retry = 0;
    QM_CUDA(cudaMemcpyAsync(&n_retry, d_rcount.p, sizeof(n_retry), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaStreamSynchronize(stream));
    if (n_retry > A.retry_cap)
        return fail(QM_ERR_CAPACITY, "qm_paint_grid_surrogate: " + std::to_string(n_retry) +
                                         " paths to re-run, more than the re-run list holds");
    if (n_retry > 0) {
        st = rerun_failed(scene, A, static_cast<uint2 *>(d_retry.p), n_retry, max_chunks, cells, stream);
        if (st != QM_OK) return st;
    }
    ReduceArgs R{};
    R.cells = cells;
    R.n_chunks = slices;
    R.partial = A.partial;
    R.level_min = g.level_min_db;
    R.bin_db = g.bin_db;
    R.n_bins = histogram ? g.n_bins : 0;
    R.dba_scratch = static_cast<float *>(d_dba.p);
    if (cell_bands) QM_CUDA(cudaMalloc(&d_bands.p, (size_t)cells * 8 * sizeof(float)));
    if (cell_dba) QM_CUDA(cudaMalloc(&d_dbaout.p, (size_t)cells * sizeof(float)));
    if (cell_lden) QM_CUDA(cudaMalloc(&d_lden.p, (size_t)cells * sizeof(float)));
    if (histogram) {
        QM_CUDA(cudaMalloc(&d_hist.p, g.n_bins * sizeof(uint32_t)));
        QM_CUDA(cudaMemsetAsync(d_hist.p, 0, g.n_bins * sizeof(uint32_t), stream));
    }
    R.cell_bands = static_cast<float *>(d_bands.p);
    R.cell_dba = static_cast<float *>(d_dbaout.p);
    R.cell_lden = static_cast<float *>(d_lden.p);
    R.histogram = static_cast<uint32_t *>(d_hist.p);
    size_t smem = histogram ? g.n_bins * sizeof(uint32_t) : 0;
    if (smem > 48 * 1024) QM_CUDA(cudaFuncSetAttribute(reduce_cells_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    reduce_cells_kernel<<<(cells + 255) / 256, 256, smem, stream>>>(R);
    QM_CUDA(cudaGetLastError());
    QM_CUDA(cudaEventRecord(ev.e1, stream));
    unsigned long long counters[6], taken = 0;
    unsigned net_error = 0;
    QM_CUDA(cudaMemcpyAsync(counters, d_counters.p, sizeof(counters), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaMemcpyAsync(&taken, d_taken.p, sizeof(taken), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaMemcpyAsync(&net_error, net->net.error, sizeof(net_error), cudaMemcpyDeviceToHost, stream));
    if (cell_bands) QM_CUDA(cudaMemcpyAsync(cell_bands, d_bands.p, (size_t)cells * 8 * sizeof(float), cudaMemcpyDeviceToHost, stream));
    if (cell_dba) QM_CUDA(cudaMemcpyAsync(cell_dba, d_dbaout.p, (size_t)cells * sizeof(float), cudaMemcpyDeviceToHost, stream));
    if (cell_lden) QM_CUDA(cudaMemcpyAsync(cell_lden, d_lden.p, (size_t)cells * sizeof(float), cudaMemcpyDeviceToHost, stream));
    if (histogram) QM_CUDA(cudaMemcpyAsync(histogram, d_hist.p, g.n_bins * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaStreamSynchronize(stream));
    float ms = 0.f, front_ms = 0.f;
    QM_CUDA(cudaEventElapsedTime(&ms, ev.e0, ev.e1));
    QM_CUDA(cudaEventElapsedTime(&front_ms, ev.e0, ev.e2));
    if (stats) {
        stats->paths = counters[0];
        stats->crossings = counters[1];
        stats->failed_paths = counters[3];
        stats->edge_tests = counters[2];
        stats->vertices = counters[4];
        stats->candidates = counters[5];
        stats->kernel_ms = ms;
        stats->paint_ms = front_ms;
    }
    if (net_error) return fail(QM_ERR_TIMEOUT, "qm_paint_grid_surrogate: a bounded wait of the inference kernel gave up");
    if (surrogate_paths) *surrogate_paths = taken;
    return QM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Batches of uneven tiles (include/qm_tiles.h).

struct qm_batch_plan {
    qm_scene *scene = nullptr;
    uint64_t n_cells = 0;
    bool use_graph = false;
    std::vector<TileDev> tiles;
    struct Launch {
        int threads = 128;
        uint32_t n_items = 0, grid = 0;
        Scratch items, next;
    };
    std::vector<Launch> launches;  // one per threads-per-CTA value in use
    Scratch d_tiles, d_cell_tile, d_rcv_xy, d_alt, d_own, d_partial, d_retry, d_rcount, d_counters, d_retry_acc,
        d_bands, d_dba, d_lden;
    uint32_t retry_cap = 0;
    size_t partial_slots = 0;
    float lden_w[3];
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~qm_batch_plan() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

namespace {

const qm_tile_config TILE_BLOCKS[5] = {{16, 8, 128, 0}, {16, 16, 256, 0}, {32, 16, 128, 0}, {32, 32, 256, 0}, {64, 64, 256, 0}};
const uint32_t TILE_CHUNKS[5] = {128, 256, 512, 1024, 2048};

qm_tile_config tile_candidate(int k) {
    qm_tile_config c = TILE_BLOCKS[k / 5];
    c.chunk = TILE_CHUNKS[k % 5];
    return c;
}

bool tile_config_ok(const qm_tile_config &c) {
    return c.block_w >= 8 && c.block_w <= 64 && c.block_w % 8 == 0 && c.block_h >= 8 && c.block_h <= 64 &&
           c.block_h % 8 == 0 && (c.threads == 128 || c.threads == 256) && c.chunk >= 32 && c.chunk <= 65536;
}

// The batch's launches (queue resets, persistent CTAs) on the stream, graph or not.
cudaError_t batch_launch(qm_batch_plan *P, cudaStream_t stream) {
    cudaError_t e;
    if ((e = cudaMemsetAsync(P->d_rcount.p, 0, sizeof(unsigned int), stream)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(P->d_counters.p, 0, 6 * sizeof(unsigned long long), stream)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(P->d_retry_acc.p, 0, P->n_cells * GRID_SLOTS * sizeof(float), stream)) != cudaSuccess)
        return e;
    const bool terrain = terrain_caps(P->scene);
    for (auto &L : P->launches) {
        if ((e = cudaMemsetAsync(L.next.p, 0, sizeof(unsigned int), stream)) != cudaSuccess) return e;
        BatchArgs B{};
        B.tiles = static_cast<TileDev *>(P->d_tiles.p);
        B.items = static_cast<WorkItem *>(L.items.p);
        B.n_items = L.n_items;
        B.next = static_cast<unsigned int *>(L.next.p);
        B.rcv_alt = static_cast<float *>(P->d_alt.p);
        B.rcv_own = static_cast<uint32_t *>(P->d_own.p);
        B.partial = static_cast<float *>(P->d_partial.p);
        B.retry = static_cast<uint2 *>(P->d_retry.p);
        B.retry_cap = P->retry_cap;
        B.retry_count = static_cast<unsigned int *>(P->d_rcount.p);
        B.counters = static_cast<unsigned long long *>(P->d_counters.p);
        for (int k = 0; k < 3; ++k) B.lden_w[k] = P->lden_w[k];
        B.want_fav = P->scene->any_favourable;
        if (L.threads == 256) {
            if (terrain)
                batch_paint_kernel<CapsTerrain, 256><<<L.grid, 256, 0, stream>>>(P->scene->dev, B);
            else
                batch_paint_kernel<CapsFlat, 256><<<L.grid, 256, 0, stream>>>(P->scene->dev, B);
        } else {
            if (terrain)
                batch_paint_kernel<CapsTerrain, 128><<<L.grid, 128, 0, stream>>>(P->scene->dev, B);
            else
                batch_paint_kernel<CapsFlat, 128><<<L.grid, 128, 0, stream>>>(P->scene->dev, B);
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace

extern "C" {

uint32_t qm_tile_bucket(const qm_tile_desc *tile) {
    int side = std::max(tile->nx, tile->ny);
    return side < 64 ? 0u : side < 128 ? 1u : side < 256 ? 2u : 3u;
}

void qm_tune_default(qm_tune_table *table) {
    for (int b = 0; b < QM_TILE_BUCKETS; ++b) table->bucket[b] = qm_tile_config{16, 8, 128, 512};
}

void qm_batch_plan_free(qm_batch_plan *plan) {
    if (!plan) return;
    qm_scene *scene = plan->scene;
    qm_ctx *ctx = scene->ctx;
    bool scene_done;
    {
        std::lock_guard<std::mutex> guard(ctx->lock);
        cudaSetDevice(ctx->device);
        delete plan;
        scene_done = --scene->plans == 0 && scene->freed;
    }
    if (!scene_done) return;
    delete scene;  // freed by its owner while this plan still held it
    ctx_release(ctx);
}

qm_status qm_batch_plan_create(qm_scene *scene, const qm_tile_desc *tiles, size_t n_tiles, uint64_t n_cells,
                               const qm_tune_table *table, uint32_t flags, qm_batch_plan **out) {
    NvtxRange nvtx_range("qm_batch_plan_create");
    if (!scene || !out || (n_tiles && !tiles)) return fail(QM_ERR_ARGUMENT, "qm_batch_plan_create: null scene, tiles or out");
    if (n_tiles == 0 || n_tiles > (1u << 20)) return fail(QM_ERR_ARGUMENT, "qm_batch_plan_create: 1 to 2^20 tiles");
    if (n_cells == 0 || n_cells > (1ull << 31)) return fail(QM_ERR_ARGUMENT, "qm_batch_plan_create: n_cells in [1, 2^31]");
    qm_tune_table tab;
    if (table)
        tab = *table;
    else
        qm_tune_default(&tab);
    for (int b = 0; b < QM_TILE_BUCKETS; ++b)
        if (!tile_config_ok(tab.bucket[b]))
            return fail(QM_ERR_ARGUMENT, "qm_batch_plan_create: table bucket " + std::to_string(b) +
                                             ": block sides multiples of 8 in [8, 64], threads 128 or 256, chunk in [32, 65536]");
    // Tiles: inside the scene, cells within n_cells and disjoint.
    std::vector<std::pair<uint64_t, uint64_t>> ranges(n_tiles);
    for (size_t t = 0; t < n_tiles; ++t) {
        const qm_tile_desc &d = tiles[t];
        const std::string name = "qm_batch_plan_create: tile " + std::to_string(t);
        if (d.nx <= 0 || d.ny <= 0 || d.spacing <= 0 || (int64_t)d.nx * d.ny > (int64_t(1) << 26))
            return fail(QM_ERR_ARGUMENT, name + ": nx, ny or spacing");
        int64_t last_x = d.origin[0] + (int64_t)(d.nx - 1) * d.spacing, last_y = d.origin[1] + (int64_t)(d.ny - 1) * d.spacing;
        if (d.origin[0] < 0 || d.origin[1] < 0 || last_x >= scene->extent[0] || last_y >= scene->extent[1])
            return fail(QM_ERR_ARGUMENT, name + ": receivers outside the scene extent");
        if (d.source_end > d.source_begin && d.source_end > scene->n_sources)
            return fail(QM_ERR_ARGUMENT, name + ": source range beyond the scene's sources");
        uint64_t cells = (uint64_t)d.nx * d.ny;
        if (d.cell_offset + cells > n_cells) return fail(QM_ERR_ARGUMENT, name + ": cells beyond n_cells");
        ranges[t] = {d.cell_offset, d.cell_offset + cells};
    }
    {
        std::vector<std::pair<uint64_t, uint64_t>> sorted = ranges;
        std::sort(sorted.begin(), sorted.end());
        for (size_t k = 1; k < sorted.size(); ++k)
            if (sorted[k].first < sorted[k - 1].second) return fail(QM_ERR_ARGUMENT, "qm_batch_plan_create: tiles share output cells");
    }
    qm_ctx *ctx = scene->ctx;
    std::lock_guard<std::mutex> guard(ctx->lock);
    QM_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t stream = ctx->stream;
    auto *P = new qm_batch_plan;
    std::unique_ptr<qm_batch_plan> hold(P);
    P->scene = scene;
    P->n_cells = n_cells;
    P->use_graph = (flags & QM_BATCH_GRAPH) != 0;
    for (int p = 0; p < 3; ++p) P->lden_w[p] = (float)LDEN_W[p];
    std::vector<float> alt(n_cells, 0.0f);
    std::vector<uint32_t> own(n_cells, 0), cell_tile(n_cells, ~0u);
    std::vector<int2> xy(n_cells, make_int2(0, 0));
    struct Pending {
        WorkItem item;
        uint64_t work;
    };
    std::vector<Pending> pending[2];  // 128 and 256 threads
    uint64_t total_paths = 0;
    for (size_t t = 0; t < n_tiles; ++t) {
        const qm_tile_desc &d = tiles[t];
        const qm_tile_config &c = tab.bucket[qm_tile_bucket(&d)];
        uint32_t sb = d.source_begin, se = d.source_end;
        if (se <= sb) {
            sb = 0;
            se = scene->n_sources;
        }
        TileDev T{};
        T.origin_x = d.origin[0];
        T.origin_y = d.origin[1];
        T.spacing = d.spacing;
        T.nx = d.nx;
        T.ny = d.ny;
        T.source_begin = sb;
        T.source_end = se;
        T.block_w = c.block_w;
        T.block_h = c.block_h;
        T.chunk = c.chunk;
        T.n_chunks = se > sb ? (se - sb + c.chunk - 1) / c.chunk : 0;
        T.cell_offset = d.cell_offset;
        T.partial_offset = P->partial_slots;
        const uint64_t cells = (uint64_t)d.nx * d.ny;
        P->partial_slots += cells * T.n_chunks;
        total_paths += cells * (se - sb);
        P->tiles.push_back(T);
        qm_grid_desc g{};
        g.origin[0] = d.origin[0];
        g.origin[1] = d.origin[1];
        g.spacing = d.spacing;
        g.nx = d.nx;
        g.ny = d.ny;
        g.height_m = d.height_m;
        std::vector<float> a;
        std::vector<uint32_t> o;
        grid_receivers(scene, &g, a, o);
        for (uint64_t k = 0; k < cells; ++k) {
            uint64_t gc = d.cell_offset + k;
            alt[gc] = a[k];
            own[gc] = o[k];
            cell_tile[gc] = (uint32_t)t;
            xy[gc] = make_int2(d.origin[0] + (int)(k % d.nx) * d.spacing, d.origin[1] + (int)(k / d.nx) * d.spacing);
        }
        const uint32_t bx = (d.nx + c.block_w - 1) / c.block_w, by = (d.ny + c.block_h - 1) / c.block_h;
        for (uint32_t b = 0; b < bx * by; ++b) {
            uint32_t w = std::min<uint32_t>(c.block_w, d.nx - (b % bx) * c.block_w);
            uint32_t h = std::min<uint32_t>(c.block_h, d.ny - (b / bx) * c.block_h);
            for (uint32_t ch = 0; ch < T.n_chunks; ++ch) {
                uint32_t n = std::min<uint32_t>(c.chunk, se - sb - ch * c.chunk);
                pending[c.threads == 256 ? 1 : 0].push_back(Pending{WorkItem{(uint32_t)t, b, ch, 0}, (uint64_t)w * h * n});
            }
        }
    }
    if (P->partial_slots > (size_t(1) << 31))
        return fail(QM_ERR_CAPACITY, "qm_batch_plan_create: the batch's partial sums exceed 2^31 slots; use larger chunks");
    // Largest items first: the persistent CTAs then finish together.
    for (int k = 0; k < 2; ++k) {
        if (pending[k].empty()) continue;
        std::stable_sort(pending[k].begin(), pending[k].end(), [](const Pending &a, const Pending &b) { return a.work > b.work; });
        if (pending[k].size() >= (1ull << 32)) return fail(QM_ERR_CAPACITY, "qm_batch_plan_create: too many work items");
        P->launches.emplace_back();
        auto &L = P->launches.back();
        L.threads = k == 1 ? 256 : 128;
        L.n_items = (uint32_t)pending[k].size();
        L.grid = (uint32_t)std::min<uint64_t>(L.n_items, (uint64_t)ctx->sm_count * (512 / L.threads));
        std::vector<WorkItem> items(L.n_items);
        for (uint32_t i = 0; i < L.n_items; ++i) items[i] = pending[k][i].item;
        QM_CUDA(cudaMalloc(&L.items.p, items.size() * sizeof(WorkItem)));
        QM_CUDA(cudaMalloc(&L.next.p, sizeof(unsigned int)));
        QM_CUDA(cudaMemcpyAsync(L.items.p, items.data(), items.size() * sizeof(WorkItem), cudaMemcpyHostToDevice, stream));
        QM_CUDA(cudaStreamSynchronize(stream));
    }
    P->retry_cap = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(total_paths / 16, 1 << 20), 1 << 27);
    QM_CUDA(cudaMalloc(&P->d_tiles.p, P->tiles.size() * sizeof(TileDev)));
    QM_CUDA(cudaMalloc(&P->d_cell_tile.p, n_cells * sizeof(uint32_t)));
    QM_CUDA(cudaMalloc(&P->d_rcv_xy.p, n_cells * sizeof(int2)));
    QM_CUDA(cudaMalloc(&P->d_alt.p, n_cells * sizeof(float)));
    QM_CUDA(cudaMalloc(&P->d_own.p, n_cells * sizeof(uint32_t)));
    QM_CUDA(cudaMalloc(&P->d_partial.p, std::max<size_t>(P->partial_slots, 1) * GRID_SLOTS * sizeof(float)));
    QM_CUDA(cudaMalloc(&P->d_retry.p, (size_t)P->retry_cap * sizeof(uint2)));
    QM_CUDA(cudaMalloc(&P->d_rcount.p, sizeof(unsigned int)));
    QM_CUDA(cudaMalloc(&P->d_counters.p, 6 * sizeof(unsigned long long)));
    QM_CUDA(cudaMalloc(&P->d_retry_acc.p, n_cells * GRID_SLOTS * sizeof(float)));
    QM_CUDA(cudaMalloc(&P->d_bands.p, n_cells * QM_BANDS * sizeof(float)));
    QM_CUDA(cudaMalloc(&P->d_dba.p, n_cells * sizeof(float)));
    QM_CUDA(cudaMalloc(&P->d_lden.p, n_cells * sizeof(float)));
    QM_CUDA(cudaMemcpyAsync(P->d_tiles.p, P->tiles.data(), P->tiles.size() * sizeof(TileDev), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(P->d_cell_tile.p, cell_tile.data(), n_cells * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(P->d_rcv_xy.p, xy.data(), n_cells * sizeof(int2), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(P->d_alt.p, alt.data(), n_cells * sizeof(float), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(P->d_own.p, own.data(), n_cells * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaStreamSynchronize(stream));
    if (P->use_graph) {
        QM_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = batch_launch(P, stream);
        cudaGraph_t graph = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(stream, &graph);
        if (e != cudaSuccess || e2 != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            return fail(QM_ERR_CUDA, std::string("cuda: graph capture: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
        }
        P->graph = graph;
        QM_CUDA(cudaGraphInstantiate(&P->exec, P->graph, 0));
    }
    ++scene->plans;
    *out = hold.release();
    return QM_OK;
}

qm_status qm_batch_plan_run(qm_batch_plan *P, qm_paint_stats *stats) {
    NvtxRange nvtx_range("qm_batch_plan_run");
    if (!P) return fail(QM_ERR_ARGUMENT, "qm_batch_plan_run: null plan");
    qm_scene *scene = P->scene;
    qm_ctx *ctx = scene->ctx;
    std::lock_guard<std::mutex> guard(ctx->lock);
    QM_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t stream = ctx->stream;
    Events ev;
    QM_CUDA(ev.create());
    QM_CUDA(cudaEventRecord(ev.e0, stream));
    if (P->use_graph)
        QM_CUDA(cudaGraphLaunch(P->exec, stream));
    else
        QM_CUDA(batch_launch(P, stream));
    QM_CUDA(cudaEventRecord(ev.e2, stream));
    unsigned int n_retry = 0;
    QM_CUDA(cudaMemcpyAsync(&n_retry, P->d_rcount.p, sizeof(n_retry), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaStreamSynchronize(stream));
    if (n_retry > P->retry_cap)
        return fail(QM_ERR_CAPACITY, "qm_batch_plan_run: " + std::to_string(n_retry) + " over-capacity paths, more than the re-run list holds");
    if (n_retry > 0) {
        std::vector<uint2> list(n_retry);
        QM_CUDA(cudaMemcpy(list.data(), P->d_retry.p, n_retry * sizeof(uint2), cudaMemcpyDeviceToHost));
        std::sort(list.begin(), list.end(), [](uint2 a, uint2 b) { return a.x != b.x ? a.x < b.x : a.y < b.y; });
        std::vector<uint32_t> cids, cstart;
        for (uint32_t i = 0; i < n_retry; ++i)
            if (cids.empty() || cids.back() != list[i].x) {
                cids.push_back(list[i].x);
                cstart.push_back(i);
            }
        cstart.push_back(n_retry);
        const uint32_t threads = std::min<uint32_t>(((n_retry + 63) / 64) * 64, 8192);
        using Large = PathWork<CapsLarge::C, CapsLarge::K, CapsLarge::H>;
        Scratch d_sorted, d_cids, d_cstart, d_works, d_results, d_rstatus;
        QM_CUDA(cudaMalloc(&d_sorted.p, n_retry * sizeof(uint2)));
        QM_CUDA(cudaMalloc(&d_cids.p, cids.size() * sizeof(uint32_t)));
        QM_CUDA(cudaMalloc(&d_cstart.p, cstart.size() * sizeof(uint32_t)));
        QM_CUDA(cudaMalloc(&d_works.p, (size_t)threads * sizeof(Large)));
        QM_CUDA(cudaMalloc(&d_results.p, (size_t)n_retry * GRID_SLOTS * sizeof(float)));
        QM_CUDA(cudaMalloc(&d_rstatus.p, (size_t)n_retry * sizeof(uint32_t)));
        QM_CUDA(cudaMemcpyAsync(d_sorted.p, list.data(), n_retry * sizeof(uint2), cudaMemcpyHostToDevice, stream));
        QM_CUDA(cudaMemcpyAsync(d_cids.p, cids.data(), cids.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        QM_CUDA(cudaMemcpyAsync(d_cstart.p, cstart.data(), cstart.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        BatchRetryArgs RA{};
        RA.rcv_xy = static_cast<int2 *>(P->d_rcv_xy.p);
        RA.rcv_alt = static_cast<float *>(P->d_alt.p);
        RA.rcv_own = static_cast<uint32_t *>(P->d_own.p);
        for (int k = 0; k < 3; ++k) RA.lden_w[k] = P->lden_w[k];
        RA.want_fav = scene->any_favourable;
        batch_retry_kernel<<<threads / 64, 64, 0, stream>>>(scene->dev, RA, static_cast<uint2 *>(d_sorted.p), n_retry,
                                                            static_cast<Large *>(d_works.p),
                                                            static_cast<float *>(d_results.p),
                                                            static_cast<uint32_t *>(d_rstatus.p));
        QM_CUDA(cudaGetLastError());
        fold_retry_kernel<<<(unsigned)((cids.size() + 127) / 128), 128, 0, stream>>>(
            static_cast<uint32_t *>(d_cids.p), static_cast<uint32_t *>(d_cstart.p), (uint32_t)cids.size(),
            static_cast<float *>(d_results.p), static_cast<float *>(P->d_retry_acc.p), 0, (int)P->n_cells);
        QM_CUDA(cudaGetLastError());
        std::vector<uint32_t> rstatus(n_retry);
        QM_CUDA(cudaMemcpyAsync(rstatus.data(), d_rstatus.p, n_retry * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        QM_CUDA(cudaStreamSynchronize(stream));
        size_t still = 0;
        for (uint32_t v : rstatus) still += v != 0;
        if (still)
            return fail(QM_ERR_CAPACITY, "qm_batch_plan_run: " + std::to_string(still) + " paths exceed even the large per-path capacities");
    }
    BatchReduceArgs R{};
    R.tiles = static_cast<TileDev *>(P->d_tiles.p);
    R.cell_tile = static_cast<uint32_t *>(P->d_cell_tile.p);
    R.n_cells = P->n_cells;
    R.partial = static_cast<float *>(P->d_partial.p);
    R.retry_acc = static_cast<float *>(P->d_retry_acc.p);
    R.cell_bands = static_cast<float *>(P->d_bands.p);
    R.cell_dba = static_cast<float *>(P->d_dba.p);
    R.cell_lden = static_cast<float *>(P->d_lden.p);
    batch_reduce_kernel<<<(unsigned)((P->n_cells + 255) / 256), 256, 0, stream>>>(R);
    QM_CUDA(cudaGetLastError());
    QM_CUDA(cudaEventRecord(ev.e1, stream));
    unsigned long long counters[6];
    QM_CUDA(cudaMemcpyAsync(counters, P->d_counters.p, sizeof(counters), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaStreamSynchronize(stream));
    float ms = 0.f, paint_ms = 0.f;
    QM_CUDA(cudaEventElapsedTime(&ms, ev.e0, ev.e1));
    QM_CUDA(cudaEventElapsedTime(&paint_ms, ev.e0, ev.e2));
    if (stats) {
        stats->paths = counters[0];
        stats->crossings = counters[1];
        stats->edge_tests = counters[2];
        stats->failed_paths = counters[3];
        stats->vertices = counters[4];
        stats->candidates = counters[5];
        stats->kernel_ms = ms;
        stats->paint_ms = paint_ms;
    }
    return QM_OK;
}

qm_status qm_batch_plan_read(qm_batch_plan *P, float *cell_bands, float *cell_dba, float *cell_lden) {
    if (!P) return fail(QM_ERR_ARGUMENT, "qm_batch_plan_read: null plan");
    qm_ctx *ctx = P->scene->ctx;
    std::lock_guard<std::mutex> guard(ctx->lock);
    QM_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t stream = ctx->stream;
    if (cell_bands)
        QM_CUDA(cudaMemcpyAsync(cell_bands, P->d_bands.p, P->n_cells * QM_BANDS * sizeof(float), cudaMemcpyDeviceToHost, stream));
    if (cell_dba) QM_CUDA(cudaMemcpyAsync(cell_dba, P->d_dba.p, P->n_cells * sizeof(float), cudaMemcpyDeviceToHost, stream));
    if (cell_lden) QM_CUDA(cudaMemcpyAsync(cell_lden, P->d_lden.p, P->n_cells * sizeof(float), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaStreamSynchronize(stream));
    return QM_OK;
}

qm_status qm_batch_autotune(qm_scene *scene, const qm_tile_desc *sample, size_t n_sample, qm_tune_table *table,
                            float *timings) {
    NvtxRange nvtx_range("qm_batch_autotune");
    if (!scene || !table || (n_sample && !sample)) return fail(QM_ERR_ARGUMENT, "qm_batch_autotune: null scene, sample or table");
    qm_tune_default(table);
    if (timings)
        for (int k = 0; k < QM_TILE_BUCKETS * QM_TILE_CANDIDATES; ++k) timings[k] = -1.0f;
    for (int b = 0; b < QM_TILE_BUCKETS; ++b) {
        // This bucket's samples, clipped to their first 64 x 64 receivers and 4,096 sources.
        std::vector<qm_tile_desc> tiles;
        uint64_t cells = 0;
        for (size_t k = 0; k < n_sample; ++k) {
            if ((int)qm_tile_bucket(&sample[k]) != b) continue;
            qm_tile_desc d = sample[k];
            d.nx = std::min(d.nx, 64);
            d.ny = std::min(d.ny, 64);
            uint32_t sb = d.source_begin, se = d.source_end;
            if (se <= sb) {
                sb = 0;
                se = scene->n_sources;
            }
            d.source_begin = sb;
            d.source_end = std::min(se, sb + 4096u);
            d.cell_offset = cells;
            cells += (uint64_t)d.nx * d.ny;
            tiles.push_back(d);
        }
        if (tiles.empty()) continue;
        float best = INFINITY;
        for (int k = 0; k < QM_TILE_CANDIDATES; ++k) {
            qm_tune_table t;
            for (int q = 0; q < QM_TILE_BUCKETS; ++q) t.bucket[q] = tile_candidate(k);
            qm_batch_plan *plan = nullptr;
            qm_status st = qm_batch_plan_create(scene, tiles.data(), tiles.size(), cells, &t, 0, &plan);
            if (st != QM_OK) return st;
            qm_paint_stats s1{}, s2{};
            st = qm_batch_plan_run(plan, &s1);
            if (st == QM_OK) st = qm_batch_plan_run(plan, &s2);
            qm_batch_plan_free(plan);
            if (st != QM_OK) return st;
            float ms = (float)s2.paint_ms;
            if (timings) timings[b * QM_TILE_CANDIDATES + k] = ms;
            if (ms < best) {
                best = ms;
                table->bucket[b] = tile_candidate(k);
            }
        }
    }
    return QM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Line-source levels in time (physics/src/percentile.rs). The quantile table is made here by the
// reference's own seeded simulation (physics/src/percentile_tests.rs:1-102): one SplitMix64
// stream over the rows in order, per sample a Poisson count of emitters uniform on the simulated
// length, their intensities 1 / (1 + x^2) summed with the mean of those beyond, over the line's
// mean; each row's samples sorted and read at probabilities (k + 0.5) / 100.

namespace {

struct LineLevelRandom {
    uint64_t state;
    double uniform() {
        state += 0x9e3779b97f4a7c15ull;
        uint64_t z = state;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return (double)((z ^ (z >> 31)) >> 11) / (double)(1ull << 53);
    }
    size_t poisson(double mean) {  // a normal approximation above a mean of 50
        const double pi = 3.14159265358979323846;
        if (mean > 50.0) {
            const double radius = std::sqrt(-2.0 * std::log(1.0 - uniform()));
            const double normal = radius * std::cos(2.0 * pi * uniform());
            return (size_t)std::max(std::round(mean + std::sqrt(mean) * normal), 0.0);
        }
        const double limit = std::exp(-mean);
        size_t count = 0;
        double product = uniform();
        while (product > limit) {
            ++count;
            product *= uniform();
        }
        return count;
    }
};

const std::vector<float> &line_level_table() {
    static const std::vector<float> table = [] {
        const double pi = 3.14159265358979323846;
        std::vector<float> t((size_t)LINE_LEVEL_ROWS * LINE_LEVEL_QUANTILES);
        LineLevelRandom random{0x5eed1971ull};
        std::vector<double> samples;
        for (int row = 0; row < LINE_LEVEL_ROWS; ++row) {
            const double lambda = LINE_LEVEL_LAMBDA_MIN * std::pow(10.0, (double)row / LINE_LEVEL_STEPS_PER_DECADE);
            // At least 200 distances each side and ten emitters on average; 20,000 samples, up to
            // a million for sparse lines whose upper quantiles rest on rare passes.
            const double half_length = std::max(5.0 / lambda, 200.0);
            const size_t count = (size_t)std::min(20000.0 * std::max(0.01 / lambda, 1.0), 1000000.0);
            const double mean_inside = lambda * 2.0 * half_length;
            const double outside = lambda * 2.0 * (pi / 2.0 - std::atan(half_length));
            const double mean = lambda * pi;
            samples.resize(count);
            for (size_t i = 0; i < count; ++i) {
                const size_t emitters = random.poisson(mean_inside);
                double inside = 0.0;
                for (size_t e = 0; e < emitters; ++e) {
                    const double x = (2.0 * random.uniform() - 1.0) * half_length;
                    inside += 1.0 / (1.0 + x * x);
                }
                samples[i] = (inside + outside) / mean;
            }
            std::sort(samples.begin(), samples.end());
            for (int k = 0; k < LINE_LEVEL_QUANTILES; ++k)
                t[(size_t)row * LINE_LEVEL_QUANTILES + k] =
                    (float)samples[(size_t)(((double)k + 0.5) / LINE_LEVEL_QUANTILES * (double)count)];
        }
        return t;
    }();
    return table;
}

}  // namespace

namespace qm {
const std::vector<float> &line_level_table_shared() { return line_level_table(); }
}  // namespace qm

namespace {

// The line-level table on the context's device, uploaded on first use (the context's lock held,
// its device current).
qm_status device_line_table(qm_ctx *ctx) {
    if (ctx->line_table) return QM_OK;
    const std::vector<float> &table = line_level_table();
    QM_CUDA(cudaMalloc(&ctx->line_table, table.size() * sizeof(float)));
    QM_CUDA(cudaMemcpyAsync(ctx->line_table, table.data(), table.size() * sizeof(float), cudaMemcpyHostToDevice,
                            ctx->stream));
    return QM_OK;
}

}  // namespace

extern "C" {

qm_status qm_line_level_table(float *table) {
    if (!table) return fail(QM_ERR_ARGUMENT, "qm_line_level_table: null table");
    const std::vector<float> &t = line_level_table();
    std::memcpy(table, t.data(), t.size() * sizeof(float));
    return QM_OK;
}

qm_status qm_line_level_quantiles(qm_ctx *ctx, const double *lambda, const double *p, size_t n, double *out) {
    NvtxRange nvtx_range("qm_line_level_quantiles");
    if (!ctx) return fail(QM_ERR_ARGUMENT, "qm_line_level_quantiles: null ctx");
    if (n == 0) return QM_OK;
    if (!lambda || !p || !out) return fail(QM_ERR_ARGUMENT, "qm_line_level_quantiles: null lambda, p or out");
    std::lock_guard<std::mutex> guard(ctx->lock);
    QM_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t stream = ctx->stream;
    const qm_status table_status = device_line_table(ctx);
    if (table_status != QM_OK) return table_status;
    Scratch d_lambda, d_p, d_out;
    QM_CUDA(cudaMalloc(&d_lambda.p, n * sizeof(double)));
    QM_CUDA(cudaMalloc(&d_p.p, n * sizeof(double)));
    QM_CUDA(cudaMalloc(&d_out.p, n * sizeof(double)));
    QM_CUDA(cudaMemcpyAsync(d_lambda.p, lambda, n * sizeof(double), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(d_p.p, p, n * sizeof(double), cudaMemcpyHostToDevice, stream));
    const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)ctx->sm_count * 8);
    line_level_kernel<<<blocks, 256, 0, stream>>>(ctx->line_table, static_cast<const double *>(d_lambda.p),
                                                  static_cast<const double *>(d_p.p), n, static_cast<double *>(d_out.p));
    QM_CUDA(cudaGetLastError());
    QM_CUDA(cudaMemcpyAsync(out, d_out.p, n * sizeof(double), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaStreamSynchronize(stream));
    return QM_OK;
}

}  // extern "C"

// =============================================================================================
// Batch::loudness on the device (qm_distribution.h, qm_pixel.cuh).

extern "C" {

qm_status qm_pixel_loudness(qm_ctx *ctx, const float *input, size_t n_floats, const uint64_t *offsets,
                            size_t n_pixels, uint32_t n_layers, double bin_db, const double *shares,
                            size_t n_profiles, const uint32_t *runs, float *ndens, double *kernel_ms) {
    NvtxRange nvtx_range("qm_pixel_loudness");
    using namespace qm::pix;
    if (!ctx) return fail(QM_ERR_ARGUMENT, "qm_pixel_loudness: null ctx");
    if (n_pixels == 0) return QM_OK;
    if (!input || !offsets || !ndens) return fail(QM_ERR_ARGUMENT, "qm_pixel_loudness: null input, offsets or ndens");
    if (n_layers > (uint32_t)MAX_LAYERS)
        return fail(QM_ERR_ARGUMENT, "qm_pixel_loudness: " + std::to_string(n_layers) + " layers, at most " +
                                         std::to_string(MAX_LAYERS));
    if (!(bin_db > 0.0) || !std::isfinite(bin_db))
        return fail(QM_ERR_ARGUMENT, "qm_pixel_loudness: bin_db must be positive and finite");
    const double bins_f = std::round(qm::dist::SPAN_DB / bin_db);
    if (!(bins_f >= 1.0) || bins_f > MAX_BINS)
        return fail(QM_ERR_ARGUMENT, "qm_pixel_loudness: bin_db gives " + std::to_string(bins_f) + " bins, at most " +
                                         std::to_string(MAX_BINS) + " on the device");
    if (n_pixels > 0xFFFFFFFFu) return fail(QM_ERR_ARGUMENT, "qm_pixel_loudness: too many pixels");
    for (size_t k = 0; k < n_pixels; ++k) {
        const uint64_t end = k + 1 < n_pixels ? offsets[k + 1] : n_floats;
        if (offsets[k] > end || end > n_floats)
            return fail(QM_ERR_ARGUMENT, "qm_pixel_loudness: pixel " + std::to_string(k) +
                                             " does not lie within the input before the next pixel");
    }
    // The periods' groups of hours (the caller's hourly shares, as qm_pixel_distributions groups them).
    std::vector<double> factors((size_t)3 * MAX_GROUPS * std::max<size_t>(n_profiles, 1), 1.0);
    std::vector<uint32_t> group_hours(3 * MAX_GROUPS, 0);
    uint32_t n_groups[3] = {0, 0, 0};
    if (n_profiles > 0) {
        if (!shares) return fail(QM_ERR_ARGUMENT, "qm_pixel_loudness: null shares with profiles");
        for (uint32_t p = 0; p < 3; ++p) {
            uint32_t slot_group[12];
            size_t groups = 0;
            const qm_status st = qm_hour_groups(shares, n_profiles, p, runs ? runs[p] : 0, slot_group,
                                                group_hours.data() + p * MAX_GROUPS,
                                                factors.data() + (size_t)p * MAX_GROUPS * n_profiles, &groups);
            if (st != QM_OK) return st;
            n_groups[p] = (uint32_t)groups;
        }
    }
    std::lock_guard<std::mutex> guard(ctx->lock);
    QM_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t stream = ctx->stream;
    qm_status st = device_line_table(ctx);
    if (st != QM_OK) return st;
    const uint32_t L = n_layers;
    Scratch d_in, d_off, d_fac, d_groups, d_nden, d_status;
    QM_CUDA(cudaMalloc(&d_in.p, std::max<size_t>(n_floats, 1) * sizeof(float)));
    QM_CUDA(cudaMalloc(&d_off.p, n_pixels * sizeof(uint64_t)));
    QM_CUDA(cudaMalloc(&d_fac.p, factors.size() * sizeof(double)));
    QM_CUDA(cudaMalloc(&d_groups.p, group_hours.size() * sizeof(uint32_t)));
    QM_CUDA(cudaMalloc(&d_nden.p, n_pixels * (L + 1) * sizeof(float)));
    QM_CUDA(cudaMalloc(&d_status.p, n_pixels * sizeof(uint32_t)));
    if (n_floats) QM_CUDA(cudaMemcpyAsync(d_in.p, input, n_floats * sizeof(float), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(d_off.p, offsets, n_pixels * sizeof(uint64_t), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(d_fac.p, factors.data(), factors.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
    QM_CUDA(cudaMemcpyAsync(d_groups.p, group_hours.data(), group_hours.size() * sizeof(uint32_t),
                            cudaMemcpyHostToDevice, stream));
    Args A{};
    A.input = static_cast<const float *>(d_in.p);
    A.offsets = static_cast<const uint64_t *>(d_off.p);
    A.n_floats = n_floats;
    A.n_pixels = (uint32_t)n_pixels;
    A.n_layers = L;
    A.bin_db = bin_db;
    A.n_bins = (int)bins_f;
    A.table = ctx->line_table;
    A.factors = static_cast<const double *>(d_fac.p);
    A.group_hours = static_cast<const uint32_t *>(d_groups.p);
    for (int p = 0; p < 3; ++p) A.n_groups[p] = n_groups[p];
    A.n_profiles = (uint32_t)n_profiles;
    A.ndens = static_cast<float *>(d_nden.p);
    A.status = static_cast<uint32_t *>(d_status.p);
    const size_t smem = shared_bytes(A.n_bins);
    QM_CUDA(cudaFuncSetAttribute(pixel_loudness_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    Events ev;
    QM_CUDA(ev.create());
    QM_CUDA(cudaEventRecord(ev.e0, stream));
    pixel_loudness_kernel<<<(unsigned)n_pixels, THREADS, smem, stream>>>(A);
    QM_CUDA(cudaGetLastError());
    QM_CUDA(cudaEventRecord(ev.e1, stream));
    std::vector<uint32_t> status(n_pixels);
    QM_CUDA(cudaMemcpyAsync(ndens, d_nden.p, n_pixels * (L + 1) * sizeof(float), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaMemcpyAsync(status.data(), d_status.p, n_pixels * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    QM_CUDA(cudaStreamSynchronize(stream));
    if (kernel_ms) {
        float ms = 0.0f;
        QM_CUDA(cudaEventElapsedTime(&ms, ev.e0, ev.e1));
        *kernel_ms = ms;
    }
    for (size_t k = 0; k < n_pixels; ++k) {
        if (status[k] == 0) continue;
        std::string why = (status[k] & BAD_PACKING) ? "its counts run past its floats or leave floats over"
                          : (status[k] & BAD_PROFILE) ? "a line follows a profile past n_profiles"
                          : (status[k] & BAD_LINE)    ? "a line or steady energy fails the host's checks"
                                                      : "a moving line has more than 256 values";
        return fail(QM_ERR_ARGUMENT, "qm_pixel_loudness: pixel " + std::to_string(k) + ": " + why);
    }
    return QM_OK;
}

}  // extern "C"
