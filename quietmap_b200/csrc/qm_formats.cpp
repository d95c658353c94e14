// The reference's file formats read on the host: `obstacles` tiles into scene outlines,
// `terrain` and `terrain-fine` tiles into their nodes and the ground at a point, and the global
// weather table into a place's weather (include/qm_obstacles.h, include/qm_terrain.h,
// include/qm_weather.h). No device work: these entry points need no context.

#include <dlfcn.h>
#include <sys/types.h>

#include <algorithm>
#include <cerrno>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/qm_obstacles.h"
#include "../../include/qm_terrain.h"
#include "../../include/qm_weather.h"
#include "qm_host.h"

namespace {

qm_status fail(qm_status status, const std::string &message) { return qm::set_error(status, message); }

}  // namespace

// ---------------------------------------------------------------------------------------------
// `obstacles` tiles (qmobs2; tiles/src/obstacles.rs:1-24 gives the layout, parse.rs:23-128 the
// checks, whose order and messages these follow).

namespace {

uint16_t le16(const uint8_t *p) { return (uint16_t)(p[0] | (p[1] << 8)); }
uint32_t le32(const uint8_t *p) {
    return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
uint64_t le64(const uint8_t *p) { return (uint64_t)le32(p) | ((uint64_t)le32(p + 4) << 32); }

// A checked tile: its sections, every index inside them verified.
struct ObstaclesView {
    static constexpr size_t HEADER = 32, CELLS = 128 * 128, WORDS = CELLS / 64;
    static constexpr size_t RUN = 8, OUTLINE = 12, VERTEX = 4, MAX_SQUARES = 256;
    const uint8_t *words, *before, *first_runs, *squares, *runs, *outlines, *vertices;
    size_t occupied, n_squares, n_runs, n_outlines, n_vertices;

    uint64_t word(size_t w) const { return le64(words + 8 * w); }
    size_t first_run(size_t rank) const { return le32(first_runs + 4 * rank); }
    const uint8_t *outline(size_t i) const { return outlines + OUTLINE * i; }
    size_t first_vertex(size_t i) const { return le32(outline(i)); }
    size_t end_vertex(size_t i) const { return i + 1 < n_outlines ? first_vertex(i + 1) : n_vertices; }
    uint64_t footprint_id(const uint8_t *rec) const {
        return ((uint64_t)le32(squares + 4 * (size_t)rec[10]) << 32) | le32(rec + 4);
    }
    uint32_t vertex(size_t k) const { return le32(vertices + VERTEX * k); }  // both int16, packed
};

qm_status obstacles_view(const uint8_t *b, size_t n, ObstaclesView &v) {
    using V = ObstaclesView;
    auto bad = [](const char *message) { return fail(QM_ERR_ARGUMENT, message); };
    if (!b && n) return fail(QM_ERR_ARGUMENT, "obstacles: null bytes");
    if (n < V::HEADER || std::memcmp(b, "qmobs2\n\0", 8) != 0) return bad("obstacles: bad magic");
    const uint64_t outlines = le32(b + 8), vertices = le32(b + 12), runs = le32(b + 16), occupied = le32(b + 20),
                   squares = le32(b + 24);
    if (le32(b + 28) != 0 || occupied > V::CELLS || squares > V::MAX_SQUARES) return bad("obstacles: bad header");
    const uint64_t lengths[7] = {8 * V::WORDS,   2 * V::WORDS,          4 * (occupied + 1),   4 * squares,
                                 V::RUN * runs, V::OUTLINE * outlines, V::VERTEX * vertices};
    uint64_t at[8];
    at[0] = V::HEADER;
    for (int k = 0; k < 7; ++k) at[k + 1] = at[k] + lengths[k];
    if ((uint64_t)n != at[7]) return bad("obstacles: length does not match the counts");
    v.words = b + at[0];
    v.before = b + at[1];
    v.first_runs = b + at[2];
    v.squares = b + at[3];
    v.runs = b + at[4];
    v.outlines = b + at[5];
    v.vertices = b + at[6];
    v.occupied = occupied;
    v.n_squares = squares;
    v.n_runs = runs;
    v.n_outlines = outlines;
    v.n_vertices = vertices;
    size_t before = 0;
    for (size_t w = 0; w < V::WORDS; ++w) {
        if ((size_t)le16(v.before + 2 * w) != before) return bad("obstacles: occupied cells miscounted");
        before += (size_t)__builtin_popcountll(v.word(w));
    }
    bool ordered = before == v.occupied && v.first_run(0) == 0 && v.first_run(v.occupied) == v.n_runs;
    for (size_t r = 0; ordered && r < v.occupied; ++r) ordered = v.first_run(r + 1) > v.first_run(r);
    if (!ordered) return bad("obstacles: cell runs out of order");
    for (size_t r = 1; r < v.n_squares; ++r)
        if (le32(v.squares + 4 * r) <= le32(v.squares + 4 * r - 4)) return bad("obstacles: footprint squares out of order");
    if (v.n_outlines > 0 && v.first_vertex(0) != 0) return bad("obstacles: vertices before the first outline");
    uint64_t previous_id = 0;
    for (size_t i = 0; i < v.n_outlines; ++i) {
        const uint8_t *rec = v.outline(i);
        const int kind = rec[11] & 3, envelope = rec[11] >> 2;
        if (kind > 2 || envelope > 5) return bad("obstacles: unknown outline kind or envelope");
        if (le16(rec + 8) == 0 || (size_t)rec[10] >= v.n_squares) return bad("obstacles: zero height or a missing square");
        const size_t first = v.first_vertex(i), end = v.end_vertex(i);
        const uint64_t id = v.footprint_id(rec);
        if (end < first || end > v.n_vertices || id < previous_id) return bad("obstacles: outline out of range or order");
        const size_t count = end - first;
        const bool well_formed = kind == 2 ? count >= 2 : count >= 4 && v.vertex(first) == v.vertex(end - 1);
        if (!well_formed) return bad("obstacles: open ring or short outline");
        previous_id = id;
    }
    for (size_t r = 0; r < v.n_runs; ++r) {
        const uint8_t *run = v.runs + V::RUN * r;
        const size_t outline = le32(run), first_edge = le16(run + 4), edge_count = le16(run + 6);
        if (outline >= v.n_outlines || edge_count == 0 ||
            first_edge + edge_count >= v.end_vertex(outline) - v.first_vertex(outline))
            return bad("obstacles: run out of range");
    }
    return QM_OK;
}

}  // namespace

extern "C" {

qm_status qm_obstacles_check(const uint8_t *bytes, size_t n_bytes, qm_obstacles_counts *counts) {
    ObstaclesView v;
    qm_status st = obstacles_view(bytes, n_bytes, v);
    if (st != QM_OK) return st;
    if (counts) {
        counts->outlines = (uint32_t)v.n_outlines;
        counts->vertices = (uint32_t)v.n_vertices;
        counts->runs = (uint32_t)v.n_runs;
        counts->occupied_cells = (uint32_t)v.occupied;
        counts->footprint_squares = (uint32_t)v.n_squares;
        counts->pad_ = 0;
    }
    return QM_OK;
}

qm_status qm_obstacles_outlines(const uint8_t *bytes, size_t n_bytes, int32_t offset_x, int32_t offset_y,
                                uint32_t first_vertex_base, qm_outline *outlines, int32_t *vertices_xy,
                                uint8_t *envelope) {
    ObstaclesView v;
    qm_status st = obstacles_view(bytes, n_bytes, v);
    if (st != QM_OK) return st;
    if ((v.n_outlines && !outlines) || (v.n_vertices && !vertices_xy))
        return fail(QM_ERR_ARGUMENT, "qm_obstacles_outlines: null outlines or vertices_xy");
    if ((uint64_t)first_vertex_base + v.n_vertices > UINT32_MAX)
        return fail(QM_ERR_ARGUMENT, "qm_obstacles_outlines: vertex indices beyond 2^32");
    for (size_t k = 0; k < v.n_vertices; ++k) {
        const uint8_t *p = v.vertices + ObstaclesView::VERTEX * k;
        const int64_t x = (int64_t)(int16_t)le16(p) + offset_x, y = (int64_t)(int16_t)le16(p + 2) + offset_y;
        if (x < INT32_MIN || x > INT32_MAX || y < INT32_MIN || y > INT32_MAX)
            return fail(QM_ERR_ARGUMENT, "qm_obstacles_outlines: a vertex leaves the int32 lattice");
        vertices_xy[2 * k] = (int32_t)x;
        vertices_xy[2 * k + 1] = (int32_t)y;
    }
    for (size_t i = 0; i < v.n_outlines; ++i) {
        const uint8_t *rec = v.outline(i);
        qm_outline &o = outlines[i];
        o.first_vertex = first_vertex_base + (uint32_t)v.first_vertex(i);
        o.vertex_count = (uint32_t)(v.end_vertex(i) - v.first_vertex(i));
        o.footprint_id = v.footprint_id(rec);
        o.height_m = (float)((double)le16(rec + 8) / 10.0);
        o.building = (rec[11] & 3) != 2 ? 1u : 0u;
        if (envelope) envelope[i] = rec[11] >> 2;
    }
    return QM_OK;
}

qm_status qm_obstacles_merge(const uint8_t *const *bytes, const size_t *n_bytes, const int32_t *offsets_xy,
                             size_t n_tiles, qm_outline *outlines, uint32_t *n_outlines, int32_t *vertices_xy,
                             uint32_t *n_vertices, uint8_t *envelope) {
    if (!n_outlines || !n_vertices) return fail(QM_ERR_ARGUMENT, "qm_obstacles_merge: null n_outlines or n_vertices");
    if (n_tiles && (!bytes || !n_bytes || !offsets_xy))
        return fail(QM_ERR_ARGUMENT, "qm_obstacles_merge: null bytes, n_bytes or offsets_xy");
    const bool counting = !outlines && !vertices_xy;
    if (!counting && (!outlines || !vertices_xy))
        return fail(QM_ERR_ARGUMENT, "qm_obstacles_merge: outlines and vertices_xy are given together");
    struct Kept {
        uint64_t id;
        uint32_t first, count;
        uint16_t height_dm;
        uint8_t kind, envelope;
    };
    std::vector<Kept> kept;
    std::vector<int32_t> xy;  // the kept outlines' global vertices
    std::unordered_map<uint64_t, std::vector<uint32_t>> by_key;
    std::vector<int32_t> g;
    for (size_t t = 0; t < n_tiles; ++t) {
        ObstaclesView v;
        qm_status st = obstacles_view(bytes[t], n_bytes[t], v);
        if (st != QM_OK) return fail(st, "qm_obstacles_merge: tile " + std::to_string(t) + ": " + qm::last_error());
        for (size_t i = 0; i < v.n_outlines; ++i) {
            const uint8_t *rec = v.outline(i);
            const size_t first = v.first_vertex(i), count = v.end_vertex(i) - first;
            g.resize(2 * count);
            uint64_t key = v.footprint_id(rec) * 0x9E3779B97F4A7C15ull ^ (uint64_t)(rec[11] & 3) ^ ((uint64_t)count << 40);
            for (size_t k = 0; k < count; ++k) {
                const uint8_t *p = v.vertices + ObstaclesView::VERTEX * (first + k);
                const int64_t x = (int64_t)(int16_t)le16(p) + offsets_xy[2 * t];
                const int64_t y = (int64_t)(int16_t)le16(p + 2) + offsets_xy[2 * t + 1];
                if (x < INT32_MIN || x > INT32_MAX || y < INT32_MIN || y > INT32_MAX)
                    return fail(QM_ERR_ARGUMENT, "qm_obstacles_merge: a vertex leaves the int32 lattice");
                g[2 * k] = (int32_t)x;
                g[2 * k + 1] = (int32_t)y;
                key = (key ^ (uint32_t)x) * 0x100000001B3ull;
                key = (key ^ (uint32_t)y) * 0x100000001B3ull;
            }
            const uint64_t id = v.footprint_id(rec);
            const uint8_t kind = rec[11] & 3;
            bool duplicate = false;
            auto &bucket = by_key[key];
            for (uint32_t j : bucket) {
                const Kept &o = kept[j];
                if (o.id == id && o.kind == kind && o.count == count &&
                    std::equal(g.begin(), g.end(), xy.begin() + 2 * (size_t)o.first)) {
                    duplicate = true;
                    break;
                }
            }
            if (duplicate) continue;
            if (xy.size() / 2 + count > UINT32_MAX) return fail(QM_ERR_CAPACITY, "qm_obstacles_merge: more than 2^32 vertices");
            bucket.push_back((uint32_t)kept.size());
            kept.push_back(Kept{id, (uint32_t)(xy.size() / 2), (uint32_t)count, le16(rec + 8), kind, (uint8_t)(rec[11] >> 2)});
            xy.insert(xy.end(), g.begin(), g.end());
        }
    }
    const uint32_t cap_outlines = *n_outlines, cap_vertices = *n_vertices;
    *n_outlines = (uint32_t)kept.size();
    *n_vertices = (uint32_t)(xy.size() / 2);
    if (counting) return QM_OK;
    if (kept.size() > cap_outlines || xy.size() / 2 > cap_vertices)
        return fail(QM_ERR_CAPACITY, "qm_obstacles_merge: outlines or vertices_xy too short (" +
                                         std::to_string(kept.size()) + " outlines, " + std::to_string(xy.size() / 2) +
                                         " vertices)");
    std::copy(xy.begin(), xy.end(), vertices_xy);
    for (size_t j = 0; j < kept.size(); ++j) {
        qm_outline &o = outlines[j];
        o.first_vertex = kept[j].first;
        o.vertex_count = kept[j].count;
        o.footprint_id = kept[j].id;
        o.height_m = (float)((double)kept[j].height_dm / 10.0);
        o.building = kept[j].kind != 2 ? 1u : 0u;
        if (envelope) envelope[j] = kept[j].envelope;
    }
    return QM_OK;
}

qm_status qm_obstacles_cell_runs(const uint8_t *bytes, size_t n_bytes, uint32_t column, uint32_t row, uint32_t *runs,
                                 uint32_t cap, uint32_t *count) {
    ObstaclesView v;
    qm_status st = obstacles_view(bytes, n_bytes, v);
    if (st != QM_OK) return st;
    if (!count || (cap && !runs)) return fail(QM_ERR_ARGUMENT, "qm_obstacles_cell_runs: null count or runs");
    if (column >= QM_OBSTACLES_CELLS_PER_SIDE || row >= QM_OBSTACLES_CELLS_PER_SIDE)
        return fail(QM_ERR_ARGUMENT, "qm_obstacles_cell_runs: cell outside the tile");
    const size_t cell = (size_t)row * QM_OBSTACLES_CELLS_PER_SIDE + column;
    const uint64_t word = v.word(cell / 64);
    const unsigned bit = (unsigned)(cell % 64);
    *count = 0;
    if (!((word >> bit) & 1)) return QM_OK;
    const size_t rank = le16(v.before + 2 * (cell / 64)) + (size_t)__builtin_popcountll(word & ((1ull << bit) - 1));
    const size_t r0 = v.first_run(rank), r1 = v.first_run(rank + 1);
    *count = (uint32_t)(r1 - r0);
    for (size_t r = r0; r < r1 && r - r0 < cap; ++r) {
        const uint8_t *run = v.runs + ObstaclesView::RUN * r;
        runs[3 * (r - r0)] = le32(run);
        runs[3 * (r - r0) + 1] = le16(run + 4);
        runs[3 * (r - r0) + 2] = le16(run + 6);
    }
    return QM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// The global weather table (qmwthr2; physics/src/weather.rs).

namespace {

constexpr size_t WEATHER_NODE = QM_WEATHER_NODE_BYTES;

bool weather_percentages_valid(const uint8_t *node) {  // weather.rs:168-170
    for (int k = 0; k < QM_PERIODS * QM_SECTORS; ++k)
        if (node[k] > 100) return false;
    return true;
}

// The four nodes around a place and their bilinear weights, longitude wrapping (weather.rs:172-187).
void weather_corners(double lat, double lon, size_t index[4], double weight[4]) {
    const double nodes = 2.0;
    const double y = std::min(std::max((90.0 - lat) * nodes, 0.0), (double)(QM_WEATHER_ROWS - 1));
    double wrapped = std::fmod(lon, 360.0);
    if (wrapped < 0.0) wrapped += 360.0;
    const double x = wrapped * nodes;
    const size_t row = std::min((size_t)std::floor(y), (size_t)QM_WEATHER_ROWS - 2), column = (size_t)std::floor(x);
    const double fy = y - (double)row, fx = x - (double)column;
    auto at = [](size_t r, size_t c) { return r * QM_WEATHER_COLUMNS + c % QM_WEATHER_COLUMNS; };
    index[0] = at(row, column);
    weight[0] = (1.0 - fy) * (1.0 - fx);
    index[1] = at(row, column + 1);
    weight[1] = (1.0 - fy) * fx;
    index[2] = at(row + 1, column);
    weight[2] = fy * (1.0 - fx);
    index[3] = at(row + 1, column + 1);
    weight[3] = fy * fx;
}

// A place's weather from its four nodes (weather.rs:189-214): each value the weighted sum in
// corner order, over 100.
void weather_place_of(const uint8_t *const node[4], const double weight[4], double *favourable, double *alpha) {
    for (int k = 0; k < QM_PERIODS * QM_SECTORS; ++k) {
        double sum = 0.0;
        for (int c = 0; c < 4; ++c) sum += weight[c] * (double)node[c][k];
        favourable[k] = sum / 100.0;
    }
    for (int b = 0; b < QM_BANDS; ++b) {
        const size_t at = QM_PERIODS * QM_SECTORS + 2 * b;
        double sum = 0.0;
        for (int c = 0; c < 4; ++c) sum += weight[c] * (double)le16(node[c] + at);
        alpha[b] = sum / 100.0;
    }
}

}  // namespace

extern "C" {

qm_status qm_weather_place(const uint8_t *table, size_t n_bytes, double lat, double lon, double *favourable,
                           double *alpha_db_per_km) {
    if (!favourable || !alpha_db_per_km) return fail(QM_ERR_ARGUMENT, "qm_weather_place: null outputs");
    if (!table || n_bytes != (size_t)QM_WEATHER_TABLE_BYTES || std::memcmp(table, "qmwthr2\n", 8) != 0)
        return fail(QM_ERR_ARGUMENT, "weather table: bad magic or length");
    const uint8_t *nodes = table + 8;
    for (size_t k = 0; k < (size_t)QM_WEATHER_ROWS * QM_WEATHER_COLUMNS; ++k)
        if (!weather_percentages_valid(nodes + k * WEATHER_NODE))
            return fail(QM_ERR_ARGUMENT, "weather table: a percentage above 100");
    if (!std::isfinite(lat) || !std::isfinite(lon)) return fail(QM_ERR_ARGUMENT, "qm_weather_place: lat and lon finite");
    size_t index[4];
    double weight[4];
    weather_corners(lat, lon, index, weight);
    const uint8_t *node[4];
    for (int c = 0; c < 4; ++c) node[c] = nodes + index[c] * WEATHER_NODE;
    weather_place_of(node, weight, favourable, alpha_db_per_km);
    return QM_OK;
}

qm_status qm_weather_read_place(const char *path, double lat, double lon, double *favourable,
                                double *alpha_db_per_km) {
    if (!path || !favourable || !alpha_db_per_km) return fail(QM_ERR_ARGUMENT, "qm_weather_read_place: null argument");
    if (!std::isfinite(lat) || !std::isfinite(lon))
        return fail(QM_ERR_ARGUMENT, "qm_weather_read_place: lat and lon finite");
    const std::string name(path);
    std::FILE *f = std::fopen(path, "rb");
    if (!f) return fail(QM_ERR_ARGUMENT, name + ": " + std::strerror(errno));
    std::unique_ptr<std::FILE, int (*)(std::FILE *)> hold(f, std::fclose);
    if (fseeko(f, 0, SEEK_END) != 0) return fail(QM_ERR_ARGUMENT, name + ": " + std::strerror(errno));
    const off_t length = ftello(f);
    uint8_t magic[8];
    auto read_at = [&](void *dst, size_t bytes, off_t at) {
        return fseeko(f, at, SEEK_SET) == 0 && std::fread(dst, 1, bytes, f) == bytes;
    };
    if (length != (off_t)QM_WEATHER_TABLE_BYTES || !read_at(magic, 8, 0) || std::memcmp(magic, "qmwthr2\n", 8) != 0)
        return fail(QM_ERR_ARGUMENT, name + ": weather table: bad magic or length");
    size_t index[4];
    double weight[4];
    weather_corners(lat, lon, index, weight);
    uint8_t bytes[4][WEATHER_NODE];
    const uint8_t *node[4];
    for (int c = 0; c < 4; ++c) {
        if (!read_at(bytes[c], WEATHER_NODE, (off_t)(8 + index[c] * WEATHER_NODE)))
            return fail(QM_ERR_ARGUMENT, name + ": short read");
        if (!weather_percentages_valid(bytes[c]))
            return fail(QM_ERR_ARGUMENT, name + ": weather table: a percentage above 100");
        node[c] = bytes[c];
    }
    weather_place_of(node, weight, favourable, alpha_db_per_km);
    return QM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// `terrain` tiles (qmterr2; tiles/src/terrain.rs).

namespace {

// The two functions of zstd's public C API the decoder needs, from the system's libzstd.
struct Zstd {
    size_t (*decompress)(void *dst, size_t capacity, const void *src, size_t size) = nullptr;
    unsigned (*is_error)(size_t code) = nullptr;
    bool loaded() const { return decompress && is_error; }
};

const Zstd &zstd() {
    static const Zstd z = [] {
        Zstd out;
        void *h = dlopen("libzstd.so.1", RTLD_NOW | RTLD_LOCAL);
        if (!h) return out;
        out.decompress = reinterpret_cast<size_t (*)(void *, size_t, const void *, size_t)>(dlsym(h, "ZSTD_decompress"));
        out.is_error = reinterpret_cast<unsigned (*)(size_t)>(dlsym(h, "ZSTD_isError"));
        return out;
    }();
    return z;
}

}  // namespace

extern "C" {

qm_status qm_terrain_decode(const uint8_t *bytes, size_t n_bytes, qm_terrain_window *window, uint16_t *height_codes,
                            uint8_t *impervious, uint8_t *forest, uint8_t *canopy) {
    constexpr size_t HEADER = 24, PLANES = 5;
    if (!window) return fail(QM_ERR_ARGUMENT, "qm_terrain_decode: null window");
    if (!bytes || n_bytes < HEADER || std::memcmp(bytes, "qmterr2\n", 8) != 0)
        return fail(QM_ERR_ARGUMENT, "terrain: bad magic");
    qm_terrain_window w;
    w.north_node = (int32_t)le32(bytes + 8);
    w.west_node = (int32_t)le32(bytes + 12);
    w.rows = le32(bytes + 16);
    w.columns = le32(bytes + 20);
    if (w.rows < 1 || w.rows > QM_TERRAIN_MAX_WINDOW_NODES || w.columns < 1 || w.columns > QM_TERRAIN_MAX_WINDOW_NODES)
        return fail(QM_ERR_ARGUMENT, "terrain: a window no tile has");
    *window = w;
    if (!height_codes) return QM_OK;
    const Zstd &z = zstd();
    if (!z.loaded()) return fail(QM_ERR_UNSUPPORTED, "qm_terrain_decode: libzstd.so.1 is not available");
    const size_t n = (size_t)w.rows * w.columns, columns = w.columns;
    std::vector<uint8_t> planes(PLANES * n);
    const size_t got = z.decompress(planes.data(), planes.size(), bytes + HEADER, n_bytes - HEADER);
    if (z.is_error(got)) return fail(QM_ERR_ARGUMENT, "terrain: the frame does not decode");
    if (got != PLANES * n) return fail(QM_ERR_ARGUMENT, "terrain: the frame does not match the window");
    // The planar prediction undone row by row (terrain.rs:157-180): code = residual + west + north
    // - north-west in the u16 ring, the residual zigzag-decoded from its two byte planes.
    const uint8_t *low = planes.data(), *high = low + n;
    std::vector<uint16_t> north_row(columns, 0);
    for (size_t r = 0; r < w.rows; ++r) {
        uint16_t west = 0, north_west = 0;
        for (size_t c = 0; c < columns; ++c) {
            const size_t at = r * columns + c;
            const uint16_t zigzag = (uint16_t)(low[at] | (high[at] << 8));
            const uint16_t residual = (uint16_t)((uint16_t)(zigzag >> 1) ^ (uint16_t)(-(int)(zigzag & 1)));
            const uint16_t code = (uint16_t)(residual + (uint16_t)(west + north_row[c] - north_west));
            north_west = north_row[c];
            north_row[c] = code;
            west = code;
            height_codes[at] = code;
        }
    }
    if (impervious) std::memcpy(impervious, planes.data() + 2 * n, n);
    if (forest) std::memcpy(forest, planes.data() + 3 * n, n);
    if (canopy) std::memcpy(canopy, planes.data() + 4 * n, n);
    return QM_OK;
}

void qm_mercator_from_degrees(double lat_deg, double lon_deg, double *x, double *y) {
    const double pi = 3.14159265358979323846, n = 4096.0, max_lat = 85.05112877980659;
    double lon = std::fmod(lon_deg + 180.0, 360.0);
    if (lon < 0.0) lon += 360.0;
    lon -= 180.0;
    const double phi = std::min(std::max(lat_deg, -max_lat), max_lat) * (pi / 180.0);
    if (x) *x = (lon + 180.0) / 360.0 * n;
    if (y) *y = (1.0 - std::asinh(std::tan(phi)) / pi) / 2.0 * n;
}

qm_status qm_terrain_window_of_tile(uint32_t tile_x, uint32_t tile_y, qm_terrain_window *window) {
    if (!window) return fail(QM_ERR_ARGUMENT, "qm_terrain_window_of_tile: null window");
    if (tile_x >= 4096 || tile_y >= 4096) return fail(QM_ERR_ARGUMENT, "qm_terrain_window_of_tile: tile outside z12");
    const int64_t axis = 4096, longitude_nodes = 360 * 3600;
    // Longitude edges have denominator 4096: exact integer floor and ceiling.
    const int64_t west = (int64_t)tile_x * longitude_nodes / axis - longitude_nodes / 2;
    const int64_t east = (((int64_t)tile_x + 1) * longitude_nodes + axis - 1) / axis - longitude_nodes / 2;
    const double pi = 3.14159265358979323846;
    auto edge_latitude_nodes = [&](uint32_t y) {
        const double mercator = pi * (1.0 - 2.0 * (double)y / 4096.0);
        return std::atan(std::sinh(mercator)) * (180.0 / pi) * 3600.0;
    };
    const int32_t north = (int32_t)std::ceil(edge_latitude_nodes(tile_y));
    const int32_t south = (int32_t)std::floor(edge_latitude_nodes(tile_y + 1));
    window->north_node = north;
    window->west_node = (int32_t)west;
    window->rows = (uint32_t)(north - south + 1);
    window->columns = (uint32_t)(east - west + 1);
    return QM_OK;
}

double qm_terrain_column_of(const qm_terrain_window *window, double mercator_x) {
    const double world = 360.0 * 3600.0;
    const double column = mercator_x * world / 4096.0 - world / 2.0 - (double)window->west_node;
    double wrapped = std::fmod(column + world / 2.0, world);
    if (wrapped < 0.0) wrapped += world;
    return wrapped - world / 2.0;
}

qm_status qm_terrain_sample(const qm_terrain_window *window, const uint16_t *height_codes, const uint8_t *impervious,
                            const uint8_t *forest, const uint8_t *canopy, const double *mercator_xy, size_t n,
                            qm_ground_sample *out, uint8_t *found) {
    if (!window || (n && (!height_codes || !impervious || !forest || !canopy || !mercator_xy || !out || !found)))
        return fail(QM_ERR_ARGUMENT, "qm_terrain_sample: null argument");
    const qm_terrain_window w = *window;
    if (w.rows < 1 || w.columns < 1) return fail(QM_ERR_ARGUMENT, "qm_terrain_sample: empty window");
    // Web Mercator y of every node row (terrain.rs:261-267).
    std::vector<double> rows(w.rows);
    for (uint32_t r = 0; r < w.rows; ++r)
        qm_mercator_from_degrees((double)(w.north_node - (int32_t)r) / 3600.0, 0.0, nullptr, &rows[r]);
    const double spacing = (rows[w.rows - 1] - rows[0]) / (double)std::max<uint32_t>(w.rows - 1, 1);
    for (size_t k = 0; k < n; ++k) {
        found[k] = 0;
        const double px = mercator_xy[2 * k], py = mercator_xy[2 * k + 1];
        // locate (terrain.rs:289-331)
        double column_position = qm_terrain_column_of(&w, px);
        if (column_position > -1e-6) column_position = std::max(column_position, 0.0);
        const double column = std::floor(column_position), cf = column_position - column;
        const double guess = std::floor((py - rows[0]) / spacing);
        int64_t row = std::isfinite(guess) ? (int64_t)std::min(std::max(guess, 0.0), (double)(w.rows - 1)) : 0;
        while (row > 0 && py < rows[row]) --row;
        while (row + 1 < (int64_t)w.rows && py >= rows[row + 1]) ++row;
        if (py < rows[0] - 1e-9 || column < 0.0) continue;
        const double rf = row + 1 < (int64_t)w.rows ? (py - rows[row]) / (rows[row + 1] - rows[row]) : 0.0;
        const uint64_t r0 = (uint64_t)row, c0 = column >= 4294967295.0 ? 4294967295ull : (uint64_t)column;
        const uint64_t r1 = r0 + (rf > 0.0 ? 1 : 0), c1 = c0 + (cf > 0.0 ? 1 : 0);
        if (r1 >= w.rows || c1 >= w.columns) continue;
        // sample_at (terrain.rs:339-387)
        const size_t at[4] = {(size_t)(r0 * w.columns + c0), (size_t)(r0 * w.columns + c1), (size_t)(r1 * w.columns + c0),
                              (size_t)(r1 * w.columns + c1)};
        const size_t nearest = at[(rf >= 0.5 ? 2 : 0) + (cf >= 0.5 ? 1 : 0)];
        bool missing = forest[nearest] > 100;
        for (size_t c : at) missing = missing || height_codes[c] == QM_TERRAIN_HEIGHT_MISSING || impervious[c] > 100;
        if (missing) continue;
        const double weight[4] = {(1.0 - rf) * (1.0 - cf), (1.0 - rf) * cf, rf * (1.0 - cf), rf * cf};
        double height = 0.0, imp = 0.0;
        for (int c = 0; c < 4; ++c) {
            height += weight[c] * (-500.0 + (double)height_codes[at[c]] / 5.0);
            imp += weight[c] * (double)impervious[at[c]];
        }
        out[k].height_m = height;
        out[k].ground_factor = 1.0 - imp / 100.0;
        out[k].forest_cover = (double)forest[nearest] / 100.0;
        out[k].canopy_m = (double)canopy[nearest];
        found[k] = 1;
    }
    return QM_OK;
}

qm_status qm_terrain_fine_decode(const uint8_t *bytes, size_t n_bytes, qm_terrain_window *window, int16_t *details) {
    constexpr size_t HEADER = 24;
    constexpr uint32_t BLOCK = 128, FINE = 6;
    if (!window) return fail(QM_ERR_ARGUMENT, "qm_terrain_fine_decode: null window");
    if (!bytes || n_bytes < HEADER || std::memcmp(bytes, "qmtfin2\n", 8) != 0)
        return fail(QM_ERR_ARGUMENT, "terrain-fine: bad magic");
    qm_terrain_window w;
    w.north_node = (int32_t)le32(bytes + 8);
    w.west_node = (int32_t)le32(bytes + 12);
    w.rows = le32(bytes + 16);
    w.columns = le32(bytes + 20);
    const uint32_t most = (QM_TERRAIN_MAX_WINDOW_NODES - 1) * FINE + 1;
    if (w.rows < 2 || w.rows > most || w.columns < 2 || w.columns > most)
        return fail(QM_ERR_ARGUMENT, "terrain-fine: a window no tile has");
    // Blocks along an axis of `nodes` nodes, and the first and last node block b stores
    // (terrain_fine.rs:47-56).
    auto blocks_along = [](uint32_t nodes) { return std::max<uint32_t>((nodes - 1 + BLOCK - 1) / BLOCK, 1); };
    const uint32_t down = blocks_along(w.rows), across = blocks_along(w.columns);
    const size_t count = (size_t)down * across, first = HEADER + 4 * count;
    if (n_bytes < first) return fail(QM_ERR_ARGUMENT, "terrain-fine: the directory is cut");
    std::vector<std::pair<size_t, size_t>> frames(count);
    size_t start = first;
    for (size_t b = 0; b < count; ++b) {
        const size_t end = first + le32(bytes + HEADER + 4 * b);
        if (end < start || end > n_bytes) return fail(QM_ERR_ARGUMENT, "terrain-fine: a frame outside the tile");
        frames[b] = {start, end};
        start = end;
    }
    *window = w;
    if (!details) return QM_OK;
    const Zstd &z = zstd();
    if (!z.loaded()) return fail(QM_ERR_UNSUPPORTED, "qm_terrain_fine_decode: libzstd.so.1 is not available");
    std::vector<uint8_t> planes;
    std::vector<uint16_t> north_row;
    // Blocks in row-major order, so a node two blocks share is the later block's, the block the
    // reference reads it from (terrain_fine.rs:150-155).
    for (uint32_t br = 0; br < down; ++br) {
        const uint32_t r0 = br * BLOCK, r1 = std::min(r0 + BLOCK, w.rows - 1);
        for (uint32_t bc = 0; bc < across; ++bc) {
            const uint32_t c0 = bc * BLOCK, c1 = std::min(c0 + BLOCK, w.columns - 1);
            const size_t rows = r1 - r0 + 1, columns = c1 - c0 + 1, nodes = rows * columns;
            const auto &f = frames[(size_t)br * across + bc];
            planes.resize(2 * nodes);
            const size_t got = z.decompress(planes.data(), planes.size(), bytes + f.first, f.second - f.first);
            if (z.is_error(got) || got != 2 * nodes) return fail(QM_ERR_ARGUMENT, "terrain-fine: a block does not decode");
            const uint8_t *low = planes.data(), *high = low + nodes;
            north_row.assign(columns, 0);
            for (size_t r = 0; r < rows; ++r) {
                uint16_t west = 0, north_west = 0;
                for (size_t c = 0; c < columns; ++c) {
                    const size_t at = r * columns + c;
                    const uint16_t zigzag = (uint16_t)(low[at] | (high[at] << 8));
                    const uint16_t residual = (uint16_t)((uint16_t)(zigzag >> 1) ^ (uint16_t)(-(int)(zigzag & 1)));
                    const uint16_t code = (uint16_t)(residual + (uint16_t)(west + north_row[c] - north_west));
                    north_west = north_row[c];
                    north_row[c] = code;
                    west = code;
                    details[(size_t)(r0 + r) * w.columns + c0 + c] = (int16_t)code;
                }
            }
        }
    }
    return QM_OK;
}

}  // extern "C"
