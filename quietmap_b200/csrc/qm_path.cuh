// One receiver-source path on the device: the obstacle crossings (exact integer walk), the
// vertical path's tops and roofs, a streamed walk of the ground profile that sums segment moments
// and builds each state's rubber band as it goes, and the CNOSSOS boundary per state.
//
// Follows, in order: popup/src/obstacles/crossings.rs:13-226 (crossings), physics/src/ray.rs:125-404
// (ray_terms, PathBuffers::fill, crests_of, clip_roofs_in_closing_order), physics/src/cnossos/
// {mod.rs:123-176, rubber_band.rs:373-444, diffraction.rs:64-197} (state boundaries),
// popup/src/evaluate.rs:171-214 (a point source's ray and divergence).
#pragma once

#include <climits>

#include "qm_physics.cuh"
#include "qm_stage.cuh"

namespace qm {

// Pair failure bits (paint-gpu/kernels/common.cuh:27-31), plus a timeout bit.
constexpr uint32_t FAILED_NOT_READ = 1u;
constexpr uint32_t FAILED_NO_TERRAIN = 2u;
constexpr uint32_t FAILED_CAPACITY = 4u;
constexpr uint32_t FAILED_LINE_CUTOFF = 8u;
constexpr uint32_t FAILED_TIMEOUT = 16u;

struct OutlineDev {
    uint32_t first, count, fp, building;
    float height;
    uint32_t pad[3];
};

// A point source as the kernels read it: 128 bytes.
struct SourceDev {
    int32_t x, y;
    float height, gf, excl, platform;
    uint32_t fp, layer;
    float energy[QM_PERIODS * QM_BANDS];
};
static_assert(sizeof(SourceDev) == 128, "SourceDev layout");

struct SceneDev {
    float step_m;
    int cell_steps, cells_x, cells_y;
    const uint2 *cell_range;     // [cells_y][cells_x]: each cell's first entry and one past its last
    const int4 *cell_seg;        // per entry: the edge's ends (ax, ay, bx, by)
    const uint2 *cell_ref;       // per entry: (edge start vertex, outline)
    // The same entries column by column ([cells_x][cells_y]), so that a column's cells are one
    // contiguous run of entries: what a warp sweeping along x stages with one bulk copy.
    const uint2 *col_range;
    const int4 *col_seg;
    const uint2 *col_ref;
    const int2 *vertices;
    const OutlineDev *outlines;
    int dem_nx, dem_ny, dem_ox, dem_oy, dem_sp;
    const float2 *dem;  // (altitude, ground factor) per node, [ny][nx]
    float flat_z, flat_g;
    const SourceDev *sources;
    uint32_t n_sources;
    float fav[QM_PERIODS][QM_SECTORS];
    float alpha[QM_BANDS];
    float air_per_m[QM_BANDS];  // alpha * ln(10) / 10 / 1000: the air's exponent per metre of slant
};

__device__ __forceinline__ int floor_div(int a, int b) {
    int q = a / b;
    return (a % b != 0 && ((a < 0) != (b < 0))) ? q - 1 : q;
}
__device__ __forceinline__ long long floor_div64(long long a, long long b) {
    long long q = a / b;
    return (a % b != 0 && ((a < 0) != (b < 0))) ? q - 1 : q;
}

// ---------------------------------------------------------------------------------------------
// Crossings

// One crossing: chainage, crossed edge (its first vertex), the outline index with flags (bit 30
// building, bit 31 bounds_roof), and the outline's height and dense footprint, copied from the
// outline when the crossing is listed so that the path's later steps read no outline records.
struct XRec {
    double t;
    uint32_t edge;
    uint32_t info;
    float height;
    uint32_t fp;
};
constexpr uint32_t X_OUTLINE = 0x3fffffffu, X_BUILDING = 0x40000000u, X_BOUNDS = 0x80000000u;

__device__ __forceinline__ uint32_t xrec_fp(const SceneDev &, const XRec &r) { return r.fp; }

__device__ __forceinline__ int sgn64(long long v) { return (v > 0) - (v < 0); }

// 32 x 32 -> 64-bit product (one wide multiply): lattice coordinates and their differences fit in
// 32 bits (scenes are limited to 2^27 steps).
__device__ __forceinline__ long long mulw(int a, int b) { return (long long)a * (long long)b; }

// Whether an edge hit enters or leaves its ring (crossings.rs:80-111); exact on lattice points.
__device__ __noinline__ bool edge_bounds_roof(const SceneDev &S, long long sx, long long sy, long long dx, long long dy,
                                        uint32_t edge, uint32_t first, uint32_t count) {
    auto side = [&](uint32_t index) {
        int2 v = S.vertices[index];
        return mulw((int)dx, v.y - (int)sy) - mulw((int)dy, v.x - (int)sx);
    };
    long long a = side(edge), b = side(edge + 1);
    if (a != 0 && b != 0) return true;
    uint32_t distinct = count - 1;
    uint32_t vertex = ((a == 0 ? edge : edge + 1) - first) % distinct;
    int n0 = 0, n1 = 0;
    for (uint32_t offset = 1; offset < distinct; ++offset) {
        if (n0 == 0) n0 = sgn64(side(first + (vertex + distinct - offset) % distinct));
        if (n1 == 0) n1 = sgn64(side(first + (vertex + offset) % distinct));
        if (n0 != 0 && n1 != 0) break;
    }
    return n0 * n1 < 0;
}

// A lane's listed crossings sorted by (t, footprint, edge), deduplicated as the reference does
// (crossings.rs:34-56) and without the receiver's own walls; returns the count kept.
__device__ __forceinline__ int finish_crossings(const SceneDev &S, XRec *xs, int n, uint32_t rcv_own) {
    // The walk's cells come in order, so the list is nearly sorted; an edge listed in several cells
    // appears once per visited cell, its copies side by side after.
    for (int i = 1; i < n; ++i) {
        XRec v = xs[i];
        int j = i - 1;
        while (j >= 0) {
            const XRec &u = xs[j];
            bool after = u.t > v.t;
            if (!after && u.t == v.t) {
                uint32_t fu = xrec_fp(S, u), fv = xrec_fp(S, v);
                after = fu > fv || (fu == fv && u.edge > v.edge);
            }
            if (!after) break;
            xs[j + 1] = u;
            --j;
        }
        xs[j + 1] = v;
    }
    // One crossing per footprint and chainage within 1e-9 (crossings.rs:39-55); copies of one edge
    // (equal t and edge) are the common case of it.
    int kept = 0;
    for (int i = 0; i < n; ++i) {
        XRec c = xs[i];
        if (kept > 0 && xs[kept - 1].edge == c.edge && xs[kept - 1].t == c.t) continue;
        bool merged = false;
        if (kept > 0 && c.t - xs[kept - 1].t < 1e-9) {
            uint32_t fc = xrec_fp(S, c);
            for (int k = kept - 1; k >= 0; --k) {
                if (!(c.t - xs[k].t < 1e-9)) break;
                if (xrec_fp(S, xs[k]) == fc) {
                    xs[k].info |= (c.info & X_BOUNDS);
                    merged = true;
                    break;
                }
            }
        }
        if (!merged) xs[kept++] = c;
    }
    // The receiver's own walls (popup/src/evaluate.rs:293-297).
    if (rcv_own != 0) {
        int m = 0;
        for (int i = 0; i < kept; ++i)
            if (xrec_fp(S, xs[i]) != rcv_own) xs[m++] = xs[i];
        kept = m;
    }
    return kept;
}

// Every crossing of the segment (sx, sy) -> (rx, ry) with an obstacle edge, sorted by (t, footprint)
// and deduplicated as the reference does (crossings.rs:34-56), without the receiver's own walls.
// The walk visits the cells the segment passes (exact integer decisions); an edge meets the segment
// when the exact integer cross products say so, and t is rounded once from the exact quotient, so t
// and the list are those of the reference's f64 test (its products of lattice integers are exact).
template <int MAXC>
__device__ int list_crossings(const SceneDev &S, int sx, int sy, int rx, int ry, uint32_t rcv_own, XRec *xs,
                              uint32_t &status, uint32_t &edges_tested) {
    int n = 0;
    const int idx = rx - sx, idy = ry - sy;
    long long dx = idx, dy = idy;
    const int C = S.cell_steps;
    int cx = floor_div(sx, C), cy = floor_div(sy, C);
    const int lx = floor_div(rx, C), ly = floor_div(ry, C);
    const int stx = dx >= 0 ? 1 : -1, sty = dy >= 0 ? 1 : -1;
    long long bx = (long long)(cx + (dx >= 0 ? 1 : 0)) * C;  // next vertical boundary ahead
    long long by = (long long)(cy + (dy >= 0 ? 1 : 0)) * C;
    const long long adx = dx >= 0 ? dx : -dx, ady = dy >= 0 ? dy : -dy;
    const int minx = min(sx, rx), maxx = max(sx, rx), miny = min(sy, ry), maxy = max(sy, ry);
    int guard = abs(lx - cx) + abs(ly - cy) + 2;
    // The walk is software-pipelined: the next cell is found and its entry range requested before
    // the current cell's entries are tested, so the range's load overlaps the tests.
    auto range_of = [&](int x, int y) {
        return (x >= 0 && y >= 0 && x < S.cells_x && y < S.cells_y) ? __ldg(S.cell_range + y * S.cells_x + x)
                                                                    : make_uint2(0u, 0u);
    };
    uint2 range = range_of(cx, cy);
    for (; guard > 0; --guard) {
        const bool last = cx == lx && cy == ly;
        int ncx = cx, ncy = cy;
        if (!last) {
            int axis;
            if (cx == lx)
                axis = 1;
            else if (cy == ly)
                axis = 0;
            else {
                int ax_ = (int)(bx - sx), ay_ = (int)(by - sy);
                if (ax_ < 0) ax_ = -ax_;
                if (ay_ < 0) ay_ = -ay_;
                axis = (mulw(ax_, (int)ady) < mulw(ay_, (int)adx)) ? 0 : 1;  // a tie steps the row
            }
            if (axis == 0) {
                ncx += stx;
                bx += (long long)stx * C;
            } else {
                ncy += sty;
                by += (long long)sty * C;
            }
        }
        const uint2 next_range = last ? make_uint2(0u, 0u) : range_of(ncx, ncy);
        for (uint32_t k = range.x; k < range.y; ++k) {
            int4 seg = __ldg(S.cell_seg + k);
            if (max(seg.x, seg.z) < minx || min(seg.x, seg.z) > maxx || max(seg.y, seg.w) < miny ||
                min(seg.y, seg.w) > maxy)
                continue;
            ++edges_tested;
            const int ex = seg.z - seg.x, ey = seg.w - seg.y;
            long long den = mulw(idx, ey) - mulw(idy, ex);
            if (den == 0) continue;
            const int wx = seg.x - sx, wy = seg.y - sy;
            long long tn = mulw(wx, ey) - mulw(wy, ex);
            long long un = mulw(wx, idy) - mulw(wy, idx);
            long long d = den;
            if (d < 0) {
                d = -d;
                tn = -tn;
                un = -un;
            }
            if (!(tn > 0 && tn < d && un >= 0 && un <= d)) continue;
            if (n >= MAXC) {
                status |= FAILED_CAPACITY;
                return n;
            }
            uint2 ref = __ldg(S.cell_ref + k);
            OutlineDev o = S.outlines[ref.y];
            bool building = o.building != 0;
            // The segment's side of the edge's ends is -un and den - un: when the segment passes
            // through neither end the hit bounds the roof (edge_bounds_roof's first case), so
            // the ring is walked only for hits through a vertex.
            bool bounds = building && ((un != 0 && un != d) || edge_bounds_roof(S, sx, sy, dx, dy, ref.x, o.first, o.count));
            xs[n++] = XRec{(double)tn / (double)d, ref.x, ref.y | (building ? X_BUILDING : 0u) | (bounds ? X_BOUNDS : 0u),
                           o.height, o.fp};
        }
        if (last) break;
        cx = ncx;
        cy = ncy;
        range = next_range;
    }
    return finish_crossings(S, xs, n, rcv_own);
}

// ---------------------------------------------------------------------------------------------
// Crossings of a warp's rays, found together

// Entries staged per buffer; each warp has two buffers (2 KB) in shared memory.
constexpr int STAGE_ENTRIES = 64;

struct __align__(16) CrossStage {
    int4 seg[2][STAGE_ENTRIES];
    uint64_t bar[2];
};

// The staging state a warp carries from one source to the next: the parity each buffer's barrier
// waits for next, and whether a copy ever failed to land (the warp then stages nothing more).
struct StageState {
    unsigned phases;
    bool dead;
};

__device__ __forceinline__ void stage_init(CrossStage &st) {
    if ((threadIdx.x & 31) == 0) {
        mbar_init(&st.bar[0], 1);
        mbar_init(&st.bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
}

__device__ __forceinline__ int warp_min_i(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ int warp_max_i(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// The crossings of each lane's segment (sx, sy) -> (rx, ry) (`ray` false: none), listed as
// list_crossings lists them, by the whole warp at once. Every lane must call it, with warp-uniform
// staging state. The rays of a warp run from one source to nearby receivers and so meet nearly the
// same obstacle cells. The warp sweeps the union of their cells a column at a time along the
// leading lane's main axis: each lane finds the cell rows its own segment touches in the column
// (with a margin, so the union never misses a cell), the warp takes their span, and the span's
// entries, contiguous in the column-ordered (or, sweeping along y, the row-ordered) copy of the cell
// lists, arrive in shared memory by one bulk copy per piece of at most STAGE_ENTRIES, the next piece's
// copy in flight while the current one is tested. Each lane tests every staged entry against its own
// segment by the exact integer test. An edge a segment crosses is listed in the cell holding the
// crossing point, which lies in the span, so each lane finds every crossing it would find alone
// (some more than once, as the lone walk does for an edge listed in several cells), and
// finish_crossings then yields the same list.
template <int MAXC>
__device__ int warp_list_crossings(const SceneDev &S, CrossStage &st, StageState &ss, int sx, int sy, int rx, int ry,
                                   bool ray, uint32_t rcv_own, XRec *xs, uint32_t &status, uint32_t &edges_tested) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    ray = ray && (rx != sx || ry != sy);
    const unsigned rays = __ballot_sync(FULL, ray);
    if (rays == 0) return 0;
    if (ss.dead) {
        status |= FAILED_TIMEOUT;
        return 0;
    }
    const int leader = __ffs(rays) - 1;
    const int ldx = __shfl_sync(FULL, rx - sx, leader), ldy = __shfl_sync(FULL, ry - sy, leader);
    const bool xmajor = abs(ldx) >= abs(ldy);
    const int su = xmajor ? sx : sy, sv = xmajor ? sy : sx, ru = xmajor ? rx : ry, rv = xmajor ? ry : rx;
    const int C = S.cell_steps;
    const int cells_u = xmajor ? S.cells_x : S.cells_y, cells_v = xmajor ? S.cells_y : S.cells_x;
    const int dir = (xmajor ? ldx : ldy) >= 0 ? 1 : -1;
    const int u_lo = ray ? min(su, ru) : INT_MAX, u_hi = ray ? max(su, ru) : INT_MIN;
    int cu = max(floor_div(warp_min_i(u_lo), C), 0), cu_end = min(floor_div(warp_max_i(u_hi), C), cells_u - 1);
    if (dir < 0) {
        const int t = cu;
        cu = cu_end;
        cu_end = t;
    }
    bool columns_left = dir > 0 ? cu <= cu_end : cu >= cu_end;
    const uint2 *ranges = xmajor ? S.col_range : S.cell_range;
    const int4 *segs = xmajor ? S.col_seg : S.cell_seg;
    const uint2 *refs = xmajor ? S.col_ref : S.cell_ref;
    const double slope = (ray && ru != su) ? (double)(rv - sv) / (double)(ru - su) : 0.0;
    const double inv_c = 1.0 / (double)C;
    const int minx = min(sx, rx), maxx = max(sx, rx), miny = min(sy, ry), maxy = max(sy, ry);
    const int idx = rx - sx, idy = ry - sy;
    const long long dx = idx, dy = idy;
    uint32_t cb = 0, ce = 0;  // entries of the current column not yet staged
    // The next piece of entries in sweep order; warp-uniform.
    auto next_piece = [&](uint32_t &start, uint32_t &count) -> bool {
        while (cb == ce) {
            if (!columns_left) return false;
            int vlo = INT_MAX, vhi = INT_MIN;
            if (ray) {
                const long long x0 = max((long long)cu * C, (long long)u_lo), x1 = min((long long)(cu + 1) * C, (long long)u_hi);
                if (x0 <= x1) {
                    double v0, v1;
                    if (ru == su) {
                        v0 = min(sv, rv);
                        v1 = max(sv, rv);
                    } else {
                        v0 = (double)sv + (double)(x0 - su) * slope;
                        v1 = (double)sv + (double)(x1 - su) * slope;
                        if (v0 > v1) {
                            const double t = v0;
                            v0 = v1;
                            v1 = t;
                        }
                    }
                    vlo = (int)floor((v0 - 1e-3) * inv_c);
                    vhi = (int)floor((v1 + 1e-3) * inv_c);
                }
            }
            const int wlo = max(warp_min_i(vlo), 0), whi = min(warp_max_i(vhi), cells_v - 1);
            if (wlo <= whi) {
                cb = __ldg(&ranges[(size_t)cu * cells_v + wlo].x);
                ce = __ldg(&ranges[(size_t)cu * cells_v + whi].y);
            }
            cu += dir;
            columns_left = dir > 0 ? cu <= cu_end : cu >= cu_end;
        }
        start = cb;
        count = min(ce - cb, (uint32_t)STAGE_ENTRIES);
        cb += count;
        return true;
    };
    int n = 0;
    bool full = false;
    uint32_t g_cur = 0, n_cur = 0;
    bool have = next_piece(g_cur, n_cur);
    if (have && lane == 0) bulk_load(st.seg[0], segs + g_cur, n_cur * (unsigned)sizeof(int4), &st.bar[0]);
    int b = 0;
    while (have) {
        uint32_t g_next = 0, n_next = 0;
        const bool have_next = next_piece(g_next, n_next);
        if (have_next && lane == 0) {
            // Buffer b ^ 1 was read in the previous round, before the warp's last __syncwarp.
            fence_proxy_async_shared();
            bulk_load(st.seg[b ^ 1], segs + g_next, n_next * (unsigned)sizeof(int4), &st.bar[b ^ 1]);
        }
        const bool landed = __all_sync(FULL, mbar_wait(&st.bar[b], (ss.phases >> b) & 1u));
        ss.phases ^= 1u << b;
        if (!landed) {
            // Wait once more, bounded, for the copy still in flight, then stage nothing more.
            if (have_next) {
                mbar_wait(&st.bar[b ^ 1], (ss.phases >> (b ^ 1)) & 1u);
                ss.phases ^= 1u << (b ^ 1);
            }
            __syncwarp();
            ss.dead = true;
            status |= FAILED_TIMEOUT;
            return n;
        }
        if (ray) {
            const int4 *piece = st.seg[b];
            for (uint32_t j = 0; j < n_cur; ++j) {
                const int4 seg = piece[j];
                if (max(seg.x, seg.z) < minx || min(seg.x, seg.z) > maxx || max(seg.y, seg.w) < miny ||
                    min(seg.y, seg.w) > maxy)
                    continue;
                ++edges_tested;
                const int ex = seg.z - seg.x, ey = seg.w - seg.y;
                long long den = mulw(idx, ey) - mulw(idy, ex);
                if (den == 0) continue;
                const int wx = seg.x - sx, wy = seg.y - sy;
                long long tn = mulw(wx, ey) - mulw(wy, ex);
                long long un = mulw(wx, idy) - mulw(wy, idx);
                long long d = den;
                if (d < 0) {
                    d = -d;
                    tn = -tn;
                    un = -un;
                }
                if (!(tn > 0 && tn < d && un >= 0 && un <= d)) continue;
                const uint2 ref = __ldg(refs + g_cur + j);
                // An edge listed in several swept cells is met again; a segment meets an edge at most
                // once, so a repeat of an edge among the lane's last few hits is that crossing again.
                bool repeat = false;
                for (int k = n - 1; k >= 0 && k >= n - 4; --k) repeat |= xs[k].edge == ref.x;
                if (repeat) continue;
                if (n >= MAXC) {
                    status |= FAILED_CAPACITY;
                    full = true;
                    continue;
                }
                const OutlineDev o = S.outlines[ref.y];
                const bool building = o.building != 0;
                const bool bounds =
                    building && ((un != 0 && un != d) || edge_bounds_roof(S, sx, sy, dx, dy, ref.x, o.first, o.count));
                xs[n++] = XRec{(double)tn / (double)d, ref.x, ref.y | (building ? X_BUILDING : 0u) | (bounds ? X_BOUNDS : 0u),
                               o.height, o.fp};
            }
        }
        __syncwarp();
        g_cur = g_next;
        n_cur = n_next;
        have = have_next;
        b ^= 1;
    }
    if (full) return n;
    return finish_crossings(S, xs, n, rcv_own);
}

// ---------------------------------------------------------------------------------------------
// Terrain

// Bilinear ground at a lattice point (the ray's ends).
__device__ inline float2 terrain_point(const SceneDev &S, int x, int y) {
    if (S.dem_nx == 0) return make_float2(S.flat_z, S.flat_g);
    long long nx = (long long)x - S.dem_ox, ny = (long long)y - S.dem_oy;
    long long i0 = floor_div64(nx, S.dem_sp), j0 = floor_div64(ny, S.dem_sp);
    float fx = (float)(nx - i0 * S.dem_sp) / (float)S.dem_sp;
    float fy = (float)(ny - j0 * S.dem_sp) / (float)S.dem_sp;
    if (i0 < 0) {
        i0 = 0;
        fx = 0.f;
    }
    if (j0 < 0) {
        j0 = 0;
        fy = 0.f;
    }
    if (i0 > S.dem_nx - 2) {
        fx = 1.f;
        i0 = S.dem_nx - 2;
    }
    if (j0 > S.dem_ny - 2) {
        fy = 1.f;
        j0 = S.dem_ny - 2;
    }
    const float2 *row0 = S.dem + j0 * S.dem_nx, *row1 = row0 + S.dem_nx;
    float2 a = __ldg(row0 + i0), b = __ldg(row0 + i0 + 1), c = __ldg(row1 + i0), d = __ldg(row1 + i0 + 1);
    float lz = a.x + fx * (b.x - a.x), hz = c.x + fx * (d.x - c.x);
    float lg = a.y + fx * (b.y - a.y), hg = c.y + fx * (d.y - c.y);
    return make_float2(lz + fy * (hz - lz), lg + fy * (hg - lg));
}

__device__ __forceinline__ float2 dem_node(const SceneDev &S, int i, int j) {
    i = i < 0 ? 0 : (i >= S.dem_nx ? S.dem_nx - 1 : i);
    j = j < 0 ? 0 : (j >= S.dem_ny ? S.dem_ny - 1 : j);
    return __ldg(S.dem + (size_t)j * S.dem_nx + i);
}

struct TV {
    float x, z, g;
};

// The ground profile under a ray (popup/src/scene.rs:242-296 on one metric lattice): the source end,
// a vertex wherever the ray crosses a DEM row or column line strictly inside, the receiver end.
// Orders of crossing are decided exactly on integers (a tie takes the row line first); each line
// vertex's node pair and fraction follow incrementally from exact rationals. Every step is additions
// only: the order test compares running products (steps to the next row line x |dx| against steps
// to the next column line x |dy|), and a vertex's node index and remainder advance by a fixed
// quotient and remainder taken once, carrying one when the remainder passes its denominator.
struct TerrainWalk {
    long long adx, ady;
    long long a_col, a_row;          // steps along x (y) from the source to the next column (row) line
    long long p_col, p_row;          // a_col * ady and a_row * adx: the order of the next two lines
    long long step_pc, step_pr;      // sp * ady and sp * adx: their increments per line
    long long sp;
    long long col_rem, col_den, col_qrem;  // column vertex: remainder of its node row (in den units)
    long long row_rem, row_den, row_qrem;  // row vertex: remainder of its node column
    int col_i, row_i;                // node row (column) index of the next column (row) vertex
    int col_q, row_q;                // whole nodes the index advances per line
    int next_col, next_row;          // line indices ahead
    int col_step, row_step;
    float length, inv_adx, inv_ady, inv_col_den, inv_row_den;
    bool dem;
    int stage;  // 0 start, 1 inner, 2 end, 3 done
    float2 start_zg, end_zg;

    __device__ __forceinline__ void init(const SceneDev &S, int x0, int y0, int x1, int y1, float length_m) {
        long long dx = (long long)x1 - x0, dy = (long long)y1 - y0;
        adx = dx >= 0 ? dx : -dx;
        ady = dy >= 0 ? dy : -dy;
        length = length_m;
        dem = S.dem_nx != 0;
        stage = 0;
        start_zg = terrain_point(S, x0, y0);
        end_zg = terrain_point(S, x1, y1);
        if (!dem) return;
        sp = S.dem_sp;
        long long rx = (long long)x0 - S.dem_ox, ry = (long long)y0 - S.dem_oy;
        long long fc = floor_div64(rx, sp), fr = floor_div64(ry, sp);
        bool on_col = fc * sp == rx, on_row = fr * sp == ry;
        col_step = dx > 0 ? 1 : -1;
        row_step = dy > 0 ? 1 : -1;
        long long nc = dx > 0 ? fc + 1 : (on_col ? fc - 1 : fc);
        long long nr = dy > 0 ? fr + 1 : (on_row ? fr - 1 : fr);
        next_col = (int)nc;
        next_row = (int)nr;
        a_col = dx != 0 ? (nc * sp - rx) * col_step : -1;
        a_row = dy != 0 ? (nr * sp - ry) * row_step : -1;
        p_col = a_col * ady;
        p_row = a_row * adx;
        step_pc = sp * ady;
        step_pr = sp * adx;
        inv_adx = adx ? 1.0f / (float)adx : 0.0f;
        inv_ady = ady ? 1.0f / (float)ady : 0.0f;
        if (dy != 0) {
            // x of the row line's vertex relative to the DEM origin, in units of sp: num / den.
            long long num = (rx * dy + (nr * sp - ry) * dx) * row_step;
            row_den = ady * sp;
            long long inc = sp * dx;  // per row step (both signs folded in)
            long long i = floor_div64(num, row_den);
            row_i = (int)i;
            row_rem = num - i * row_den;
            long long q = floor_div64(inc, row_den);
            row_q = (int)q;
            row_qrem = inc - q * row_den;
            inv_row_den = 1.0f / (float)row_den;
        }
        if (dx != 0) {
            long long num = (ry * dx + (nc * sp - rx) * dy) * col_step;
            col_den = adx * sp;
            long long inc = sp * dy;
            long long i = floor_div64(num, col_den);
            col_i = (int)i;
            col_rem = num - i * col_den;
            long long q = floor_div64(inc, col_den);
            col_q = (int)q;
            col_qrem = inc - q * col_den;
            inv_col_den = 1.0f / (float)col_den;
        }
    }

    // The next vertex; false when the walk is done.
    __device__ __forceinline__ bool next(const SceneDev &S, TV &v) {
        if (stage == 0) {
            stage = dem ? 1 : 2;
            v = TV{0.0f, start_zg.x, start_zg.y};
            return true;
        }
        if (stage == 1) {
            bool col_ok = adx != 0 && a_col < adx;
            bool row_ok = ady != 0 && a_row < ady;
            if (col_ok || row_ok) {
                bool take_row = !col_ok || (row_ok && p_row <= p_col);
                if (take_row) {
                    float t = (float)a_row * inv_ady;
                    float f = (float)row_rem * inv_row_den;
                    float2 a = dem_node(S, row_i, next_row), b = dem_node(S, row_i + 1, next_row);
                    v = TV{t * length, a.x + f * (b.x - a.x), a.y + f * (b.y - a.y)};
                    next_row += row_step;
                    a_row += sp;
                    p_row += step_pr;
                    row_i += row_q;
                    row_rem += row_qrem;
                    if (row_rem >= row_den) {
                        row_rem -= row_den;
                        ++row_i;
                    }
                } else {
                    float t = (float)a_col * inv_adx;
                    float f = (float)col_rem * inv_col_den;
                    float2 a = dem_node(S, next_col, col_i), b = dem_node(S, next_col, col_i + 1);
                    v = TV{t * length, a.x + f * (b.x - a.x), a.y + f * (b.y - a.y)};
                    next_col += col_step;
                    a_col += sp;
                    p_col += step_pc;
                    col_i += col_q;
                    col_rem += col_qrem;
                    if (col_rem >= col_den) {
                        col_rem -= col_den;
                        ++col_i;
                    }
                }
                return true;
            }
            stage = 2;
        }
        if (stage == 2) {
            stage = 3;
            v = TV{length, end_zg.x, end_zg.y};
            return true;
        }
        return false;
    }
};

// ---------------------------------------------------------------------------------------------
// The path

struct Roof {
    float x0, x1, top0, top1, zt0, zt1, g0, g1;  // roof ends, tops, terrain and G at the ends
    uint32_t fp;
};

struct BuildingHit {
    uint32_t fp;
    float x, top, zt, g;
};

// 32 bytes: the next segment's origin is the profile at the entry's own x (the source end's at x = 0).
struct HullEntry {
    float x, z;    // the point of the band
    float oz;      // the profile's height at x: the next segment's origin is (x, oz)
    float og;      // G at x
    Moments seg;   // profile from the previous entry's origin to x, about that origin
};

template <int CAP_C, int CAP_K, int CAP_H>
struct PathWork {
    XRec xs[CAP_C];
    PlanePoint tops[CAP_C];
    BuildingHit hits[CAP_C];
    Roof roofs[CAP_C / 2 + 1];
    PlanePoint crests[CAP_K];
    HullEntry hull[2][CAP_H];
};

struct PathResult {
    float boundary[2][QM_BANDS];  // 10^(-A_boundary/10) per state
    float slant;
    float weight;          // point divergence 1/(d^2 10^1.1)
    float p[QM_PERIODS];   // favourable probability per period
    uint32_t status;
    uint32_t crossings;
    uint32_t edges_tested;
    uint32_t vertices;    // profile vertices streamed (terrain and roofs)
    uint32_t candidates;  // diffraction candidates fed to the bands
};

// One state's rubber band, built as the candidates stream in sorted order
// (rubber_band.rs:373-444 with the equal-distance collapse and the monotone chain), with the
// profile's segment moments carried on the hull so the side planes need no stored profile.
template <int STATE, int CAP_H>
struct Band {
    float radius;
    PlanePoint S, R;
    float slope_sr;  // (R.z - S.z) / (R.x - S.x): the line of sight, taken once
    float chord_sr;  // |SR|
    Sag sag_sr;
    HullEntry *h;
    int n;
    bool blocked;
    bool have_best;
    float best_value;
    PlanePoint best;
    Moments best_src;  // profile [0, best] about (0, z0)
    float best_oz, best_og;
    float oox, ooz;  // origin of the open segment
    Moments open;
    bool failed;

    __device__ __forceinline__ void init(HullEntry *storage, PlanePoint s, PlanePoint r, float z0, float g0) {
        S = s;
        R = r;
        float dx = r.x - s.x, dz = r.z - s.z;
        chord_sr = sqrtf(dx * dx + dz * dz);
        radius = fmaxf(1000.0f, 8.0f * chord_sr);
        slope_sr = dz / dx;
        if (STATE == QM_FAV) sag_sr = make_sag(radius, s, r);
        h = storage;
        h[0] = HullEntry{s.x, s.z, z0, g0, moments_zero()};
        n = 1;
        blocked = false;
        have_best = false;
        best_value = 0.0f;
        oox = 0.0f;
        ooz = z0;
        open = moments_zero();
        failed = false;
    }

    // Adds the profile segment since the last event (moments about (sx0, sz0)) to the open segment.
    __device__ __forceinline__ void fold(const Moments &seg, float sx0, float sz0) {
        open = join(open, rebase(seg, sx0, sz0, oox, ooz));
    }

    __device__ __forceinline__ void push(float px, float pz, float oz, float og) {
        Moments seg = open;
        while (n >= 2) {
            const HullEntry &a = h[n - 2];
            const HullEntry &b = h[n - 1];
            bool under;
            if (STATE == QM_HOM) {
                // b on or under the chord a -> p, without the division (p.x > a.x).
                under = (b.z - a.z) * (px - a.x) <= (pz - a.z) * (b.x - a.x);
            } else {
                under = b.z <= ray_altitude<STATE>(radius, PlanePoint{a.x, a.z}, PlanePoint{px, pz}, b.x);
            }
            if (under) {
                seg = join(b.seg, rebase(seg, b.x, b.oz, a.x, a.oz));
                --n;
            } else {
                break;
            }
        }
        if (n >= CAP_H) {
            failed = true;
            return;
        }
        h[n++] = HullEntry{px, pz, oz, og, seg};
        open = moments_zero();
        oox = px;
        ooz = oz;
    }

    // A candidate at x with the profile moments [0, x] about (0, z0) and the profile at x.
    __device__ __forceinline__ void candidate(PlanePoint c, const Moments &total, float z0, float oz, float og) {
        if (failed) return;
        float line = S.z + slope_sr * (c.x - S.x);
        if (STATE == QM_FAV) line += sag_sr.at(c.x - S.x);
        if (c.z > line) {
            // Blocking: the first opens the band (from the total so far), an equal-x one higher than
            // the hull's last replaces it, any other extends the hull; one push for all three.
            if (!blocked) {
                blocked = true;
                open = total;
                oox = 0.0f;
                ooz = z0;
            } else if (h[n - 1].x == c.x && n >= 2) {
                if (!(c.z > h[n - 1].z)) return;
                const HullEntry &b = h[n - 1];
                const HullEntry &a = h[n - 2];
                open = join(b.seg, rebase(open, b.x, b.oz, a.x, a.oz));
                oox = a.x;
                ooz = a.oz;
                --n;
            }
            push(c.x, c.z, oz, og);
            return;
        }
        if (blocked) return;
        float delta = single_path_difference_f<STATE>(radius, S, c, R, chord_sr);
        if (!have_best || delta > best_value) {
            have_best = true;
            best_value = delta;
            best = c;
            best_src = total;
            best_oz = oz;
            best_og = og;
            open = moments_zero();
            oox = c.x;
            ooz = oz;
        }
    }
};

// boundary_for_candidates (diffraction.rs:64-197) from the band's result.
template <int STATE, int CAP_H>
__device__ __noinline__ void state_boundary(Band<STATE, CAP_H> &band, const EqGeometry &direct, float path_ground, float near_source,
                               float source_gf, float z0, float g0, float L, float out[QM_BANDS]) {
    float whole[QM_BANDS];
    ground_attenuation_bands(direct, source_side_factors(STATE, path_ground, near_source), STATE, whole);
#pragma unroll
    for (int b = 0; b < QM_BANDS; ++b) out[b] = whole[b];
    PlanePoint pts_local[1];
    const PlanePoint *points;
    int np;
    Moments src_m, rcv_m;
    float last_ox, last_oz, last_og, first_og;
    bool blocked = band.blocked;
    // Points: the hull interior, or the best unblocked candidate.
    PlanePoint hull_pts[CAP_H];
    if (blocked) {
        band.push(band.R.x, band.R.z, 0.0f, 0.0f);
        if (band.failed) return;
        np = band.n - 2;
        if (np <= 0) return;  // a blocked band keeps its highest blocking point; never empty
        for (int i = 0; i < np; ++i) hull_pts[i] = PlanePoint{band.h[i + 1].x, band.h[i + 1].z};
        points = hull_pts;
        src_m = band.h[1].seg;
        first_og = band.h[1].og;
        rcv_m = band.h[band.n - 1].seg;
        last_ox = band.h[band.n - 2].x;
        last_oz = band.h[band.n - 2].oz;
        last_og = band.h[band.n - 2].og;
    } else if (band.have_best) {
        pts_local[0] = band.best;
        points = pts_local;
        np = 1;
        src_m = band.best_src;
        first_og = band.best_og;
        rcv_m = band.open;
        last_ox = band.best.x;
        last_oz = band.best_oz;
        last_og = band.best_og;
    } else {
        return;
    }
    (void)first_og;
    PlanePoint S = band.S, R = band.R;
    PlanePoint first = points[0], last = points[np - 1];
    PointD Sd{S.x, S.z}, Rd{R.x, R.z};
    double radius = band.radius;
    double delta = path_difference_d(STATE, radius, Sd, points, np, Rd);
    float span = 0.0f;
    if (np > 1)
        for (int i = 0; i + 1 < np; ++i) {
            float dx = points[i + 1].x - points[i].x, dz = points[i + 1].z - points[i].z;
            float chord = sqrtf(dx * dx + dz * dz);
            span += chord + arc_excess_f<STATE>(chord, band.radius);
        }
    float c2[QM_BANDS];
#pragma unroll
    for (int b = 0; b < QM_BANDS; ++b) {
        if (np > 1 && span > MULTIPLE_DIFFRACTION_MINIMUM_SPAN) {
            float x = 5.0f * c_band.lambda[b] / span;
            c2[b] = (1.0f + x * x) / (1.0f / 3.0f + x * x);
        } else {
            c2[b] = 1.0f;
        }
    }
    // Side planes (mean_plane.rs:204-249) and geometries.
    MeanPlane sp = plane_of(src_m, 0.0f, first.x, z0);
    EqGeometry source_side = geometry_over(sp, S, first);
    float rlen = L - last_ox;
    MeanPlane rp = plane_of(rcv_m, last_ox, rlen, last_oz);
    EqGeometry receiver_side = geometry_over(rp, last, R);
    PointD Si, Ri;
    mirror_d(sp, S.x, S.z, Si.x, Si.z);
    mirror_d(rp, R.x, R.z, Ri.x, Ri.z);
    double delta_si = path_difference_d(STATE, radius, Si, points, np, Rd);
    double delta_ri = path_difference_d(STATE, radius, Sd, points, np, Ri);
    float source_side_ground = mean_ground_of(src_m, first.x, g0);
    float source_side_near = ground_factor_near_source(source_side, source_side_ground, source_gf);
    float ground_so[QM_BANDS], ground_or[QM_BANDS];
    ground_attenuation_bands(source_side, source_side_factors(STATE, source_side_ground, source_side_near), STATE,
                             ground_so);
    float receiver_side_ground = mean_ground_of(rcv_m, rlen, last_og);
    ground_attenuation_bands(receiver_side, GroundFactors{receiver_side_ground, receiver_side_ground, receiver_side_ground},
                             STATE, ground_or);
    double rayleigh_star = blocked ? 0.0 : path_difference_d(STATE, radius, Si, points, np, Ri);
    const float delta_f = (float)delta, delta_si_f = (float)delta_si, delta_ri_f = (float)delta_ri;
#pragma unroll
    for (int b = 0; b < QM_BANDS; ++b) {
        bool admitted = blocked || (delta > -c_band.lambda_over_20_d[b] && delta > c_band.lambda_over_4_d[b] - rayleigh_star);
        if (!admitted) continue;
        float direct_db = diffraction_db(delta_f, c2[b], b);
        float source_image_db = diffraction_db(delta_si_f, c2[b], b);
        float receiver_image_db = diffraction_db(delta_ri_f, c2[b], b);
        float sr = direct_db;
        float split_so;
        if (source_side.source_below) {
            sr = source_image_db;
            split_so = ground_so[b];
        } else {
            split_so = ground_split_db(ground_so[b], source_image_db, direct_db);
        }
        if (!isfinite(split_so)) {
            split_so = ground_so[b];
            sr = source_image_db;
        }
        float split_or;
        if (receiver_side.receiver_below) {
            sr = receiver_image_db;
            split_or = ground_or[b];
        } else {
            split_or = ground_split_db(ground_or[b], receiver_image_db, sr);
        }
        if (!isfinite(split_or)) {
            split_or = ground_or[b];
            sr = receiver_image_db;
        }
        out[b] = fminf(fmaxf(sr, 0.0f), DIFFRACTION_CAP_DB) + split_so + split_or;
    }
}

// p of a period for a direction (physics/src/weather.rs:61-70).
__device__ __forceinline__ float favourable_at(const float row[QM_SECTORS], float azimuth_rad) {
    float bearing = 90.0f - azimuth_rad * (180.0f / 3.14159265358979f);
    bearing = bearing - 360.0f * floorf(bearing / 360.0f);
    if (bearing >= 360.0f) bearing -= 360.0f;
    float position = bearing / (360.0f / QM_SECTORS);
    float fl = floorf(position);
    int lower = ((int)fl) % QM_SECTORS;
    int upper = (lower + 1) % QM_SECTORS;
    float fraction = position - fl;
    return row[lower] + fraction * (row[upper] - row[lower]);
}

// A walk's start: the lattice walk from the source's lattice point, the f64 walk
// (qm_offlattice.cuh) from its fractional position.
__device__ __forceinline__ void start_walk(TerrainWalk &walk, const SceneDev &S, double, double, int sx, int sy, int rx,
                                           int ry, float L) {
    walk.init(S, sx, sy, rx, ry, L);
}

// The rest of a path once its crossings are listed in w.xs[0, nx): terrain, roofs, both states'
// bands and boundaries, slant, divergence and p. out.status and out.edges_tested hold what the
// listing set. The ray starts at (sxd, syd) steps: the source's lattice point for a point source,
// a quadrature node's fractional position with the f64 walk (Walk = TerrainWalkD) for a line.
template <int CAP_C, int CAP_K, int CAP_H, class Walk = TerrainWalk>
__device__ void evaluate_listed(const SceneDev &S, const SourceDev &src, int rx, int ry, float rcv_alt, bool want_fav,
                                PathWork<CAP_C, CAP_K, CAP_H> &w, int nx, PathResult &out, double sxd, double syd) {
    const int sx = src.x, sy = src.y;
    const float dxm = (float)((double)rx - sxd) * S.step_m, dym = (float)((double)ry - syd) * S.step_m;
    const float dist = sqrtf(dxm * dxm + dym * dym);
    const float L = fmaxf(dist, 1.0f);
    out.crossings = nx;
    // Pass 1: terrain heights and G at the crossings, and the crests (physics/src/ray.rs:255-309).
    Walk walk;
    start_walk(walk, S, sxd, syd, sx, sy, rx, ry, L);
    const float z0 = walk.start_zg.x, g0 = walk.start_zg.y;
    const float source_ground = z0;
    const float platform = src.platform;
    const float src_alt = source_ground + src.height;
    int nk = 0;
    {
        TV prev{0.f, 0.f, 0.f}, v;
        bool have_prev = false;
        int ci = 0;
        bool open = false;
        PlanePoint best{0.f, 0.f};
        long long at = 0;
        // The next crossing's place along the ray, kept in a register (infinite past the last).
        float xc = nx > 0 ? (float)w.xs[0].t * L : INFINITY;
        while (walk.next(S, v)) {
            if (v.x < platform) v.z = fminf(v.z, source_ground);
            // Crossings whose interpolation interval ends here (first vertex with x > crossing x).
            if (have_prev)
                while (xc < v.x) {
                    float f = v.x > prev.x ? fminf(fmaxf((xc - prev.x) / (v.x - prev.x), 0.f), 1.f) : 0.f;
                    w.tops[ci] = PlanePoint{prev.z + f * (v.z - prev.z), prev.g + f * (v.g - prev.g)};
                    ++ci;
                    xc = ci < nx ? (float)w.xs[ci].t * L : INFINITY;
                }
            // crests_of (ray.rs:360-385)
            if (walk.dem) {
                bool middle = v.x > 300.0f && v.x < L - 300.0f;
                long long group = (long long)floorf(v.x / 150.0f);
                if (open && (!middle || at != group)) {
                    if (nk < CAP_K) w.crests[nk++] = best;
                    else out.status |= FAILED_CAPACITY;
                    open = false;
                }
                if (!middle) {
                    if (nk < CAP_K) w.crests[nk++] = PlanePoint{v.x, v.z};
                    else out.status |= FAILED_CAPACITY;
                } else if (!(open && v.z <= best.z)) {
                    open = true;
                    best = PlanePoint{v.x, v.z};
                    at = group;
                }
            }
            prev = v;
            have_prev = true;
        }
        if (open) {
            if (nk < CAP_K) w.crests[nk++] = best;
            else out.status |= FAILED_CAPACITY;
        }
        // Crossings at or beyond the last vertex read the last interval at its end.
        for (; ci < nx; ++ci) w.tops[ci] = PlanePoint{prev.z, prev.g};
    }
    // Tops and building hits (ray.rs:293-309); w.tops[i] holds (terrain z, G) at crossing i.
    int nt = 0, nb = 0;
    {
        uint32_t own = src.fp;
        for (int i = 0; i < nx; ++i) {
            const uint32_t fp = w.xs[i].fp;
            bool bounds = (w.xs[i].info & X_BOUNDS) != 0;
            if (own != 0) {
                // containing_footprints (ray.rs:201-226): the own footprint and every footprint with an
                // odd count of roof-bounding crossings.
                bool contained = fp == own;
                if (!contained) {
                    int count = 0;
                    for (int k = 0; k < nx; ++k)
                        if ((w.xs[k].info & X_BOUNDS) && xrec_fp(S, w.xs[k]) == fp) ++count;
                    contained = (count & 1) != 0;
                }
                if (contained) continue;
            }
            float x = (float)w.xs[i].t * L;
            float zt = w.tops[i].x, g = w.tops[i].z;
            float top = zt + w.xs[i].height;
            if (bounds) w.hits[nb++] = BuildingHit{fp, x, top, zt, g};
            w.tops[nt++] = PlanePoint{x, top};
        }
    }
    // Roofs: each footprint's hits in order of x, paired consecutively (ray.rs:312-323). The hits
    // already come in order of x, so a forward scan finds each one's partner; `hits[k].fp` is
    // cleared once paired.
    int nr = 0;
    for (int k = 0; k < nb; ++k) {
        uint32_t fp = w.hits[k].fp;
        if (fp == 0u) continue;
        for (int j = k + 1; j < nb; ++j)
            if (w.hits[j].fp == fp) {
                const BuildingHit &a = w.hits[k], &b = w.hits[j];
                w.roofs[nr++] = Roof{a.x, b.x, a.top, b.top, a.zt, b.zt, a.g, b.g, fp};
                w.hits[j].fp = 0u;
                break;
            }
        w.hits[k].fp = 0u;
    }
    // clip_roofs_in_closing_order (ray.rs:389-404): sorted by (x1, x0), stable over roofs grouped by
    // footprint, so equal keys keep footprint order.
    for (int i = 1; i < nr; ++i) {
        Roof v = w.roofs[i];
        int j = i - 1;
        while (j >= 0 && (w.roofs[j].x1 > v.x1 ||
                          (w.roofs[j].x1 == v.x1 && (w.roofs[j].x0 > v.x0 || (w.roofs[j].x0 == v.x0 && w.roofs[j].fp > v.fp))))) {
            w.roofs[j + 1] = w.roofs[j];
            --j;
        }
        w.roofs[j + 1] = v;
    }
    {
        float covered_to = -INFINITY, cov_zt = 0.f, cov_g = 0.f;
        int kept = 0;
        for (int i = 0; i < nr; ++i) {
            Roof r = w.roofs[i];
            if (r.x1 <= covered_to) continue;
            if (r.x0 < covered_to) {
                float span = r.x1 - r.x0;
                r.top0 += (covered_to - r.x0) / span * (r.top1 - r.top0);
                r.x0 = covered_to;
                r.zt0 = cov_zt;
                r.g0 = cov_g;
            }
            covered_to = r.x1;
            cov_zt = r.zt1;
            cov_g = r.g1;
            w.roofs[kept++] = r;
        }
        nr = kept;
    }
    // Pass 2: the vertical profile (terrain with roofs raised as hard ground, ray.rs:326-353)
    // streamed in order, candidates (crests and tops strictly inside, terrain first at equal x:
    // cnossos/mod.rs:154-176) fed to each state's band at their place in the stream.
    const PlanePoint Sp{0.0f, src_alt}, Rp{L, rcv_alt};
    Band<QM_HOM, CAP_H> hom;
    Band<QM_FAV, CAP_H> fav;
    hom.init(w.hull[0], Sp, Rp, z0, g0);
    if (want_fav) fav.init(w.hull[1], Sp, Rp, z0, g0);
    Moments total = moments_zero();
    {
        start_walk(walk, S, sxd, syd, sx, sy, rx, ry, L);
        // Profile stream state: pending roof vertices, covered_to, current terrain vertex.
        TV vprev, tv;
        walk.next(S, tv);  // x = 0
        if (tv.x < platform) tv.z = fminf(tv.z, source_ground);
        vprev = tv;
        int ri = 0;
        float covered_to = 0.0f;
        // The roof being emitted (its four vertices: ground, top, top, ground) and the next roof's
        // start, kept in registers.
        Roof roof;
        int roof_stage = 4;
        float next_roof_x0 = nr > 0 ? w.roofs[0].x0 : INFINITY;
        bool have_tv = walk.next(S, tv);
        if (have_tv && tv.x < platform) tv.z = fminf(tv.z, source_ground);
        // The next vertex of the vertical profile.
        auto next_vertex = [&](TV &out_v) -> bool {
            for (;;) {
                if (roof_stage < 4) {
                    const bool first_end = roof_stage < 2, ground = roof_stage == 0 || roof_stage == 3;
                    out_v = TV{first_end ? roof.x0 : roof.x1,
                               roof_stage == 0 ? roof.zt0 : roof_stage == 1 ? roof.top0 : roof_stage == 2 ? roof.top1 : roof.zt1,
                               ground ? (first_end ? roof.g0 : roof.g1) : 0.0f};
                    ++roof_stage;
                    return true;
                }
                if (!have_tv) return false;
                if (next_roof_x0 < tv.x) {
                    roof = w.roofs[ri];
                    roof_stage = 0;
                    covered_to = roof.x1;
                    ++ri;
                    next_roof_x0 = ri < nr ? w.roofs[ri].x0 : INFINITY;
                    continue;
                }
                TV t = tv;
                have_tv = walk.next(S, tv);
                if (have_tv && tv.x < platform) tv.z = fminf(tv.z, source_ground);
                if (t.x > covered_to) {
                    out_v = t;
                    return true;
                }
            }
        };
        TV vnext;
        bool have_next = next_vertex(vnext);
        uint32_t n_vertices = 0, n_candidates = 0;
        // The profile since the last candidate, about that candidate's place (seg_x, seg_z); folded
        // into the total and into each band's open segment at the next candidate.
        Moments seg = moments_zero();
        float seg_x = 0.0f, seg_z = z0;
        auto consume = [&](const TV &v) {
            ++n_vertices;
            add_stretch(seg, seg_x, seg_z, vprev.x, vprev.z, vprev.g, v.x, v.z, v.g);
            vprev = v;
        };
        auto fold = [&]() {
            total = join(total, rebase(seg, seg_x, seg_z, 0.0f, z0));
            hom.fold(seg, seg_x, seg_z);
            if (want_fav) fav.fold(seg, seg_x, seg_z);
            seg = moments_zero();
            seg_x = vprev.x;
            seg_z = vprev.z;
        };
        // The next crest and the next top strictly inside (0, L), kept in registers.
        int ik = 0, it = 0;
        auto next_crest = [&](PlanePoint &c) -> bool {
            while (ik < nk) {
                c = w.crests[ik++];
                if (c.x > 0.0f && c.x < L) return true;
            }
            return false;
        };
        auto next_top = [&](PlanePoint &c) -> bool {
            while (it < nt) {
                c = w.tops[it++];
                if (c.x > 0.0f && c.x < L) return true;
            }
            return false;
        };
        PlanePoint crest_c, top_c;
        bool have_crest = next_crest(crest_c), have_top = next_top(top_c);
        for (;;) {
            // Next candidate, terrain first at equal x.
            PlanePoint c;
            if (have_crest && (!have_top || !(top_c.x < crest_c.x))) {
                c = crest_c;
                have_crest = next_crest(crest_c);
            } else if (have_top) {
                c = top_c;
                have_top = next_top(top_c);
            } else {
                break;
            }
            while (have_next && vnext.x <= c.x) {
                consume(vnext);
                have_next = next_vertex(vnext);
            }
            if (vprev.x < c.x && have_next) {
                float f = (c.x - vprev.x) / (vnext.x - vprev.x);
                consume(TV{c.x, vprev.z + f * (vnext.z - vprev.z), vprev.g + f * (vnext.g - vprev.g)});
            }
            ++n_candidates;
            fold();
            hom.candidate(c, total, z0, vprev.z, vprev.g);
            if (want_fav) fav.candidate(c, total, z0, vprev.z, vprev.g);
        }
        while (have_next) {
            consume(vnext);
            have_next = next_vertex(vnext);
        }
        fold();
        out.vertices = n_vertices;
        out.candidates = n_candidates;
    }
    // The direct path (diffraction.rs:44-61) and each state's boundary.
    MeanPlane dplane = plane_of(total, 0.0f, L, z0);
    EqGeometry direct = geometry_over(dplane, Sp, Rp);
    float path_ground = mean_ground_of(total, L, g0);
    float source_gf = src.gf >= 0.0f ? src.gf : g0;
    float near_source = ground_factor_near_source(direct, path_ground, source_gf);
    float att[QM_BANDS];
    // Each band goes to state_boundary as a copy: the band itself never has its address taken, so its
    // fields can stay in registers through the candidate loop.
    {
        Band<QM_HOM, CAP_H> done = hom;
        state_boundary<QM_HOM, CAP_H>(done, direct, path_ground, near_source, source_gf, z0, g0, L, att);
        if (done.failed) out.status |= FAILED_CAPACITY;
    }
#pragma unroll
    for (int b = 0; b < QM_BANDS; ++b) out.boundary[0][b] = __expf(-att[b] * LN10_OVER_10);
    if (want_fav) {
        Band<QM_FAV, CAP_H> done = fav;
        state_boundary<QM_FAV, CAP_H>(done, direct, path_ground, near_source, source_gf, z0, g0, L, att);
        if (done.failed) out.status |= FAILED_CAPACITY;
#pragma unroll
        for (int b = 0; b < QM_BANDS; ++b) out.boundary[1][b] = __expf(-att[b] * LN10_OVER_10);
    } else {
#pragma unroll
        for (int b = 0; b < QM_BANDS; ++b) out.boundary[1][b] = out.boundary[0][b];
    }
    // Slant, divergence, p (ray.rs:132-137; evaluate.rs:199-204, 317-322).
    float dz = rcv_alt - src_alt;
    out.slant = fmaxf(sqrtf(L * L + dz * dz), 1.0f);
    float dh = fmaxf(dist, src.excl);
    float d = fmaxf(sqrtf(dh * dh + dz * dz), 1.0f);
    out.weight = 1.0f / (d * d * 12.589254117941673f);
    float azimuth = atan2f(dym, dxm);
#pragma unroll
    for (int p = 0; p < QM_PERIODS; ++p) out.p[p] = want_fav ? favourable_at(S.fav[p], azimuth) : 0.0f;
}

// One point source at one receiver: boundary transfer per state, slant, divergence weight and p.
// `want_fav` false skips the favourable state (its p is zero everywhere).
template <int CAP_C, int CAP_K, int CAP_H>
__device__ void evaluate_path(const SceneDev &S, const SourceDev &src, int rx, int ry, float rcv_alt, uint32_t rcv_own,
                              bool want_fav, PathWork<CAP_C, CAP_K, CAP_H> &w, PathResult &out) {
    out.status = 0;
    out.edges_tested = 0;
    const int nx = list_crossings<CAP_C>(S, src.x, src.y, rx, ry, rcv_own, w.xs, out.status, out.edges_tested);
    evaluate_listed<CAP_C, CAP_K, CAP_H>(S, src, rx, ry, rcv_alt, want_fav, w, nx, out, (double)src.x, (double)src.y);
}

}  // namespace qm
