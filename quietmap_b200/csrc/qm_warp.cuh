// The warp-per-path painter: one warp evaluates one receiver-source path at a time, its lists in
// shared memory, its lanes sharing every phase — the cells and edges of the crossing walk, the sort
// of the crossings, the DEM lines of the terrain walk, the candidates of the rubber bands, and the
// bands of the two states' boundaries. Long terrain rays (tens of crossings, hundreds of profile
// vertices and candidates) are where thread-per-path loses its lanes to divergence and its lists to
// local memory; here the lanes stay converged and the lists never leave the SM.
//
// It computes what `evaluate_path` (qm_path.cuh) computes, following the same reference code:
// popup/src/obstacles/crossings.rs:13-226, physics/src/ray.rs:125-404, physics/src/cnossos/
// {mod.rs:123-176, mean_plane.rs:19-64, rubber_band.rs:373-444, diffraction.rs:64-197}. Two
// reorganisations keep the results: the rubber band is found by gift wrapping (each next point is
// the candidate with the steepest chord, or the steepest initial arc tangent downwind, from the last
// one; ties to the farthest), which yields the monotone chain's strict upper chain; and the mean
// planes' integrals are summed by the lanes over the profile's pieces within each range.
#pragma once

#include "qm_path.cuh"
#include "qm_warp_util.cuh"

namespace qm {

// Capacities of one warp's path: raw crossings (duplicates of an edge listed in several cells
// included), roofs, crests, hull points per state, blocking candidates.
constexpr int WX = 256, WR = 96, WK = 448, WH = 48, WB = 256;

struct WarpShared {
    unsigned long long key[WX];
    uint32_t idx[WX];
    double t[WX];      // crossing chainage; later (zt, g) at the crossing as float2
    uint32_t edge[WX];
    uint32_t info[WX];  // outline index | bounds_roof << 31
    float2 top[WX];     // (x, top) of the tops
    float r_x0[WR], r_x1[WR], r_top0[WR], r_top1[WR], r_zt0[WR], r_zt1[WR], r_g0[WR], r_g1[WR];
    uint32_t r_fp[WR];
    float2 crest[WK];
    float2 hull[2][WH]; // each state's band points (interior)
    // One state's blocking candidates live in `key`'s storage, free once the crossings are sorted.
    __device__ __forceinline__ float2 *block() { return reinterpret_cast<float2 *>(key); }
};
static_assert(sizeof(unsigned long long) * WX >= sizeof(float2) * WB, "blocking list fits the key storage");

__device__ __forceinline__ uint32_t outline_fp(const SceneDev &S, uint32_t info) { return S.outlines[info & 0x7fffffffu].fp; }

// ------------------------------------------------------------------------------------------------
// A. Crossings

__device__ inline int warp_crossings(const SceneDev &S, int sx, int sy, int rx, int ry, uint32_t rcv_own,
                                     WarpShared &W, uint32_t &status, uint32_t &tested) {
    const int l = lane_id();
    const long long dx = (long long)rx - sx, dy = (long long)ry - sy;
    const long long adx = dx >= 0 ? dx : -dx, ady = dy >= 0 ? dy : -dy;
    const int C = S.cell_steps;
    const int cx0 = floor_div(sx, C), cy0 = floor_div(sy, C);
    const int lx = floor_div(rx, C), ly = floor_div(ry, C);
    const int stx = dx >= 0 ? 1 : -1, sty = dy >= 0 ? 1 : -1;
    // Cell boundaries crossed along x and y: distances (in steps along the axis) to the i-th one.
    const long long bx0 = (long long)(cx0 + (dx >= 0 ? 1 : 0)) * C, by0 = (long long)(cy0 + (dy >= 0 ? 1 : 0)) * C;
    Merge2 m;
    m.a0 = (bx0 - sx) * stx;
    m.pa = C;
    m.da = adx > 0 ? adx : 1;
    m.na = lx > cx0 ? lx - cx0 : cx0 - lx;
    m.b0 = (by0 - sy) * sty;
    m.pb = C;
    m.db = ady > 0 ? ady : 1;
    m.nb = ly > cy0 ? ly - cy0 : cy0 - ly;
    const long long n_cells = m.na + m.nb + 1;
    const int minx = min(sx, rx), maxx = max(sx, rx), miny = min(sy, ry), maxy = max(sy, ry);
    int n_raw = 0;
    bool overflow = false;
    unsigned my_tested = 0;
    for (long long base = 0; base < n_cells; base += 32) {
        long long k = base + l;
        uint32_t b = 0, e = 0;
        if (k < n_cells) {
            long long ca = m.count_a(k, 0, 0);
            int cx = cx0 + stx * (int)ca, cy = cy0 + sty * (int)(k - ca);
            if (cx >= 0 && cy >= 0 && cx < S.cells_x && cy < S.cells_y) {
                int c = cy * S.cells_x + cx;
                b = __ldg(S.cell_start + c);
                e = __ldg(S.cell_start + c + 1);
            }
        }
        int count = (int)(e - b), total;
        int offset = warp_exclusive_scan(count, total);
        for (int q0 = 0; q0 < total; q0 += 32) {
            int q = q0 + l;
            bool hit = false;
            double t = 0.0;
            uint32_t info = 0, edge_v = 0;
            // The lane holding entry q: the last lane whose offset is <= q (all lanes shuffle).
            int owner = 0;
#pragma unroll
            for (int s = 16; s > 0; s >>= 1) {
                int cand = owner + s;
                int off_c = __shfl_sync(FULL, offset, cand & 31);
                int qq = q < total ? q : -1;
                if (cand < 32 && qq >= 0 && off_c <= qq) owner = cand;
            }
            uint32_t ob = __shfl_sync(FULL, b, owner);
            int ooff = __shfl_sync(FULL, offset, owner);
            if (q < total) {
                uint32_t entry = ob + (uint32_t)(q - ooff);
                int4 seg = __ldg(S.cell_seg + entry);
                if (!(max(seg.x, seg.z) < minx || min(seg.x, seg.z) > maxx || max(seg.y, seg.w) < miny ||
                      min(seg.y, seg.w) > maxy)) {
                    ++my_tested;
                    long long ex = (long long)seg.z - seg.x, ey = (long long)seg.w - seg.y;
                    long long den = dx * ey - dy * ex;
                    if (den != 0) {
                        long long wx = (long long)seg.x - sx, wy = (long long)seg.y - sy;
                        long long tn = wx * ey - wy * ex, un = wx * dy - wy * dx;
                        if (den < 0) {
                            den = -den;
                            tn = -tn;
                            un = -un;
                        }
                        if (tn > 0 && tn < den && un >= 0 && un <= den) {
                            uint2 ref = __ldg(S.cell_ref + entry);
                            OutlineDev o = S.outlines[ref.y];
                            bool bounds = o.building != 0 && edge_bounds_roof(S, sx, sy, dx, dy, ref.x, o.first, o.count);
                            hit = true;
                            t = (double)tn / (double)den;
                            info = ref.y | (bounds ? 0x80000000u : 0u);
                            edge_v = ref.x;
                        }
                    }
                }
            }
            unsigned mask = __ballot_sync(FULL, hit);
            int pos = n_raw + __popc(mask & ((1u << l) - 1));
            if (hit) {
                if (pos < WX) {
                    W.t[pos] = t;
                    W.edge[pos] = edge_v;
                    W.info[pos] = info;
                } else {
                    overflow = true;
                }
            }
            n_raw += __popc(mask);
        }
    }
    tested += warp_sum(my_tested);
    if (__any_sync(FULL, overflow) || n_raw > WX) {
        status |= FAILED_CAPACITY;
        return 0;
    }
    __syncwarp();
    // Sort by t (bit patterns of positive doubles order as the values), padded to a power of two.
    int n_pad = 1;
    while (n_pad < n_raw) n_pad <<= 1;
    for (int i = l; i < n_pad; i += 32) {
        W.key[i] = i < n_raw ? (unsigned long long)__double_as_longlong(W.t[i]) : ~0ull;
        W.idx[i] = i;
    }
    __syncwarp();
    if (n_raw > 1) warp_bitonic_sort(W.key, W.idx, n_pad);
    // Permute (t, edge, info) into sorted order through registers.
    double rt[WX / 32];
    uint32_t re[WX / 32], ri[WX / 32];
#pragma unroll
    for (int s = 0; s < WX / 32; ++s) {
        int i = l + 32 * s;
        if (i < n_raw) {
            uint32_t j = W.idx[i];
            rt[s] = W.t[j];
            re[s] = W.edge[j];
            ri[s] = W.info[j];
        }
    }
    __syncwarp();
#pragma unroll
    for (int s = 0; s < WX / 32; ++s) {
        int i = l + 32 * s;
        if (i < n_raw) {
            W.t[i] = rt[s];
            W.edge[i] = re[s];
            W.info[i] = ri[s];
        }
    }
    __syncwarp();
    // Equal chainages (an edge found in several cells, or two edges meeting the ray at one point)
    // are ordered by (footprint, edge) like the reference's sort; such runs are short and rare.
    bool any_tie = false;
    for (int i = l + 1; i < n_raw; i += 32)
        if (W.t[i] == W.t[i - 1]) any_tie = true;
    if (__any_sync(FULL, any_tie)) {
        if (l == 0) {
            for (int i = 1; i < n_raw; ++i) {
                double tv = W.t[i];
                uint32_t ev = W.edge[i], iv = W.info[i];
                uint32_t fv = outline_fp(S, iv);
                int j = i - 1;
                while (j >= 0 && W.t[j] == tv) {
                    uint32_t fj = outline_fp(S, W.info[j]);
                    if (fj < fv || (fj == fv && W.edge[j] < ev)) break;
                    W.t[j + 1] = W.t[j];
                    W.edge[j + 1] = W.edge[j];
                    W.info[j + 1] = W.info[j];
                    --j;
                }
                W.t[j + 1] = tv;
                W.edge[j + 1] = ev;
                W.info[j + 1] = iv;
            }
        }
        __syncwarp();
    }
    // An edge listed in several cells meets the ray at one t: its copies sit side by side now and
    // merge (their flags are equal).
    {
        int n = 0;
        for (int base = 0; base < n_raw; base += 32) {
            int i = base + l;
            bool keep = false;
            double tv = 0.0;
            uint32_t ev = 0, iv = 0;
            if (i < n_raw) {
                tv = W.t[i];
                ev = W.edge[i];
                iv = W.info[i];
                keep = i == 0 || W.edge[i - 1] != ev;
            }
            unsigned mask = __ballot_sync(FULL, keep);
            int pos = n + __popc(mask & ((1u << l) - 1));
            __syncwarp();
            if (keep) {
                W.t[pos] = tv;
                W.edge[pos] = ev;
                W.info[pos] = iv;
            }
            n += __popc(mask);
            __syncwarp();
        }
        n_raw = n;
    }
    // One crossing per footprint and chainage within 1e-9 (crossings.rs:39-55): the window rarely
    // holds two crossings; when it does anywhere, lane 0 applies the rule in order.
    bool suspect = false;
    for (int i = l + 1; i < n_raw; i += 32)
        if (W.t[i] - W.t[i - 1] < 1e-9) suspect = true;
    int kept = 0;
    if (__any_sync(FULL, suspect)) {
        if (l == 0) {
            for (int i = 0; i < n_raw; ++i) {
                double tv = W.t[i];
                uint32_t fv = outline_fp(S, W.info[i]);
                bool merged = false;
                for (int k2 = kept - 1; k2 >= 0; --k2) {
                    if (!(tv - W.t[k2] < 1e-9)) break;
                    if (outline_fp(S, W.info[k2]) == fv) {
                        W.info[k2] |= W.info[i] & 0x80000000u;
                        merged = true;
                        break;
                    }
                }
                if (!merged) {
                    W.t[kept] = tv;
                    W.edge[kept] = W.edge[i];
                    W.info[kept] = W.info[i];
                    ++kept;
                }
            }
        }
        kept = __shfl_sync(FULL, kept, 0);
        __syncwarp();
    } else {
        kept = n_raw;
    }
    // The receiver's own walls (popup/src/evaluate.rs:293-297), compacted in order.
    if (rcv_own != 0) {
        int n = 0;
        for (int base = 0; base < kept; base += 32) {
            int i = base + l;
            bool keep = false;
            double tv = 0.0;
            uint32_t ev = 0, iv = 0;
            if (i < kept) {
                tv = W.t[i];
                ev = W.edge[i];
                iv = W.info[i];
                keep = outline_fp(S, iv) != rcv_own;
            }
            unsigned mask = __ballot_sync(FULL, keep);
            int pos = n + __popc(mask & ((1u << l) - 1));
            __syncwarp();
            if (keep) {
                W.t[pos] = tv;
                W.edge[pos] = ev;
                W.info[pos] = iv;
            }
            n += __popc(mask);
            __syncwarp();
        }
        kept = n;
    }
    return kept;
}

// ------------------------------------------------------------------------------------------------
// Terrain along the ray: the DEM-line merge (rows first on ties) and vertex evaluation.

struct RayTerrain {
    bool dem;
    long long rx, ry, dx, dy, adx, ady, sp;
    int col_step, row_step;
    long long next_col0, next_row0;  // first lines ahead
    Merge2 m;                        // A = column lines, B = row lines
    float length;
    float platform, source_ground;
    float2 start_zg, end_zg;

    __device__ void init(const SceneDev &S, int x0, int y0, int x1, int y1, float L, float platform_m) {
        dx = (long long)x1 - x0;
        dy = (long long)y1 - y0;
        adx = dx >= 0 ? dx : -dx;
        ady = dy >= 0 ? dy : -dy;
        length = L;
        dem = S.dem_nx != 0;
        start_zg = terrain_point(S, x0, y0);
        end_zg = terrain_point(S, x1, y1);
        platform = platform_m;
        source_ground = start_zg.x;
        m.na = m.nb = 0;
        if (!dem) return;
        sp = S.dem_sp;
        rx = (long long)x0 - S.dem_ox;
        ry = (long long)y0 - S.dem_oy;
        long long fc = floor_div64(rx, sp), fr = floor_div64(ry, sp);
        bool on_col = fc * sp == rx, on_row = fr * sp == ry;
        col_step = dx > 0 ? 1 : -1;
        row_step = dy > 0 ? 1 : -1;
        next_col0 = dx > 0 ? fc + 1 : (on_col ? fc - 1 : fc);
        next_row0 = dy > 0 ? fr + 1 : (on_row ? fr - 1 : fr);
        m.a0 = (next_col0 * sp - rx) * col_step;
        m.pa = sp;
        m.da = adx > 0 ? adx : 1;
        m.na = adx > 0 && m.a0 < adx ? (adx - m.a0 + sp - 1) / sp : 0;
        m.b0 = (next_row0 * sp - ry) * row_step;
        m.pb = sp;
        m.db = ady > 0 ? ady : 1;
        m.nb = ady > 0 && m.b0 < ady ? (ady - m.b0 + sp - 1) / sp : 0;
    }

    __device__ __forceinline__ long long inner() const { return m.na + m.nb; }

    // The inner vertex on column line index i (is_col) or row line j, with the platform clamp.
    __device__ __forceinline__ TV vertex(const SceneDev &S, bool is_col, long long k) const {
        TV v;
        if (is_col) {
            long long a = m.a0 + k * sp;
            long long line = next_col0 + k * col_step;
            // y on column line: (ry dx + (line sp - rx) dy) / (dx sp)
            long long num = (ry * dx + (line * sp - rx) * dy) * col_step, den = adx * sp;
            long long j0 = floor_div_pos(num, den);
            float f = (float)(num - j0 * den) / (float)den;
            float2 p = dem_node(S, line, j0), q = dem_node(S, line, j0 + 1);
            v = TV{(float)a / (float)adx * length, p.x + f * (q.x - p.x), p.y + f * (q.y - p.y)};
        } else {
            long long a = m.b0 + k * sp;
            long long line = next_row0 + k * row_step;
            long long num = (rx * dy + (line * sp - ry) * dx) * row_step, den = ady * sp;
            long long i0 = floor_div_pos(num, den);
            float f = (float)(num - i0 * den) / (float)den;
            float2 p = dem_node(S, i0, line), q = dem_node(S, i0 + 1, line);
            v = TV{(float)a / (float)ady * length, p.x + f * (q.x - p.x), p.y + f * (q.y - p.y)};
        }
        if (v.x < platform) v.z = fminf(v.z, source_ground);
        return v;
    }

    // The vertex with merged index k in [0, inner() + 2): 0 the source end, inner()+1 the receiver end.
    __device__ __forceinline__ TV vertex_at(const SceneDev &S, long long k) const {
        if (k == 0) return TV{0.0f, start_zg.x, start_zg.y};
        if (k == inner() + 1) {
            TV v{length, end_zg.x, end_zg.y};
            if (v.x < platform) v.z = fminf(v.z, source_ground);
            return v;
        }
        long long mi = k - 1;
        long long c1 = m.count_a(mi + 1, 0, 0), c0 = m.count_a(mi, 0, 0);
        return c1 > c0 ? vertex(S, true, c1 - 1) : vertex(S, false, mi - c0);
    }

    // The terrain at chainage t (as the reference's `interpolate` over the terrain polyline, ray.rs
    // :406-417): between the last vertex at or before x and the first one after it.
    __device__ float2 at_t(const SceneDev &S, double t, float x) const {
        if (!dem) return start_zg;
        // Inner vertices at or before t: columns with a0 + i sp <= t adx, rows likewise.
        long long nc = 0, nr = 0;
        if (m.na > 0) {
            double lim = t * (double)adx;
            long long c = (long long)floor((lim - (double)m.a0) / (double)sp) + 1;
            c = c < 0 ? 0 : (c > m.na ? m.na : c);
            nc = c;
        }
        if (m.nb > 0) {
            double lim = t * (double)ady;
            long long r = (long long)floor((lim - (double)m.b0) / (double)sp) + 1;
            r = r < 0 ? 0 : (r > m.nb ? m.nb : r);
            nr = r;
        }
        long long k = nc + nr;  // inner vertices before; the bracket is merged indices k and k + 1
        TV a = vertex_at(S, k), b = vertex_at(S, k + 1);
        // Float chainages may place x a hair outside the exact bracket; step to the reference's.
        while (a.x > x && k > 0) {
            --k;
            b = a;
            a = vertex_at(S, k);
        }
        while (b.x <= x && k + 1 < inner() + 1) {
            ++k;
            a = b;
            b = vertex_at(S, k + 1);
        }
        float f = b.x > a.x ? fminf(fmaxf((x - a.x) / (b.x - a.x), 0.f), 1.f) : 0.f;
        return make_float2(a.z + f * (b.z - a.z), a.g + f * (b.g - a.g));
    }
};

// ------------------------------------------------------------------------------------------------
// B. Tops and roofs (physics/src/ray.rs:293-323, 389-404)

__device__ inline void warp_tops_roofs(const SceneDev &S, const RayTerrain &T, int n_x, uint32_t own, float L,
                                       WarpShared &W, int &n_t, int &n_r, uint32_t &status) {
    const int l = lane_id();
    // Terrain (z, G) at each crossing, kept in W.t's storage as float2 once t is read.
    for (int i = l; i < n_x; i += 32) {
        double t = W.t[i];
        float x = (float)t * L;
        float2 zg = T.at_t(S, t, x);
        W.key[i] = ((unsigned long long)__float_as_uint(zg.y) << 32) | __float_as_uint(zg.x);
        W.top[i] = make_float2(x, 0.0f);
    }
    __syncwarp();
    // Containing footprints (ray.rs:201-226): the source's own and every footprint with an odd
    // count of roof-bounding crossings; they never screen it.
    n_t = 0;
    for (int base = 0; base < n_x; base += 32) {
        int i = base + l;
        bool keep = false;
        float2 tp{0.f, 0.f};
        if (i < n_x) {
            uint32_t info = W.info[i];
            uint32_t fp = outline_fp(S, info);
            keep = true;
            if (own != 0) {
                bool contained = fp == own;
                if (!contained) {
                    int cnt = 0;
                    for (int k = 0; k < n_x; ++k)
                        if ((W.info[k] & 0x80000000u) && outline_fp(S, W.info[k]) == fp) ++cnt;
                    contained = (cnt & 1) != 0;
                }
                keep = !contained;
            }
            float zt = __uint_as_float((uint32_t)W.key[i]);
            tp = make_float2(W.top[i].x, zt + S.outlines[info & 0x7fffffffu].height);
            if (!keep) W.info[i] &= 0x7fffffffu;  // a contained crossing bounds no roof
        }
        unsigned mask = __ballot_sync(FULL, keep);
        int pos = n_t + __popc(mask & ((1u << l) - 1));
        __syncwarp();
        if (keep) W.top[pos] = tp;  // pos <= i: in order, never ahead of a value still to read
        // The roof data of crossing i stays indexed by i: (x, top) are recomputed below from key/info.
        if (i < n_x) W.idx[i] = keep ? pos : 0xffffffffu;
        n_t += __popc(mask);
        __syncwarp();
    }
    // Roofs: each footprint's roof-bounding hits in order, paired consecutively: hit i opens a roof
    // when an even number of same-footprint hits precede it, with the next one as its end.
    n_r = 0;
    bool overflow = false;
    for (int base = 0; base < n_x; base += 32) {
        int i = base + l;
        bool opens = false;
        int partner = -1;
        if (i < n_x && (W.info[i] & 0x80000000u) && W.idx[i] != 0xffffffffu) {
            uint32_t fp = outline_fp(S, W.info[i]);
            int before = 0;
            for (int k = 0; k < i; ++k)
                if ((W.info[k] & 0x80000000u) && W.idx[k] != 0xffffffffu && outline_fp(S, W.info[k]) == fp) ++before;
            if ((before & 1) == 0)
                for (int k = i + 1; k < n_x; ++k)
                    if ((W.info[k] & 0x80000000u) && W.idx[k] != 0xffffffffu && outline_fp(S, W.info[k]) == fp) {
                        partner = k;
                        break;
                    }
            opens = partner >= 0;
        }
        unsigned mask = __ballot_sync(FULL, opens);
        int pos = n_r + __popc(mask & ((1u << l) - 1));
        if (opens) {
            if (pos < WR) {
                float2 a = W.top[W.idx[i]], b = W.top[W.idx[partner]];
                unsigned long long ka = W.key[i], kb = W.key[partner];
                W.r_x0[pos] = a.x;
                W.r_x1[pos] = b.x;
                W.r_top0[pos] = a.y;
                W.r_top1[pos] = b.y;
                W.r_zt0[pos] = __uint_as_float((uint32_t)ka);
                W.r_g0[pos] = __uint_as_float((uint32_t)(ka >> 32));
                W.r_zt1[pos] = __uint_as_float((uint32_t)kb);
                W.r_g1[pos] = __uint_as_float((uint32_t)(kb >> 32));
                W.r_fp[pos] = outline_fp(S, W.info[i]);
            } else {
                overflow = true;
            }
        }
        n_r += __popc(mask);
    }
    if (__any_sync(FULL, overflow)) {
        status |= FAILED_CAPACITY;
        n_r = 0;
        return;
    }
    __syncwarp();
    // Closing order (x1, x0, footprint), stable: roofs come out nearly sorted, lane 0 inserts.
    if (l == 0) {
        for (int i = 1; i < n_r; ++i) {
            float x0 = W.r_x0[i], x1 = W.r_x1[i], t0 = W.r_top0[i], t1 = W.r_top1[i], z0 = W.r_zt0[i], z1 = W.r_zt1[i];
            float g0 = W.r_g0[i], g1 = W.r_g1[i];
            uint32_t fp = W.r_fp[i];
            int j = i - 1;
            while (j >= 0 && (W.r_x1[j] > x1 || (W.r_x1[j] == x1 && (W.r_x0[j] > x0 || (W.r_x0[j] == x0 && W.r_fp[j] > fp))))) {
                W.r_x0[j + 1] = W.r_x0[j];
                W.r_x1[j + 1] = W.r_x1[j];
                W.r_top0[j + 1] = W.r_top0[j];
                W.r_top1[j + 1] = W.r_top1[j];
                W.r_zt0[j + 1] = W.r_zt0[j];
                W.r_zt1[j + 1] = W.r_zt1[j];
                W.r_g0[j + 1] = W.r_g0[j];
                W.r_g1[j + 1] = W.r_g1[j];
                W.r_fp[j + 1] = W.r_fp[j];
                --j;
            }
            W.r_x0[j + 1] = x0;
            W.r_x1[j + 1] = x1;
            W.r_top0[j + 1] = t0;
            W.r_top1[j + 1] = t1;
            W.r_zt0[j + 1] = z0;
            W.r_zt1[j + 1] = z1;
            W.r_g0[j + 1] = g0;
            W.r_g1[j + 1] = g1;
            W.r_fp[j + 1] = fp;
        }
        // clip_roofs_in_closing_order: a roof ending where cover already ends is dropped, one
        // starting under cover starts where the cover ends, its top interpolated there.
        float covered_to = -INFINITY, cov_zt = 0.f, cov_g = 0.f;
        int kept = 0;
        for (int i = 0; i < n_r; ++i) {
            float x0 = W.r_x0[i], x1 = W.r_x1[i], t0 = W.r_top0[i], t1 = W.r_top1[i];
            float z0 = W.r_zt0[i], z1 = W.r_zt1[i], g0 = W.r_g0[i], g1 = W.r_g1[i];
            if (x1 <= covered_to) continue;
            if (x0 < covered_to) {
                float span = x1 - x0;
                t0 += (covered_to - x0) / span * (t1 - t0);
                x0 = covered_to;
                z0 = cov_zt;
                g0 = cov_g;
            }
            covered_to = x1;
            cov_zt = z1;
            cov_g = g1;
            W.r_x0[kept] = x0;
            W.r_x1[kept] = x1;
            W.r_top0[kept] = t0;
            W.r_top1[kept] = t1;
            W.r_zt0[kept] = z0;
            W.r_zt1[kept] = z1;
            W.r_g0[kept] = g0;
            W.r_g1[kept] = g1;
            ++kept;
        }
        W.r_fp[0] = kept;  // hand the count over through shared memory
    }
    __syncwarp();
    n_r = n_r > 0 ? (int)W.r_fp[0] : 0;
    __syncwarp();
}

// ------------------------------------------------------------------------------------------------
// C. Crests (ray.rs:360-385): every terrain vertex within 300 m of an end, beyond it the highest of
// each 150 m group (the first of equals). Returns the count, or -1 over capacity.

__device__ inline int warp_crests(const SceneDev &S, const RayTerrain &T, float L, WarpShared &W) {
    const int l = lane_id();
    if (!T.dem) return 0;  // flat: the ends only, never inside (0, L)
    const long long n_vertices = T.inner() + 2;
    int n_k = 0;
    bool open = false;
    float2 best = make_float2(0.f, 0.f);
    long long at = 0;
    bool overflow = false;
    long long ia = 0, ib = 0;
    for (long long base = 0; base < n_vertices; base += 32) {
        long long k = base + l;
        TV v{0.f, 0.f, 0.f};
        bool valid = k < n_vertices;
        if (valid) v = T.vertex_at(S, k);
        (void)ia;
        (void)ib;
        bool middle = valid && v.x > 300.0f && v.x < L - 300.0f;
        long long group = valid ? (long long)floorf(v.x / 150.0f) : -1;
        // Segments of consecutive middle vertices of one group; a segment's best (max z, first of
        // equals) is emitted at its last vertex, the open segment carries across chunks.
        long long prev_group = __shfl_up_sync(FULL, group, 1);
        bool prev_middle = __shfl_up_sync(FULL, middle, 1);
        if (l == 0) {
            prev_group = open ? at : -2;
            prev_middle = open;
        }
        bool starts = middle && !(prev_middle && prev_group == group);
        // Segmented argmax by shuffles over runs (segment heads at `starts`).
        float bz = middle ? v.z : -INFINITY;
        float bx = v.x;
        // Carry the open group into lane 0's segment.
        if (l == 0 && middle && !starts) {
            if (!(v.z > best.y)) {
                bz = best.y;
                bx = best.x;
            }
        }
        // Inclusive segmented scan of (bz, bx) keeping the first maximum.
        int head = starts ? l : -1;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int h2 = __shfl_up_sync(FULL, head, o);
            if (l >= o && h2 > head) head = h2;
        }
        // head = index of this lane's segment head (or -1 when the segment began before the chunk).
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            float z2 = __shfl_up_sync(FULL, bz, o);
            float x2 = __shfl_up_sync(FULL, bx, o);
            int src = l - o;
            bool same = l >= o && src >= head && middle;
            if (same && z2 >= bz) {
                // The earlier one wins ties (first of equals).
                bz = z2;
                bx = x2;
            }
        }
        // A middle lane whose segment continues beyond the chunk or into the next lane stays open.
        long long next_group = __shfl_down_sync(FULL, group, 1);
        bool next_middle = __shfl_down_sync(FULL, middle, 1);
        bool last_in_chunk = l == 31 || !(base + l + 1 < n_vertices) ;
        if (l == 31) {
            next_middle = false;
            next_group = -3;
        }
        bool closes_here = middle && !last_in_chunk && !(next_middle && next_group == group);
        bool emit_self = valid && !middle;
        // Emission order by position: a closing segment emits its best, a non-middle vertex itself.
        bool emits = closes_here || emit_self;
        // The open segment from the previous chunk closes at lane 0 when lane 0 does not continue it.
        bool prev_open_closes = (l == 0) && open && !(middle && !starts);
        unsigned pmask = __ballot_sync(FULL, prev_open_closes);
        if (pmask) {
            if (l == 0) {
                if (n_k < WK)
                    W.crest[n_k] = best;
                else
                    overflow = true;
            }
            n_k += 1;
        }
        unsigned mask = __ballot_sync(FULL, emits);
        int pos = n_k + __popc(mask & ((1u << l) - 1));
        if (emits) {
            float2 c = closes_here ? make_float2(bx, bz) : make_float2(v.x, v.z);
            if (pos < WK)
                W.crest[pos] = c;
            else
                overflow = true;
        }
        n_k += __popc(mask);
        // The segment still open at the chunk's end (its last valid lane is middle and unclosed).
        int last_lane = (int)min((long long)31, n_vertices - 1 - base);
        bool lm = __shfl_sync(FULL, middle, last_lane);
        float obz = __shfl_sync(FULL, bz, last_lane), obx = __shfl_sync(FULL, bx, last_lane);
        long long og = __shfl_sync(FULL, group, last_lane);
        open = lm;
        if (open) {
            best = make_float2(obx, obz);
            at = og;
        }
    }
    if (open) {
        if (n_k < WK && l == 0) W.crest[n_k] = best;
        if (n_k >= WK) overflow = true;
        n_k += 1;
    }
    __syncwarp();
    return __any_sync(FULL, overflow) ? -1 : n_k;
}

// ------------------------------------------------------------------------------------------------
// D. Rubber bands: gift wrapping over the blocking candidates (or the best unblocked one).

struct BandResult {
    int np;           // band points (0: no candidate)
    bool blocked;
    float2 best;      // the unblocked candidate
};

// The state's ray leaves `a` toward `c` at this angle: the chord's, plus half the arc's central
// angle downwind (asin(chord / 2G)), which orders the arcs of one radius through `a` as they stand.
template <int STATE>
__device__ __forceinline__ float leave_angle(float radius, float2 a, float2 c) {
    float dx = c.x - a.x, dz = c.y - a.y;
    float ang = atan2f(dz, dx);
    if (STATE == QM_FAV) ang += asinf(fminf(sqrtf(dx * dx + dz * dz) / (2.0f * radius), 1.0f));
    return ang;
}

template <int STATE>
__device__ BandResult warp_band(const SceneDev &S, float2 Sp, float2 Rp, int n_k, int n_t, float L, WarpShared &W,
                                int &status_flags) {
    const int l = lane_id();
    BandResult res{0, false, make_float2(0.f, 0.f)};
    float dxr = Rp.x - Sp.x, dzr = Rp.y - Sp.y;
    float radius = fmaxf(1000.0f, 8.0f * sqrtf(dxr * dxr + dzr * dzr));
    Sag sag{};
    if (STATE == QM_FAV) sag = make_sag(radius, PlanePoint{Sp.x, Sp.y}, PlanePoint{Rp.x, Rp.y});
    const int n_c = n_k + n_t;
    // Blocking candidates, compacted in order (crests and tops as two sorted lists).
    int n_b = 0;
    bool overflow = false;
    for (int base = 0; base < n_c; base += 32) {
        int i = base + l;
        bool blocks = false;
        float2 c = make_float2(0.f, 0.f);
        if (i < n_c) {
            c = i < n_k ? W.crest[i] : W.top[i - n_k];
            if (c.x > 0.0f && c.x < L) {
                float line = chord_altitude(PlanePoint{Sp.x, Sp.y}, PlanePoint{Rp.x, Rp.y}, c.x);
                if (STATE == QM_FAV) line += sag.at(c.x - Sp.x);
                blocks = c.y > line;
            }
        }
        unsigned mask = __ballot_sync(FULL, blocks);
        int pos = n_b + __popc(mask & ((1u << l) - 1));
        if (blocks) {
            if (pos < WB)
                W.block()[pos] = c;
            else
                overflow = true;
        }
        n_b += __popc(mask);
    }
    if (__any_sync(FULL, overflow)) {
        status_flags |= FAILED_CAPACITY;
        return res;
    }
    __syncwarp();
    if (n_b > 0) {
        res.blocked = true;
        float2 a = Sp;
        int np = 0;
        for (int guard = 0; guard < WH + 1; ++guard) {
            // The steepest candidate beyond a (R included); ties to the farthest.
            float best_ang = leave_angle<STATE>(radius, a, Rp);
            float best_x = Rp.x;
            float2 best_c = Rp;
            for (int i = l; i < n_b; i += 32) {
                float2 c = W.block()[i];
                if (c.x <= a.x) continue;
                float ang = leave_angle<STATE>(radius, a, c);
                if (ang > best_ang || (ang == best_ang && c.x > best_x)) {
                    best_ang = ang;
                    best_x = c.x;
                    best_c = c;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                float oa = __shfl_xor_sync(FULL, best_ang, o);
                float ox = __shfl_xor_sync(FULL, best_x, o);
                float oz = __shfl_xor_sync(FULL, best_c.y, o);
                if (oa > best_ang || (oa == best_ang && ox > best_x)) {
                    best_ang = oa;
                    best_x = ox;
                    best_c = make_float2(ox, oz);
                }
            }
            if (best_c.x >= Rp.x) break;
            if (np >= WH) {
                status_flags |= FAILED_CAPACITY;
                break;
            }
            if (l == 0) W.hull[STATE][np] = best_c;
            ++np;
            a = best_c;
        }
        __syncwarp();
        res.np = np;
        return res;
    }
    // Unblocked: the candidate with the largest path difference, the first in candidate order
    // (by x, terrain first at equal x) among equals.
    float chord_sr = sqrtf(dxr * dxr + dzr * dzr);
    float best_v = -INFINITY;
    float2 best_c = make_float2(0.f, 0.f);
    float best_x = INFINITY;
    int best_kind = 2;
    bool have = false;
    for (int i = l; i < n_c; i += 32) {
        float2 c = i < n_k ? W.crest[i] : W.top[i - n_k];
        if (!(c.x > 0.0f && c.x < L)) continue;
        int kind = i < n_k ? 0 : 1;
        float v = single_path_difference_f<STATE>(radius, PlanePoint{Sp.x, Sp.y}, PlanePoint{c.x, c.y},
                                                  PlanePoint{Rp.x, Rp.y}, chord_sr);
        bool better = !have || v > best_v || (v == best_v && (c.x < best_x || (c.x == best_x && kind < best_kind)));
        if (better) {
            have = true;
            best_v = v;
            best_c = c;
            best_x = c.x;
            best_kind = kind;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        float ov = __shfl_xor_sync(FULL, best_v, o);
        float ox = __shfl_xor_sync(FULL, best_c.x, o);
        float oz = __shfl_xor_sync(FULL, best_c.y, o);
        int ok = __shfl_xor_sync(FULL, best_kind, o);
        bool oh = __shfl_xor_sync(FULL, have, o);
        bool better = oh && (!have || ov > best_v || (ov == best_v && (ox < best_c.x || (ox == best_c.x && ok < best_kind))));
        if (better) {
            have = true;
            best_v = ov;
            best_c = make_float2(ox, oz);
            best_kind = ok;
        }
    }
    if (have) {
        res.np = 1;
        res.best = best_c;
        if (l == 0) W.hull[STATE][0] = best_c;
    }
    __syncwarp();
    return res;
}

// ------------------------------------------------------------------------------------------------
// E. Integrals of the vertical profile over ranges (mean_plane.rs:204-249, mod.rs:42-58): the
// terrain polyline, with each roof's span replaced by its roof line (G = 0 there).

struct Range {
    float a, b;    // [a, b]
    float xo, zo;  // origin
};

// The profile's upper-side value at x (ground_altitude_at): a roof's line on [x0, x1), else terrain.
__device__ inline float2 profile_at(const SceneDev &S, const RayTerrain &T, const WarpShared &W, int n_r, double t_hint,
                                    float x) {
    for (int r = 0; r < n_r; ++r)
        if (x >= W.r_x0[r] && x < W.r_x1[r]) {
            float span = W.r_x1[r] - W.r_x0[r];
            float f = span > 0.f ? (x - W.r_x0[r]) / span : 0.f;
            return make_float2(W.r_top0[r] + f * (W.r_top1[r] - W.r_top0[r]), 0.0f);
        }
    return T.at_t(S, t_hint, x);
}

// Adds the piece [p0, p1] of a linear stretch (z0 at x0 .. z1 at x1, G likewise) clipped to each range.
__device__ __forceinline__ void add_piece(Moments *acc, const Range *R, int nR, float x0, float z0, float g0, float x1,
                                          float z1, float g1, float p0, float p1) {
    float span = x1 - x0;
    for (int q = 0; q < nR; ++q) {
        float a = fmaxf(p0, R[q].a), b = fminf(p1, R[q].b);
        if (!(b > a)) continue;
        float fa = span > 0.f ? (a - x0) / span : 0.f, fb = span > 0.f ? (b - x0) / span : 0.f;
        float za = z0 + fa * (z1 - z0), zb = z0 + fb * (z1 - z0);
        float ga = g0 + fa * (g1 - g0), gb = g0 + fb * (g1 - g0);
        add_stretch(acc[q], R[q].xo, R[q].zo, a, za, ga, b, zb, gb);
    }
}

template <int NR_MAX>
__device__ void warp_profile_moments(const SceneDev &S, const RayTerrain &T, const WarpShared &W, int n_r, float L,
                                     const Range *R, int nR, Moments *out) {
    const int l = lane_id();
    Moments acc[NR_MAX];
#pragma unroll
    for (int q = 0; q < NR_MAX; ++q) acc[q] = moments_zero();
    const long long n_vertices = T.inner() + 2;
    // Terrain stretches outside the roofs: lane l holds vertex base + l, its neighbour by shuffle.
    for (long long base = 0; base < n_vertices - 1; base += 32) {
        long long k = base + l;
        TV a{0.f, 0.f, 0.f};
        if (k < n_vertices) a = T.vertex_at(S, k);
        TV b;
        b.x = __shfl_down_sync(FULL, a.x, 1);
        b.z = __shfl_down_sync(FULL, a.z, 1);
        b.g = __shfl_down_sync(FULL, a.g, 1);
        if (l == 31 && k + 1 < n_vertices) b = T.vertex_at(S, k + 1);
        if (k < n_vertices - 1 && b.x > a.x) {
            // First roof ending after a.x (roofs are disjoint, sorted by their ends).
            int lo = 0, hi = n_r;
            while (lo < hi) {
                int mid = (lo + hi) >> 1;
                if (W.r_x1[mid] <= a.x)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            float p = a.x;
            for (int r = lo; r < n_r && p < b.x; ++r) {
                if (W.r_x0[r] >= b.x) break;
                if (W.r_x0[r] > p) add_piece(acc, R, nR, a.x, a.z, a.g, b.x, b.z, b.g, p, W.r_x0[r]);
                p = fmaxf(p, W.r_x1[r]);
            }
            if (p < b.x) add_piece(acc, R, nR, a.x, a.z, a.g, b.x, b.z, b.g, p, b.x);
        }
    }
    // The roofs' lines (hard ground, G = 0).
    for (int r = l; r < n_r; r += 32)
        add_piece(acc, R, nR, W.r_x0[r], W.r_top0[r], 0.0f, W.r_x1[r], W.r_top1[r], 0.0f, W.r_x0[r], W.r_x1[r]);
#pragma unroll
    for (int q = 0; q < NR_MAX; ++q) {
        if (q >= nR) break;
        out[q].z = warp_sum(acc[q].z);
        out[q].xz = warp_sum(acc[q].xz);
        out[q].g = warp_sum(acc[q].g);
        out[q].len = warp_sum(acc[q].len);
    }
}

// ------------------------------------------------------------------------------------------------
// F. The boundary of one state, one band per lane (diffraction.rs:64-197). Every lane of the warp
// calls it (lanes 8k..8k+7 for state k & 1); the four path differences of a state are taken once, on
// that state's lanes 0-3, and shared.

__device__ inline float lane_state_boundary(int state, int b, const EqGeometry &direct, float path_ground,
                                            float near_source, float source_gf, const WarpShared &W,
                                            const BandResult &res, float2 Sp, float2 Rp, const Moments &src_m,
                                            float first_x, float z0, float g0, const Moments &rcv_m, float last_x,
                                            float last_zat, float last_gat, float L) {
    const int l = lane_id();
    float whole = ground_attenuation_band(direct, source_side_factors(state, path_ground, near_source), state, b);
    const PlanePoint *points = reinterpret_cast<const PlanePoint *>(W.hull[state]);
    const int np = res.np;
    float dxr = Rp.x - Sp.x, dzr = Rp.y - Sp.y;
    double radius = fmaxf(1000.0f, 8.0f * sqrtf(dxr * dxr + dzr * dzr));
    PointD Sd{Sp.x, Sp.y}, Rd{Rp.x, Rp.y};
    PlanePoint first = np > 0 ? points[0] : PlanePoint{0.5f * L, 0.f};
    PlanePoint last = np > 0 ? points[np - 1] : first;
    MeanPlane sp = plane_of(src_m, 0.0f, first.x, z0);
    EqGeometry source_side = geometry_over(sp, PlanePoint{Sp.x, Sp.y}, first);
    float rlen = L - last_x;
    MeanPlane rp = plane_of(rcv_m, last_x, rlen, last_zat);
    EqGeometry receiver_side = geometry_over(rp, last, PlanePoint{Rp.x, Rp.y});
    PointD Si, Ri;
    mirror_d(sp, Sp.x, Sp.y, Si.x, Si.z);
    mirror_d(rp, Rp.x, Rp.y, Ri.x, Ri.z);
    // The state's path differences: delta, source image, receiver image, Rayleigh's S*R*.
    int j = l & 7;
    double mine = 0.0;
    if (np > 0 && j < 4 && !(j == 3 && res.blocked)) {
        PointD from = (j == 1 || j == 3) ? Si : Sd;
        PointD to = (j == 2 || j == 3) ? Ri : Rd;
        mine = path_difference_d(state, radius, from, points, np, to);
    }
    int g0l = l & ~7;
    double delta = __shfl_sync(FULL, mine, g0l);
    double delta_si = __shfl_sync(FULL, mine, g0l + 1);
    double delta_ri = __shfl_sync(FULL, mine, g0l + 2);
    double rayleigh_star = __shfl_sync(FULL, mine, g0l + 3);
    if (np == 0) return whole;
    float span = 0.0f;
    for (int i = 0; i + 1 < np; ++i) {
        float dx = points[i + 1].x - points[i].x, dz = points[i + 1].z - points[i].z;
        float chord = sqrtf(dx * dx + dz * dz);
        span += chord + (state == QM_FAV ? arc_excess_f<QM_FAV>(chord, (float)radius) : 0.0f);
    }
    float c2 = 1.0f;
    if (np > 1 && span > MULTIPLE_DIFFRACTION_MINIMUM_SPAN) {
        float x = 5.0f * c_band.lambda[b] / span;
        c2 = (1.0f + x * x) / (1.0f / 3.0f + x * x);
    }
    bool admitted = res.blocked || (delta > -c_band.lambda_over_20_d[b] && delta > c_band.lambda_over_4_d[b] - rayleigh_star);
    if (!admitted) return whole;
    float source_side_ground = mean_ground_of(src_m, first.x, g0);
    float source_side_near = ground_factor_near_source(source_side, source_side_ground, source_gf);
    float ground_so =
        ground_attenuation_band(source_side, source_side_factors(state, source_side_ground, source_side_near), state, b);
    float receiver_side_ground = mean_ground_of(rcv_m, rlen, last_gat);
    float ground_or = ground_attenuation_band(
        receiver_side, GroundFactors{receiver_side_ground, receiver_side_ground, receiver_side_ground}, state, b);
    float direct_db = diffraction_db((float)delta, c2, b);
    float source_image_db = diffraction_db((float)delta_si, c2, b);
    float receiver_image_db = diffraction_db((float)delta_ri, c2, b);
    float sr = direct_db;
    float split_so;
    if (source_side.source_below) {
        sr = source_image_db;
        split_so = ground_so;
    } else {
        split_so = ground_split_db(ground_so, source_image_db, direct_db);
    }
    if (!isfinite(split_so)) {
        split_so = ground_so;
        sr = source_image_db;
    }
    float split_or;
    if (receiver_side.receiver_below) {
        sr = receiver_image_db;
        split_or = ground_or;
    } else {
        split_or = ground_split_db(ground_or, receiver_image_db, sr);
    }
    if (!isfinite(split_or)) {
        split_or = ground_or;
        sr = receiver_image_db;
    }
    return fminf(fmaxf(sr, 0.0f), DIFFRACTION_CAP_DB) + split_so + split_or;
}

// ------------------------------------------------------------------------------------------------
// One path by one warp. On return every lane holds out.status, slant, weight, p; lane b (< 8) holds
// the homogeneous boundary transfer of band b in out.boundary[0][0] and the favourable one in
// out.boundary[1][0].

__device__ void warp_evaluate_path(const SceneDev &S, const SourceDev &src, int rx, int ry, float rcv_alt,
                                   uint32_t rcv_own, bool want_fav, WarpShared &W, PathResult &out) {
    const int l = lane_id();
    out.status = 0;
    out.edges_tested = 0;
    out.vertices = 0;
    out.candidates = 0;
    const int sx = src.x, sy = src.y;
    const float dxm = (float)(rx - sx) * S.step_m, dym = (float)(ry - sy) * S.step_m;
    const float dist = sqrtf(dxm * dxm + dym * dym);
    const float L = fmaxf(dist, 1.0f);
    uint32_t status = 0, tested = 0;
    int n_x = warp_crossings(S, sx, sy, rx, ry, rcv_own, W, status, tested);
    out.crossings = n_x;
    out.edges_tested = tested;
    RayTerrain T;
    T.init(S, sx, sy, rx, ry, L, src.platform);
    const float z0 = T.start_zg.x, g0 = T.start_zg.y;
    const float src_alt = z0 + src.height;
    int n_t = 0, n_r = 0;
    if (!status) warp_tops_roofs(S, T, n_x, src.fp, L, W, n_t, n_r, status);
    int n_k = 0;
    if (!status) {
        n_k = warp_crests(S, T, L, W);
        if (n_k < 0) {
            status |= FAILED_CAPACITY;
            n_k = 0;
        }
    }
    out.vertices = (uint32_t)(T.inner() + 2) + 4u * n_r;
    out.candidates = n_k + n_t;
    const float2 Sp = make_float2(0.0f, src_alt), Rp = make_float2(L, rcv_alt);
    int flags = (int)status;
    BandResult bh{0, false}, bf{0, false};
    if (!status) {
        bh = warp_band<QM_HOM>(S, Sp, Rp, n_k, n_t, L, W, flags);
        if (want_fav) bf = warp_band<QM_FAV>(S, Sp, Rp, n_k, n_t, L, W, flags);
    }
    status = (uint32_t)flags;
    // Ranges: direct, then per state its source side and receiver side.
    Range R[5];
    int nR = 0;
    R[nR++] = Range{0.0f, L, 0.0f, z0};
    float first_x[2] = {0.f, 0.f}, last_x[2] = {0.f, 0.f}, last_zat[2] = {0.f, 0.f}, last_gat[2] = {0.f, 0.f};
    int src_q[2] = {-1, -1}, rcv_q[2] = {-1, -1};
    BandResult bands[2] = {bh, bf};
    for (int st = 0; st < (want_fav ? 2 : 1); ++st) {
        if (status || bands[st].np == 0) continue;
        int np = bands[st].np;
        float2 fpnt = W.hull[st][0], lpnt = W.hull[st][np - 1];
        first_x[st] = fpnt.x;
        last_x[st] = lpnt.x;
        float2 zg = profile_at(S, T, W, n_r, (double)(lpnt.x / L), lpnt.x);
        last_zat[st] = zg.x;
        last_gat[st] = zg.y;
        src_q[st] = nR;
        R[nR++] = Range{0.0f, fpnt.x, 0.0f, z0};
        rcv_q[st] = nR;
        R[nR++] = Range{lpnt.x, L, lpnt.x, zg.x};
    }
    Moments M[5];
    if (!status) warp_profile_moments<5>(S, T, W, n_r, L, R, nR, M);
    out.status = status;
    // Boundaries: lane = state * 8 + band.
    MeanPlane dplane = plane_of(M[0], 0.0f, L, z0);
    EqGeometry direct = geometry_over(dplane, PlanePoint{Sp.x, Sp.y}, PlanePoint{Rp.x, Rp.y});
    float path_ground = mean_ground_of(M[0], L, g0);
    float source_gf = src.gf >= 0.0f ? src.gf : g0;
    float near_source = ground_factor_near_source(direct, path_ground, source_gf);
    float att = 0.0f;
    int st = (l >> 3) & 1, b = l & 7;
    if (!status) {  // warp-uniform: every lane takes part (lanes 16-31 repeat states 0 and 1)
        Moments sm = src_q[st] >= 0 ? M[src_q[st]] : moments_zero();
        Moments rm = rcv_q[st] >= 0 ? M[rcv_q[st]] : moments_zero();
        att = lane_state_boundary(st, b, direct, path_ground, near_source, source_gf, W, bands[st], Sp, Rp, sm,
                                  first_x[st], z0, g0, rm, last_x[st], last_zat[st], last_gat[st], L);
    }
    float tr = __expf(-att * LN10_OVER_10);
    float hom = __shfl_sync(FULL, tr, b);
    float fav = want_fav ? __shfl_sync(FULL, tr, 8 + b) : hom;
    out.boundary[0][0] = hom;
    out.boundary[1][0] = fav;
    float dz = rcv_alt - src_alt;
    out.slant = fmaxf(sqrtf(L * L + dz * dz), 1.0f);
    float dh = fmaxf(dist, src.excl);
    float d = fmaxf(sqrtf(dh * dh + dz * dz), 1.0f);
    out.weight = 1.0f / (d * d * 12.589254117941673f);
    float azimuth = atan2f(dym, dxm);
#pragma unroll
    for (int p = 0; p < QM_PERIODS; ++p) out.p[p] = want_fav ? favourable_at(S.fav[p], azimuth) : 0.0f;
    __syncwarp();
}

// The grid painter with one warp per path: CTA = 4 warps over 4 receivers of the grid and a chunk
// of sources; lane b (< 8) keeps band b's compensated day sum, lane 8 the Lden sum.
__global__ void __launch_bounds__(128) paint_grid_warp_kernel(SceneDev S, GridArgs A) {
    extern __shared__ unsigned char smem_raw[];
    WarpShared &W = reinterpret_cast<WarpShared *>(smem_raw)[threadIdx.x >> 5];
    __shared__ unsigned long long s_counts[6];
    if (threadIdx.x < 6) s_counts[threadIdx.x] = 0;
    __syncthreads();
    const int l = lane_id();
    const int cell = blockIdx.x * 4 + (threadIdx.x >> 5);
    const int chunk = blockIdx.y;
    const int cells = A.nx * A.ny;
    unsigned long long paths = 0, crossings = 0, tested = 0, failed_paths = 0, vertices = 0, candidates = 0;
    if (cell < cells) {
        const int ix = cell % A.nx, iy = cell / A.nx;
        const int rx = A.origin_x + ix * A.spacing, ry = A.origin_y + iy * A.spacing;
        const float alt = A.rcv_alt[cell];
        const uint32_t own = A.rcv_own[cell];
        KSum acc{0.f, 0.f};
        uint32_t failed = 0;
        const uint32_t s0 = A.source_begin + chunk * A.chunk;
        const uint32_t s1 = min(s0 + A.chunk, A.source_end);
        for (uint32_t s = s0; s < s1; ++s) {
            const SourceDev &src = S.sources[s];
            PathResult r;
            warp_evaluate_path(S, src, rx, ry, alt, own, A.want_fav, W, r);
            ++paths;
            crossings += r.crossings;
            tested += r.edges_tested;
            vertices += r.vertices;
            candidates += r.candidates;
            if (r.status) {
                failed |= r.status;
                ++failed_paths;
                if (l == 0) {
                    unsigned int slot = atomicAdd(A.retry_count, 1u);
                    if (slot < A.retry_cap) A.retry[slot] = make_uint2((uint32_t)cell, s);
                }
                continue;
            }
            // Lane b: band b's energy per period; the Lden-weighted A sum over bands by warp sum.
            float air = l < 8 ? __expf(-S.air_per_m[l] * r.slant) : 0.f;
            float lsum = 0.f, day = 0.f;
            if (l < 8) {
#pragma unroll
                for (int p = 0; p < QM_PERIODS; ++p) {
                    float pp = r.p[p];
                    float t = air * (pp * r.boundary[1][0] + (1.0f - pp) * r.boundary[0][0]);
                    float e = r.weight * __ldg(&src.energy[p * QM_BANDS + l]) * t;
                    if (p == 0) day = e;
                    lsum += A.lden_w[p] * e;
                }
            }
            lsum = warp_sum(lsum);
            if (l < 8) acc.add(day);
            if (l == 8) acc.add(lsum);
        }
        float *out = A.partial + ((size_t)chunk * cells + cell) * GRID_SLOTS;
        if (l < GRID_SLOTS) out[l] = acc.value();
        if (failed && l == 0) atomicOr(A.failed + cell, failed);
    }
    if (l == 0) {
        atomicAdd(&s_counts[0], paths);
        atomicAdd(&s_counts[1], crossings);
        atomicAdd(&s_counts[2], tested);
        atomicAdd(&s_counts[3], failed_paths);
        atomicAdd(&s_counts[4], vertices);
        atomicAdd(&s_counts[5], candidates);
    }
    __syncthreads();
    if (threadIdx.x < 6) atomicAdd(A.counters + threadIdx.x, s_counts[threadIdx.x]);
}

}  // namespace qm
