// Device physics of one source-receiver path in the vertical plane, FP32 (FP64 only for path
// differences delta). CNOSSOS-EU 2.5 ground and diffraction as the reference's Rust states it:
// physics/src/cnossos/{mean_plane,ground,rubber_band,diffraction}.rs. The vertical profile is never
// stored: mean planes and mean ground factors come from segment moments the walk sums
// (qm_path.cuh), so every function here takes moments, not polylines.
#pragma once

#include <cstdint>

#define QM_BANDS 8
#define QM_PERIODS 3
#define QM_SECTORS 16
#define QM_HOM 0
#define QM_FAV 1

namespace qm {

// Band constants computed on the host in double and rounded once (the reference does the same:
// paint-gpu/src/device.rs:57-77): f^2.5, f^1.5, f^0.75, wavenumber k, wavelength lambda.
struct BandConstants {
    float f25[QM_BANDS];
    float f15[QM_BANDS];
    float f075[QM_BANDS];
    float k[QM_BANDS];
    float lambda[QM_BANDS];
    float inv_lambda[QM_BANDS];
    double lambda_d[QM_BANDS];
    double lambda_over_20_d[QM_BANDS];  // lambda / 20 and lambda / 4, exactly as the criteria divide
    double lambda_over_4_d[QM_BANDS];
};

// Defined once: only the library's main translation unit includes this header.
__constant__ BandConstants c_band;

constexpr float LN10_OVER_10 = 0.2302585092994046f;
constexpr float LOG10_2 = 0.30102999566398120f;

__device__ __forceinline__ float log10_fast(float x) { return __log2f(x) * LOG10_2; }
__device__ __forceinline__ float energy_of(float level_db) { return __expf(level_db * LN10_OVER_10); }
__device__ __forceinline__ float amplitude_of(float level_db) { return __expf(level_db * (LN10_OVER_10 * 0.5f)); }

struct PlanePoint {
    float x, z;
};

// Integrals of the ground over a range, about the range's origin (x_o, z_o):
// z = int (z - z_o) dx, xz = int (x - x_o)(z - z_o) dx, g = int G dx, len = range length.
struct Moments {
    float z, xz, g, len;
};

__device__ __forceinline__ Moments moments_zero() { return Moments{0.f, 0.f, 0.f, 0.f}; }

// One linear stretch (a, za, ga) -> (b, zb, gb) added exactly (mean_plane.rs:217-227; the
// trapezoid of VerticalProfile::mean_ground_factor, mod.rs:52-55).
__device__ __forceinline__ void add_stretch(Moments &m, float xo, float zo, float a, float za, float ga, float b,
                                            float zb, float gb) {
    float width = b - a;
    if (width <= 0.0f) return;
    float u0 = a - xo, u1 = b - xo, w0 = za - zo, w1 = zb - zo;
    m.z += 0.5f * (w0 + w1) * width;
    m.xz += width * (u0 * (2.0f * w0 + w1) + u1 * (w0 + 2.0f * w1)) * (1.0f / 6.0f);
    m.g += 0.5f * (ga + gb) * width;
    m.len += width;
}

// Moments about (x1, z1) re-taken about (x0, z0) (the range starts at x1).
__device__ __forceinline__ Moments rebase(const Moments &m, float x1, float z1, float x0, float z0) {
    float dx = x1 - x0, dz = z1 - z0;
    Moments r;
    r.z = m.z + dz * m.len;
    r.xz = m.xz + dx * m.z + dz * (0.5f * m.len * m.len + dx * m.len);
    r.g = m.g;
    r.len = m.len;
    return r;
}

// Two adjacent ranges about the first one's origin.
__device__ __forceinline__ Moments join(const Moments &a, const Moments &b_about_a) {
    return Moments{a.z + b_about_a.z, a.xz + b_about_a.xz, a.g + b_about_a.g, a.len + b_about_a.len};
}

struct MeanPlane {
    float slope, intercept;
};

// fit_mean_plane (mean_plane.rs:204-249) of the range [start, start + length] from its moments about
// (start, z_ref); a range under a millimetre is a level plane through z_ref.
__device__ __forceinline__ MeanPlane plane_of(const Moments &m, float start, float length, float z_ref) {
    if (length < 1e-3f) return MeanPlane{0.0f, z_ref};
    float slope = 12.0f * (m.xz - 0.5f * length * m.z) / (length * length * length);
    return MeanPlane{slope, z_ref + (m.z / length - 0.5f * slope * length) - slope * start};
}

// VerticalProfile::mean_ground_factor (mod.rs:42-58) from the range's moments.
__device__ __forceinline__ float mean_ground_of(const Moments &m, float length, float g_at_start) {
    return length < 1e-3f ? g_at_start : m.g / length;
}

__device__ __forceinline__ float plane_altitude(const MeanPlane &p, float x) { return p.slope * x + p.intercept; }

struct EqGeometry {
    MeanPlane plane;
    float zs, zr;
    bool source_below, receiver_below;
    float dp;
};

// EquivalentGeometry::over (mean_plane.rs:293-306).
__device__ __forceinline__ EqGeometry geometry_over(const MeanPlane &p, PlanePoint from, PlanePoint to) {
    float inv = rsqrtf(1.0f + p.slope * p.slope);
    float hs = (from.z - plane_altitude(p, from.x)) * inv;
    float hr = (to.z - plane_altitude(p, to.x)) * inv;
    EqGeometry g;
    g.plane = p;
    g.zs = fmaxf(hs, 0.0f);
    g.zr = fmaxf(hr, 0.0f);
    g.source_below = hs < 0.0f;
    g.receiver_below = hr < 0.0f;
    g.dp = fabsf((to.x - from.x) + p.slope * (to.z - from.z)) * inv;
    return g;
}

// MeanPlane::mirror (mean_plane.rs:274-278), in double for the images' path differences.
__device__ __forceinline__ void mirror_d(const MeanPlane &p, double x, double z, double &ox, double &oz) {
    double slope = p.slope;
    double norm_sq = 1.0 + slope * slope;
    double offset = (z - (slope * x + (double)p.intercept)) / norm_sq;
    ox = x + 2.0 * offset * slope;
    oz = z - 2.0 * offset;
}

// ---------------------------------------------------------------------------------------------
// Ground: physics/src/cnossos/ground.rs
constexpr float SHORT_PATH_HEIGHT_FACTOR = 30.0f;
constexpr float FAVOURABLE_CURVATURE_A0 = 2e-4f;
constexpr float FAVOURABLE_TERRAIN_COEFF = 6e-3f;
constexpr float MINIMUM_HEIGHT_SUM = 1e-3f;
constexpr float HARD_GROUND_BELOW = 1e-3f;

struct GroundFactors {
    float path, impedance, floor;
};

// ground.rs:40-53
__device__ __forceinline__ float ground_factor_near_source(const EqGeometry &g, float path_gf, float source_gf) {
    float height_sum = fmaxf(g.zs + g.zr, MINIMUM_HEIGHT_SUM);
    float ratio = g.dp / (SHORT_PATH_HEIGHT_FACTOR * height_sum);
    return ratio <= 1.0f ? path_gf * ratio + source_gf * (1.0f - ratio) : path_gf;
}

// ground.rs:78-89
__device__ __forceinline__ float analytic_ground_db(int b, float dp, float zs, float zr, float gw13) {
    float k = c_band.k[b];
    float gw26 = gw13 * gw13;
    float w = 0.0185f * c_band.f25[b] * gw26 / (c_band.f15[b] * gw26 + 1.3e3f * c_band.f075[b] * gw13 + 1.16e6f);
    float wd = w * dp;
    float cf = dp * (1.0f + 3.0f * wd * __expf(-sqrtf(wd))) / (1.0f + wd);
    float cfk = cf / k;
    float root = sqrtf(2.0f * cfk);
    float product = (zs * zs - root * zs + cfk) * (zr * zr - root * zr + cfk);
    return -10.0f * log10_fast(4.0f * k * k / (dp * dp) * product);
}

// ground.rs:92-102
__device__ __forceinline__ float favourable_floor_db(const EqGeometry &g, float floor_factor) {
    float height_sum = fmaxf(g.zs + g.zr, MINIMUM_HEIGHT_SUM);
    float base = -3.0f * (1.0f - floor_factor);
    float limit = SHORT_PATH_HEIGHT_FACTOR * height_sum;
    return g.dp <= limit ? base : base * (1.0f + 2.0f * (1.0f - limit / g.dp));
}

// ground.rs:105-139
// Out of line: called three times per state; inlining each copy would crowd the instruction
// cache the crossing walk needs.
__device__ __noinline__ void ground_attenuation_bands(const EqGeometry &g, GroundFactors f, int state,
                                                      float out[QM_BANDS]) {
    float dp = fmaxf(g.dp, 1e-6f);
    float zs = g.zs, zr = g.zr;
    float imp = fmaxf(f.impedance, 0.0f);
    float gw13 = imp > 0.0f ? __expf(1.3f * __logf(imp)) : 0.0f;
    if (state == QM_HOM) {
        if (f.path < HARD_GROUND_BELOW) {
#pragma unroll
            for (int b = 0; b < QM_BANDS; ++b) out[b] = -3.0f;
            return;
        }
        float floor = -3.0f * (1.0f - f.floor);
#pragma unroll
        for (int b = 0; b < QM_BANDS; ++b) out[b] = fmaxf(analytic_ground_db(b, dp, zs, zr, gw13), floor);
    } else {
        float floor = favourable_floor_db(g, f.floor);
        if (f.path < HARD_GROUND_BELOW) {
#pragma unroll
            for (int b = 0; b < QM_BANDS; ++b) out[b] = floor;
            return;
        }
        float height_sum = fmaxf(zs + zr, MINIMUM_HEIGHT_SUM);
        float curvature = FAVOURABLE_CURVATURE_A0 * dp * dp * 0.5f;
        float terrain = FAVOURABLE_TERRAIN_COEFF * dp / height_sum;
        float rs = zs / height_sum, rr = zr / height_sum;
        float zsf = zs + curvature * rs * rs + terrain;
        float zrf = zr + curvature * rr * rr + terrain;
#pragma unroll
        for (int b = 0; b < QM_BANDS; ++b) out[b] = fmaxf(analytic_ground_db(b, dp, zsf, zrf, gw13), floor);
    }
}

// One band of ground_attenuation_bands (ground.rs:105-139), for a lane that owns that band.
__device__ __noinline__ float ground_attenuation_band(const EqGeometry &g, GroundFactors f, int state, int b) {
    float dp = fmaxf(g.dp, 1e-6f);
    float zs = g.zs, zr = g.zr;
    float imp = fmaxf(f.impedance, 0.0f);
    float gw13 = imp > 0.0f ? __expf(1.3f * __logf(imp)) : 0.0f;
    if (state == QM_HOM) {
        if (f.path < HARD_GROUND_BELOW) return -3.0f;
        return fmaxf(analytic_ground_db(b, dp, zs, zr, gw13), -3.0f * (1.0f - f.floor));
    }
    float floor = favourable_floor_db(g, f.floor);
    if (f.path < HARD_GROUND_BELOW) return floor;
    float height_sum = fmaxf(zs + zr, MINIMUM_HEIGHT_SUM);
    float curvature = FAVOURABLE_CURVATURE_A0 * dp * dp * 0.5f;
    float terrain = FAVOURABLE_TERRAIN_COEFF * dp / height_sum;
    float rs = zs / height_sum, rr = zr / height_sum;
    return fmaxf(analytic_ground_db(b, dp, zs + curvature * rs * rs + terrain, zr + curvature * rr * rr + terrain, gw13),
                 floor);
}

// diffraction.rs:200-213
__device__ __forceinline__ GroundFactors source_side_factors(int state, float path_ground, float near_source) {
    return GroundFactors{path_ground, state == QM_HOM ? near_source : path_ground, near_source};
}

// ---------------------------------------------------------------------------------------------
// Rubber band: physics/src/cnossos/rubber_band.rs

__device__ __forceinline__ float chord_altitude(PlanePoint from, PlanePoint to, float x) {
    return from.z + (to.z - from.z) * (x - from.x) / (to.x - from.x);
}

// Favourable-ray height above the S-R chord (rubber_band.rs:319-340); zero homogeneous.
struct Sag {
    float along_per_x, chord, gamma2, centre_term;
    __device__ __forceinline__ float at(float x_from_source) const {
        float along = x_from_source * along_per_x;
        float offset = along - 0.5f * chord;
        float perpendicular = along * (chord - along) / (sqrtf(fmaxf(gamma2 - offset * offset, 0.0f)) + centre_term);
        return perpendicular * along_per_x;
    }
};

__device__ __forceinline__ Sag make_sag(float radius, PlanePoint source, PlanePoint receiver) {
    float horizontal = receiver.x - source.x;
    float dx = receiver.x - source.x, dz = receiver.z - source.z;
    float chord = sqrtf(dx * dx + dz * dz);
    float gamma2 = radius * radius;
    return Sag{chord / horizontal, chord, gamma2, sqrtf(gamma2 - 0.25f * chord * chord)};
}

// The state's ray altitude at x on the leg from -> to (chord plus the favourable sag).
template <int STATE>
__device__ __forceinline__ float ray_altitude(float radius, PlanePoint from, PlanePoint to, float x) {
    float c = chord_altitude(from, to, x);
    if (STATE == QM_HOM) return c;
    return c + make_sag(radius, from, to).at(x - from.x);
}

// The arc's excess over its chord, 2 G asin(l / 2G) - l (rubber_band.rs:231-251), FP32 (screening).
template <int STATE>
__device__ __forceinline__ float arc_excess_f(float chord, float radius) {
    if (STATE == QM_HOM) return 0.0f;
    float x = chord / (2.0f * radius);
    if (x > 1.0f / 16.0f) return 2.0f * radius * asinf(fminf(x, 1.0f)) - chord;
    float x2 = x * x;
    return 2.0f * radius * x * x2 * (1.0f / 6.0f + x2 * (3.0f / 40.0f + x2 * (5.0f / 112.0f + x2 * (35.0f / 1152.0f))));
}

__device__ __forceinline__ double arc_excess_d(int state, double chord, double radius) {
    if (state == QM_HOM) return 0.0;
    double x = chord / (2.0 * radius);
    if (x > 1.0 / 16.0) return 2.0 * radius * asin(fmin(x, 1.0)) - chord;
    double x2 = x * x;
    return 2.0 * radius * x * x2 * (1.0 / 6.0 + x2 * (3.0 / 40.0 + x2 * (5.0 / 112.0 + x2 * (35.0 / 1152.0))));
}

// |SO| + |OR| - |SR| without cancellation (rubber_band.rs:352-364).
__device__ __forceinline__ float triangle_excess_f(PlanePoint s, PlanePoint o, PlanePoint r) {
    float ux = o.x - s.x, uz = o.z - s.z, vx = r.x - o.x, vz = r.z - o.z;
    float lu = sqrtf(ux * ux + uz * uz), lv = sqrtf(vx * vx + vz * vz);
    float wx = ux + vx, wz = uz + vz;
    float lw = sqrtf(wx * wx + wz * wz);
    float dot = ux * vx + uz * vz;
    if (dot <= 0.0f) return lu + lv - lw;
    float cross = ux * vz - uz * vx;
    return 2.0f * cross * cross / ((lu * lv + dot) * (lu + lv + lw));
}

struct PointD {
    double x, z;
};

__device__ __forceinline__ double distance_d(PointD a, PointD b) {
    double dx = b.x - a.x, dz = b.z - a.z;
    return sqrt(dx * dx + dz * dz);
}

__device__ __forceinline__ double triangle_excess_d(PointD s, PointD o, PointD r) {
    double ux = o.x - s.x, uz = o.z - s.z, vx = r.x - o.x, vz = r.z - o.z;
    double lu = sqrt(ux * ux + uz * uz), lv = sqrt(vx * vx + vz * vz);
    double wx = ux + vx, wz = uz + vz;
    double lw = sqrt(wx * wx + wz * wz);
    double dot = ux * vx + uz * vz;
    if (dot <= 0.0) return lu + lv - lw;
    double cross = ux * vz - uz * vx;
    return 2.0 * cross * cross / ((lu * lv + dot) * (lu + lv + lw));
}

// StateRay::path_difference (rubber_band.rs:257-301) in FP64: the diffraction path difference
// cancels catastrophically near grazing, so delta alone is taken in double.
__device__ __noinline__ double path_difference_d(int state, double radius, PointD from, const PlanePoint *points, int n,
                                           PointD to) {
    if (n == 0) return 0.0;
    double chords = 0.0, arcs = 0.0;
    PointD start = from;
    for (int i = 0; i < n; ++i) {
        PointD p{points[i].x, points[i].z};
        chords += triangle_excess_d(start, p, to);
        if (state != QM_HOM) arcs += arc_excess_d(state, distance_d(start, p), radius);
        start = p;
    }
    // Homogeneous rays are straight: every arc excess is exactly zero.
    if (state != QM_HOM)
        arcs += arc_excess_d(state, distance_d(start, to), radius) - arc_excess_d(state, distance_d(from, to), radius);
    double excess = chords + arcs;
    if (n > 1) return excess;
    PointD first{points[0].x, points[0].z};
    double chord = from.z + (to.z - from.z) * (first.x - from.x) / (to.x - from.x);
    if (state == QM_HOM) return first.z >= chord ? excess : -excess;
    if (first.z >= chord) return excess;
    PointD on_chord{first.x, chord};
    return 2.0 * triangle_excess_d(from, on_chord, to) - triangle_excess_d(from, first, to) +
           2.0 * arc_excess_d(state, distance_d(from, on_chord), radius) +
           2.0 * arc_excess_d(state, distance_d(on_chord, to), radius) -
           arc_excess_d(state, distance_d(from, first), radius) - arc_excess_d(state, distance_d(first, to), radius) -
           arc_excess_d(state, distance_d(from, to), radius);
}

// The single-point path difference in FP32, used only to choose the unblocked candidate; the
// chosen one's delta is recomputed in FP64.
template <int STATE>
__device__ __forceinline__ float single_path_difference_f(float radius, PlanePoint from, PlanePoint o, PlanePoint to,
                                                          float chord_sr) {
    float dso = sqrtf((o.x - from.x) * (o.x - from.x) + (o.z - from.z) * (o.z - from.z));
    float dor = sqrtf((to.x - o.x) * (to.x - o.x) + (to.z - o.z) * (to.z - o.z));
    float excess = triangle_excess_f(from, o, to);
    if (STATE == QM_FAV)
        excess += arc_excess_f<STATE>(dso, radius) + arc_excess_f<STATE>(dor, radius) -
                  arc_excess_f<STATE>(chord_sr, radius);
    float chord = chord_altitude(from, to, o.x);
    if (STATE == QM_HOM) return o.z >= chord ? excess : -excess;
    if (o.z >= chord) return excess;
    PlanePoint on_chord{o.x, chord};
    float dsa = sqrtf((on_chord.x - from.x) * (on_chord.x - from.x) + (on_chord.z - from.z) * (on_chord.z - from.z));
    float dar = sqrtf((to.x - on_chord.x) * (to.x - on_chord.x) + (to.z - on_chord.z) * (to.z - on_chord.z));
    return 2.0f * triangle_excess_f(from, on_chord, to) - triangle_excess_f(from, o, to) +
           2.0f * arc_excess_f<STATE>(dsa, radius) + 2.0f * arc_excess_f<STATE>(dar, radius) -
           arc_excess_f<STATE>(dso, radius) - arc_excess_f<STATE>(dor, radius) - arc_excess_f<STATE>(chord_sr, radius);
}

// ---------------------------------------------------------------------------------------------
// Diffraction: physics/src/cnossos/diffraction.rs
constexpr float DIFFRACTION_CAP_DB = 25.0f;
constexpr float MULTIPLE_DIFFRACTION_MINIMUM_SPAN = 0.3f;

// diffraction.rs:19-29
// delta arrives as FP32: its cancellation was taken care of in FP64, and 24 bits of relative
// precision leave the level within 1e-6 dB.
__device__ __forceinline__ float diffraction_db(float delta, float c2, int b) {
    float x = 40.0f * c2 * delta * c_band.inv_lambda[b];
    return x >= -2.0f ? 10.0f * log10_fast(3.0f + x) : 0.0f;
}

// diffraction.rs:32-34
__device__ __forceinline__ float ground_split_db(float ground_db, float mirrored_db, float direct_db) {
    return -20.0f * log10_fast(1.0f + (amplitude_of(-ground_db) - 1.0f) * amplitude_of(-(mirrored_db - direct_db)));
}

}  // namespace qm
