// Line pieces: the CNOSSOS-EU point sum of a straight source piece by quadrature in the in-plane
// angle (Directive 2015/996 2.5.3; physics/src/line.rs). For a straight piece and a receiver R,
// dx / r^2 = dphi / d_perp with phi the angle in the plane holding the line and R, so the sum of
// point sources with A_div = 20 lg r + 11 is W' / (10^1.1 d_perp) times the integral of the path's
// transfer over dphi. Five buckets of equal dphi take one node each (one bucket for a piece seen
// under 3 degrees); a bucket spanning more than 3 degrees of azimuth with an obstacle edge in
// front of it replaces its node by nodes placed on the blocked runs and clear gaps of a 128-bin
// mask over its azimuths, each weighted by its own dphi.
//
// Everything here is __host__ __device__ and allocates nothing: the nodes go to a callback one
// at a time and the mask is four 32-bit words, so one device thread can walk a piece's nodes
// while it evaluates their rays. The templates take host-only functors too (the host entry
// points' C callbacks), hence nv_exec_check_disable on each. Positions are metres relative to
// the receiver: x east, y north, z up.
#pragma once

#include <cuda_runtime.h>

#include <math.h>
#include <stdint.h>

namespace qm {
namespace line {

constexpr double PI = 3.14159265358979323846;
constexpr int BUCKETS = 5;                               // line.rs:19
constexpr double ONE_BUCKET_SPAN_RAD = 3.0 * PI / 180.0;  // line.rs:23
constexpr double WIDE_MIN_SPAN_RAD = 3.0 * PI / 180.0;    // line.rs:26
constexpr int MASK_BINS = 128;                           // line.rs:28
constexpr int MASK_WORDS = MASK_BINS / 32;
constexpr double PART_MAX_SPAN_RAD = 0.26;               // line.rs:30
constexpr int MAX_PARTS = 9;                             // line.rs:31
constexpr double PERPENDICULAR_FLOOR_M = 0.5;            // line.rs:34
constexpr double POINT_DIVERGENCE = 12.589254117941673;  // 10^1.1, line.rs:36

// Most nodes one piece can take: per bucket one node per mask run plus the extra parts a run
// wider than PART_MAX_SPAN_RAD takes (a bucket spans under pi of azimuth), five buckets.
constexpr int MAX_NODES = BUCKETS * (MASK_BINS + 13);

// An angle wrapped into (-pi, pi] (line.rs:39-48).
__host__ __device__ inline double wrap_to_pi(double angle) {
    const double tau = 2.0 * PI;
    const double a = fmod(angle, tau);
    if (a > PI) return a - tau;
    if (a <= -PI) return a + tau;
    return a;
}

// A straight piece in the receiver's frame (line.rs:53-62, 86-170): its start, unit direction
// and length, the foot of the perpendicular from the receiver (along the piece, metres), the
// floored perpendicular and the in-plane angles of the two ends.
struct Piece {
    double start[3], unit[3], length, foot, perp, angle0, angle1;

    // False for a piece shorter than a millimetre, which radiates nothing.
    __host__ __device__ bool make(const double s[3], const double e[3]) {
        const double a[3] = {e[0] - s[0], e[1] - s[1], e[2] - s[2]};
        length = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        if (length < 1e-3) return false;
        for (int k = 0; k < 3; ++k) {
            start[k] = s[k];
            unit[k] = a[k] / length;
        }
        foot = -(s[0] * unit[0] + s[1] * unit[1] + s[2] * unit[2]);
        const double f[3] = {s[0] + foot * unit[0], s[1] + foot * unit[1], s[2] + foot * unit[2]};
        perp = fmax(sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]), PERPENDICULAR_FLOOR_M);
        angle0 = atan((0.0 - foot) / perp);
        angle1 = atan((length - foot) / perp);
        return true;
    }
    __host__ __device__ double span() const { return angle1 - angle0; }
    // 1 / (10^1.1 d_perp) times the horizontal share of the piece's direction.
    __host__ __device__ double divergence() const { return hypot(unit[0], unit[1]) / (POINT_DIVERGENCE * perp); }
    __host__ __device__ double angle_at(double along) const { return atan((along - foot) / perp); }
    __host__ __device__ double along_at_angle(double angle) const {
        return fmin(fmax(foot + perp * tan(angle), 0.0), length);
    }
    __host__ __device__ void point(double along, double p[3]) const {
        for (int k = 0; k < 3; ++k) p[k] = start[k] + along * unit[k];
    }
    // Where the horizontal ray at `azimuth` meets the piece's ground track, clamped to the piece;
    // false when the two are parallel.
    __host__ __device__ bool along_at_azimuth(double azimuth, double &along) const {
        const double dx = cos(azimuth), dy = sin(azimuth);
        const double ux = unit[0] * length, uy = unit[1] * length;
        const double den = dx * uy - dy * ux;
        if (fabs(den) < 1e-12) return false;
        const double fraction = (dy * start[0] - dx * start[1]) / den;
        along = fmin(fmax(fraction, 0.0), 1.0) * length;
        return true;
    }
    __host__ __device__ double azimuth_at(double along) const {
        double p[3];
        point(along, p);
        return atan2(p[1], p[0]);
    }
    __host__ __device__ double range_at(double along) const {
        double p[3];
        point(along, p);
        return hypot(p[0], p[1]);
    }
};

__host__ __device__ inline bool mask_bit(const uint32_t mask[MASK_WORDS], int bin) {
    return (mask[bin >> 5] >> (bin & 31)) & 1u;
}

// The bins of the span [lo, hi] (bin width `width`) that one edge's arc blocks: where the edge
// stands at least a metre nearer than the piece seen through the middle of their overlap, the
// arc also tried a turn either way (line.rs:317-355).
__host__ __device__ inline void mark_blocked(const Piece &g, double arc_lo, double arc_hi, double nearest,
                                             double radius, double lo, double hi, double width,
                                             uint32_t mask[MASK_WORDS]) {
    if (nearest > radius) return;
    const double shifts[3] = {0.0, 2.0 * PI, -2.0 * PI};
    for (int s = 0; s < 3; ++s) {
        const double piece_lo = fmax(arc_lo + shifts[s], lo), piece_hi = fmin(arc_hi + shifts[s], hi);
        if (piece_hi <= piece_lo) continue;
        double along;
        if (!g.along_at_azimuth(0.5 * (piece_lo + piece_hi), along)) continue;
        if (g.range_at(along) - nearest <= 1.0) continue;
        // A first bin past the end (an overlap rounded onto the span's far edge) marks nothing.
        const double down = floor((piece_lo - lo) / width);
        const int first = down > 0.0 ? (int)fmin(down, (double)MASK_BINS) : 0;
        const double up = ceil((piece_hi - lo) / width);
        int last = up > 1.0 ? (int)fmin(up - 1.0, (double)MASK_BINS) : 0;
        if (last < first) last = first;
        if (last > MASK_BINS - 1) last = MASK_BINS - 1;
        for (int b = first; b <= last; ++b) mask[b >> 5] |= 1u << (b & 31);
    }
}

// The geometry-placed nodes of one bucket [angle_lo, angle_hi] of in-plane angle, or none when
// the bucket keeps its centre node: narrow in azimuth, or nothing in front of it
// (line.rs:208-315). `skyline(lo, hi, radius, visit)` hands visit(arc_lo, arc_hi, nearest) every
// obstacle edge within `radius` whose arc may meet the wedge [lo, hi]; it is asked only here.
// Returns how many nodes went to emit(along, weight, obstacles_on_ray).
#pragma nv_exec_check_disable
template <class Skyline, class Emit>
__host__ __device__ int wide_bucket_nodes(const Piece &g, double angle_lo, double angle_hi, Skyline &skyline,
                                          Emit &emit) {
    const double along_lo = g.along_at_angle(angle_lo), along_hi = g.along_at_angle(angle_hi);
    const double azimuth_a = g.azimuth_at(along_lo);
    const double turn = wrap_to_pi(g.azimuth_at(along_hi) - azimuth_a);
    const double span = fabs(turn);
    if (span < WIDE_MIN_SPAN_RAD) return 0;
    const double span_lo = turn < 0.0 ? azimuth_a + turn : azimuth_a;
    const double span_hi = turn < 0.0 ? azimuth_a : azimuth_a + turn;
    double a[3], b[3];
    g.point(along_lo, a);
    g.point(along_hi, b);
    const double chord = hypot(a[0] - b[0], a[1] - b[1]);
    const double centre_range = g.range_at(g.along_at_angle(0.5 * (angle_lo + angle_hi)));
    const double radius = fmin(fmin(g.range_at(along_lo), g.range_at(along_hi)), centre_range) + chord;
    const double width = span / MASK_BINS;
    uint32_t mask[MASK_WORDS] = {0u, 0u, 0u, 0u};
    auto visit = [&](double arc_lo, double arc_hi, double nearest) {
        mark_blocked(g, arc_lo, arc_hi, nearest, radius, span_lo, span_hi, width, mask);
    };
    skyline(span_lo, span_hi, radius, visit);
    if ((mask[0] | mask[1] | mask[2] | mask[3]) == 0u) return 0;
    const double lo_a = fmin(along_lo, along_hi), hi_a = fmax(along_lo, along_hi);
    const double angle_at_span_lo = turn < 0.0 ? angle_hi : angle_lo;
    const double angle_at_span_hi = turn < 0.0 ? angle_lo : angle_hi;
    auto angle_at_azimuth = [&](double azimuth, double fallback) {
        double along;
        if (!g.along_at_azimuth(azimuth, along)) return fallback;
        return g.angle_at(fmin(fmax(along, lo_a), hi_a));
    };
    int emitted = 0, bin = 0;
    while (bin < MASK_BINS) {
        const bool blocked = mask_bit(mask, bin);
        int run_end = bin;
        while (run_end < MASK_BINS && mask_bit(mask, run_end) == blocked) ++run_end;
        const double run_lo = span_lo + bin * width;
        const double run_hi = run_end == MASK_BINS ? span_hi : span_lo + run_end * width;
        const int parts = (int)fmin(fmax(ceil((run_hi - run_lo) / PART_MAX_SPAN_RAD), 1.0), (double)MAX_PARTS);
        const double step = (run_hi - run_lo) / parts;
        for (int part = 0; part < parts; ++part) {
            const double part_lo = run_lo + part * step;
            const bool last_part = part + 1 == parts && run_end == MASK_BINS;
            const double part_hi = last_part ? span_hi : part_lo + step;
            const double edge_lo = (bin == 0 && part == 0) ? angle_at_span_lo : angle_at_azimuth(part_lo, angle_at_span_lo);
            const double edge_hi = last_part ? angle_at_span_hi : angle_at_azimuth(part_hi, angle_at_span_hi);
            double along;
            if (!g.along_at_azimuth(0.5 * (part_lo + part_hi), along)) along = g.along_at_angle(0.5 * (edge_lo + edge_hi));
            emit(along, fabs(edge_hi - edge_lo), blocked);
            ++emitted;
        }
        bin = run_end;
    }
    return emitted;
}

// The quadrature nodes of one piece in order (line.rs:178-206): per bucket its geometry-placed
// nodes, else its centre node with the bucket's angle as weight and obstacles on its ray.
// Returns the number of nodes emitted.
#pragma nv_exec_check_disable
template <class Skyline, class Emit>
__host__ __device__ int quadrature_nodes(const Piece &g, Skyline &skyline, Emit &emit) {
    const double span = g.span();
    const int buckets = span < ONE_BUCKET_SPAN_RAD ? 1 : BUCKETS;
    const double bucket_angle = span / buckets;
    int total = 0;
    for (int bucket = 0; bucket < buckets; ++bucket) {
        const double angle_lo = g.angle0 + bucket * bucket_angle, angle_hi = angle_lo + bucket_angle;
        const int placed = wide_bucket_nodes(g, angle_lo, angle_hi, skyline, emit);
        if (placed == 0) {
            emit(g.along_at_angle(angle_lo + 0.5 * bucket_angle), angle_hi - angle_lo, true);
            total += 1;
        } else {
            total += placed;
        }
    }
    return total;
}

}  // namespace line
}  // namespace qm
