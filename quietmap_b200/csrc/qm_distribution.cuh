// How levels add over time (popup/src/distribution.rs:44-298): a distribution of the summed level
// over a period on a grid of bin_db decibels from -30 dB over 180 dB, per bin its share of the
// time and that share times its moments' mean intensity (so adding an independent sound loses no
// energy to the grid), and the share in silence. A line's values are intensities with their
// shares of the time, ascending, with running sums of the shares and of the shares times the
// intensities; adding a line to a distribution visits, per moment of the distribution, the runs
// of values whose sums share a bin, found by a logarithm for the first and a short search each
// after it.
//
// __host__ __device__ over caller-provided arrays, allocating nothing: a device thread or warp
// keeps a distribution in shared memory (360 bins of 16 bytes at 0.5 dB, 90 at 2 dB), the host
// entry points run the same source.
#pragma once

#include <cuda_runtime.h>

#include <math.h>
#include <stdint.h>

namespace qm {
namespace dist {

constexpr double LEVEL_MIN_DB = -30.0;  // distribution.rs:11
constexpr double SPAN_DB = 180.0;       // distribution.rs:12
constexpr double LN_10 = 2.302585092994046;

// A level's intensity (physics/src/bands.rs:34-36).
__host__ __device__ inline double energy(double level_db) { return exp(level_db * (LN_10 / 10.0)); }

// The grid's bins at bin_db: the span over the step, rounded half away from zero.
__host__ __device__ inline int bin_count(double bin_db) { return (int)round(SPAN_DB / bin_db); }

// The bin of a level; a level under the grid (or NaN) is held in the lowest bin, one over it in
// the highest (distribution.rs:69-73).
__host__ __device__ inline int bin_of(double level_db, double bin_db, int n_bins) {
    const double at = round((level_db - LEVEL_MIN_DB) / bin_db);
    if (!(at > 0.0)) return 0;
    return at >= (double)(n_bins - 1) ? n_bins - 1 : (int)at;
}

// A line's values: pairs[k] = (intensity, share) ascending by intensity, sums[k] = (shares,
// shares times intensities) of the first k pairs, k = 0 .. n.
struct Values {
    const double *pairs;  // [n][2]
    const double *sums;   // [n + 1][2]
    int n;
};

// The first pair from `from` whose intensity reaches `limit` (n if none): probing one, two,
// four... ahead, then halving, as a run is mostly a few values (distribution.rs:223-233).
__host__ __device__ inline int first_at_or_above(const Values &v, int from, double limit) {
    int low = from, step = 1;
    while (low + step - 1 < v.n && v.pairs[2 * (low + step - 1)] < limit) {
        low += step;
        step *= 2;
    }
    int high = low + step - 1 < v.n ? low + step - 1 : v.n;
    while (low < high) {
        const int mid = low + (high - low) / 2;
        if (v.pairs[2 * mid] < limit)
            low = mid + 1;
        else
            high = mid;
    }
    return low;
}

// The bins a moment at `intensity` (0: silent) moves to with each of the line's values times
// `scale` (above 0) added, each visited once in increasing order as visit(bin, shares, weighted)
// with the shares of the values that take it there and their shares times their scaled
// intensities; bin -1 is silence (distribution.rs:86-145).
#pragma nv_exec_check_disable
template <class Visit>
__host__ __device__ void runs(double bin_db, int n_bins, double intensity, const Values &line, double scale,
                              Visit &visit) {
    auto run = [&](int a, int b, double &shares, double &weighted) {
        shares = line.sums[2 * b] - line.sums[2 * a];
        weighted = scale * (line.sums[2 * b + 1] - line.sums[2 * a + 1]);
    };
    int from = 0;
    double shares, weighted;
    if (intensity <= 0.0) {
        // The values at or under zero (ascending, so a prefix) keep the moment silent.
        int lo = 0, hi = line.n;
        while (lo < hi) {
            const int mid = lo + (hi - lo) / 2;
            if (line.pairs[2 * mid] <= 0.0)
                lo = mid + 1;
            else
                hi = mid;
        }
        from = lo;
        if (from > 0) {
            run(0, from, shares, weighted);
            visit(-1, shares, weighted);
        }
    }
    if (from == line.n) return;
    const int last = n_bins - 1;
    const double step = energy(bin_db);
    int bin = bin_of(10.0 * log10(intensity + scale * line.pairs[2 * from]), bin_db, n_bins);
    double ceiling = energy(LEVEL_MIN_DB + ((double)bin + 0.5) * bin_db);
    for (;;) {
        const int to = bin == last ? line.n : first_at_or_above(line, from + 1, (ceiling - intensity) / scale);
        run(from, to, shares, weighted);
        visit(bin, shares, weighted);
        from = to;
        if (from >= line.n) break;
        const double value = line.pairs[2 * from];
        for (;;) {
            bin += 1;
            ceiling *= step;
            if (bin == last || intensity + scale * value < ceiling) break;
        }
    }
}

// out = in with the line (values times `scale`) added at every moment: each sum in the bin of its
// level, its intensity kept exact (distribution.rs:176-196). bins are [n_bins][2] (share,
// share x mean intensity); out is overwritten and must not alias in.
__host__ __device__ inline void with_line(double bin_db, int n_bins, const double *in_bins, double in_silent,
                                          const Values &line, double scale, double *out_bins, double *out_silent) {
    for (int b = 0; b < 2 * n_bins; ++b) out_bins[b] = 0.0;
    double silent = 0.0;
    auto add = [&](double intensity, double share) {
        auto visit = [&](int bin, double shares, double weighted) {
            if (bin < 0) {
                silent += share * shares;
            } else {
                out_bins[2 * bin] += share * shares;
                out_bins[2 * bin + 1] += share * (intensity * shares + weighted);
            }
        };
        runs(bin_db, n_bins, intensity, line, scale, visit);
    };
    if (in_silent > 0.0) add(0.0, in_silent);
    for (int b = 0; b < n_bins; ++b) {
        const double share = in_bins[2 * b];
        if (share > 0.0) add(in_bins[2 * b + 1] / share, share);
    }
    *out_silent = silent;
}

// The level exceeded `exceeded` of the time, -inf where silence is (distribution.rs:152-162).
__host__ __device__ inline double exceeded_db(const double *bins, int n_bins, double exceeded) {
    double above = 0.0;
    for (int b = n_bins - 1; b >= 0; --b) {
        const double share = bins[2 * b];
        above += share;
        if (share > 0.0 && above > exceeded * (1.0 - 1e-12)) return 10.0 * log10(bins[2 * b + 1] / share);
    }
    return -INFINITY;
}

// into += from x weight, silence included (distribution.rs:213-220).
__host__ __device__ inline void add_scaled(double *into_bins, double *into_silent, const double *from_bins,
                                           double from_silent, int n_bins, double weight) {
    *into_silent += from_silent * weight;
    for (int b = 0; b < 2 * n_bins; ++b) into_bins[b] += from_bins[b] * weight;
}

// The node probabilities of a line's values (distribution.rs:17-32): every percent to 0.99, then
// evenly in log(1 - p) to 1 - 1e-8, each with the share of the time it stands for.
constexpr int NODES = 99 + 24 + 1;
__host__ __device__ inline void node(int k, double &p, double &share) {
    if (k < 99) {
        p = ((double)k + 0.5) / 100.0;
        share = 0.01;
    } else if (k < 99 + 24) {
        const double a = 2.0 + (double)(k - 99) * 0.25, b = 2.25 + (double)(k - 99) * 0.25;
        p = 1.0 - pow(10.0, -((a + b) / 2.0));
        share = (1.0 - pow(10.0, -b)) - (1.0 - pow(10.0, -a));
    } else {
        p = 1.0 - 0.5e-8;
        share = 1e-8;
    }
}

}  // namespace dist
}  // namespace qm
