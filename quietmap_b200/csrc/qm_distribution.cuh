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

// A single steady intensity as a line's values: one pair (intensity, all the time) and its sums.
struct Steady {
    double pairs[2], sums[4];
    __host__ __device__ explicit Steady(double intensity) {
        pairs[0] = intensity;
        pairs[1] = 1.0;
        sums[0] = sums[1] = 0.0;
        sums[2] = 0.0 + 1.0;
        sums[3] = 0.0 + 1.0 * intensity;
    }
    __host__ __device__ Values view() const { return Values{pairs, sums, 1}; }
};

// out = in with a steady intensity added at every moment (distribution.rs:208-211).
__host__ __device__ inline void over(double bin_db, int n_bins, const double *in_bins, double in_silent,
                                     double intensity, double *out_bins, double *out_silent) {
    const Steady steady(intensity);
    with_line(bin_db, n_bins, in_bins, in_silent, steady.view(), 1.0, out_bins, out_silent);
}

// out = in with an independent distribution `other` added at every moment: its bins' mean
// intensities and its silence as a line's values, ascending, equal ones in bin order with the
// silence first (distribution.rs:198-206). scratch_pairs holds 2 (n_bins + 1) doubles and
// scratch_sums 2 (n_bins + 2).
__host__ __device__ inline void with_distribution(double bin_db, int n_bins, const double *in_bins, double in_silent,
                                                  const double *other_bins, double other_silent,
                                                  double *scratch_pairs, double *scratch_sums, double *out_bins,
                                                  double *out_silent) {
    int n = 0;
    // The silence is 0, under every bin's mean intensity, and comes first in a stable sort.
    if (other_silent > 0.0) {
        scratch_pairs[0] = 0.0;
        scratch_pairs[1] = other_silent;
        n = 1;
    }
    for (int b = 0; b < n_bins; ++b) {
        const double share = other_bins[2 * b];
        if (!(share > 0.0)) continue;
        const double intensity = other_bins[2 * b + 1] / share;
        // Insertion into the ascending run so far (stable: after every equal value); bins' means
        // rise with the bin, so this is mostly an append.
        int at = n;
        while (at > 0 && scratch_pairs[2 * (at - 1)] > intensity) {
            scratch_pairs[2 * at] = scratch_pairs[2 * (at - 1)];
            scratch_pairs[2 * at + 1] = scratch_pairs[2 * (at - 1) + 1];
            --at;
        }
        scratch_pairs[2 * at] = intensity;
        scratch_pairs[2 * at + 1] = share;
        ++n;
    }
    scratch_sums[0] = scratch_sums[1] = 0.0;
    for (int k = 0; k < n; ++k) {
        scratch_sums[2 * (k + 1)] = scratch_sums[2 * k] + scratch_pairs[2 * k + 1];
        scratch_sums[2 * (k + 1) + 1] = scratch_sums[2 * k + 1] + scratch_pairs[2 * k + 1] * scratch_pairs[2 * k];
    }
    with_line(bin_db, n_bins, in_bins, in_silent, Values{scratch_pairs, scratch_sums, n}, 1.0, out_bins, out_silent);
}

// Lines over a period (popup/src/percentiles.rs:172-282, percentiles/lines.rs:172-195), every
// line at its period's mean flow.
constexpr int WEATHER_STATES = 10;                                 // percentiles/weather.rs:131
constexpr double HOLDS_MEAN_LAMBDA = 10.0;                         // lines.rs:240
constexpr double PASSES_HOLD_MEAN = 2.0 * 3.14159265358979323846 * HOLDS_MEAN_LAMBDA;  // lines.rs:243
constexpr double HELD_EXCEEDED = 1e-3;                             // lines.rs:247
constexpr double HELD_SHARE = 1e-2;                                // lines.rs:248

// How a line sounds in a period: holding its mean, silent (an event off then), moving the level
// (an event while it sounds, a stream of passes), or a sparse line that moves the level unless
// its intensity exceeded a thousandth of the time stays under a hundredth of the steady energy.
enum ShapeKind : int { SHAPE_HOLDS = 0, SHAPE_SILENT = 1, SHAPE_MOVES = 2, SHAPE_SPARSE = 3 };

struct PeriodLine {
    double energy;         // the period's mean energy: a line at or under 0 is silent
    const double *means;   // [WEATHER_STATES]
    double factor;         // its flow in the hours against the period's mean (1 without a profile)
    int kind;              // ShapeKind
    Values values;         // SHAPE_MOVES, SHAPE_SPARSE: intensities relative to the mean
    double exceeded;       // SHAPE_SPARSE: the relative intensity exceeded a thousandth of the time
};

// The moment of a layer's lines in a weather state (percentiles.rs:236-282): the steady energy
// with the lines that hold their mean, and the steady energy the sparse lines are held against.
__host__ __device__ inline double moment_floor(const PeriodLine *lines, int n, int state, double steady,
                                               double &steady_energy) {
    double floor = steady, held = 0.0;
    for (int k = 0; k < n; ++k) {
        const double mean = lines[k].means[state] * lines[k].factor;
        if (lines[k].energy <= 0.0 || mean <= 0.0) continue;
        if (lines[k].kind == SHAPE_HOLDS) floor += mean;
        if (lines[k].kind == SHAPE_SPARSE) held += mean;
    }
    steady_energy = floor + held;
    for (int k = 0; k < n; ++k) {
        const double mean = lines[k].means[state] * lines[k].factor;
        if (lines[k].energy <= 0.0 || mean <= 0.0 || lines[k].kind != SHAPE_SPARSE) continue;
        if (mean * lines[k].exceeded < HELD_SHARE * steady_energy) floor += mean;
    }
    return floor;
}

// The lines that move the level in that moment, in the reference's order: the events and
// streams, then the sparse lines not held; visit(k, mean).
#pragma nv_exec_check_disable
template <class Visit>
__host__ __device__ void moving_lines(const PeriodLine *lines, int n, int state, double steady_energy, Visit &visit) {
    for (int pass = 0; pass < 2; ++pass)
        for (int k = 0; k < n; ++k) {
            const double mean = lines[k].means[state] * lines[k].factor;
            if (lines[k].energy <= 0.0 || mean <= 0.0) continue;
            if (pass == 0 && lines[k].kind == SHAPE_MOVES) visit(k, mean);
            if (pass == 1 && lines[k].kind == SHAPE_SPARSE && !(mean * lines[k].exceeded < HELD_SHARE * steady_energy))
                visit(k, mean);
        }
}

// A layer's distribution in one weather state (percentiles.rs:172-211): its floor, then each
// moving line added. Returns true where no line moves (the layer holds its floor, written to
// *floor). a and b are [n_bins][2] work buffers; the result is in *out (a or b).
__host__ __device__ inline bool layer_state(double bin_db, int n_bins, const PeriodLine *lines, int n, int state,
                                            double steady, double *a, double *b, double **out, double *out_silent,
                                            double *floor) {
    double steady_energy;
    *floor = moment_floor(lines, n, state, steady, steady_energy);
    for (int k = 0; k < 2 * n_bins; ++k) a[k] = 0.0;
    double silent;
    over(bin_db, n_bins, a, 1.0, *floor, b, &silent);
    double *current = b, *spare = a;
    bool moved = false;
    auto add = [&](int k, double mean) {
        double next_silent;
        with_line(bin_db, n_bins, current, silent, lines[k].values, mean, spare, &next_silent);
        double *t = current;
        current = spare;
        spare = t;
        silent = next_silent;
        moved = true;
    };
    moving_lines(lines, n, state, steady_energy, add);
    *out = current;
    *out_silent = silent;
    return !moved;
}

// The weather states merged where their difference cannot show (popup/src/percentiles/
// weather.rs:132-176) for one period's lines, means[n][WEATHER_STATES] in place: each run of
// consecutive states in which every line's mean is finite and within `spread` (largest over
// smallest) gives each line its mean over the run in all of the run's states.
__host__ __device__ inline void merge_close_states(double *means, int n, double spread) {
    auto within = [&](int start, int end) {  // states start..=end, every line
        for (int k = 0; k < n; ++k) {
            double low = INFINITY, high = 0.0;
            for (int st = start; st <= end; ++st) {
                const double mean = means[k * WEATHER_STATES + st];
                if (!isfinite(mean)) return false;
                low = fmin(low, mean);
                high = fmax(high, mean);
            }
            if (!(high <= spread * low)) return false;
        }
        return true;
    };
    int start = 0;
    while (start < WEATHER_STATES) {
        int end = start + 1;
        while (end < WEATHER_STATES && within(start, end)) ++end;
        if (end - start > 1) {
            for (int k = 0; k < n; ++k) {
                double *run = means + k * WEATHER_STATES + start;
                bool differ = false;
                for (int st = 0; st < end - start; ++st) differ = differ || run[st] != run[0];
                if (!differ) continue;
                double total = 0.0;
                for (int st = 0; st < end - start; ++st) total += run[st];
                const double mean = total / (double)(end - start);
                for (int st = 0; st < end - start; ++st) run[st] = mean;
            }
        }
        start = end;
    }
}

// Loudness from the distributions (popup/src/loudness.rs:68-130, 236-269): a period's curve is
// Zwicker's loudness of its received spectrum set to each whole A-weighted decibel from -30 to
// 160 (191 values), linear between; its mean loudness the levels' shares times the curve there.
constexpr double CURVE_LOW_DB = -30.0, CURVE_HIGH_DB = 160.0;  // loudness.rs:68-69
constexpr int CURVE_STEPS = 190;
constexpr double PERIOD_HOURS[3] = {12.0, 4.0, 8.0};            // physics/src/bands.rs:16
constexpr double PERIOD_PENALTY_DB[3] = {0.0, 5.0, 10.0};       // physics/src/bands.rs:18

__host__ __device__ inline double curve_at(const double *table, double level_db) {
    const double position = fmin(fmax(level_db - CURVE_LOW_DB, 0.0), (double)CURVE_STEPS);
    const double down = floor(position);
    const int below = down < (double)(CURVE_STEPS - 1) ? (int)down : CURVE_STEPS - 1;
    const double low = table[below], high = table[below + 1];
    return low + (high - low) * (position - (double)below);
}

// The mean loudness over a distribution with `penalty_db` added to its levels (silence is 0).
__host__ __device__ inline double mean_loudness(const double *bins, int n_bins, const double *table,
                                                double penalty_db) {
    double total = 0.0;
    for (int b = 0; b < n_bins; ++b) {
        const double share = bins[2 * b];
        if (!(share > 0.0)) continue;
        total += share * curve_at(table, 10.0 * log10(bins[2 * b + 1] / share) + penalty_db);
    }
    return total;
}

// A line's means in the weather states from its pieces' energies in the two meteorological
// states (popup/src/percentiles/weather.rs:1-127). Pieces are binned by their favourable share,
// pieces louder in calm air in bins of their own; each bin's calm energy counts in every state,
// its excess downwind in the states wholly under its share and in part in the state its share
// falls in.
constexpr int SHARE_BINS = 10;                           // weather.rs:6
constexpr double F64_EPSILON = 2.220446049250313e-16;

__host__ __device__ inline double favourable_share(double mean, double homogeneous, double favourable) {
    if (fabs(favourable - homogeneous) <= F64_EPSILON * fabs(favourable)) return 0.0;
    return fmin(fmax((mean - homogeneous) / (favourable - homogeneous), 0.0), 1.0);
}

// A whole non-negative position's integer part, NaN as 0, held to `most`.
__host__ __device__ inline int truncated(double position, int most) {
    if (!(position > 0.0)) return 0;
    return position >= (double)most ? most : (int)position;
}

struct WeatherBins {
    double bins[2 * SHARE_BINS][3][3];  // [bin][homogeneous, favourable, mixed][period]
    uint32_t active;

    __host__ __device__ void clear() {
        for (int b = 0; b < 2 * SHARE_BINS; ++b)
            for (int st = 0; st < 3; ++st)
                for (int p = 0; p < 3; ++p) bins[b][st][p] = 0.0;
        active = 0;
    }
    // A piece of `energy` in one period, the mix of its homogeneous and favourable energies (a
    // piece without states holds its mean in either).
    __host__ __device__ void add(int period, double energy, double homogeneous, double favourable) {
        if (!(homogeneous > 0.0 || favourable > 0.0)) homogeneous = favourable = energy;
        const double share = favourable_share(energy, homogeneous, favourable);
        const int bin = (favourable < homogeneous ? SHARE_BINS : 0) + truncated(share * SHARE_BINS, SHARE_BINS - 1);
        active |= 1u << bin;
        bins[bin][0][period] += homogeneous;
        bins[bin][1][period] += favourable;
        bins[bin][2][period] += energy;
    }
    // The period's mean of `energy` in each weather state.
    __host__ __device__ void means(int period, double energy, double out[WEATHER_STATES]) const {
        if (active == 0) {
            for (int st = 0; st < WEATHER_STATES; ++st) out[st] = energy;
            return;
        }
        double whole[WEATHER_STATES + 1], part[WEATHER_STATES + 1];
        for (int st = 0; st <= WEATHER_STATES; ++st) whole[st] = part[st] = 0.0;
        double calm = 0.0;
        bool silent = true;
        for (int b = 0; b < 2 * SHARE_BINS; ++b) {
            if (!((active >> b) & 1u)) continue;
            const double homogeneous = bins[b][0][period], favourable = bins[b][1][period];
            silent = silent && homogeneous + favourable <= 0.0;
            const double share = favourable_share(bins[b][2][period], homogeneous, favourable);
            const double position = share * WEATHER_STATES;
            const int state = truncated(position, WEATHER_STATES);
            whole[state] += favourable - homogeneous;
            part[state] += (position - (double)state) * (favourable - homogeneous);
            calm += homogeneous;
        }
        if (silent) {
            for (int st = 0; st < WEATHER_STATES; ++st) out[st] = energy;
            return;
        }
        double above = 0.0;
        for (int st = WEATHER_STATES - 1; st >= 0; --st) {
            above += whole[st + 1];
            out[st] = calm + above + part[st];
        }
    }
};

}  // namespace dist
}  // namespace qm
