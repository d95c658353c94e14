// Distributions of the summed level over time on the host side of the library: the C entry
// points that run the shared __host__ __device__ arithmetic (qm_distribution.cuh) on the calling
// thread, and the values of the lines added to them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <utility>
#include <vector>

#include "../../include/qm_distribution.h"
#include "qm_distribution.cuh"
#include "qm_host.h"
#include "qm_percentile.cuh"

static_assert(QM_DISTRIBUTION_LINE_NODES == qm::dist::NODES, "the header's node count is the grid's");
static_assert(QM_WEATHER_STATES == qm::dist::WEATHER_STATES, "the header's weather states are the mixture's");
static_assert(QM_LOUDNESS_CURVE_POINTS == qm::dist::CURVE_STEPS + 1, "the header's curve is the table's");

namespace {

qm_status grid(const char *who, double bin_db, int &n_bins) {
    if (!(bin_db > 0.0) || !std::isfinite(bin_db))
        return qm::set_error(QM_ERR_ARGUMENT, std::string(who) + ": bin_db must be positive and finite");
    const double count = std::round(qm::dist::SPAN_DB / bin_db);
    if (!(count >= 1.0) || count > QM_DISTRIBUTION_MAX_BINS)
        return qm::set_error(QM_ERR_ARGUMENT, std::string(who) + ": bin_db gives " + std::to_string(count) +
                                                  " bins, at most " + std::to_string(QM_DISTRIBUTION_MAX_BINS));
    n_bins = (int)count;
    return QM_OK;
}

// Values in increasing order of intensity, equal ones in their given order, with their running
// sums (distribution.rs:243-256).
struct OwnedValues {
    std::vector<double> pairs, sums;
    qm::dist::Values view() const { return qm::dist::Values{pairs.data(), sums.data(), (int)(pairs.size() / 2)}; }
};

OwnedValues sorted_values(const double *values, size_t n) {
    std::vector<std::pair<double, double>> list(n);
    // An intensity of -0 is one of 0: the sort sees them as equal.
    for (size_t k = 0; k < n; ++k) list[k] = {values[2 * k] + 0.0, values[2 * k + 1]};
    std::stable_sort(list.begin(), list.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
    OwnedValues out;
    out.pairs.resize(2 * n);
    out.sums.resize(2 * (n + 1));
    out.sums[0] = out.sums[1] = 0.0;
    for (size_t k = 0; k < n; ++k) {
        out.pairs[2 * k] = list[k].first;
        out.pairs[2 * k + 1] = list[k].second;
        out.sums[2 * (k + 1)] = out.sums[2 * k] + list[k].second;
        out.sums[2 * (k + 1) + 1] = out.sums[2 * k + 1] + list[k].second * list[k].first;
    }
    return out;
}

// pass_values (distribution.rs:283-298) for a mean in (0, 700], in the order they arise.
std::vector<double> pass_pairs(double mean) {
    std::vector<double> out;
    double share = std::exp(-mean);
    out.insert(out.end(), {0.0, share});
    double time_left = -std::expm1(-mean), mean_left = 1.0, count = 0.0;
    for (;;) {
        count += 1.0;
        share *= mean / count;
        if (time_left - share <= 1e-12) {
            out.insert(out.end(), {mean_left / time_left, time_left});
            return out;
        }
        time_left -= share;
        mean_left -= share * count / mean;
        out.insert(out.end(), {count / mean, share});
    }
}

// Kurze's values at lambda at the node probabilities, by the library's sampler.
std::vector<double> kurze_pairs(double lambda) {
    const float *table = qm::line_level_table_shared().data();
    std::vector<double> out(2 * qm::dist::NODES);
    for (int k = 0; k < qm::dist::NODES; ++k) {
        double p, share;
        qm::dist::node(k, p, share);
        out[2 * k] = qm::line_relative_intensity(table, lambda, p);
        out[2 * k + 1] = share;
    }
    return out;
}

}  // namespace

extern "C" {

qm_status qm_distribution_bins(double bin_db, size_t *n_bins) {
    if (n_bins == nullptr) return qm::set_error(QM_ERR_ARGUMENT, "qm_distribution_bins: null n_bins");
    int n = 0;
    const qm_status status = grid("qm_distribution_bins", bin_db, n);
    if (status != QM_OK) return status;
    *n_bins = (size_t)n;
    return QM_OK;
}

qm_status qm_distribution_with_line(double bin_db, const double *bins, double silent, const double *values,
                                    size_t n_values, double scale, double *out_bins, double *out_silent) {
    int n_bins = 0;
    const qm_status status = grid("qm_distribution_with_line", bin_db, n_bins);
    if (status != QM_OK) return status;
    if (bins == nullptr || out_bins == nullptr || out_silent == nullptr || (n_values > 0 && values == nullptr))
        return qm::set_error(QM_ERR_ARGUMENT, "qm_distribution_with_line: null bins, values or output");
    if (bins == out_bins) return qm::set_error(QM_ERR_ARGUMENT, "qm_distribution_with_line: out_bins aliases bins");
    if (!(scale > 0.0) || !std::isfinite(scale))
        return qm::set_error(QM_ERR_ARGUMENT, "qm_distribution_with_line: scale must be above 0 and finite");
    if (n_values > (size_t)INT32_MAX / 2)
        return qm::set_error(QM_ERR_ARGUMENT, "qm_distribution_with_line: too many values");
    for (size_t k = 0; k < n_values; ++k)
        if (!(values[2 * k] >= 0.0) || !(values[2 * k + 1] >= 0.0))
            return qm::set_error(QM_ERR_ARGUMENT, "qm_distribution_with_line: value " + std::to_string(k) +
                                                      " has a negative or NaN intensity or share");
    const OwnedValues line = sorted_values(values, n_values);
    qm::dist::with_line(bin_db, n_bins, bins, silent, line.view(), scale, out_bins, out_silent);
    return QM_OK;
}

qm_status qm_distribution_exceeded_db(double bin_db, const double *bins, double exceeded, double *level_db) {
    int n_bins = 0;
    const qm_status status = grid("qm_distribution_exceeded_db", bin_db, n_bins);
    if (status != QM_OK) return status;
    if (bins == nullptr || level_db == nullptr)
        return qm::set_error(QM_ERR_ARGUMENT, "qm_distribution_exceeded_db: null bins or level_db");
    *level_db = qm::dist::exceeded_db(bins, n_bins, exceeded);
    return QM_OK;
}

qm_status qm_distribution_line_values(double lambda, double duty, double *values, size_t cap, size_t *n_values) {
    if (n_values == nullptr || (cap > 0 && values == nullptr))
        return qm::set_error(QM_ERR_ARGUMENT, "qm_distribution_line_values: null values or n_values");
    if (!std::isnan(duty)) {
        if (!(duty > 0.0 && duty <= 1.0))
            return qm::set_error(QM_ERR_ARGUMENT, "qm_distribution_line_values: duty must lie in (0, 1]");
        *n_values = 2;
        if (cap < 2)
            return qm::set_error(QM_ERR_CAPACITY, "qm_distribution_line_values: 2 values, room for " + std::to_string(cap));
        values[0] = 0.0;
        values[1] = 1.0 - duty;
        values[2] = 1.0 / duty;
        values[3] = duty;
        return QM_OK;
    }
    if (std::isnan(lambda)) return qm::set_error(QM_ERR_ARGUMENT, "qm_distribution_line_values: lambda is NaN");
    *n_values = qm::dist::NODES;
    if (cap < (size_t)qm::dist::NODES)
        return qm::set_error(QM_ERR_CAPACITY, "qm_distribution_line_values: " + std::to_string(qm::dist::NODES) +
                                                  " values, room for " + std::to_string(cap));
    const float *table = qm::line_level_table_shared().data();
    for (int k = 0; k < qm::dist::NODES; ++k) {
        double p, share;
        qm::dist::node(k, p, share);
        values[2 * k] = qm::line_relative_intensity(table, lambda, p);
        values[2 * k + 1] = share;
    }
    return QM_OK;
}

qm_status qm_distribution_layers_grouped(double bin_db, const qm_period_line *lines, size_t n_lines,
                                         const double *steady, size_t n_layers, uint32_t hours,
                                         const uint32_t *group_hours, size_t n_groups, const double *factors,
                                         const uint8_t *profiled, double *layer_bins, double *layer_silent,
                                         double *place_bins, double *place_silent) {
    const char *who = "qm_distribution_layers";
    int n_bins = 0;
    const qm_status status = grid(who, bin_db, n_bins);
    if (status != QM_OK) return status;
    if ((n_lines > 0 && lines == nullptr) || (n_layers > 0 && (steady == nullptr || layer_bins == nullptr ||
                                                               layer_silent == nullptr)) ||
        place_bins == nullptr || place_silent == nullptr)
        return qm::set_error(QM_ERR_ARGUMENT, std::string(who) + ": null lines, steady or output");
    if (n_lines > (size_t)INT32_MAX) return qm::set_error(QM_ERR_ARGUMENT, std::string(who) + ": too many lines");
    if (n_groups == 0 || group_hours == nullptr || (n_lines > 0 && (factors == nullptr || profiled == nullptr)))
        return qm::set_error(QM_ERR_ARGUMENT, std::string(who) + ": no groups of hours, or null factors");
    uint64_t grouped = 0;
    for (size_t g = 0; g < n_groups; ++g) grouped += group_hours[g];
    if (hours == 0 || grouped != hours)
        return qm::set_error(QM_ERR_ARGUMENT, std::string(who) + ": the groups hold " + std::to_string(grouped) +
                                                  " hours of a period of " + std::to_string(hours));
    for (size_t l = 0; l < n_layers; ++l)
        if (!(steady[l] >= 0.0) || !std::isfinite(steady[l]))
            return qm::set_error(QM_ERR_ARGUMENT, std::string(who) + ": steady energy of layer " + std::to_string(l) +
                                                      " is negative or not finite");
    std::vector<char> alike(n_layers, 1);
    for (size_t k = 0; k < n_lines; ++k) {
        const qm_period_line &line = lines[k];
        const std::string which = std::string(who) + ": line " + std::to_string(k);
        if (line.layer >= n_layers) return qm::set_error(QM_ERR_ARGUMENT, which + " names layer " + std::to_string(line.layer));
        if (std::isnan(line.energy) || std::isnan(line.lambda))
            return qm::set_error(QM_ERR_ARGUMENT, which + " has a NaN energy or lambda");
        if (!std::isnan(line.duty) && line.duty > 1.0)
            return qm::set_error(QM_ERR_ARGUMENT, which + " has a duty above 1");
        for (int st = 0; st < QM_WEATHER_STATES; ++st)
            if (!(line.means[st] >= 0.0) || !std::isfinite(line.means[st]))
                return qm::set_error(QM_ERR_ARGUMENT, which + " has a negative or non-finite mean");
        for (size_t g = 0; g < n_groups; ++g)
            if (profiled[k] && (!(factors[g * n_lines + k] >= 0.0) || !std::isfinite(factors[g * n_lines + k])))
                return qm::set_error(QM_ERR_ARGUMENT, which + " has a negative or non-finite flow factor");
        if (profiled[k]) alike[line.layer] = 0;
    }
    const double min_positive = 2.2250738585072014e-308;
    const float *table = qm::line_level_table_shared().data();
    // A layer's lines with their shapes at the flow factors of group g (lines.rs:172-195); g < 0:
    // every line at its period's mean flow. `owned` keeps the values the entries point at.
    auto shape_layer = [&](size_t layer, long g, std::vector<OwnedValues> &owned, std::vector<qm::dist::PeriodLine> &out) {
        out.clear();
        owned.clear();
        owned.reserve(n_lines);
        for (size_t k = 0; k < n_lines; ++k) {
            const qm_period_line &line = lines[k];
            if (line.layer != layer) continue;
            const double factor = (g >= 0 && profiled[k]) ? factors[(size_t)g * n_lines + k] : 1.0;
            qm::dist::PeriodLine entry{line.energy, line.means, factor, qm::dist::SHAPE_HOLDS,
                                       qm::dist::Values{nullptr, nullptr, 0}, 0.0};
            std::vector<double> pairs;
            const double lambda = line.lambda * factor;
            if (!std::isnan(line.passing)) {
                if (line.passing >= min_positive && line.passing < qm::dist::PASSES_HOLD_MEAN) {
                    entry.kind = qm::dist::SHAPE_MOVES;
                    pairs = pass_pairs(line.passing);
                }
            } else if (!std::isnan(line.duty)) {
                if (line.duty > 0.0) {
                    entry.kind = qm::dist::SHAPE_MOVES;
                    pairs = {0.0, 1.0 - line.duty, 1.0 / line.duty, line.duty};
                } else {
                    entry.kind = qm::dist::SHAPE_SILENT;
                }
            } else if (!(lambda >= qm::dist::HOLDS_MEAN_LAMBDA)) {
                entry.kind = qm::dist::SHAPE_SPARSE;
                pairs = kurze_pairs(lambda);
                entry.exceeded = qm::line_relative_intensity(table, lambda, 1.0 - qm::dist::HELD_EXCEEDED);
            }
            if (!pairs.empty()) {
                owned.push_back(sorted_values(pairs.data(), pairs.size() / 2));
                entry.values = owned.back().view();
            }
            out.push_back(entry);
        }
    };
    const size_t bins2 = 2 * (size_t)n_bins;
    const int S = qm::dist::WEATHER_STATES;
    // Per layer and state: its distribution, silence, floor and whether it holds.
    std::vector<double> state_bins(n_layers * S * bins2), state_silent(n_layers * S), floors(n_layers * S);
    std::vector<char> holds(n_layers * S);
    std::vector<double> a(bins2), b(bins2), c(bins2), d(bins2), pairs(2 * ((size_t)n_bins + 1)),
        sums(2 * ((size_t)n_bins + 2));
    std::vector<OwnedValues> owned;
    std::vector<qm::dist::PeriodLine> entries;
    auto layer_states = [&](size_t l, long g) {
        shape_layer(l, g, owned, entries);
        for (int state = 0; state < S; ++state) {
            double *out = nullptr, silent = 0.0;
            const size_t at = l * S + state;
            holds[at] = qm::dist::layer_state(bin_db, n_bins, entries.data(), (int)entries.size(), state, steady[l],
                                              a.data(), b.data(), &out, &silent, &floors[at]);
            std::copy(out, out + bins2, state_bins.begin() + at * bins2);
            state_silent[at] = silent;
        }
    };
    for (size_t b2 = 0; b2 < n_layers * bins2; ++b2) layer_bins[b2] = 0.0;
    for (size_t l = 0; l < n_layers; ++l) layer_silent[l] = 0.0;
    for (size_t b2 = 0; b2 < bins2; ++b2) place_bins[b2] = 0.0;
    *place_silent = 0.0;
    // The layers no profiled line moves, once at their mean flow, a tenth of the time a state.
    for (size_t l = 0; l < n_layers; ++l) {
        if (!alike[l]) continue;
        layer_states(l, -1);
        for (int state = 0; state < S; ++state)
            qm::dist::add_scaled(layer_bins + l * bins2, layer_silent + l, state_bins.data() + (l * S + state) * bins2,
                                 state_silent[l * S + state], n_bins, 1.0 / (double)S);
    }
    for (size_t g = 0; g < n_groups; ++g) {
        const double weight = (double)group_hours[g] / (double)((uint64_t)hours * S);
        for (size_t l = 0; l < n_layers; ++l) {
            if (alike[l]) continue;
            layer_states(l, (long)g);
            for (int state = 0; state < S; ++state)
                qm::dist::add_scaled(layer_bins + l * bins2, layer_silent + l,
                                     state_bins.data() + (l * S + state) * bins2, state_silent[l * S + state], n_bins,
                                     weight);
        }
        // The place in each state: the floors of the layers that hold, then each moving layer.
        for (int state = 0; state < S; ++state) {
            double floor = 0.0;
            for (size_t l = 0; l < n_layers; ++l)
                if (holds[l * S + state]) floor += floors[l * S + state];
            std::fill(c.begin(), c.end(), 0.0);
            double silent;
            qm::dist::over(bin_db, n_bins, c.data(), 1.0, floor, d.data(), &silent);
            double *current = d.data(), *spare = c.data();
            for (size_t l = 0; l < n_layers; ++l) {
                if (holds[l * S + state]) continue;
                double next_silent;
                qm::dist::with_distribution(bin_db, n_bins, current, silent, state_bins.data() + (l * S + state) * bins2,
                                            state_silent[l * S + state], pairs.data(), sums.data(), spare, &next_silent);
                std::swap(current, spare);
                silent = next_silent;
            }
            qm::dist::add_scaled(place_bins, place_silent, current, silent, n_bins, weight);
        }
    }
    return QM_OK;
}

qm_status qm_distribution_layers(double bin_db, const qm_period_line *lines, size_t n_lines, const double *steady,
                                 size_t n_layers, double *layer_bins, double *layer_silent, double *place_bins,
                                 double *place_silent) {
    const uint32_t one = 1;
    const std::vector<uint8_t> unprofiled(n_lines, 0);
    const std::vector<double> unit(n_lines, 1.0);
    return qm_distribution_layers_grouped(bin_db, lines, n_lines, steady, n_layers, 1, &one, 1, unit.data(),
                                          unprofiled.data(), layer_bins, layer_silent, place_bins, place_silent);
}

qm_status qm_distribution_merge_states(qm_period_line *lines, size_t n_lines, double spread) {
    if (n_lines > 0 && lines == nullptr) return qm::set_error(QM_ERR_ARGUMENT, "qm_distribution_merge_states: null lines");
    if (std::isnan(spread)) return qm::set_error(QM_ERR_ARGUMENT, "qm_distribution_merge_states: spread is NaN");
    if (n_lines > (size_t)INT32_MAX) return qm::set_error(QM_ERR_ARGUMENT, "qm_distribution_merge_states: too many lines");
    std::vector<double> means(n_lines * QM_WEATHER_STATES);
    for (size_t k = 0; k < n_lines; ++k) std::copy(lines[k].means, lines[k].means + QM_WEATHER_STATES, &means[k * QM_WEATHER_STATES]);
    qm::dist::merge_close_states(means.data(), (int)n_lines, spread);
    for (size_t k = 0; k < n_lines; ++k) std::copy(&means[k * QM_WEATHER_STATES], &means[k * QM_WEATHER_STATES] + QM_WEATHER_STATES, lines[k].means);
    return QM_OK;
}

qm_status qm_loudness_curve_shape(const double *thirds, double *shape_db, int *has_shape) {
    if (thirds == nullptr || shape_db == nullptr || has_shape == nullptr)
        return qm::set_error(QM_ERR_ARGUMENT, "qm_loudness_curve_shape: null argument");
    // Third-octave A-weighting, 25 Hz to 12.5 kHz (IEC 61672-1; physics/src/loudness.rs:14-17).
    static const double a_weighting_db[28] = {-44.7, -39.4, -34.6, -30.2, -26.2, -22.5, -19.1, -16.1, -13.4, -10.9,
                                              -8.6,  -6.6,  -4.8,  -3.2,  -1.9,  -0.8,  0.0,   0.6,   1.0,   1.2,
                                              1.3,   1.2,   1.0,   0.5,   -0.1,  -1.1,  -2.5,  -4.3};
    double a_weighted = 0.0;
    for (int k = 0; k < 28; ++k) {
        if (!(thirds[k] >= 0.0) || !std::isfinite(thirds[k]))
            return qm::set_error(QM_ERR_ARGUMENT, "qm_loudness_curve_shape: band " + std::to_string(k) +
                                                      " is negative or not finite");
        a_weighted += thirds[k] * qm::dist::energy(a_weighting_db[k]);
    }
    *has_shape = a_weighted > 0.0 ? 1 : 0;
    for (int k = 0; k < 28; ++k)
        shape_db[k] = (*has_shape && thirds[k] > 0.0) ? 10.0 * std::log10(thirds[k] / a_weighted) : -INFINITY;
    return QM_OK;
}

qm_status qm_distribution_loudness(double bin_db, const double *bins, const double *curves, double *mean_sone,
                                   double *nden_sone) {
    int n_bins = 0;
    const qm_status status = grid("qm_distribution_loudness", bin_db, n_bins);
    if (status != QM_OK) return status;
    if (bins == nullptr || curves == nullptr || mean_sone == nullptr || nden_sone == nullptr)
        return qm::set_error(QM_ERR_ARGUMENT, "qm_distribution_loudness: null argument");
    double day = 0.0;
    for (int p = 0; p < 3; ++p) {
        const double *period_bins = bins + (size_t)p * 2 * n_bins;
        const double *curve = curves + (size_t)p * QM_LOUDNESS_CURVE_POINTS;
        mean_sone[p] = qm::dist::mean_loudness(period_bins, n_bins, curve, 0.0);
        day += qm::dist::PERIOD_HOURS[p] *
               qm::dist::mean_loudness(period_bins, n_bins, curve, qm::dist::PERIOD_PENALTY_DB[p]);
    }
    *nden_sone = day / 24.0;
    return QM_OK;
}

namespace {

// qm_pixel_read without its capacity error: the lines past `cap` are counted, not written.
qm_status read_pixel(const float *packed, size_t n_floats, uint32_t n_layers, uint32_t period, qm_period_line *lines,
                     int32_t *profiles, size_t cap, size_t *n_lines, double *steady, double *shapes,
                     uint8_t *has_shape) {
    if ((n_floats > 0 && packed == nullptr) || n_lines == nullptr || steady == nullptr || shapes == nullptr ||
        has_shape == nullptr || (cap > 0 && (lines == nullptr || profiles == nullptr)))
        return qm::set_error(QM_ERR_ARGUMENT, "qm_pixel_read: null argument");
    if (period >= 3) return qm::set_error(QM_ERR_ARGUMENT, "qm_pixel_read: period must be 0, 1 or 2");
    const int P = 3, S = QM_WEATHER_STATES;
    size_t at = 0, count = 0;
    auto need = [&](size_t floats, const std::string &what) {
        if (at > n_floats || n_floats - at < floats)
            return qm::set_error(QM_ERR_ARGUMENT, "qm_pixel_read: " + what + " runs past the pixel's " +
                                                      std::to_string(n_floats) + " floats");
        return QM_OK;
    };
    for (uint32_t l = 0; l < n_layers; ++l) {
        const std::string layer = "layer " + std::to_string(l);
        if (need(P + 1, layer) != QM_OK) return QM_ERR_ARGUMENT;
        steady[l] = (double)packed[at + period];
        const float lines_f = packed[at + P];
        at += P + 1;
        if (!(lines_f >= 0.0f) || lines_f != std::floor(lines_f) || lines_f > (float)INT32_MAX)
            return qm::set_error(QM_ERR_ARGUMENT, "qm_pixel_read: " + layer + " has no whole line count");
        const size_t n = (size_t)lines_f;
        if (need(n * QM_PACKED_LINE_FLOATS, layer + "'s lines") != QM_OK) return QM_ERR_ARGUMENT;
        for (size_t k = 0; k < n; ++k, at += QM_PACKED_LINE_FLOATS) {
            const float *f = packed + at;
            if (count < cap) {
                qm_period_line &line = lines[count];
                line.layer = l;
                line.reserved = 0;
                line.energy = (double)f[period];
                for (int st = 0; st < S; ++st) line.means[st] = (double)f[P + period * S + st];
                line.lambda = (double)f[P + P * S + period];
                profiles[count] = f[2 * P + P * S] < 0.0f ? -1 : (int32_t)f[2 * P + P * S];
                line.duty = (double)f[2 * P + P * S + 1 + period];
                line.passing = (double)f[3 * P + P * S + 1 + period];
            }
            ++count;
        }
    }
    for (uint32_t c = 0; c <= n_layers; ++c) {
        if (need((size_t)P * 28, "curve " + std::to_string(c)) != QM_OK) return QM_ERR_ARGUMENT;
        const float *shape = packed + at + (size_t)period * 28;
        has_shape[c] = std::isnan(shape[0]) ? 0 : 1;
        for (int k = 0; k < 28; ++k) shapes[(size_t)c * 28 + k] = has_shape[c] ? (double)shape[k] : -INFINITY;
        at += (size_t)P * 28;
    }
    if (at != n_floats)
        return qm::set_error(QM_ERR_ARGUMENT, "qm_pixel_read: " + std::to_string(n_floats - at) +
                                                  " floats left over after the curves");
    *n_lines = count;
    return QM_OK;
}

}  // namespace

qm_status qm_pixel_read(const float *packed, size_t n_floats, uint32_t n_layers, uint32_t period,
                        qm_period_line *lines, int32_t *profiles, size_t cap, size_t *n_lines, double *steady,
                        double *shapes, uint8_t *has_shape) {
    const qm_status status =
        read_pixel(packed, n_floats, n_layers, period, lines, profiles, cap, n_lines, steady, shapes, has_shape);
    if (status != QM_OK) return status;
    if (*n_lines > cap)
        return qm::set_error(QM_ERR_CAPACITY, "qm_pixel_read: " + std::to_string(*n_lines) + " lines, room for " +
                                                  std::to_string(cap));
    return QM_OK;
}

qm_status qm_distribution_state_means(const double *piece_energy, const double *piece_states, size_t n_pieces,
                                      const double *energy, double *means) {
    if ((n_pieces > 0 && (piece_energy == nullptr || piece_states == nullptr)) || energy == nullptr || means == nullptr)
        return qm::set_error(QM_ERR_ARGUMENT, "qm_distribution_state_means: null argument");
    for (size_t k = 0; k < n_pieces; ++k)
        for (int v = 0; v < 9; ++v) {
            const double x = v < 3 ? piece_energy[3 * k + v] : piece_states[6 * k + (v - 3)];
            if (!(x >= 0.0) || !std::isfinite(x))
                return qm::set_error(QM_ERR_ARGUMENT, "qm_distribution_state_means: piece " + std::to_string(k) +
                                                          " has a negative or non-finite energy");
        }
    qm::dist::WeatherBins weather;
    weather.clear();
    for (size_t k = 0; k < n_pieces; ++k)
        for (int p = 0; p < 3; ++p)
            weather.add(p, piece_energy[3 * k + p], piece_states[6 * k + p], piece_states[6 * k + 3 + p]);
    for (int p = 0; p < 3; ++p) weather.means(p, energy[p], means + (size_t)p * QM_WEATHER_STATES);
    return QM_OK;
}

qm_status qm_hour_groups(const double *shares, size_t n_profiles, uint32_t period, uint32_t runs,
                         uint32_t *group_of_slot, uint32_t *group_hours, double *factors, size_t *n_groups) {
    if ((n_profiles > 0 && shares == nullptr) || group_of_slot == nullptr || group_hours == nullptr ||
        (n_profiles > 0 && factors == nullptr) || n_groups == nullptr)
        return qm::set_error(QM_ERR_ARGUMENT, "qm_hour_groups: null argument");
    if (period >= 3) return qm::set_error(QM_ERR_ARGUMENT, "qm_hour_groups: period must be 0, 1 or 2");
    static const int first_hour[3] = {7, 19, 23};  // traffic.rs:31
    const int hours = (int)qm::dist::PERIOD_HOURS[period];
    if (runs > (uint32_t)hours)
        return qm::set_error(QM_ERR_ARGUMENT, "qm_hour_groups: more runs than the period's " + std::to_string(hours) + " hours");
    for (size_t k = 0; k < 24 * n_profiles; ++k)
        if (!(shares[k] > 0.0) || !std::isfinite(shares[k]))
            return qm::set_error(QM_ERR_ARGUMENT, "qm_hour_groups: share " + std::to_string(k) + " is not positive and finite");
    auto share = [&](size_t profile, int slot) { return shares[profile * 24 + (first_hour[period] + slot) % 24]; };
    std::vector<double> mean(n_profiles);
    for (size_t profile = 0; profile < n_profiles; ++profile) {
        double total = 0.0;
        for (int slot = 0; slot < hours; ++slot) total += share(profile, slot);
        mean[profile] = total / (double)hours;
    }
    auto factor = [&](size_t profile, int slot) { return share(profile, slot) / mean[profile]; };
    std::vector<std::vector<int>> groups;
    if (runs == 0) {
        for (int slot = 0; slot < hours; ++slot) groups.push_back({slot});
    } else {
        std::vector<double> flow(hours);
        for (int slot = 0; slot < hours; ++slot) {
            double total = 0.0;
            for (size_t profile = 0; profile < n_profiles; ++profile) total += factor(profile, slot);
            flow[slot] = total;
        }
        std::vector<int> slots(hours);
        for (int slot = 0; slot < hours; ++slot) slots[slot] = slot;
        std::sort(slots.begin(), slots.end(), [&](int a, int b) { return flow[a] < flow[b] || (flow[a] == flow[b] && a < b); });
        for (uint32_t run = 0; run < runs; ++run) {
            std::vector<int> group(slots.begin() + run * hours / runs, slots.begin() + (run + 1) * hours / runs);
            std::sort(group.begin(), group.end());
            groups.push_back(group);
        }
    }
    for (size_t g = 0; g < groups.size(); ++g) {
        group_hours[g] = (uint32_t)groups[g].size();
        for (int slot : groups[g]) group_of_slot[slot] = (uint32_t)g;
        for (size_t profile = 0; profile < n_profiles; ++profile) {
            double total = 0.0;
            for (int slot : groups[g]) total += factor(profile, slot);
            factors[g * n_profiles + profile] = total / (double)groups[g].size();
        }
    }
    *n_groups = groups.size();
    return QM_OK;
}

qm_status qm_pixel_distributions(const float *packed, size_t n_floats, uint32_t n_layers, double bin_db,
                                 const double *shares, size_t n_profiles, const uint32_t *runs, double *layer_bins,
                                 double *layer_silent, double *place_bins, double *place_silent) {
    int n_bins = 0;
    const qm_status status = grid("qm_pixel_distributions", bin_db, n_bins);
    if (status != QM_OK) return status;
    if ((n_layers > 0 && (layer_bins == nullptr || layer_silent == nullptr)) || place_bins == nullptr ||
        place_silent == nullptr)
        return qm::set_error(QM_ERR_ARGUMENT, "qm_pixel_distributions: null output");
    const size_t bins2 = 2 * (size_t)n_bins;
    std::vector<double> steady(n_layers), shapes(((size_t)n_layers + 1) * 28), each(n_layers * bins2),
        each_silent(n_layers);
    std::vector<uint8_t> has_shape(n_layers + 1);
    for (uint32_t period = 0; period < 3; ++period) {
        // The period's lines: counted first, then read.
        size_t n_lines = 0;
        qm_status read = read_pixel(packed, n_floats, n_layers, period, nullptr, nullptr, 0, &n_lines, steady.data(),
                                    shapes.data(), has_shape.data());
        if (read != QM_OK) return read;
        std::vector<qm_period_line> lines(n_lines);
        std::vector<int32_t> profiles(n_lines);
        read = qm_pixel_read(packed, n_floats, n_layers, period, lines.data(), profiles.data(), n_lines, &n_lines,
                             steady.data(), shapes.data(), has_shape.data());
        if (read != QM_OK) return read;
        std::vector<uint8_t> profiled(n_lines, 0);
        bool any = false;
        for (size_t k = 0; k < n_lines; ++k) {
            if (profiles[k] < 0) continue;
            if ((size_t)profiles[k] >= n_profiles)
                return qm::set_error(QM_ERR_ARGUMENT, "qm_pixel_distributions: line " + std::to_string(k) +
                                                          " follows profile " + std::to_string(profiles[k]) + " of " +
                                                          std::to_string(n_profiles));
            profiled[k] = 1;
            any = true;
        }
        // The period's groups of hours (traffic.rs:251-279): one at the mean flow unless a line
        // follows a profile.
        uint32_t hours = 1;
        std::vector<uint32_t> group_hours(1, 1);
        std::vector<double> factors(n_lines, 1.0);
        if (any) {
            hours = (uint32_t)qm::dist::PERIOD_HOURS[period];
            std::vector<uint32_t> slot_group(12);
            std::vector<double> profile_factors(12 * n_profiles);
            group_hours.assign(12, 0);
            size_t n_groups = 0;
            const qm_status grouped = qm_hour_groups(shares, n_profiles, period, runs ? runs[period] : 0,
                                                     slot_group.data(), group_hours.data(), profile_factors.data(),
                                                     &n_groups);
            if (grouped != QM_OK) return grouped;
            group_hours.resize(n_groups);
            factors.assign(n_groups * n_lines, 1.0);
            for (size_t g = 0; g < n_groups; ++g)
                for (size_t k = 0; k < n_lines; ++k)
                    if (profiled[k]) factors[g * n_lines + k] = profile_factors[g * n_profiles + (size_t)profiles[k]];
        }
        double silent = 0.0;
        const qm_status layered = qm_distribution_layers_grouped(
            bin_db, lines.data(), n_lines, steady.data(), n_layers, hours, group_hours.data(), group_hours.size(),
            factors.data(), profiled.data(), each.data(), each_silent.data(), place_bins + period * bins2, &silent);
        if (layered != QM_OK) return layered;
        place_silent[period] = silent;
        for (uint32_t l = 0; l < n_layers; ++l) {
            std::copy(each.begin() + l * bins2, each.begin() + (l + 1) * bins2, layer_bins + ((size_t)l * 3 + period) * bins2);
            layer_silent[(size_t)l * 3 + period] = each_silent[l];
        }
    }
    return QM_OK;
}

qm_status qm_pixel_ndens(const float *packed, size_t n_floats, uint32_t n_layers, double bin_db, const double *shares,
                         size_t n_profiles, const uint32_t *runs, const double *curves, double *ndens) {
    if (curves == nullptr || ndens == nullptr) return qm::set_error(QM_ERR_ARGUMENT, "qm_pixel_ndens: null curves or ndens");
    int n_bins = 0;
    const qm_status status = grid("qm_pixel_ndens", bin_db, n_bins);
    if (status != QM_OK) return status;
    const size_t bins2 = 2 * (size_t)n_bins, curve = 3 * (size_t)QM_LOUDNESS_CURVE_POINTS;
    std::vector<double> layer_bins(n_layers * 3 * bins2), layer_silent(n_layers * 3), place_bins(3 * bins2),
        place_silent(3);
    const qm_status made = qm_pixel_distributions(packed, n_floats, n_layers, bin_db, shares, n_profiles, runs,
                                                  layer_bins.data(), layer_silent.data(), place_bins.data(),
                                                  place_silent.data());
    if (made != QM_OK) return made;
    double mean[3];
    for (uint32_t l = 0; l <= n_layers; ++l) {
        const double *bins = l < n_layers ? layer_bins.data() + (size_t)l * 3 * bins2 : place_bins.data();
        const qm_status read = qm_distribution_loudness(bin_db, bins, curves + l * curve, mean, ndens + l);
        if (read != QM_OK) return read;
    }
    return QM_OK;
}

qm_status qm_distribution_percentiles(double bin_db, const double *bins, double *levels) {
    int n_bins = 0;
    const qm_status status = grid("qm_distribution_percentiles", bin_db, n_bins);
    if (status != QM_OK) return status;
    if (bins == nullptr || levels == nullptr)
        return qm::set_error(QM_ERR_ARGUMENT, "qm_distribution_percentiles: null bins or levels");
    static const double exceeded[4] = {0.05, 0.1, 0.5, 0.9};
    for (int k = 0; k < 4; ++k)
        for (int p = 0; p < 3; ++p)
            levels[k * 3 + p] = qm::dist::exceeded_db(bins + (size_t)p * 2 * n_bins, n_bins, exceeded[k]);
    return QM_OK;
}

qm_status qm_distribution_pass_values(double mean, double *values, size_t cap, size_t *n_values) {
    if (n_values == nullptr || (cap > 0 && values == nullptr))
        return qm::set_error(QM_ERR_ARGUMENT, "qm_distribution_pass_values: null values or n_values");
    // Above about 745 the silence's share exp(-mean) underflows to 0, every share after it stays
    // 0 and the time left never falls under 1e-12: the stream is then steady to any decibel grid.
    if (!(mean > 0.0) || !(mean <= 700.0))
        return qm::set_error(QM_ERR_ARGUMENT, "qm_distribution_pass_values: mean must lie in (0, 700]");
    size_t n = 0;
    auto push = [&](double value, double share) {
        if (n < cap) {
            values[2 * n] = value;
            values[2 * n + 1] = share;
        }
        ++n;
    };
    // Poisson numbers of passes in progress, each at the stream's mean over `mean`, up to the
    // number a moment in 1e12 exceeds, which takes what is left of the time and of the mean;
    // the time left after the silence is -expm1(-mean), exact for tiny means.
    double share = std::exp(-mean);
    push(0.0, share);
    double time_left = -std::expm1(-mean), mean_left = 1.0, count = 0.0;
    for (;;) {
        count += 1.0;
        share *= mean / count;
        if (time_left - share <= 1e-12) {
            push(mean_left / time_left, time_left);
            break;
        }
        time_left -= share;
        mean_left -= share * count / mean;
        push(count / mean, share);
    }
    *n_values = n;
    if (n > cap)
        return qm::set_error(QM_ERR_CAPACITY,
                             "qm_distribution_pass_values: " + std::to_string(n) + " values, room for " + std::to_string(cap));
    return QM_OK;
}

}  // extern "C"
