// Batch::loudness on the device (paint/src/exact.rs:171-175; the reference's card does it in
// paint-gpu/kernels/loudness.cuh:42-81 and 166-226): for each packed pixel (paint/src/sone.rs:32-51,
// 217-234), its layers' and its place's distributions of level over each period
// (popup/src/percentiles.rs:88-282), then each on its curve (popup/src/loudness.rs:179-205) for Nden.
//
// One CTA a pixel, one warp a weather state. A warp builds, for its state and the period's group of
// hours, each layer's distribution in shared memory (its floor, then each moving line added with
// the lanes over the distribution's moments, qm_distribution.cuh `runs`) and the place's (the
// holding layers' floors, then each moving layer added as an independent distribution). After each
// layer the CTA adds the ten states' distributions into the period's mixture in state order, as the
// host composition (qm_distribution_layers_grouped) adds them, so the mixtures hold no atomics'
// order. The period's curves are Zwicker's loudness of the pixel's shapes at the whole decibels its
// mixtures need; Nden weighs the periods' mean loudness by their hours and penalties.
#pragma once

#include "qm_distribution.cuh"
#include "qm_percentile.cuh"
#include "qm_zwicker.cuh"

namespace qm {
namespace pix {

constexpr int PERIODS = 3;
constexpr int STATES = dist::WEATHER_STATES;
constexpr int LINE_FLOATS = 43;  // QM_PACKED_LINE_FLOATS
constexpr int THIRDS = 28;
constexpr int MAX_LAYERS = 8;
constexpr int MAX_BINS = 96;     // bin_db of at least 1.875 dB (the map's grid is 2 dB: 90 bins)
constexpr int MAX_VALUES = 256;  // a moving line's values: Kurze's 124 nodes, a stream's passes
constexpr int MAX_GROUPS = 12;
constexpr int THREADS = STATES * 32;

// A period's hours and penalty (physics/src/bands.rs:16-18), as dist::PERIOD_HOURS and
// dist::PERIOD_PENALTY_DB give them to the host.
__device__ __forceinline__ double period_hours(int p) { return p == 0 ? 12.0 : p == 1 ? 4.0 : 8.0; }
__device__ __forceinline__ double period_penalty_db(int p) { return p == 0 ? 0.0 : p == 1 ? 5.0 : 10.0; }

// A pixel's status bits.
constexpr uint32_t BAD_PACKING = 1u, BAD_PROFILE = 2u, TOO_MANY_VALUES = 4u, BAD_LINE = 8u;

struct Args {
    const float *input;
    const uint64_t *offsets;  // each pixel's first float
    uint64_t n_floats;
    uint32_t n_pixels, n_layers;
    double bin_db;
    int n_bins;
    const float *table;          // the line-level quantile table
    const double *factors;       // [PERIODS][MAX_GROUPS][n_profiles]: a profile's flow in a group
    const uint32_t *group_hours; // [PERIODS][MAX_GROUPS]
    uint32_t n_groups[PERIODS];
    uint32_t n_profiles;
    float *ndens;      // [n_pixels][n_layers + 1]
    uint32_t *status;  // [n_pixels]
};

// Doubles of a warp's shared memory: layer and place buffers (cur/spare each), a moving line's
// values and their running sums, and the accumulator of a sum's silence.
__host__ __device__ inline int warp_doubles(int n_bins) { return 8 * n_bins + 2 * MAX_VALUES + 2 * (MAX_VALUES + 1) + 2; }
// Doubles of the CTA's mixtures: per curve (layers, then the place) its bins and its silence.
__host__ __device__ inline int mixture_doubles(int n_bins) { return (MAX_LAYERS + 1) * (2 * n_bins + 1); }
__host__ __device__ inline size_t shared_bytes(int n_bins) {
    return ((size_t)STATES * warp_doubles(n_bins) + mixture_doubles(n_bins) + (MAX_LAYERS + 1) + STATES +
            (size_t)STATES * 4 * MAX_LAYERS) * sizeof(double) +
           192 * sizeof(float) + 192;
}

// A line's view of one period from its 43 packed floats (sone.rs:217-234 order): energy per period,
// means per period and state, lambda per period, profile, duty per period, passes per period.
struct LineIn {
    const float *f;
    int p;
    __device__ double energy() const { return (double)f[p]; }
    __device__ double mean(int state) const { return (double)f[PERIODS + p * STATES + state]; }
    __device__ double lambda() const { return (double)f[PERIODS + PERIODS * STATES + p]; }
    __device__ int profile() const { return f[2 * PERIODS + PERIODS * STATES] < 0.0f ? -1 : (int)f[2 * PERIODS + PERIODS * STATES]; }
    __device__ double duty() const { return (double)f[2 * PERIODS + PERIODS * STATES + 1 + p]; }
    __device__ double passing() const { return (double)f[3 * PERIODS + PERIODS * STATES + 1 + p]; }
};

// How a line sounds at a flow factor (the host's shape_layer, lines.rs:172-195): its kind and, for
// a sparse line, the relative intensity it exceeds a thousandth of the time.
__device__ inline int line_kind(const LineIn &line, double factor, const float *table, double &exceeded) {
    constexpr double MIN_POSITIVE = 2.2250738585072014e-308;
    exceeded = 0.0;
    const double passing = line.passing(), duty = line.duty(), lambda = line.lambda() * factor;
    if (!isnan(passing)) return (passing >= MIN_POSITIVE && passing < dist::PASSES_HOLD_MEAN) ? dist::SHAPE_MOVES : dist::SHAPE_HOLDS;
    if (!isnan(duty)) return duty > 0.0 ? dist::SHAPE_MOVES : dist::SHAPE_SILENT;
    if (!(lambda >= dist::HOLDS_MEAN_LAMBDA)) {
        exceeded = line_relative_intensity(table, lambda, 1.0 - dist::HELD_EXCEEDED);
        return dist::SHAPE_SPARSE;
    }
    return dist::SHAPE_HOLDS;
}

// Values in increasing order of intensity (stable), with their running sums, by one lane
// (distribution.rs:243-256, as the host's sorted_values): pairs[n][2] in place, sums[n + 1][2].
__device__ inline void sort_and_sum(double *pairs, double *sums, int n) {
    for (int i = 0; i < n; ++i) pairs[2 * i] += 0.0;
    for (int i = 1; i < n; ++i) {
        const double v = pairs[2 * i], s = pairs[2 * i + 1];
        int j = i;
        while (j > 0 && pairs[2 * (j - 1)] > v) {
            pairs[2 * j] = pairs[2 * (j - 1)];
            pairs[2 * j + 1] = pairs[2 * (j - 1) + 1];
            --j;
        }
        pairs[2 * j] = v;
        pairs[2 * j + 1] = s;
    }
    sums[0] = sums[1] = 0.0;
    for (int k = 0; k < n; ++k) {
        sums[2 * (k + 1)] = __dadd_rn(sums[2 * k], pairs[2 * k + 1]);
        sums[2 * (k + 1) + 1] = __dadd_rn(sums[2 * k + 1], __dmul_rn(pairs[2 * k + 1], pairs[2 * k]));
    }
}

// A moving line's values into pairs/sums (the warp together); returns their count, -1 past
// MAX_VALUES. Passes (distribution.rs:283-298) and an event's two values by one lane, Kurze's nodes
// (distribution.rs:17-32 with physics/src/percentile.rs's sampler) a lane a node.
__device__ inline int line_values(const LineIn &line, double factor, const float *table, double *pairs, double *sums) {
    const int lane = threadIdx.x & 31;
    int n = 0;
    const double passing = line.passing(), duty = line.duty();
    if (!isnan(passing)) {
        if (lane == 0) {
            double share = exp(-passing);
            pairs[0] = 0.0;
            pairs[1] = share;
            n = 1;
            double time_left = -expm1(-passing), mean_left = 1.0, count = 0.0;
            for (;;) {
                count += 1.0;
                share *= passing / count;
                if (n >= MAX_VALUES) {
                    n = -1;
                    break;
                }
                if (time_left - share <= 1e-12) {
                    pairs[2 * n] = mean_left / time_left;
                    pairs[2 * n + 1] = time_left;
                    ++n;
                    break;
                }
                time_left -= share;
                mean_left -= share * count / passing;
                pairs[2 * n] = count / passing;
                pairs[2 * n + 1] = share;
                ++n;
            }
        }
        n = __shfl_sync(0xffffffffu, n, 0);
    } else if (!isnan(duty)) {
        if (lane == 0) {
            pairs[0] = 0.0;
            pairs[1] = 1.0 - duty;
            pairs[2] = 1.0 / duty;
            pairs[3] = duty;
        }
        n = 2;
    } else {
        const double lambda = line.lambda() * factor;
        for (int k = lane; k < dist::NODES; k += 32) {
            double p, share;
            dist::node(k, p, share);
            pairs[2 * k] = line_relative_intensity(table, lambda, p);
            pairs[2 * k + 1] = share;
        }
        n = dist::NODES;
    }
    __syncwarp();
    if (n > 0 && lane == 0) sort_and_sum(pairs, sums, n);
    __syncwarp();
    return n;
}

// out = in with the line (values times `scale`) added at every moment (dist::with_line), the lanes
// over the moments: each moment's runs (dist::runs) added into out's bins by shared-memory atomics.
// out's silence lands in *out_silent.
__device__ inline void warp_with_line(double bin_db, int n_bins, const double *in_bins, double in_silent,
                                      const dist::Values &line, double scale, double *out_bins, double *out_silent) {
    const int lane = threadIdx.x & 31;
    for (int k = lane; k < 2 * n_bins; k += 32) out_bins[k] = 0.0;
    if (lane == 0) *out_silent = 0.0;
    __syncwarp();
    auto add = [&](double intensity, double share) {
        auto visit = [&](int bin, double shares, double weighted) {
            if (bin < 0) {
                atomicAdd(out_silent, share * shares);
            } else {
                atomicAdd(&out_bins[2 * bin], share * shares);
                atomicAdd(&out_bins[2 * bin + 1], share * (intensity * shares + weighted));
            }
        };
        dist::runs(bin_db, n_bins, intensity, line, scale, visit);
    };
    if (lane == 0 && in_silent > 0.0) add(0.0, in_silent);
    for (int b = lane; b < n_bins; b += 32) {
        const double share = in_bins[2 * b];
        if (share > 0.0) add(in_bins[2 * b + 1] / share, share);
    }
    __syncwarp();
}

// out = in with an independent distribution `other` added (dist::with_distribution): its bins'
// mean intensities and its silence as a line's values, built by one lane in the host's order.
__device__ inline void warp_with_distribution(double bin_db, int n_bins, const double *in_bins, double in_silent,
                                              const double *other_bins, double other_silent, double *pairs,
                                              double *sums, double *out_bins, double *out_silent) {
    const int lane = threadIdx.x & 31;
    int n = 0;
    if (lane == 0) {
        if (other_silent > 0.0) {
            pairs[0] = 0.0;
            pairs[1] = other_silent;
            n = 1;
        }
        for (int b = 0; b < n_bins; ++b) {
            const double share = other_bins[2 * b];
            if (!(share > 0.0)) continue;
            const double intensity = other_bins[2 * b + 1] / share;
            int at = n;
            while (at > 0 && pairs[2 * (at - 1)] > intensity) {
                pairs[2 * at] = pairs[2 * (at - 1)];
                pairs[2 * at + 1] = pairs[2 * (at - 1) + 1];
                --at;
            }
            pairs[2 * at] = intensity;
            pairs[2 * at + 1] = share;
            ++n;
        }
        sums[0] = sums[1] = 0.0;
        for (int k = 0; k < n; ++k) {
            sums[2 * (k + 1)] = __dadd_rn(sums[2 * k], pairs[2 * k + 1]);
            sums[2 * (k + 1) + 1] = __dadd_rn(sums[2 * k + 1], __dmul_rn(pairs[2 * k + 1], pairs[2 * k]));
        }
    }
    n = __shfl_sync(0xffffffffu, n, 0);
    __syncwarp();
    warp_with_line(bin_db, n_bins, in_bins, in_silent, dist::Values{pairs, sums, n}, 1.0, out_bins, out_silent);
}

// A single steady intensity over an all-silent distribution (dist::over from silence): the
// steady values written to pairs/sums, then added.
__device__ inline void warp_steady(double bin_db, int n_bins, double intensity, double *zero_bins, double *pairs,
                                   double *sums, double *out_bins, double *out_silent) {
    const int lane = threadIdx.x & 31;
    for (int k = lane; k < 2 * n_bins; k += 32) zero_bins[k] = 0.0;
    if (lane == 0) {
        const dist::Steady steady(intensity);
        pairs[0] = steady.pairs[0];
        pairs[1] = steady.pairs[1];
        for (int k = 0; k < 4; ++k) sums[k] = steady.sums[k];
    }
    __syncwarp();
    warp_with_line(bin_db, n_bins, zero_bins, 1.0, dist::Values{pairs, sums, 1}, 1.0, out_bins, out_silent);
}

__global__ void __launch_bounds__(THREADS, 1) pixel_loudness_kernel(Args A) {
    extern __shared__ __align__(16) double smem[];
    const int nb = A.n_bins, warp = threadIdx.x >> 5, lane = threadIdx.x & 31, state = warp;
    const int L = (int)A.n_layers;
    // Shared layout: the warps' areas, the mixtures, the Nden sums, per warp the layers' floors
    // and holds (and the current buffers' places), one curve's points, its needed steps.
    double *area = smem + (size_t)warp * warp_doubles(nb);
    double *mix = smem + (size_t)STATES * warp_doubles(nb);
    double *nden = mix + mixture_doubles(nb);
    double *silents = nden + (MAX_LAYERS + 1);  // [STATES]: each warp's current distribution's silence
    double *floors_all = silents + STATES;
    double *floors = floors_all + (size_t)warp * 4 * MAX_LAYERS;  // floors, holds, then spare
    float *curve = reinterpret_cast<float *>(floors_all + STATES * 4 * MAX_LAYERS);
    unsigned char *needed = reinterpret_cast<unsigned char *>(curve + 192);
    __shared__ int s_start[MAX_LAYERS], s_count[MAX_LAYERS], s_curves, s_cur[STATES];
    __shared__ uint32_t s_status;
    __shared__ int s_groups, s_hours;
    double *bufA = area, *bufB = area + 2 * nb, *bufC = area + 4 * nb, *bufD = area + 6 * nb;
    double *pairs = area + 8 * nb, *sums = pairs + 2 * MAX_VALUES, *acc_silent = sums + 2 * (MAX_VALUES + 1);
    const uint32_t pixel = blockIdx.x;
    const float *in = A.input + A.offsets[pixel];
    const uint64_t end = pixel + 1 < A.n_pixels ? A.offsets[pixel + 1] : A.n_floats;
    const uint64_t n_floats = end - A.offsets[pixel];
    if (threadIdx.x == 0) {
        // The packing (read_pixel's checks): per layer its steady energies and its line count,
        // whole and non-negative, its lines within the pixel, then the curves, nothing left over.
        uint32_t st = 0;
        uint64_t at = 0;
        for (int l = 0; l < L && st == 0; ++l) {
            if (at + PERIODS + 1 > n_floats) {
                st = BAD_PACKING;
                break;
            }
            const float count = in[at + PERIODS];
            if (!(count >= 0.0f) || count != floorf(count) || count > 1e7f) {
                st = BAD_PACKING;
                break;
            }
            s_start[l] = (int)(at + PERIODS + 1);
            s_count[l] = (int)count;
            at += PERIODS + 1 + (uint64_t)count * LINE_FLOATS;
        }
        s_curves = (int)at;
        if (st == 0 && at + (uint64_t)(L + 1) * PERIODS * THIRDS != n_floats) st = BAD_PACKING;
        s_status = st;
        for (int c = 0; c <= L; ++c) nden[c] = 0.0;
    }
    __syncthreads();
    if (s_status != 0) {
        if (threadIdx.x == 0) A.status[pixel] = s_status;
        for (int c = threadIdx.x; c <= L; c += blockDim.x) A.ndens[(size_t)pixel * (L + 1) + c] = NAN;
        return;
    }
    const int mix_stride = 2 * nb + 1;
    for (int p = 0; p < PERIODS; ++p) {
        for (int k = threadIdx.x; k < (L + 1) * mix_stride; k += blockDim.x) mix[k] = 0.0;
        if (threadIdx.x == 0) {
            // The period's lines checked as the host checks them, and whether any follows a profile.
            bool any = false;
            uint32_t st = 0;
            for (int l = 0; l < L; ++l) {
                const double steady = (double)in[s_start[l] - PERIODS - 1 + p];
                if (!(steady >= 0.0) || !isfinite(steady)) st |= BAD_LINE;
                for (int k = 0; k < s_count[l]; ++k) {
                    const LineIn line{in + s_start[l] + k * LINE_FLOATS, p};
                    if (isnan(line.energy()) || isnan(line.lambda()) || (!isnan(line.duty()) && line.duty() > 1.0))
                        st |= BAD_LINE;
                    for (int s = 0; s < STATES; ++s)
                        if (!(line.mean(s) >= 0.0) || !isfinite(line.mean(s))) st |= BAD_LINE;
                    const int profile = line.profile();
                    if (profile >= 0) {
                        any = true;
                        if ((uint32_t)profile >= A.n_profiles) st |= BAD_PROFILE;
                    }
                }
            }
            s_status |= st;
            s_groups = any ? (int)A.n_groups[p] : 1;
            s_hours = any ? (int)period_hours(p) : 1;
        }
        __syncthreads();
        if (s_status != 0) break;
        const int groups = s_groups, hours = s_hours;
        for (int g = 0; g < groups; ++g) {
            const double weight = (double)(hours == 1 ? 1u : A.group_hours[p * MAX_GROUPS + g]) / (double)((uint64_t)hours * STATES);
            // A line's flow factor in this group: its profile's (a layer none of whose lines follows a
            // profile stays at its mean flow, as do its lines).
            auto factor_of = [&](const LineIn &line) {
                const int profile = line.profile();
                return (hours == 1 || profile < 0) ? 1.0 : A.factors[((size_t)p * MAX_GROUPS + g) * A.n_profiles + profile];
            };
            auto layer_alike = [&](int l) {
                for (int k = 0; k < s_count[l]; ++k)
                    if (LineIn{in + s_start[l] + k * LINE_FLOATS, p}.profile() >= 0) return false;
                return true;
            };
            // The floors and holds of every layer in this warp's state (dist::moment_floor,
            // dist::moving_lines), warp-uniform.
            double place_floor = 0.0;
            for (int l = 0; l < L; ++l) {
                const bool alike = hours == 1 || layer_alike(l);
                double floor = (double)in[s_start[l] - PERIODS - 1 + p], held = 0.0;
                bool moves = false;
                for (int k = 0; k < s_count[l]; ++k) {
                    const LineIn line{in + s_start[l] + k * LINE_FLOATS, p};
                    const double f = alike ? 1.0 : factor_of(line);
                    const double mean = line.mean(state) * f;
                    if (line.energy() <= 0.0 || mean <= 0.0) continue;
                    double exceeded;
                    const int kind = line_kind(line, f, A.table, exceeded);
                    if (kind == dist::SHAPE_HOLDS) floor += mean;
                    if (kind == dist::SHAPE_SPARSE) held += mean;
                    if (kind == dist::SHAPE_MOVES) moves = true;
                }
                const double steady_energy = floor + held;
                for (int k = 0; k < s_count[l]; ++k) {
                    const LineIn line{in + s_start[l] + k * LINE_FLOATS, p};
                    const double f = alike ? 1.0 : factor_of(line);
                    const double mean = line.mean(state) * f;
                    if (line.energy() <= 0.0 || mean <= 0.0) continue;
                    double exceeded;
                    if (line_kind(line, f, A.table, exceeded) != dist::SHAPE_SPARSE) continue;
                    if (mean * exceeded < dist::HELD_SHARE * steady_energy)
                        floor += mean;
                    else
                        moves = true;
                }
                if (lane == 0) {
                    floors[l] = floor;
                    floors[MAX_LAYERS + l] = moves ? 0.0 : 1.0;
                    floors[2 * MAX_LAYERS + l] = steady_energy;
                }
                if (!moves) place_floor += floor;
            }
            __syncwarp();
            // The place: the holding layers' floors, then each moving layer in order.
            double place_silent;
            warp_steady(A.bin_db, nb, place_floor, bufC, pairs, sums, bufD, acc_silent);
            place_silent = *acc_silent;
            double *place = bufD, *place_spare = bufC;
            for (int l = 0; l < L; ++l) {
                const bool alike = hours == 1 || layer_alike(l);
                // The layer in this state: its floor, then its moving lines (events and streams, then
                // the sparse lines not held), in the host's order.
                warp_steady(A.bin_db, nb, floors[l], bufA, pairs, sums, bufB, acc_silent);
                double silent = *acc_silent;
                double *cur = bufB, *spare = bufA;
                const double steady_energy = floors[2 * MAX_LAYERS + l];
                for (int pass = 0; pass < 2; ++pass)
                    for (int k = 0; k < s_count[l]; ++k) {
                        const LineIn line{in + s_start[l] + k * LINE_FLOATS, p};
                        const double f = alike ? 1.0 : factor_of(line);
                        const double mean = line.mean(state) * f;
                        if (line.energy() <= 0.0 || mean <= 0.0) continue;
                        double exceeded;
                        const int kind = line_kind(line, f, A.table, exceeded);
                        const bool take = pass == 0 ? kind == dist::SHAPE_MOVES
                                                    : (kind == dist::SHAPE_SPARSE &&
                                                       !(mean * exceeded < dist::HELD_SHARE * steady_energy));
                        if (!take) continue;
                        const int n = line_values(line, f, A.table, pairs, sums);
                        if (n < 0) {
                            if (lane == 0) atomicOr(&s_status, TOO_MANY_VALUES);
                            continue;
                        }
                        warp_with_line(A.bin_db, nb, cur, silent, dist::Values{pairs, sums, n}, mean, spare, acc_silent);
                        silent = *acc_silent;
                        double *t = cur;
                        cur = spare;
                        spare = t;
                    }
                if (lane == 0) {
                    s_cur[warp] = cur == bufA ? 0 : 1;
                    silents[warp] = silent;
                }
                __syncthreads();
                // The layer's mixture: every state's distribution in state order (alike layers once).
                if (!alike || g == 0) {
                    const double w = alike ? 1.0 / (double)STATES : weight;
                    double *into = mix + (size_t)l * mix_stride;
                    for (int k = threadIdx.x; k <= 2 * nb; k += blockDim.x) {
                        double v = into[k];
                        for (int s = 0; s < STATES; ++s) {
                            const double *src = smem + (size_t)s * warp_doubles(nb) + (s_cur[s] ? 2 * nb : 0);
                            v = __dadd_rn(v, __dmul_rn(k < 2 * nb ? src[k] : silents[s], w));
                        }
                        into[k] = v;
                    }
                }
                __syncthreads();
                if (floors[MAX_LAYERS + l] == 0.0) {
                    warp_with_distribution(A.bin_db, nb, place, place_silent, cur, silent, pairs, sums, place_spare,
                                           acc_silent);
                    place_silent = *acc_silent;
                    double *t = place;
                    place = place_spare;
                    place_spare = t;
                }
                __syncwarp();
            }
            if (lane == 0) {
                s_cur[warp] = place == bufC ? 0 : 1;
                silents[warp] = place_silent;
            }
            __syncthreads();
            {
                double *into = mix + (size_t)L * mix_stride;
                for (int k = threadIdx.x; k <= 2 * nb; k += blockDim.x) {
                    double v = into[k];
                    for (int s = 0; s < STATES; ++s) {
                        const double *src = smem + (size_t)s * warp_doubles(nb) + (s_cur[s] ? 6 * nb : 4 * nb);
                        v = __dadd_rn(v, __dmul_rn(k < 2 * nb ? src[k] : silents[s], weight));
                    }
                    into[k] = v;
                }
            }
            __syncthreads();
        }
        // The period's loudness on each curve (dist::mean_loudness with the period's penalty): the
        // whole decibels the mixture's levels need, their Zwicker loudness, then the sum over bins.
        const double penalty = period_penalty_db(p);
        for (int c = 0; c <= L; ++c) {
            const float *shape = in + s_curves + ((size_t)c * PERIODS + p) * THIRDS;
            if (isnan(shape[0])) continue;  // no shape: the curve reads 0
            const double *bins = mix + (size_t)c * mix_stride;
            for (int k = threadIdx.x; k <= dist::CURVE_STEPS; k += blockDim.x) needed[k] = 0;
            __syncthreads();
            for (int b = threadIdx.x; b < nb; b += blockDim.x) {
                const double share = bins[2 * b];
                if (!(share > 0.0)) continue;
                const double level = 10.0 * log10(bins[2 * b + 1] / share) + penalty;
                const double position = fmin(fmax(level - dist::CURVE_LOW_DB, 0.0), (double)dist::CURVE_STEPS);
                const double down = floor(position);
                const int below = down < (double)(dist::CURVE_STEPS - 1) ? (int)down : dist::CURVE_STEPS - 1;
                needed[below] = 1;
                needed[below + 1] = 1;
            }
            __syncthreads();
            for (int k = threadIdx.x; k <= dist::CURVE_STEPS; k += blockDim.x) {
                if (!needed[k]) continue;
                float levels[THIRDS];
                for (int t = 0; t < THIRDS; ++t) levels[t] = shape[t] + (float)(dist::CURVE_LOW_DB + (double)k);
                curve[k] = zwicker_sone(levels);
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                double total = 0.0;
                for (int b = 0; b < nb; ++b) {
                    const double share = bins[2 * b];
                    if (!(share > 0.0)) continue;
                    const double level = 10.0 * log10(bins[2 * b + 1] / share) + penalty;
                    const double position = fmin(fmax(level - dist::CURVE_LOW_DB, 0.0), (double)dist::CURVE_STEPS);
                    const double down = floor(position);
                    const int below = down < (double)(dist::CURVE_STEPS - 1) ? (int)down : dist::CURVE_STEPS - 1;
                    const double low = (double)curve[below], high = (double)curve[below + 1];
                    total += share * (low + (high - low) * (position - (double)below));
                }
                nden[c] += period_hours(p) * total;
            }
            __syncthreads();
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) A.status[pixel] = s_status;
    for (int c = threadIdx.x; c <= L; c += blockDim.x)
        A.ndens[(size_t)pixel * (L + 1) + c] = s_status ? NAN : (float)(nden[c] / 24.0);
}

}  // namespace pix
}  // namespace qm
