/* How levels add over time: distributions of the summed level over a period on a decibel grid,
 * and the values of the lines added to them (popup/src/distribution.rs).
 *
 * The arithmetic is one __host__ __device__ source (quietmap_b200/csrc/qm_distribution.cuh) for
 * the per-pixel distributions on the device; these entry points run it on the calling host
 * thread, as the reference's click detail (popup) does for one point, and for checking it
 * without a GPU. They need no device and allocate no device memory. A distribution is
 * bins[n][2] (share of the time, share x the moments' mean intensity) on a grid of bin_db from
 * -30 dB over 180 dB, plus its share in silence. */
#ifndef QM_DISTRIBUTION_H
#define QM_DISTRIBUTION_H

#include <stddef.h>
#include <stdint.h>

#include "qm_batch.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The finest grid: 0.1 dB, 1800 bins. */
#define QM_DISTRIBUTION_MAX_BINS 1800
/* A line's values at the reference's node probabilities (popup/src/distribution.rs:17-32). */
#define QM_DISTRIBUTION_LINE_NODES 124

/* The bins of a grid of bin_db (180 dB over the step, rounded; distribution.rs:55-62);
 * QM_ERR_ARGUMENT for a step that is not positive and finite or gives more than
 * QM_DISTRIBUTION_MAX_BINS. */
qm_status qm_distribution_bins(double bin_db, size_t *n_bins);

/* Distribution::with_line (distribution.rs:86-145, 176-196): `out` is `in` with a line of
 * `n_values` (intensity, share) pairs, in any order, times `scale` added at every moment; each
 * sum lands in the bin of its level with its intensity kept exact. Intensities must be at
 * least 0 and shares at least 0, scale above 0. out_bins may not alias bins. */
qm_status qm_distribution_with_line(double bin_db, const double *bins, double silent, const double *values,
                                    size_t n_values, double scale, double *out_bins, double *out_silent);

/* Distribution::exceeded_db (distribution.rs:152-162): the level exceeded `exceeded` of the
 * time, -inf where silence is. */
qm_status qm_distribution_exceeded_db(double bin_db, const double *bins, double exceeded, double *level_db);

/* line_values (distribution.rs:264-281): a line's intensities relative to its mean with their
 * shares, Kurze's quantiles at `lambda` emitters per distance of its closest point at the node
 * probabilities (QM_DISTRIBUTION_LINE_NODES pairs, by the library's line-level sampler), or
 * with `duty` in (0, 1] an event's mean over its duty while it sounds and silence otherwise
 * (2 pairs). Pass NaN as duty for a line. values[n][2]. */
qm_status qm_distribution_line_values(double lambda, double duty, double *values, size_t cap, size_t *n_values);

/* pass_values (distribution.rs:283-298): the relative intensities of a stream of passes of one
 * level of which `mean` are in progress on average, with their shares. `mean` lies in (0, 700]:
 * above about 745 the silence's share underflows to 0 and the reference's loop does not end.
 * values[n][2]; more than `cap`: the first `cap` are written, *n_values holds the count and the
 * call returns QM_ERR_CAPACITY. */
qm_status qm_distribution_pass_values(double mean, double *values, size_t cap, size_t *n_values);

/* One line over one period (popup/src/percentiles/lines.rs:8-24, that period's fields): the
 * layer it sounds in, its mean energy, its means in the weather states, Kurze's lambda (infinite
 * for a steady source), an event's duty (NaN: not an event) and a stream's passes in progress
 * (NaN: not a stream). */
#define QM_WEATHER_STATES 10
typedef struct {
    uint32_t layer;
    uint32_t reserved;
    double energy;
    double means[QM_WEATHER_STATES];
    double lambda;
    double duty;
    double passing;
} qm_period_line;

/* layered_distributions for one period and one group of hours (popup/src/percentiles.rs:88-160
 * with layer_states and moment, :172-282): each layer's distribution of the summed level over the
 * period and the place's, each weather state a tenth of the time; in a state each layer is its
 * steady energy and its lines that hold their mean, with its moving lines added (events, passes,
 * sparse lines not held), and the place is the steady layers' floors with the moving layers'
 * distributions added. Lines keep their order within a layer; every line runs at its period's
 * mean flow. layer_bins[n_layers][n_bins][2], layer_silent[n_layers], place_bins[n_bins][2]. */
qm_status qm_distribution_layers(double bin_db, const qm_period_line *lines, size_t n_lines, const double *steady,
                                 size_t n_layers, double *layer_bins, double *layer_silent, double *place_bins,
                                 double *place_silent);

/* merge_close_states for one period's lines, in place (popup/src/percentiles/weather.rs:132-176):
 * each run of consecutive weather states in which every line's mean is finite and within `spread`
 * (largest over smallest; the map uses 1.2) gives each line its mean over the run in all of the
 * run's states. The energy stays; equal states then cost one state. */
qm_status qm_distribution_merge_states(qm_period_line *lines, size_t n_lines, double spread);

/* Loudness from the distributions (popup/src/loudness.rs:74-130, 236-269). A period's curve is
 * the loudness (sone) of its received spectrum set to each whole A-weighted decibel from -30 to
 * 160 dB: curve[191], linear between; `qm_loudness_curve_shape` gives the spectrum at an
 * A-weighted 0 dB (thirds[28] energies from 25 Hz to 12.5 kHz; -inf where a band is silent;
 * *has_shape 0 and no shape for a spectrum without A-weighted energy, whose curve is 0), and
 * `qm_zwicker` of that shape plus each whole decibel fills the curve. */
#define QM_LOUDNESS_CURVE_POINTS 191
qm_status qm_loudness_curve_shape(const double *thirds, double *shape_db, int *has_shape);

/* Each period's mean loudness over its distribution (bins[3][n_bins][2]) on its curve
 * (curves[3][191]) and Nden: the periods' means with the evening's 5 dB and the night's 10 dB
 * added to their levels, weighed by their 12, 4 and 8 hours over 24. */
qm_status qm_distribution_loudness(double bin_db, const double *bins, const double *curves, double *mean_sone,
                                   double *nden_sone);

/* One pixel of the reference's packed loudness input (paint/src/sone.rs:32-51, 217-234; read by
 * its card, paint-gpu/kernels/loudness.cuh), read for one period: per layer (n_layers of them,
 * six in the reference) its steady energy per period, its line count and its lines of
 * QM_PACKED_LINE_FLOATS floats (energy per period, means per period and weather state, lambda
 * per period, hourly profile or -1, duty per period or NaN, passes in progress per period or
 * NaN); then each layer's curves and the place's, per period 28 third-octave levels at an
 * A-weighted 0 dB (NaN: no shape). Writes the period's lines (their layers set; at most `cap`,
 * *n_lines the count, QM_ERR_CAPACITY beyond), each line's profile (-1: none) into profiles,
 * steady[n_layers], shapes[n_layers + 1][28] and has_shape[n_layers + 1]. Rejects a pixel
 * whose counts run past `n_floats` or leave floats over. */
#define QM_PACKED_LINE_FLOATS 43
qm_status qm_pixel_read(const float *packed, size_t n_floats, uint32_t n_layers, uint32_t period,
                        qm_period_line *lines, int32_t *profiles, size_t cap, size_t *n_lines, double *steady,
                        double *shapes, uint8_t *has_shape);

/* A line's means in the weather states (popup/src/percentiles/weather.rs:1-127, `Weather::add`
 * over its pieces then `weather_means`): piece k's energy per period piece_energy[k][3], the mix
 * of its homogeneous and favourable energies piece_states[k][2][3] (both 0: it holds its mean in
 * either); `energy[3]` the line's energy, kept in every state where no piece has any. Writes
 * means[3][QM_WEATHER_STATES], ready for qm_period_line.means. */
qm_status qm_distribution_state_means(const double *piece_energy, const double *piece_states, size_t n_pieces,
                                      const double *energy, double *means);

/* hour_factor and hour_groups (popup/src/percentiles/traffic.rs:31-39, 251-279) over the caller's
 * hourly shares[n_profiles][24] (by hour of the day; the reference's are measured road profiles):
 * a period's 12, 4 or 8 hours (from 7, 19 and 23 h) each apart when `runs` is 0, else sorted by
 * their flow summed over the profiles (ties by hour) and cut into `runs` runs (the map: 4, 1, 3).
 * Writes group_of_slot[hours], group_hours[n_groups] and factors[n_groups][n_profiles], each
 * profile's mean hour factor over the group (its flow there against the period's mean), for
 * qm_distribution_layers_grouped; at most 12 groups. */
qm_status qm_hour_groups(const double *shares, size_t n_profiles, uint32_t period, uint32_t runs,
                         uint32_t *group_of_slot, uint32_t *group_hours, double *factors, size_t *n_groups);

/* A packed pixel's distributions for all three periods (layered_distributions on its placed
 * layers, popup/src/percentiles.rs:88-160): the pixel read as qm_pixel_read reads it; where any
 * line follows an hourly profile, each period's hours grouped as qm_hour_groups groups them over
 * shares[n_profiles][24] with runs[3] runs (NULL: every hour apart), each profiled line at its
 * profile's factor in each group; else one group at the mean flow. Writes
 * layer_bins[n_layers][3][n_bins][2], layer_silent[n_layers][3], place_bins[3][n_bins][2] and
 * place_silent[3]. A line naming a profile past n_profiles is refused. */
qm_status qm_pixel_distributions(const float *packed, size_t n_floats, uint32_t n_layers, double bin_db,
                                 const double *shares, size_t n_profiles, const uint32_t *runs, double *layer_bins,
                                 double *layer_silent, double *place_bins, double *place_silent);

/* A packed pixel's Nden per layer and for the place (popup/src/loudness.rs:179-205
 * `layers_loudness`, as paint/src/sone.rs:197-215 gathers them): qm_pixel_distributions, then each
 * layer's distributions on its own curves and the place's on the place's
 * (curves[n_layers + 1][3][191], each the loudness of that curve's shape at each whole decibel
 * from -30 dB; a curve without a shape is all 0 and reads 0). ndens[n_layers + 1]. */
qm_status qm_pixel_ndens(const float *packed, size_t n_floats, uint32_t n_layers, double bin_db, const double *shares,
                         size_t n_profiles, const uint32_t *runs, const double *curves, double *ndens);

/* Batch::loudness on the device (paint/src/exact.rs:171-175; the reference's card:
 * paint-gpu/src/loudness.rs:270-372, kernels/loudness.cuh): `n_pixels` packed pixels laid end to
 * end in input[n_floats], pixel k starting at offsets[k] and ending where the next starts (the last
 * at n_floats), each read as qm_pixel_read reads it. Per pixel, what qm_pixel_ndens computes on the
 * host: its layers' and place's distributions over each period (hours grouped by shares[n_profiles]
 * [24] and runs[3] as qm_pixel_distributions groups them), then Nden per layer and for the place on
 * curves made on the device from the pixel's own shapes (Zwicker's loudness of each shape at every
 * whole decibel a level needs). ndens[n_pixels][n_layers + 1] (a layer without a shape reads 0).
 * Limits: n_layers at most 8; bin_db at least 1.875 dB (at most 96 bins; the map's grid is 2 dB);
 * a moving line of at most 256 values. A malformed pixel, a line that breaks the host's checks or
 * names a profile past n_profiles, or a line over the values limit fails the call with the pixel's
 * index; its Nden is NaN. kernel_ms (nullable) receives the kernel's device time. */
qm_status qm_pixel_loudness(qm_ctx *ctx, const float *input, size_t n_floats, const uint64_t *offsets,
                            size_t n_pixels, uint32_t n_layers, double bin_db, const double *shares,
                            size_t n_profiles, const uint32_t *runs, float *ndens, double *kernel_ms);

/* Percentiles::of (popup/src/percentiles.rs:284-296): the levels exceeded 5, 10, 50 and 90 % of
 * each period's time (dB, -inf where silence is), from bins[3][n_bins][2]; levels[4][3] (L5,
 * L10, L50, L90 by period). */
qm_status qm_distribution_percentiles(double bin_db, const double *bins, double *levels);

/* The same over a period's groups of hours (popup/src/percentiles.rs:88-160 with hour_groups,
 * percentiles/traffic.rs:251-279): a period of `hours` hours whose groups hold group_hours[g]
 * hours each, together every hour of the period; profiled[k] marks a line that follows an hourly profile and factors[g][n_lines]
 * its flow in group g against the period's mean (the mean of its profile's hour factors there,
 * which scales its lambda and its means). A layer none of whose lines is profiled is computed
 * once at its mean flow; the others per group, each group weighing its hours' share. The hourly
 * profiles themselves are the caller's (the reference's measured shares). */
qm_status qm_distribution_layers_grouped(double bin_db, const qm_period_line *lines, size_t n_lines,
                                         const double *steady, size_t n_layers, uint32_t hours,
                                         const uint32_t *group_hours, size_t n_groups, const double *factors,
                                         const uint8_t *profiled, double *layer_bins, double *layer_silent,
                                         double *place_bins, double *place_silent);

#ifdef __cplusplus
}
#endif

#endif /* QM_DISTRIBUTION_H */
