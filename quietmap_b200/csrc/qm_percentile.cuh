// How a line of moving emitters' level varies in time (Kurze 1971, "Statistics of road traffic
// noise", J. Sound Vib. 18): the intensity, relative to its mean, that a line with `lambda`
// emitters per distance of its closest point stays below with probability p. The sampler follows
// physics/src/percentile.rs:27-160 over a 41 x 100 quantile table the host builds by the
// reference's own seeded simulation (physics/src/percentile_tests.rs:1-102).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace qm {

constexpr int LINE_LEVEL_ROWS = 41, LINE_LEVEL_QUANTILES = 100;
constexpr double LINE_LEVEL_LAMBDA_MIN = 1e-4, LINE_LEVEL_STEPS_PER_DECADE = 8.0, LINE_LEVEL_DENSE = 10.0;

// The standard normal quantile by Acklam's published rational approximation (relative error
// about 1e-9): one rational function in the centre, its tail form within 0.02425 of either end.
__host__ __device__ inline double line_level_normal_quantile(double p) {
    const double a0 = -3.969683028665376e1, a1 = 2.209460984245205e2, a2 = -2.759285104469687e2,
                 a3 = 1.38357751867269e2, a4 = -3.066479806614716e1, a5 = 2.506628277459239;
    const double b0 = -5.447609879822406e1, b1 = 1.615858368580409e2, b2 = -1.556989798598866e2,
                 b3 = 6.680131188771972e1, b4 = -1.328068155288572e1;
    const double c0 = -7.784894002430293e-3, c1 = -3.223964580411365e-1, c2 = -2.400758277161838,
                 c3 = -2.549671010366478, c4 = 4.374664141464968, c5 = 2.938163982698783;
    const double d0 = 7.784695709041462e-3, d1 = 3.224671290700398e-1, d2 = 2.445134137142996,
                 d3 = 3.754408661907416;
    auto tail = [&](double q) {
        return (((((c0 * q + c1) * q + c2) * q + c3) * q + c4) * q + c5) /
               ((((d0 * q + d1) * q + d2) * q + d3) * q + 1.0);
    };
    if (p < 0.02425) return tail(sqrt(-2.0 * log(p)));
    if (p > 1.0 - 0.02425) return -tail(sqrt(-2.0 * log(1.0 - p)));
    const double q = p - 0.5, r = q * q;
    return (((((a0 * r + a1) * r + a2) * r + a3) * r + a4) * r + a5) * q /
           (((((b0 * r + b1) * r + b2) * r + b3) * r + b4) * r + 1.0);
}

__host__ __device__ inline double line_level_probability(int k) { return ((double)k + 0.5) / LINE_LEVEL_QUANTILES; }

// The table's log intensity at lambda (LINE_LEVEL_LAMBDA_MIN <= lambda < LINE_LEVEL_DENSE) and
// p (at most the last quantile's probability): log-linear between rows, and between quantiles
// linear in the log of 1 - p.
__host__ __device__ inline double line_level_table_value(const float *table, double lambda, double p) {
    const double position = fmin(fmax(log10(lambda / LINE_LEVEL_LAMBDA_MIN) * LINE_LEVEL_STEPS_PER_DECADE, 0.0),
                                 (double)(LINE_LEVEL_ROWS - 1));
    const int row = (int)floor(position);
    const double fraction = position - trunc(position);
    const double pq = fmax(p, line_level_probability(0));
    const int k0 = (int)floor(pq * LINE_LEVEL_QUANTILES - 0.5);
    const int k = k0 < LINE_LEVEL_QUANTILES - 2 ? k0 : LINE_LEVEL_QUANTILES - 2;
    const double t = (log(1.0 - pq) - log(1.0 - line_level_probability(k))) /
                     (log(1.0 - line_level_probability(k + 1)) - log(1.0 - line_level_probability(k)));
    auto log_quantile = [&](int r) {
        const double here = log(fmax((double)table[r * LINE_LEVEL_QUANTILES + k], 1e-30));
        const double next = log(fmax((double)table[r * LINE_LEVEL_QUANTILES + k + 1], 1e-30));
        return here + t * (next - here);
    };
    const double low = log_quantile(row), high = log_quantile(row + 1 < LINE_LEVEL_ROWS ? row + 1 : row);
    return exp(low + fraction * (high - low));
}

// The intensity relative to the mean: silence without emitters, 1 for a steady source, normal
// for a dense line; above the last quantile the table goes on as its nearest emitter's passing
// (an emitter within s distances, probability 1 - exp(-2 lambda s), gives 1 / (lambda pi
// (1 + s^2))); a line sparser than the table is the first row scaled by lambda.
__host__ __device__ inline double line_relative_intensity(const float *table, double lambda, double p) {
    const double pi = 3.14159265358979323846;
    if (!isfinite(lambda)) return 1.0;
    if (lambda <= 0.0) return 0.0;
    const double bottom = line_level_probability(0), top = line_level_probability(LINE_LEVEL_QUANTILES - 1);
    if (lambda >= LINE_LEVEL_DENSE) {
        const double deviation = 1.0 / sqrt(2.0 * pi * lambda);
        return fmax(1.0 + deviation * line_level_normal_quantile(fmin(fmax(p, bottom), top)), 0.0);
    }
    auto passing = [&](double ln_p) {
        const double s = -ln_p / (2.0 * lambda);
        return 1.0 / (lambda * pi * (1.0 + s * s));
    };
    const double q = p > top ? top : p;
    double value = lambda < LINE_LEVEL_LAMBDA_MIN
                       ? lambda / LINE_LEVEL_LAMBDA_MIN * line_level_table_value(table, LINE_LEVEL_LAMBDA_MIN, q)
                       : line_level_table_value(table, lambda, q);
    if (p > top) value = value + passing(log(p)) - passing(log(top));
    return value;
}

// Internal linkage: every translation unit that includes this header for the sampler gets its
// own copy of the kernel, and only qm_lib.cu launches it.
static __global__ void __launch_bounds__(256) line_level_kernel(const float *table, const double *lambda, const double *p,
                                                                size_t n, double *out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = line_relative_intensity(table, lambda[i], p[i]);
}

}  // namespace qm
