// Doc 29 aircraft noise on a receiver grid: one thread per receiver cell, the flight segments
// streamed through shared memory tile by tile by TMA bulk copies (cp.async.bulk with an mbarrier,
// double buffered), NPD rows and type spectra staged once per CTA. Each (cell, segment) pair is the
// reference's segment SEL at a receiver with no horizons (physics/src/doc29/segment.rs:223-345,
// npd.rs:115-277, corrections.rs:21-85) in FP32; energies are summed per aircraft type with Kahan
// compensation, then spread over the types' third-octave spectra.
#pragma once

#include <cstdint>

#include "../../include/qm_aircraft.h"
#include "qm_stage.cuh"

namespace qm {

// One NPD power row on the device (npd.rs:238-277): SEL and SEL - LAmax at the ten distances, the
// tail's absorption, d0 of the scaled distance, and whether LAmax is the 12 dB placeholder.
struct AcRow {
    float sel[10];
    float sml[10];
    float tail_alpha;
    float d0;
    uint32_t dipole;
    uint32_t pad;
};

struct AcType {
    float v_ref_kt;
    uint32_t installation;
    float share[28];  // unweighted band energy per unit of A-weighted energy
    uint32_t pad[2];
};

struct FlightGridArgs {
    const qm_flight_segment *segs;
    uint32_t n_segs;
    const float4 *boxes;  // per flight: x0, y0, x1, y1
    const AcRow *rows;    // [type][op][row]
    const AcType *types;
    uint32_t n_types;
    double ox, oy, spacing;
    int nx, ny;
    float height;
    double reach2;  // squared reach (<= 0: none)
    float inv_duration;
    float *lae;
    float *thirds;
    unsigned *error;
    unsigned long long *pairs;  // (cell, segment) pairs evaluated, culled ones not counted
};

constexpr int AC_TILE = 128;  // segments per TMA tile (6 KB)
constexpr int AC_THREADS = 256;
__constant__ float LOG10_NPD_FT[10] = {2.3010299956639813f, 2.6020599913279625f, 2.7993405494535817f, 3.0f,
                                    3.3010299956639813f, 3.6020599913279625f, 3.7993405494535817f, 4.0f,
                                    4.2041199826559246f, 4.3979400086720376f};

// What a segment contributes at every receiver, worked out once per tile by one thread a segment:
// its start, direction and lengths, the lower power row and the lerp weight, and the speed
// correction as an energy factor (corrections.rs:21-27 depends on the segment alone).
struct SegPre {
    float sx, sy, sz, dx, dy, dz;
    float inv_l2, inv_h;  // inv_h 0: a vertical segment (no horizontal extent)
    float sqrt_l2, length;
    float w, gain;        // power-row weight; 10^(speed correction / 10)
    uint32_t row_base;    // the lower power row: type * 20 + departure * 10 + row
    uint32_t type, flight, pad;
};

__device__ __forceinline__ SegPre prepare_segment(const qm_flight_segment &g, const AcType *types) {
    SegPre p;
    p.sx = g.start[0];
    p.sy = g.start[1];
    p.sz = g.start[2];
    p.dx = g.end[0] - g.start[0];
    p.dy = g.end[1] - g.start[1];
    p.dz = g.end[2] - g.start[2];
    const float h2 = p.dx * p.dx + p.dy * p.dy, l2 = h2 + p.dz * p.dz;
    p.inv_l2 = l2 > 0.0f ? 1.0f / l2 : 0.0f;
    p.inv_h = h2 <= 1e-6f ? 0.0f : rsqrtf(h2);
    p.sqrt_l2 = sqrtf(l2);
    p.length = fmaxf(p.sqrt_l2, 1.0f);
    const int row = min((int)floorf(g.power), 8);
    p.w = g.power - (float)row;
    p.row_base = g.type * 20 + (g.departure ? 10 : 0) + row;
    const float speed_kt = g.speed_mps * (3600.0f / 1852.0f);
    p.gain = speed_kt > 10.0f ? types[g.type].v_ref_kt / speed_kt : 1.0f;
    p.type = g.type;
    p.flight = g.flight;
    p.pad = 0;
    return p;
}

// The A-weighted sound exposure (energy, 10^(SEL/10)) of one segment at a receiver
// (segment.rs:317-345, no horizons): the NPD level with the speed, installation, lateral and
// finite-segment corrections, the corrections applied as energy factors.
__device__ __forceinline__ float segment_energy(const SegPre &p, const AcRow *rows, const AcType &T, float rx, float ry,
                                                float rz) {
    const float s0 = p.sx - rx, s1 = p.sy - ry, s2 = p.sz - rz;
    const float d0 = p.dx, d1 = p.dy, d2 = p.dz;
    // closest_points (segment.rs:223-265)
    float along, ol0, ol1, ol2, lateral, height, lambda_height;
    if (p.inv_h == 0.0f) {
        along = 0.f;
        ol0 = s0;
        ol1 = s1;
        ol2 = s2;
        lateral = sqrtf(s0 * s0 + s1 * s1);
        height = s2;
        lambda_height = s2;
    } else {
        along = -(s0 * d0 + s1 * d1 + s2 * d2) * p.inv_l2;
        const float c = fminf(fmaxf(along, 0.f), 1.f);
        ol0 = s0 + along * d0;
        ol1 = s1 + along * d1;
        ol2 = s2 + along * d2;
        lateral = fabsf(s0 * d1 - s1 * d0) * p.inv_h;
        const float slant2 = ol0 * ol0 + ol1 * ol1 + ol2 * ol2;
        height = copysignf(sqrtf(fmaxf(slant2 - lateral * lateral, 0.f)), ol2);
        lambda_height = (along >= 0.f && along <= 1.f) ? height : (s2 + c * d2) * p.sqrt_l2 * p.inv_h;
    }
    const float length = p.length;
    const float slant = sqrtf(ol0 * ol0 + ol1 * ol1 + ol2 * ol2);
    // NpdPosition::at (npd.rs:122-135)
    const float sl = fmaxf(slant, 100.0f * 0.3048f);
    const float log_d = __log2f(sl * (1.0f / 0.3048f)) * 0.30102999566f;
    int interval = 0;
#pragma unroll
    for (int k = 8; k >= 1; --k)
        if (interval == 0 && log_d > LOG10_NPD_FT[k]) interval = k;
    const float frac = (log_d - LOG10_NPD_FT[interval]) / (LOG10_NPD_FT[interval + 1] - LOG10_NPD_FT[interval]);
    const bool tail = sl >= 25000.0f * 0.3048f;
    const float tail_db = 20.0f * __log2f(sl * (1.0f / (25000.0f * 0.3048f))) * 0.30102999566f;
    // read_npd: two power rows lerped (npd.rs:189-203).
    const AcRow *rp = rows + p.row_base;
    float sel_v[2], scaled[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const AcRow &R = rp[q];
        const float lin = R.sel[interval] + frac * (R.sel[interval + 1] - R.sel[interval]);
        sel_v[q] = tail ? R.sel[9] - tail_db - R.tail_alpha * (sl - 25000.0f * 0.3048f) : lin;
        const float sml = R.sml[interval] + frac * (R.sml[interval + 1] - R.sml[interval]);
        scaled[q] = R.dipole ? sl : R.d0 * __expf(sml * 0.23025850930f);
    }
    const float w = p.w;
    const float sel = w != 0.f ? sel_v[0] + w * (sel_v[1] - sel_v[0]) : sel_v[0];
    const float dl = w != 0.f ? scaled[0] + w * (scaled[1] - scaled[0]) : scaled[0];
    float fraction = 1.0f;
    if (!(length < 1.0f || dl < 1.0f)) {
        // (e(a1) - e(a0)) / pi with e(a) = a / (1 + a^2) + atan(a) (corrections.rs:33-42), written
        // without the cancellation of two values near pi/2 far ahead of or behind the segment.
        const float a0 = -(along * length) / dl, a1 = -(along * length - length) / dl, da = length / dl;
        const float p0 = 1.0f + a0 * a0, p1 = 1.0f + a1 * a1;
        const float diff = atan2f(da, 1.0f + a0 * a1) + da * (1.0f - a0 * a1) / (p0 * p1);
        fraction = fmaxf(diff * 0.31830988618f, 1e-15f);
    }
    const float beta = atanf(lambda_height / fmaxf(lateral, 0.01f)) * 57.295779513f;
    float lat = 0.0f;
    if (!(beta > 50.0f)) {
        const float gamma = lateral <= 914.0f ? 1.089f * (1.0f - __expf(-0.00274f * lateral)) : 1.0f;
        const float lam = beta < 0.0f ? 10.857f : 1.137f - 0.0229f * beta + 9.72f * __expf(-0.142f * beta);
        lat = gamma * lam;
    }
    float inst = 1.0f;
    if (T.installation < 2) {
        const float a = T.installation == 0 ? 0.0039f : 0.1225f, b = T.installation == 0 ? 0.062f : 0.329f,
                    c = T.installation == 0 ? 0.8786f : 1.0f;
        const float h = fmaxf(height, 0.0f);
        const float s2_ = h * h / fmaxf(slant * slant, 1e-12f);
        const float c2_ = 1.0f - s2_;
        const float num = a * c2_ + s2_, den = c * 4.0f * s2_ * c2_ + (c2_ - s2_) * (c2_ - s2_);
        if (den > 0.0f && num > 0.0f) inst = __expf(b * __logf(num)) / den;
    }
    return exp2f((sel - lat) * 0.33219280948873623f) * p.gain * inst * fraction;
}

// One CTA: 16 x 16 cells; segments in TMA tiles; per (thread, type) compensated sums in smem.
__global__ void __launch_bounds__(AC_THREADS) flight_grid_kernel(FlightGridArgs A) {
    extern __shared__ __align__(128) unsigned char smem[];
    qm_flight_segment *tiles = reinterpret_cast<qm_flight_segment *>(smem);  // [2][AC_TILE]
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + 2 * AC_TILE * sizeof(qm_flight_segment));
    AcRow *rows = reinterpret_cast<AcRow *>(smem + 2 * AC_TILE * sizeof(qm_flight_segment) + 16);
    AcType *types = reinterpret_cast<AcType *>(rows + A.n_types * 20);
    float *acc = reinterpret_cast<float *>(types + A.n_types);  // [n_types][2][AC_THREADS]
    SegPre *pre = reinterpret_cast<SegPre *>(acc + A.n_types * 2 * AC_THREADS);  // [AC_TILE]
    const int tid = threadIdx.x;
    for (uint32_t i = tid; i < A.n_types * 20; i += AC_THREADS) rows[i] = A.rows[i];
    for (uint32_t i = tid; i < A.n_types; i += AC_THREADS) types[i] = A.types[i];
    for (uint32_t i = tid; i < A.n_types * 2 * AC_THREADS; i += AC_THREADS) acc[i] = 0.0f;
    const int bx = blockIdx.x % ((A.nx + 15) / 16), by = blockIdx.x / ((A.nx + 15) / 16);
    const int ix = bx * 16 + (tid & 15), iy = by * 16 + (tid >> 4);
    const bool active = ix < A.nx && iy < A.ny;
    const double rxd = A.ox + ix * A.spacing, ryd = A.oy + iy * A.spacing;
    const float rx = (float)rxd, ry = (float)ryd, rz = A.height;
    const uint32_t n_tiles = (A.n_segs + AC_TILE - 1) / AC_TILE;
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    auto issue = [&](uint32_t t) {
        uint32_t first = t * AC_TILE;
        uint32_t count = min((uint32_t)AC_TILE, A.n_segs - first);
        bulk_load(tiles + (t & 1) * AC_TILE, A.segs + first, count * (unsigned)sizeof(qm_flight_segment), &bars[t & 1]);
    };
    if (tid == 0) {
        if (n_tiles > 0) issue(0);
        if (n_tiles > 1) issue(1);
    }
    bool ok = true;
    uint32_t stopped = n_tiles;
    unsigned long long evaluated = 0;
    uint32_t cached_flight = 0xffffffffu;
    bool cached_near = true;
    for (uint32_t t = 0; t < n_tiles; ++t) {
        if (!mbar_wait(&bars[t & 1], (t >> 1) & 1)) {
            ok = false;
            atomicOr(A.error, 1u);
        }
        ok = __syncthreads_and(ok);
        if (!ok) {
            stopped = t;
            break;
        }
        const qm_flight_segment *tile = tiles + (t & 1) * AC_TILE;
        uint32_t count = min((uint32_t)AC_TILE, A.n_segs - t * AC_TILE);
        if (tid < count) pre[tid] = prepare_segment(tile[tid], types);
        __syncthreads();
        if (active) {
            for (uint32_t i = 0; i < count; ++i) {
                const SegPre &g = pre[i];
                if (A.reach2 > 0.0) {
                    // Whole flights are culled by their horizontal box (segments come grouped by flight).
                    if (g.flight != cached_flight) {
                        float4 box = __ldg(A.boxes + g.flight);
                        double dx = fmax(fmax((double)box.x - rxd, 0.0), rxd - (double)box.z);
                        double dy = fmax(fmax((double)box.y - ryd, 0.0), ryd - (double)box.w);
                        cached_flight = g.flight;
                        cached_near = dx * dx + dy * dy <= A.reach2;
                    }
                    if (!cached_near) continue;
                }
                ++evaluated;
                const float e = segment_energy(g, rows, types[g.type], rx, ry, rz);
                // Kahan sum of this thread's type energy.
                float *s = acc + (g.type * 2) * AC_THREADS + tid;
                float *c = s + AC_THREADS;
                float y = __fsub_rn(e, *c);
                float tt = __fadd_rn(*s, y);
                *c = __fsub_rn(__fsub_rn(tt, *s), y);
                *s = tt;
            }
        }
        __syncthreads();  // the buffer is free again
        if (tid == 0 && t + 2 < n_tiles) issue(t + 2);
    }
    // Pairs evaluated (not culled): a warp sum, then one atomic a warp.
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) evaluated += __shfl_down_sync(0xffffffffu, evaluated, o);
    if ((tid & 31) == 0 && A.pairs) atomicAdd(A.pairs, evaluated);
    if (!ok) {
        // A copy may still be in flight: wait for both barriers once more, bounded, then leave.
        if (tid == 0)
            for (uint32_t t = stopped; t < n_tiles && t < stopped + 2; ++t) mbar_wait(&bars[t & 1], (t >> 1) & 1);
        __syncthreads();
        return;
    }
    if (!active) return;
    const int cell = iy * A.nx + ix;
    float total = 0.0f;
    for (uint32_t t = 0; t < A.n_types; ++t) total += acc[(t * 2) * AC_THREADS + tid] - acc[(t * 2 + 1) * AC_THREADS + tid];
    if (A.lae) A.lae[cell] = 10.0f * log10f(total);
    if (A.thirds) {
        for (int b = 0; b < 28; ++b) {
            float e = 0.0f;
            for (uint32_t t = 0; t < A.n_types; ++t)
                e += (acc[(t * 2) * AC_THREADS + tid] - acc[(t * 2 + 1) * AC_THREADS + tid]) * types[t].share[b];
            A.thirds[(size_t)cell * 28 + b] = 10.0f * log10f(e * A.inv_duration);
        }
    }
}

}  // namespace qm
