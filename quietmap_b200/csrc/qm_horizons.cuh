// Receivers' horizons for aircraft screening on the device (popup/src/aircraft/horizons.rs:145-198
// Horizons::build, laid out as write_f32 lays them out, horizons.rs:50-64 and 196-201). One CTA a
// point: 32 threads sample the terrain of a sector each (48 samples from 30 m to 8 km growing
// geometrically), 256 threads walk a 512 m ray each through the scene's obstacle cells (the f64
// crossing walk, qm_offlattice.cuh) and keep per range band the steepest roof edge; the steepest
// tangents of all come from a block reduction.
#pragma once

#include "../../include/qm_flights.h"
#include "qm_offlattice.cuh"

namespace qm {
namespace hz {

constexpr int BANDS = QM_HORIZON_BANDS;
constexpr int TSECT = QM_TERRAIN_SECTORS, BSECT = QM_BUILDING_SECTORS;
constexpr int SAMPLES = 48;
constexpr int THREADS = BSECT;
constexpr int PER_SECTOR = 1 + 2 * BANDS;
constexpr int MAX_CROSSINGS = 256;  // a 512 m ray's crossings; more fails the point

struct Args {
    const double *xy;          // [n][2] lattice steps
    const double *altitude_m;  // [n]
    const uint32_t *own;       // [n] dense footprint ids (0 none)
    uint32_t n;
    double growth;             // (8 km / 30 m)^(1/47), taken on the host as the cores take it
    float *out;                // [n][QM_HORIZON_FLOATS]
    unsigned *failed;          // [n] a ray's crossings exceeded MAX_CROSSINGS
};

__device__ __forceinline__ int band_of(double range, const double *limits) {
    for (int k = 0; k < BANDS; ++k)
        if (range <= limits[k] + 0.5) return k;
    return BANDS - 1;
}

// The steepest edge per band of one sector, then written as its 1 + 2 x BANDS floats.
struct SectorBands {
    double range[BANDS], tangent[BANDS];
    bool set[BANDS];
    double steepest;
    __device__ void clear() {
        for (int k = 0; k < BANDS; ++k) set[k] = false;
        steepest = -CUDART_INF;
    }
    // SectorEdges::offer (horizons.rs:73-80)
    __device__ void offer(int band, double r, double t) {
        if (!set[band] || t > tangent[band]) {
            set[band] = true;
            range[band] = r;
            tangent[band] = t;
        }
        steepest = fmax(steepest, t);
    }
    __device__ void write(float *e) const {
        e[0] = (float)steepest;
        for (int k = 0; k < BANDS; ++k) {
            e[1 + 2 * k] = set[k] ? (float)range[k] : CUDART_NAN_F;
            e[2 + 2 * k] = set[k] ? (float)tangent[k] : CUDART_NAN_F;
        }
    }
};

__global__ void __launch_bounds__(THREADS) flight_horizons_kernel(SceneDev S, Args A) {
    __shared__ double s_max[2][THREADS / 32];
    const uint32_t i = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const double px = A.xy[2 * i], py = A.xy[2 * i + 1], alt = A.altitude_m[i];
    float *out = A.out + (size_t)i * QM_HORIZON_FLOATS;
    const double tau = 6.283185307179586;
    const double m = (double)S.step_m;
    double t_all = -CUDART_INF, b_all = -CUDART_INF;
    SectorBands sb;
    // Terrain (horizons.rs:154-173): a sample outside the DEM is no terrain.
    if (tid < TSECT) {
        const double terrain_limits[BANDS] = {500.0, 1000.0, 2000.0, 3500.0, 5500.0, 8000.0};
        sb.clear();
        double dy, dx;
        sincos(((double)tid + 0.5) * tau / (double)TSECT, &dy, &dx);
        const bool dem = S.dem_nx != 0;
        const double x1 = dem ? (double)S.dem_ox + (double)(S.dem_nx - 1) * (double)S.dem_sp : 0.0;
        const double y1 = dem ? (double)S.dem_oy + (double)(S.dem_ny - 1) * (double)S.dem_sp : 0.0;
        double range = 30.0;
        for (int j = 0; j < SAMPLES; ++j) {
            const double qx = px + dx * range / m, qy = py + dy * range / m;
            if (!dem || (qx >= (double)S.dem_ox && qx <= x1 && qy >= (double)S.dem_oy && qy <= y1)) {
                double z, g;
                terrain_at_d(S, qx, qy, z, g);
                sb.offer(band_of(range, terrain_limits), range, (z - alt) / range);
            }
            range *= A.growth;
        }
        sb.write(out + 1 + tid * PER_SECTOR);
        t_all = sb.steepest;
    }
    // Buildings (horizons.rs:174-196): every building crossing of the sector's 512 m ray but the
    // point's own footprint's walls (finish_crossings drops them) and those within 1 cm.
    {
        const double building_limits[BANDS] = {16.0, 32.0, 64.0, 128.0, 256.0, 512.0};
        const double reach = 512.0;
        sb.clear();
        double dy, dx;
        sincos(((double)tid + 0.5) * tau / (double)BSECT, &dy, &dx);
        XRec xs[MAX_CROSSINGS];
        uint32_t status = 0, tested = 0;
        const int nx = list_crossings_d<MAX_CROSSINGS>(S, px, py, px + dx * reach / m, py + dy * reach / m, A.own[i],
                                                       xs, status, tested);
        if (status) atomicOr(A.failed + i, 1u);
        for (int k = 0; k < nx; ++k) {
            if (!(xs[k].info & X_BUILDING)) continue;
            const double range = xs[k].t * reach;
            if (range <= 0.01) continue;
            double z, g;
            terrain_at_d(S, px + dx * range / m, py + dy * range / m, z, g);
            sb.offer(band_of(range, building_limits), range, (z + (double)xs[k].height - alt) / range);
        }
        sb.write(out + QM_TERRAIN_HORIZON_FLOATS + 1 + tid * PER_SECTOR);
        b_all = sb.steepest;
    }
    // The steepest tangent of all, per horizon.
    for (int o = 16; o > 0; o >>= 1) {
        t_all = fmax(t_all, __shfl_xor_sync(0xffffffffu, t_all, o));
        b_all = fmax(b_all, __shfl_xor_sync(0xffffffffu, b_all, o));
    }
    if (lane == 0) {
        s_max[0][warp] = t_all;
        s_max[1][warp] = b_all;
    }
    __syncthreads();
    if (tid == 0) {
        double t = -CUDART_INF, b = -CUDART_INF;
        for (int w = 0; w < THREADS / 32; ++w) {
            t = fmax(t, s_max[0][w]);
            b = fmax(b, s_max[1][w]);
        }
        out[0] = (float)t;
        out[QM_TERRAIN_HORIZON_FLOATS] = (float)b;
    }
}

}  // namespace hz
}  // namespace qm
