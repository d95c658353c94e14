// The surrogate's front end on the device: the features of a path over flat ground (its exact
// crossing list, then the vertical path's roofs as the exact path builds them), the training
// samples (features with the exact path's A_boundary as the label), and the painter's first pass
// (eligible paths become feature rows for the network; the others run the exact path).
#pragma once

#include <cuda_bf16.h>

#include "qm_kernels.cuh"

namespace qm {

constexpr int SURR_F = 32, SURR_ROOFS = 8;

// Where the training-sample kernels write: rows of raw features, labels and eligibility.
struct SampleArgs {
    GridArgs g;
    float *features;  // [cells * n_src][32]
    float *labels;    // [cells * n_src][8]
    uint8_t *eligible;
};

// Features of one path (the layout is the one in include/qm_surrogate.h) and whether its
// geometry is eligible: every obstacle top pairs into a roof and at most 8 roofs are crossed.
// The tops, roof pairing and clipping follow evaluate_path (physics/src/ray.rs:293-323,
// 389-404) on flat ground, where every top stands on the one ground altitude.
template <int CAP_C>
__device__ __noinline__ bool surrogate_front(const SceneDev &S, const SourceDev &src, int rx, int ry, float rcv_alt,
                                             uint32_t rcv_own, XRec *xs, float f[SURR_F], uint32_t &status,
                                             uint32_t &edges_tested, uint32_t &n_crossings) {
    status = 0;
    edges_tested = 0;
    const int sx = src.x, sy = src.y;
    const float dxm = (float)(rx - sx) * S.step_m, dym = (float)(ry - sy) * S.step_m;
    const float dist = sqrtf(dxm * dxm + dym * dym);
    const float L = fmaxf(dist, 1.0f);
    const int nx = list_crossings<CAP_C>(S, sx, sy, rx, ry, rcv_own, xs, status, edges_tested);
    n_crossings = nx;
    const float2 zs = terrain_point(S, sx, sy), zr = terrain_point(S, rx, ry);
    BuildingHit hits[2 * SURR_ROOFS];
    int nb = 0, nt = 0;
    bool over = false;
    const uint32_t own = src.fp;
    for (int i = 0; i < nx; ++i) {
        const OutlineDev &o = S.outlines[xs[i].info & X_OUTLINE];
        const uint32_t fp = o.fp;
        const bool bounds = (xs[i].info & X_BOUNDS) != 0;
        if (own != 0) {
            bool contained = fp == own;
            if (!contained) {
                int count = 0;
                for (int k = 0; k < nx; ++k)
                    if ((xs[k].info & X_BOUNDS) && xrec_fp(S, xs[k]) == fp) ++count;
                contained = (count & 1) != 0;
            }
            if (contained) continue;
        }
        ++nt;
        if (!bounds) continue;
        if (nb == 2 * SURR_ROOFS) {
            over = true;
            continue;
        }
        hits[nb++] = BuildingHit{fp, (float)xs[i].t * L, zs.x + o.height, zs.x, zs.y};
    }
    Roof roofs[SURR_ROOFS];
    int nr = 0, paired = 0;
    for (int k = 0; k < nb; ++k) {
        const uint32_t fp = hits[k].fp;
        if (fp == 0u) continue;
        for (int j = k + 1; j < nb; ++j)
            if (hits[j].fp == fp) {
                const BuildingHit &a = hits[k], &b = hits[j];
                roofs[nr++] = Roof{a.x, b.x, a.top, b.top, a.zt, b.zt, a.g, b.g, fp};
                hits[j].fp = 0u;
                paired += 2;
                break;
            }
        hits[k].fp = 0u;
    }
    const bool eligible = !over && status == 0 && nt == nb && paired == nb;
    // clip_roofs_in_closing_order: sorted by (x1, x0, footprint), then clipped to what is uncovered.
    for (int i = 1; i < nr; ++i) {
        Roof v = roofs[i];
        int j = i - 1;
        while (j >= 0 && (roofs[j].x1 > v.x1 ||
                          (roofs[j].x1 == v.x1 && (roofs[j].x0 > v.x0 || (roofs[j].x0 == v.x0 && roofs[j].fp > v.fp))))) {
            roofs[j + 1] = roofs[j];
            --j;
        }
        roofs[j + 1] = v;
    }
    int kept = 0;
    {
        float covered_to = -INFINITY;
        for (int i = 0; i < nr; ++i) {
            Roof r = roofs[i];
            if (r.x1 <= covered_to) continue;
            if (r.x0 < covered_to) {
                float span = r.x1 - r.x0;
                r.top0 += (covered_to - r.x0) / span * (r.top1 - r.top0);
                r.x0 = covered_to;
            }
            covered_to = r.x1;
            roofs[kept++] = r;
        }
    }
    f[0] = L * 1e-3f;
    f[1] = src.height * 0.1f;
    f[2] = (rcv_alt - zr.x) * 0.1f;
    f[3] = (zr.x - zs.x) * 0.1f;
    f[4] = 0.0f;
    f[5] = src.gf >= 0.0f ? src.gf : zs.y;
    f[6] = terrain_point(S, (int)(((long long)sx + rx) / 2), (int)(((long long)sy + ry) / 2)).y;
    f[7] = zr.y;
    const float inv_l = 1.0f / L;
#pragma unroll
    for (int k = 0; k < SURR_ROOFS; ++k) {
        bool present = k < kept;
        f[8 + 3 * k] = present ? roofs[k].x0 * inv_l : 0.0f;
        f[9 + 3 * k] = present ? roofs[k].x1 * inv_l : 0.0f;
        f[10 + 3 * k] = present ? ((roofs[k].top0 + roofs[k].top1) - (roofs[k].zt0 + roofs[k].zt1)) * 0.05f : 0.0f;
    }
    return eligible;
}

constexpr int SURR_STRETCHES = 12, SURR_SAMPLES = 36;
// Stretch ends along the path, finer near the source and the receiver (where obstacles and the
// ground shape decide diffraction most).
__device__ __forceinline__ float surr_stretch_end(int j) {
    constexpr float E[SURR_STRETCHES + 1] = {0.0f, 0.02f, 0.05f, 0.1f, 0.2f, 0.35f, 0.5f,
                                             0.65f, 0.8f, 0.9f, 0.95f, 0.98f, 1.0f};
    return E[j];
}

// The terrain feature set (include/qm_surrogate.h) of one path, f4 left 0 for the caller to set;
// eligible when its crossing list fits. Positions along the path are rounded to the lattice
// (x = sx + rint(t * dx)) and the ground there is the DEM's bilinear value.
template <int CAP_C>
__device__ __noinline__ bool surrogate_front_terrain(const SceneDev &S, const SourceDev &src, int rx, int ry,
                                                     float rcv_alt, uint32_t rcv_own, XRec *xs, float f[SURR_F],
                                                     uint32_t &status, uint32_t &edges_tested, uint32_t &n_crossings) {
    status = 0;
    edges_tested = 0;
    const int sx = src.x, sy = src.y;
    const int dx = rx - sx, dy = ry - sy;
    const float dxm = (float)dx * S.step_m, dym = (float)dy * S.step_m;
    const float L = fmaxf(sqrtf(dxm * dxm + dym * dym), 1.0f);
    const int nx = list_crossings<CAP_C>(S, sx, sy, rx, ry, rcv_own, xs, status, edges_tested);
    n_crossings = nx;
    const float2 zs = terrain_point(S, sx, sy), zr = terrain_point(S, rx, ry);
    const float src_alt = zs.x + src.height;
    const float rise = (rcv_alt - src_alt) / L;  // the straight line's slope
    auto ground_at = [&](double t) {
        int px = sx + (int)rint(t * (double)dx), py = sy + (int)rint(t * (double)dy);
        return terrain_point(S, px, py);
    };
    // Terrain above the line, stretch by stretch.
    float gsum = 0.0f;
#pragma unroll 1
    for (int j = 0; j < SURR_STRETCHES; ++j) {
        float top = -INFINITY;
        const float e0 = surr_stretch_end(j), e1 = surr_stretch_end(j + 1);
        for (int q = 0; q < SURR_SAMPLES / SURR_STRETCHES; ++q) {
            const double t = (double)e0 + (q + 0.5) / (SURR_SAMPLES / SURR_STRETCHES) * (double)(e1 - e0);
            const float2 zg = ground_at(t);
            top = fmaxf(top, zg.x - (src_alt + rise * (float)t * L));
            gsum += zg.y;
        }
        f[8 + j] = top * 0.1f;
    }
    // Obstacle tops (every wall the path crosses, standing on the ground at its crossing point):
    // their largest rise above the line, stretch by stretch (-10, i.e. 100 m below, where none).
#pragma unroll
    for (int j = 0; j < SURR_STRETCHES; ++j) f[20 + j] = -10.0f;
    const uint32_t own = src.fp;
    for (int i = 0; i < nx; ++i) {
        const OutlineDev &o = S.outlines[xs[i].info & X_OUTLINE];
        const uint32_t fp = o.fp;
        if (own != 0) {
            bool contained = fp == own;
            if (!contained) {
                int count = 0;
                for (int k = 0; k < nx; ++k)
                    if ((xs[k].info & X_BOUNDS) && xrec_fp(S, xs[k]) == fp) ++count;
                contained = (count & 1) != 0;
            }
            if (contained) continue;
        }
        const double t = xs[i].t;
        const float top = ground_at(t).x + o.height;
        int j = 0;
        while (j < SURR_STRETCHES - 1 && t >= (double)surr_stretch_end(j + 1)) ++j;
        f[20 + j] = fmaxf(f[20 + j], (top - (src_alt + rise * (float)t * L)) * 0.1f);
    }
    const bool eligible = status == 0;
    f[0] = L * 1e-3f;
    f[1] = src.height * 0.1f;
    f[2] = (rcv_alt - zr.x) * 0.1f;
    f[3] = (zr.x - zs.x) * 0.1f;
    f[4] = 0.0f;
    f[5] = src.gf >= 0.0f ? src.gf : zs.y;
    f[6] = gsum * (1.0f / SURR_SAMPLES);
    f[7] = zr.y;
    return eligible;
}

// Terrain training samples: two rows per path (homogeneous, favourable) with the exact path's
// A_boundary of each state as the label.
__global__ void __launch_bounds__(128, QM_PAINT_MIN_BLOCKS) surrogate_samples_terrain_kernel(SceneDev S, SampleArgs P) {
    const GridArgs &A = P.g;
    const int tiles_x = (A.nx + A.tile_w - 1) / A.tile_w;
    const int tx = blockIdx.x % tiles_x, ty = blockIdx.x / tiles_x;
    const int2 slot = tile_slot(A.tile_w, A.tile_h);
    const int ix = tx * A.tile_w + slot.x, iy = ty * A.tile_h + slot.y;
    if (ix >= A.nx || iy >= A.ny) return;
    const int cell = iy * A.nx + ix;
    const int rx = A.origin_x + ix * A.spacing, ry = A.origin_y + iy * A.spacing;
    const float alt = A.rcv_alt[cell];
    const uint32_t own = A.rcv_own[cell];
    const uint32_t n_src = A.source_end - A.source_begin;
    PathWork<CapsTerrain::C, CapsTerrain::K, CapsTerrain::H> work;
    const uint32_t s0 = A.source_begin + blockIdx.y * A.chunk, s1 = min(s0 + A.chunk, A.source_end);
    for (uint32_t s = s0; s < s1; ++s) {
        const SourceDev &src = S.sources[s];
        const size_t row = ((size_t)cell * n_src + (s - A.source_begin)) * 2;
        float f[SURR_F];
        uint32_t st, tested, nc;
        bool ok = surrogate_front_terrain<CapsTerrain::C>(S, src, rx, ry, alt, own, work.xs, f, st, tested, nc);
        PathResult r;
        evaluate_path<CapsTerrain::C, CapsTerrain::K, CapsTerrain::H>(S, src, rx, ry, alt, own, true, work, r);
        ok = ok && r.status == 0;
        for (int state = 0; state < 2; ++state) {
            P.eligible[row + state] = ok ? 1 : 0;
            f[4] = (float)state;
#pragma unroll
            for (int k = 0; k < SURR_F; ++k) P.features[(row + state) * SURR_F + k] = f[k];
#pragma unroll
            for (int b = 0; b < QM_BANDS; ++b)
                P.labels[(row + state) * QM_BANDS + b] = r.status ? 0.0f : -10.0f * log10f(r.boundary[state][b]);
        }
    }
}

// Training samples: thread = receiver of a tile, looping over its chunk of sources; each path's
// raw features, eligibility and exact A_boundary (homogeneous state) per band.

__global__ void __launch_bounds__(128, QM_PAINT_MIN_BLOCKS) surrogate_samples_kernel(SceneDev S, SampleArgs P) {
    const GridArgs &A = P.g;
    const int tiles_x = (A.nx + A.tile_w - 1) / A.tile_w;
    const int tx = blockIdx.x % tiles_x, ty = blockIdx.x / tiles_x;
    const int2 slot = tile_slot(A.tile_w, A.tile_h);
    const int ix = tx * A.tile_w + slot.x, iy = ty * A.tile_h + slot.y;
    if (ix >= A.nx || iy >= A.ny) return;
    const int cell = iy * A.nx + ix;
    const int rx = A.origin_x + ix * A.spacing, ry = A.origin_y + iy * A.spacing;
    const float alt = A.rcv_alt[cell];
    const uint32_t own = A.rcv_own[cell];
    const uint32_t n_src = A.source_end - A.source_begin;
    PathWork<CapsFlat::C, CapsFlat::K, CapsFlat::H> work;
    const uint32_t s0 = A.source_begin + blockIdx.y * A.chunk, s1 = min(s0 + A.chunk, A.source_end);
    for (uint32_t s = s0; s < s1; ++s) {
        const SourceDev &src = S.sources[s];
        const size_t row = (size_t)cell * n_src + (s - A.source_begin);
        float f[SURR_F];
        uint32_t st, tested, nc;
        bool ok = surrogate_front<CapsFlat::C>(S, src, rx, ry, alt, own, work.xs, f, st, tested, nc);
        PathResult r;
        evaluate_path<CapsFlat::C, CapsFlat::K, CapsFlat::H>(S, src, rx, ry, alt, own, false, work, r);
        ok = ok && r.status == 0;
        P.eligible[row] = ok ? 1 : 0;
#pragma unroll
        for (int k = 0; k < SURR_F; ++k) P.features[row * SURR_F + k] = f[k];
#pragma unroll
        for (int b = 0; b < QM_BANDS; ++b)
            P.labels[row * QM_BANDS + b] = r.status ? 0.0f : -10.0f * log10f(r.boundary[0][b]);
    }
}

// The painter's first pass: eligible paths inside the trained feature ranges become normalised
// BF16 rows with their energy coefficients; the others run the exact path here and add their
// energies to the chunk's partial slice.
struct SurrPaintArgs {
    GridArgs g;
    __nv_bfloat16 *x;   // [cells * rows_per_cell][32]
    float *coef;        // [cells * rows_per_cell][16]
    uint8_t *eligible;  // [cells * rows_per_cell]
    uint32_t rows_per_cell;
    float in_shift[SURR_F], in_scale[SURR_F], lo[SURR_F], hi[SURR_F];
};

__global__ void __launch_bounds__(128, QM_PAINT_MIN_BLOCKS) surrogate_front_kernel(SceneDev S, SurrPaintArgs P) {
    __shared__ unsigned long long s_counts[6];
    if (threadIdx.x < 6) s_counts[threadIdx.x] = 0;
    __syncthreads();
    const GridArgs &A = P.g;
    const int tiles_x = (A.nx + A.tile_w - 1) / A.tile_w;
    const int tx = blockIdx.x % tiles_x, ty = blockIdx.x / tiles_x;
    const int2 slot = tile_slot(A.tile_w, A.tile_h);
    const int ix = tx * A.tile_w + slot.x, iy = ty * A.tile_h + slot.y;
    const bool active = ix < A.nx && iy < A.ny;
    const int cell = iy * A.nx + ix;
    unsigned long long paths = 0, crossings = 0, tested = 0, failed_paths = 0, vertices = 0, candidates = 0;
    if (active) {
        const int rx = A.origin_x + ix * A.spacing, ry = A.origin_y + iy * A.spacing;
        const float alt = A.rcv_alt[cell];
        const uint32_t own = A.rcv_own[cell];
        KSum bands[QM_BANDS];
        KSum lden{0.f, 0.f};
#pragma unroll
        for (int b = 0; b < QM_BANDS; ++b) bands[b] = KSum{0.f, 0.f};
        uint32_t failed = 0;
        PathWork<CapsFlat::C, CapsFlat::K, CapsFlat::H> work;
        const uint32_t s0 = A.source_begin + blockIdx.y * A.chunk, s1 = min(s0 + A.chunk, A.source_end);
        for (uint32_t s = s0; s < s1; ++s) {
            const SourceDev &src = S.sources[s];
            ++paths;
            float f[SURR_F];
            uint32_t st, et, nc;
            bool ok = surrogate_front<CapsFlat::C>(S, src, rx, ry, alt, own, work.xs, f, st, et, nc);
#pragma unroll
            for (int k = 0; k < SURR_F; ++k) ok = ok && f[k] >= P.lo[k] && f[k] <= P.hi[k];
            if (ok) {
                crossings += nc;
                tested += et;
                const size_t row = (size_t)cell * P.rows_per_cell + (s - A.source_begin);
                uint4 *xr = reinterpret_cast<uint4 *>(P.x + row * SURR_F);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    uint32_t w[4];
#pragma unroll
                    for (int h = 0; h < 4; ++h) {
                        int k = 8 * q + 2 * h;
                        __nv_bfloat162 v = __floats2bfloat162_rn((f[k] - P.in_shift[k]) * P.in_scale[k],
                                                                 (f[k + 1] - P.in_shift[k + 1]) * P.in_scale[k + 1]);
                        w[h] = *reinterpret_cast<uint32_t *>(&v);
                    }
                    xr[q] = make_uint4(w[0], w[1], w[2], w[3]);
                }
                // Energy coefficients: divergence and air absorption (evaluate_path's tail and
                // path_energies, homogeneous state).
                const float dxm = (float)(rx - src.x) * S.step_m, dym = (float)(ry - src.y) * S.step_m;
                const float dist = sqrtf(dxm * dxm + dym * dym), L = fmaxf(dist, 1.0f);
                const float src_alt = terrain_point(S, src.x, src.y).x + src.height;
                const float dz = alt - src_alt;
                const float slant = fmaxf(sqrtf(L * L + dz * dz), 1.0f);
                const float dh = fmaxf(dist, src.excl);
                const float d = fmaxf(sqrtf(dh * dh + dz * dz), 1.0f);
                const float weight = 1.0f / (d * d * 12.589254117941673f);
                float4 *cr = reinterpret_cast<float4 *>(P.coef + row * 16);
                float c[16];
#pragma unroll
                for (int b = 0; b < QM_BANDS; ++b) {
                    float wa = weight * __expf(-S.air_per_m[b] * slant);
                    float e0 = __ldg(&src.energy[b]);
                    float el = A.lden_w[0] * e0 + A.lden_w[1] * __ldg(&src.energy[QM_BANDS + b]) +
                               A.lden_w[2] * __ldg(&src.energy[2 * QM_BANDS + b]);
                    c[b] = wa * e0;
                    c[8 + b] = wa * el;
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) cr[q] = make_float4(c[4 * q], c[4 * q + 1], c[4 * q + 2], c[4 * q + 3]);
                P.eligible[row] = 1;
                continue;
            }
            PathResult r;
            evaluate_path<CapsFlat::C, CapsFlat::K, CapsFlat::H>(S, src, rx, ry, alt, own, false, work, r);
            crossings += r.crossings;
            tested += r.edges_tested;
            vertices += r.vertices;
            candidates += r.candidates;
            if (r.status) {
                failed |= r.status;
                ++failed_paths;
                unsigned int slot = atomicAdd(A.retry_count, 1u);
                if (slot < A.retry_cap) A.retry[slot] = make_uint2((uint32_t)cell, s);
                continue;
            }
            float day[QM_BANDS], le;
            path_energies(S, r, src, A.lden_w, day, le);
#pragma unroll
            for (int b = 0; b < QM_BANDS; ++b) bands[b].add(day[b]);
            lden.add(le);
        }
        float *out = A.partial + ((size_t)blockIdx.y * (A.nx * A.ny) + cell) * GRID_SLOTS;
#pragma unroll
        for (int b = 0; b < QM_BANDS; ++b) out[b] += bands[b].value();
        out[8] += lden.value();
        if (failed) atomicOr(A.failed + cell, failed);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        paths += __shfl_down_sync(0xffffffffu, paths, o);
        crossings += __shfl_down_sync(0xffffffffu, crossings, o);
        tested += __shfl_down_sync(0xffffffffu, tested, o);
        failed_paths += __shfl_down_sync(0xffffffffu, failed_paths, o);
        vertices += __shfl_down_sync(0xffffffffu, vertices, o);
        candidates += __shfl_down_sync(0xffffffffu, candidates, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&s_counts[0], paths);
        atomicAdd(&s_counts[1], crossings);
        atomicAdd(&s_counts[2], tested);
        atomicAdd(&s_counts[3], failed_paths);
        atomicAdd(&s_counts[4], vertices);
        atomicAdd(&s_counts[5], candidates);
    }
    __syncthreads();
    if (threadIdx.x < 6) atomicAdd(A.counters + threadIdx.x, s_counts[threadIdx.x]);
}

// The painter's first pass on terrain: two rows per eligible path (homogeneous, favourable), each
// with its state's share of the energy coefficients; the others run the exact path here.
__global__ void __launch_bounds__(128, QM_PAINT_MIN_BLOCKS) surrogate_front_terrain_kernel(SceneDev S, SurrPaintArgs P) {
    __shared__ unsigned long long s_counts[6];
    if (threadIdx.x < 6) s_counts[threadIdx.x] = 0;
    __syncthreads();
    const GridArgs &A = P.g;
    const int tiles_x = (A.nx + A.tile_w - 1) / A.tile_w;
    const int tx = blockIdx.x % tiles_x, ty = blockIdx.x / tiles_x;
    const int2 slot = tile_slot(A.tile_w, A.tile_h);
    const int ix = tx * A.tile_w + slot.x, iy = ty * A.tile_h + slot.y;
    const bool active = ix < A.nx && iy < A.ny;
    const int cell = iy * A.nx + ix;
    unsigned long long paths = 0, crossings = 0, tested = 0, failed_paths = 0, vertices = 0, candidates = 0;
    if (active) {
        const int rx = A.origin_x + ix * A.spacing, ry = A.origin_y + iy * A.spacing;
        const float alt = A.rcv_alt[cell];
        const uint32_t own = A.rcv_own[cell];
        KSum bands[QM_BANDS];
        KSum lden{0.f, 0.f};
#pragma unroll
        for (int b = 0; b < QM_BANDS; ++b) bands[b] = KSum{0.f, 0.f};
        uint32_t failed = 0;
        PathWork<CapsTerrain::C, CapsTerrain::K, CapsTerrain::H> work;
        const uint32_t s0 = A.source_begin + blockIdx.y * A.chunk, s1 = min(s0 + A.chunk, A.source_end);
        for (uint32_t s = s0; s < s1; ++s) {
            const SourceDev &src = S.sources[s];
            ++paths;
            float f[SURR_F];
            uint32_t st, et, nc;
            bool ok = surrogate_front_terrain<CapsTerrain::C>(S, src, rx, ry, alt, own, work.xs, f, st, et, nc);
#pragma unroll
            for (int k = 0; k < SURR_F; ++k)
                ok = ok && (k == 4 || (f[k] >= P.lo[k] && f[k] <= P.hi[k]));
            if (ok) {
                crossings += nc;
                tested += et;
                const size_t row = (size_t)cell * P.rows_per_cell + 2 * (size_t)(s - A.source_begin);
                const float dxm = (float)(rx - src.x) * S.step_m, dym = (float)(ry - src.y) * S.step_m;
                const float dist = sqrtf(dxm * dxm + dym * dym), L = fmaxf(dist, 1.0f);
                const float src_alt = terrain_point(S, src.x, src.y).x + src.height;
                const float dz = alt - src_alt;
                const float slant = fmaxf(sqrtf(L * L + dz * dz), 1.0f);
                const float dh = fmaxf(dist, src.excl);
                const float d = fmaxf(sqrtf(dh * dh + dz * dz), 1.0f);
                const float weight = 1.0f / (d * d * 12.589254117941673f);
                const float azimuth = atan2f(dym, dxm);
                float p[QM_PERIODS];
#pragma unroll
                for (int q = 0; q < QM_PERIODS; ++q) p[q] = A.want_fav ? favourable_at(S.fav[q], azimuth) : 0.0f;
                for (int state = 0; state < 2; ++state) {
                    f[4] = (float)state;
                    uint4 *xr = reinterpret_cast<uint4 *>(P.x + (row + state) * SURR_F);
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        uint32_t w[4];
#pragma unroll
                        for (int h = 0; h < 4; ++h) {
                            int k = 8 * q + 2 * h;
                            __nv_bfloat162 v = __floats2bfloat162_rn((f[k] - P.in_shift[k]) * P.in_scale[k],
                                                                     (f[k + 1] - P.in_shift[k + 1]) * P.in_scale[k + 1]);
                            w[h] = *reinterpret_cast<uint32_t *>(&v);
                        }
                        xr[q] = make_uint4(w[0], w[1], w[2], w[3]);
                    }
                    float4 *cr = reinterpret_cast<float4 *>(P.coef + (row + state) * 16);
                    float c[16];
#pragma unroll
                    for (int b = 0; b < QM_BANDS; ++b) {
                        const float wa = weight * __expf(-S.air_per_m[b] * slant);
                        float share[QM_PERIODS];
#pragma unroll
                        for (int q = 0; q < QM_PERIODS; ++q) share[q] = state ? p[q] : 1.0f - p[q];
                        const float e0 = __ldg(&src.energy[b]), e1 = __ldg(&src.energy[QM_BANDS + b]),
                                    e2 = __ldg(&src.energy[2 * QM_BANDS + b]);
                        c[b] = wa * e0 * share[0];
                        c[8 + b] = wa * (A.lden_w[0] * e0 * share[0] + A.lden_w[1] * e1 * share[1] +
                                         A.lden_w[2] * e2 * share[2]);
                    }
#pragma unroll
                    for (int q = 0; q < 4; ++q) cr[q] = make_float4(c[4 * q], c[4 * q + 1], c[4 * q + 2], c[4 * q + 3]);
                    P.eligible[row + state] = 1;
                }
                continue;
            }
            PathResult r;
            evaluate_path<CapsTerrain::C, CapsTerrain::K, CapsTerrain::H>(S, src, rx, ry, alt, own, A.want_fav, work, r);
            crossings += r.crossings;
            tested += r.edges_tested;
            vertices += r.vertices;
            candidates += r.candidates;
            if (r.status) {
                failed |= r.status;
                ++failed_paths;
                unsigned int slot = atomicAdd(A.retry_count, 1u);
                if (slot < A.retry_cap) A.retry[slot] = make_uint2((uint32_t)cell, s);
                continue;
            }
            float day[QM_BANDS], le;
            path_energies(S, r, src, A.lden_w, day, le);
#pragma unroll
            for (int b = 0; b < QM_BANDS; ++b) bands[b].add(day[b]);
            lden.add(le);
        }
        float *out = A.partial + ((size_t)blockIdx.y * (A.nx * A.ny) + cell) * GRID_SLOTS;
#pragma unroll
        for (int b = 0; b < QM_BANDS; ++b) out[b] += bands[b].value();
        out[8] += lden.value();
        if (failed) atomicOr(A.failed + cell, failed);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        paths += __shfl_down_sync(0xffffffffu, paths, o);
        crossings += __shfl_down_sync(0xffffffffu, crossings, o);
        tested += __shfl_down_sync(0xffffffffu, tested, o);
        failed_paths += __shfl_down_sync(0xffffffffu, failed_paths, o);
        vertices += __shfl_down_sync(0xffffffffu, vertices, o);
        candidates += __shfl_down_sync(0xffffffffu, candidates, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&s_counts[0], paths);
        atomicAdd(&s_counts[1], crossings);
        atomicAdd(&s_counts[2], tested);
        atomicAdd(&s_counts[3], failed_paths);
        atomicAdd(&s_counts[4], vertices);
        atomicAdd(&s_counts[5], candidates);
    }
    __syncthreads();
    if (threadIdx.x < 6) atomicAdd(A.counters + threadIdx.x, s_counts[threadIdx.x]);
}

}  // namespace qm
