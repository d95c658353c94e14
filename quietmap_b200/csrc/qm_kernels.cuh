// Kernels of the painter: the fused grid painter (receivers x a chunk of sources, compensated
// per-cell sums), its per-cell reduction with levels and the level histogram, and the pair
// evaluator behind Batch::evaluate / Batch::pair_spectra.
#pragma once

#include "qm_path.cuh"

namespace qm {

// Kahan-compensated FP32 sum: the energetic sums of 10^(L/10) keep their low bits.
struct KSum {
    float s, c;
    __device__ __forceinline__ void add(float v) {
        float y = __fsub_rn(v, c);
        float t = __fadd_rn(s, y);
        c = __fsub_rn(__fsub_rn(t, s), y);
        s = t;
    }
    __device__ __forceinline__ float value() const { return __fsub_rn(s, c); }
};

// Path capacities per workload kind: crossings, crests, hull points per state.
struct CapsFlat {
    static constexpr int C = 96, K = 2, H = 24;
};
struct CapsTerrain {
    static constexpr int C = 256, K = 512, H = 64;
};
struct CapsLarge {
    static constexpr int C = 1024, K = 4096, H = 256;
};

// Per-cell output slots of the grid painter: 8 day band energies and the Lden-weighted A energy.
constexpr int GRID_SLOTS = 9;

struct GridArgs {
    int origin_x, origin_y, spacing, nx, ny;
    float height_m;
    uint32_t source_begin, source_end;
    uint32_t chunk;          // sources per chunk
    uint32_t n_chunks;
    const float *rcv_alt;    // [cells] receiver altitude (ground + height)
    const uint32_t *rcv_own; // [cells] dense own footprint
    float *partial;          // [n_chunks][cells][GRID_SLOTS]
    uint32_t *failed;        // [cells] bitwise-or of path failures
    unsigned long long *counters;  // paths, crossings, edge tests, failed paths, vertices, candidates
    uint2 *retry;            // failed (cell, source) paths, re-run with large capacities
    uint32_t retry_cap;
    unsigned int *retry_count;
    float lden_w[QM_PERIODS];
    bool want_fav;
    int tile_w, tile_h;      // receiver tile per CTA
};

// The 9 energies one path adds to its cell: day bands (transfer of period 0) and the Lden-weighted
// A energy over the periods (popup/src/evaluate.rs:135-142; physics/src/bands.rs:59-66).
__device__ __forceinline__ void path_energies(const SceneDev &S, const PathResult &r, const SourceDev &src,
                                              const float lden_w[QM_PERIODS], float day[QM_BANDS], float &lden) {
    float air[QM_BANDS];
#pragma unroll
    for (int b = 0; b < QM_BANDS; ++b) air[b] = __expf(-S.air_per_m[b] * r.slant);
    float lsum = 0.f;
#pragma unroll
    for (int p = 0; p < QM_PERIODS; ++p) {
        float pp = r.p[p];
        float psum = 0.f;
#pragma unroll
        for (int b = 0; b < QM_BANDS; ++b) {
            float t = air[b] * (pp * r.boundary[1][b] + (1.0f - pp) * r.boundary[0][b]);
            float e = r.weight * __ldg(&src.energy[p * QM_BANDS + b]) * t;
            if (p == 0) day[b] = e;
            psum += e;
        }
        lsum += lden_w[p] * psum;
    }
    lden = lsum;
}

// Receiver r (0 <= r < block_w * block_h) of a block of receivers: each 32 consecutive r (a warp)
// cover an 8 x 4 patch when the block's sides are multiples of 8 and 4, else the block is
// row-major. A warp's rays to a source then lie closer together than along a row of 16 or 32, so
// their crossing walks and profiles diverge less (a terrain tile, 16 x 8 receivers x 80,000
// sources: 699 ms against 742 ms with two rows of 16 a warp, cell results bit for bit the same;
// 4 x 8 patches measured the same as 8 x 4).
__device__ __forceinline__ int2 block_slot(uint32_t r, uint32_t block_w, uint32_t block_h) {
    if (block_w % 8 == 0 && block_h % 4 == 0) {
        const uint32_t g = r >> 5, l = r & 31, groups_x = block_w / 8;
        return make_int2((int)((g % groups_x) * 8 + (l & 7)), (int)((g / groups_x) * 4 + (l >> 3)));
    }
    return make_int2((int)(r % block_w), (int)(r / block_w));
}

// A thread's receiver inside its CTA's tile (one thread per receiver).
__device__ __forceinline__ int2 tile_slot(int tile_w, int tile_h) {
    return block_slot(threadIdx.x, (uint32_t)tile_w, (uint32_t)tile_h);
}

#ifndef QM_PAINT_MIN_BLOCKS
// CTAs of 128 resident per SM: 3 caps registers at 170 a thread. Measured on a terrain tile
// (16 x 8 receivers x 80,000 sources): 2 CTAs 847 ms, 3 CTAs 741 ms, 4 CTAs 786 ms, 5 CTAs 814 ms,
// 6 CTAs 880 ms; the road square is within 2 % for 3 and 4.
#define QM_PAINT_MIN_BLOCKS 3
#endif

// Thread = one receiver of a tile; CTA = (receiver tile, source chunk). Each thread walks its chunk
// of sources and keeps its cell's band energies in compensated registers; one store per cell. On
// terrain the warp lists the crossings of its 32 rays to each source together (warp_list_crossings:
// the obstacle entries staged in shared memory by bulk copies); on flat scenes each lane lists its
// own ray's. Each lane then follows its own path.
template <class Caps>
__global__ void __launch_bounds__(128, QM_PAINT_MIN_BLOCKS) paint_grid_kernel(SceneDev S, GridArgs A) {
    __shared__ unsigned long long s_counts[6];
    __shared__ CrossStage s_stage[4];
    if (threadIdx.x < 6) s_counts[threadIdx.x] = 0;
    CrossStage &stage = s_stage[threadIdx.x >> 5];
    stage_init(stage);
    __syncthreads();
    const int tiles_x = (A.nx + A.tile_w - 1) / A.tile_w;
    const int tile = blockIdx.x;
    const int chunk = blockIdx.y;
    const int tx = tile % tiles_x, ty = tile / tiles_x;
    const int2 slot = tile_slot(A.tile_w, A.tile_h);
    const int ix = tx * A.tile_w + slot.x;
    const int iy = ty * A.tile_h + slot.y;
    const bool active = ix < A.nx && iy < A.ny;
    const int cell = iy * A.nx + ix;
    KSum bands[QM_BANDS];
    KSum lden{0.f, 0.f};
#pragma unroll
    for (int b = 0; b < QM_BANDS; ++b) bands[b] = KSum{0.f, 0.f};
    uint32_t failed = 0;
    unsigned long long paths = 0, crossings = 0, tested = 0, failed_paths = 0, vertices = 0, candidates = 0;
    const int rx = A.origin_x + ix * A.spacing, ry = A.origin_y + iy * A.spacing;
    const float alt = active ? A.rcv_alt[cell] : 0.0f;
    const uint32_t own = active ? A.rcv_own[cell] : 0u;
    PathWork<Caps::C, Caps::K, Caps::H> work;
    StageState ss{0u, false};
    const uint32_t s0 = A.source_begin + chunk * A.chunk;
    const uint32_t s1 = min(s0 + A.chunk, A.source_end);
    for (uint32_t s = s0; s < s1; ++s) {
        const SourceDev &src = S.sources[s];
        PathResult r;
        r.status = 0;
        r.edges_tested = 0;
        // Flat scenes' short rays cross few cells: each lane walks its own (the warp's shared sweep
        // pays off on the long terrain rays).
        int nx;
        if constexpr (Caps::C == CapsFlat::C) {
            if (!active) continue;
            nx = list_crossings<Caps::C>(S, src.x, src.y, rx, ry, own, work.xs, r.status, r.edges_tested);
        } else {
            nx = warp_list_crossings<Caps::C>(S, stage, ss, src.x, src.y, rx, ry, active, own, work.xs, r.status,
                                              r.edges_tested);
            if (!active) continue;
        }
        if (r.status == 0) {
            evaluate_listed<Caps::C, Caps::K, Caps::H>(S, src, rx, ry, alt, A.want_fav, work, nx, r, (double)src.x,
                                                       (double)src.y);
        } else {
            r.crossings = nx;
            r.vertices = 0;
            r.candidates = 0;
        }
        ++paths;
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
    if (active) {
        float *out = A.partial + ((size_t)chunk * (A.nx * A.ny) + cell) * GRID_SLOTS;
#pragma unroll
        for (int b = 0; b < QM_BANDS; ++b) out[b] = bands[b].value();
        out[8] = lden.value();
        if (failed) atomicOr(A.failed + cell, failed);
    }
    // Counters: warp sums, then one atomic per CTA.
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

// Failed paths again, with large per-path capacities held in global scratch (one work area per
// thread, grid-stride over the sorted list): each path's 9 energies into `out`.
__global__ void __launch_bounds__(64) retry_paths_kernel(SceneDev S, GridArgs A, const uint2 *pairs, uint32_t n,
                                                         PathWork<CapsLarge::C, CapsLarge::K, CapsLarge::H> *works,
                                                         float *out, uint32_t *status) {
    uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t stride = gridDim.x * blockDim.x;
    PathWork<CapsLarge::C, CapsLarge::K, CapsLarge::H> &work = works[tid];
    for (uint32_t i = tid; i < n; i += stride) {
        uint2 pr = pairs[i];
        int cell = (int)pr.x;
        int ix = cell % A.nx, iy = cell / A.nx;
        const SourceDev &src = S.sources[pr.y];
        PathResult r;
        evaluate_path<CapsLarge::C, CapsLarge::K, CapsLarge::H>(S, src, A.origin_x + ix * A.spacing,
                                                                A.origin_y + iy * A.spacing, A.rcv_alt[cell],
                                                                A.rcv_own[cell], A.want_fav, work, r);
        status[i] = r.status;
        float day[QM_BANDS], le = 0.f;
        if (r.status == 0) path_energies(S, r, src, A.lden_w, day, le);
#pragma unroll
        for (int b = 0; b < QM_BANDS; ++b) out[(size_t)i * GRID_SLOTS + b] = r.status ? 0.f : day[b];
        out[(size_t)i * GRID_SLOTS + 8] = le;
    }
}

// The re-run paths of each failing cell, summed in (cell, source) order into the partial slice
// `slice` (deterministic).
__global__ void fold_retry_kernel(const uint32_t *cell_ids, const uint32_t *cell_start, uint32_t n_cells,
                                  const float *results, float *partial, uint32_t slice, int cells) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_cells) return;
    KSum acc[GRID_SLOTS];
#pragma unroll
    for (int j = 0; j < GRID_SLOTS; ++j) acc[j] = KSum{0.f, 0.f};
    for (uint32_t i = cell_start[k]; i < cell_start[k + 1]; ++i)
#pragma unroll
        for (int j = 0; j < GRID_SLOTS; ++j) acc[j].add(results[(size_t)i * GRID_SLOTS + j]);
    float *dst = partial + ((size_t)slice * cells + cell_ids[k]) * GRID_SLOTS;
#pragma unroll
    for (int j = 0; j < GRID_SLOTS; ++j) dst[j] = acc[j].value();
}

// The bin of a level (popup/src/distribution.rs:69-72): round((L - L_min) / bin) with Rust's
// saturating cast (negative and NaN to 0), clamped to the last bin; taken in double from the FP32
// level so the count is exact given the level.
__device__ __forceinline__ uint32_t level_bin(float level, double level_min, double bin_db, uint32_t n_bins) {
    double r = round(((double)level - level_min) / bin_db);
    if (!(r > 0.0)) return 0;
    if (r >= (double)(n_bins - 1)) return n_bins - 1;
    return (uint32_t)r;
}

struct ReduceArgs {
    int cells;
    uint32_t n_chunks;
    const float *partial;
    float *cell_bands;  // [cells][8] dB (nullable)
    float *cell_dba;    // [cells] (nullable)
    float *cell_lden;   // [cells] (nullable)
    float *dba_scratch; // [cells] always written (histogram input)
    uint32_t *histogram;
    double level_min, bin_db;
    uint32_t n_bins;
};

// Per cell: the chunks' partial energies summed in chunk order (compensated, deterministic), the
// band levels, dBA and Lden, and the cell's dBA counted into a block histogram in shared memory.
__global__ void __launch_bounds__(256) reduce_cells_kernel(ReduceArgs A) {
    extern __shared__ uint32_t s_hist[];
    for (uint32_t k = threadIdx.x; k < A.n_bins; k += blockDim.x) s_hist[k] = 0;
    __syncthreads();
    int cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell < A.cells) {
        KSum acc[GRID_SLOTS];
#pragma unroll
        for (int k = 0; k < GRID_SLOTS; ++k) acc[k] = KSum{0.f, 0.f};
        for (uint32_t c = 0; c < A.n_chunks; ++c) {
            const float *p = A.partial + ((size_t)c * A.cells + cell) * GRID_SLOTS;
#pragma unroll
            for (int k = 0; k < GRID_SLOTS; ++k) acc[k].add(p[k]);
        }
        KSum total{0.f, 0.f};
#pragma unroll
        for (int b = 0; b < QM_BANDS; ++b) {
            float e = acc[b].value();
            total.add(e);
            if (A.cell_bands) A.cell_bands[(size_t)cell * QM_BANDS + b] = 10.0f * log10f(e);
        }
        float dba = 10.0f * log10f(total.value());
        float lden = 10.0f * log10f(acc[8].value());
        if (A.cell_dba) A.cell_dba[cell] = dba;
        if (A.cell_lden) A.cell_lden[cell] = lden;
        A.dba_scratch[cell] = dba;
        if (A.histogram) atomicAdd(&s_hist[level_bin(dba, A.level_min, A.bin_db, A.n_bins)], 1u);
    }
    __syncthreads();
    if (A.histogram)
        for (uint32_t k = threadIdx.x; k < A.n_bins; k += blockDim.x)
            if (s_hist[k]) atomicAdd(A.histogram + k, s_hist[k]);
}

// Standalone level histogram (qm_level_histogram).
__global__ void __launch_bounds__(256) histogram_kernel(const float *levels, size_t n, double level_min, double bin_db,
                                                        uint32_t n_bins, uint32_t *counts) {
    extern __shared__ uint32_t s_hist[];
    for (uint32_t k = threadIdx.x; k < n_bins; k += blockDim.x) s_hist[k] = 0;
    __syncthreads();
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        atomicAdd(&s_hist[level_bin(__ldg(levels + i), level_min, bin_db, n_bins)], 1u);
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < n_bins; k += blockDim.x)
        if (s_hist[k]) atomicAdd(counts + k, s_hist[k]);
}

// Map cells (qm_quantize_cells; paint/src/levels.rs). The products and sums are rounded one by
// one (no fused multiply-add), as the reference's f64 arithmetic is.
__device__ __forceinline__ uint8_t lden_cell_of(double energy) {  // levels.rs:87-98, energy valid
    if (energy < 1.0) return QM_CELL_SILENCE;
    return (uint8_t)fmin(round(__dmul_rn(2.0, __dmul_rn(10.0, log10(energy)))), (double)(QM_CELL_SILENCE - 1));
}

__device__ __forceinline__ uint8_t nden_cell_of(double sone) {  // levels.rs:25-33
    const double byte = __dadd_rn(80.0, __dmul_rn(20.0, log2(sone)));
    if (isnan(byte) || byte < 0.0) return QM_CELL_SILENCE;
    return (uint8_t)fmin(round(byte), (double)(QM_CELL_SILENCE - 1));
}

// Thread = pixel (grid-stride). An invalid Lden energy of an assessed pixel lowers *first_bad to
// pixel * 8 + layer (layer QM_LAYERS: the total); that pixel's bytes are then not meaningful.
__global__ void __launch_bounds__(256) quantize_cells_kernel(const double *lden_energy, const double *sone,
                                                             const uint8_t *assessed, size_t n, uint8_t *lden_cells,
                                                             uint8_t *nden_cells, unsigned long long *first_bad) {
    constexpr int W = QM_LAYERS + 1;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        uint8_t lc[W], nc[W];
        if (assessed && assessed[p] == 0) {
#pragma unroll
            for (int l = 0; l < W; ++l) lc[l] = nc[l] = QM_CELL_NO_LEVEL;
        } else {
#pragma unroll
            for (int l = 0; l < W; ++l) lc[l] = nc[l] = QM_CELL_SILENCE;
            double total = 0.0;
            int bad = -1;
#pragma unroll
            for (int l = 0; l < QM_LAYERS; ++l) {
                const double e = lden_energy[p * QM_LAYERS + l];
                if (bad < 0 && !(isfinite(e) && e >= 0.0)) bad = l;
                if (bad < 0) lc[l] = lden_cell_of(e);
                total = __dadd_rn(total, e);  // in layer order, as the reference's sum
            }
            if (bad < 0 && !(isfinite(total) && total >= 0.0)) bad = QM_LAYERS;
            if (bad < 0) lc[QM_LAYERS] = lden_cell_of(total);
            if (bad >= 0) atomicMin(first_bad, (unsigned long long)p * 8ull + (unsigned long long)bad);
            if (nden_cells) {
#pragma unroll
                for (int l = 0; l < W; ++l) nc[l] = nden_cell_of(sone[p * W + l]);
            }
        }
#pragma unroll
        for (int l = 0; l < W; ++l) lden_cells[p * W + l] = lc[l];
        if (nden_cells) {
#pragma unroll
            for (int l = 0; l < W; ++l) nden_cells[p * W + l] = nc[l];
        }
    }
}

// HM3 / HMD stream bytes before Brotli (qm_hm3_predict; paint/src/hm3.rs:68-109). Thread = one
// output byte of one tile (grid-stride); the tile's first thread also writes its header.
__device__ __forceinline__ uint8_t paeth_residual(const uint8_t *tile, uint32_t at) {
    constexpr uint32_t P = QM_HM3_TILE_PX;
    const bool has_left = (at % P) != 0, has_above = at >= P;
    const int left = has_left ? tile[at - 1] : 0;
    const int above = has_above ? tile[at - P] : 0;
    const int corner = (has_left && has_above) ? tile[at - P - 1] : 0;
    const int estimate = left + above - corner;
    const int dl = abs(estimate - left), da = abs(estimate - above), dc = abs(estimate - corner);
    const int predicted = (dl <= da && dl <= dc) ? left : (da <= dc ? above : corner);
    return (uint8_t)(tile[at] - predicted);
}

__global__ void __launch_bounds__(256) hm3_predict_kernel(const uint8_t *cells, const uint8_t *layers, size_t n_tiles,
                                                          uint32_t header_word, uint8_t header_last,
                                                          uint8_t *streams) {
    constexpr size_t PIX = (size_t)QM_HM3_TILE_PX * QM_HM3_TILE_PX;
    const size_t total = n_tiles * PIX;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t tile = i / PIX;
        const uint32_t at = (uint32_t)(i - tile * PIX);
        uint8_t *out = streams + tile * (size_t)QM_HM3_STREAM_BYTES;
        if (at == 0) {
#pragma unroll
            for (int k = 0; k < 4; ++k) out[k] = (uint8_t)(header_word >> (8 * k));
            out[4] = header_last;
            out[5] = layers[tile];
        }
        out[6 + at] = paeth_residual(cells + tile * PIX, at);
    }
}

struct PairArgs {
    const int2 *rcv_xy;
    const float *rcv_alt;
    const uint32_t *rcv_own;
    const uint32_t *source_of_pair;
    const uint32_t *receiver_of_pair;
    size_t n_pairs;
    float *pair_sums;   // [n][9]
    float *pair_bands;  // [n][3][8]
    uint32_t *status;   // [n]
};

// A pair's PairEnergy sums and its bands per period from its path.
__device__ __forceinline__ void pair_outputs(const SceneDev &S, const SourceDev &src, const PathResult &res, float *sums,
                                             float *bands) {
    float air[QM_BANDS];
#pragma unroll
    for (int b = 0; b < QM_BANDS; ++b) air[b] = __expf(-S.air_per_m[b] * res.slant);
#pragma unroll
    for (int p = 0; p < QM_PERIODS; ++p) {
        float mixed = 0.f, calm = 0.f, down = 0.f;
        float pp = res.p[p];
#pragma unroll
        for (int b = 0; b < QM_BANDS; ++b) {
            float power = res.weight * src.energy[p * QM_BANDS + b];
            float e = power * air[b] * (pp * res.boundary[1][b] + (1.0f - pp) * res.boundary[0][b]);
            bands[p * QM_BANDS + b] = e;
            mixed += e;
            calm += power * air[b] * res.boundary[0][b];
            down += power * air[b] * res.boundary[1][b];
        }
        sums[p] = mixed;
        sums[3 + p] = calm;
        sums[6 + p] = down;
    }
}

// One thread per pair: the pair's ray with both states, its PairEnergy (exact.rs:128-132,
// 200-203) and its bands per period (received_bands, evaluate.rs:270-290).
template <class Caps>
__global__ void __launch_bounds__(128) evaluate_pairs_kernel(SceneDev S, PairArgs A) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= A.n_pairs) return;
    if (A.source_of_pair[i] >= S.n_sources) return;  // a line piece: the line pairs' kernel
    uint32_t r = A.receiver_of_pair[i];
    const SourceDev &src = S.sources[A.source_of_pair[i]];
    int2 xy = A.rcv_xy[r];
    PathWork<Caps::C, Caps::K, Caps::H> work;
    PathResult res;
    evaluate_path<Caps::C, Caps::K, Caps::H>(S, src, xy.x, xy.y, A.rcv_alt[r], A.rcv_own[r], true, work, res);
    pair_outputs(S, src, res, A.pair_sums + i * 9, A.pair_bands + i * QM_PERIODS * QM_BANDS);
    A.status[i] = res.status;
}

// Failed pairs again with large per-path capacities held in global scratch (grid-stride).
__global__ void __launch_bounds__(64) retry_pairs_kernel(SceneDev S, PairArgs A, const uint32_t *indices, uint32_t n,
                                                         PathWork<CapsLarge::C, CapsLarge::K, CapsLarge::H> *works) {
    uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t stride = gridDim.x * blockDim.x;
    PathWork<CapsLarge::C, CapsLarge::K, CapsLarge::H> &work = works[tid];
    for (uint32_t k = tid; k < n; k += stride) {
        size_t i = indices[k];
        uint32_t r = A.receiver_of_pair[i];
        const SourceDev &src = S.sources[A.source_of_pair[i]];
        int2 xy = A.rcv_xy[r];
        PathResult res;
        evaluate_path<CapsLarge::C, CapsLarge::K, CapsLarge::H>(S, src, xy.x, xy.y, A.rcv_alt[r], A.rcv_own[r], true,
                                                                work, res);
        pair_outputs(S, src, res, A.pair_sums + i * 9, A.pair_bands + i * QM_PERIODS * QM_BANDS);
        A.status[i] = res.status;
    }
}

// Point bands (add_bands, exact.rs:208-215): pairs grouped by point (a stable order), one thread per
// (point, layer-period-band slot) summing its pairs in order.
__global__ void point_bands_kernel(const uint32_t *order, const uint32_t *point_start, const uint32_t *point_ids,
                                   uint32_t n_groups, const float *pair_bands, const float *band_weight,
                                   const uint32_t *pair_layer, float *point_bands) {
    size_t g = blockIdx.x;
    if (g >= n_groups) return;
    uint32_t slot = threadIdx.x;  // layer * 24 + period * 8 + band
    if (slot >= 6 * QM_PERIODS * QM_BANDS) return;
    uint32_t layer = slot / (QM_PERIODS * QM_BANDS), pb = slot % (QM_PERIODS * QM_BANDS);
    KSum acc{0.f, 0.f};
    for (uint32_t k = point_start[g]; k < point_start[g + 1]; ++k) {
        uint32_t i = order[k];
        if (pair_layer[i] != layer) continue;
        float w = band_weight ? band_weight[i] : 1.0f;
        acc.add(w * pair_bands[(size_t)i * QM_PERIODS * QM_BANDS + pb]);
    }
    point_bands[(size_t)point_ids[g] * 6 * QM_PERIODS * QM_BANDS + slot] += acc.value();
}

// The crossing lists of rays (qm_list_crossings): the same walk the painter runs.
template <int CAP>
__global__ void __launch_bounds__(128) list_crossings_kernel(SceneDev S, const int2 *from, const int2 *to, size_t n,
                                                             uint32_t cap, uint32_t *counts, uint32_t *edges,
                                                             double *t, uint32_t *flags, uint32_t *status) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    XRec xs[CAP];
    uint32_t st = 0, tested = 0;
    int2 a = from[i], b = to[i];
    int k = list_crossings<CAP>(S, a.x, a.y, b.x, b.y, 0, xs, st, tested);
    counts[i] = k;
    status[i] = st;
    for (int j = 0; j < k && j < (int)cap; ++j) {
        edges[i * cap + j] = xs[j].edge;
        t[i * cap + j] = xs[j].t;
        flags[i * cap + j] = ((xs[j].info & X_BUILDING) ? 1u : 0u) | ((xs[j].info & X_BOUNDS) ? 2u : 0u);
    }
}

}  // namespace qm
