// Batches of uneven receiver tiles: persistent CTAs take (tile, receiver block, source chunk) work
// items from a device queue (largest first), paint them with the exact path code and write each
// item's compensated cell sums to its own partial slot; a reduce pass sums each cell's chunks in
// chunk order. The queue is a counter: a CTA takes the next item until none is left, so nothing
// waits on anything.
#pragma once

#include "qm_kernels.cuh"

namespace qm {

struct TileDev {
    int origin_x, origin_y, spacing, nx, ny;
    uint32_t source_begin, source_end;
    uint32_t block_w, block_h, chunk, n_chunks;
    uint32_t pad;
    unsigned long long cell_offset;     // global index of the tile's first cell
    unsigned long long partial_offset;  // first partial slot: [n_chunks][cells] slots of 9 floats
};

struct WorkItem {
    uint32_t tile, block, chunk, pad;
};

struct BatchArgs {
    const TileDev *tiles;
    const WorkItem *items;
    uint32_t n_items;
    unsigned int *next;  // the queue head
    const float *rcv_alt;
    const uint32_t *rcv_own;
    float *partial;
    uint2 *retry;  // (global cell, source) of over-capacity paths
    uint32_t retry_cap;
    unsigned int *retry_count;
    unsigned long long *counters;  // paths, crossings, edge tests, failed paths, vertices, candidates
    float lden_w[QM_PERIODS];
    bool want_fav;
};

template <class Caps, int THREADS>
__global__ void __launch_bounds__(THREADS, 512 / THREADS) batch_paint_kernel(SceneDev S, BatchArgs B) {
    __shared__ unsigned int s_item;
    __shared__ unsigned long long s_counts[6];
    if (threadIdx.x < 6) s_counts[threadIdx.x] = 0;
    unsigned long long paths = 0, crossings = 0, tested = 0, failed_paths = 0, vertices = 0, candidates = 0;
    PathWork<Caps::C, Caps::K, Caps::H> work;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_item = atomicAdd(B.next, 1u);
        __syncthreads();
        const unsigned int item = s_item;
        if (item >= B.n_items) break;
        const WorkItem w = B.items[item];
        const TileDev T = B.tiles[w.tile];
        const uint32_t blocks_x = (T.nx + T.block_w - 1) / T.block_w;
        const uint32_t bx = w.block % blocks_x, by = w.block / blocks_x;
        const uint32_t per = T.block_w * T.block_h;
        const uint32_t s0 = T.source_begin + w.chunk * T.chunk, s1 = min(s0 + T.chunk, T.source_end);
        const uint32_t cells_t = (uint32_t)T.nx * T.ny;
        for (uint32_t r = threadIdx.x; r < per; r += THREADS) {
            const int2 slot = block_slot(r, T.block_w, T.block_h);
            const uint32_t ix = bx * T.block_w + (uint32_t)slot.x, iy = by * T.block_h + (uint32_t)slot.y;
            if (ix >= (uint32_t)T.nx || iy >= (uint32_t)T.ny) continue;
            const uint32_t cell = iy * T.nx + ix;
            const unsigned long long gcell = T.cell_offset + cell;
            const int rx = T.origin_x + (int)ix * T.spacing, ry = T.origin_y + (int)iy * T.spacing;
            const float alt = B.rcv_alt[gcell];
            const uint32_t own = B.rcv_own[gcell];
            KSum bands[QM_BANDS];
            KSum lden{0.f, 0.f};
#pragma unroll
            for (int b = 0; b < QM_BANDS; ++b) bands[b] = KSum{0.f, 0.f};
            for (uint32_t s = s0; s < s1; ++s) {
                const SourceDev &src = S.sources[s];
                PathResult res;
                evaluate_path<Caps::C, Caps::K, Caps::H>(S, src, rx, ry, alt, own, B.want_fav, work, res);
                ++paths;
                crossings += res.crossings;
                tested += res.edges_tested;
                vertices += res.vertices;
                candidates += res.candidates;
                if (res.status) {
                    ++failed_paths;
                    unsigned int slot = atomicAdd(B.retry_count, 1u);
                    if (slot < B.retry_cap) B.retry[slot] = make_uint2((uint32_t)gcell, s);
                    continue;
                }
                float day[QM_BANDS], le;
                path_energies(S, res, src, B.lden_w, day, le);
#pragma unroll
                for (int b = 0; b < QM_BANDS; ++b) bands[b].add(day[b]);
                lden.add(le);
            }
            float *out = B.partial + (T.partial_offset + (unsigned long long)w.chunk * cells_t + cell) * GRID_SLOTS;
#pragma unroll
            for (int b = 0; b < QM_BANDS; ++b) out[b] = bands[b].value();
            out[8] = lden.value();
        }
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
    if (threadIdx.x < 6) atomicAdd(B.counters + threadIdx.x, s_counts[threadIdx.x]);
}

// Over-capacity paths of a batch again, with large capacities; receivers from the batch's tables.
struct BatchRetryArgs {
    const int2 *rcv_xy;
    const float *rcv_alt;
    const uint32_t *rcv_own;
    float lden_w[QM_PERIODS];
    bool want_fav;
};

__global__ void __launch_bounds__(64) batch_retry_kernel(SceneDev S, BatchRetryArgs A, const uint2 *pairs, uint32_t n,
                                                         PathWork<CapsLarge::C, CapsLarge::K, CapsLarge::H> *works,
                                                         float *out, uint32_t *status) {
    uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t stride = gridDim.x * blockDim.x;
    PathWork<CapsLarge::C, CapsLarge::K, CapsLarge::H> &work = works[tid];
    for (uint32_t i = tid; i < n; i += stride) {
        uint2 pr = pairs[i];
        int2 xy = A.rcv_xy[pr.x];
        const SourceDev &src = S.sources[pr.y];
        PathResult r;
        evaluate_path<CapsLarge::C, CapsLarge::K, CapsLarge::H>(S, src, xy.x, xy.y, A.rcv_alt[pr.x], A.rcv_own[pr.x],
                                                                A.want_fav, work, r);
        status[i] = r.status;
        float day[QM_BANDS], le = 0.f;
        if (r.status == 0) path_energies(S, r, src, A.lden_w, day, le);
#pragma unroll
        for (int b = 0; b < QM_BANDS; ++b) out[(size_t)i * GRID_SLOTS + b] = r.status ? 0.f : day[b];
        out[(size_t)i * GRID_SLOTS + 8] = le;
    }
}

// Per global cell: its tile's chunk slots in chunk order plus its re-run paths, then the levels.
struct BatchReduceArgs {
    const TileDev *tiles;
    const uint32_t *cell_tile;  // tile of each global cell (~0u: none)
    unsigned long long n_cells;
    const float *partial;
    const float *retry_acc;  // [n_cells][9]
    float *cell_bands, *cell_dba, *cell_lden;
};

__global__ void __launch_bounds__(256) batch_reduce_kernel(BatchReduceArgs R) {
    const unsigned long long g = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
    if (g >= R.n_cells) return;
    const uint32_t t = R.cell_tile[g];
    if (t == ~0u) {
#pragma unroll
        for (int b = 0; b < QM_BANDS; ++b) R.cell_bands[g * QM_BANDS + b] = -INFINITY;
        R.cell_dba[g] = -INFINITY;
        R.cell_lden[g] = -INFINITY;
        return;
    }
    const TileDev T = R.tiles[t];
    const unsigned long long cell = g - T.cell_offset, cells_t = (unsigned long long)T.nx * T.ny;
    KSum acc[GRID_SLOTS];
#pragma unroll
    for (int k = 0; k < GRID_SLOTS; ++k) acc[k] = KSum{0.f, 0.f};
    for (uint32_t c = 0; c < T.n_chunks; ++c) {
        const float *p = R.partial + (T.partial_offset + c * cells_t + cell) * GRID_SLOTS;
#pragma unroll
        for (int k = 0; k < GRID_SLOTS; ++k) acc[k].add(p[k]);
    }
#pragma unroll
    for (int k = 0; k < GRID_SLOTS; ++k) acc[k].add(R.retry_acc[g * GRID_SLOTS + k]);
    KSum total{0.f, 0.f};
#pragma unroll
    for (int b = 0; b < QM_BANDS; ++b) {
        float e = acc[b].value();
        total.add(e);
        R.cell_bands[g * QM_BANDS + b] = 10.0f * log10f(e);
    }
    R.cell_dba[g] = 10.0f * log10f(total.value());
    R.cell_lden[g] = 10.0f * log10f(acc[8].value());
}

}  // namespace qm
