// Line pieces as candidates of Batch::evaluate on the device: one thread a (receiver, piece) pair.
// The piece's quadrature nodes are placed as the reference places them (physics/src/line.rs:178-206,
// qm_line.cuh), each wide bucket asking the receiver's skyline (popup/src/evaluate.rs:225-242,
// qm_skyline.cuh) with the source's height as the floor; each node's ray runs from its fractional
// point along the piece by the f64 walks (qm_offlattice.cuh), with obstacles only where the mask
// leaves its ray open, through the exact path (evaluate_listed), weighted by the node's angle times
// the piece's divergence (the oracle's evaluate_line_piece restates popup/src/evaluate.rs:171-267).
#pragma once

#include "qm_kernels.cuh"
#include "qm_line.cuh"
#include "qm_offlattice.cuh"
#include "qm_skyline.cuh"

namespace qm {

// A line piece on the device: its ends (lattice steps, fractional allowed) and its source
// properties, energy per metre of the piece.
struct PieceDev {
    double ax, ay, bx, by;
    SourceDev src;
};

// The skyline query the quadrature calls, from the receiver at (rx, ry) above the source's height.
struct DeviceSkyline {
    const skyline::Index *ix;
    int64_t rx, ry;
    double floor_m;
    template <class Visit>
    __device__ void operator()(double lo, double hi, double radius, Visit &visit) const {
        skyline::arcs(*ix, rx, ry, lo, hi, radius, floor_m, visit);
    }
};

// One (receiver, piece) pair: PairEnergy sums[9] and bands[3][8] summed over the piece's nodes.
template <int CAP_C, int CAP_K, int CAP_H>
__device__ void evaluate_line_pair(const SceneDev &S, const skyline::Index &sky, const PieceDev &pc, int rx, int ry,
                                   float alt, uint32_t own, PathWork<CAP_C, CAP_K, CAP_H> &work, float *sums,
                                   float *bands, uint32_t &status) {
#pragma unroll
    for (int k = 0; k < 9; ++k) sums[k] = 0.0f;
#pragma unroll
    for (int k = 0; k < QM_PERIODS * QM_BANDS; ++k) bands[k] = 0.0f;
    double za, ga, zb, gb;
    terrain_at_d(S, pc.ax, pc.ay, za, ga);
    terrain_at_d(S, pc.bx, pc.by, zb, gb);
    const double m = (double)S.step_m;
    const double h = (double)pc.src.height;
    const double start[3] = {(pc.ax - (double)rx) * m, (pc.ay - (double)ry) * m, za + h - (double)alt};
    const double end[3] = {(pc.bx - (double)rx) * m, (pc.by - (double)ry) * m, zb + h - (double)alt};
    line::Piece g;
    if (!g.make(start, end)) return;
    const double divergence = g.divergence();
    DeviceSkyline query{&sky, rx, ry, fmax(h, 0.0)};
    auto emit = [&](double along, double weight, bool on_ray) {
        const double fraction = along / g.length;
        const double px = pc.ax + fraction * (pc.bx - pc.ax), py = pc.ay + fraction * (pc.by - pc.ay);
        PathResult res;
        res.status = 0;
        res.edges_tested = 0;
        const int nx = on_ray ? list_crossings_d<CAP_C>(S, px, py, rx, ry, own, work.xs, res.status, res.edges_tested) : 0;
        evaluate_listed<CAP_C, CAP_K, CAP_H, TerrainWalkD>(S, pc.src, rx, ry, alt, true, work, nx, res, px, py);
        status |= res.status;
        res.weight = (float)(weight * divergence);
        float node_sums[9], node_bands[QM_PERIODS * QM_BANDS];
        pair_outputs(S, pc.src, res, node_sums, node_bands);
#pragma unroll
        for (int k = 0; k < 9; ++k) sums[k] += node_sums[k];
#pragma unroll
        for (int k = 0; k < QM_PERIODS * QM_BANDS; ++k) bands[k] += node_bands[k];
    };
    line::quadrature_nodes(g, query, emit);
}

struct LinePairArgs {
    const PieceDev *pieces;
    skyline::Index sky;
    const uint32_t *line_pairs;  // the pairs whose candidate is a piece
    uint32_t n_line_pairs;
};

// One thread a line pair, the per-path work areas in local memory.
template <class Caps>
__global__ void __launch_bounds__(128) evaluate_line_pairs_kernel(SceneDev S, PairArgs A, LinePairArgs L) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= L.n_line_pairs) return;
    const size_t i = L.line_pairs[k];
    const uint32_t r = A.receiver_of_pair[i];
    const PieceDev &pc = L.pieces[A.source_of_pair[i] - S.n_sources];
    const int2 xy = A.rcv_xy[r];
    PathWork<Caps::C, Caps::K, Caps::H> work;
    uint32_t status = 0;
    evaluate_line_pair<Caps::C, Caps::K, Caps::H>(S, L.sky, pc, xy.x, xy.y, A.rcv_alt[r], A.rcv_own[r], work,
                                                  A.pair_sums + i * 9, A.pair_bands + i * QM_PERIODS * QM_BANDS, status);
    A.status[i] = status;
}

// Line pairs over the per-path capacities again with large ones in global scratch (grid-stride).
__global__ void __launch_bounds__(64) retry_line_pairs_kernel(SceneDev S, PairArgs A, LinePairArgs L,
                                                              const uint32_t *indices, uint32_t n,
                                                              PathWork<CapsLarge::C, CapsLarge::K, CapsLarge::H> *works) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    PathWork<CapsLarge::C, CapsLarge::K, CapsLarge::H> &work = works[tid];
    for (uint32_t k = tid; k < n; k += stride) {
        const size_t i = indices[k];
        const uint32_t r = A.receiver_of_pair[i];
        const PieceDev &pc = L.pieces[A.source_of_pair[i] - S.n_sources];
        const int2 xy = A.rcv_xy[r];
        uint32_t status = 0;
        evaluate_line_pair<CapsLarge::C, CapsLarge::K, CapsLarge::H>(S, L.sky, pc, xy.x, xy.y, A.rcv_alt[r], A.rcv_own[r],
                                                                     work, A.pair_sums + i * 9,
                                                                     A.pair_bands + i * QM_PERIODS * QM_BANDS, status);
        A.status[i] = status;
    }
}

}  // namespace qm
