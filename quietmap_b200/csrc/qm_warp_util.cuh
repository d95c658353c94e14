// Warp-level building blocks of the warp-per-path painter: reductions, ballot compaction, a bitonic
// sort in shared memory, and the exact merge of two arithmetic sequences of line crossings (the
// cells a ray walks and the DEM lines it crosses are both such merges).
#pragma once

#include <cstdint>

namespace qm {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

__device__ __forceinline__ int warp_exclusive_scan(int v, int &total) {
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(FULL, x, o);
        if (lane_id() >= o) x += y;
    }
    total = __shfl_sync(FULL, x, 31);
    return x - v;
}

// Two crossing sequences along a ray: A_i = (a0 + i*pa) / da for i < na and B_j = (b0 + j*pb) / db
// for j < nb (integers, da, db > 0; each sequence increasing). Merged in increasing order; on a tie
// B comes first. All decisions are exact integer comparisons.
struct Merge2 {
    long long a0, pa, da, na;
    long long b0, pb, db, nb;

    __device__ __forceinline__ bool a_before_b(long long i, long long j) const {
        // A_i < B_j strictly (a tie puts B first).
        return (a0 + i * pa) * db < (b0 + j * pb) * da;
    }
    // The number of A among the first m merged elements starting from (ia, ib).
    __device__ __forceinline__ long long count_a(long long m, long long ia, long long ib) const {
        long long ra = na - ia, rb = nb - ib;
        long long lo = m - rb > 0 ? m - rb : 0;  // at least this many A
        long long hi = m < ra ? m : ra;          // at most this many
        // Largest p in [lo, hi] with p == lo or A[ia + p - 1] before B[ib + m - p].
        while (lo < hi) {
            long long p = (lo + hi + 1) >> 1;
            long long j = ib + m - p;
            bool ok = (j >= nb) || a_before_b(ia + p - 1, j);
            if (ok)
                lo = p;
            else
                hi = p - 1;
        }
        return lo;
    }
};

// Lane l's element of the next chunk of 32 merged elements from (ia, ib): `is_a`, its index, and
// whether it exists; (ia, ib) advance past the chunk. Returns the number of elements in the chunk.
__device__ __forceinline__ int merge_chunk(const Merge2 &m, long long &ia, long long &ib, bool &is_a, long long &index,
                                           bool &valid) {
    long long remaining = (m.na - ia) + (m.nb - ib);
    int n = remaining < 32 ? (int)remaining : 32;
    int l = lane_id();
    valid = l < n;
    long long c1 = valid ? m.count_a(l + 1, ia, ib) : 0;
    long long c0 = __shfl_up_sync(FULL, c1, 1);
    if (l == 0) c0 = 0;
    is_a = c1 > c0;
    index = is_a ? ia + c1 - 1 : ib + (l - c1);
    long long last_c = __shfl_sync(FULL, c1, n > 0 ? n - 1 : 0);
    if (n > 0) {
        ia += last_c;
        ib += n - last_c;
    }
    return n;
}

// Bitonic sort of `n` (a power of two) 64-bit keys with 32-bit payloads in shared memory, ascending.
__device__ inline void warp_bitonic_sort(unsigned long long *keys, uint32_t *vals, int n) {
    for (int k = 2; k <= n; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane_id(); i < n; i += 32) {
                int p = i ^ j;
                if (p > i) {
                    bool up = (i & k) == 0;
                    unsigned long long a = keys[i], b = keys[p];
                    if ((a > b) == up) {
                        keys[i] = b;
                        keys[p] = a;
                        uint32_t t = vals[i];
                        vals[i] = vals[p];
                        vals[p] = t;
                    }
                }
            }
            __syncwarp();
        }
    }
}

}  // namespace qm
