// ISO 532-1 stationary Zwicker loudness on the device: one thread per spectrum of 28 third-octave
// levels (qm_zwicker.cuh).

#include <cstdint>

#include "qm_zwicker.cuh"

namespace qm {

// One thread per spectrum; spectra are read as 28 consecutive floats (coalesced through L1).
__global__ void __launch_bounds__(128) zwicker_kernel(const float *thirds, size_t n, float *sone) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float levels[28];
    const float *p = thirds + i * 28;
#pragma unroll
    for (int k = 0; k < 28; ++k) levels[k] = __ldg(p + k);
    sone[i] = zwicker_sone(levels);
}

void launch_zwicker(const float *thirds, size_t n, float *sone, cudaStream_t stream) {
    if (n == 0) return;
    unsigned blocks = (unsigned)((n + 127) / 128);
    zwicker_kernel<<<blocks, 128, 0, stream>>>(thirds, n, sone);
}

}  // namespace qm
