// ISO 532-1 stationary Zwicker loudness on the device, FP32, built without fast math (the
// reference's loudness module is too: paint-gpu/src/device.rs:287). Restates
// physics/src/loudness.rs:100-182; tables loudness.rs:24-97. Included by every translation unit
// whose kernels take loudness: the tables are per unit.
#pragma once

#include <cstdint>

namespace qm {

static __constant__ float c_rap[8] = {45.0f, 55.0f, 65.0f, 71.0f, 80.0f, 90.0f, 100.0f, 120.0f};
static __constant__ float c_dll[8][11] = {
    {-32.0f, -24.0f, -16.0f, -10.0f, -5.0f, 0.0f, -7.0f, -3.0f, 0.0f, -2.0f, 0.0f},
    {-29.0f, -22.0f, -15.0f, -10.0f, -4.0f, 0.0f, -7.0f, -2.0f, 0.0f, -2.0f, 0.0f},
    {-27.0f, -19.0f, -14.0f, -9.0f, -4.0f, 0.0f, -6.0f, -2.0f, 0.0f, -2.0f, 0.0f},
    {-25.0f, -17.0f, -12.0f, -9.0f, -3.0f, 0.0f, -5.0f, -2.0f, 0.0f, -2.0f, 0.0f},
    {-23.0f, -16.0f, -11.0f, -7.0f, -3.0f, 0.0f, -4.0f, -1.0f, 0.0f, -1.0f, 0.0f},
    {-20.0f, -14.0f, -10.0f, -6.0f, -3.0f, 0.0f, -4.0f, -1.0f, 0.0f, -1.0f, 0.0f},
    {-18.0f, -12.0f, -9.0f, -6.0f, -2.0f, 0.0f, -3.0f, -1.0f, 0.0f, -1.0f, 0.0f},
    {-15.0f, -10.0f, -8.0f, -4.0f, -2.0f, 0.0f, -3.0f, -1.0f, 0.0f, -1.0f, 0.0f},
};
static __constant__ float c_ltq[20] = {30.0f, 18.0f, 12.0f, 8.0f, 7.0f, 6.0f, 5.0f, 4.0f, 3.0f, 3.0f,
                                3.0f,  3.0f,  3.0f,  3.0f, 3.0f, 3.0f, 3.0f, 3.0f, 3.0f, 3.0f};
static __constant__ float c_a0[20] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f,
                               -0.5f, -1.6f, -3.2f, -5.4f, -5.6f, -4.0f, -1.5f, 2.0f, 5.0f, 12.0f};
static __constant__ float c_dcb[20] = {-0.25f, -0.6f, -0.8f, -0.8f, -0.5f, 0.0f, 0.5f, 1.1f, 1.5f, 1.7f,
                                1.8f,   1.8f,  1.7f,  1.6f,  1.4f,  1.2f, 0.8f, 0.5f, 0.0f, -0.5f};
static __constant__ float c_zup[21] = {0.9f,  1.8f,  2.8f,  3.5f,  4.4f,  5.4f,  6.6f,  7.9f,  9.2f,  10.6f, 12.3f,
                                13.8f, 15.2f, 16.7f, 18.1f, 19.3f, 20.6f, 21.8f, 22.7f, 23.6f, 24.0f};
static __constant__ float c_rns[18] = {21.5f, 18.0f, 15.1f, 11.5f, 9.0f, 6.1f, 4.4f, 3.1f, 2.13f,
                                1.36f, 0.82f, 0.42f, 0.30f, 0.22f, 0.15f, 0.10f, 0.035f, 0.0f};
static __constant__ float c_usl[18][8] = {
    {13.0f, 8.2f, 6.3f, 5.5f, 5.5f, 5.5f, 5.5f, 5.5f},         {9.0f, 7.5f, 6.0f, 5.1f, 4.5f, 4.5f, 4.5f, 4.5f},
    {7.8f, 6.7f, 5.6f, 4.9f, 4.4f, 3.9f, 3.9f, 3.9f},          {6.2f, 5.4f, 4.6f, 4.0f, 3.5f, 3.2f, 3.2f, 3.2f},
    {4.5f, 3.8f, 3.6f, 3.2f, 2.9f, 2.7f, 2.7f, 2.7f},          {3.7f, 3.0f, 2.8f, 2.35f, 2.2f, 2.2f, 2.2f, 2.2f},
    {2.9f, 2.3f, 2.1f, 1.9f, 1.8f, 1.7f, 1.7f, 1.7f},          {2.4f, 1.7f, 1.5f, 1.35f, 1.3f, 1.3f, 1.3f, 1.3f},
    {1.95f, 1.45f, 1.3f, 1.15f, 1.1f, 1.1f, 1.1f, 1.1f},       {1.5f, 1.2f, 0.94f, 0.86f, 0.82f, 0.82f, 0.82f, 0.82f},
    {0.72f, 0.67f, 0.64f, 0.63f, 0.62f, 0.62f, 0.62f, 0.62f},  {0.59f, 0.53f, 0.51f, 0.50f, 0.42f, 0.42f, 0.42f, 0.42f},
    {0.40f, 0.33f, 0.26f, 0.24f, 0.24f, 0.22f, 0.22f, 0.22f},  {0.27f, 0.21f, 0.20f, 0.18f, 0.17f, 0.17f, 0.17f, 0.17f},
    {0.16f, 0.15f, 0.14f, 0.12f, 0.11f, 0.11f, 0.11f, 0.11f},  {0.12f, 0.11f, 0.10f, 0.08f, 0.08f, 0.08f, 0.08f, 0.08f},
    {0.09f, 0.08f, 0.07f, 0.06f, 0.06f, 0.06f, 0.06f, 0.05f},  {0.06f, 0.05f, 0.03f, 0.02f, 0.02f, 0.02f, 0.02f, 0.02f},
};

static __device__ __forceinline__ float energy_db(float level) { return expf(level * 0.2302585092994046f); }

// zwicker_loudness_sone (loudness.rs:148-182) of one spectrum.
static __device__ float zwicker_sone(const float *in) {
    float levels[28];
#pragma unroll
    for (int i = 0; i < 28; ++i) levels[i] = fmaxf(in[i], -60.0f);
    // core_loudness (loudness.rs:100-144)
    float corrected[11];
#pragma unroll
    for (int band = 0; band < 11; ++band) {
        float level = levels[band];
        int range = 7;
        for (int k = 0; k < 8; ++k)
            if (level <= c_rap[k] - c_dll[k][band]) {
                range = k;
                break;
            }
        corrected[band] = energy_db(level + c_dll[range][band]);
    }
    float lowest[3];
    {
        float s0 = 0.f, s1 = 0.f, s2 = 0.f;
#pragma unroll
        for (int b = 0; b < 6; ++b) s0 += corrected[b];
#pragma unroll
        for (int b = 6; b < 9; ++b) s1 += corrected[b];
        s2 = corrected[9] + corrected[10];
        lowest[0] = s0 > 0.f ? 10.0f * log10f(s0) : -INFINITY;
        lowest[1] = s1 > 0.f ? 10.0f * log10f(s1) : -INFINITY;
        lowest[2] = s2 > 0.f ? 10.0f * log10f(s2) : -INFINITY;
    }
    float core[21];
#pragma unroll
    for (int band = 0; band < 20; ++band) {
        float level = (band < 3 ? lowest[band] : levels[band + 8]) - c_a0[band];
        float v = 0.0f;
        if (level > c_ltq[band]) {
            level -= c_dcb[band];
            float threshold = energy_db(c_ltq[band] / 4.0f);
            v = fmaxf(0.0635f * threshold * (sqrtf(sqrtf(0.75f + 0.25f * energy_db(level - c_ltq[band]))) - 1.0f), 0.0f);
        }
        core[band] = v;
    }
    core[20] = 0.0f;
    float correction = 0.4f + 0.32f * powf(core[0], 0.2f);
    if (correction <= 1.0f) core[0] *= correction;
    float total = 0.0f, z1 = 0.0f, n1 = 0.0f;
    for (int band = 0; band < 21; ++band) {
        float upper = c_zup[band] + 0.0001f;
        int group = min(max(band - 1, 0), 7);
        float c = core[band];
        // Each band ends in at most 19 slope pieces (one per RNS range) plus one flat piece.
        for (int guard = 0; guard < 24 && z1 < upper; ++guard) {
            if (n1 <= c) {
                total += c * (upper - z1);
                z1 = upper;
                n1 = c;
            } else {
                int range = 17;
                for (int k = 0; k < 18; ++k)
                    if (n1 > c_rns[k]) {
                        range = k;
                        break;
                    }
                float steepness = c_usl[range][group];
                float n2 = fmaxf(c_rns[range], c);
                float z2 = z1 + (n1 - n2) / steepness;
                if (z2 > upper) {
                    z2 = upper;
                    n2 = n1 - (z2 - z1) * steepness;
                }
                total += (z2 - z1) * (n1 + n2) * 0.5f;
                z1 = z2;
                n1 = n2;
            }
        }
    }
    return fmaxf(total, 0.0f);
}

}  // namespace qm
