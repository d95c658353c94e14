// The surrogate network's kernels: BF16 tensor-core matrix products with FP32 accumulation
// (mma.sync m16n8k16), fused five-layer inference with the activations chained through
// registers, training products for the backward pass, and Adam on FP32 master weights.
#include "qm_mlp.h"
#include "qm_stage.cuh"

#include <algorithm>
#include <cmath>

namespace qm {
namespace {

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}

// D += A (16x16, row) * B (16x8, col), BF16 in, FP32 accumulate.
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ void ldsm_x4(uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3, const void *p) {
    unsigned a = (unsigned)__cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(a));
}

__device__ __forceinline__ void ldsm_x2(uint32_t &r0, uint32_t &r1, const void *p) {
    unsigned a = (unsigned)__cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];" : "=r"(r0), "=r"(r1) : "r"(a));
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    unsigned a = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// GELU in its tanh form (Hendrycks and Gimpel, 2016): 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))),
// with the hardware tanh; and its derivative. Training and inference use the same function.
__device__ __forceinline__ float tanh_hw(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
constexpr float GELU_C = 0.7978845608028654f, GELU_A = 0.044715f;
__device__ __forceinline__ float gelu(float z) {
    float t = tanh_hw(GELU_C * fmaf(GELU_A * z, z * z, z));
    return 0.5f * z * (1.0f + t);
}
__device__ __forceinline__ float gelu_grad(float z) {
    float t = tanh_hw(GELU_C * fmaf(GELU_A * z, z * z, z));
    return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * GELU_C * fmaf(3.0f * GELU_A * z, z, 1.0f);
}

// ---------------------------------------------------------------------------------------------
// Fused inference: a CTA of 8 warps takes 128 rows (16 a warp) through all five layers. The
// weights stream through shared memory in chunks of 64 output rows (cp.async, double buffered);
// each layer's FP32 results become the next layer's BF16 A fragments in registers (the m16n8
// accumulator layout is the m16k16 operand layout, two n-tiles per k-tile).

constexpr int FT_ROWS = 128, FT_THREADS = 256;
constexpr int CH_ROWS = 64, CH_STRIDE = 256 + 8;  // padded rows: conflict-free ldmatrix
constexpr int CH_ELEMS = CH_ROWS * CH_STRIDE;
constexpr int CHUNKS = 17;  // 4 per hidden layer, 1 for the output layer

struct FusedArgs {
    const __nv_bfloat16 *w16;
    const float *master;
    float out_shift[MLP_OUT], out_scale[MLP_OUT], lab_lo[MLP_OUT], lab_hi[MLP_OUT];
    const __nv_bfloat16 *x;
    size_t rows;
    float *out;      // forward mode: [rows][8]
    MlpPaintArgs p;  // paint mode
};

__device__ __forceinline__ void issue_chunk(const __nv_bfloat16 *w16, int q, __nv_bfloat16 *buf) {
    const int l = q < 16 ? q / 4 : 4, c = q < 16 ? q % 4 : 0;
    const int K = l == 0 ? 32 : 256, rows = l == 4 ? 8 : CH_ROWS;
    const __nv_bfloat16 *src = w16 + mlp_w16_offset(l) + (size_t)c * CH_ROWS * K;
    const int per_row = K / 8, total = rows * per_row;
    for (int v = threadIdx.x; v < total; v += FT_THREADS) {
        int r = v / per_row, k8 = (v - r * per_row) * 8;
        cp_async16(buf + r * CH_STRIDE + k8, src + (size_t)r * K + k8);
    }
}

struct Pipe {
    __nv_bfloat16 *bufs;
    const __nv_bfloat16 *w16;
    int sel;
    __device__ __forceinline__ const __nv_bfloat16 *begin(int q_next, bool has_next) {
        if (has_next) issue_chunk(w16, q_next, bufs + (sel ^ 1) * CH_ELEMS);
        cp_commit();
        cp_wait<1>();
        __syncthreads();
        return bufs + sel * CH_ELEMS;
    }
    __device__ __forceinline__ void end() {
        __syncthreads();
        sel ^= 1;
    }
};

// One chunk of 64 outputs over KT k-tiles of input.
template <int KT>
__device__ __forceinline__ void chunk_mma(const __nv_bfloat16 *buf, const uint32_t (&a)[KT][4], float (&acc)[8][4],
                                          int lane) {
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
        for (int i = 0; i < 4; ++i) acc[nt][i] = 0.0f;
    const int j = lane >> 3, i = lane & 7;
#pragma unroll
    for (int kt = 0; kt < KT; ++kt) {
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            uint32_t b0, b1, b2, b3;
            ldsm_x4(b0, b1, b2, b3, buf + (16 * p + i + 8 * (j >> 1)) * CH_STRIDE + 16 * kt + 8 * (j & 1));
            mma_bf16(acc[2 * p], a[kt], b0, b1);
            mma_bf16(acc[2 * p + 1], a[kt], b2, b3);
        }
    }
}

// Bias + GELU of a chunk's accumulators into k-tiles 4c..4c+3 of the next layer's A fragments.
__device__ __forceinline__ void chunk_gelu(const float (&acc)[8][4], const float *bias, int c, int t,
                                           uint32_t (&next)[16][4]) {
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        int col = 64 * c + 8 * nt + 2 * t;
        float b0 = __ldg(bias + col), b1 = __ldg(bias + col + 1);
        uint32_t lo = pack_bf16(gelu(acc[nt][0] + b0), gelu(acc[nt][1] + b1));
        uint32_t hi = pack_bf16(gelu(acc[nt][2] + b0), gelu(acc[nt][3] + b1));
        int q = 4 * c + nt / 2;
        if ((nt & 1) == 0) {
            next[q][0] = lo;
            next[q][1] = hi;
        } else {
            next[q][2] = lo;
            next[q][3] = hi;
        }
    }
}

template <int KT>
__device__ __forceinline__ void hidden_layer(Pipe &pipe, int first_q, const uint32_t (&in)[KT][4], const float *bias,
                                             uint32_t (&out)[16][4], int lane, bool has_next_tile) {
    const int t = lane & 3;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        int q = first_q + c;
        const __nv_bfloat16 *buf = pipe.begin((q + 1) % CHUNKS, q + 1 < CHUNKS || has_next_tile);
        float acc[8][4];
        chunk_mma<KT>(buf, in, acc, lane);
        chunk_gelu(acc, bias, c, t, out);
        pipe.end();
    }
}

template <int MODE>
__global__ void __launch_bounds__(FT_THREADS, 1) mlp_fused_kernel(FusedArgs A) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ float s_red[8][9];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const size_t n_tiles = (A.rows + FT_ROWS - 1) / FT_ROWS;
    Pipe pipe{reinterpret_cast<__nv_bfloat16 *>(smem_raw), A.w16, 0};
    if (blockIdx.x >= n_tiles) return;
    issue_chunk(A.w16, 0, pipe.bufs);
    cp_commit();
    const float *bias[MLP_LAYERS];
#pragma unroll
    for (int l = 0; l < MLP_LAYERS; ++l) bias[l] = A.master + mlp_b_offset(l);
    for (size_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const bool has_next = tile + gridDim.x < n_tiles;
        const size_t r0 = tile * FT_ROWS + warp * 16 + g, r1 = r0 + 8;
        // Layer 1 input fragments straight from the feature rows.
        uint32_t xa[2][4];
#pragma unroll
        for (int kt = 0; kt < 2; ++kt) {
            int col = 16 * kt + 2 * t;
            const uint32_t *x0 = reinterpret_cast<const uint32_t *>(A.x + r0 * MLP_IN + col);
            const uint32_t *x1 = reinterpret_cast<const uint32_t *>(A.x + r1 * MLP_IN + col);
            xa[kt][0] = r0 < A.rows ? __ldg(x0) : 0u;
            xa[kt][1] = r1 < A.rows ? __ldg(x1) : 0u;
            xa[kt][2] = r0 < A.rows ? __ldg(x0 + 4) : 0u;
            xa[kt][3] = r1 < A.rows ? __ldg(x1 + 4) : 0u;
        }
        uint32_t ha[16][4], hb[16][4];
        hidden_layer<2>(pipe, 0, xa, bias[0], ha, lane, has_next);
        hidden_layer<16>(pipe, 4, ha, bias[1], hb, lane, has_next);
        hidden_layer<16>(pipe, 8, hb, bias[2], ha, lane, has_next);
        hidden_layer<16>(pipe, 12, ha, bias[3], hb, lane, has_next);
        // Output layer: 8 outputs, one n-tile.
        float y[4] = {0.f, 0.f, 0.f, 0.f};
        {
            const __nv_bfloat16 *buf = pipe.begin(0, has_next);
            const int i = lane & 7, j = (lane >> 3) & 1;
#pragma unroll
            for (int kt = 0; kt < 16; ++kt) {
                uint32_t b0, b1;
                ldsm_x2(b0, b1, buf + i * CH_STRIDE + 16 * kt + 8 * j);
                mma_bf16(y, hb[kt], b0, b1);
            }
            pipe.end();
        }
        const int o = 2 * t;
        float a00 = (y[0] + __ldg(bias[4] + o)) * A.out_scale[o] + A.out_shift[o];
        float a01 = (y[1] + __ldg(bias[4] + o + 1)) * A.out_scale[o + 1] + A.out_shift[o + 1];
        float a10 = (y[2] + __ldg(bias[4] + o)) * A.out_scale[o] + A.out_shift[o];
        float a11 = (y[3] + __ldg(bias[4] + o + 1)) * A.out_scale[o + 1] + A.out_shift[o + 1];
        if (MODE == 0) {
            if (r0 < A.rows) *reinterpret_cast<float2 *>(A.out + r0 * MLP_OUT + o) = make_float2(a00, a01);
            if (r1 < A.rows) *reinterpret_cast<float2 *>(A.out + r1 * MLP_OUT + o) = make_float2(a10, a11);
        } else {
            const MlpPaintArgs &P = A.p;
            float v[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) v[k] = 0.0f;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const size_t r = h ? r1 : r0;
                const float x0 = h ? a10 : a00, x1 = h ? a11 : a01;
                bool use = r < A.rows && P.eligible[r];
                bool out_of_range = !(x0 >= A.lab_lo[o] - 1.0f && x0 <= A.lab_hi[o] + 1.0f) ||
                                    !(x1 >= A.lab_lo[o + 1] - 1.0f && x1 <= A.lab_hi[o + 1] + 1.0f);
                // Any band of the row out of range sends the row to the exact path.
                unsigned bad = __ballot_sync(0xffffffffu, use && out_of_range);
                bool row_bad = ((bad >> (lane & ~3)) & 0xfu) != 0;
                if (use && row_bad) {
                    if (t == 0) {
                        uint32_t cell = (uint32_t)(r / P.rows_per_cell), s = (uint32_t)(r % P.rows_per_cell);
                        unsigned slot = atomicAdd(P.retry_count, 1u);
                        if (slot < P.retry_cap) P.retry[slot] = make_uint2(cell, P.source_begin + s);
                    }
                    use = false;
                }
                if (use) {
                    const float *cf = P.coef + r * 16;
                    float e0 = exp2f(-x0 * 0.33219280948873623f), e1 = exp2f(-x1 * 0.33219280948873623f);
                    float d0 = __ldg(cf + o) * e0, d1 = __ldg(cf + o + 1) * e1;
                    float l = __ldg(cf + 8 + o) * e0 + __ldg(cf + 8 + o + 1) * e1;
                    v[o] += d0;  // o varies by lane: written into the lane's own two bands
                    v[o + 1] += d1;
                    v[8] += l;
                    if (t == 0) atomicAdd(P.taken, 1ull);
                }
            }
            // v[k] is nonzero only for k in {o, o+1, 8}: sum over the warp per band, then over warps.
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                float s = v[k];
#pragma unroll
                for (int m = 16; m > 0; m >>= 1) s += __shfl_xor_sync(0xffffffffu, s, m);
                v[k] = s;
            }
            if (lane == 0)
#pragma unroll
                for (int k = 0; k < 9; ++k) s_red[warp][k] = v[k];
            __syncthreads();
            if (threadIdx.x < 9) {
                float s = 0.0f;
                for (int w = 0; w < 8; ++w) s += s_red[w][threadIdx.x];
                const size_t row0 = tile * FT_ROWS;
                const size_t cell = row0 / P.rows_per_cell, slice = (row0 % P.rows_per_cell) / FT_ROWS;
                float *dst = P.partial + (slice * (size_t)P.cells + cell) * 9 + threadIdx.x;
                *dst += s;
            }
            __syncthreads();
        }
    }
    cp_wait<0>();
}

// ---------------------------------------------------------------------------------------------
// Fused inference on the fifth-generation tensor cores (tcgen05). A CTA of 8 warps takes 128 rows
// (the MMA's M) through all five layers: one thread issues tcgen05.mma (BF16 operands from shared
// memory through matrix descriptors, FP32 accumulators in tensor memory, 128 x 256 per layer), the
// layer's weights arrive by one TMA bulk copy into shared memory while the previous layer's
// epilogue runs, and the epilogue (tcgen05.ld, bias, GELU, BF16) writes the next layer's A operand
// back into shared memory. Operands use the canonical K-major layout without swizzle: 8-row x
// 16-byte core matrices, adjacent along K 128 bytes apart (LBO), 8-row groups K/8 * 128 bytes
// apart (SBO). Every wait on an mbarrier is bounded by %globaltimer.

constexpr int UM_THREADS = 512;
// Warps share a lane quarter of tensor memory (a warp reads only its quarter's 32 rows): UM_GROUPS
// warps a quarter, each taking UM_GROUP_COLS of a hidden layer's 256 columns in the epilogue.
constexpr int UM_GROUPS = UM_THREADS / 128;
constexpr int UM_GROUP_COLS = 256 / UM_GROUPS;
constexpr int UM_A_BYTES = 128 * 256 * 2;   // layer input, 128 rows x 256
constexpr int UM_B_BYTES = 256 * 256 * 2;   // one layer's weights
constexpr int UM_X_BYTES = 128 * MLP_IN * 2; // feature rows as they arrive (row-major)
constexpr int UM_BIAS_FLOATS = 4 * 256 + 16;
constexpr size_t UM_SMEM = UM_A_BYTES + UM_B_BYTES + UM_X_BYTES + UM_BIAS_FLOATS * 4 + 64;
constexpr int UM_TMEM_COLS = 256;
static_assert(UM_SMEM <= 227 * 1024, "shared memory");

// Rows and columns of layer l's B operand as packed (the output layer padded to 16 rows).
__host__ __device__ constexpr int um_n(int l) { return l == MLP_LAYERS - 1 ? 16 : MLP_HID; }
__host__ __device__ constexpr int um_k(int l) { return mlp_dim(l); }
__host__ __device__ constexpr size_t um_w_offset(int l) {  // bytes
    size_t o = 0;
    for (int k = 0; k < l; ++k) o += (size_t)um_n(k) * um_k(k) * 2;
    return o;
}
constexpr size_t UM_W_BYTES = um_w_offset(MLP_LAYERS);

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of tcgen05; base offset 0, no swizzle
    return d;
}
// kind::f16 instruction descriptor: FP32 accumulate, BF16 A and B, both K-major, N and M.
__host__ __device__ constexpr uint32_t umma_idesc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void async_proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void um_mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void um_bulk(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// Waits for the barrier's phase for at most about a second (qm_stage.cuh); false when it gave up.
__device__ __forceinline__ bool um_wait(uint64_t *bar, unsigned phase) { return mbar_wait(bar, phase); }

// Packs the BF16 matrices into the tcgen05 operand layout (output layer padded to 16 rows).
__global__ void pack_umma_kernel(const __nv_bfloat16 *w16, __nv_bfloat16 *packed) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= UM_W_BYTES / 2) return;
    int l = 0;
    while (l < MLP_LAYERS - 1 && i >= um_w_offset(l + 1) / 2) ++l;
    const size_t e = i - um_w_offset(l) / 2;
    const int K = um_k(l), sbo = K / 8 * 64;  // in elements
    const int n = (int)(e / K), k = (int)(e % K);
    const size_t dst = um_w_offset(l) / 2 + (size_t)(n / 8) * sbo + (k / 8) * 64 + (n % 8) * 8 + (k % 8);
    packed[dst] = n < mlp_dim(l + 1) ? w16[mlp_w16_offset(l) + (size_t)n * K + k] : __float2bfloat16(0.0f);
}

struct UmmaArgs {
    const __nv_bfloat16 *wpack;  // [UM_W_BYTES] packed matrices
    const float *master;
    float out_shift[MLP_OUT], out_scale[MLP_OUT], lab_lo[MLP_OUT], lab_hi[MLP_OUT];
    const __nv_bfloat16 *x;
    size_t rows;
    float *out;
    MlpPaintArgs p;
    unsigned *error;
};

template <int MODE>
__global__ void __launch_bounds__(UM_THREADS, 1) mlp_umma_kernel(UmmaArgs A) {
    extern __shared__ __align__(1024) unsigned char um_smem[];
    unsigned char *sA = um_smem;
    unsigned char *sB = sA + UM_A_BYTES;
    unsigned char *sX = sB + UM_B_BYTES;
    float *sBias = reinterpret_cast<float *>(sX + UM_X_BYTES);
    uint64_t *bars = reinterpret_cast<uint64_t *>(sBias + UM_BIAS_FLOATS);  // w, x, mma
    uint32_t *sTmem = reinterpret_cast<uint32_t *>(bars + 3);
    __shared__ float s_red[4][9];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const size_t n_tiles = (A.rows + 127) / 128;
    if (blockIdx.x >= n_tiles) return;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(sTmem)),
                     "r"(UM_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        um_mbar_init(&bars[0], 1);
        um_mbar_init(&bars[1], 1);
        um_mbar_init(&bars[2], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = tid; i < UM_BIAS_FLOATS; i += UM_THREADS) {
        int l = i / 256, c = i % 256;
        float v = 0.0f;
        if (l < 4) v = A.master[mlp_b_offset(l) + c];
        else if (c < MLP_OUT) v = A.master[mlp_b_offset(4) + c];
        sBias[i] = v;
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem = *sTmem;
    unsigned pw = 0, px = 0, pm = 0;
    bool ok = true;
    auto x_bytes = [&](size_t tile) { return (unsigned)(min((size_t)128, A.rows - tile * 128) * MLP_IN * 2); };
    if (tid == 0) {
        um_bulk(sB, A.wpack, (unsigned)(um_n(0) * um_k(0) * 2), &bars[0]);
        um_bulk(sX, A.x + blockIdx.x * 128 * MLP_IN, x_bytes(blockIdx.x), &bars[1]);
    }
    const int lq = warp & 3, ch = warp >> 2;  // TMEM lane quarter and column group of this warp
    const int row = 32 * lq + lane;            // this thread's row of the tile
    for (size_t tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x) {
        const bool has_next = tile + gridDim.x < n_tiles;
        const size_t r_global = tile * 128 + row;
        const int rows_here = (int)min((size_t)128, A.rows - tile * 128);
        ok = __syncthreads_and(um_wait(&bars[1], px));
        px ^= 1;
        if (!ok) break;
        // Feature rows (row-major, 64 B) into the A layout (K = 32: SBO 512 B); missing rows zero.
        if (tid < 128) {
            const uint4 *src = reinterpret_cast<const uint4 *>(sX + tid * 64);
            for (int q = 0; q < 4; ++q) {
                uint4 v = tid < rows_here ? src[q] : make_uint4(0, 0, 0, 0);
                *reinterpret_cast<uint4 *>(sA + (tid / 8) * 512 + q * 128 + (tid % 8) * 16) = v;
            }
        }
        async_proxy_fence();
        __syncthreads();
        if (tid == 0 && has_next) um_bulk(sX, A.x + (tile + gridDim.x) * 128 * MLP_IN, x_bytes(tile + gridDim.x), &bars[1]);
        for (int l = 0; l < MLP_LAYERS && ok; ++l) {
            ok = __syncthreads_and(um_wait(&bars[0], pw));
            pw ^= 1;
            if (!ok) break;
            const int K = um_k(l), N = um_n(l);
            if (tid == 0) {
                tc_after_sync();
                const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
                const uint32_t sbo = (uint32_t)(K / 8 * 128);
                for (int s = 0; s < K / 16; ++s)
                    umma_bf16(tmem, umma_desc(a0 + 256 * s, 128, sbo), umma_desc(b0 + 256 * s, 128, sbo),
                              umma_idesc(128, N), s > 0 ? 1u : 0u);
                umma_commit(&bars[2]);
            }
            ok = __syncthreads_and(um_wait(&bars[2], pm));
            pm ^= 1;
            if (!ok) break;
            tc_after_sync();
            // The weights are consumed: fetch the next layer's (or the next tile's first).
            if (tid == 0 && (l + 1 < MLP_LAYERS || has_next)) {
                const int nl = (l + 1) % MLP_LAYERS;
                um_bulk(sB, reinterpret_cast<const unsigned char *>(A.wpack) + um_w_offset(nl),
                        (unsigned)(um_n(nl) * um_k(nl) * 2), &bars[0]);
            }
            const uint32_t t_row = tmem + ((uint32_t)(32 * lq) << 16);
            if (l < MLP_LAYERS - 1) {
                // Hidden epilogue: this warp's UM_GROUP_COLS columns of its 32 rows -> GELU -> BF16 A layout (K = 256).
                const float *bias = sBias + l * 256;
                for (int c = 0; c < UM_GROUP_COLS / 16; ++c) {
                    const int col = UM_GROUP_COLS * ch + 16 * c;
                    float v[16];
                    tmem_ld16(t_row + col, v);
                    uint32_t pk[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        __nv_bfloat162 h = __floats2bfloat162_rn(gelu(v[2 * q] + bias[col + 2 * q]),
                                                                 gelu(v[2 * q + 1] + bias[col + 2 * q + 1]));
                        pk[q] = *reinterpret_cast<uint32_t *>(&h);
                    }
                    unsigned char *dst = sA + (row / 8) * 4096 + (col / 8) * 128 + (row % 8) * 16;
                    *reinterpret_cast<uint4 *>(dst) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                    *reinterpret_cast<uint4 *>(dst + 128) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
                }
                async_proxy_fence();
                tc_before_sync();
                __syncthreads();
            } else {
                // Output epilogue: warps 0..3, one row each thread.
                float y[MLP_OUT];
                bool use = false, bad = false;
                if (ch == 0) {
                    float v[16];
                    tmem_ld16(t_row, v);
#pragma unroll
                    for (int o = 0; o < MLP_OUT; ++o) {
                        y[o] = (v[o] + sBias[4 * 256 + o]) * A.out_scale[o] + A.out_shift[o];
                        bad = bad || !(y[o] >= A.lab_lo[o] - 1.0f && y[o] <= A.lab_hi[o] + 1.0f);
                    }
                }
                if (MODE == 0) {
                    if (ch == 0 && r_global < A.rows) {
                        float4 *o4 = reinterpret_cast<float4 *>(A.out + r_global * MLP_OUT);
                        o4[0] = make_float4(y[0], y[1], y[2], y[3]);
                        o4[1] = make_float4(y[4], y[5], y[6], y[7]);
                    }
                } else {
                    const MlpPaintArgs &P = A.p;
                    float e[9];
#pragma unroll
                    for (int k = 0; k < 9; ++k) e[k] = 0.0f;
                    if (ch == 0) {
                        use = r_global < A.rows && P.eligible[r_global] != 0;
                        // A path whose row (or, with two rows a path, either row) leaves the label
                        // range goes to the exact re-run once, and none of its rows is used.
                        bool drop = use && bad;
                        if (P.rows_per_path == 2) {
                            // Every lane takes part in the shuffle (no short-circuit around it).
                            const bool partner = __shfl_xor_sync(0xffffffffu, drop, 1) != 0;
                            drop = drop || partner;
                        }
                        if (drop) {
                            if (P.rows_per_path == 1 || (lane & 1) == 0) {
                                uint32_t cell = (uint32_t)(r_global / P.rows_per_cell),
                                         s = (uint32_t)((r_global % P.rows_per_cell) / P.rows_per_path);
                                unsigned slot = atomicAdd(P.retry_count, 1u);
                                if (slot < P.retry_cap) P.retry[slot] = make_uint2(cell, P.source_begin + s);
                            }
                            use = false;
                        }
                    }
                    if (ch == 0 && use) {
                        {
                            const float4 *cf = reinterpret_cast<const float4 *>(P.coef + r_global * 16);
                            float c[16];
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                float4 f = __ldg(cf + q);
                                c[4 * q] = f.x;
                                c[4 * q + 1] = f.y;
                                c[4 * q + 2] = f.z;
                                c[4 * q + 3] = f.w;
                            }
#pragma unroll
                            for (int o = 0; o < MLP_OUT; ++o) {
                                float en = exp2f(-y[o] * 0.33219280948873623f);
                                e[o] = c[o] * en;
                                e[8] += c[8 + o] * en;
                            }
                        }
                    }
                    if (ch == 0) {
                        unsigned taken = __popc(__ballot_sync(0xffffffffu, use && (P.rows_per_path == 1 || (lane & 1) == 0)));
                        if (lane == 0 && taken) atomicAdd(P.taken, (unsigned long long)taken);
#pragma unroll
                        for (int k = 0; k < 9; ++k) {
                            float sum = e[k];
#pragma unroll
                            for (int m = 16; m > 0; m >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, m);
                            if (lane == 0) s_red[lq][k] = sum;
                        }
                    }
                    __syncthreads();
                    if (tid < 9) {
                        float sum = s_red[0][tid] + s_red[1][tid] + s_red[2][tid] + s_red[3][tid];
                        const size_t row0 = tile * 128;
                        const size_t cell = row0 / P.rows_per_cell, slice = (row0 % P.rows_per_cell) / 128;
                        P.partial[(slice * (size_t)P.cells + cell) * 9 + tid] += sum;
                    }
                }
                tc_before_sync();
                __syncthreads();
            }
        }
    }
    if (!ok && tid == 0) atomicOr(A.error, 1u);
    tc_after_sync();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(UM_TMEM_COLS) : "memory");
}

// ---------------------------------------------------------------------------------------------
// Training product: C[M][N] (op) A(m, k) * B(k, n), BF16 operands, FP32 accumulation, on the
// fifth-generation tensor cores. A is stored [M][K] (A_MK) or [K][M]; B is stored [N][K] (B_NK) or
// [K][N]. A CTA computes a 128 x 128 tile of C over its share of K (split-K over blockIdx.z): the
// threads stage each 64-wide K chunk of both operands into shared memory in the canonical K-major
// layout (transposing an operand stored [K][...] on the way), one thread issues the chunk's
// `tcgen05.mma` (M 128, N 128, K 16) into 128 tensor-memory columns and commits them to the
// chunk's mbarrier, and the next chunk is staged into the other buffer meanwhile. The epilogue reads
// the accumulators with `tcgen05.ld` and applies the layer's bias, GELU or GELU gradient.

enum { EPI_STORE = 0, EPI_ATOMIC = 1, EPI_BIAS_GELU = 2, EPI_BIAS = 3, EPI_GELU_GRAD = 4 };

struct GemmArgs {
    const __nv_bfloat16 *a, *b;
    int M, N, K;       // each a multiple of 8
    int lda, ldb;      // row strides of the stored matrices (multiples of 8)
    int k_per_split;   // multiple of GT_KC
    float *c;          // [M][N] FP32 (EPI_STORE, EPI_ATOMIC, EPI_BIAS: output; EPI_BIAS_GELU: Z)
    const float *bias; // [N]
    __nv_bfloat16 *h;  // [M][N] BF16 (EPI_BIAS_GELU: GELU(Z); EPI_GELU_GRAD: dZ of the layer below)
    const float *z;    // [M][N] (EPI_GELU_GRAD: the layer below's pre-activation)
    unsigned *error;   // set when a bounded wait gave up
};

constexpr int GT_M = 128, GT_N = 128, GT_KC = 64;
constexpr int GT_TILE_BYTES = 128 * GT_KC * 2;      // one operand's chunk: 16 KB
constexpr int GT_SBO = GT_KC / 8 * 128;             // bytes between 8-row groups of a chunk
constexpr int GT_TILE_STRIDE = 128 + 1;              // floats a row of the epilogue's accumulator tile
constexpr size_t GT_EPI_BYTES = 128 * GT_TILE_STRIDE * 4;
// Two buffers of A and B (reused by the epilogue's accumulator tile), then two barriers and the
// tensor-memory address.
constexpr size_t GT_DATA_BYTES = GT_EPI_BYTES > 4 * GT_TILE_BYTES ? GT_EPI_BYTES : 4 * GT_TILE_BYTES;
constexpr size_t GT_SMEM = (GT_DATA_BYTES + 15) / 16 * 16 + 64;
constexpr int GT_TMEM_COLS = 128;

// One operand's chunk [kb, kb + GT_KC) of rows [r0, r0 + 128): each thread loads 4 groups of 8
// elements into registers (rows at or past `rows` and columns at or past `k_end` read zero), then
// stores them in the canonical K-major layout without swizzle: element (row, k) at
// (row / 8) * GT_SBO + (k / 8) * 128 + (row % 8) * 16 + (k % 8) * 2.
template <bool ROW_K>
__device__ __forceinline__ void load_operand(uint4 (&r)[4], const __nv_bfloat16 *src, int ld, int r0, int rows, int kb,
                                             int k_end, int tid) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int v = tid + 256 * i;  // 1024 groups of 8 elements
        if (ROW_K) {
            // Stored [row][k]: a group is 8 consecutive k of one row.
            const int row = v >> 3, k = kb + 8 * (v & 7);
            const bool ok = r0 + row < rows && k < k_end;
            r[i] = ok ? *reinterpret_cast<const uint4 *>(src + (size_t)(r0 + row) * ld + k) : make_uint4(0, 0, 0, 0);
        } else {
            // Stored [k][row]: a group is 8 consecutive rows at one k.
            const int row = 8 * (v >> 6), k = kb + (v & 63);
            const bool ok = r0 + row < rows && k < k_end;
            r[i] = ok ? *reinterpret_cast<const uint4 *>(src + (size_t)k * ld + r0 + row) : make_uint4(0, 0, 0, 0);
        }
    }
}

template <bool ROW_K>
__device__ __forceinline__ void store_operand(unsigned char *dst, const uint4 (&r)[4], int tid) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int v = tid + 256 * i;
        if (ROW_K) {
            const int row = v >> 3, k8 = v & 7;
            *reinterpret_cast<uint4 *>(dst + (row >> 3) * GT_SBO + k8 * 128 + (row & 7) * 16) = r[i];
        } else {
            // The group's 8 rows scattered to their places at column k.
            const int rg = v >> 6, kl = v & 63;
            const __nv_bfloat16 *e = reinterpret_cast<const __nv_bfloat16 *>(&r[i]);
            unsigned char *base = dst + rg * GT_SBO + (kl >> 3) * 128 + (kl & 7) * 2;
#pragma unroll
            for (int q = 0; q < 8; ++q) *reinterpret_cast<__nv_bfloat16 *>(base + q * 16) = e[q];
        }
    }
}

template <bool A_MK, bool B_NK, int EPI>
__global__ void __launch_bounds__(256) gemm_kernel(GemmArgs G) {
    extern __shared__ __align__(1024) unsigned char gt_smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(gt_smem + (GT_DATA_BYTES + 15) / 16 * 16);
    uint32_t *sTmem = reinterpret_cast<uint32_t *>(bars + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * GT_M, n0 = blockIdx.x * GT_N;
    const int k_begin = blockIdx.z * G.k_per_split;
    const int k_end = min(G.K, k_begin + G.k_per_split);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(sTmem)),
                     "r"(GT_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        um_mbar_init(&bars[0], 1);
        um_mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem = *sTmem;
    unsigned phases = 0u;  // bit b: the parity buffer b's barrier completes next
    bool ok = true;
    int chunk = 0;
    // Each chunk's operands are loaded into registers one chunk ahead, while the tensor cores work
    // on the chunk before.
    uint4 ra[4], rb[4];
    if (k_begin < k_end) {
        load_operand<A_MK>(ra, G.a, G.lda, m0, G.M, k_begin, k_end, tid);
        load_operand<B_NK>(rb, G.b, G.ldb, n0, G.N, k_begin, k_end, tid);
    }
    for (int kb = k_begin; kb < k_end && ok; kb += GT_KC, ++chunk) {
        const int b = chunk & 1;
        if (chunk >= 2) {
            // The MMAs that read this buffer two chunks ago must be done before it is refilled.
            ok = __syncthreads_and(um_wait(&bars[b], (phases >> b) & 1u));
            phases ^= 1u << b;
            if (!ok) break;
        }
        unsigned char *sA = gt_smem + b * GT_TILE_BYTES, *sB = gt_smem + (2 + b) * GT_TILE_BYTES;
        store_operand<A_MK>(sA, ra, tid);
        store_operand<B_NK>(sB, rb, tid);
        async_proxy_fence();
        __syncthreads();
        if (kb + GT_KC < k_end) {
            load_operand<A_MK>(ra, G.a, G.lda, m0, G.M, kb + GT_KC, k_end, tid);
            load_operand<B_NK>(rb, G.b, G.ldb, n0, G.N, kb + GT_KC, k_end, tid);
        }
        if (tid == 0) {
            tc_after_sync();
            const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
            for (int s = 0; s < GT_KC / 16; ++s)
                umma_bf16(tmem, umma_desc(a0 + 256 * s, 128, GT_SBO), umma_desc(b0 + 256 * s, 128, GT_SBO),
                          umma_idesc(GT_M, GT_N), (chunk > 0 || s > 0) ? 1u : 0u);
            umma_commit(&bars[b]);
        }
    }
    // The last commit tracks every MMA this thread issued before it.
    if (ok && chunk > 0) {
        const int b = (chunk - 1) & 1;
        ok = __syncthreads_and(um_wait(&bars[b], (phases >> b) & 1u));
    }
    tc_after_sync();
    if (ok && chunk > 0) {
        // The accumulators through shared memory (the operand buffers are free now): each lane holds
        // a row of tensor memory, and rows written straight to global memory would scatter.
        float *tile = reinterpret_cast<float *>(gt_smem);  // [128][GT_TILE_STRIDE]
        const int lq = warp & 3, ch = warp >> 2;           // TMEM lane quarter and column half
        const int row = 32 * lq + lane;
        const uint32_t t_row = tmem + ((uint32_t)(32 * lq) << 16);
        for (int c = 0; c < 4; ++c) {
            const int col = 64 * ch + 16 * c;
            float v[16];
            tmem_ld16(t_row + col, v);
#pragma unroll
            for (int j = 0; j < 16; ++j) tile[row * GT_TILE_STRIDE + col + j] = v[j];
        }
        __syncthreads();
        // Then by pairs of columns along rows, a warp writing 64 consecutive columns of one row.
        for (int p = tid; p < 128 * 64; p += 256) {
            const int r = p >> 6, cp = 2 * (p & 63);
            const int m = m0 + r, n = n0 + cp;
            if (m >= G.M || n >= G.N) continue;
            float v0 = tile[r * GT_TILE_STRIDE + cp], v1 = tile[r * GT_TILE_STRIDE + cp + 1];
            const size_t idx = (size_t)m * G.N + n;
            if (EPI == EPI_STORE) {
                *reinterpret_cast<float2 *>(G.c + idx) = make_float2(v0, v1);
            } else if (EPI == EPI_ATOMIC) {
                atomicAdd(G.c + idx, v0);
                atomicAdd(G.c + idx + 1, v1);
            } else if (EPI == EPI_BIAS || EPI == EPI_BIAS_GELU) {
                v0 += G.bias[n];
                v1 += G.bias[n + 1];
                *reinterpret_cast<float2 *>(G.c + idx) = make_float2(v0, v1);
                if (EPI == EPI_BIAS_GELU)
                    *reinterpret_cast<uint32_t *>(G.h + idx) = pack_bf16(gelu(v0), gelu(v1));
            } else {  // EPI_GELU_GRAD
                const float2 z = *reinterpret_cast<const float2 *>(G.z + idx);
                *reinterpret_cast<uint32_t *>(G.h + idx) = pack_bf16(v0 * gelu_grad(z.x), v1 * gelu_grad(z.y));
            }
        }
    }
    if (!ok && tid == 0 && G.error) atomicOr(G.error, 1u);
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(GT_TMEM_COLS) : "memory");
}

template <bool A_MK, bool B_NK, int EPI>
cudaError_t gemm(const GemmArgs &g, int splits, cudaStream_t stream) {
    if (g.M % 8 || g.N % 8 || g.K % 8 || g.lda % 8 || g.ldb % 8) return cudaErrorInvalidValue;
    // Set on every call: the attribute belongs to the current device.
    cudaError_t e = cudaFuncSetAttribute(gemm_kernel<A_MK, B_NK, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)GT_SMEM);
    if (e != cudaSuccess) return e;
    GemmArgs a = g;
    int k_chunks = (g.K + GT_KC - 1) / GT_KC;
    splits = std::max(1, std::min(splits, k_chunks));
    a.k_per_split = ((k_chunks + splits - 1) / splits) * GT_KC;
    splits = (g.K + a.k_per_split - 1) / a.k_per_split;
    dim3 grid((g.N + GT_N - 1) / GT_N, (g.M + GT_M - 1) / GT_M, splits);
    gemm_kernel<A_MK, B_NK, EPI><<<grid, 256, GT_SMEM, stream>>>(a);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// Element-wise kernels.

__global__ void cast_kernel(const float *master, __nv_bfloat16 *w16) {
    // Matrices only: layer l's [out][in] block of the master vector -> its BF16 block.
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= MLP_W16) return;
    int l = 0;
    size_t base16 = 0, base32 = 0;
    for (; l < MLP_LAYERS; ++l) {
        size_t n = (size_t)mlp_dim(l + 1) * mlp_dim(l);
        if (i < base16 + n) break;
        base16 += n;
        base32 += n + mlp_dim(l + 1);
    }
    w16[i] = __float2bfloat16_rn(master[base32 + (i - base16)]);
}

__global__ void normalise_kernel(MlpScales s, const float *raw, size_t n, __nv_bfloat16 *out) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n * MLP_IN) return;
    int f = (int)(i % MLP_IN);
    out[i] = __float2bfloat16_rn((raw[i] - s.in_shift[f]) * s.in_scale[f]);
}

// MSE on n rows of 8: dOut = 2 (out - y) / (8 n) as BF16; the loss summed into *loss.
__global__ void loss_kernel(const float *out, const float *y, size_t n, __nv_bfloat16 *dout, double *loss) {
    __shared__ float s[256];
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    float e2 = 0.0f;
    if (i < n * MLP_OUT) {
        float d = out[i] - y[i];
        e2 = d * d;
        dout[i] = __float2bfloat16_rn(2.0f * d / (float)(n * MLP_OUT));
    }
    s[threadIdx.x] = e2;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
        if (threadIdx.x < k) s[threadIdx.x] += s[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss, (double)s[0] / (double)(n * MLP_OUT));
}

// Column sums of a BF16 matrix [n][w] into db (added).
__global__ void bias_grad_kernel(const __nv_bfloat16 *dz, size_t n, int w, float *db) {
    int col = blockIdx.x * 32 + (threadIdx.x & 31);
    int lane_row = threadIdx.x >> 5;  // 8 row lanes
    float s = 0.0f;
    if (col < w)
        for (size_t r = blockIdx.y * 8 + lane_row; r < n; r += 8 * gridDim.y) s += __bfloat162float(dz[r * w + col]);
    __shared__ float red[8][33];
    red[lane_row][threadIdx.x & 31] = s;
    __syncthreads();
    if (threadIdx.x < 32 && col < w) {
        float t = 0.0f;
        for (int k = 0; k < 8; ++k) t += red[k][threadIdx.x];
        atomicAdd(db + col, t);
    }
}

__global__ void adam_kernel(float *p, const float *g, float *m, float *v, size_t n, float lr, float c1, float c2) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    float gi = g[i];
    float mi = b1 * m[i] + (1.0f - b1) * gi;
    float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
}

__global__ void gather_kernel(const __nv_bfloat16 *x, const float *y, const uint32_t *index, size_t n,
                              __nv_bfloat16 *bx, float *by) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    size_t r = index[i];
    const uint4 *src = reinterpret_cast<const uint4 *>(x + r * MLP_IN);
    uint4 *dst = reinterpret_cast<uint4 *>(bx + i * MLP_IN);
#pragma unroll
    for (int k = 0; k < 4; ++k) dst[k] = src[k];
    const float4 *ys = reinterpret_cast<const float4 *>(y + r * MLP_OUT);
    float4 *yd = reinterpret_cast<float4 *>(by + i * MLP_OUT);
    yd[0] = ys[0];
    yd[1] = ys[1];
}

__device__ __forceinline__ void atomic_min_f(float *a, float v) {
    int *ai = reinterpret_cast<int *>(a);
    int old = *ai;
    while (__int_as_float(old) > v) {
        int prev = atomicCAS(ai, old, __float_as_int(v));
        if (prev == old) break;
        old = prev;
    }
}
__device__ __forceinline__ void atomic_max_f(float *a, float v) {
    int *ai = reinterpret_cast<int *>(a);
    int old = *ai;
    while (__int_as_float(old) < v) {
        int prev = atomicCAS(ai, old, __float_as_int(v));
        if (prev == old) break;
        old = prev;
    }
}

// One thread per (row block, column): sums over its rows, then one atomic each.
__global__ void stats_kernel(const float *rows, const uint8_t *keep, size_t n, int w, double *sum, double *sumsq,
                             float *lo, float *hi) {
    int col = threadIdx.x % w;
    int lanes = blockDim.x / w;
    int sub = threadIdx.x / w;
    if (sub >= lanes) return;
    double s = 0.0, s2 = 0.0;
    float mn = INFINITY, mx = -INFINITY;
    for (size_t r = blockIdx.x * (size_t)lanes + sub; r < n; r += (size_t)gridDim.x * lanes) {
        if (keep && !keep[r]) continue;
        float v = rows[r * w + col];
        s += v;
        s2 += (double)v * v;
        mn = fminf(mn, v);
        mx = fmaxf(mx, v);
    }
    atomicAdd(sum + col, s);
    atomicAdd(sumsq + col, s2);
    atomic_min_f(lo + col, mn);
    atomic_max_f(hi + col, mx);
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// Host side.

namespace {

cudaError_t set_umma_smem() {
    cudaError_t e = cudaFuncSetAttribute(mlp_umma_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)UM_SMEM);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(mlp_umma_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)UM_SMEM);
    return e;
}

UmmaArgs umma_args(const MlpDev &net) {
    UmmaArgs a{};
    a.wpack = net.wpack;
    a.master = net.master;
    for (int o = 0; o < MLP_OUT; ++o) {
        a.out_shift[o] = net.scales.out_shift[o];
        a.out_scale[o] = net.scales.out_scale[o];
        a.lab_lo[o] = net.scales.lab_lo[o];
        a.lab_hi[o] = net.scales.lab_hi[o];
    }
    a.error = net.error;
    return a;
}

cudaError_t set_fused_smem() {
    const int smem = 2 * CH_ELEMS * (int)sizeof(__nv_bfloat16);
    cudaError_t e = cudaFuncSetAttribute(mlp_fused_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(mlp_fused_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    return e;
}

FusedArgs fused_args(const MlpDev &net) {
    FusedArgs a{};
    a.w16 = net.w16;
    a.master = net.master;
    for (int o = 0; o < MLP_OUT; ++o) {
        a.out_shift[o] = net.scales.out_shift[o];
        a.out_scale[o] = net.scales.out_scale[o];
        a.lab_lo[o] = net.scales.lab_lo[o];
        a.lab_hi[o] = net.scales.lab_hi[o];
    }
    return a;
}

unsigned fused_grid(size_t rows) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    size_t tiles = (rows + FT_ROWS - 1) / FT_ROWS;
    return (unsigned)std::max<size_t>(1, std::min<size_t>(tiles, (size_t)sms));
}

}  // namespace

size_t mlp_packed_bytes() { return UM_W_BYTES; }

cudaError_t mlp_cast(const MlpDev &net, cudaStream_t stream) {
    cast_kernel<<<(unsigned)((MLP_W16 + 255) / 256), 256, 0, stream>>>(net.master, net.w16);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || !net.wpack) return e;
    pack_umma_kernel<<<(unsigned)((UM_W_BYTES / 2 + 255) / 256), 256, 0, stream>>>(net.w16, net.wpack);
    return cudaGetLastError();
}

cudaError_t mlp_normalise(const MlpScales &s, const float *raw, size_t n, __nv_bfloat16 *out, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    size_t total = n * MLP_IN;
    normalise_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(s, raw, n, out);
    return cudaGetLastError();
}

cudaError_t mlp_forward(const MlpDev &net, const __nv_bfloat16 *x, size_t n, float *out, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    if (net.kernel == 0) {
        cudaError_t e = set_umma_smem();
        if (e != cudaSuccess) return e;
        UmmaArgs a = umma_args(net);
        a.x = x;
        a.rows = n;
        a.out = out;
        mlp_umma_kernel<0><<<fused_grid(n), UM_THREADS, UM_SMEM, stream>>>(a);
        return cudaGetLastError();
    }
    cudaError_t e = set_fused_smem();
    if (e != cudaSuccess) return e;
    FusedArgs a = fused_args(net);
    a.x = x;
    a.rows = n;
    a.out = out;
    mlp_fused_kernel<0><<<fused_grid(n), FT_THREADS, 2 * CH_ELEMS * sizeof(__nv_bfloat16), stream>>>(a);
    return cudaGetLastError();
}

cudaError_t mlp_paint(const MlpDev &net, const MlpPaintArgs &p, cudaStream_t stream) {
    if (p.rows == 0) return cudaSuccess;
    if (net.kernel == 0 || p.rows_per_path == 2) {  // the mma.sync kernel takes one row a path only
        cudaError_t e = set_umma_smem();
        if (e != cudaSuccess) return e;
        UmmaArgs a = umma_args(net);
        a.x = p.x;
        a.rows = p.rows;
        a.p = p;
        mlp_umma_kernel<1><<<fused_grid(p.rows), UM_THREADS, UM_SMEM, stream>>>(a);
        return cudaGetLastError();
    }
    cudaError_t e = set_fused_smem();
    if (e != cudaSuccess) return e;
    FusedArgs a = fused_args(net);
    a.x = p.x;
    a.rows = p.rows;
    a.p = p;
    mlp_fused_kernel<1><<<fused_grid(p.rows), FT_THREADS, 2 * CH_ELEMS * sizeof(__nv_bfloat16), stream>>>(a);
    return cudaGetLastError();
}

struct MlpWork {
    size_t max_rows = 0;
    float *z[MLP_LAYERS] = {};           // pre-activations (the last: the outputs)
    __nv_bfloat16 *h[MLP_LAYERS - 1] = {};  // GELU of the hidden pre-activations
    __nv_bfloat16 *dz[2] = {};
    __nv_bfloat16 *dout = nullptr;
};

MlpWork *mlp_work_create(size_t max_rows) {
    MlpWork *w = new MlpWork;
    w->max_rows = max_rows;
    bool ok = true;
    for (int l = 0; l < MLP_LAYERS; ++l) ok &= cudaMalloc(&w->z[l], max_rows * mlp_dim(l + 1) * sizeof(float)) == cudaSuccess;
    for (int l = 0; l < MLP_LAYERS - 1; ++l)
        ok &= cudaMalloc(&w->h[l], max_rows * MLP_HID * sizeof(__nv_bfloat16)) == cudaSuccess;
    for (int k = 0; k < 2; ++k) ok &= cudaMalloc(&w->dz[k], max_rows * MLP_HID * sizeof(__nv_bfloat16)) == cudaSuccess;
    ok &= cudaMalloc(&w->dout, max_rows * MLP_OUT * sizeof(__nv_bfloat16)) == cudaSuccess;
    if (!ok) {
        mlp_work_free(w);
        return nullptr;
    }
    return w;
}

void mlp_work_free(MlpWork *w) {
    if (!w) return;
    for (auto p : w->z) cudaFree(p);
    for (auto p : w->h) cudaFree(p);
    for (auto p : w->dz) cudaFree(p);
    cudaFree(w->dout);
    delete w;
}

cudaError_t mlp_gradients(const MlpDev &net, MlpWork *w, const __nv_bfloat16 *x, const float *y, size_t n,
                          float *grads, double *loss, cudaStream_t stream) {
    if (n == 0 || n > w->max_rows || n % 8 != 0) return cudaErrorInvalidValue;
    cudaError_t e;
    if ((e = cudaMemsetAsync(grads, 0, MLP_WEIGHTS * sizeof(float), stream)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(loss, 0, sizeof(double), stream)) != cudaSuccess) return e;
    const int M = (int)n;
    // Forward, keeping the pre-activations.
    const __nv_bfloat16 *in = x;
    for (int l = 0; l < MLP_LAYERS; ++l) {
        GemmArgs g{};
        g.a = in;
        g.lda = mlp_dim(l);
        g.b = net.w16 + mlp_w16_offset(l);
        g.ldb = mlp_dim(l);
        g.M = M;
        g.N = mlp_dim(l + 1);
        g.K = mlp_dim(l);
        g.c = w->z[l];
        g.bias = net.master + mlp_b_offset(l);
        g.error = net.error;
        if (l < MLP_LAYERS - 1) {
            g.h = w->h[l];
            e = gemm<true, true, EPI_BIAS_GELU>(g, 1, stream);
            in = w->h[l];
        } else {
            e = gemm<true, true, EPI_BIAS>(g, 1, stream);
        }
        if (e != cudaSuccess) return e;
    }
    size_t outs = n * MLP_OUT;
    loss_kernel<<<(unsigned)((outs + 255) / 256), 256, 0, stream>>>(w->z[MLP_LAYERS - 1], y, n, w->dout, loss);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    // Backward.
    const __nv_bfloat16 *dz = w->dout;
    int flip = 0;
    for (int l = MLP_LAYERS - 1; l >= 0; --l) {
        const int out_w = mlp_dim(l + 1), in_w = mlp_dim(l);
        const __nv_bfloat16 *layer_in = l > 0 ? w->h[l - 1] : x;
        GemmArgs g{};
        g.a = dz;
        g.lda = out_w;
        g.b = layer_in;
        g.ldb = in_w;
        g.M = out_w;
        g.N = in_w;
        g.K = M;
        g.c = grads + mlp_w_offset(l);
        g.error = net.error;
        int splits = std::max(1, std::min(128, M / 256));
        if ((e = gemm<false, false, EPI_ATOMIC>(g, splits, stream)) != cudaSuccess) return e;
        dim3 bg((out_w + 31) / 32, (unsigned)std::max<size_t>(1, std::min<size_t>(256, n / 64)));
        bias_grad_kernel<<<bg, 256, 0, stream>>>(dz, n, out_w, grads + mlp_b_offset(l));
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if (l > 0) {
            GemmArgs d{};
            d.a = dz;
            d.lda = out_w;
            d.b = net.w16 + mlp_w16_offset(l);
            d.ldb = in_w;
            d.M = M;
            d.N = in_w;
            d.K = out_w;
            d.z = w->z[l - 1];
            d.h = w->dz[flip];
            d.error = net.error;
            if ((e = gemm<true, false, EPI_GELU_GRAD>(d, 1, stream)) != cudaSuccess) return e;
            dz = w->dz[flip];
            flip ^= 1;
        }
    }
    return cudaSuccess;
}

cudaError_t mlp_adam(MlpDev &net, const float *grads, float lr, int step, cudaStream_t stream) {
    float c1 = 1.0f / (1.0f - std::pow(0.9f, (float)step)), c2 = 1.0f / (1.0f - std::pow(0.999f, (float)step));
    adam_kernel<<<(unsigned)((MLP_WEIGHTS + 255) / 256), 256, 0, stream>>>(net.master, grads, net.adam_m, net.adam_v,
                                                                          MLP_WEIGHTS, lr, c1, c2);
    cudaError_t e = cudaGetLastError();
    return e != cudaSuccess ? e : mlp_cast(net, stream);
}

cudaError_t mlp_gather(const __nv_bfloat16 *x, const float *y, const uint32_t *index, size_t n, __nv_bfloat16 *bx,
                       float *by, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    gather_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(x, y, index, n, bx, by);
    return cudaGetLastError();
}

cudaError_t mlp_column_stats(const float *rows, const uint8_t *keep, size_t n, int w, double *sum, double *sumsq,
                             float *lo, float *hi, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    int lanes = 256 / w;
    unsigned blocks = (unsigned)std::max<size_t>(1, std::min<size_t>(1184, (n + lanes - 1) / lanes));
    stats_kernel<<<blocks, lanes * w, 0, stream>>>(rows, keep, n, w, sum, sumsq, lo, hi);
    return cudaGetLastError();
}

}  // namespace qm
