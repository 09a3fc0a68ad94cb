// surrogate_fused.cuh -- the calibration surrogate's whole inference pass
// (4 -> 256 -> 256 -> 256 -> 3, GELU, BF16 weights and activations, FP32
// accumulation) in one persistent kernel.
//
// One CTA of 512 threads per SM walks tiles of 128 samples. A tile's
// activations never leave the SM:
//   layer 1 (K = 4, too short for the tensor cores): CUDA cores, from the raw
//     inputs normalised as the unfused path does, written as BF16 into the
//     activation tile in shared memory (the UMMA K-major canonical layout);
//   layers 2 and 3: tcgen05.mma (M = 128, N = 128, K = 16 steps) from the
//     activation tile and a weight half (128 output features x 256 inputs),
//     accumulating in tensor memory (128 lanes x 256 FP32 columns); the
//     epilogue reads it back with tcgen05.ld, adds the bias, applies GELU and
//     writes the BF16 activations over the tile they came from;
//   layer 4 (N = 3): folded into layer 3's epilogue, each thread summing its
//     row's products over its 64 columns, the four parts of a row added in a
//     fixed order.
// The four weight halves of a tile (64 KB each, two of layer 2, two of layer
// 3) stream from L2 into two shared buffers with cp.async while the other
// buffer's MMAs or an epilogue run: a layer's halves are loaded while the
// previous layer's epilogue (or the previous tile's) works.
// Shared memory: activation tile 64 KB + two weight buffers 128 KB, plus the
// small tables (W1, biases, W4) -- one CTA per SM.
// Every mbarrier wait is bounded: a wait that runs out sets the error word,
// the CTA stops issuing work, and tensor memory is released.
#pragma once
#include "surrogate_gemm.cuh"

namespace surrogate {

constexpr int FUSED_THREADS = 512;   // 16 warps: 4 per tensor-memory lane quarter
constexpr int FUSED_TILE = 128;       // samples per tile (UMMA M)
constexpr int FUSED_NH = 256;         // hidden width
constexpr int FUSED_HALF = 128;       // output features per weight half (UMMA N)
constexpr int FUSED_CHUNK = 16384;    // one 64-wide K chunk of a 128-row operand
constexpr int FUSED_OPERAND = 4 * FUSED_CHUNK; // 128 rows x 256 K in BF16 = 64 KB
constexpr int FUSED_SMEM = 3 * FUSED_OPERAND + 1024; // + alignment slack

struct FusedArgs {
    const float* x;            // raw inputs [n][4]
    const float* norm;         // in_mean[4], in_std[4], ...
    const __nv_bfloat16* wb;   // the parameter vector in BF16
    const float* p;            // the parameter vector in FP32 (biases)
    long long off_w1, off_b1, off_w2, off_b2, off_w3, off_b3, off_w4, off_b4;
    int n;
    float* y;                  // normalised outputs [n][3]
    unsigned int* error;
};

// byte offset of element (row, k) of a 128-row K-major operand (no swizzle:
// 8 x 16-byte core matrices; 1024 B between 8-row groups, 128 B between
// 8-wide K groups, 16 KB per 64-wide K chunk)
__device__ __forceinline__ int fused_at(int row, int k)
{
    return (k >> 6) * FUSED_CHUNK + (row >> 3) * 1024 + ((k & 63) >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

// rows [half * 128, half * 128 + 128) of a 256 x 256 weight matrix (output
// feature x input) into a weight buffer, 16 bytes per cp.async
__device__ __forceinline__ void fused_load_half(unsigned char* dst, const __nv_bfloat16* w, int half)
{
    for (int it = threadIdx.x; it < FUSED_HALF * (FUSED_NH / 8); it += FUSED_THREADS) {
        const int r = it >> 5, g = it & 31; // row, 8-wide K group
        const __nv_bfloat16* src = w + (long long)(half * FUSED_HALF + r) * FUSED_NH + g * 8;
        const uint32_t d = smem_u32(dst + fused_at(r, g * 8));
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
    }
}

// one layer's MMAs: both output halves over K = 256, then one commit
__device__ __forceinline__ void fused_mma_layer(uint32_t tmem, const unsigned char* sA, unsigned char* const sW[2],
                                                uint64_t* bar)
{
    constexpr uint32_t idesc = umma_idesc_bf16(FUSED_HALF);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int s = 0; s < FUSED_NH / 16; ++s) {
            const uint32_t off = (uint32_t)((s >> 2) * FUSED_CHUNK + (s & 3) * 256);
            const uint64_t ad = umma_desc(smem_u32(sA) + off, 128, 1024);
            const uint64_t bd = umma_desc(smem_u32(sW[h]) + off, 128, 1024);
            umma_bf16(tmem + (uint32_t)(h * FUSED_HALF), ad, bd, idesc, s > 0 ? 1u : 0u);
        }
    umma_commit(bar);
}

// 8 consecutive BF16 values (rounded to nearest, two per conversion) as one 16-byte word
__device__ __forceinline__ uint4 fused_pack8(const float* f)
{
    uint32_t w[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(f[2 * j], f[2 * j + 1]);
        w[j] = *reinterpret_cast<const uint32_t*>(&h);
    }
    return make_uint4(w[0], w[1], w[2], w[3]);
}

__global__ void __launch_bounds__(FUSED_THREADS, 1) k_mlp_forward_fused(FusedArgs a)
{
    extern __shared__ unsigned char smem_raw[];
    __shared__ float4 w1s[FUSED_NH];               // layer 1: the 4 weights of each feature
    __shared__ __align__(16) float b1s[FUSED_NH], b2s[FUSED_NH], b3s[FUSED_NH];
    __shared__ float4 w4s[FUSED_NH];               // layer 4: (w0, w1, w2, 0) of each input column
    __shared__ float b4s[3];
    __shared__ float part[3][FUSED_TILE][3];       // layer 4 sums of column parts 1..3
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_slot;
    __shared__ int failed;
    unsigned char* smem = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    unsigned char* sA = smem;
    unsigned char* const sW[2] = {smem + FUSED_OPERAND, smem + 2 * FUSED_OPERAND};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int quarter = warp & 3, cpart = warp >> 2; // lane quarter, 64-column part
    const int ntiles = (a.n + FUSED_TILE - 1) / FUSED_TILE;

    for (int i = threadIdx.x; i < FUSED_NH; i += FUSED_THREADS)
        w1s[i] = make_float4(__bfloat162float(a.wb[a.off_w1 + 4 * i]), __bfloat162float(a.wb[a.off_w1 + 4 * i + 1]),
                             __bfloat162float(a.wb[a.off_w1 + 4 * i + 2]), __bfloat162float(a.wb[a.off_w1 + 4 * i + 3]));
    for (int i = threadIdx.x; i < FUSED_NH; i += FUSED_THREADS) {
        b1s[i] = a.p[a.off_b1 + i];
        b2s[i] = a.p[a.off_b2 + i];
        b3s[i] = a.p[a.off_b3 + i];
    }
    for (int i = threadIdx.x; i < FUSED_NH; i += FUSED_THREADS)
        w4s[i] = make_float4(__bfloat162float(a.wb[a.off_w4 + i]), __bfloat162float(a.wb[a.off_w4 + FUSED_NH + i]),
                             __bfloat162float(a.wb[a.off_w4 + 2 * FUSED_NH + i]), 0.0f);
    if (threadIdx.x < 3) b4s[threadIdx.x] = a.p[a.off_b4 + threadIdx.x];
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(256));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    const __nv_bfloat16* w2 = a.wb + a.off_w2;
    const __nv_bfloat16* w3 = a.wb + a.off_w3;
    unsigned phase = 0;

    if (blockIdx.x < ntiles) { // layer 2's weights for the first tile
        fused_load_half(sW[0], w2, 0);
        fused_load_half(sW[1], w2, 1);
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    for (int tile = blockIdx.x; tile < ntiles && !failed; tile += gridDim.x) {
        const int m0 = tile * FUSED_TILE;
        // ---- layer 1: thread = (row, quarter of the features) ----
        {
            constexpr int FQ = FUSED_NH / (FUSED_THREADS / FUSED_TILE); // 64 features
            const int r = threadIdx.x & (FUSED_TILE - 1), fq = threadIdx.x >> 7;
            const int m = m0 + r;
            float xn[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const float raw = m < a.n ? a.x[(long long)m * 4 + k] : a.norm[k];
                xn[k] = __bfloat162float(__float2bfloat16_rn((raw - a.norm[k]) / a.norm[4 + k]));
            }
#pragma unroll 1
            for (int j0 = fq * FQ; j0 < fq * FQ + FQ; j0 += 8) {
                float h[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const float4 w = w1s[j0 + j];
                    float acc = 0.0f;
                    acc = fmaf(xn[0], w.x, acc);
                    acc = fmaf(xn[1], w.y, acc);
                    acc = fmaf(xn[2], w.z, acc);
                    acc = fmaf(xn[3], w.w, acc);
                    h[j] = gelu_f(acc + b1s[j0 + j]);
                }
                *reinterpret_cast<uint4*>(sA + fused_at(r, j0)) = fused_pack8(h);
            }
        }
        // ---- layers 2 and 3 ----
#pragma unroll 1
        for (int layer = 2; layer <= 3; ++layer) {
            asm volatile("cp.async.wait_group 0;" ::: "memory");   // this layer's weights have landed
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); // activations and weights -> MMA
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
            if (threadIdx.x == 0) fused_mma_layer(tmem, sA, sW, &bar);
            if (!mbar_wait(&bar, phase & 1)) failed = 1;
            ++phase;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            __syncthreads();
            if (failed) break;
            // the weight buffers are free: the next layer's (or the next tile's) halves start moving
            const bool more = layer == 2 || tile + (int)gridDim.x < ntiles;
            if (more) {
                const __nv_bfloat16* wn = layer == 2 ? w3 : w2;
                fused_load_half(sW[0], wn, 0);
                fused_load_half(sW[1], wn, 1);
                asm volatile("cp.async.commit_group;" ::: "memory");
            }
            // ---- epilogue: thread = row (tensor-memory lane), its 64-column part ----
            const int row = quarter * 32 + lane;
            const float* bias = layer == 2 ? b2s : b3s;
            float y0 = 0.0f, y1 = 0.0f, y2 = 0.0f;
#pragma unroll 1
            for (int cc = 0; cc < 2; ++cc) {
                const int c0 = cpart * 64 + cc * 32;
                float v[32];
                tmem_ld32(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)c0, v);
                const float4* b4 = reinterpret_cast<const float4*>(bias + c0);
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const float4 bb = b4[i];
                    v[4 * i] = gelu_f(v[4 * i] + bb.x);
                    v[4 * i + 1] = gelu_f(v[4 * i + 1] + bb.y);
                    v[4 * i + 2] = gelu_f(v[4 * i + 2] + bb.z);
                    v[4 * i + 3] = gelu_f(v[4 * i + 3] + bb.w);
                }
                if (layer == 2) {
#pragma unroll
                    for (int g = 0; g < 4; ++g)
                        *reinterpret_cast<uint4*>(sA + fused_at(row, c0 + 8 * g)) = fused_pack8(v + 8 * g);
                } else {
#pragma unroll
                    for (int i = 0; i < 32; i += 2) { // layer 4 on the BF16 activations
                        const float2 hb = __bfloat1622float2(__floats2bfloat162_rn(v[i], v[i + 1]));
                        const float4 wa = w4s[c0 + i], wb = w4s[c0 + i + 1];
                        y0 = fmaf(hb.x, wa.x, y0);
                        y1 = fmaf(hb.x, wa.y, y1);
                        y2 = fmaf(hb.x, wa.z, y2);
                        y0 = fmaf(hb.y, wb.x, y0);
                        y1 = fmaf(hb.y, wb.y, y1);
                        y2 = fmaf(hb.y, wb.z, y2);
                    }
                }
            }
            if (layer == 3) {
                if (cpart > 0) {
                    part[cpart - 1][row][0] = y0;
                    part[cpart - 1][row][1] = y1;
                    part[cpart - 1][row][2] = y2;
                }
                __syncthreads();
                const int m = m0 + row;
                if (cpart == 0 && m < a.n) { // the parts in column order
                    a.y[(long long)m * 3 + 0] = (((y0 + part[0][row][0]) + part[1][row][0]) + part[2][row][0]) + b4s[0];
                    a.y[(long long)m * 3 + 1] = (((y1 + part[0][row][1]) + part[1][row][1]) + part[2][row][1]) + b4s[1];
                    a.y[(long long)m * 3 + 2] = (((y2 + part[0][row][2]) + part[1][row][2]) + part[2][row][2]) + b4s[2];
                }
            }
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (failed && threadIdx.x == 0) atomicExch(a.error, 1u);
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256));
}

} // namespace surrogate
