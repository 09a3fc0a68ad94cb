// surrogate_gemm.cuh -- BF16 x BF16 -> FP32 GEMM on the 5th-generation tensor
// cores (tcgen05.mma, accumulator in tensor memory) for the calibration
// surrogate's multilayer perceptron.
//
//   C[m, n] = sum_k A(m, k) B(n, k)      A(m, k) = A[m * a_sm + k * a_sk]
//                                        B(n, k) = B[n * b_sn + k * b_sk]
//
// One CTA of 256 threads computes a 128 x BN tile (BN <= 256, a multiple of
// 16) over the whole K range: K is staged 64 at a time into shared memory in
// the K-major canonical layout without swizzle (8 x 16-byte core matrices;
// LBO = 128 B between the two K halves of an instruction, SBO = 1024 B
// between 8-row groups), two stages deep; one elected thread issues four
// K=16 tcgen05.mma per stage and commits them to the stage's mbarrier; the
// accumulator lives in tensor memory (128 lanes x BN columns of FP32) and the
// eight warps read it back with tcgen05.ld (each lane quarter by two warps,
// alternate 32-column runs) for the fused epilogue.
// Operand staging uses plain loads, so any strides (transposes) are allowed:
// the backward pass reads its operands transposed without extra copies.
//
// Every wait is bounded: a wait that runs out sets an error word and the
// kernel finishes without using the missing result; tensor memory is
// always released.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace surrogate {

constexpr int GEMM_BM = 128;
constexpr int GEMM_BK = 64;
constexpr int GEMM_THREADS = 256; // 8 warps: warps w and w + 4 share TMEM lanes 32 (w % 4) ..
constexpr int GEMM_MAX_BN = 256;
constexpr unsigned long long WAIT_LIMIT = 1ull << 26; // try_wait polls before giving up

enum Epilogue : int {
    EPI_STORE_F32 = 0,    // out_f32[m, n] = acc
    EPI_BIAS_GELU = 1,    // z = acc + bias[n]; out_f32 = z; out_bf16 = gelu(z)
    EPI_BIAS_F32 = 2,     // out_f32 = acc + bias[n]
    EPI_DGELU_BF16 = 3,   // out_bf16 = acc * gelu'(z[m, n]) with z = aux_f32
    EPI_BIAS_GELU_H = 4,  // out_bf16 = gelu(acc + bias[n]) (inference: no pre-activation kept)
};

struct GemmArgs {
    const __nv_bfloat16* A;
    const __nv_bfloat16* B;
    long long a_sm, a_sk, b_sn, b_sk;
    int M, N, K;
    int epilogue;
    const float* bias;       // EPI_BIAS_*
    const float* aux_f32;    // EPI_DGELU_BF16: pre-activations z, ld = ldc
    float* out_f32;
    __nv_bfloat16* out_bf16;
    int ldc;
    unsigned int* error;     // set to 1 when a wait runs out
};

__device__ __forceinline__ float gelu_f(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }

// d/dz of z Phi(z): Phi(z) + z phi(z)
__device__ __forceinline__ float gelu_grad_f(float z)
{
    const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
    return cdf + z * pdf;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// UMMA shared-memory matrix descriptor: start, leading and stride byte
// offsets (16-byte units), version 1, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B, both
// K-major, N = bn, M = 128.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int bn)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(bn >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

// bounded wait; false when the limit ran out
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity)
{
    for (unsigned long long i = 0; i < WAIT_LIMIT; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
                 "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32])
{
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                 "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                   "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                   "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Stage rows [row0, row0 + rows) x k [k0, k0 + 64) of a strided BF16 matrix
// into the K-major no-swizzle layout: core matrix (row / 8, k / 8) at
// (row / 8) * 1024 + (k / 8) * 128 bytes, row % 8 selecting its 16-byte row.
// Out-of-range elements are zero.
__device__ __forceinline__ void stage_tile(unsigned char* dst, const __nv_bfloat16* src, long long s_row,
                                           long long s_k, int row0, int rows, int nrows, int k0, int K)
{
    const int items = rows * (GEMM_BK / 8); // (row, 8-element k group)
    for (int it = threadIdx.x; it < items; it += GEMM_THREADS) {
        const int r = it >> 3, g = it & 7;
        const int row = row0 + r;
        const int kb = k0 + g * 8;
        unsigned short e[8];
        if (row < nrows && kb + 8 <= K && s_k == 1 && ((((long long)row * s_row + kb) & 7) == 0)) {
            const uint4 v = *reinterpret_cast<const uint4*>(src + (long long)row * s_row + kb);
            *reinterpret_cast<uint4*>(dst + (r >> 3) * 1024 + g * 128 + (r & 7) * 16) = v;
            continue;
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int k = kb + q;
            e[q] = (row < nrows && k < K) ? __bfloat16_as_ushort(src[(long long)row * s_row + (long long)k * s_k]) : 0;
        }
        uint4 v;
        v.x = e[0] | ((uint32_t)e[1] << 16);
        v.y = e[2] | ((uint32_t)e[3] << 16);
        v.z = e[4] | ((uint32_t)e[5] << 16);
        v.w = e[6] | ((uint32_t)e[7] << 16);
        *reinterpret_cast<uint4*>(dst + (r >> 3) * 1024 + g * 128 + (r & 7) * 16) = v;
    }
}

// The same staging for a row-contiguous matrix with 16-byte aligned rows:
// one cp.async of 16 bytes per (row, 8-element k group), zero-filled past
// the matrix edge, in flight together (cp.async.commit_group by the caller).
__device__ __forceinline__ void stage_tile_async(unsigned char* dst, const __nv_bfloat16* src, long long s_row,
                                                 int row0, int rows, int nrows, int k0, int K)
{
    const int items = rows * (GEMM_BK / 8);
    for (int it = threadIdx.x; it < items; it += GEMM_THREADS) {
        const int r = it >> 3, g = it & 7;
        const int row = row0 + r;
        const int kb = k0 + g * 8;
        int bytes = 0;
        const __nv_bfloat16* p = src;
        if (row < nrows && kb < K) {
            bytes = (K - kb >= 8) ? 16 : (K - kb) * 2;
            p = src + (long long)row * s_row + kb;
        }
        const uint32_t d = smem_u32(dst + (r >> 3) * 1024 + g * 128 + (r & 7) * 16);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(p), "r"(bytes) : "memory");
    }
}

} // namespace surrogate

namespace surrogate {

template <int BN>
struct GemmSmem {
    static constexpr int A_BYTES = GEMM_BM * GEMM_BK * 2; // 16 KB per stage
    static constexpr int B_BYTES = BN * GEMM_BK * 2;
    static constexpr int BYTES = 2 * A_BYTES + 2 * B_BYTES + 1024; // + alignment slack
    static constexpr uint32_t TMEM_COLS = BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));
};

template <int BN>
__global__ void __launch_bounds__(GEMM_THREADS, 1) k_gemm_bf16(GemmArgs g)
{
    static_assert(BN % 16 == 0 && BN >= 16 && BN <= GEMM_MAX_BN, "UMMA N for M = 128");
    using L = GemmSmem<BN>;
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ uint32_t tmem_slot;
    __shared__ int failed;
    unsigned char* smem = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    unsigned char* sA[2] = {smem, smem + L::A_BYTES};
    unsigned char* sB[2] = {smem + 2 * L::A_BYTES, smem + 2 * L::A_BYTES + L::B_BYTES};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * GEMM_BM, n0 = blockIdx.y * BN;

    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(L::TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    constexpr uint32_t idesc = umma_idesc_bf16(BN);

    const int nk = (g.K + GEMM_BK - 1) / GEMM_BK;
    // row-contiguous operands with 16-byte rows are staged with cp.async, so
    // the next chunk's copies run while this chunk's MMAs do
    const bool a_async = g.a_sk == 1 && (g.a_sm & 7) == 0 && ((reinterpret_cast<uintptr_t>(g.A) & 15) == 0);
    const bool b_async = g.b_sk == 1 && (g.b_sn & 7) == 0 && ((reinterpret_cast<uintptr_t>(g.B) & 15) == 0);
    auto stage = [&](int c, int b) {
        if (a_async) stage_tile_async(sA[b], g.A, g.a_sm, m0, GEMM_BM, g.M, c * GEMM_BK, g.K);
        else stage_tile(sA[b], g.A, g.a_sm, g.a_sk, m0, GEMM_BM, g.M, c * GEMM_BK, g.K);
        if (b_async) stage_tile_async(sB[b], g.B, g.b_sn, n0, BN, g.N, c * GEMM_BK, g.K);
        else stage_tile(sB[b], g.B, g.b_sn, g.b_sk, n0, BN, g.N, c * GEMM_BK, g.K);
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    stage(0, 0);
    for (int c = 0; c < nk; ++c) {
        const int b = c & 1;
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); // generic/cp.async writes -> async-proxy reads
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int j = 0; j < GEMM_BK / 16; ++j) {
                const uint64_t ad = umma_desc(smem_u32(sA[b]) + j * 256, 128, 1024);
                const uint64_t bd = umma_desc(smem_u32(sB[b]) + j * 256, 128, 1024);
                umma_bf16(tmem, ad, bd, idesc, (c > 0 || j > 0) ? 1u : 0u);
            }
            umma_commit(&bar[b]);
        }
        if (c + 1 < nk) {
            const int b1 = (c + 1) & 1;
            // the MMAs of chunk c - 1 read buffer b1: wait for them before overwriting it
            if (c >= 1 && !mbar_wait(&bar[b1], ((c - 1) >> 1) & 1)) failed = 1;
            stage(c + 1, b1);
        }
    }
    const int last = nk - 1;
    if (!mbar_wait(&bar[last & 1], (last >> 1) & 1)) failed = 1;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __syncthreads();
    if (failed) {
        if (threadIdx.x == 0) atomicExch(g.error, 1u);
    } else {
        // ---- epilogue: thread = accumulator row (tensor-memory lane); the two
        // warps of a lane quarter take alternate 32-column runs ----
        const int quarter = warp & 3, half = warp >> 2;
        const int row = m0 + quarter * 32 + lane;
        const bool row_ok = row < g.M;
#pragma unroll 1
        for (int cc = half; cc < (BN + 31) / 32; cc += 2) { // a 16-wide tile reads 32 allocated columns
            float v[32];
            tmem_ld32(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(cc * 32), v);
            if (!row_ok) continue;
            const long long base = (long long)row * g.ldc;
            const int nb0 = n0 + cc * 32;
            if (cc * 32 + 32 <= BN && nb0 + 32 <= g.N && (g.ldc & 7) == 0) {
                // a whole 32-column run of this row: 16-byte stores (the row's
                // 64 or 128 bytes are contiguous)
                float r[32];
                if (g.epilogue == EPI_BIAS_GELU || g.epilogue == EPI_BIAS_F32 || g.epilogue == EPI_BIAS_GELU_H) {
                    const float4* b4 = reinterpret_cast<const float4*>(g.bias + nb0);
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const float4 bb = b4[i];
                        r[4 * i] = v[4 * i] + bb.x;
                        r[4 * i + 1] = v[4 * i + 1] + bb.y;
                        r[4 * i + 2] = v[4 * i + 2] + bb.z;
                        r[4 * i + 3] = v[4 * i + 3] + bb.w;
                    }
                } else if (g.epilogue == EPI_DGELU_BF16) {
                    const float4* z4 = reinterpret_cast<const float4*>(g.aux_f32 + base + nb0);
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const float4 zz = z4[i];
                        r[4 * i] = v[4 * i] * gelu_grad_f(zz.x);
                        r[4 * i + 1] = v[4 * i + 1] * gelu_grad_f(zz.y);
                        r[4 * i + 2] = v[4 * i + 2] * gelu_grad_f(zz.z);
                        r[4 * i + 3] = v[4 * i + 3] * gelu_grad_f(zz.w);
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < 32; ++i) r[i] = v[i];
                }
                if (g.epilogue == EPI_STORE_F32 || g.epilogue == EPI_BIAS_F32 || g.epilogue == EPI_BIAS_GELU) {
                    float4* o4 = reinterpret_cast<float4*>(g.out_f32 + base + nb0);
#pragma unroll
                    for (int i = 0; i < 8; ++i) o4[i] = make_float4(r[4 * i], r[4 * i + 1], r[4 * i + 2], r[4 * i + 3]);
                }
                if (g.epilogue == EPI_BIAS_GELU || g.epilogue == EPI_BIAS_GELU_H || g.epilogue == EPI_DGELU_BF16) {
                    const bool act = g.epilogue != EPI_DGELU_BF16;
                    uint4* o4 = reinterpret_cast<uint4*>(g.out_bf16 + base + nb0);
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        uint32_t w[4];
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const float x0 = act ? gelu_f(r[8 * i + 2 * j]) : r[8 * i + 2 * j];
                            const float x1 = act ? gelu_f(r[8 * i + 2 * j + 1]) : r[8 * i + 2 * j + 1];
                            w[j] = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(x0)) |
                                   ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(x1)) << 16);
                        }
                        o4[i] = make_uint4(w[0], w[1], w[2], w[3]);
                    }
                }
                continue;
            }
#pragma unroll
            for (int i = 0; i < 32; ++i) {
                const int n = nb0 + i;
                if (cc * 32 + i >= BN || n >= g.N) break;
                const float a = v[i];
                switch (g.epilogue) {
                case EPI_STORE_F32: g.out_f32[base + n] = a; break;
                case EPI_BIAS_F32: g.out_f32[base + n] = a + g.bias[n]; break;
                case EPI_BIAS_GELU: {
                    const float z = a + g.bias[n];
                    g.out_f32[base + n] = z;
                    g.out_bf16[base + n] = __float2bfloat16_rn(gelu_f(z));
                    break;
                }
                case EPI_BIAS_GELU_H:
                    g.out_bf16[base + n] = __float2bfloat16_rn(gelu_f(a + g.bias[n]));
                    break;
                default: // EPI_DGELU_BF16
                    g.out_bf16[base + n] = __float2bfloat16_rn(a * gelu_grad_f(g.aux_f32[base + n]));
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(L::TMEM_COLS));
}

} // namespace surrogate
