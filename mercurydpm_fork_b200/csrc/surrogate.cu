// surrogate.cu -- the calibration surrogate: a 4-256-256-256-3 GELU
// multilayer perceptron with BF16 weights and activations and FP32
// accumulation, trained with Adam, every GEMM on tcgen05 tensor cores
// (surrogate_gemm.cuh). C ABI in include/dem_surrogate.h.
//
// The reference has no such component: its calibration loop
// (Drivers/Calibration/py/smc.py:168-350) proposes parameters by sequential
// Monte Carlo over plain DEM runs; this network learns the map from contact
// parameters to bulk responses from batched DEM runs and proposes candidates
// for them, with DEM kept as the judge of its error.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/dem_surrogate.h"
#include "surrogate_gemm.cuh"
#include "surrogate_fused.cuh"

using namespace surrogate;

namespace {

constexpr int NI = DEM_MLP_INPUTS, NH = DEM_MLP_HIDDEN, NO = DEM_MLP_OUTPUTS;

// offsets of the flat FP32 parameter vector (include/dem_surrogate.h)
constexpr long long OFF_W1 = 0, OFF_B1 = OFF_W1 + (long long)NH * NI;
constexpr long long OFF_W2 = OFF_B1 + NH, OFF_B2 = OFF_W2 + (long long)NH * NH;
constexpr long long OFF_W3 = OFF_B2 + NH, OFF_B3 = OFF_W3 + (long long)NH * NH;
constexpr long long OFF_W4 = OFF_B3 + NH, OFF_B4 = OFF_W4 + (long long)NO * NH;
constexpr long long NPARAM = OFF_B4 + NO;
static_assert(NPARAM == DEM_MLP_NPARAMS, "parameter layout");

struct Mlp {
    int device = 0;
    int capacity = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    unsigned* d_error = nullptr;
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr; // params, grads, Adam moments (FP32)
    __nv_bfloat16* wb = nullptr;                                    // BF16 copy of the whole vector
    long long step = 0;
    float norm[2 * NI + 2 * NO];                                    // in_mean, in_std, out_mean, out_std
    float* d_norm = nullptr;
    // activations for `capacity` rows
    float *x = nullptr, *t = nullptr;        // raw inputs, raw targets (FP32)
    __nv_bfloat16* xb = nullptr;             // normalised inputs
    float *z1 = nullptr, *z2 = nullptr, *z3 = nullptr, *y = nullptr;
    __nv_bfloat16 *h1 = nullptr, *h2 = nullptr, *h3 = nullptr;
    __nv_bfloat16 *dyb = nullptr, *dz1 = nullptr, *dz2 = nullptr, *dz3 = nullptr;
    float* loss = nullptr;
};

int fail(Mlp* h, int code, const std::string& msg)
{
    if (h) h->err = msg;
    return code;
}

#define CK(call)                                                                                      \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) return fail(h, DEM_MLP_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

unsigned grid1(long long n, int b) { return (unsigned)std::max<long long>(1, (n + b - 1) / b); }

} // namespace

// ---------------------------------------------------------------------------
// element-wise and reduction kernels
// ---------------------------------------------------------------------------
namespace {

// x (raw, [n][4]) -> (x - mean) / std in BF16
__global__ void k_norm_inputs(const float* x, const float* norm, int n, __nv_bfloat16* xb)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * NI) return;
    const int c = i % NI;
    xb[i] = __float2bfloat16_rn((x[i] - norm[c]) / norm[NI + c]);
}

// y (normalised, [n][3]) -> raw units
__global__ void k_denorm_outputs(const float* y, const float* norm, int n, float* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * NO) return;
    const int c = i % NO;
    out[i] = y[i] * norm[2 * NI + NO + c] + norm[2 * NI + c];
}

// loss = mean (y - t')^2 with t' the normalised target; dy = 2 (y - t') / (3 n)
// in BF16. One block, rows in a fixed order.
__global__ void __launch_bounds__(256) k_loss(const float* y, const float* t, const float* norm, int n,
                                              __nv_bfloat16* dyb, float* loss)
{
    __shared__ float sh[256];
    float acc = 0.f;
    const float scale = 2.0f / (3.0f * (float)n);
    for (int i = threadIdx.x; i < n * NO; i += blockDim.x) {
        const int c = i % NO;
        const float tn = (t[i] - norm[2 * NI + c]) / norm[2 * NI + NO + c];
        const float d = y[i] - tn;
        acc += d * d;
        dyb[i] = __float2bfloat16_rn(scale * d);
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) *loss = sh[0] / (3.0f * (float)n);
}

// bias gradient: column sums of a [n][cols] BF16 matrix
__global__ void k_colsum(const __nv_bfloat16* d, int n, int cols, float* out)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.f;
    for (int r = 0; r < n; ++r) s += __bfloat162float(d[(long long)r * cols + c]);
    out[c] = s;
}

__global__ void k_to_bf16(const float* p, long long n, __nv_bfloat16* out)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = __float2bfloat16_rn(p[i]);
}

// Adam (Kingma and Ba 2015) with bias correction; refreshes the BF16 copy
__global__ void k_adam(float* p, const float* g, float* m, float* v, long long n, float lr, float bc1, float bc2,
                       __nv_bfloat16* wb)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = 0.9f * m[i] + 0.1f * gi;
    const float vi = 0.999f * v[i] + 0.001f * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + 1e-8f);
    p[i] = pi;
    wb[i] = __float2bfloat16_rn(pi);
}

template <int BN>
int launch_gemm(Mlp* h, GemmArgs a)
{
    using L = GemmSmem<BN>;
    static bool configured[64] = {false};
    if (!configured[h->device & 63]) {
        CK(cudaFuncSetAttribute(k_gemm_bf16<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, L::BYTES));
        configured[h->device & 63] = true;
    }
    a.error = h->d_error;
    const dim3 grid(grid1(a.M, GEMM_BM), grid1(a.N, BN));
    k_gemm_bf16<BN><<<grid, GEMM_THREADS, L::BYTES, h->stream>>>(a);
    CK(cudaGetLastError());
    return DEM_MLP_OK;
}

// C = A . B^T with the operand strides of GemmArgs; N <= 16 uses 16-wide tiles
int gemm(Mlp* h, const __nv_bfloat16* A, long long a_sm, long long a_sk, const __nv_bfloat16* B, long long b_sn,
         long long b_sk, int M, int N, int K, int epi, const float* bias, const float* aux, float* out_f32,
         __nv_bfloat16* out_bf16, int ldc)
{
    GemmArgs a{A, B, a_sm, a_sk, b_sn, b_sk, M, N, K, epi, bias, aux, out_f32, out_bf16, ldc, nullptr};
    if (N <= 16) return launch_gemm<16>(h, a);
    return launch_gemm<256>(h, a);
}

} // namespace

// ---------------------------------------------------------------------------
// forward and backward passes (n rows already in h->x, h->t)
// ---------------------------------------------------------------------------
namespace {

// Inference: the whole pass in one kernel (surrogate_fused.cuh), one CTA per
// SM over 128-sample tiles; the activations stay on the SM.
int forward_fused(Mlp* h, int n)
{
    static bool configured[64] = {false};
    static int sms[64] = {0};
    if (!configured[h->device & 63]) {
        CK(cudaFuncSetAttribute(k_mlp_forward_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, FUSED_SMEM));
        CK(cudaDeviceGetAttribute(&sms[h->device & 63], cudaDevAttrMultiProcessorCount, h->device));
        configured[h->device & 63] = true;
    }
    const int tiles = (n + FUSED_TILE - 1) / FUSED_TILE;
    FusedArgs a{h->x, h->d_norm, h->wb, h->p, OFF_W1, OFF_B1, OFF_W2, OFF_B2, OFF_W3, OFF_B3, OFF_W4, OFF_B4,
                n, h->y, h->d_error};
    k_mlp_forward_fused<<<std::min(tiles, sms[h->device & 63]), FUSED_THREADS, FUSED_SMEM, h->stream>>>(a);
    CK(cudaGetLastError());
    return DEM_MLP_OK;
}

// keep_z: store the pre-activations for a backward pass (training, one GEMM
// per layer); without, the fused inference kernel
int forward(Mlp* h, int n, bool keep_z = true)
{
    if (!keep_z) return forward_fused(h, n);
    const int epi = keep_z ? EPI_BIAS_GELU : EPI_BIAS_GELU_H;
    int rc;
    const __nv_bfloat16* W = h->wb;
    const float* P = h->p;
    k_norm_inputs<<<grid1((long long)n * NI, 256), 256, 0, h->stream>>>(h->x, h->d_norm, n, h->xb);
    // z1 = x W1^T + b1, h1 = gelu(z1), ... (A rows = samples, B rows = output features)
    if ((rc = gemm(h, h->xb, NI, 1, W + OFF_W1, NI, 1, n, NH, NI, epi, P + OFF_B1, nullptr, h->z1, h->h1, NH)))
        return rc;
    if ((rc = gemm(h, h->h1, NH, 1, W + OFF_W2, NH, 1, n, NH, NH, epi, P + OFF_B2, nullptr, h->z2, h->h2, NH)))
        return rc;
    if ((rc = gemm(h, h->h2, NH, 1, W + OFF_W3, NH, 1, n, NH, NH, epi, P + OFF_B3, nullptr, h->z3, h->h3, NH)))
        return rc;
    return gemm(h, h->h3, NH, 1, W + OFF_W4, NH, 1, n, NO, NH, EPI_BIAS_F32, P + OFF_B4, nullptr, h->y, nullptr, NO);
}

// gradient of the mean squared error into h->g; loss into h->loss
int backward(Mlp* h, int n)
{
    int rc;
    const __nv_bfloat16* W = h->wb;
    float* G = h->g;
    k_loss<<<1, 256, 0, h->stream>>>(h->y, h->t, h->d_norm, n, h->dyb, h->loss);
    // layer 4: dW4[o][i] = sum_b dy[b][o] h3[b][i]; db4 = colsum(dy); dz3 = (dy W4) gelu'(z3)
    if ((rc = gemm(h, h->dyb, 1, NO, h->h3, 1, NH, NO, NH, n, EPI_STORE_F32, nullptr, nullptr, G + OFF_W4, nullptr, NH)))
        return rc;
    k_colsum<<<1, 32, 0, h->stream>>>(h->dyb, n, NO, G + OFF_B4);
    if ((rc = gemm(h, h->dyb, NO, 1, W + OFF_W4, 1, NH, n, NH, NO, EPI_DGELU_BF16, nullptr, h->z3, nullptr, h->dz3, NH)))
        return rc;
    // layer 3
    if ((rc = gemm(h, h->dz3, 1, NH, h->h2, 1, NH, NH, NH, n, EPI_STORE_F32, nullptr, nullptr, G + OFF_W3, nullptr, NH)))
        return rc;
    k_colsum<<<1, NH, 0, h->stream>>>(h->dz3, n, NH, G + OFF_B3);
    if ((rc = gemm(h, h->dz3, NH, 1, W + OFF_W3, 1, NH, n, NH, NH, EPI_DGELU_BF16, nullptr, h->z2, nullptr, h->dz2, NH)))
        return rc;
    // layer 2
    if ((rc = gemm(h, h->dz2, 1, NH, h->h1, 1, NH, NH, NH, n, EPI_STORE_F32, nullptr, nullptr, G + OFF_W2, nullptr, NH)))
        return rc;
    k_colsum<<<1, NH, 0, h->stream>>>(h->dz2, n, NH, G + OFF_B2);
    if ((rc = gemm(h, h->dz2, NH, 1, W + OFF_W2, 1, NH, n, NH, NH, EPI_DGELU_BF16, nullptr, h->z1, nullptr, h->dz1, NH)))
        return rc;
    // layer 1 (its input gradient is not needed)
    if ((rc = gemm(h, h->dz1, 1, NH, h->xb, 1, NI, NH, NI, n, EPI_STORE_F32, nullptr, nullptr, G + OFF_W1, nullptr, NI)))
        return rc;
    k_colsum<<<1, NH, 0, h->stream>>>(h->dz1, n, NH, G + OFF_B1);
    CK(cudaGetLastError());
    return DEM_MLP_OK;
}

int check_device_status(Mlp* h)
{
    unsigned e = 0;
    CK(cudaMemcpyAsync(&e, h->d_error, sizeof(e), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (e) {
        CK(cudaMemsetAsync(h->d_error, 0, sizeof(unsigned), h->stream));
        return fail(h, DEM_MLP_ERR_TIMEOUT, "a tensor-core wait ran out");
    }
    return DEM_MLP_OK;
}

int load_batch(Mlp* h, const float* x, const float* t, int n)
{
    if (n <= 0 || n > h->capacity || !x) return fail(h, DEM_MLP_ERR_BAD_INPUT, "batch size out of range");
    CK(cudaSetDevice(h->device));
    CK(cudaMemcpyAsync(h->x, x, (size_t)n * NI * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    if (t) CK(cudaMemcpyAsync(h->t, t, (size_t)n * NO * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    return DEM_MLP_OK;
}

} // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
struct dem_mlp : Mlp {};

extern "C" {

int dem_mlp_create(int device, int capacity, uint64_t seed, dem_mlp** out)
{
    if (!out || capacity <= 0 || capacity > (1 << 24)) return DEM_MLP_ERR_BAD_INPUT;
    *out = nullptr;
    dem_mlp* h = new dem_mlp();
    h->device = device;
    h->capacity = capacity;
    auto cleanup = [&](int rc) {
        if (rc) dem_mlp_destroy(h);
        return rc;
    };
    if (cudaSetDevice(device) != cudaSuccess) return cleanup(DEM_MLP_ERR_CUDA);
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) return cleanup(DEM_MLP_ERR_CUDA);
    const size_t c = (size_t)capacity;
    bool ok = true;
    auto alloc = [&](auto** p, size_t count) {
        if (ok && cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(count, 1) * sizeof(**p)) != cudaSuccess)
            ok = false;
    };
    alloc(&h->d_error, 1);
    alloc(&h->p, NPARAM); alloc(&h->g, NPARAM); alloc(&h->m, NPARAM); alloc(&h->v, NPARAM);
    alloc(&h->wb, NPARAM);
    alloc(&h->d_norm, 2 * NI + 2 * NO);
    alloc(&h->x, c * NI); alloc(&h->t, c * NO); alloc(&h->xb, c * NI);
    alloc(&h->z1, c * NH); alloc(&h->z2, c * NH); alloc(&h->z3, c * NH); alloc(&h->y, c * NO);
    alloc(&h->h1, c * NH); alloc(&h->h2, c * NH); alloc(&h->h3, c * NH);
    alloc(&h->dyb, c * NO); alloc(&h->dz1, c * NH); alloc(&h->dz2, c * NH); alloc(&h->dz3, c * NH);
    alloc(&h->loss, 1);
    if (!ok) return cleanup(fail(h, DEM_MLP_ERR_CUDA, "cudaMalloc failed"));
    // He-uniform weights, zero biases
    std::vector<float> p(NPARAM, 0.0f);
    std::mt19937_64 rng(seed);
    auto fill = [&](long long off, int rows, int cols) {
        const float a = std::sqrt(6.0f / (float)cols);
        std::uniform_real_distribution<float> u(-a, a);
        for (long long i = 0; i < (long long)rows * cols; ++i) p[off + i] = u(rng);
    };
    fill(OFF_W1, NH, NI);
    fill(OFF_W2, NH, NH);
    fill(OFF_W3, NH, NH);
    fill(OFF_W4, NO, NH);
    for (int k = 0; k < NI; ++k) { h->norm[k] = 0.f; h->norm[NI + k] = 1.f; }
    for (int k = 0; k < NO; ++k) { h->norm[2 * NI + k] = 0.f; h->norm[2 * NI + NO + k] = 1.f; }
    int rc = dem_mlp_set_params(h, p.data());
    if (rc) return cleanup(rc);
    if (cudaMemcpyAsync(h->d_norm, h->norm, sizeof(h->norm), cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
        cudaMemsetAsync(h->d_error, 0, sizeof(unsigned), h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess)
        return cleanup(DEM_MLP_ERR_CUDA);
    *out = h;
    return DEM_MLP_OK;
}

int dem_mlp_set_normalisation(dem_mlp* h, const float* in_mean, const float* in_std, const float* out_mean,
                              const float* out_std)
{
    if (!h || !in_mean || !in_std || !out_mean || !out_std) return DEM_MLP_ERR_BAD_INPUT;
    for (int k = 0; k < NI; ++k) {
        if (!(in_std[k] > 0.f)) return fail(h, DEM_MLP_ERR_BAD_INPUT, "input std must be positive");
        h->norm[k] = in_mean[k];
        h->norm[NI + k] = in_std[k];
    }
    for (int k = 0; k < NO; ++k) {
        if (!(out_std[k] > 0.f)) return fail(h, DEM_MLP_ERR_BAD_INPUT, "output std must be positive");
        h->norm[2 * NI + k] = out_mean[k];
        h->norm[2 * NI + NO + k] = out_std[k];
    }
    CK(cudaSetDevice(h->device));
    CK(cudaMemcpyAsync(h->d_norm, h->norm, sizeof(h->norm), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return DEM_MLP_OK;
}

int dem_mlp_get_params(dem_mlp* h, float* params)
{
    if (!h || !params) return DEM_MLP_ERR_BAD_INPUT;
    CK(cudaSetDevice(h->device));
    CK(cudaMemcpyAsync(params, h->p, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return DEM_MLP_OK;
}

int dem_mlp_set_params(dem_mlp* h, const float* params)
{
    if (!h || !params) return DEM_MLP_ERR_BAD_INPUT;
    CK(cudaSetDevice(h->device));
    CK(cudaMemcpyAsync(h->p, params, NPARAM * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemsetAsync(h->m, 0, NPARAM * sizeof(float), h->stream));
    CK(cudaMemsetAsync(h->v, 0, NPARAM * sizeof(float), h->stream));
    k_to_bf16<<<grid1(NPARAM, 256), 256, 0, h->stream>>>(h->p, NPARAM, h->wb);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    h->step = 0;
    return DEM_MLP_OK;
}

int dem_mlp_forward(dem_mlp* h, const float* x, int n, float* y)
{
    if (!h || !y) return DEM_MLP_ERR_BAD_INPUT;
    int rc;
    if ((rc = load_batch(h, x, nullptr, n)) || (rc = forward(h, n, false))) return rc;
    k_denorm_outputs<<<grid1((long long)n * NO, 256), 256, 0, h->stream>>>(h->y, h->d_norm, n, h->t);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(y, h->t, (size_t)n * NO * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    return check_device_status(h);
}

int dem_mlp_gradients(dem_mlp* h, const float* x, const float* t, int n, float* loss, float* grads)
{
    if (!h || !t || !loss || !grads) return DEM_MLP_ERR_BAD_INPUT;
    int rc;
    if ((rc = load_batch(h, x, t, n)) || (rc = forward(h, n)) || (rc = backward(h, n))) return rc;
    CK(cudaMemcpyAsync(loss, h->loss, sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(grads, h->g, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    return check_device_status(h);
}

int dem_mlp_train_step(dem_mlp* h, const float* x, const float* t, int n, float lr, float* loss)
{
    if (!h || !t || !(lr > 0.f)) return DEM_MLP_ERR_BAD_INPUT;
    int rc;
    if ((rc = load_batch(h, x, t, n)) || (rc = forward(h, n)) || (rc = backward(h, n))) return rc;
    h->step += 1;
    const float bc1 = 1.0f - std::pow(0.9f, (float)h->step);
    const float bc2 = 1.0f - std::pow(0.999f, (float)h->step);
    k_adam<<<grid1(NPARAM, 256), 256, 0, h->stream>>>(h->p, h->g, h->m, h->v, NPARAM, lr, bc1, bc2, h->wb);
    CK(cudaGetLastError());
    if (loss) CK(cudaMemcpyAsync(loss, h->loss, sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    return check_device_status(h);
}

int dem_mlp_time_forward(dem_mlp* h, int n, int reps, float* ms)
{
    if (!h || !ms || n <= 0 || n > h->capacity || reps <= 0) return DEM_MLP_ERR_BAD_INPUT;
    CK(cudaSetDevice(h->device));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    int rc = forward(h, n, false); // warm-up
    CK(cudaEventRecord(e0, h->stream));
    for (int r = 0; r < reps && !rc; ++r) rc = forward(h, n, false);
    CK(cudaEventRecord(e1, h->stream));
    CK(cudaEventSynchronize(e1));
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    *ms = t / reps;
    return check_device_status(h);
}

const char* dem_mlp_last_error(dem_mlp* h) { return h ? h->err.c_str() : "null handle"; }

void dem_mlp_destroy(dem_mlp* h)
{
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    void* ptrs[] = {h->d_error, h->p, h->g, h->m, h->v, h->wb, h->d_norm, h->x, h->t, h->xb, h->z1, h->z2,
                    h->z3, h->y, h->h1, h->h2, h->h3, h->dyb, h->dz1, h->dz2, h->dz3, h->loss};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

} // extern "C"
