// Kernels of the learned initial-guess network: a multilayer perceptron over
// atom-pair descriptors whose outputs are density-matrix blocks.  Training
// runs in FP32 (forward with the pre-activations kept, backward, masked mean
// squared error, Adam); inference reads BF16 weights and BF16-rounded inputs
// on the tensor cores (mma.sync, FP32 accumulation).  The layer shapes are
// small (inputs of about a hundred features, width 128, outputs up to 196),
// so each layer is one tiled GEMM launch with bias and SiLU fused into its
// epilogue; the FP32 kernel serves the forward pass of training and the three
// products of the backward pass through operand strides.
// No counterpart in the reference (its initial guesses are SAD / core / read).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/vlx_b200.h"

namespace {

constexpr int kTile = 64;  // output tile (rows and columns)
constexpr int kTileK = 16; // reduction slice staged in shared memory

__device__ __forceinline__ float load_f(const float* p, size_t i) { return __ldg(p + i); }
__device__ __forceinline__ float load_f(const __nv_bfloat16* p, size_t i) { return __bfloat162float(p[i]); }

__device__ __forceinline__ float silu(float z) { return z / (1.0f + expf(-z)); }

// C(m, n) = sum_k A(m, k) B(k, n) (+ bias[n]), A(m, k) = A[m sam + k sak],
// B(k, n) = B[k sbk + n sbn]; Z (optional) gets the value, Y gets SiLU of it
// (or the value itself).  round_a: round A to BF16 before use (inference).
template <typename TB>
__global__ void __launch_bounds__(256) gemm_kernel(const float* __restrict__ A, const long sam, const long sak,
                                                   const TB* __restrict__ B, const long sbk, const long sbn,
                                                   const float* __restrict__ bias, float* __restrict__ Z,
                                                   float* __restrict__ Y, const int M, const int N, const int K,
                                                   const int act, const int round_a)
{
    __shared__ float As[kTileK][kTile + 4];
    __shared__ float Bs[kTileK][kTile + 4];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int m0 = blockIdx.y * kTile, n0 = blockIdx.x * kTile;
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0.0f;
    for (int k0 = 0; k0 < K; k0 += kTileK) {
        for (int t = threadIdx.x; t < kTile * kTileK; t += blockDim.x) {
            const int r = t / kTileK, kk = t % kTileK;
            const int m = m0 + r, k = k0 + kk;
            float v = (m < M && k < K) ? __ldg(A + (size_t)m * sam + (size_t)k * sak) : 0.0f;
            if (round_a) v = __bfloat162float(__float2bfloat16_rn(v));
            As[kk][r] = v;
        }
        for (int t = threadIdx.x; t < kTile * kTileK; t += blockDim.x) {
            const int kk = t / kTile, c = t % kTile;
            const int n = n0 + c, k = k0 + kk;
            Bs[kk][c] = (n < N && k < K) ? load_f(B, (size_t)k * sbk + (size_t)n * sbn) : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kTileK; kk++) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = As[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; j++) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int m = m0 + ty * 4 + i;
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int n = n0 + tx * 4 + j;
            if (n >= N) continue;
            const float z = acc[i][j] + (bias ? __ldg(bias + n) : 0.0f);
            if (Z) Z[(size_t)m * N + n] = z;
            Y[(size_t)m * N + n] = act ? silu(z) : z;
        }
    }
}

// Inference layer on the tensor cores: Y[M, N] = act(X[M, K] W[N, K]^T + b)
// with X rounded to BF16 as it is staged, W in BF16, FP32 accumulation
// (mma.sync m16n8k16 BF16, operand fragments read straight from shared
// memory).  Block: 4 warps on a 64 x 64 output tile, each warp 32 x 32
// (2 x 4 MMA tiles); K in steps of 16, zero-padded at the edges.
constexpr int kMmaTile = 64;
constexpr int kMmaK = 16;
constexpr int kMmaPad = kMmaK + 8;  // row stride 48 B: the fragment loads of a warp hit 32 distinct banks

__device__ __forceinline__ void mma_bf16_16816(float* c, const uint32_t* a, const uint32_t* b)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__global__ void __launch_bounds__(128) gemm_bf16_mma_kernel(const float* __restrict__ X,
                                                            const __nv_bfloat16* __restrict__ W,
                                                            const float* __restrict__ bias, float* __restrict__ Y,
                                                            const int M, const int N, const int K, const int act)
{
    __shared__ __align__(16) __nv_bfloat16 As[kMmaTile][kMmaPad];
    __shared__ __align__(16) __nv_bfloat16 Bs[kMmaTile][kMmaPad];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, tq = lane & 3;
    const int m0 = blockIdx.y * kMmaTile, n0 = blockIdx.x * kMmaTile;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int e = 0; e < 4; e++) acc[i][j][e] = 0.0f;
    const __nv_bfloat16 zero = __float2bfloat16_rn(0.0f);
    for (int k0 = 0; k0 < K; k0 += kMmaK) {
        for (int t = threadIdx.x; t < kMmaTile * kMmaK; t += blockDim.x) {
            const int r = t / kMmaK, kk = t % kMmaK, k = k0 + kk;
            const int m = m0 + r, n = n0 + r;
            As[r][kk] = (m < M && k < K) ? __float2bfloat16_rn(__ldg(X + (size_t)m * K + k)) : zero;
            Bs[r][kk] = (n < N && k < K) ? W[(size_t)n * K + k] : zero;
        }
        __syncthreads();
        uint32_t a[2][4], b[4][2];
#pragma unroll
        for (int i = 0; i < 2; i++) {
            const int r = wm + i * 16 + g;
            a[i][0] = *reinterpret_cast<const uint32_t*>(&As[r][2 * tq]);
            a[i][1] = *reinterpret_cast<const uint32_t*>(&As[r + 8][2 * tq]);
            a[i][2] = *reinterpret_cast<const uint32_t*>(&As[r][2 * tq + 8]);
            a[i][3] = *reinterpret_cast<const uint32_t*>(&As[r + 8][2 * tq + 8]);
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int c = wn + j * 8 + g;
            b[j][0] = *reinterpret_cast<const uint32_t*>(&Bs[c][2 * tq]);
            b[j][1] = *reinterpret_cast<const uint32_t*>(&Bs[c][2 * tq + 8]);
        }
#pragma unroll
        for (int i = 0; i < 2; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) mma_bf16_16816(acc[i][j], a[i], b[j]);
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int m = m0 + wm + i * 16 + g + ((e & 2) ? 8 : 0);
                const int n = n0 + wn + j * 8 + 2 * tq + (e & 1);
                if (m < M && n < N) {
                    const float z = acc[i][j][e] + (bias ? __ldg(bias + n) : 0.0f);
                    Y[(size_t)m * N + n] = act ? silu(z) : z;
                }
            }
}

// dZ = dY * SiLU'(Z), SiLU'(z) = s (1 + z (1 - s)), s = 1 / (1 + e^-z)
__global__ void silu_backward_kernel(const float* __restrict__ dY, const float* __restrict__ Z, float* __restrict__ dZ,
                                     const size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float z = Z[i];
        const float s = 1.0f / (1.0f + expf(-z));
        dZ[i] = dY[i] * s * (1.0f + z * (1.0f - s));
    }
}

// db[n] = sum_m dZ[m N + n]
__global__ void column_sum_kernel(const float* __restrict__ dZ, float* __restrict__ db, const int M, const int N)
{
    __shared__ float part[8][33];
    const int c = blockIdx.x * 32 + threadIdx.x;
    float s = 0.0f;
    if (c < N)
        for (int m = threadIdx.y; m < M; m += blockDim.y) s += dZ[(size_t)m * N + c];
    part[threadIdx.y][threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.y == 0 && c < N) {
        float t = 0.0f;
        for (int r = 0; r < 8; r++) t += part[r][threadIdx.x];
        db[c] = t;
    }
}

// masked squared error: dY = 2 w (Y - T) / count, loss += sum w (Y - T)^2
__global__ void mse_kernel(const float* __restrict__ Y, const float* __restrict__ T, const float* __restrict__ W,
                           float* __restrict__ dY, double* __restrict__ loss, const size_t n, const float inv_count)
{
    __shared__ double part[256];
    double acc = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float w = W[i];
        const float r = Y[i] - T[i];
        dY[i] = 2.0f * w * r * inv_count;
        acc += (double)(w * r * r);
    }
    part[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss, part[0]);
}

// Adam with bias-corrected moments (Kingma & Ba 2015); c1 = 1 - beta1^t, c2 = 1 - beta2^t
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, const size_t n, const float lr, const float b1, const float b2,
                            const float eps, const float c1, const float c2)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

__global__ void to_bf16_kernel(const float* __restrict__ x, __nv_bfloat16* __restrict__ y, const size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] = __float2bfloat16_rn(x[i]);
}

int grid_1d(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 8); }

}  // namespace

extern "C" int vlx_b200_set_error_internal(int code, const char* msg);

#define MLP_CHECK()                                                                       \
    do {                                                                                  \
        cudaError_t e_ = cudaGetLastError();                                              \
        if (e_ != cudaSuccess) return vlx_b200_set_error_internal(VLX_B200_ERR_CUDA, cudaGetErrorString(e_)); \
    } while (0)

extern "C" {

int vlx_b200_mlp_linear(const float* X, const float* W, const float* b, float* Z, float* Y, int M, int K, int N,
                        int silu_act, void* stream)
{
    if (!X || !W || !Y || M < 0 || K < 1 || N < 1)
        return vlx_b200_set_error_internal(VLX_B200_ERR_ARGUMENT, "mlp_linear: bad arguments");
    if (M == 0) return VLX_B200_OK;
    const dim3 grid((N + kTile - 1) / kTile, (M + kTile - 1) / kTile);
    gemm_kernel<float><<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(X, K, 1, W, 1, K, b, Z, Y, M, N, K,
                                                                            silu_act, 0);
    MLP_CHECK();
    return VLX_B200_OK;
}

int vlx_b200_mlp_linear_bf16(const float* X, const void* W_bf16, const float* b, float* Y, int M, int K, int N,
                             int silu_act, void* stream)
{
    if (!X || !W_bf16 || !Y || M < 0 || K < 1 || N < 1)
        return vlx_b200_set_error_internal(VLX_B200_ERR_ARGUMENT, "mlp_linear_bf16: bad arguments");
    if (M == 0) return VLX_B200_OK;
    const dim3 grid((N + kMmaTile - 1) / kMmaTile, (M + kMmaTile - 1) / kMmaTile);
    gemm_bf16_mma_kernel<<<grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        X, static_cast<const __nv_bfloat16*>(W_bf16), b, Y, M, N, K, silu_act);
    MLP_CHECK();
    return VLX_B200_OK;
}

int vlx_b200_mlp_linear_backward(const float* X, const float* W, const float* Z, const float* dY, float* dZ,
                                 float* dX, float* dW, float* db, int M, int K, int N, int silu_act, void* stream)
{
    if (!X || !W || !dY || !dW || !db || (silu_act && (!Z || !dZ)) || M < 1 || K < 1 || N < 1)
        return vlx_b200_set_error_internal(VLX_B200_ERR_ARGUMENT, "mlp_linear_backward: bad arguments");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t n = (size_t)M * N;
    const float* g = dY;
    if (silu_act) {
        silu_backward_kernel<<<grid_1d(n), 256, 0, st>>>(dY, Z, dZ, n);
        g = dZ;
    }
    // dW[N, K] = g^T X: rows n, reduction over m
    gemm_kernel<float><<<dim3((K + kTile - 1) / kTile, (N + kTile - 1) / kTile), 256, 0, st>>>(
        g, 1, N, X, K, 1, nullptr, nullptr, dW, N, K, M, 0, 0);
    column_sum_kernel<<<(N + 31) / 32, dim3(32, 8), 0, st>>>(g, db, M, N);
    // dX[M, K] = g W
    if (dX)
        gemm_kernel<float><<<dim3((K + kTile - 1) / kTile, (M + kTile - 1) / kTile), 256, 0, st>>>(
            g, N, 1, W, K, 1, nullptr, nullptr, dX, M, K, N, 0, 0);
    MLP_CHECK();
    return VLX_B200_OK;
}

int vlx_b200_mlp_mse(const float* Y, const float* T, const float* mask, float* dY, double* d_loss_sum, long long n,
                     double count, void* stream)
{
    if (!Y || !T || !mask || !dY || !d_loss_sum || n < 0 || !(count > 0.0))
        return vlx_b200_set_error_internal(VLX_B200_ERR_ARGUMENT, "mlp_mse: bad arguments");
    if (n == 0) return VLX_B200_OK;
    mse_kernel<<<grid_1d(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(Y, T, mask, dY, d_loss_sum, (size_t)n,
                                                                         (float)(1.0 / count));
    MLP_CHECK();
    return VLX_B200_OK;
}

int vlx_b200_adam_step(float* params, const float* grads, float* m, float* v, long long n, float lr, float beta1,
                       float beta2, float eps, int step, void* stream)
{
    if (!params || !grads || !m || !v || n < 0 || step < 1)
        return vlx_b200_set_error_internal(VLX_B200_ERR_ARGUMENT, "adam_step: bad arguments");
    if (n == 0) return VLX_B200_OK;
    const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
    adam_kernel<<<grid_1d(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(params, grads, m, v, (size_t)n, lr, beta1,
                                                                          beta2, eps, c1, c2);
    MLP_CHECK();
    return VLX_B200_OK;
}

int vlx_b200_to_bf16(const float* x, void* y, long long n, void* stream)
{
    if (!x || !y || n < 0) return vlx_b200_set_error_internal(VLX_B200_ERR_ARGUMENT, "to_bf16: bad arguments");
    if (n == 0) return VLX_B200_OK;
    to_bf16_kernel<<<grid_1d(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(x, static_cast<__nv_bfloat16*>(y),
                                                                             (size_t)n);
    MLP_CHECK();
    return VLX_B200_OK;
}

}  // extern "C"
