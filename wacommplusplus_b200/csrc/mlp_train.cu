// Training of the advection surrogate's MLP (388 -> 256 -> 256 -> 256 -> 3, GELU tanh form, the
// outputs multiplied by the stencil's uniformity gate) with the library's own kernels: the forward
// pass, the mean-squared loss against the targets, the backward pass through all four layers and
// an Adam update, in FP32 on the CUDA cores. The parameters use the flat layout of
// wacomm_b200_set_surrogate (w1 [256][388], b1, w2 [256][256], b2, w3, b3, w4 [3][256], b4), so
// trained weights go to the inference kernels unchanged.
//
// One tiled GEMM kernel covers the three products of a layer: the forward Z = X W^T (bias and
// GELU fused into its epilogue), the input gradient dX = dZ W, and the weight gradient
// dW = dZ^T X (the reduction over the batch).
#include <cmath>

#include "engine.h"

namespace wb {
namespace {

constexpr int T_HID = 256, T_STENCIL = 384, T_PARTICLE = 4, T_IN = T_STENCIL + T_PARTICLE,
              T_OUT = 3;
constexpr size_t OFF_TW1 = 0, OFF_TB1 = OFF_TW1 + (size_t)T_HID * T_IN, OFF_TW2 = OFF_TB1 + T_HID,
                 OFF_TB2 = OFF_TW2 + (size_t)T_HID * T_HID, OFF_TW3 = OFF_TB2 + T_HID,
                 OFF_TB3 = OFF_TW3 + (size_t)T_HID * T_HID, OFF_TW4 = OFF_TB3 + T_HID,
                 OFF_TB4 = OFF_TW4 + (size_t)T_OUT * T_HID, T_PARAMS = OFF_TB4 + T_OUT;

__device__ __forceinline__ float gelu_exact_tanh(float x, float *derivative) {
    const float c0 = 0.7978845608028654f, c1 = 0.044715f;
    const float t = tanhf(c0 * (x + c1 * x * x * x));
    if (derivative) *derivative = 0.5f * (1.f + t) + 0.5f * x * (1.f - t * t) * c0 * (1.f + 3.f * c1 * x * x);
    return 0.5f * x * (1.f + t);
}

// C[M][N] = sum_k a(m, k) b(k, n) with a(m, k) = TA ? A[k lda + m] : A[m lda + k] and
// b(k, n) = TB ? B[n ldb + k] : B[k ldb + n]. EPI 0: store; 1: add bias[n] and store; 2: add
// bias[n], store Z and GELU(Z) into H; 3: add into C atomically (the K range split over
// gridDim.z, C zeroed beforehand). 64 x 64 tiles, 256 threads of 4 x 4 outputs, K steps of 16;
// each operand tile is read with its contiguous index fastest.
template <bool TA, bool TB, int EPI>
__global__ void __launch_bounds__(256) gemm_kernel(int M, int N, int K, const float *A, int lda,
                                                   const float *B, int ldb, const float *bias,
                                                   float *C, float *H, int ldc) {
    __shared__ float As[16][64 + 1], Bs[16][64 + 1];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
    const int kPer = ((K + gridDim.z - 1) / gridDim.z + 15) / 16 * 16;
    const int kBegin = blockIdx.z * kPer, kEnd = min(K, kBegin + kPer);
    float acc[4][4] = {};
    for (int k0 = kBegin; k0 < kEnd; k0 += 16) {
        for (int e = threadIdx.x; e < 16 * 64; e += 256) {
            // A: m contiguous when transposed, k contiguous otherwise
            const int kk = TA ? e / 64 : e % 16, r = TA ? e % 64 : e / 16;
            const int m = m0 + r, k = k0 + kk;
            As[kk][r] = (m < M && k < kEnd) ? (TA ? A[(size_t)k * lda + m] : A[(size_t)m * lda + k])
                                            : 0.f;
        }
        for (int e = threadIdx.x; e < 16 * 64; e += 256) {
            // B: k contiguous when transposed, n contiguous otherwise
            const int kk = TB ? e % 16 : e / 64, r = TB ? e / 16 : e % 64;
            const int n = n0 + r, k = k0 + kk;
            Bs[kk][r] = (n < N && k < kEnd) ? (TB ? B[(size_t)n * ldb + k] : B[(size_t)k * ldb + n])
                                            : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; kk++) {
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
            float z = acc[i][j];
            if (EPI == 3) {
                atomicAdd(C + (size_t)m * ldc + n, z);
                continue;
            }
            if (EPI >= 1) z += bias[n];
            C[(size_t)m * ldc + n] = z;
            if (EPI == 2) H[(size_t)m * ldc + n] = gelu_exact_tanh(z, nullptr);
        }
    }
}

template <bool TA, bool TB, int EPI>
void gemm(int M, int N, int K, const float *A, int lda, const float *B, int ldb, const float *bias,
          float *C, float *H, int ldc, cudaStream_t stream) {
    // the batch reductions (EPI 3) are split so that about two blocks run per SM
    const int tiles = ((N + 63) / 64) * ((M + 63) / 64);
    int splits = EPI == 3 ? (296 + tiles - 1) / tiles : 1;
    if (splits > (K + 63) / 64) splits = (K + 63) / 64 > 0 ? (K + 63) / 64 : 1;
    dim3 grid((N + 63) / 64, (M + 63) / 64, splits);
    gemm_kernel<TA, TB, EPI><<<grid, 256, 0, stream>>>(M, N, K, A, lda, B, ldb, bias, C, H, ldc);
}

// X = [stencil | particle], [batch][388].
__global__ void concat_kernel(const float *stencil, const float *particle, int batch, float *X) {
    const size_t total = (size_t)batch * T_IN;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
         e += (size_t)gridDim.x * blockDim.x) {
        const size_t b = e / T_IN, c = e % T_IN;
        X[e] = c < T_STENCIL ? stencil[b * T_STENCIL + c] : particle[b * T_PARTICLE + (c - T_STENCIL)];
    }
}

// Y = O g; loss = mean over batch and outputs of (Y - target)^2; dO = 2 (Y - target) g / (3 batch).
__global__ void loss_kernel(const float *O, const float *gate, const float *target, int batch,
                            float *dO, float *loss) {
    __shared__ float partial[256];
    float sum = 0.f;
    const float scale = 1.f / (3.f * batch);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < batch * T_OUT; e += gridDim.x * blockDim.x) {
        const float g = gate[e / T_OUT];
        const float d = O[e] * g - target[e];
        sum += d * d;
        dO[e] = 2.f * d * g * scale;
    }
    partial[threadIdx.x] = sum;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) partial[threadIdx.x] += partial[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss, partial[0] * scale);
}

// dZ = dH * GELU'(Z), in place in dH.
__global__ void gelu_backward_kernel(const float *Z, float *dH, size_t n) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x) {
        float d;
        gelu_exact_tanh(Z[e], &d);
        dH[e] *= d;
    }
}

// db[n] = sum over the batch of dZ[b][n]; one block per column.
__global__ void column_sum_kernel(const float *dZ, int batch, int N, float *db) {
    __shared__ float partial[256];
    const int n = blockIdx.x;
    float sum = 0.f;
    for (int b = threadIdx.x; b < batch; b += blockDim.x) sum += dZ[(size_t)b * N + n];
    partial[threadIdx.x] = sum;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) partial[threadIdx.x] += partial[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) db[n] = partial[0];
}

// Adam (beta1 0.9, beta2 0.999, eps 1e-8, bias-corrected at `step`).
__global__ void adam_kernel(float *p, const float *g, float *m, float *v, size_t n, float lr,
                            float c1, float c2) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x) {
        const float gi = g[e];
        const float mi = 0.9f * m[e] + 0.1f * gi, vi = 0.999f * v[e] + 0.001f * gi * gi;
        m[e] = mi;
        v[e] = vi;
        p[e] -= lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
    }
}

int blocks_for(size_t n) {
    const size_t b = (n + 255) / 256;
    return (int)(b < 148 * 8 ? (b > 0 ? b : 1) : 148 * 8);
}

}  // namespace

size_t mlp_train_work_floats(int batch) {
    return (size_t)batch * (T_IN + 6 * T_HID + 2 * T_OUT + 2 * T_HID);
}

cudaError_t mlp_train_step(const float *stencil, const float *particle, const float *gate,
                           const float *target, int batch, float *params, float *grads, float *m,
                           float *v, float *work, float *loss, int step, float lr, bool update,
                           cudaStream_t stream) {
    const int B = batch;
    float *X = work, *Z1 = X + (size_t)B * T_IN, *H1 = Z1 + (size_t)B * T_HID,
          *Z2 = H1 + (size_t)B * T_HID, *H2 = Z2 + (size_t)B * T_HID, *Z3 = H2 + (size_t)B * T_HID,
          *H3 = Z3 + (size_t)B * T_HID, *O = H3 + (size_t)B * T_HID, *dO = O + (size_t)B * T_OUT,
          *dA = dO + (size_t)B * T_OUT, *dB = dA + (size_t)B * T_HID;
    const float *W1 = params + OFF_TW1, *W2 = params + OFF_TW2, *W3 = params + OFF_TW3,
                *W4 = params + OFF_TW4;
    cudaError_t e = cudaMemsetAsync(loss, 0, sizeof(float), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(grads, 0, T_PARAMS * sizeof(float), stream);
    if (e != cudaSuccess) return e;
    concat_kernel<<<blocks_for((size_t)B * T_IN), 256, 0, stream>>>(stencil, particle, B, X);
    // forward
    gemm<false, true, 2>(B, T_HID, T_IN, X, T_IN, W1, T_IN, params + OFF_TB1, Z1, H1, T_HID, stream);
    gemm<false, true, 2>(B, T_HID, T_HID, H1, T_HID, W2, T_HID, params + OFF_TB2, Z2, H2, T_HID, stream);
    gemm<false, true, 2>(B, T_HID, T_HID, H2, T_HID, W3, T_HID, params + OFF_TB3, Z3, H3, T_HID, stream);
    gemm<false, true, 1>(B, T_OUT, T_HID, H3, T_HID, W4, T_HID, params + OFF_TB4, O, nullptr, T_OUT, stream);
    loss_kernel<<<blocks_for((size_t)B * T_OUT), 256, 0, stream>>>(O, gate, target, B, dO, loss);
    // backward: layer 4
    gemm<true, false, 3>(T_OUT, T_HID, B, dO, T_OUT, H3, T_HID, nullptr, grads + OFF_TW4, nullptr, T_HID, stream);
    column_sum_kernel<<<T_OUT, 256, 0, stream>>>(dO, B, T_OUT, grads + OFF_TB4);
    gemm<false, false, 0>(B, T_HID, T_OUT, dO, T_OUT, W4, T_HID, nullptr, dA, nullptr, T_HID, stream);
    // layer 3
    gelu_backward_kernel<<<blocks_for((size_t)B * T_HID), 256, 0, stream>>>(Z3, dA, (size_t)B * T_HID);
    gemm<true, false, 3>(T_HID, T_HID, B, dA, T_HID, H2, T_HID, nullptr, grads + OFF_TW3, nullptr, T_HID, stream);
    column_sum_kernel<<<T_HID, 256, 0, stream>>>(dA, B, T_HID, grads + OFF_TB3);
    gemm<false, false, 0>(B, T_HID, T_HID, dA, T_HID, W3, T_HID, nullptr, dB, nullptr, T_HID, stream);
    // layer 2
    gelu_backward_kernel<<<blocks_for((size_t)B * T_HID), 256, 0, stream>>>(Z2, dB, (size_t)B * T_HID);
    gemm<true, false, 3>(T_HID, T_HID, B, dB, T_HID, H1, T_HID, nullptr, grads + OFF_TW2, nullptr, T_HID, stream);
    column_sum_kernel<<<T_HID, 256, 0, stream>>>(dB, B, T_HID, grads + OFF_TB2);
    gemm<false, false, 0>(B, T_HID, T_HID, dB, T_HID, W2, T_HID, nullptr, dA, nullptr, T_HID, stream);
    // layer 1 (no input gradient)
    gelu_backward_kernel<<<blocks_for((size_t)B * T_HID), 256, 0, stream>>>(Z1, dA, (size_t)B * T_HID);
    gemm<true, false, 3>(T_HID, T_IN, B, dA, T_HID, X, T_IN, nullptr, grads + OFF_TW1, nullptr, T_IN, stream);
    column_sum_kernel<<<T_HID, 256, 0, stream>>>(dA, B, T_HID, grads + OFF_TB1);
    if (update) {
        const float c1 = 1.f - powf(0.9f, (float)step), c2 = 1.f - powf(0.999f, (float)step);
        adam_kernel<<<blocks_for(T_PARAMS), 256, 0, stream>>>(params, grads, m, v, T_PARAMS, lr, c1, c2);
    }
    return cudaGetLastError();
}

}  // namespace wb

extern "C" size_t wacomm_b200_mlp_train_work_floats(int batch) {
    return batch > 0 ? wb::mlp_train_work_floats(batch) : 0;
}

extern "C" int wacomm_b200_mlp_train_step(const float *stencil, const float *particle,
                                          const float *gate, const float *target, int batch,
                                          float *params, float *grads, float *m, float *v,
                                          float *work, float *loss, int step, float lr, int update,
                                          void *stream) {
    if (!stencil || !particle || !gate || !target || batch <= 0 || !params || !grads || !work ||
        !loss || (update && (!m || !v || step < 1)))
        return WACOMM_B200_ERR_ARGUMENT;
    const cudaError_t e = wb::mlp_train_step(stencil, particle, gate, target, batch, params, grads,
                                             m, v, work, loss, step, lr, update != 0,
                                             static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? WACOMM_B200_OK : WACOMM_B200_ERR_CUDA;
}
