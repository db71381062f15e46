// Training of the advection surrogate's MLP (388 -> 256 -> 256 -> 256 -> 3, GELU tanh form, the
// outputs multiplied by the stencil's uniformity gate) with the library's own kernels: the forward
// pass, the mean-squared loss against the targets, the backward pass through all four layers and
// an Adam update. The GEMMs of layers 1-3 (forward, input gradients) and every weight gradient
// run on the tcgen05 tensor cores with BF16 operands and FP32 accumulation; the three-output layer
// 4 forward and input gradient, the loss, GELU derivatives, bias sums and Adam are FP32 on the
// CUDA cores. The parameters use the flat layout of
// wacomm_b200_set_surrogate (w1 [256][388], b1, w2 [256][256], b2, w3, b3, w4 [3][256], b4), so
// trained weights go to the inference kernels unchanged.
//
// The tensor-core GEMM covers the three products of a layer: the forward Z = X W^T (bias and GELU
// fused into its epilogue), the input gradient dX = dZ W, and the weight gradient dW = dZ^T X (the
// reduction over the batch, split over the SMs and summed in a fixed order). A tiled FP32 GEMM on
// the CUDA cores serves layer 4, whose three outputs are too few for a tensor-core tile.
#include <cmath>

#include <cuda_bf16.h>

#include "engine.h"
#include "umma.cuh"

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

// ------------------------------------------------------------------ tcgen05 GEMM (layers 1-3)
//
// C[M][N] = sum_k a(m, k) b(n, k), a(m, k) = A[m sam + k sak], b(n, k) = B[n sbn + k sbk]: BF16
// operands, FP32 accumulation in tensor memory. A block owns a 128-row by up to 256-column tile
// and a range of K; its 256 threads read the FP32 operands (coalesced along whichever index is
// contiguous in memory, so transposed operands need no separate pass), round them to BF16 and
// write them into shared memory in the K-major 128-byte-swizzle layout of umma.cuh, two K-blocks
// of 64 in flight: while one thread issues the four MMAs of block kb, the others fill block kb+1.
// Epilogues: 0 store; 1 add bias[n]; 2 add bias[n], store Z and GELU(Z); 3 store the block's
// partial sum of its K range to partial[blockIdx.z] (reduced afterwards in a fixed order, so the
// weight gradients are reproducible bit for bit).
constexpr int UM = 128, UK = 64, UN = 256, UTHREADS = 256;
constexpr uint32_t UA_BYTES = UM * 128, UB_BYTES = UN * 128;
constexpr size_t USMEM = 2 * ((size_t)UA_BYTES + UB_BYTES) + 1024;

struct UmmaGemm {
    int M, N, K, kPerSplit;
    const float *A;
    long long sam, sak;
    const float *B;
    long long sbn, sbk;
    const float *bias;
    float *C, *H, *partial;
    int ldc;
    int *err;
};

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t *>(&v);
}

__device__ __forceinline__ uint4 pack8(float4 a, float4 b) {
    return make_uint4(pack_bf16x2(a.x, a.y), pack_bf16x2(a.z, a.w), pack_bf16x2(b.x, b.y),
                      pack_bf16x2(b.z, b.w));
}

// One rows x 64 operand block, a(r, k) = src[r sRow + k sK], rounded to BF16 into its swizzled
// shared-memory image; rows at or past `rows` and k at or past kEnd read as zero. Three ways to
// read it, chosen per block: with k contiguous, each item is a row's 16-byte chunk of 8 k values
// (two float4 loads); with rows contiguous, each item is 4 rows x 8 k values (eight float4 loads
// along the rows, written as four chunks); otherwise scalar pairs. Every thread issues its loads
// before its stores, so many loads are in flight.
__device__ __forceinline__ void stage_block(uint8_t *dst, int rowsInBlock, const float *src,
                                            long long sRow, long long sK, int row0, int rows,
                                            int k0, int kEnd, int tid) {
    const bool aligned = (((uintptr_t)src) & 15) == 0 && k0 + UK <= kEnd;
    if (aligned && sK == 1 && (sRow & 3) == 0) {
        const int items = rowsInBlock * 8;
        for (int base = 0; base < items; base += 4 * UTHREADS) {
            float4 v[4][2];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int it = base + u * UTHREADS + tid, r = it >> 3, c = it & 7;
                v[u][0] = v[u][1] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (it < items && row0 + r < rows) {
                    const float4 *q =
                        reinterpret_cast<const float4 *>(src + (long long)(row0 + r) * sRow + k0 + c * 8);
                    v[u][0] = __ldg(q);
                    v[u][1] = __ldg(q + 1);
                }
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int it = base + u * UTHREADS + tid;
                if (it < items)
                    *reinterpret_cast<uint4 *>(dst + umma::sw128_offset(it >> 3, (it & 7) * 8)) =
                        pack8(v[u][0], v[u][1]);
            }
        }
        return;
    }
    if (aligned && sRow == 1 && (sK & 3) == 0 && (row0 & 3) == 0) {
        const int groups = (rowsInBlock + 3) / 4, items = groups * 8;
        for (int it = tid; it < items; it += UTHREADS) {
            const int g = it % groups, c = it / groups, r0 = 4 * g, gr0 = row0 + r0;
            float4 v[8];
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const float *col = src + (long long)(k0 + c * 8 + q) * sK;
                if (gr0 + 3 < rows) {
                    v[q] = __ldg(reinterpret_cast<const float4 *>(col + gr0));
                } else {
                    v[q].x = gr0 < rows ? __ldg(col + gr0) : 0.f;
                    v[q].y = gr0 + 1 < rows ? __ldg(col + gr0 + 1) : 0.f;
                    v[q].z = gr0 + 2 < rows ? __ldg(col + gr0 + 2) : 0.f;
                    v[q].w = 0.f;
                }
            }
            *reinterpret_cast<uint4 *>(dst + umma::sw128_offset(r0 + 0, c * 8)) =
                pack8(make_float4(v[0].x, v[1].x, v[2].x, v[3].x), make_float4(v[4].x, v[5].x, v[6].x, v[7].x));
            *reinterpret_cast<uint4 *>(dst + umma::sw128_offset(r0 + 1, c * 8)) =
                pack8(make_float4(v[0].y, v[1].y, v[2].y, v[3].y), make_float4(v[4].y, v[5].y, v[6].y, v[7].y));
            *reinterpret_cast<uint4 *>(dst + umma::sw128_offset(r0 + 2, c * 8)) =
                pack8(make_float4(v[0].z, v[1].z, v[2].z, v[3].z), make_float4(v[4].z, v[5].z, v[6].z, v[7].z));
            *reinterpret_cast<uint4 *>(dst + umma::sw128_offset(r0 + 3, c * 8)) =
                pack8(make_float4(v[0].w, v[1].w, v[2].w, v[3].w), make_float4(v[4].w, v[5].w, v[6].w, v[7].w));
        }
        return;
    }
    const int pairs = rowsInBlock * (UK / 2);
    for (int e = tid; e < pairs; e += UTHREADS) {
        int r, kp;
        if (sK == 1) {
            r = e / (UK / 2);
            kp = e % (UK / 2);
        } else {
            kp = e / rowsInBlock;
            r = e % rowsInBlock;
        }
        const int gr = row0 + r, gk = k0 + 2 * kp;
        float v0 = 0.f, v1 = 0.f;
        if (gr < rows) {
            const float *p = src + (long long)gr * sRow;
            if (gk < kEnd) v0 = __ldg(p + (long long)gk * sK);
            if (gk + 1 < kEnd) v1 = __ldg(p + (long long)(gk + 1) * sK);
        }
        *reinterpret_cast<uint32_t *>(dst + umma::sw128_offset(r, 2 * kp)) = pack_bf16x2(v0, v1);
    }
}

template <int EPI>
__global__ void __launch_bounds__(UTHREADS, 1) umma_gemm_kernel(const UmmaGemm g) {
    using namespace umma;
    extern __shared__ uint8_t dynSmem[];
    uint8_t *sA = reinterpret_cast<uint8_t *>(((uintptr_t)dynSmem + 1023) & ~(uintptr_t)1023);
    uint8_t *sB = sA + 2 * UA_BYTES;
    __shared__ __align__(8) uint64_t freed[2], accFull;
    __shared__ uint32_t tmemSlot;
    __shared__ int abortFlag;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * UM, n0 = blockIdx.x * UN;
    const int nLeft = g.N - n0;
    const int nTile = nLeft >= UN ? UN : ((nLeft + 15) / 16) * 16;  // MMA N: multiple of 16
    const int kBegin = blockIdx.z * g.kPerSplit;
    const int kEnd = min(g.K, kBegin + g.kPerSplit);
    const int nkb = kEnd > kBegin ? (kEnd - kBegin + UK - 1) / UK : 0;
    if (tid == 0) {
        mbar_init(&freed[0], 1);
        mbar_init(&freed[1], 1);
        mbar_init(&accFull, 1);
        abortFlag = 0;
        fence_barrier_init();
    }
    if (warp == 0) tmem_alloc(&tmemSlot, UN);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = tmemSlot;
    const uint32_t idesc = idesc_bf16(UM, nTile);
    bool ok = true;
    for (int kb = 0; kb < nkb && ok; kb++) {
        const int s = kb & 1;
        // the MMAs of block kb-2 read this stage: wait for their commit
        if (kb >= 2) ok = mbar_wait(&freed[s], (uint32_t)(((kb >> 1) + 1) & 1), &abortFlag);
        __syncwarp();
        if (!ok) break;
        const int k0 = kBegin + kb * UK;
        stage_block(sA + s * UA_BYTES, UM, g.A, g.sam, g.sak, m0, g.M, k0, kEnd, tid);
        stage_block(sB + s * UB_BYTES, nTile, g.B, g.sbn, g.sbk, n0, g.N, k0, kEnd, tid);
        fence_async_shared();
        fence_before_sync();
        __syncthreads();
        fence_after_sync();
        if (abortFlag) {
            ok = false;
            break;
        }
        if (tid == 0) {
#pragma unroll
            for (int ks = 0; ks < UK / 16; ks++)
                mma_bf16(tmem, desc_sw128(smem_u32(sA + s * UA_BYTES + ks * 32)),
                         desc_sw128(smem_u32(sB + s * UB_BYTES + ks * 32)), idesc, (kb | ks) != 0);
            mma_commit(&freed[s]);
        }
    }
    // every MMA issued so far lands before the accumulator is read (or the block exits)
    if (tid == 0) mma_commit(&accFull);
    const bool done = mbar_wait_bounded(&accFull, 0);
    __syncwarp();
    fence_after_sync();
    const bool valid = ok && done && !abortFlag;
    if (valid) {
        const int quarter = warp & 3, half = warp >> 2;
        const int m = m0 + quarter * 32 + lane;
        for (int c0 = half * (UN / 2); c0 < (half + 1) * (UN / 2) && c0 < nTile; c0 += 32) {
            float v[32];
            if (nkb > 0) {
                tmem_ld32(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)c0, v);
            } else {
#pragma unroll
                for (int c = 0; c < 32; c++) v[c] = 0.f;
            }
            if (m >= g.M) continue;
#pragma unroll
            for (int c = 0; c < 32; c++) {
                const int n = n0 + c0 + c;
                if (n >= g.N) break;
                float z = v[c];
                if (EPI == 3) {
                    g.partial[((size_t)blockIdx.z * g.M + m) * g.N + n] = z;
                    continue;
                }
                if (EPI >= 1) z += __ldg(g.bias + n);
                g.C[(size_t)m * g.ldc + n] = z;
                if (EPI == 2) g.H[(size_t)m * g.ldc + n] = gelu_exact_tanh(z, nullptr);
            }
        }
    }
    if (!valid && tid == 0) atomicOr(g.err, 1);
    fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        fence_after_sync();
        tmem_dealloc(tmem, UN);
    }
}

// out[m][n] = sum over the splits z (in order) of partial[z][m][n].
__global__ void split_sum_kernel(const float *partial, int splits, size_t cells, float *out) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < cells;
         e += (size_t)gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int z = 0; z < splits; z++) s += partial[(size_t)z * cells + e];
        out[e] = s;
    }
}

// Floats of the weight-gradient partial sums: at most 148 / (output tiles) splits of M x N, the
// most for a 256 x 256 weight (two tiles, 74 splits).
constexpr size_t UMMA_PARTIAL_FLOATS = (size_t)(148 / 2) * T_HID * T_HID;

cudaError_t umma_prepare() {
    static bool done[64] = {};
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    if (device >= 0 && device < 64 && done[device]) return cudaSuccess;
    for (auto fn : {umma_gemm_kernel<0>, umma_gemm_kernel<1>, umma_gemm_kernel<2>, umma_gemm_kernel<3>}) {
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)USMEM);
        if (e != cudaSuccess) return e;
    }
    if (device >= 0 && device < 64) done[device] = true;
    return cudaSuccess;
}

// C (M x N, leading dimension ldc) from a(m, k) = A[m sam + k sak] and b(n, k) = B[n sbn + k sbk]
// on the tensor cores. EPI 3 (a reduction over a long K, the batch) splits K over about one block
// per SM and sums the splits in order into C (ldc must be N).
template <int EPI>
cudaError_t umma_gemm(int M, int N, int K, const float *A, long long sam, long long sak,
                      const float *B, long long sbn, long long sbk, const float *bias, float *C,
                      float *H, int ldc, float *partial, int *err, cudaStream_t stream) {
    cudaError_t e = umma_prepare();
    if (e != cudaSuccess) return e;
    UmmaGemm g;
    g.M = M;
    g.N = N;
    g.K = K;
    g.A = A;
    g.sam = sam;
    g.sak = sak;
    g.B = B;
    g.sbn = sbn;
    g.sbk = sbk;
    g.bias = bias;
    g.C = C;
    g.H = H;
    g.partial = partial;
    g.ldc = ldc;
    g.err = err;
    const int tilesN = (N + UN - 1) / UN, tilesM = (M + UM - 1) / UM;
    int splits = 1;
    g.kPerSplit = ((K + UK - 1) / UK) * UK;
    if (EPI == 3) {
        splits = 148 / (tilesN * tilesM);
        if (splits < 1) splits = 1;
        const int kBlocks = (K + UK - 1) / UK;
        if (splits > kBlocks) splits = kBlocks > 0 ? kBlocks : 1;
        g.kPerSplit = ((kBlocks + splits - 1) / splits) * UK;
        splits = (K + g.kPerSplit - 1) / g.kPerSplit;
        if (splits < 1) splits = 1;
        if ((size_t)splits * M * N > UMMA_PARTIAL_FLOATS || ldc != N) return cudaErrorInvalidValue;
    }
    dim3 grid(tilesN, tilesM, splits);
    umma_gemm_kernel<EPI><<<grid, UTHREADS, USMEM, stream>>>(g);
    e = cudaGetLastError();
    if (e != cudaSuccess || EPI != 3) return e;
    const size_t cells = (size_t)M * N;
    split_sum_kernel<<<(int)((cells + 255) / 256), 256, 0, stream>>>(partial, splits, cells, C);
    return cudaGetLastError();
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

// db[n] = sum over the batch of dZ[b][n], in two passes with a fixed order: block (x, y) sums the
// 32 columns 32x.. over the rows of chunk y (warp w takes rows w, w + 8, ..., its lanes one column
// each, so every row is read as one 128-byte line), adding its 8 warps' sums in order into
// partial[y][n]; then the chunks are added in order.
constexpr int COLUMN_CHUNKS = 64;

__global__ void column_partial_kernel(const float *dZ, int batch, int N, float *partial) {
    __shared__ float warpSum[8][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n = blockIdx.x * 32 + lane;
    const int per = (batch + COLUMN_CHUNKS - 1) / COLUMN_CHUNKS;
    const int b0 = blockIdx.y * per, b1 = min(batch, b0 + per);
    float sum = 0.f;
    if (n < N)
        for (int b = b0 + warp; b < b1; b += 8) sum += dZ[(size_t)b * N + n];
    warpSum[warp][lane] = sum;
    __syncthreads();
    if (warp == 0 && n < N) {
        float total = 0.f;
        for (int w = 0; w < 8; w++) total += warpSum[w][lane];
        partial[(size_t)blockIdx.y * N + n] = total;
    }
}

__global__ void column_final_kernel(const float *partial, int N, float *db) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float total = 0.f;
    for (int c = 0; c < COLUMN_CHUNKS; c++) total += partial[(size_t)c * N + n];
    db[n] = total;
}

void column_sum(const float *dZ, int batch, int N, float *partial, float *db, cudaStream_t stream) {
    column_partial_kernel<<<dim3((N + 31) / 32, COLUMN_CHUNKS), 256, 0, stream>>>(dZ, batch, N, partial);
    column_final_kernel<<<(N + 255) / 256, 256, 0, stream>>>(partial, N, db);
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
    // an error word (padded to 16 bytes), the weight-gradient partial sums, then the
    // activations and gradients of the batch
    return 4 + UMMA_PARTIAL_FLOATS + (size_t)batch * (T_IN + 6 * T_HID + 2 * T_OUT + 2 * T_HID);
}

cudaError_t mlp_train_step(const float *stencil, const float *particle, const float *gate,
                           const float *target, int batch, float *params, float *grads, float *m,
                           float *v, float *work, float *loss, int step, float lr, bool update,
                           cudaStream_t stream) {
    const int B = batch;
    int *err = reinterpret_cast<int *>(work);
    float *partial = work + 4;
    float *X = partial + UMMA_PARTIAL_FLOATS, *Z1 = X + (size_t)B * T_IN,
          *H1 = Z1 + (size_t)B * T_HID, *Z2 = H1 + (size_t)B * T_HID, *H2 = Z2 + (size_t)B * T_HID,
          *Z3 = H2 + (size_t)B * T_HID, *H3 = Z3 + (size_t)B * T_HID, *O = H3 + (size_t)B * T_HID,
          *dO = O + (size_t)B * T_OUT, *dA = dO + (size_t)B * T_OUT, *dB = dA + (size_t)B * T_HID;
    const float *W1 = params + OFF_TW1, *W2 = params + OFF_TW2, *W3 = params + OFF_TW3,
                *W4 = params + OFF_TW4;
    cudaError_t e = cudaMemsetAsync(loss, 0, sizeof(float), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(grads, 0, T_PARAMS * sizeof(float), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), stream);
    if (e != cudaSuccess) return e;
    concat_kernel<<<blocks_for((size_t)B * T_IN), 256, 0, stream>>>(stencil, particle, B, X);
#define UMMA(call)                              \
    do {                                        \
        if ((e = (call)) != cudaSuccess) return e; \
    } while (0)
    // forward: layers 1-3 on the tensor cores (BF16 operands, bias and GELU in the epilogue),
    // layer 4 (three outputs) on the CUDA cores
    UMMA(umma_gemm<2>(B, T_HID, T_IN, X, T_IN, 1, W1, T_IN, 1, params + OFF_TB1, Z1, H1, T_HID,
                      partial, err, stream));
    UMMA(umma_gemm<2>(B, T_HID, T_HID, H1, T_HID, 1, W2, T_HID, 1, params + OFF_TB2, Z2, H2,
                      T_HID, partial, err, stream));
    UMMA(umma_gemm<2>(B, T_HID, T_HID, H2, T_HID, 1, W3, T_HID, 1, params + OFF_TB3, Z3, H3,
                      T_HID, partial, err, stream));
    gemm<false, true, 1>(B, T_OUT, T_HID, H3, T_HID, W4, T_HID, params + OFF_TB4, O, nullptr, T_OUT, stream);
    loss_kernel<<<blocks_for((size_t)B * T_OUT), 256, 0, stream>>>(O, gate, target, B, dO, loss);
    // backward, layer 4: dW4 = dO^T H3 (tensor cores, reduction over the batch), dA = dO W4
    UMMA(umma_gemm<3>(T_OUT, T_HID, B, dO, 1, T_OUT, H3, 1, T_HID, nullptr, grads + OFF_TW4,
                      nullptr, T_HID, partial, err, stream));
    column_sum(dO, B, T_OUT, partial, grads + OFF_TB4, stream);
    gemm<false, false, 0>(B, T_HID, T_OUT, dO, T_OUT, W4, T_HID, nullptr, dA, nullptr, T_HID, stream);
    // layer 3: dZ3 = dA GELU'(Z3); dW3 = dZ3^T H2; dB = dZ3 W3
    gelu_backward_kernel<<<blocks_for((size_t)B * T_HID), 256, 0, stream>>>(Z3, dA, (size_t)B * T_HID);
    UMMA(umma_gemm<3>(T_HID, T_HID, B, dA, 1, T_HID, H2, 1, T_HID, nullptr, grads + OFF_TW3,
                      nullptr, T_HID, partial, err, stream));
    column_sum(dA, B, T_HID, partial, grads + OFF_TB3, stream);
    UMMA(umma_gemm<0>(B, T_HID, T_HID, dA, T_HID, 1, W3, 1, T_HID, nullptr, dB, nullptr, T_HID,
                      partial, err, stream));
    // layer 2
    gelu_backward_kernel<<<blocks_for((size_t)B * T_HID), 256, 0, stream>>>(Z2, dB, (size_t)B * T_HID);
    UMMA(umma_gemm<3>(T_HID, T_HID, B, dB, 1, T_HID, H1, 1, T_HID, nullptr, grads + OFF_TW2,
                      nullptr, T_HID, partial, err, stream));
    column_sum(dB, B, T_HID, partial, grads + OFF_TB2, stream);
    UMMA(umma_gemm<0>(B, T_HID, T_HID, dB, T_HID, 1, W2, 1, T_HID, nullptr, dA, nullptr, T_HID,
                      partial, err, stream));
    // layer 1 (no input gradient)
    gelu_backward_kernel<<<blocks_for((size_t)B * T_HID), 256, 0, stream>>>(Z1, dA, (size_t)B * T_HID);
    UMMA(umma_gemm<3>(T_HID, T_IN, B, dA, 1, T_HID, X, 1, T_IN, nullptr, grads + OFF_TW1,
                      nullptr, T_IN, partial, err, stream));
    column_sum(dA, B, T_HID, partial, grads + OFF_TB1, stream);
#undef UMMA
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
