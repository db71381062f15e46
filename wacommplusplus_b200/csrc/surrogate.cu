// Learned one-interval advection surrogate on the tensor cores (tcgen05, sm_100a).
//
// The MLP 388 -> 256 -> 256 -> 256 -> 3 (GELU, tanh form) is split in two kernels:
//
// * surrogate_cell_kernel: the stencil part of layer 1 depends only on the cell and level a
//   particle starts in, so it is evaluated once per cell-level as a GEMM
//   [cell-levels x 384] x [384 x 256] (BF16 operands, FP32 accumulation in TMEM) and stored as
//   FP16 pre-activations z, together with the uniformity gate of the stencil;
// * surrogate_step_kernel: per tile of 128 particles (taken in slot order: the particle state is
//   read coalesced, and the per-cell z rows and corner records it gathers stay in L2), layer 1 is
//   finished on the CUDA cores from z and the four particle features, layers 2 and 3 run as two
//   [128 x 256] x [256 x 256] tcgen05 GEMMs with the weights streamed through a 2-stage
//   shared-memory ring by bulk copies, each accumulating onto its bias (stored into TMEM by the
//   rows), and layer 3's epilogue folds in the 3-output layer 4. The three outputs and a row tag
//   go to rows[] per work item;
// * surrogate_post_kernel: one thread per work item applies the displacement with the closures in
//   closed form, updates the state and the fused concentration, and appends the particles the
//   surrogate does not cover to a fallback list for the plain kernel. Run apart from the GEMM
//   pipeline, its dependent loads overlap across a full SM of warps instead of stalling the row
//   warps of the step kernel.
//
// Warp roles of the step kernel (576 threads): warps 0-15 own the tile's rows (warp w holds rows
// 32(w%4).. -- the TMEM lane quarter it may access -- and columns 64(w/4).. of the accumulator),
// warp 16 streams weights, warp 17 issues the MMAs and owns the TMEM allocation. Every wait is bounded; a timeout raises an error flag and the block drains and
// exits.
#include <cstring>
#include <type_traits>

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "engine.h"
#include "move_kernels.cuh"
#include "umma.cuh"

namespace wb {

namespace {

constexpr int HID = 256;
constexpr int N_STENCIL = 384;
constexpr int N_INPUT = 388;
constexpr int TILE = 128;
constexpr uint32_t KBLOCK_A = TILE * 128;  // 16 KB: 128 rows x 64 BF16
constexpr uint32_t KBLOCK_W = HID * 128;   // 32 KB: 256 rows x 64 BF16
constexpr int CELL_KB = N_STENCIL / 64;    // 6
constexpr int HID_KB = HID / 64;           // 4
constexpr float W_FEATURE = 1000.f;        // 1 / (w feature scale, m/s)
constexpr float OUT_H = 100.f, OUT_V = 1.f;
constexpr float GATE_SIGMA = 0.01f;
constexpr int GATE_REF = (1 * 4 + 1) * 4 + 1;

// Offsets in the packed weight buffer (bytes; every block starts on 1024 bytes).
constexpr size_t OFF_W1 = 0;
constexpr size_t OFF_W2 = OFF_W1 + (size_t)CELL_KB * KBLOCK_W;
constexpr size_t OFF_W3 = OFF_W2 + (size_t)HID_KB * KBLOCK_W;
constexpr size_t OFF_B1 = OFF_W3 + (size_t)HID_KB * KBLOCK_W;
constexpr size_t OFF_B2 = OFF_B1 + 1024;
constexpr size_t OFF_B3 = OFF_B2 + 1024;
constexpr size_t OFF_W1P = OFF_B3 + 1024;
constexpr size_t OFF_W4 = OFF_W1P + 4096;
constexpr size_t OFF_B4 = OFF_W4 + 3072;
constexpr size_t PACKED_BYTES = OFF_B4 + 1024;

// Twice the GELU, tanh form, of two units: 2 h = x + x tanh(x (c0 + c1 x^2)), c0 = sqrt(2/pi),
// c1 = 0.044715 c0, with the packed FP32x2 multiply and multiply-add of sm_100 (half the
// instructions of the scalar form, the same roundings). The factor 1/2 of the GELU is carried by
// the consumer instead: the packed weights of layers 2, 3 and 4 are stored halved. Scaling by a
// power of two is exact in FP32 and BF16, so the rounded activations and every product are those
// of the unscaled network, one multiply fewer per unit.
__device__ __forceinline__ float2 gelu2_pair(float2 x) {
    const float2 p = __ffma2_rn(__fmul2_rn(x, x), make_float2(0.035677408136300125f, 0.035677408136300125f),
                                make_float2(0.7978845608028654f, 0.7978845608028654f));
    const float2 inner = __fmul2_rn(x, p);
    float2 t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t.x) : "f"(inner.x));
    asm("tanh.approx.f32 %0, %1;" : "=f"(t.y) : "f"(inner.y));
    return __ffma2_rn(x, t, x);
}

// Asynchronous 16-byte copy global -> shared (cached in L1), completed by cp_async_wait_all of
// the issuing thread.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(umma::smem_u32(smem)), "l"(gmem)
                 : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t *>(&v);
}

__device__ __forceinline__ uint8_t *align1024(uint8_t *p) {
    return (uint8_t *)(((uintptr_t)p + 1023) & ~(uintptr_t)1023);
}

// ------------------------------------------------------------------ per-cell layer 1

// What the displacement step needs from the forcing at a start cell-level, in one contiguous
// record: corners in the order (j,i), (j+1,i), (j+1,i+1), (j,i+1) of records t0 and t1.
struct alignas(16) CellCorners {
    float u[2][4], v[2][4];    // rho level kI
    float wU[2][4], wL[2][4];  // w levels kI and kI-1
    float zeta[2][4];
    float h[4];
    double invXdist, invYdist, depth;  // reciprocal cell metric, depthIntervals(kI)
    float gate;   // min(1, sigma / GATE_SIGMA): the weight of the network's correction
    float sigma;  // RMS deviation (m/s) of the stencil's u, v from the cell's own corner
};
static_assert(sizeof(CellCorners) == 208, "corner record layout");

struct CellArgs {
    int eta, xi, sW, sRho;
    long long nCL;  // (eta-1) * (xi-1) * (sW-1) cell-levels, index ((j*(xi-1)) + i)*(sW-1) + kI+sW-2
    const float *u0, *v0, *w0, *u1, *v1, *w1, *z0, *z1;
    const double *h, *depthIntervals;
    const double2 *metric;
    const uint8_t *weights;
    __half *z;             // [nCL][256]
    CellCorners *corners;  // [nCL]
    int *err;
};

constexpr size_t CELL_SMEM = (size_t)CELL_KB * KBLOCK_A + 2 * (size_t)KBLOCK_W + 1024;

__global__ void __launch_bounds__(128, 1) surrogate_cell_kernel(const CellArgs a) {
    using namespace umma;
    extern __shared__ uint8_t dynSmem[];
    uint8_t *sA = align1024(dynSmem);
    uint8_t *sW = sA + CELL_KB * KBLOCK_A;
    __shared__ __align__(8) uint64_t full[2], empty[2], accFull;
    __shared__ uint32_t tmemSlot;
    __shared__ int abortFlag;
    __shared__ float b1s[HID];
    const int tid = threadIdx.x, warp = tid >> 5;
    if (tid == 0) {
        for (int s = 0; s < 2; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&accFull, 1);
        abortFlag = 0;
        fence_barrier_init();
    }
    const float *b1 = reinterpret_cast<const float *>(a.weights + OFF_B1);
    for (int c = tid; c < HID; c += 128) b1s[c] = b1[c];
    if (warp == 0) tmem_alloc(&tmemSlot, 256);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = tmemSlot;
    const int levels = a.sW - 1;
    const long long nTiles = (a.nCL + TILE - 1) / TILE;
    const uint32_t idesc = idesc_bf16(TILE, HID);
    uint32_t g = 0;                      // weight blocks loaded so far (thread 0)
    int issued[2] = {-1, -1}, consumed[2] = {-1, -1};
    int it = 0;
    for (long long tile = blockIdx.x; tile < nTiles; tile += gridDim.x, it++) {
        // ---- gather: thread = row = cell-level
        const long long cl = tile * TILE + tid;
        float gsum = 0.f;
        if (cl < a.nCL) {
            const int lev = (int)(cl % levels);
            const long long cell = cl / levels;
            const int j = (int)(cell / (a.xi - 1)), i = (int)(cell % (a.xi - 1));
            const int kI = lev - (a.sW - 2);
#pragma unroll 1
            for (int q = 0; q < N_STENCIL / 8; q++) {
                const int f = q * 8;
                const int rec = f / 192, field = (f / 64) % 3, c = (f / 16) % 4, a0 = (f % 16) / 4;
                const float *src = rec == 0 ? (field == 0 ? a.u0 : field == 1 ? a.v0 : a.w0)
                                            : (field == 0 ? a.u1 : field == 1 ? a.v1 : a.w1);
                const int nlev = field == 2 ? a.sW : a.sRho;
                int L = kI - 2 + c;
                L = L < -nlev + 1 ? -nlev + 1 : (L > 0 ? 0 : L);
                L += nlev - 1;
                const float scale = field == 2 ? W_FEATURE : 1.f;
                float v[8];
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    int jj = j - 1 + a0 + e / 4, ii = i - 1 + e % 4;
                    jj = jj < 0 ? 0 : (jj > a.eta - 1 ? a.eta - 1 : jj);
                    ii = ii < 0 ? 0 : (ii > a.xi - 1 ? a.xi - 1 : ii);
                    v[e] = __ldg(src + ((size_t)L * a.eta + jj) * a.xi + ii) * scale;
                }
                uint4 pk;
                pk.x = pack_bf16(v[0], v[1]);
                pk.y = pack_bf16(v[2], v[3]);
                pk.z = pack_bf16(v[4], v[5]);
                pk.w = pack_bf16(v[6], v[7]);
                *reinterpret_cast<uint4 *>(sA + (f / 64) * KBLOCK_A + sw128_offset(tid, f % 64)) = pk;
            }
            // uniformity gate from the FP32 forcing: squared deviations of the u and v blocks of
            // both records from each block's node GATE_REF
            auto node = [&](const float *src, int n) {
                int lv = kI - 2 + n / 16;
                lv = lv < -a.sRho + 1 ? -a.sRho + 1 : (lv > 0 ? 0 : lv);
                lv += a.sRho - 1;
                int jj = j - 1 + (n % 16) / 4, ii = i - 1 + n % 4;
                jj = jj < 0 ? 0 : (jj > a.eta - 1 ? a.eta - 1 : jj);
                ii = ii < 0 ? 0 : (ii > a.xi - 1 ? a.xi - 1 : ii);
                return __ldg(src + ((size_t)lv * a.eta + jj) * a.xi + ii);
            };
            const float *blocks[4] = {a.u0, a.v0, a.u1, a.v1};
#pragma unroll 1
            for (int blk = 0; blk < 4; blk++) {
                const float x0 = node(blocks[blk], GATE_REF);
                float sum = 0.f;
                for (int n = 0; n < 64; n++) {
                    const float d = node(blocks[blk], n) - x0;
                    sum = fmaf(d, d, sum);
                }
                gsum += sum;
            }
        } else {
            const uint4 zero = make_uint4(0, 0, 0, 0);
            for (int q = 0; q < N_STENCIL / 8; q++)
                *reinterpret_cast<uint4 *>(sA + (q * 8 / 64) * KBLOCK_A + sw128_offset(tid, (q * 8) % 64)) = zero;
        }
        fence_async_shared();
        fence_before_sync();
        __syncthreads();
        fence_after_sync();
        if (abortFlag) break;
        // ---- weights through a 2-stage ring and the MMAs (thread 0)
        if (tid == 0) {
            bool ok = true;
            auto load = [&](uint32_t gg, int kb) {
                const uint32_t s = gg & 1, n = gg >> 1;
                if (!mbar_wait(&empty[s], (n & 1) ^ 1, &abortFlag)) return false;
                mbar_expect_tx(&full[s], KBLOCK_W);
                bulk_g2s(sW + s * KBLOCK_W, a.weights + OFF_W1 + (size_t)kb * KBLOCK_W, KBLOCK_W, &full[s]);
                issued[s] = (int)n;
                return true;
            };
            ok = load(g, 0) && load(g + 1, 1);
            for (int kb = 0; kb < CELL_KB && ok; kb++) {
                const uint32_t gg = g + kb, s = gg & 1, n = gg >> 1;
                if (!mbar_wait(&full[s], n & 1, &abortFlag)) {
                    ok = false;
                    break;
                }
                consumed[s] = (int)n;
                fence_after_sync();
#pragma unroll
                for (int ks = 0; ks < 4; ks++)
                    mma_bf16(tmem, desc_sw128(smem_u32(sA + kb * KBLOCK_A + ks * 32)),
                             desc_sw128(smem_u32(sW + s * KBLOCK_W + ks * 32)), idesc, (kb | ks) != 0);
                mma_commit(&empty[s]);
                if (kb + 2 < CELL_KB) ok = load(gg + 2, kb + 2);
            }
            mma_commit(&accFull);
            g += CELL_KB;
        }
        __syncwarp();
        mbar_wait(&accFull, it & 1, &abortFlag);
        __syncwarp();
        fence_after_sync();
        // ---- epilogue: z = acc + b1 (FP16), gate
        const bool write = cl < a.nCL && !abortFlag;
#pragma unroll 1
        for (int c0 = 0; c0 < HID; c0 += 32) {
            float v[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            if (write) {
                uint4 *dst = reinterpret_cast<uint4 *>(a.z + (size_t)cl * HID + c0);
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    __half2 h0 = __floats2half2_rn(v[8 * q + 0] + b1s[c0 + 8 * q + 0], v[8 * q + 1] + b1s[c0 + 8 * q + 1]);
                    __half2 h1 = __floats2half2_rn(v[8 * q + 2] + b1s[c0 + 8 * q + 2], v[8 * q + 3] + b1s[c0 + 8 * q + 3]);
                    __half2 h2 = __floats2half2_rn(v[8 * q + 4] + b1s[c0 + 8 * q + 4], v[8 * q + 5] + b1s[c0 + 8 * q + 5]);
                    __half2 h3 = __floats2half2_rn(v[8 * q + 6] + b1s[c0 + 8 * q + 6], v[8 * q + 7] + b1s[c0 + 8 * q + 7]);
                    uint4 pk;
                    pk.x = *reinterpret_cast<uint32_t *>(&h0);
                    pk.y = *reinterpret_cast<uint32_t *>(&h1);
                    pk.z = *reinterpret_cast<uint32_t *>(&h2);
                    pk.w = *reinterpret_cast<uint32_t *>(&h3);
                    dst[q] = pk;
                }
            }
        }
        if (write) {
            const int lev = (int)(cl % levels);
            const long long cell = cl / levels;
            const int j = (int)(cell / (a.xi - 1)), i = (int)(cell % (a.xi - 1));
            const int kI = lev - (a.sW - 2);
            const size_t plane = (size_t)a.eta * a.xi, c00 = (size_t)j * a.xi + i;
            const size_t corner[4] = {c00, c00 + a.xi, c00 + a.xi + 1, c00 + 1};
            const size_t lr = (size_t)(kI + a.sRho - 1) * plane, lu = (size_t)(kI + a.sW - 1) * plane,
                         ll = (size_t)(kI + a.sW - 2) * plane;
            CellCorners c;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                c.u[0][q] = a.u0[lr + corner[q]];
                c.u[1][q] = a.u1[lr + corner[q]];
                c.v[0][q] = a.v0[lr + corner[q]];
                c.v[1][q] = a.v1[lr + corner[q]];
                c.wU[0][q] = a.w0[lu + corner[q]];
                c.wU[1][q] = a.w1[lu + corner[q]];
                c.wL[0][q] = a.w0[ll + corner[q]];
                c.wL[1][q] = a.w1[ll + corner[q]];
                c.zeta[0][q] = a.z0[corner[q]];
                c.zeta[1][q] = a.z1[corner[q]];
                c.h[q] = (float)a.h[corner[q]];
            }
            const double2 m = a.metric[c00];
            c.invXdist = 1.0 / m.x;
            c.invYdist = 1.0 / m.y;
            c.depth = a.depthIntervals[kI + a.sW - 2];
            c.sigma = sqrtf(gsum / 256.f);
            c.gate = fminf(c.sigma / GATE_SIGMA, 1.f);
            a.corners[cl] = c;
        }
        fence_before_sync();
        __syncthreads();
        if (abortFlag) break;
    }
    if (tid == 0) {
        for (int s = 0; s < 2; s++)
            if (issued[s] > consumed[s]) mbar_wait_bounded(&full[s], (uint32_t)issued[s] & 1);
        if (abortFlag) atomicOr(a.err, ERR_SURROGATE_WAIT);
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        fence_after_sync();
        tmem_dealloc(tmem, 256);
    }
}

// ------------------------------------------------------------------ per-particle step

struct StepArgs {
    int eta, xi, sW, sRho;
    double start, length, dti, tau0, survprob, sv;
    double invLength, invDti, invTau0;  // reciprocals: the row epilogue multiplies
    int upper, lower, horizontal;
    int fallbackAll;  // run parameters outside the surrogate: every active particle falls back
    float maxError;   // metres per interval (INFINITY: off); see surrogate_trusted
    int drift;        // driftModel == 1: drifting objects fall back
    const int *dry;   // inclusive 2-D prefix sums of dry nodes, [(eta+1)][(xi+1)]
    const __half *z;  // [nCL][256]
    const CellCorners *corners;
    const uint8_t *weights;
    uint32_t *fallback, *fallbackCount;
    unsigned long long *runCount;
    float4 *rows;     // per work item: layer-4 sums (with b4, before the gate), row tag
};

// Row warps in column groups of four TMEM lane quarters, a bulk-copy producer warp and an MMA
// warp. Group g holds accumulator columns [g GROUP_COLS, (g+1) GROUP_COLS), the last group the rest.
// Sixteen row warps (four groups of 64 columns, 96 registers) run 9 % faster than eight (two
// groups of 128, 132 registers) and 3 % faster than twelve: the row work per thread shrinks and
// each scheduler holds four row warps instead of two.
constexpr int ROW_WARPS = 16, ROW_THREADS = ROW_WARPS * 32, GROUPS = ROW_WARPS / 4;
constexpr int PRODUCER_WARP = ROW_WARPS, MMA_WARP = ROW_WARPS + 1;
constexpr int STEP_THREADS = ROW_THREADS + 64;
constexpr int GROUP_COLS = (HID / 32 + GROUPS - 1) / GROUPS * 32;
constexpr int LAST_GROUP_COLS = HID - (GROUPS - 1) * GROUP_COLS;
constexpr int WRING = 2;
constexpr uint32_t A_BYTES = HID_KB * KBLOCK_A;  // 64 KB: one tile's activations
constexpr size_t STEP_SMEM = 2 * (size_t)A_BYTES + WRING * (size_t)KBLOCK_W + 1024;

enum : int { ROW_NONE = 0, ROW_RUN = 1, ROW_FALLBACK = 2, ROW_EMPTY = 3 };
// Row tag of a work item in rows[]: the cell-level (>= 0) of a row the surrogate moves, or one of
// these.
constexpr int ROW_CODE_NONE = -1, ROW_CODE_FALLBACK = -2;

// A tile's row as the prologue classified it.
struct RowTag {
    uint32_t slot;
    int status;
    int cl;
};

// Bilinear value from the four corners (j,i), (j+1,i), (j+1,i+1), (j,i+1) held in x, y, z, w, as
// nested linear blends: equal corners give their value exactly.
__device__ __forceinline__ float bil4(const float4 c, float jF, float iF) {
    const float lo = fmaf(c.w - c.x, iF, c.x), hi = fmaf(c.z - c.y, iF, c.y);
    return fmaf(hi - lo, jF, lo);
}

__device__ __forceinline__ float blend(float a, float b, float t) { return fmaf(b - a, t, a); }

// End of nSub equal substeps d = disp/nSub along one axis of [0, maximum): a particle leaving the
// domain at substep m under repeated reflectDomain alternates its overshoot e and d - e.
__device__ double pinned_axis(double x0, double disp, double d, double nSub, double maximum,
                              double &m) {
    const double end = x0 + disp, big = nSub + 1;
    const bool up = end >= maximum, down = end < 0;
    if (!up && !down) {
        m = big;
        return end;
    }
    double mm = up ? (d > 0 ? floor((maximum - x0) / d) + 1 : big) : (d < 0 ? floor(x0 / -d) + 1 : big);
    mm = fmin(mm, big);
    const double r = nSub - mm;
    double e = up ? x0 + mm * d - maximum : -(x0 + mm * d);
    e = fmax(e, 0.0);
    if (fmod(r, 2.0) != 0.0) e = fmax(fabs(d) - e, 0.0);
    double x = up ? maximum - e : e;
    x = fmin(fmax(x, 0.0), nextafter(maximum, 0.0));
    m = mm;
    return x;
}

// Whether the one-interval prediction is trusted: an estimate of the start-point method's error
// over the remaining time, |grad u| |u| t^2 / 2, with the velocity gradient taken as the stencil's
// RMS deviation sigma over 1.5 cells of the finer axis, must not exceed maxError (metres). A
// uniform stencil (sigma = 0) is always trusted: there the start-point displacement is exact.
__device__ __forceinline__ bool surrogate_trusted(float sigma, double invX, double invY, float ub,
                                                  float vb, double trem, float maxError) {
    const float grad = sigma * (float)fmax(invX, invY) * (1.f / 1.5f);
    const float t = (float)trem;
    return grad * sqrtf(ub * ub + vb * vb) * 0.5f * t * t <= maxError;
}

__device__ __forceinline__ int dry_in_box(const int *pre, int xi, int ja, int jb, int ia, int ib) {
    const int w = xi + 1;
    return pre[(jb + 1) * w + ib + 1] - pre[ja * w + ib + 1] - pre[(jb + 1) * w + ia] + pre[ja * w + ia];
}

// The MMA jobs of a block in the order the row warps make their operands ready: layers 2 and 3 of
// tile 0, 1, ... (the rows take prologue k+1, epilogue 3 of k, epilogue 2 of k+1, so layer 2 of
// tile k+1 runs on the tensor cores while the rows finish layer 3 of tile k, and layer 3 of tile
// k+1 while they build the operand of tile k+2). fn(tile, layer) returns false to stop.
template <class Fn>
__device__ __forceinline__ void for_each_job(int nT, Fn fn) {
    for (int k = 0; k < nT; k++) {
        if (!fn(k, 0)) return;
        if (!fn(k, 1)) return;
    }
}

__global__ void __launch_bounds__(STEP_THREADS, 1)
    surrogate_step_kernel(const StepArgs a, ParticleSoA S, const MoveLaunch L) {
    using namespace umma;
    extern __shared__ uint8_t dynSmem[];
    uint8_t *sA0 = align1024(dynSmem);
    uint8_t *ring = sA0 + 2 * A_BYTES;
    __shared__ __align__(8) uint64_t full[WRING], empty[WRING], aFull[2], accFull[2];
    __shared__ uint32_t tmemSlot;
    __shared__ int abortFlag;
    __shared__ int quarterStop[2][4];  // stop decisions per TMEM lane quarter, by tile parity
    __shared__ __align__(16) float w1ps[4 * HID];  // feature-major: pairs of units as float2
    __shared__ float b2s[HID], b3s[HID], w4s[3 * HID], b4s[4];
    // layer-4 partial sums of column groups 1.., by tile parity
    __shared__ float red[2][GROUPS - 1][TILE * 3];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        for (int s = 0; s < WRING; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&aFull[b], ROW_WARPS);  // one arrival per row warp
            mbar_init(&accFull[b], 1);
        }
        abortFlag = 0;
        for (int q = 0; q < 8; q++) quarterStop[q / 4][q % 4] = 0;
        fence_barrier_init();
    }
    {
        const float *w1p = reinterpret_cast<const float *>(a.weights + OFF_W1P);
        const float *b2 = reinterpret_cast<const float *>(a.weights + OFF_B2);
        const float *b3 = reinterpret_cast<const float *>(a.weights + OFF_B3);
        const float *w4 = reinterpret_cast<const float *>(a.weights + OFF_W4);
        const float *b4 = reinterpret_cast<const float *>(a.weights + OFF_B4);
        for (int c = tid; c < HID * 4; c += STEP_THREADS) w1ps[(c & 3) * HID + (c >> 2)] = w1p[c];
        for (int c = tid; c < HID; c += STEP_THREADS) {
            b2s[c] = b2[c];
            b3s[c] = b3[c];
        }
        for (int c = tid; c < 3 * HID; c += STEP_THREADS) w4s[c] = w4[c];
        if (tid < 3) b4s[tid] = b4[tid];
    }
    if (warp == MMA_WARP) tmem_alloc(&tmemSlot, 512);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = tmemSlot;
    const long long nTiles = ((long long)L.count + TILE - 1) / TILE;
    const int nT = blockIdx.x < nTiles ? (int)((nTiles - 1 - blockIdx.x) / gridDim.x + 1) : 0;
    const uint32_t idesc = idesc_bf16(TILE, HID);

    if (warp == PRODUCER_WARP) {
        // ---------------------------------------------------------- weight producer
        if (lane == 0) {
            int issued0 = -1, issued1 = -1;
            uint32_t g = 0;
            for_each_job(nT, [&](int, int layer) {
                for (int b = 0; b < HID_KB; b++, g++) {
                    const uint32_t s = g % WRING, n = g / WRING;
                    if (!mbar_wait(&empty[s], (n & 1) ^ 1, &abortFlag)) return false;
                    mbar_expect_tx(&full[s], KBLOCK_W);
                    const size_t off = (layer == 0 ? OFF_W2 : OFF_W3) + (size_t)b * KBLOCK_W;
                    bulk_g2s(ring + s * KBLOCK_W, a.weights + off, KBLOCK_W, &full[s]);
                    if (s == 0) issued0 = (int)n;
                    else issued1 = (int)n;
                }
                return true;
            });
            // copies still in flight land before the block exits
            if (issued0 >= 0) mbar_wait_bounded(&full[0], (uint32_t)issued0 & 1);
            if (issued1 >= 0) mbar_wait_bounded(&full[1], (uint32_t)issued1 & 1);
        }
        __syncwarp();
    } else if (warp == MMA_WARP) {
        // ---------------------------------------------------------- MMA issuer
        if (lane == 0) {
            uint32_t g = 0;
            for_each_job(nT, [&](int tile, int layer) {
                const int buf = tile & 1;
                if (!mbar_wait(&aFull[buf], (uint32_t)layer, &abortFlag)) return false;
                fence_after_sync();
                const uint32_t d = tmem + (uint32_t)(buf * HID);
                const uint8_t *A = sA0 + buf * A_BYTES;
                for (int kb = 0; kb < HID_KB; kb++, g++) {
                    const uint32_t s = g % WRING, n = g / WRING;
                    if (!mbar_wait(&full[s], n & 1, &abortFlag)) return false;
                    fence_after_sync();
#pragma unroll
                    for (int ks = 0; ks < 4; ks++)
                        mma_bf16(d, desc_sw128(smem_u32(A + kb * KBLOCK_A + ks * 32)),
                                 desc_sw128(smem_u32(ring + s * KBLOCK_W + ks * 32)), idesc,
                                 true);  // onto the bias the rows stored
                    mma_commit(&empty[s]);
                }
                mma_commit(&accFull[buf]);
                return true;
            });
        }
        __syncwarp();
    } else {
        // ---------------------------------------------------------- rows (warps 0-11)
        const int quarter = warp & 3, group = warp >> 2;
        const int r = quarter * 32 + lane;
        const uint32_t tlane = (uint32_t)(quarter * 32) << 16;
        const int cBase = group * GROUP_COLS;
        const int chunks = (group == GROUPS - 1 ? LAST_GROUP_COLS : GROUP_COLS) / 32;  // TMEM loads
        const double T0 = a.start, T1 = a.start + a.length;
        const double kLower = -a.sW + 2;
        auto tileOf = [&](int x) { return (long long)blockIdx.x + (long long)x * gridDim.x; };
        // each row warp signals its own part of an operand buffer (no block-wide barrier): its
        // lanes' shared-memory writes are fenced for the tensor cores, then lane 0 arrives
        auto arrive = [&](int buf) {
            fence_async_shared();
            fence_before_sync();
            __syncwarp();
            if (lane == 0) mbar_arrive(&aFull[buf]);
        };

        // A row's particle state, gathered ahead of the prologue that classifies it.
        struct RowState {
            uint32_t slot;
            bool valid;
            double pj, pi, pk, ptime, phealth;
            int ptype;
        };
        auto fetch = [&](int x) {
            RowState st{0u, false, 0.0, 0.0, 0.0, 0.0, 0.0, 0};
            const long long n = tileOf(x) * TILE + r;
            if (n < L.count) {
                st.valid = true;
                st.slot = L.order ? L.order[n] : (uint32_t)n;
                st.pj = S.j[st.slot];
                st.pi = S.i[st.slot];
                st.pk = S.k[st.slot];
                st.ptime = S.time[st.slot];
                st.phealth = S.health[st.slot];
                st.ptype = S.type[st.slot];
            }
            return st;
        };
        // A row's classification and layer-1 features, taken from its gathered state.
        struct Pending {
            RowTag tag;
            float jF, iF, kF, a0;
        };
        auto classify = [&](const RowState &st) {
            RowTag tag{0u, ROW_EMPTY, 0};
            float jF = 0.f, iF = 0.f, kF = 0.f, a0 = 0.f;
            if (st.valid) {
                tag.slot = st.slot;
                const double pj = st.pj, pi = st.pi, pk = st.pk;
                const double ptime = st.ptime, phealth = st.phealth;
                const int ptype = st.ptype;
                tag.status = ROW_NONE;
                if (phealth > 0 && ptime < T1) {
                    const double fj = floor(pj), fi = floor(pi), ck = ceil(pk);
                    const bool cellOk = fj >= 0 && fi >= 0 && fj + 1 < a.eta && fi + 1 < a.xi;
                    if (a.fallbackAll || phealth < a.survprob || pk > 0 || pk < kLower ||
                        (a.drift && ptype != 0) || !cellOk) {
                        tag.status = ROW_FALLBACK;
                    } else {
                        tag.status = ROW_RUN;
                        const int jI = (int)fj, iI = (int)fi, kI = (int)ck;
                        jF = (float)(pj - fj);
                        iF = (float)(pi - fi);
                        kF = (float)(ck - pk);
                        a0 = ptime > T0 ? (float)((ptime - T0) / a.length) : 0.f;
                        tag.cl = (jI * (a.xi - 1) + iI) * (a.sW - 1) + (kI + a.sW - 2);
                    }
                }
            }
            return Pending{tag, jF, iF, kF, a0};
        };
        // The row's per-cell layer-1 sums (FP16) for tile x, copied asynchronously into this
        // thread's own part of operand buffer A[x & 1]: 16-byte chunk q at the swizzled slot where
        // chunk q of the row's layer-1 output goes, so that the prologue converts them in place.
        // Issued once the tensor cores are done with the buffer, they land while the rows work on
        // the tiles before x.
        auto stage = [&](int x, const Pending &pd) {
            if (pd.tag.status == ROW_RUN) {
                uint8_t *A = sA0 + (x & 1) * A_BYTES;
                const uint4 *zrow = reinterpret_cast<const uint4 *>(a.z + (size_t)pd.tag.cl * HID + cBase);
                for (int q = 0; q < chunks * 4; q++) {
                    const int col = cBase + q * 8;
                    cp_async16(A + (col / 64) * KBLOCK_A + sw128_offset(r, col % 64), zrow + q);
                }
            }
            cp_async_commit();
        };
        // layer 1 of tile x from its staged sums: 2 GELU(z + features) -> A[x & 1], in place
        auto prologue = [&](int x, const Pending &pd) {
            const RowTag tag = pd.tag;
            const float jF = pd.jF, iF = pd.iF, kF = pd.kF, a0 = pd.a0;
            uint8_t *A = sA0 + (x & 1) * A_BYTES;
            cp_async_wait_all();
#pragma unroll 1
            for (int q0 = 0; q0 < chunks * 4; q0 += 4) {
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int col = cBase + (q0 + q) * 8;
                    uint4 *slotPtr = reinterpret_cast<uint4 *>(A + (col / 64) * KBLOCK_A + sw128_offset(r, col % 64));
                    uint4 out = make_uint4(0, 0, 0, 0);
                    if (tag.status == ROW_RUN) {
                        const uint4 zz = *slotPtr;
                        const __half2 *hz = reinterpret_cast<const __half2 *>(&zz);
                        const float2 fj = make_float2(jF, jF), fi = make_float2(iF, iF);
                        const float2 fk = make_float2(kF, kF), fa = make_float2(a0, a0);
                        uint32_t o[4];
#pragma unroll
                        for (int e = 0; e < 4; e++) {
                            // units col + 2e, col + 2e + 1: z + w_j jF + w_i iF + w_k kF + w_a a0
                            const int u = col + 2 * e;
                            float2 h = __half22float2(hz[e]);
                            h = __ffma2_rn(*reinterpret_cast<const float2 *>(w1ps + u), fj, h);
                            h = __ffma2_rn(*reinterpret_cast<const float2 *>(w1ps + HID + u), fi, h);
                            h = __ffma2_rn(*reinterpret_cast<const float2 *>(w1ps + 2 * HID + u), fk, h);
                            h = __ffma2_rn(*reinterpret_cast<const float2 *>(w1ps + 3 * HID + u), fa, h);
                            h = gelu2_pair(h);
                            o[e] = pack_bf16(h.x, h.y);
                        }
                        out = make_uint4(o[0], o[1], o[2], o[3]);
                    }
                    *slotPtr = out;
                }
            }
            // layer 2 accumulates onto its bias: this warp's columns of the tile's accumulator
            // (free since the rows read layer 3 of tile x-2 out of it) start as b2
            const uint32_t acc = tmem + (uint32_t)((x & 1) * HID) + tlane;
            for (int t = 0; t < chunks; t++) tmem_st32(acc + (uint32_t)(cBase + 32 * t), b2s + cBase + 32 * t);
            tmem_wait_st();
            arrive(x & 1);
            return tag;
        };

        // layer-2 epilogue of tile x: 2 GELU(acc) -> A[x & 1] (the halved W3 takes the 2 back); the
        // accumulator holds b2 + layer 2 and is reset to b3 for layer 3
        auto epilogue2 = [&](int x) {
            const int buf = x & 1;
            const bool ok = mbar_wait(&accFull[buf], 0, &abortFlag);
            __syncwarp();
            fence_after_sync();
            uint8_t *A = sA0 + buf * A_BYTES;
            const uint32_t acc = tmem + (uint32_t)(buf * HID) + tlane;
#pragma unroll 1
            for (int t = 0; t < chunks; t++) {
                const int c0 = cBase + 32 * t;
                float v[32];
                tmem_ld32(acc + (uint32_t)c0, v);
                tmem_st32(acc + (uint32_t)c0, b3s + c0);  // layer 3 accumulates onto b3
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    uint32_t o[4];
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        const float2 h = gelu2_pair(make_float2(v[8 * q + 2 * e], v[8 * q + 2 * e + 1]));
                        o[e] = pack_bf16(h.x, h.y);
                    }
                    const uint4 out = make_uint4(o[0], o[1], o[2], o[3]);
                    const int col = c0 + 8 * q;
                    *reinterpret_cast<uint4 *>(A + (col / 64) * KBLOCK_A + sw128_offset(r, col % 64)) = out;
                }
            }
            tmem_wait_st();
            arrive(buf);
            return ok;
        };

        // layer-3 epilogue of tile x with layer 4 folded in; column groups 1.. leave their partial
        // sums in red[]
        auto epilogue3 = [&](int x, float &o0, float &o1, float &o2) {
            const int buf = x & 1;
            const bool ok = mbar_wait(&accFull[buf], 1, &abortFlag);
            __syncwarp();
            fence_after_sync();
            const uint32_t acc = tmem + (uint32_t)(buf * HID) + tlane;
            o0 = o1 = o2 = 0.f;
#pragma unroll 1
            for (int t = 0; t < chunks; t++) {
                const int c0 = cBase + 32 * t;
                float v[32];
                tmem_ld32(acc + (uint32_t)c0, v);
#pragma unroll
                for (int c = 0; c < 32; c += 2) {
                    const float2 h = gelu2_pair(make_float2(v[c], v[c + 1]));
                    o0 = fmaf(h.x, w4s[c0 + c], o0);
                    o1 = fmaf(h.x, w4s[HID + c0 + c], o1);
                    o2 = fmaf(h.x, w4s[2 * HID + c0 + c], o2);
                    o0 = fmaf(h.y, w4s[c0 + c + 1], o0);
                    o1 = fmaf(h.y, w4s[HID + c0 + c + 1], o1);
                    o2 = fmaf(h.y, w4s[2 * HID + c0 + c + 1], o2);
                }
            }
            if (group > 0) {
                float *mine = red[x & 1][group - 1];
                mine[r * 3 + 0] = o0;
                mine[r * 3 + 1] = o1;
                mine[r * 3 + 2] = o2;
            }
            fence_before_sync();
            // the four warps of this lane quarter (one per column group) meet here
            named_sync(2 + quarter, 128);
            return ok;
        };

        RowTag cur{0u, ROW_EMPTY, 0}, next{0u, ROW_EMPTY, 0};
        Pending pend = classify(fetch(0));
        stage(0, pend);
        if (nT > 0) cur = prologue(0, pend);
        pend = classify(fetch(1));
        stage(1, pend);
        if (nT > 0) epilogue2(0);
        for (int k = 0; k < nT; k++) {
            // operand of tile k+1 (its layer 2 then runs while the rows finish layer 3 of tile k)
            if (k + 1 < nT) next = prologue(k + 1, pend);
            // the state gather of tile k+2 overlaps the layer-3 epilogue below
            const RowState ahead = fetch(k + 2);
            float o0, o1, o2;
            epilogue3(k, o0, o1, o2);
            // the quarter's stop decision, written by its group-0 warp in the previous tile: the
            // same value for its four warps, which therefore leave the loop together
            const int stop = quarterStop[k & 1][quarter];
            if (group == 0 && lane == 0) quarterStop[(k + 1) & 1][quarter] = abortFlag;
            if (group == 0 && cur.status != ROW_EMPTY) {
                // layer-4 sums and the row tag of the work item, for surrogate_post_kernel
                const int code = cur.status == ROW_RUN
                                     ? cur.cl
                                     : (cur.status == ROW_FALLBACK ? ROW_CODE_FALLBACK : ROW_CODE_NONE);
                float s0 = o0, s1 = o1, s2 = o2;
#pragma unroll
                for (int g = 0; g < GROUPS - 1; g++) {
                    s0 += red[k & 1][g][r * 3 + 0];
                    s1 += red[k & 1][g][r * 3 + 1];
                    s2 += red[k & 1][g][r * 3 + 2];
                }
                a.rows[tileOf(k) * TILE + r] =
                    make_float4(s0 + b4s[0], s1 + b4s[1], s2 + b4s[2], __int_as_float(code));
            }
            if (stop) break;
            // tile k+2's sums go to A[k & 1], which layer 3 of tile k no longer reads; they land
            // during the layer-2 epilogue of tile k+1
            pend = classify(ahead);
            stage(k + 2, pend);
            if (k + 1 < nT) epilogue2(k + 1);
            cur = next;
        }
        cp_async_wait_all();  // no copy into shared memory outlives the block
    }
    fence_before_sync();
    __syncthreads();
    if (warp == MMA_WARP) {
        fence_after_sync();
        tmem_dealloc(tmem, 512);
    }
    if (tid == 0 && abortFlag) atomicOr(L.err, ERR_SURROGATE_WAIT);
}

// Displacement, closures and state update of one work item from its layer-4 sums and row tag
// (rows[n], written by surrogate_step_kernel): one thread per item, so that the dependent loads
// of the particle state, the corner record and the dry-node table overlap across many warps.
// Five blocks per SM (48 registers, 20 bytes of spill): the dependent gathers overlap across more
// warps; 0.6 % of the interval faster than four blocks at 64 registers.
__global__ void __launch_bounds__(256, 5) surrogate_post_kernel(const StepArgs a, ParticleSoA S,
                                                             const MoveLaunch L) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    const double T0 = a.start;
    const double kLower = -a.sW + 2;
    // a step kernel that gave up on a wait left its rows incomplete: nothing is written
    const bool write = n < L.count && !(L.err && (*L.err & ERR_SURROGATE_WAIT));
    long long concCell = -1;
    int steps = 0;
    bool run = false;
    if (write) {
        const float4 row = a.rows[n];
        const int code = __float_as_int(row.w);
        int status = code >= 0 ? ROW_RUN : (code == ROW_CODE_FALLBACK ? ROW_FALLBACK : ROW_NONE);
        const uint32_t slot = L.order ? L.order[n] : (uint32_t)n;
        const double pj = S.j[slot], pi = S.i[slot], pk = S.k[slot];
        const double ptime = S.time[slot], page = S.age[slot], phealth = S.health[slot];
        if (status == ROW_RUN) {
            // the corner record: u[0],u[1],v[0],v[1],wU[0],wU[1],wL[0],wL[1],zeta[0],zeta[1],h
            // as float4s, then {1/xdist, 1/ydist}, then {depth, gate}
            const float4 *cf = reinterpret_cast<const float4 *>(a.corners + code);
            const float4 cu0 = __ldg(cf + 0), cu1 = __ldg(cf + 1), cv0 = __ldg(cf + 2),
                         cv1 = __ldg(cf + 3), cwU0 = __ldg(cf + 4), cwU1 = __ldg(cf + 5),
                         cwL0 = __ldg(cf + 6), cwL1 = __ldg(cf + 7), cz0 = __ldg(cf + 8),
                         cz1 = __ldg(cf + 9), ch = __ldg(cf + 10);
            const double2 inv = __ldg(reinterpret_cast<const double2 *>(cf + 11));
            const double depth = __ldg(reinterpret_cast<const double *>(cf + 12));
            const float gate = __ldg(reinterpret_cast<const float *>(cf + 12) + 2);
            const double y0 = (double)(row.x * gate);
            const double y1 = (double)(row.y * gate);
            const double y2 = (double)(row.z * gate);
            const double fj = floor(pj), fi = floor(pi), ck = ceil(pk);
            const float jF = (float)(pj - fj), iF = (float)(pi - fi), kF = (float)(ck - pk);
            const double da0 = ptime > T0 ? (ptime - T0) * a.invLength : 0.0;
            const double amid = 0.5 * (da0 + 1.0), trem = (1.0 - da0) * a.length;
            const double nSub = fmax(1.0, ceil(trem * a.invDti - 1e-9));
            const float am = (float)amid;
            const float ub = blend(bil4(cu0, jF, iF), bil4(cu1, jF, iF), am);
            const float vb = blend(bil4(cv0, jF, iF), bil4(cv1, jF, iF), am);
            const float wb = blend(blend(bil4(cwU0, jF, iF), bil4(cwL0, jF, iF), kF),
                                   blend(bil4(cwU1, jF, iF), bil4(cwL1, jF, iF), kF), am);
            const float hc = bil4(ch, jF, iF) + blend(bil4(cz0, jF, iF), bil4(cz1, jF, iF), am);
            const float sigma = __ldg(reinterpret_cast<const float *>(cf + 12) + 3);
            const bool trusted = surrogate_trusted(sigma, inv.x, inv.y, ub, vb, trem, a.maxError);
            const float zdist = hc * (float)depth;
            const double dI = ((double)ub * trem + OUT_H * y0) * inv.x;
            const double dJ = ((double)vb * trem + OUT_H * y1) * inv.y;
            const double dK = (double)(((wb + (float)a.sv) * (float)trem + OUT_V * (float)y2) *
                                       __frcp_rn(zdist));
            const double invSub = 1.0 / nSub;
            double mj, mi;
            double jn = pinned_axis(pj, dJ, dJ * invSub, nSub, (double)(a.eta - 1), mj);
            double in = pinned_axis(pi, dI, dI * invSub, nSub, (double)(a.xi - 1), mi);
            const double m = fmin(mj, mi);
            const bool crossed = m <= nSub;
            bool dead = false;
            if (a.horizontal == 1) {  // constraint: the last in-domain substep
                const double keep = crossed ? (m - 1) / nSub : 1.0;
                jn = pj + keep * dJ;
                in = pi + keep * dI;
            } else if (a.horizontal == 2 && crossed) {  // kill
                dead = true;
                jn = pj;
                in = pi;
            }
            double kn = pk + dK;
            if (kn > 0) {
                if (a.upper == 1) kn = 0;
                else if (a.upper == 2) dead = true;
                else if (a.upper == 3) kn = -kn;
            }
            if (kn < kLower) {
                if (a.lower == 1) kn = kLower;
                else if (a.lower == 2) dead = true;
                else if (a.lower == 3) kn = 2.0 * kLower - kn;
            }
            int ja = (int)floor(fmin(pj, jn)), jb = (int)floor(fmax(pj, jn)) + 1;
            int ia = (int)floor(fmin(pi, in)), ib = (int)floor(fmax(pi, in)) + 1;
            ja = ja < 0 ? 0 : (ja > a.eta - 1 ? a.eta - 1 : ja);
            jb = jb < 0 ? 0 : (jb > a.eta - 1 ? a.eta - 1 : jb);
            ia = ia < 0 ? 0 : (ia > a.xi - 1 ? a.xi - 1 : ia);
            ib = ib < 0 ? 0 : (ib > a.xi - 1 ? a.xi - 1 : ib);
            if (!trusted || dry_in_box(a.dry, a.xi, ja, jb, ia, ib) > 0) {
                status = ROW_FALLBACK;
            } else {
                const double age = page + trem;
                const double health = exp(-age * a.invTau0);
                dead = dead || health < a.survprob;
                S.j[slot] = jn;
                S.i[slot] = in;
                S.k[slot] = kn;
                S.age[slot] = age;
                S.health[slot] = dead ? -1.0 : health;
                ParticleState p;
                p.j = jn;
                p.i = in;
                p.k = kn;
                p.health = dead ? -1.0 : health;
                if (L.conc) concCell = concentration_cell(p, L.concTimeIndex, a.sRho, a.eta, a.xi);
                steps = (int)nSub;
                run = true;
            }
        } else if (status == ROW_NONE && L.conc) {
            ParticleState p;
            p.j = pj;
            p.i = pi;
            p.k = pk;
            p.health = phealth;
            concCell = concentration_cell(p, L.concTimeIndex, a.sRho, a.eta, a.xi);
        }
        if (status == ROW_FALLBACK) {
            const uint32_t at = atomicAdd(a.fallbackCount, 1u);
            a.fallback[at] = slot;
        }
    }
    if (L.steps) warp_sum_steps(L.steps, steps);
    if (L.conc) warp_count(L.conc, concCell);
    const unsigned ran = __ballot_sync(__activemask(), run);
    if ((threadIdx.x & 31) == 0 && ran) atomicAdd(a.runCount, (unsigned long long)__popc(ran));
}

// ------------------------------------------------------------------ learned advection + plain diffusion

// The cell-column forcing pair the plain FP32 step reads, for the per-substep operator.
template <int STORE>
struct WalkView {
    const CellQuad<STORE> *columns;  // [cell][sW][2] (A, B)
    const CellSurface *surface;      // [cell]
    const float2 *invMetric;         // [cell] {1/xdist, 1/ydist}
    const float *depth;              // [sW-1] FP32 depthIntervals
};

constexpr int WALK_BLOCKS = 5;  // resident blocks of 128 threads per SM the registers allow

__device__ __forceinline__ CellSurface load_surface(const CellSurface *s, int cell) {
    const float4 *q = reinterpret_cast<const float4 *>(s + cell);
    return CellSurface{__ldg(q), __ldg(q + 1)};
}

// One axis of a destination that may lie one cell beyond the domain, reflected at its edge as
// reflect_domain does (x -> 2 max - x past the last node, -x before the first): n is the
// destination cell on the axis, d its fraction there, x the fraction measured from the start cell
// and last the last valid cell. Returns whether the result is a cell and a fraction in [0, 1)
// (strictly inside (0, 1) when mirrored: a fraction of exactly 1 is the nextafter case, left to the
// FP64 landing); flip says whether the axis was mirrored.
__device__ __forceinline__ bool mirror_axis(int n, float d, float x, int last, int &cell, float &frac,
                                            bool &flip) {
    flip = false;
    cell = n;
    frac = d;
    if (n >= 0 && n <= last) return d >= 0.f && d < 1.f;
    flip = true;
    if (n == last + 1) {
        cell = last;
        frac = 2.f - x;
    } else if (n == -1) {
        cell = 0;
        frac = -x;
    } else {
        return false;
    }
    return frac > 0.f && frac < 1.f;
}

// One particle over the rest of a forward interval: the surrogate's deterministic displacement,
// spread evenly over the substeps as constant rates (m/s), plus the plain stochastic operator and
// closures of every substep, as the FP32 Euler step applies them (Particle.cpp:505-533,644-814;
// kernel.cu:262-364): sigma (1 - k/kb) Z sqrt(dt/dti) horizontally, the same times AKT crid
// vertically, the vertical cap, the vertical and horizontal closures, survival and age.
//
// The position is kept as a cell (or level) index plus an FP32 fraction, with the FP64 remainder
// of the start position carried alongside. Every substep reads its cell's surface, metric and AKT
// records and its destination's surface unconditionally (a particle stays in a cell for tens of
// substeps, so these hit L1), and a landing in water without a closure is FP32 work on the
// fraction, whether or not it changes cell: the lanes of a warp take the same path. Only a
// closure (shore, domain edge, surface, bottom) runs the plain step's FP64 landing. Returns the
// substeps taken.
template <int SEM, int STORE>
__device__ int walk_particle(const wacomm_b200_config &cfg, const IntervalParams &P,
                             const WalkView<STORE> &W, const float *depthS, int eta, int xi,
                             int sW, ParticleState &p, float rateX, float rateY, float rateZ) {
    const double length = P.length, invLength = 1.0 / length, kLower = P.kLower;
    const float shore = (float)cfg.shoreLimit, kLowerF = (float)kLower;
    const float invKLower = (float)P.invKLower, sigma = (float)cfg.sigma, crid = (float)cfg.crid;
    const float dtiF = (float)cfg.dti;
    const bool philox = P.rng == WACOMM_B200_RNG_PHILOX;
    const uint64_t prefix = fold(fold(mix64(cfg.randomSeed), p.id), (uint64_t)P.intervalKey);
    const uint64_t philoxKey = p.id ^ mix64(cfg.randomSeed);
    bool lazy = false;
    int steps = 0;
    double elapsed = p.time > P.start ? fmin(length, p.time - P.start) : 0.0;  // activation
    // Substeps left in which the lazy survival tests cannot change their outcome: while
    // age < min(ageKillLo, ageUnder) a lazily tracked particle is neither dead (age stays below
    // ageKillLo <= ageKillHi) nor without health (age below ageUnder). Counted when the
    // particle turns lazy, two substeps short of the bound for rounding; while it lasts and no
    // closure has ended the lazy tracking, both tests are skipped.
    const double ageSafe = fmin(P.ageKillLo, P.ageUnder);
    int youngLeft = 0;

    const double fj = floor(p.j), fi = floor(p.i), ck = ceil(p.k);
    int jI = to_index<SEM>(fj), iI = to_index<SEM>(fi), kI = to_index<SEM>(ck);
    float jF = (float)(p.j - fj), iF = (float)(p.i - fi), kF = (float)(ck - p.k);
    double jLo = (p.j - fj) - (double)jF, iLo = (p.i - fi) - (double)iF;
    double kLo = (ck - p.k) - (double)kF;

    // surface sums at the particle's position, carried from the previous substep's landing
    SurfaceSums here{0.f, 0.f};
    bool carried = false;
    while (elapsed < length) {
        const double stepDt = fmin(cfg.dti, length - elapsed);
        if (!(lazy && youngLeft > 0)) {
            const bool dead = lazy ? (p.age >= P.ageKillHi ||
                                      (p.age > P.ageKillLo && exp(-p.age / cfg.tau0) < cfg.survprob))
                                   : p.health < cfg.survprob;
            if (dead) {
                p.health = -1;
                lazy = false;
                break;
            }
        }
        if (!carried &&
            (!valid_cell(jI, iI, eta, xi) || (SEM == SEM_DEVICE && (kI > 0 || kI <= -sW + 1)))) {
            p.health = -1;
            lazy = false;
            break;
        }
        steps++;
        const int kM = mem_level(kI, sW);
        const int cell = jI * xi + iI;
        if (!carried) here = surface_from(load_surface(W.surface, cell), jF, iF);
        const float2 inv = __ldg(W.invMetric + cell);
        QuadPair aUp, aLo;
        const CellQuad<STORE> *col = W.columns + ((size_t)cell * sW + (size_t)(kM + sW - 1)) * 2;
        load_second<STORE>(col - 1, aLo);  // akt of W level kI-1
        load_second<STORE>(col + 1, aUp);  // akt of W level kI
        const float depth = depthS[kM + sW - 2];
        const float dt = stepDt == cfg.dti ? dtiF : (float)stepDt;
        const float alpha = (float)((elapsed + 0.5 * stepDt) * invLength);
        const float hc = here.height(alpha);
        if (hc <= shore && cfg.horizontalClosure == CLOSURE_KILL) {
            p.health = -1;
            lazy = false;
            if (SEM == SEM_DEVICE) break;
        }
        const Weights8 wa = weights8(jF, iF, alpha);
        const float au = blend(aUp, wa), al = blend(aLo, wa);
        const float aa = fmaf(al - au, kF, au);
        float n0, n1, n2;
        if (philox) {
            philox_normals3(philoxKey, P.intervalKey, (uint64_t)__double_as_longlong(elapsed), n0, n1,
                            n2);
        } else {
            const uint64_t stepKey = fold(prefix, (uint64_t)floor(elapsed / cfg.dti));
            n0 = (float)prefix_normal(stepKey, 0);
            n1 = (float)prefix_normal(stepKey, 1);
            n2 = (float)prefix_normal(stepKey, 2);
        }
        const float kNow = (float)kI - kF;
        const float sigmaDepth = sigma * (1.f - kNow * invKLower);
        const float scale = stepDt == cfg.dti ? 1.f : sqrtf(dt / dtiF);
        // the two horizontal components in pairs (packed FP32x2, the same roundings)
        const float2 rxy = __fmul2_rn(__fmul2_rn(make_float2(sigmaDepth, sigmaDepth), make_float2(n0, n1)),
                                      make_float2(scale, scale));
        const float rz = sigmaDepth * n2 * aa * crid * scale;
        const float zdist = hc * depth;
        const float rzdist = __frcp_rn(zdist);
        const float2 dIJ = __fmul2_rn(__ffma2_rn(make_float2(rateX, rateY), make_float2(dt, dt), rxy), inv);
        const float dI = dIJ.x, dJ = dIJ.y;
        float zleap = fmaf(rateZ, dt, rz);
        if (fabsf(zleap) > zdist) zleap = signf_of(zdist, zleap);
        const float2 ijN = __fadd2_rn(make_float2(iF, jF), dIJ);
        const float iN = ijN.x, jN = ijN.y, kN = fmaf(-zleap, rzdist, kF);
        // the destination: at most one cell or level away on this path (comparisons, no
        // float-to-int conversions), and its surface (this cell's, read again, in the common case)
        const int dj = (jN >= 1.f) - (jN < 0.f), di = (iN >= 1.f) - (iN < 0.f);
        const int dk = (kN >= 1.f) - (kN < 0.f);
        const float jD = jN - (float)dj, iD = iN - (float)di, kD = kN - (float)dk;
        const int nj = jI + dj, ni = iI + di;
        const bool inside = valid_cell(nj, ni, eta, xi) && jD >= 0.f && jD < 1.f && iD >= 0.f &&
                            iD < 1.f && kD >= 0.f && kD < 1.f;
        const SurfaceSums there =
            surface_from(load_surface(W.surface, inside ? nj * xi + ni : cell), jD, iD);
        const bool vertical = (float)kI - kN > 0.f || (float)kI - kN < kLowerF;
        carried = inside && !vertical && there.height(alpha) > shore;
        // The domain edge, under the closures that do not look at the land there: the destination
        // cell lies outside the valid cells and the level stays in range. Constraint drops the
        // horizontal move (the position and its surface sums stay); reflection mirrors each axis
        // that left at the edge (NumericalHelpers.hpp:67-74). FP32 work on the fractions, as a
        // landing in water, whenever the mirrored fraction lies inside (0, 1); otherwise, and for
        // the other closures, the FP64 landing below. A particle the current keeps pushing against
        // the edge takes this path every substep.
        bool edge = false;
        if (!carried && !vertical && kD >= 0.f && kD < 1.f && !valid_cell(nj, ni, eta, xi)) {
            if (cfg.horizontalClosure == CLOSURE_CONSTRAINT) {
                edge = true;
                carried = true;
            } else if (cfg.horizontalClosure == CLOSURE_REFLECTION) {
                int mj, mi;
                float mjF, miF;
                bool flipJ, flipI;
                if (mirror_axis(nj, jD, jN, eta - 2, mj, mjF, flipJ) &&
                    mirror_axis(ni, iD, iN, xi - 2, mi, miF, flipI)) {
                    edge = true;  // carried stays false: the next substep reads the new surface
                    jI = mj;
                    iI = mi;
                    jF = mjF;
                    iF = miF;
                    if (flipJ) jLo = -jLo;
                    if (flipI) iLo = -iLo;
                }
            }
            if (edge) {
                kI -= dk;
                kF = kD;
            }
        }
        if (edge) {
            // landed above
        } else if (carried) {
            jI = nj;
            iI = ni;
            jF = jD;
            iF = iD;
            kI -= dk;  // level crossing
            kF = kD;
            here = there;
        } else {
            // a closure: the plain step's FP64 landing (Particle.cpp:644-791)
            const double pj = (double)jI + (double)jF + jLo, pi = (double)iI + (double)iF + iLo;
            const double pk = (double)kI - (double)kF - kLo;
            double jdet = pj + (double)dJ, idet = pi + (double)dI;
            double kdet = pk + (double)(zleap * rzdist);
            if (kdet > 0.) close_upper(cfg, kdet, p.health, lazy);
            if (kdet < kLower) close_lower(cfg, kLower, kdet, p.health, lazy);
            double nJ = pj, nI = pi, nK = pk;
            const double fjd = floor(jdet), fid = floor(idet);
            const int jdetI = to_index<SEM>(fjd), idetI = to_index<SEM>(fid);
            if (valid_cell(jdetI, idetI, eta, xi)) {
                const CellSurface at = load_surface(W.surface, jdetI * xi + idetI);
                const float hcdet =
                    surface_from(at, (float)(jdet - fjd), (float)(idet - fid)).height(alpha);
                if (hcdet <= shore) {
                    if (cfg.horizontalClosure == CLOSURE_CONSTRAINT) {
                        idet = pi;
                        jdet = pj;
                    } else if (cfg.horizontalClosure == CLOSURE_KILL) {
                        p.health = -1;
                        lazy = false;
                    } else if (cfg.horizontalClosure == CLOSURE_REFLECTION) {
                        idet = reflect_cell(pi, iI, idet, idetI);
                        jdet = reflect_cell(pj, jI, jdet, jdetI);
                    }
                }
                nI = idet;
                nJ = jdet;
                nK = kdet;
            } else {
                if (cfg.horizontalClosure == CLOSURE_CONSTRAINT) {
                    nK = kdet;
                } else if (cfg.horizontalClosure == CLOSURE_KILL) {
                    p.health = -1;
                    lazy = false;
                } else if (cfg.horizontalClosure == CLOSURE_REFLECTION) {
                    nI = reflect_domain(idet, xi - 1);
                    nJ = reflect_domain(jdet, eta - 1);
                    nK = kdet;
                }
            }
            const double gj = floor(nJ), gi = floor(nI), gk = ceil(nK);
            jI = to_index<SEM>(gj);
            iI = to_index<SEM>(gi);
            kI = to_index<SEM>(gk);
            jF = (float)(nJ - gj);
            iF = (float)(nI - gi);
            kF = (float)(gk - nK);
            jLo = (nJ - gj) - (double)jF;
            iLo = (nI - gi) - (double)iF;
            kLo = (gk - nK) - (double)kF;
        }
        if (lazy && youngLeft > 0) {  // still lazy: no closure ended the tracking this substep
            p.age = p.age + stepDt;
            youngLeft--;
        } else {
            const bool alive = lazy ? (p.age < P.ageUnder || exp(-p.age / cfg.tau0) > 0) : p.health > 0;
            if (alive) {
                if (!lazy) {
                    // FP32 and an approximate division: the two-substep margin covers their error
                    const float n = floorf(__fdividef((float)(ageSafe - p.age), (float)cfg.dti)) - 2.f;
                    youngLeft = n > 0.f ? (n < 1.0e9f ? (int)n : 1000000000) : 0;
                }
                p.age = p.age + stepDt;
                lazy = true;
            }
        }
        elapsed += stepDt;
    }
    if (lazy) p.health = exp(-p.age / cfg.tau0);
    p.j = (double)jI + (double)jF + jLo;
    p.i = (double)iI + (double)iF + iLo;
    p.k = (double)kI - (double)kF - kLo;
    return steps;
}

// Learned advection with the plain stochastic operator per substep (diffusive forward intervals):
// one thread per work item, taken in cell order (the engine's cell sort) so that the lanes of a
// warp share their cell's records and meet the same closures. The rates come from the item's layer-4 outputs and the
// start-point velocity of its corner record, as in surrogate_post_kernel; the particle then takes
// every substep of the interval by walk_particle. Rows the step kernel handed back go to the
// fallback list.
template <int SEM, int STORE>
__global__ void __launch_bounds__(128, WALK_BLOCKS)
    surrogate_walk_kernel(const StepArgs a, const wacomm_b200_config cfg, const IntervalParams P,
                          const WalkView<STORE> W, ParticleSoA S, const MoveLaunch L) {
    __shared__ float depthS[64];  // FP32 layer thicknesses (sW - 1 <= 64 levels)
    for (int q = threadIdx.x; q < a.sW - 1 && q < 64; q += blockDim.x) depthS[q] = W.depth[q];
    __syncthreads();
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    const bool write = n < L.count && !(L.err && (*L.err & ERR_SURROGATE_WAIT));
    long long concCell = -1;
    int steps = 0;
    bool run = false;
    if (write) {
        const uint32_t slot = L.order ? L.order[n] : (uint32_t)n;  // cell order of the walk
        const float4 row = a.rows[slot];  // the step kernel's rows follow the slots
        const int code = __float_as_int(row.w);
        int status = code >= 0 ? ROW_RUN : (code == ROW_CODE_FALLBACK ? ROW_FALLBACK : ROW_NONE);
        ParticleState p;
        p.j = S.j[slot];
        p.i = S.i[slot];
        p.k = S.k[slot];
        p.health = S.health[slot];
        p.time = S.time[slot];
        if (status == ROW_RUN) {
            p.id = S.id[slot];
            p.age = S.age[slot];
            const float4 *cf = reinterpret_cast<const float4 *>(a.corners + code);
            const float4 cu0 = __ldg(cf + 0), cu1 = __ldg(cf + 1), cv0 = __ldg(cf + 2),
                         cv1 = __ldg(cf + 3), cwU0 = __ldg(cf + 4), cwU1 = __ldg(cf + 5),
                         cwL0 = __ldg(cf + 6), cwL1 = __ldg(cf + 7);
            const float gate = __ldg(reinterpret_cast<const float *>(cf + 12) + 2);
            const double fj = floor(p.j), fi = floor(p.i), ck = ceil(p.k);
            const float jF = (float)(p.j - fj), iF = (float)(p.i - fi), kF = (float)(ck - p.k);
            const double da0 = p.time > a.start ? (p.time - a.start) * a.invLength : 0.0;
            const float am = (float)(0.5 * (da0 + 1.0));
            const float invTrem = (float)(1.0 / ((1.0 - da0) * a.length));
            const float ub = blend(bil4(cu0, jF, iF), bil4(cu1, jF, iF), am);
            const float vb = blend(bil4(cv0, jF, iF), bil4(cv1, jF, iF), am);
            const float wb = blend(blend(bil4(cwU0, jF, iF), bil4(cwL0, jF, iF), kF),
                                   blend(bil4(cwU1, jF, iF), bil4(cwL1, jF, iF), kF), am);
            const double2 inv = __ldg(reinterpret_cast<const double2 *>(cf + 11));
            const float sigma = __ldg(reinterpret_cast<const float *>(cf + 12) + 3);
            if (!surrogate_trusted(sigma, inv.x, inv.y, ub, vb, (1.0 - da0) * a.length,
                                   a.maxError)) {
                status = ROW_FALLBACK;
            } else {
                const float rateX = fmaf(OUT_H * row.x * gate, invTrem, ub);
                const float rateY = fmaf(OUT_H * row.y * gate, invTrem, vb);
                const float rateZ = fmaf(OUT_V * row.z * gate, invTrem, wb + (float)a.sv);
                const float *depth = a.sW - 1 <= 64 ? depthS : W.depth;  // deeper: global copy
                steps = walk_particle<SEM, STORE>(cfg, P, W, depth, a.eta, a.xi, a.sW, p, rateX,
                                                  rateY, rateZ);
                S.j[slot] = p.j;
                S.i[slot] = p.i;
                S.k[slot] = p.k;
                S.age[slot] = p.age;
                S.health[slot] = p.health;
                if (L.conc) concCell = concentration_cell(p, L.concTimeIndex, a.sRho, a.eta, a.xi);
                run = true;
            }
        } else if (status == ROW_NONE && L.conc) {
            concCell = concentration_cell(p, L.concTimeIndex, a.sRho, a.eta, a.xi);
        }
        if (status == ROW_FALLBACK) {
            const uint32_t at = atomicAdd(a.fallbackCount, 1u);
            a.fallback[at] = slot;
        }
    }
    if (L.steps) warp_sum_steps(L.steps, steps);
    if (L.conc) warp_count(L.conc, concCell);
    const unsigned ran = __ballot_sync(__activemask(), run);
    if ((threadIdx.x & 31) == 0 && ran) atomicAdd(a.runCount, (unsigned long long)__popc(ran));
}

// ------------------------------------------------------------------ dry-node prefix sums

__global__ void dry_rows_kernel(const double *mask, const double *h, double shore, int eta, int xi,
                                int *pre) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j > eta) return;
    const int w = xi + 1;
    int run = 0;
    pre[j * w] = 0;
    for (int i = 0; i < xi; i++) {
        if (j > 0) {
            const size_t n = (size_t)(j - 1) * xi + i;
            run += ((mask && mask[n] == 0.0) || h[n] <= shore) ? 1 : 0;
        }
        pre[j * w + i + 1] = run;
    }
}

__global__ void dry_cols_kernel(int eta, int xi, int *pre) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > xi) return;
    const int w = xi + 1;
    int run = 0;
    for (int j = 0; j <= eta; j++) {
        run += pre[j * w + i];
        pre[j * w + i] = run;
    }
}

}  // namespace

// ------------------------------------------------------------------ host side

// The shared-memory sizes of the two tensor-core kernels, set once per device (the current one; a
// set-up step, kept out of stream capture).
cudaError_t surrogate_prepare() {
    static bool done[64] = {};
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    if (device >= 0 && device < 64 && done[device]) return cudaSuccess;
    e = cudaFuncSetAttribute(surrogate_cell_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)CELL_SMEM);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(surrogate_step_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)STEP_SMEM);
    if (e == cudaSuccess && device >= 0 && device < 64) done[device] = true;
    return e;
}

size_t surrogate_packed_bytes() { return PACKED_BYTES; }

size_t surrogate_corner_bytes() { return sizeof(CellCorners); }

size_t surrogate_parameter_count() {
    return (size_t)HID * N_INPUT + HID + 2 * ((size_t)HID * HID + HID) + 3 * HID + 3;
}

void surrogate_pack(const float *flat, uint8_t *out) {
    memset(out, 0, PACKED_BYTES);
    const float *w1 = flat;
    const float *b1 = w1 + HID * N_INPUT;
    const float *w2 = b1 + HID;
    const float *b2 = w2 + HID * HID;
    const float *w3 = b2 + HID;
    const float *b3 = w3 + HID * HID;
    const float *w4 = b3 + HID;
    const float *b4 = w4 + 3 * HID;
    auto put = [&](size_t base, int rows, int k, float v) {
        __nv_bfloat16 b = __float2bfloat16_rn(v);
        memcpy(out + base + (size_t)(k / 64) * KBLOCK_W + umma::sw128_offset(rows, k % 64), &b, 2);
    };
    for (int n = 0; n < HID; n++) {
        for (int k = 0; k < N_STENCIL; k++) put(OFF_W1, n, k, w1[n * N_INPUT + k]);
        for (int k = 0; k < HID; k++) {
            // halved: they multiply twice the GELU of the layer below (gelu2_pair)
            put(OFF_W2, n, k, 0.5f * w2[n * HID + k]);
            put(OFF_W3, n, k, 0.5f * w3[n * HID + k]);
        }
    }
    float *fb1 = reinterpret_cast<float *>(out + OFF_B1), *fb2 = reinterpret_cast<float *>(out + OFF_B2);
    float *fb3 = reinterpret_cast<float *>(out + OFF_B3), *fw1p = reinterpret_cast<float *>(out + OFF_W1P);
    float *fw4 = reinterpret_cast<float *>(out + OFF_W4), *fb4 = reinterpret_cast<float *>(out + OFF_B4);
    for (int n = 0; n < HID; n++) {
        fb1[n] = b1[n];
        fb2[n] = b2[n];
        fb3[n] = b3[n];
        for (int e = 0; e < 4; e++) fw1p[n * 4 + e] = w1[n * N_INPUT + N_STENCIL + e];
    }
    for (int o = 0; o < 3 * HID; o++) fw4[o] = 0.5f * w4[o];
    for (int o = 0; o < 3; o++) fb4[o] = b4[o];
}

long long surrogate_cell_levels(int eta, int xi, int sW) {
    return (long long)(eta - 1) * (xi - 1) * (sW - 1);
}

cudaError_t surrogate_cells(int eta, int xi, int sW, int sRho, const FrameDevice &f0,
                            const FrameDevice &f1, const double *h, const double *depthIntervals,
                            const double2 *metric, const uint8_t *weights, __half *z, void *corners,
                            int *err, int smCount, cudaStream_t stream) {
    CellArgs a;
    a.eta = eta;
    a.xi = xi;
    a.sW = sW;
    a.sRho = sRho;
    a.nCL = surrogate_cell_levels(eta, xi, sW);
    a.u0 = f0.u;
    a.v0 = f0.v;
    a.w0 = f0.w;
    a.u1 = f1.u;
    a.v1 = f1.v;
    a.w1 = f1.w;
    a.z0 = f0.zeta;
    a.z1 = f1.zeta;
    a.h = h;
    a.depthIntervals = depthIntervals;
    a.metric = metric;
    a.weights = weights;
    a.z = z;
    a.corners = static_cast<CellCorners *>(corners);
    a.err = err;
    if (a.nCL <= 0) return cudaSuccess;
    cudaError_t e = surrogate_prepare();
    if (e != cudaSuccess) return e;
    long long tiles = (a.nCL + TILE - 1) / TILE;
    int blocks = (int)(tiles < smCount ? tiles : smCount);
    surrogate_cell_kernel<<<blocks, 128, CELL_SMEM, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t surrogate_step(const SurrogateStep &s, const ParticleSoA &S, const MoveLaunch &L,
                           int smCount, cudaStream_t stream) {
    if (L.count <= 0) return cudaSuccess;
    StepArgs a;
    a.eta = s.eta;
    a.xi = s.xi;
    a.sW = s.sW;
    a.sRho = s.sRho;
    a.start = s.start;
    a.length = s.length;
    a.dti = s.cfg.dti;
    a.tau0 = s.cfg.tau0;
    a.invLength = s.length == 0 ? 0.0 : 1.0 / s.length;
    a.invDti = 1.0 / s.cfg.dti;
    a.invTau0 = 1.0 / s.cfg.tau0;
    a.survprob = s.cfg.survprob;
    a.sv = s.cfg.sv;
    a.upper = s.cfg.upperClosure;
    a.lower = s.cfg.lowerClosure;
    a.horizontal = s.cfg.horizontalClosure;
    a.fallbackAll = s.fallbackAll;
    a.maxError = s.maxError;
    a.drift = s.cfg.driftModel == 1;
    a.dry = s.dry;
    a.z = s.z;
    a.corners = static_cast<const CellCorners *>(s.corners);
    a.weights = s.weights;
    a.fallback = s.fallback;
    a.fallbackCount = s.fallbackCount;
    a.runCount = s.runCount;
    a.rows = s.rows;
    cudaError_t e = surrogate_prepare();
    if (e != cudaSuccess) return e;
    long long tiles = ((long long)L.count + TILE - 1) / TILE;
    int blocks = (int)(tiles < smCount ? tiles : smCount);
    surrogate_step_kernel<<<blocks, STEP_THREADS, STEP_SMEM, stream>>>(a, S, L);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (s.midEvent && (e = cudaEventRecord(s.midEvent, stream)) != cudaSuccess) return e;
    if (!s.walk) {
        surrogate_post_kernel<<<(L.count + 255) / 256, 256, 0, stream>>>(a, S, L);
        return cudaGetLastError();
    }
    const int blocks128 = (L.count + 127) / 128;
    auto walk = [&](auto semTag, auto storeTag) {
        constexpr int SEM = decltype(semTag)::value, STORE = decltype(storeTag)::value;
        WalkView<STORE> W;
        W.columns = static_cast<const CellQuad<STORE> *>(s.cells);
        W.surface = static_cast<const CellSurface *>(s.cellSurface);
        W.invMetric = s.invMetric;
        W.depth = s.depthF;
        MoveLaunch LW = L;
        LW.order = s.walkOrder;
        surrogate_walk_kernel<SEM, STORE><<<blocks128, 128, 0, stream>>>(a, s.cfg, *s.interval, W, S, LW);
        return cudaGetLastError();
    };
    using Host = std::integral_constant<int, SEM_HOST>;
    using Device = std::integral_constant<int, SEM_DEVICE>;
    using F32 = std::integral_constant<int, STORE_F32>;
    using F16 = std::integral_constant<int, STORE_F16>;
    using BF16 = std::integral_constant<int, STORE_BF16>;
    if (s.semantics == SEM_HOST) {
        if (s.storage == STORE_F16) return walk(Host{}, F16{});
        if (s.storage == STORE_BF16) return walk(Host{}, BF16{});
        return walk(Host{}, F32{});
    }
    if (s.storage == STORE_F16) return walk(Device{}, F16{});
    if (s.storage == STORE_BF16) return walk(Device{}, BF16{});
    return walk(Device{}, F32{});
}

cudaError_t surrogate_dry_prefix(const double *mask, const double *h, double shore, int eta, int xi,
                                 int *pre, cudaStream_t stream) {
    dry_rows_kernel<<<(eta + 1 + 127) / 128, 128, 0, stream>>>(mask, h, shore, eta, xi, pre);
    dry_cols_kernel<<<(xi + 1 + 127) / 128, 128, 0, stream>>>(eta, xi, pre);
    return cudaGetLastError();
}

}  // namespace wb
