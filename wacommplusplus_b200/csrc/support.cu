// Kernels around the move: forcing-pair packing, cell metric, scan, counting sort by cell,
// record layout conversion, stable dead-particle compaction and concentration grids.
#include "engine.h"
#include "move_kernels.cuh"

namespace wb {

static inline int grid_for(size_t n, int block, int maxBlocks = 148 * 16) {
    size_t blocks = (n + block - 1) / block;
    if (blocks > (size_t)maxBlocks) blocks = maxBlocks;
    return blocks < 1 ? 1 : (int)blocks;
}

size_t node_record_bytes(int storage) {
    return storage == STORE_F32 ? sizeof(NodeRecord<STORE_F32>) : sizeof(NodeRecord<STORE_F16>);
}

// ------------------------------------------------------------------ forcing pair packing

template <int STORE>
__device__ __forceinline__ void store_node(NodeRecord<STORE> *dst, float w0, float a0, float u0,
                                           float v0, float w1, float a1, float u1, float v1);
template <>
__device__ __forceinline__ void store_node<STORE_F32>(NodeRecord<STORE_F32> *dst, float w0,
                                                      float a0, float u0, float v0, float w1,
                                                      float a1, float u1, float v1) {
    dst->t0 = make_float4(w0, a0, u0, v0);
    dst->t1 = make_float4(w1, a1, u1, v1);
}
template <>
__device__ __forceinline__ void store_node<STORE_F16>(NodeRecord<STORE_F16> *dst, float w0,
                                                      float a0, float u0, float v0, float w1,
                                                      float a1, float u1, float v1) {
    NodeRecord<STORE_F16> r;
    r.wa0 = __floats2half2_rn(w0, a0);
    r.uv0 = __floats2half2_rn(u0, v0);
    r.wa1 = __floats2half2_rn(w1, a1);
    r.uv1 = __floats2half2_rn(u1, v1);
    *dst = r;
}
template <>
__device__ __forceinline__ void store_node<STORE_BF16>(NodeRecord<STORE_BF16> *dst, float w0,
                                                       float a0, float u0, float v0, float w1,
                                                       float a1, float u1, float v1) {
    NodeRecord<STORE_BF16> r;
    r.wa0 = __floats2bfloat162_rn(w0, a0);
    r.uv0 = __floats2bfloat162_rn(u0, v0);
    r.wa1 = __floats2bfloat162_rn(w1, a1);
    r.uv1 = __floats2bfloat162_rn(u1, v1);
    *dst = r;
}

// Interleaves records t0 and t1 into node records {w(L), akt(L), u(L-1), v(L-1)} x 2.
template <int STORE>
__global__ void pack_nodes_kernel(int eta, int xi, int sW, FrameDevice f0, FrameDevice f1,
                                  NodeRecord<STORE> *nodes) {
    size_t plane = (size_t)eta * xi, total = plane * sW;
    for (size_t n = blockIdx.x * (size_t)blockDim.x + threadIdx.x; n < total;
         n += (size_t)gridDim.x * blockDim.x) {
        size_t L = n / plane, cell = n - L * plane;
        float w0 = f0.w[n], a0 = f0.akt[n], w1 = f1.w[n], a1 = f1.akt[n];
        float u0 = 0, v0 = 0, u1 = 0, v1 = 0;
        if (L > 0) {
            size_t r = (L - 1) * plane + cell;
            u0 = f0.u[r];
            v0 = f0.v[r];
            u1 = f1.u[r];
            v1 = f1.v[r];
        }
        store_node<STORE>(nodes + n, w0, a0, u0, v0, w1, a1, u1, v1);
    }
}

__global__ void pack_surface_kernel(int eta, int xi, FrameDevice f0, FrameDevice f1,
                                    const double *h, SurfPair *surf, EnvPair *env) {
    size_t plane = (size_t)eta * xi;
    for (size_t n = blockIdx.x * (size_t)blockDim.x + threadIdx.x; n < plane;
         n += (size_t)gridDim.x * blockDim.x) {
        surf[n] = SurfPair{h[n], f0.zeta[n], f1.zeta[n]};
        if (env) {
            EnvPair e;
            e.wu0 = f0.windU ? f0.windU[n] : 0.f;
            e.wv0 = f0.windV ? f0.windV[n] : 0.f;
            e.su0 = f0.stokesU ? f0.stokesU[n] : 0.f;
            e.sv0 = f0.stokesV ? f0.stokesV[n] : 0.f;
            e.wu1 = f1.windU ? f1.windU[n] : 0.f;
            e.wv1 = f1.windV ? f1.windV[n] : 0.f;
            e.su1 = f1.stokesU ? f1.stokesU[n] : 0.f;
            e.sv1 = f1.stokesV ? f1.stokesV[n] : 0.f;
            env[n] = e;
        }
    }
}

cudaError_t pack_pair(int storage, int eta, int xi, int sW, const FrameDevice &f0,
                      const FrameDevice &f1, const double *h, void *nodes, SurfPair *surf,
                      EnvPair *env, cudaStream_t stream) {
    size_t total = (size_t)eta * xi * sW;
    int blocks = grid_for(total, 256);
    switch (storage) {
        case STORE_F16:
            pack_nodes_kernel<STORE_F16><<<blocks, 256, 0, stream>>>(
                eta, xi, sW, f0, f1, static_cast<NodeRecord<STORE_F16> *>(nodes));
            break;
        case STORE_BF16:
            pack_nodes_kernel<STORE_BF16><<<blocks, 256, 0, stream>>>(
                eta, xi, sW, f0, f1, static_cast<NodeRecord<STORE_BF16> *>(nodes));
            break;
        default:
            pack_nodes_kernel<STORE_F32><<<blocks, 256, 0, stream>>>(
                eta, xi, sW, f0, f1, static_cast<NodeRecord<STORE_F32> *>(nodes));
    }
    pack_surface_kernel<<<grid_for((size_t)eta * xi, 256), 256, 0, stream>>>(eta, xi, f0, f1, h,
                                                                           surf, env);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ cell-column packing

size_t cell_record_bytes(int storage) {
    return 2 * (storage == STORE_F32 ? sizeof(CellQuad<STORE_F32>) : sizeof(CellQuad<STORE_F16>));
}
size_t cell_surface_bytes() { return sizeof(CellSurface); }

template <int STORE>
__device__ __forceinline__ void store_quad(CellQuad<STORE> *dst, const float (&a0)[4],
                                           const float (&a1)[4], const float (&b0)[4],
                                           const float (&b1)[4]);
template <>
__device__ __forceinline__ void store_quad<STORE_F32>(CellQuad<STORE_F32> *dst, const float (&a0)[4],
                                                      const float (&a1)[4], const float (&b0)[4],
                                                      const float (&b1)[4]) {
    dst->a0 = make_float4(a0[0], a0[1], a0[2], a0[3]);
    dst->a1 = make_float4(a1[0], a1[1], a1[2], a1[3]);
    dst->b0 = make_float4(b0[0], b0[1], b0[2], b0[3]);
    dst->b1 = make_float4(b1[0], b1[1], b1[2], b1[3]);
}
template <>
__device__ __forceinline__ void store_quad<STORE_F16>(CellQuad<STORE_F16> *dst, const float (&a0)[4],
                                                      const float (&a1)[4], const float (&b0)[4],
                                                      const float (&b1)[4]) {
    CellQuad<STORE_F16> r;
    r.a0[0] = __floats2half2_rn(a0[0], a0[1]);
    r.a0[1] = __floats2half2_rn(a0[2], a0[3]);
    r.a1[0] = __floats2half2_rn(a1[0], a1[1]);
    r.a1[1] = __floats2half2_rn(a1[2], a1[3]);
    r.b0[0] = __floats2half2_rn(b0[0], b0[1]);
    r.b0[1] = __floats2half2_rn(b0[2], b0[3]);
    r.b1[0] = __floats2half2_rn(b1[0], b1[1]);
    r.b1[1] = __floats2half2_rn(b1[2], b1[3]);
    *dst = r;
}
template <>
__device__ __forceinline__ void store_quad<STORE_BF16>(CellQuad<STORE_BF16> *dst, const float (&a0)[4],
                                                       const float (&a1)[4], const float (&b0)[4],
                                                       const float (&b1)[4]) {
    CellQuad<STORE_BF16> r;
    r.a0[0] = __floats2bfloat162_rn(a0[0], a0[1]);
    r.a0[1] = __floats2bfloat162_rn(a0[2], a0[3]);
    r.a1[0] = __floats2bfloat162_rn(a1[0], a1[1]);
    r.a1[1] = __floats2bfloat162_rn(a1[2], a1[3]);
    r.b0[0] = __floats2bfloat162_rn(b0[0], b0[1]);
    r.b0[1] = __floats2bfloat162_rn(b0[2], b0[3]);
    r.b1[0] = __floats2bfloat162_rn(b1[0], b1[1]);
    r.b1[1] = __floats2bfloat162_rn(b1[2], b1[3]);
    *dst = r;
}

// One thread per (W level L, cell): writes A(L) and B(L) of the cell (views.cuh). Cells on the
// last row or column (never valid) are zero.
template <int STORE>
__global__ void pack_cells_kernel(int eta, int xi, int sW, FrameDevice f0, FrameDevice f1,
                                  CellQuad<STORE> *cells) {
    size_t plane = (size_t)eta * xi, total = plane * sW;
    for (size_t n = blockIdx.x * (size_t)blockDim.x + threadIdx.x; n < total;
         n += (size_t)gridDim.x * blockDim.x) {
        size_t L = n / plane, cell = n - L * plane;
        int j = (int)(cell / xi), i = (int)(cell - (size_t)j * xi);
        float u0[4] = {0, 0, 0, 0}, u1[4] = {0, 0, 0, 0}, v0[4] = {0, 0, 0, 0}, v1[4] = {0, 0, 0, 0};
        float w0[4] = {0, 0, 0, 0}, w1[4] = {0, 0, 0, 0}, a0[4] = {0, 0, 0, 0}, a1[4] = {0, 0, 0, 0};
        if (j + 1 < eta && i + 1 < xi) {
            const size_t corner[4] = {cell, cell + xi, cell + xi + 1, cell + 1};
            for (int c = 0; c < 4; c++) {
                size_t q = L * plane + corner[c];
                w0[c] = f0.w[q];
                w1[c] = f1.w[q];
                a0[c] = f0.akt[q];
                a1[c] = f1.akt[q];
                if (L > 0) {
                    size_t r = (L - 1) * plane + corner[c];
                    u0[c] = f0.u[r];
                    u1[c] = f1.u[r];
                    v0[c] = f0.v[r];
                    v1[c] = f1.v[r];
                }
            }
        }
        CellQuad<STORE> *dst = cells + (cell * sW + L) * 2;
        store_quad<STORE>(dst, u0, u1, v0, v1);
        store_quad<STORE>(dst + 1, w0, w1, a0, a1);
    }
}

__global__ void pack_cell_surface_kernel(int eta, int xi, FrameDevice f0, FrameDevice f1,
                                         const double *h, CellSurface *out) {
    size_t plane = (size_t)eta * xi;
    for (size_t cell = blockIdx.x * (size_t)blockDim.x + threadIdx.x; cell < plane;
         cell += (size_t)gridDim.x * blockDim.x) {
        int j = (int)(cell / xi), i = (int)(cell - (size_t)j * xi);
        CellSurface s;
        if (j + 1 < eta && i + 1 < xi) {
            size_t c1 = cell, c2 = cell + xi, c3 = cell + xi + 1, c4 = cell + 1;
            s.s0 = make_float4((float)h[c1] + f0.zeta[c1], (float)h[c2] + f0.zeta[c2],
                               (float)h[c3] + f0.zeta[c3], (float)h[c4] + f0.zeta[c4]);
            s.dz = make_float4(f1.zeta[c1] - f0.zeta[c1], f1.zeta[c2] - f0.zeta[c2],
                               f1.zeta[c3] - f0.zeta[c3], f1.zeta[c4] - f0.zeta[c4]);
        } else {
            s.s0 = s.dz = make_float4(0, 0, 0, 0);
        }
        out[cell] = s;
    }
}

cudaError_t pack_cells(int storage, int eta, int xi, int sW, const FrameDevice &f0,
                       const FrameDevice &f1, const double *h, void *cells, void *cellSurface,
                       cudaStream_t stream) {
    size_t total = (size_t)eta * xi * sW;
    int blocks = grid_for(total, 256);
    switch (storage) {
        case STORE_F16:
            pack_cells_kernel<STORE_F16><<<blocks, 256, 0, stream>>>(
                eta, xi, sW, f0, f1, static_cast<CellQuad<STORE_F16> *>(cells));
            break;
        case STORE_BF16:
            pack_cells_kernel<STORE_BF16><<<blocks, 256, 0, stream>>>(
                eta, xi, sW, f0, f1, static_cast<CellQuad<STORE_BF16> *>(cells));
            break;
        default:
            pack_cells_kernel<STORE_F32><<<blocks, 256, 0, stream>>>(
                eta, xi, sW, f0, f1, static_cast<CellQuad<STORE_F32> *>(cells));
    }
    pack_cell_surface_kernel<<<grid_for((size_t)eta * xi, 256), 256, 0, stream>>>(
        eta, xi, f0, f1, h, static_cast<CellSurface *>(cellSurface));
    return cudaGetLastError();
}

// ------------------------------------------------------------------ cell metric

// Cell sizes in metres along j (ydist) and i (xdist). Host rules: haversine along one grid axis
// with the cross difference dropped (Particle.cpp:548-574); device rules: full haversine between
// the nodes (kernel.cu:145-149,278-279). Cells on the last row/column are never valid.
__global__ void metric_kernel(int semantics, int eta, int xi, const double *lat,
                              const double *lon, double2 *metric, float2 *invMetric) {
    size_t plane = (size_t)eta * xi;
    for (size_t n = blockIdx.x * (size_t)blockDim.x + threadIdx.x; n < plane;
         n += (size_t)gridDim.x * blockDim.x) {
        int j = (int)(n / xi), i = (int)(n - (size_t)j * xi);
        if (j + 1 >= eta || i + 1 >= xi) {
            metric[n] = make_double2(0.0, 0.0);
            invMetric[n] = make_float2(0.f, 0.f);
            continue;
        }
        double lat0 = lat[n], lon0 = lon[n];
        double latN = lat[n + xi], lonN = lon[n + xi];
        double latE = lat[n + 1], lonE = lon[n + 1];
        double xdist, ydist;
        if (semantics == SEM_HOST) {
            double s = sin(0.5 * (latN - lat0));
            double d = s * s;
            ydist = 2.0 * atan2(sqrt(d), sqrt(1.0 - d)) * 6371000.0;
            s = sin(0.5 * (lonE - lon0));
            d = s * s * cos(latE) * cos(lat0);
            xdist = 2.0 * atan2(sqrt(d), sqrt(1.0 - d)) * 6371000.0;
        } else {
            double dLat = latN - lat0, dLon = lonN - lon0;
            double value = sin(.5 * dLat) * sin(.5 * dLat) + sin(.5 * dLon) * sin(.5 * dLon) * cos(latN) * cos(lat0);
            ydist = 2.0 * atan2(sqrt(value), sqrt(1.0 - value)) * 6371000.0;
            dLat = latE - lat0;
            dLon = lonE - lon0;
            value = sin(.5 * dLat) * sin(.5 * dLat) + sin(.5 * dLon) * sin(.5 * dLon) * cos(latE) * cos(lat0);
            xdist = 2.0 * atan2(sqrt(value), sqrt(1.0 - value)) * 6371000.0;
        }
        metric[n] = make_double2(xdist, ydist);
        invMetric[n] = make_float2((float)(1.0 / xdist), (float)(1.0 / ydist));
    }
}

cudaError_t build_metric(int semantics, int eta, int xi, const double *lonRad,
                         const double *latRad, double2 *metric, float2 *invMetric,
                         cudaStream_t stream) {
    metric_kernel<<<grid_for((size_t)eta * xi, 256), 256, 0, stream>>>(semantics, eta, xi, latRad,
                                                                      lonRad, metric, invMetric);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ exclusive scan

constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 8;
constexpr size_t SCAN_TILE = (size_t)SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ uint32_t block_exclusive(uint32_t value, uint32_t *shared,
                                                    uint32_t &blockTotal) {
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inclusive = value;
    for (int off = 1; off < 32; off <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, inclusive, off);
        if (lane >= off) inclusive += y;
    }
    if (lane == 31) shared[warp] = inclusive;
    __syncthreads();
    if (warp == 0) {
        uint32_t s = lane < (int)(blockDim.x >> 5) ? shared[lane] : 0;
        uint32_t inc = s;
        for (int off = 1; off < 32; off <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, inc, off);
            if (lane >= off) inc += y;
        }
        shared[lane] = inc - s;
        if (lane == 31) shared[32] = inc;
    }
    __syncthreads();
    uint32_t result = shared[warp] + inclusive - value;
    blockTotal = shared[32];
    __syncthreads();
    return result;
}

__global__ void __launch_bounds__(SCAN_THREADS) scan_reduce_kernel(const uint32_t *in, size_t n,
                                                                   uint32_t *sums) {
    __shared__ uint32_t shared[33];
    size_t base = blockIdx.x * SCAN_TILE + (size_t)threadIdx.x * SCAN_ITEMS;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++)
        if (base + k < n) s += in[base + k];
    uint32_t total;
    block_exclusive(s, shared, total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(SCAN_THREADS) scan_apply_kernel(const uint32_t *in, uint32_t *out,
                                                                  size_t n,
                                                                  const uint32_t *offsets,
                                                                  uint32_t *total) {
    __shared__ uint32_t shared[33];
    size_t base = blockIdx.x * SCAN_TILE + (size_t)threadIdx.x * SCAN_ITEMS;
    uint32_t v[SCAN_ITEMS];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        v[k] = base + k < n ? in[base + k] : 0;
        s += v[k];
    }
    uint32_t blockTotal;
    uint32_t run = block_exclusive(s, shared, blockTotal) + (offsets ? offsets[blockIdx.x] : 0);
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
    if (total && blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) *total = run;
}

size_t scan_temp_words(size_t n) {
    size_t words = 0;
    while (n > SCAN_TILE) {
        size_t blocks = (n + SCAN_TILE - 1) / SCAN_TILE;
        words += 2 * blocks;
        n = blocks;
    }
    return words + 2;
}

cudaError_t exclusive_scan(const uint32_t *in, uint32_t *out, size_t n, uint32_t *total,
                           uint32_t *temp, cudaStream_t stream) {
    if (n == 0) {
        if (total) cudaMemsetAsync(total, 0, sizeof(uint32_t), stream);
        return cudaGetLastError();
    }
    size_t blocks = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (blocks == 1) {
        scan_apply_kernel<<<1, SCAN_THREADS, 0, stream>>>(in, out, n, nullptr, total);
        return cudaGetLastError();
    }
    uint32_t *sums = temp, *sumOffsets = temp + blocks;
    scan_reduce_kernel<<<(unsigned)blocks, SCAN_THREADS, 0, stream>>>(in, n, sums);
    cudaError_t e = exclusive_scan(sums, sumOffsets, blocks, nullptr, temp + 2 * blocks, stream);
    if (e != cudaSuccess) return e;
    scan_apply_kernel<<<(unsigned)blocks, SCAN_THREADS, 0, stream>>>(in, out, n, sumOffsets, total);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ counting sort by cell

__device__ __forceinline__ uint32_t cell_key(double j, double i, int eta, int xi) {
    double fj = floor(j), fi = floor(i);
    if (!(fj >= 0.0 && fi >= 0.0 && fj < (double)(eta - 1) && fi < (double)(xi - 1)))
        return (uint32_t)((size_t)eta * xi);
    return (uint32_t)((int)fj * xi + (int)fi);
}

// Both passes walk the records in the sequence `seq` (a permutation of the slots, or the identity
// when null); keys are kept in sequence order. Walking in the previous interval's cell order puts
// the records of one cell next to each other, so a warp's atomics collapse to one per cell even
// where walls gather hundreds of thousands of records into a few cells.
__global__ void key_histogram_kernel(const double *j, const double *i, int n, int eta, int xi,
                                     const uint32_t *seq, uint32_t *keys, uint32_t *hist) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const uint32_t p = seq ? seq[t] : (uint32_t)t;
        uint32_t key = cell_key(j[p], i[p], eta, xi);
        keys[t] = key;
        unsigned active = __activemask();
        unsigned peers = __match_any_sync(active, key);
        if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(hist + key, (uint32_t)__popc(peers));
    }
}

__global__ void key_scatter_kernel(const uint32_t *keys, int n, const uint32_t *seq,
                                   uint32_t *cursor, uint32_t *order) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        uint32_t key = keys[t];
        unsigned active = __activemask();
        unsigned peers = __match_any_sync(active, key);
        int lane = threadIdx.x & 31;
        int leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if (lane == leader) base = atomicAdd(cursor + key, (uint32_t)__popc(peers));
        base = __shfl_sync(peers, base, leader);
        uint32_t rank = __popc(peers & ((1u << lane) - 1u));
        order[base + rank] = seq ? seq[t] : (uint32_t)t;
    }
}

cudaError_t sort_by_cell(const double *j, const double *i, int n, int eta, int xi,
                         const uint32_t *seq, uint32_t *keys, uint32_t *hist, uint32_t *offsets,
                         uint32_t *temp, uint32_t *order, cudaStream_t stream) {
    size_t bins = (size_t)eta * xi + 1;
    cudaMemsetAsync(hist, 0, bins * sizeof(uint32_t), stream);
    int blocks = grid_for((size_t)n, 256);
    key_histogram_kernel<<<blocks, 256, 0, stream>>>(j, i, n, eta, xi, seq, keys, hist);
    cudaError_t e = exclusive_scan(hist, offsets, bins, offsets + bins, temp, stream);
    if (e != cudaSuccess) return e;
    key_scatter_kernel<<<blocks, 256, 0, stream>>>(keys, n, seq, offsets, order);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ record layout

__global__ void aos_to_soa_kernel(const wacomm_b200_particle *aos, int n, ParticleSoA S) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        wacomm_b200_particle r = aos[p];
        S.id[p] = r.id;
        S.k[p] = r.k;
        S.j[p] = r.j;
        S.i[p] = r.i;
        S.health[p] = r.health;
        S.age[p] = r.age;
        S.time[p] = r.time;
        S.type[p] = r.driftObjectType;
        S.side[p] = r.driftSide;
    }
}

__global__ void soa_to_aos_kernel(ParticleSoA S, int n, wacomm_b200_particle *aos) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        wacomm_b200_particle r;
        memset(&r, 0, sizeof(r));
        r.id = S.id[p];
        r.k = S.k[p];
        r.j = S.j[p];
        r.i = S.i[p];
        r.health = S.health[p];
        r.age = S.age[p];
        r.time = S.time[p];
        r.driftObjectType = S.type[p];
        r.driftSide = S.side[p];
        aos[p] = r;
    }
}

cudaError_t aos_to_soa(const wacomm_b200_particle *aos, int n, const ParticleSoA &S,
                       cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    aos_to_soa_kernel<<<grid_for(n, 256), 256, 0, stream>>>(aos, n, S);
    return cudaGetLastError();
}

cudaError_t soa_to_aos(const ParticleSoA &S, int n, wacomm_b200_particle *aos,
                       cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    soa_to_aos_kernel<<<grid_for(n, 256), 256, 0, stream>>>(S, n, aos);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ dead-particle removal

__global__ void alive_flags_kernel(const double *health, int n, uint32_t *flags) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        flags[p] = health[p] > 0 ? 1u : 0u;
}

__global__ void compact_kernel(ParticleSoA S, int n, const uint32_t *flags,
                               const uint32_t *positions, ParticleSoA T) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        if (!flags[p]) continue;
        uint32_t q = positions[p];
        T.id[q] = S.id[p];
        T.k[q] = S.k[p];
        T.j[q] = S.j[p];
        T.i[q] = S.i[p];
        T.health[q] = S.health[p];
        T.age[q] = S.age[p];
        T.time[q] = S.time[p];
        T.type[q] = S.type[p];
        T.side[q] = S.side[p];
    }
}

cudaError_t compact_alive(const ParticleSoA &S, int n, const ParticleSoA &tmp, uint32_t *flags,
                          uint32_t *positions, uint32_t *temp, uint32_t *kept,
                          cudaStream_t stream) {
    if (n <= 0) {
        cudaMemsetAsync(kept, 0, sizeof(uint32_t), stream);
        return cudaGetLastError();
    }
    int blocks = grid_for(n, 256);
    alive_flags_kernel<<<blocks, 256, 0, stream>>>(S.health, n, flags);
    cudaError_t e = exclusive_scan(flags, positions, n, kept, temp, stream);
    if (e != cudaSuccess) return e;
    compact_kernel<<<blocks, 256, 0, stream>>>(S, n, flags, positions, tmp);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ concentration

__global__ void count_kernel(ParticleSoA S, int n, int concTime, int sRho, int eta, int xi,
                             uint32_t *conc) {
    for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        int p = base + threadIdx.x;
        long long cell = -1;
        if (p < n) {
            ParticleState s;
            s.k = S.k[p];
            s.j = S.j[p];
            s.i = S.i[p];
            s.health = S.health[p];
            cell = concentration_cell(s, concTime, sRho, eta, xi);
        }
        warp_count(conc, cell);
    }
}

__global__ void accumulate_steps_kernel(const unsigned long long *steps,
                                        unsigned long long *total) {
    *total += *steps;
}

cudaError_t accumulate_steps(const unsigned long long *steps, unsigned long long *total,
                             cudaStream_t stream) {
    accumulate_steps_kernel<<<1, 1, 0, stream>>>(steps, total);
    return cudaGetLastError();
}

cudaError_t count_concentration(const ParticleSoA &S, int n, int concTime, int sRho, int eta,
                                int xi, uint32_t *conc, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    count_kernel<<<grid_for(n, 256), 256, 0, stream>>>(S, n, concTime, sRho, eta, xi, conc);
    return cudaGetLastError();
}

// Float grid of the reference (counts as float, exact below 2^24) with the land mask of
// Wacomm.cpp:188-196,724-739 (mask != 1 -> 1e37 in every level).
__global__ void to_float_kernel(const uint32_t *conc, size_t n, int plane, const double *mask,
                                float *out) {
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
         q += (size_t)gridDim.x * blockDim.x) {
        float value = (float)conc[q];
        if (mask && mask[q % plane] != 1.0) value = 1e37f;
        out[q] = value;
    }
}

cudaError_t concentration_to_float(const uint32_t *conc, size_t n, int nTimes, int sRho, int eta,
                                   int xi, const double *mask, float *out, cudaStream_t stream) {
    (void)nTimes;
    (void)sRho;
    if (n == 0) return cudaSuccess;
    to_float_kernel<<<grid_for(n, 256), 256, 0, stream>>>(conc, n, eta * xi, mask, out);
    return cudaGetLastError();
}

}  // namespace wb
