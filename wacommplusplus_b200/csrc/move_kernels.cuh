// Move kernels: one thread per particle, the whole interval (or one chunk of it) in registers.
#pragma once

#include "step.cuh"
#include "step_fast.cuh"

namespace wb {

// Structure-of-arrays particle state resident in the engine.
struct ParticleSoA {
    uint64_t *id;
    double *k, *j, *i, *health, *age, *time;
    uint16_t *type;
    int8_t *side;
    double *elapsed;  // resume point between chunks
};

struct MoveLaunch {
    int count;                    // work items
    const uint32_t *order;        // work item -> particle slot (cell-sorted), or null
    uint32_t *conc;               // uint32 concentration grid, or null
    int concTimeIndex, concTimes;
    unsigned long long *steps;    // particle-step counter, or null
    int *err;
    // When set, the work items are the first min(count, *countDevice): a list whose length a
    // kernel earlier on the stream wrote (the launch covers `count`, blocks past the list exit).
    const uint32_t *countDevice = nullptr;
    // FP32 step: work items per thread; the grid is that many times smaller and each block
    // strides over it (results do not depend on it).
    int perThread = 1;
};

// Work items of a launch: count, or the device-side length of its list.
__device__ __forceinline__ int launch_count(const MoveLaunch &L) {
    if (!L.countDevice) return L.count;
    const uint32_t listed = *L.countDevice;
    return listed < (uint32_t)L.count ? (int)listed : L.count;
}

// Linear index of the concentration cell of an alive particle, or -1
// (Concentration.hpp:28-41: round-half-away indices, bounds 0<=j<eta, 0<=i<xi, -sRho<k<=0).
__device__ __forceinline__ long long concentration_cell(const ParticleState &p, int concTime,
                                                        int sRho, int eta, int xi) {
    if (!(p.health > 0)) return -1;
    double rk = round(p.k), rj = round(p.j), ri = round(p.i);
    if (!(rj >= 0.0 && rj < (double)eta && ri >= 0.0 && ri < (double)xi &&
          rk >= (double)(-sRho + 1) && rk <= 0.0))
        return -1;
    int k = (int)rk, j = (int)rj, i = (int)ri;
    return (((long long)concTime * sRho + (k + sRho - 1)) * eta + j) * (long long)xi + i;
}

// Warp-aggregated increment: lanes holding the same cell elect one lane that adds the count.
__device__ __forceinline__ void warp_count(uint32_t *grid, long long cell) {
    unsigned active = __activemask();
    unsigned peers = __match_any_sync(active, (unsigned long long)cell);
    int lane = threadIdx.x & 31;
    if (cell >= 0 && lane == __ffs(peers) - 1) atomicAdd(grid + cell, (uint32_t)__popc(peers));
}

__device__ __forceinline__ void warp_sum_steps(unsigned long long *counter, int steps) {
    unsigned active = __activemask();
    for (int off = 16; off > 0; off >>= 1) steps += __shfl_down_sync(active, steps, off);
    if ((threadIdx.x & 31) == 0 && counter && steps) atomicAdd(counter, (unsigned long long)steps);
}

template <int SEM, int ARITH, int STORE>
__global__ void __launch_bounds__(256) move_soa_kernel(const wacomm_b200_config cfg,
                                                       const IntervalParams P,
                                                       const PackedView<STORE> V, ParticleSoA S,
                                                       const MoveLaunch L) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    long long cell = -1;
    int steps = 0;
    if (t < L.count) {
        uint32_t slot = L.order ? L.order[t] : (uint32_t)t;
        ParticleState p;
        p.id = S.id[slot];
        p.k = S.k[slot];
        p.j = S.j[slot];
        p.i = S.i[slot];
        p.health = S.health[slot];
        p.age = S.age[slot];
        p.time = S.time[slot];
        p.type = S.type[slot];
        p.side = S.side[slot];
        double elapsed = P.firstChunk ? P.elapsed0 : S.elapsed[slot];
        steps = move_particle<SEM, ARITH>(cfg, P, V, p, elapsed, L.err);
        S.k[slot] = p.k;
        S.j[slot] = p.j;
        S.i[slot] = p.i;
        S.health[slot] = p.health;
        S.age[slot] = p.age;
        S.side[slot] = (int8_t)p.side;
        if (!P.lastChunk) S.elapsed[slot] = elapsed;
        if (L.conc && P.lastChunk) cell = concentration_cell(p, L.concTimeIndex, V.g.sRho, V.g.eta, V.g.xi);
    }
    if (L.steps) warp_sum_steps(L.steps, steps);
    if (L.conc && P.lastChunk) warp_count(L.conc, cell);
}

// Launch shapes of the FP32 kernel: threads per block and the minimum resident blocks per SM the
// register allocation must allow (WACOMM_B200 launch_shape 0..3).
template <int SHAPE>
struct LaunchShape;
template <>
struct LaunchShape<0> {
    static constexpr int threads = 256, minBlocks = 1;
};
template <>
struct LaunchShape<1> {
    static constexpr int threads = 128, minBlocks = 3;
};
template <>
struct LaunchShape<2> {
    static constexpr int threads = 256, minBlocks = 2;
};
template <>
struct LaunchShape<3> {
    static constexpr int threads = 128, minBlocks = 5;
};

// FP32 step over the cell-column pair (step_fast.cuh); same state handling as move_soa_kernel.
template <int SEM, int STORE, int SHAPE, int VARIANT>
__global__ void __launch_bounds__(LaunchShape<SHAPE>::threads, LaunchShape<SHAPE>::minBlocks)
    move_fast_kernel(const wacomm_b200_config cfg,
                                                        const IntervalParams P,
                                                        const FastView<STORE> F, ParticleSoA S,
                                                        const MoveLaunch L) {
    const int count = launch_count(L);
    // block-uniform stride loop (blocks past a device-side list take no turn)
    for (long long base = (long long)blockIdx.x * blockDim.x; base < count;
         base += (long long)gridDim.x * blockDim.x) {
        const int t = (int)base + threadIdx.x;
        long long cell = -1;
        int steps = 0;
        if (t < count) {
            uint32_t slot = L.order ? L.order[t] : (uint32_t)t;
            ParticleState p;
            p.id = S.id[slot];
            p.k = S.k[slot];
            p.j = S.j[slot];
            p.i = S.i[slot];
            p.health = S.health[slot];
            p.age = S.age[slot];
            p.time = S.time[slot];
            p.type = S.type[slot];
            p.side = S.side[slot];
            double elapsed = P.firstChunk ? P.elapsed0 : S.elapsed[slot];
            steps = move_particle_fast<SEM, STORE, VARIANT>(cfg, P, F, p, elapsed, L.err);
            S.k[slot] = p.k;
            S.j[slot] = p.j;
            S.i[slot] = p.i;
            S.health[slot] = p.health;
            S.age[slot] = p.age;
            S.side[slot] = (int8_t)p.side;
            if (!P.lastChunk) S.elapsed[slot] = elapsed;
            if (L.conc && P.lastChunk)
                cell = concentration_cell(p, L.concTimeIndex, F.V.g.sRho, F.V.g.eta, F.V.g.xi);
        }
        if (L.steps) warp_sum_steps(L.steps, steps);
        if (L.conc && P.lastChunk) warp_count(L.conc, cell);
    }
}

template <int SEM, int STORE, int SHAPE, int VARIANT>
cudaError_t launch_move_fast(const wacomm_b200_config &cfg, const IntervalParams &P,
                             const FastView<STORE> &F, const ParticleSoA &S, const MoveLaunch &L,
                             cudaStream_t stream) {
    if (L.count <= 0) return cudaSuccess;
    constexpr int threads = LaunchShape<SHAPE>::threads;
    const int per = L.perThread > 1 ? L.perThread : 1;
    int blocks = (L.count + threads * per - 1) / (threads * per);
    move_fast_kernel<SEM, STORE, SHAPE, VARIANT><<<blocks, threads, 0, stream>>>(cfg, P, F, S, L);
    return cudaGetLastError();
}

// Host launchers (one per template instance, defined in the instantiation units).
template <int SEM, int ARITH, int STORE>
cudaError_t launch_move_soa(const wacomm_b200_config &cfg, const IntervalParams &P,
                            const PackedView<STORE> &V, const ParticleSoA &S, const MoveLaunch &L,
                            int blockSize, cudaStream_t stream) {
    if (L.count <= 0) return cudaSuccess;
    int blocks = (L.count + blockSize - 1) / blockSize;
    move_soa_kernel<SEM, ARITH, STORE><<<blocks, blockSize, 0, stream>>>(cfg, P, V, S, L);
    return cudaGetLastError();
}

}  // namespace wb
