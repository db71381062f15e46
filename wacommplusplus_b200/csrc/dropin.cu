// Drop-in replacement of the reference GPU launcher (kernel.cu:370-382): same arguments, same
// in-place update of the caller's particle_data records, device rules and reference arithmetic.
// The work is ordered by horizontal cell first (key per record, histogram, exclusive scan,
// scatter into a work order), so that the threads of a warp gather the same forcing cells; each
// record still moves independently, so the order changes no result. The ordering scratch is
// stream-ordered (cudaMallocAsync/cudaFreeAsync on the caller's stream, served from the device's
// memory pool without a device-wide synchronization); if it cannot be had, the records are moved
// in caller order. Compiled with -fmad=false.
#include "engine.h"
#include "move_kernels.cuh"
#include "wacomm_b200_kernel.h"

namespace wb {

// Cell key of each record (last bin for records outside the interpolation cells) and the
// warp-aggregated histogram of the keys.
__global__ void dropin_key_kernel(const wacomm_b200_particle *particles, int n, int eta, int xi,
                                  uint32_t *keys, uint32_t *hist) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        double fj = floor(particles[p].j), fi = floor(particles[p].i);
        uint32_t key = (fj >= 0.0 && fi >= 0.0 && fj < (double)(eta - 1) && fi < (double)(xi - 1))
                           ? (uint32_t)((int)fj * xi + (int)fi)
                           : (uint32_t)((size_t)eta * xi);
        keys[p] = key;
        unsigned peers = __match_any_sync(__activemask(), key);
        if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(hist + key, (uint32_t)__popc(peers));
    }
}

// Work order: record slots grouped by key, from the exclusive offsets of the histogram.
__global__ void dropin_scatter_kernel(const uint32_t *keys, int n, uint32_t *cursor,
                                      uint32_t *order) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        uint32_t key = keys[p];
        unsigned peers = __match_any_sync(__activemask(), key);
        int lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if (lane == leader) base = atomicAdd(cursor + key, (uint32_t)__popc(peers));
        base = __shfl_sync(peers, base, leader);
        order[base + __popc(peers & ((1u << lane) - 1u))] = (uint32_t)p;
    }
}

// One thread per record, taken in the work order (null: caller order). Like the reference
// kernel, each thread derives the interval from the device copies of config and times
// (kernel.cu:158-171); the particle is read from and written back to the caller's AoS array.
__global__ void __launch_bounds__(256) dropin_move_kernel(
    const wacomm_b200_config *__restrict__ config, wacomm_b200_particle *particles,
    const uint32_t *__restrict__ order, int timeIndex, int oceanTime,
    const double *__restrict__ times, RawView V, int count) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const wacomm_b200_config &cfg = *config;
    IntervalParams P;
    make_interval(cfg, times, oceanTime, timeIndex, V.g.sW, SEM_DEVICE, P);
    if (P.skip) return;
    RawView view = V;
    view.t0 = P.t0;
    view.t1 = P.t1;
    uint32_t idx = order ? order[t] : (uint32_t)t;
    wacomm_b200_particle rec = particles[idx];
    ParticleState p;
    p.id = rec.id;
    p.k = rec.k;
    p.j = rec.j;
    p.i = rec.i;
    p.health = rec.health;
    p.age = rec.age;
    p.time = rec.time;
    p.type = rec.driftObjectType;
    p.side = rec.driftSide;
    double elapsed = P.elapsed0;
    move_particle<SEM_DEVICE, ARITH_REF>(cfg, P, view, p, elapsed, nullptr);
    rec.k = p.k;
    rec.j = p.j;
    rec.i = p.i;
    rec.health = p.health;
    rec.age = p.age;
    rec.driftSide = (int8_t)p.side;
    particles[idx] = rec;
}

int dropin_move(const wacomm_b200_config *config, wacomm_b200_particle *particles, int timeIndex,
                int oceanTime, int sW, int sRho, int eta, int xi, const double *times,
                const double *lonRad, const double *latRad, const double *depthIntervals,
                const double *h, const float *zeta, const float *u, const float *v,
                const float *w, const float *akt, const float *windU, const float *windV,
                const float *stokesU, const float *stokesV, int count, cudaStream_t stream) {
    if (count <= 0) return (int)cudaGetLastError();
    RawView V;
    V.g = GridShape{eta, xi, sW, sRho};
    V.t0 = V.t1 = 0;
    V.zeta = zeta;
    V.u = u;
    V.v = v;
    V.w = w;
    V.akt = akt;
    V.windU = windU;
    V.windV = windV;
    V.stokesU = stokesU;
    V.stokesV = stokesV;
    V.hField = h;
    V.lonRad = lonRad;
    V.latRad = latRad;
    V.depthIntervals = depthIntervals;
    V.hasWindU = windU != nullptr;
    V.hasWindV = windV != nullptr;
    V.hasStokes = stokesU != nullptr && stokesV != nullptr;
    uint32_t *order = nullptr, *scratch = nullptr;
    if (eta >= 2 && xi >= 2) {
        // keys[count] | order[count] | histogram[bins] | offsets[bins + 1] | scan partials
        size_t bins = (size_t)eta * xi + 1;
        size_t words = 2 * (size_t)count + 2 * bins + 1 + scan_temp_words(bins);
        if (cudaMallocAsync((void **)&scratch, words * sizeof(uint32_t), stream) == cudaSuccess) {
            uint32_t *keys = scratch, *hist = scratch + 2 * (size_t)count;
            uint32_t *offsets = hist + bins, *partials = offsets + bins + 1;
            int blocks = (count + 255) / 256;
            if (blocks > 148 * 16) blocks = 148 * 16;
            cudaError_t e = cudaMemsetAsync(hist, 0, bins * sizeof(uint32_t), stream);
            if (e == cudaSuccess) {
                dropin_key_kernel<<<blocks, 256, 0, stream>>>(particles, count, eta, xi, keys,
                                                              hist);
                e = exclusive_scan(hist, offsets, bins, offsets + bins, partials, stream);
            }
            if (e == cudaSuccess) {
                order = keys + count;
                dropin_scatter_kernel<<<blocks, 256, 0, stream>>>(keys, count, offsets, order);
            } else {
                cudaFreeAsync(scratch, stream);
                return (int)e;
            }
        } else {
            scratch = nullptr;
            (void)cudaGetLastError();  // no pool memory: caller order
        }
    }
    const int threads = 128;
    int blocks = count / threads + ((count % threads) == 0 ? 0 : 1);
    dropin_move_kernel<<<blocks, threads, 0, stream>>>(config, particles, order, timeIndex,
                                                       oceanTime, times, V, count);
    cudaError_t e = cudaGetLastError();
    if (scratch) {
        cudaError_t f = cudaFreeAsync(scratch, stream);
        if (e == cudaSuccess) e = f;
    }
    return (int)e;
}

}  // namespace wb

// The reference signature (cuda/kernel.h:7), C++ linkage, so that Wacomm.cpp and the reference
// parity test link against this library unchanged.
cudaError_t cudaMoveParticle(config_data *config, particle_data *particles, int timeIndex,
                             int oceanTime, int sW, int sRho, int eta, int xi, double *times,
                             double *mask, double *lonRad, double *latRad, double *depthIntervals,
                             double *h, float *zeta, float *u, float *v, float *w, float *akt,
                             float *windU10, float *windV10, float *stokesU, float *stokesV,
                             int particleCount, int numThread, int numGPU, cudaStream_t stream) {
    (void)mask;
    (void)numThread;
    (void)numGPU;
    return (cudaError_t)wb::dropin_move(
        reinterpret_cast<const wacomm_b200_config *>(config),
        reinterpret_cast<wacomm_b200_particle *>(particles), timeIndex, oceanTime, sW, sRho, eta,
        xi, times, lonRad, latRad, depthIntervals, h, zeta, u, v, w, akt, windU10, windV10,
        stokesU, stokesV, particleCount, stream);
}

extern "C" int wacomm_b200_cuda_move_particle(
    const wacomm_b200_config *config_device, wacomm_b200_particle *particles_device,
    int time_index, int ocean_time, int s_w, int s_rho, int eta, int xi, const double *times,
    const double *mask, const double *lon_rad, const double *lat_rad,
    const double *depth_intervals, const double *h, const float *zeta, const float *u,
    const float *v, const float *w, const float *akt, const float *wind_u10,
    const float *wind_v10, const float *stokes_u, const float *stokes_v, int particle_count,
    int num_thread, int num_gpu, void *stream) {
    (void)mask;
    (void)num_thread;
    (void)num_gpu;
    return wb::dropin_move(config_device, particles_device, time_index, ocean_time, s_w, s_rho,
                           eta, xi, times, lon_rad, lat_rad, depth_intervals, h, zeta, u, v, w,
                           akt, wind_u10, wind_v10, stokes_u, stokes_v, particle_count,
                           static_cast<cudaStream_t>(stream));
}
