// Drop-in replacement of the reference GPU launcher (kernel.cu:370-382): same arguments, same
// in-place update of the caller's particle_data records, device rules and reference arithmetic.
// Compiled with -fmad=false.
#include "engine.h"
#include "move_kernels.cuh"
#include "wacomm_b200_kernel.h"

namespace wb {

// One thread per record. Like the reference kernel, each thread derives the interval from the
// device copies of config and times (kernel.cu:158-171); the particle is read from and written
// back to the caller's AoS array.
__global__ void __launch_bounds__(256) dropin_move_kernel(
    const wacomm_b200_config *__restrict__ config, wacomm_b200_particle *particles,
    int timeIndex, int oceanTime, const double *__restrict__ times, RawView V, int count) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= count) return;
    const wacomm_b200_config &cfg = *config;
    IntervalParams P;
    make_interval(cfg, times, oceanTime, timeIndex, V.g.sW, SEM_DEVICE, P);
    if (P.skip) return;
    RawView view = V;
    view.t0 = P.t0;
    view.t1 = P.t1;
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
    const int threads = 128;
    int blocks = count / threads + ((count % threads) == 0 ? 0 : 1);
    dropin_move_kernel<<<blocks, threads, 0, stream>>>(config, particles, timeIndex, oceanTime,
                                                       times, V, count);
    return (int)cudaGetLastError();
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
