// Test-infrastructure shim around the reference's own CUDA kernel (cuda/kernel.cu).
//
// Ours; compiled by oracle/Makefile together with the reference kernel.cu, in place, into
// oracle/_ref/libwacomm_ref_cuda.so for sm_100a. It gives tests and bench.py a C entry point
// to the reference GPU path (the unmodified cudaMoveParticle launcher, kernel.cu:370-382) so
// that the B200 kernels can be compared and timed beside it. Never linked into the product.
#include <cuda_runtime_api.h>

#include "Config.hpp"
#include "Particle.hpp"
#include "cuda/kernel.h"

extern "C" {

// All pointers are device pointers; the call is asynchronous on `stream`.
int ref_cuda_move(void *config, void *particles, int timeIndex, int T, int sW, int sRho, int eta,
                  int xi, double *times, double *mask, double *lonRad, double *latRad,
                  double *depthIntervals, double *h, float *zeta, float *u, float *v, float *w,
                  float *akt, float *windU, float *windV, float *stokesU, float *stokesV,
                  int count, void *stream) {
    cudaError_t status = cudaMoveParticle(
        static_cast<config_data *>(config), static_cast<particle_data *>(particles), timeIndex, T,
        sW, sRho, eta, xi, times, mask, lonRad, latRad, depthIntervals, h, zeta, u, v, w, akt,
        windU, windV, stokesU, stokesV, count, 0, 0, static_cast<cudaStream_t>(stream));
    return static_cast<int>(status);
}

// The reference's per-interval GPU staging (Wacomm.cpp:386-660) around its own launcher, on one
// GPU and one section: cudaMalloc and synchronous cudaMemcpy of the whole forcing window and the
// config (Wacomm.cpp:424-477), a stream, the particle section's allocation, upload from host
// memory, the move and the download (529-596), then the frees (598, 640-660). The records are
// already particle_data here, so the host pack and unpack loops (401-408, 605-608) are left out.
// Host pointers; synchronous; returns 0 or the first CUDA error code.
int ref_cuda_interval_staged(const void *configHost, void *particlesHost, int timeIndex, int T,
                             int sW, int sRho, int eta, int xi, const double *times,
                             const double *mask, const double *lonRad, const double *latRad,
                             const double *depthIntervals, const double *h, const float *zeta,
                             const float *u, const float *v, const float *w, const float *akt,
                             int count) {
    const size_t plane = (size_t)eta * xi;
    struct Upload {
        void **device;
        const void *host;
        size_t bytes;
    };
    void *dTimes = nullptr, *dDepth = nullptr, *dLon = nullptr, *dLat = nullptr, *dMask = nullptr,
         *dH = nullptr, *dZeta = nullptr, *dU = nullptr, *dV = nullptr, *dW = nullptr,
         *dAkt = nullptr, *dConfig = nullptr, *dSection = nullptr;
    const Upload uploads[] = {
        {&dTimes, times, T * sizeof(double)},
        {&dDepth, depthIntervals, (size_t)(sW - 1) * sizeof(double)},
        {&dLon, lonRad, plane * sizeof(double)},
        {&dLat, latRad, plane * sizeof(double)},
        {&dMask, mask, plane * sizeof(double)},
        {&dH, h, plane * sizeof(double)},
        {&dZeta, zeta, T * plane * sizeof(float)},
        {&dU, u, (size_t)T * sRho * plane * sizeof(float)},
        {&dV, v, (size_t)T * sRho * plane * sizeof(float)},
        {&dW, w, (size_t)T * sW * plane * sizeof(float)},
        {&dAkt, akt, (size_t)T * sW * plane * sizeof(float)},
        {&dConfig, configHost, sizeof(config_data)},
    };
    cudaError_t e = cudaSuccess;
    for (const Upload &up : uploads) {
        if (e == cudaSuccess) e = cudaMalloc(up.device, up.bytes);
        if (e == cudaSuccess) e = cudaMemcpy(*up.device, up.host, up.bytes, cudaMemcpyHostToDevice);
    }
    cudaStream_t stream = nullptr;
    if (e == cudaSuccess) e = cudaStreamCreate(&stream);
    const size_t bytes = (size_t)count * sizeof(particle_data);
    if (e == cudaSuccess && count > 0) e = cudaMalloc(&dSection, bytes);
    if (e == cudaSuccess && count > 0)
        e = cudaMemcpyAsync(dSection, particlesHost, bytes, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess && count > 0)
        e = cudaMoveParticle(static_cast<config_data *>(dConfig),
                             static_cast<particle_data *>(dSection), timeIndex, T, sW, sRho, eta,
                             xi, static_cast<double *>(dTimes), static_cast<double *>(dMask),
                             static_cast<double *>(dLon), static_cast<double *>(dLat),
                             static_cast<double *>(dDepth), static_cast<double *>(dH),
                             static_cast<float *>(dZeta), static_cast<float *>(dU),
                             static_cast<float *>(dV), static_cast<float *>(dW),
                             static_cast<float *>(dAkt), nullptr, nullptr, nullptr, nullptr, count,
                             0, 1, stream);
    if (e == cudaSuccess && count > 0)
        e = cudaMemcpyAsync(particlesHost, dSection, bytes, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess && stream) e = cudaStreamSynchronize(stream);
    if (dSection) cudaFree(dSection);
    if (stream) cudaStreamDestroy(stream);
    for (const Upload &up : uploads)
        if (*up.device) cudaFree(*up.device);
    return static_cast<int>(e);
}

}  // extern "C"
