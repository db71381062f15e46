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

}  // extern "C"
