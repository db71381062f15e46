/*
 * Drop-in replacement of the reference's cuda/kernel.h (cuda/kernel.h:7).
 *
 * Declares cudaMoveParticle with the reference's exact C++ signature, so that host code written
 * against the reference (Wacomm.cpp:557-580, tests/CudaParticleParityTest.cu:134-137) compiles
 * and links against libwacomm_b200.so unchanged. As in the reference header, config_data and
 * particle_data are the caller's types (Config.hpp:36-72, Particle.hpp:31-41); the library only
 * needs their byte layout, which include/wacomm_b200.h restates as wacomm_b200_config and
 * wacomm_b200_particle. Every pointer is a device pointer; the call is asynchronous on `stream`
 * and returns the launch status, never aborting the process.
 */
#ifndef WACOMM_B200_KERNEL_H
#define WACOMM_B200_KERNEL_H

#include <cuda_runtime_api.h>

struct config_data;
struct particle_data;

cudaError_t cudaMoveParticle(config_data *, particle_data *, int, int, int, int, int, int, double *,
                             double *, double *, double *, double *, double *, float *, float *,
                             float *, float *, float *, float *, float *, float *, float *, int,
                             int, int, cudaStream_t stream = 0);

#endif
