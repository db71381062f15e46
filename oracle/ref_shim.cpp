// Test-infrastructure shim around the reference's own particle-move code.
//
// This file is ours; it is compiled together with the reference sources Particle.cpp and
// DriftModel.cpp, taken in place from the reference tree by oracle/Makefile, into
// oracle/_ref/libwacomm_ref.so. It exposes the reference CPU path behind plain C entry
// points so that tests and the CPU baseline of bench.py can call it on flat buffers:
//
//   * ref_move_batch       -> Particle::move over many particles, OpenMP schedule(dynamic,64)
//                             exactly like the solver loop (Wacomm.cpp:501-525).
//   * ref_concentration    -> Concentration::evaluate (Concentration.hpp:16-44).
//   * RNG / drift / schedule helpers -> NumericalHelpers.hpp, DriftModel.hpp, SourceEmission.hpp.
//
// It is never linked into the product library.
#include "Particle.hpp"
#include "Particles.hpp"
#include "Concentration.hpp"
#include "NumericalHelpers.hpp"
#include "DriftModel.hpp"
#include "SourceEmission.hpp"

#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

static_assert(sizeof(particle_data) == 64, "particle_data layout");
static_assert(sizeof(config_data) == 1248, "config_data layout");

// Particles.cpp needs NetCDF and nlohmann-json; the move path only needs the container.
Particles::Particles() = default;
Particles::~Particles() = default;

namespace {

struct Window {
    Array1<double> oceanTime;
    Array2<double> mask, lonRad, latRad, h;
    Array1<double> sW, depthIntervals;
    Array3<float> zeta;
    Array4<float> u, v, w, akt;
    Array3<float> windU, windV, stokesU, stokesV;
    bool hasWindU = false, hasWindV = false, hasStokesU = false, hasStokesV = false;
};

template <class T> T *mut(const T *p) { return const_cast<T *>(p); }

}  // namespace

extern "C" {

// Moves n particles (AoS particle_data records, updated in place) over one forcing
// interval with the reference Particle::move. Field layouts follow the device contract
// of cuda/kernel.cu: u,v [T][sRho][eta][xi], w,akt [T][sW][eta][xi] (level 0 = bottom),
// zeta and the optional wind/Stokes fields [T][eta][xi], depthIntervals[sW-1] indexed by
// kI+sW-2, sWValues[sW] indexed by k+sW-1. threads<=0 uses the OpenMP default.
int ref_move_batch(const void *config, void *particles, long n, int timeIndex, int T, int sW,
                   int sRho, int eta, int xi, const double *times, const double *mask,
                   const double *lonRad, const double *latRad, const double *sWValues,
                   const double *depthIntervals, const double *h, const float *zeta,
                   const float *u, const float *v, const float *w, const float *akt,
                   const float *windU, const float *windV, const float *stokesU,
                   const float *stokesV, int threads) {
    Window win;
    win.oceanTime.Dimension(T, mut(times));
    win.mask.Dimension(eta, xi, mut(mask));
    win.lonRad.Dimension(eta, xi, mut(lonRad));
    win.latRad.Dimension(eta, xi, mut(latRad));
    win.h.Dimension(eta, xi, mut(h));
    win.sW.Dimension(sW, mut(sWValues), -sW + 1);
    win.depthIntervals.Dimension(sW - 1, mut(depthIntervals), -sW + 2);
    win.zeta.Dimension(T, eta, xi, mut(zeta));
    win.u.Dimension(T, sRho, eta, xi, mut(u), 0, -sRho + 1, 0, 0);
    win.v.Dimension(T, sRho, eta, xi, mut(v), 0, -sRho + 1, 0, 0);
    win.w.Dimension(T, sW, eta, xi, mut(w), 0, -sW + 1, 0, 0);
    win.akt.Dimension(T, sW, eta, xi, mut(akt), 0, -sW + 1, 0, 0);
    if (windU) { win.windU.Dimension(T, eta, xi, mut(windU)); win.hasWindU = true; }
    if (windV) { win.windV.Dimension(T, eta, xi, mut(windV)); win.hasWindV = true; }
    if (stokesU) { win.stokesU.Dimension(T, eta, xi, mut(stokesU)); win.hasStokesU = true; }
    if (stokesV) { win.stokesV.Dimension(T, eta, xi, mut(stokesV)); win.hasStokesV = true; }

    config_data *cfg = mut(static_cast<const config_data *>(config));
    particle_data *records = static_cast<particle_data *>(particles);
    if (threads > 0) omp_set_num_threads(threads);
    #pragma omp parallel for schedule(dynamic, 64)
    for (long idx = 0; idx < n; idx++) {
        Particle particle(records[idx]);
        particle.move(cfg, timeIndex, win.oceanTime, win.mask, win.lonRad, win.latRad, win.sW,
                      win.depthIntervals, win.h, win.zeta, win.u, win.v, win.w, win.akt,
                      win.hasWindU ? &win.windU : nullptr, win.hasWindV ? &win.windV : nullptr,
                      win.hasStokesU ? &win.stokesU : nullptr,
                      win.hasStokesV ? &win.stokesV : nullptr);
        records[idx] = particle.data();
    }
    return 0;
}

// Concentration::evaluate over n AoS records into conc[Tc][sRho][eta][xi] (float counts,
// accumulated, not cleared), at concentration time index concTimeIdx.
int ref_concentration(const void *particles, long n, int concTimeIdx, int Tc, int sRho, int eta,
                      int xi, float *conc, int threads) {
    Particles container;
    const particle_data *records = static_cast<const particle_data *>(particles);
    for (long idx = 0; idx < n; idx++) container.push_back(Particle(records[idx]));
    Array4<float> grid(Tc, sRho, eta, xi, conc, 0, -sRho + 1, 0, 0);
    if (threads > 0) omp_set_num_threads(threads);
    Concentration::evaluate(&container, concTimeIdx, sRho, eta, xi, grid);
    return 0;
}

// Removes dead particles (health<=0) in place, keeping order (Wacomm.cpp:711-713).
long ref_remove_dead(void *particles, long n) {
    particle_data *records = static_cast<particle_data *>(particles);
    long kept = 0;
    for (long idx = 0; idx < n; idx++)
        if (Particle(records[idx]).isAlive()) records[kept++] = records[idx];
    return kept;
}

double ref_uniform(uint64_t seed, uint64_t particle, int64_t interval, uint64_t substep,
                   uint64_t component) {
    return NumericalHelpers::uniform(seed, particle, interval, substep, component);
}

double ref_normal(uint64_t seed, uint64_t particle, int64_t interval, uint64_t substep,
                  uint64_t component) {
    return NumericalHelpers::normal(seed, particle, interval, substep, component);
}

double ref_forcing_error_normal(uint64_t seed, uint64_t particle, int64_t interval,
                                uint64_t substep, uint64_t component, double longitude,
                                double latitude, double physicalTime, double spatialScale,
                                double temporalScale) {
    return forcingErrorNormal(seed, particle, interval, substep, component, longitude, latitude,
                              physicalTime, spatialScale, temporalScale);
}

void ref_drift_coefficients(int type, double *out9) {
    LeewayCoefficients c = driftObjectCoefficients(static_cast<DriftObjectType>(type));
    std::memcpy(out9, &c, sizeof(double) * 9);
}

void ref_compute_leeway(const double *coeff9, double windU, double windV, int side,
                        double downwindNormal, double crosswindNormal, double *outUV) {
    LeewayCoefficients c;
    std::memcpy(&c, coeff9, sizeof(double) * 9);
    DriftVelocity d = computeLeeway(c, windU, windV, static_cast<DriftSide>(side), downwindNormal,
                                    crosswindNormal);
    outUV[0] = d.u;
    outUV[1] = d.v;
}

double ref_jibe_step_probability(double hourly, double seconds) {
    return jibeStepProbability(hourly, seconds);
}

int ref_sample_drift_side(uint64_t seed, uint64_t particle, double rightProbability) {
    return static_cast<int>(sampleDriftSide(seed, particle, rightProbability));
}

double ref_source_position_offset(uint64_t seed, uint64_t particle, uint64_t component) {
    return sourcePositionOffset(seed, particle, component);
}

// sourceEmissionTimes; returns the count (or -1 on the reference's own error), writing at
// most cap values into out.
long ref_source_emission_times(int mode, double value, double sourceStart, double sourceEnd,
                               double intervalStart, double intervalEnd, double *out, long cap) {
    try {
        std::vector<double> times = sourceEmissionTimes(static_cast<EmissionMode>(mode), value,
                                                        sourceStart, sourceEnd, intervalStart,
                                                        intervalEnd);
        for (long idx = 0; idx < (long)times.size() && idx < cap; idx++) out[idx] = times[idx];
        return (long)times.size();
    } catch (...) {
        return -1;
    }
}

double ref_reflect_domain(double coordinate, double maximum) {
    return NumericalHelpers::reflectDomain(coordinate, maximum);
}

double ref_reflect_cell(double oldCoordinate, int oldCell, double candidate, int candidateCell) {
    NumericalHelpers::reflectCell(oldCoordinate, oldCell, candidate, candidateCell);
    return candidate;
}

double ref_restart_elapsed(double intervalStart, double intervalEnd, double checkpoint) {
    return NumericalHelpers::restartElapsed(intervalStart, intervalEnd, checkpoint);
}

int ref_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
