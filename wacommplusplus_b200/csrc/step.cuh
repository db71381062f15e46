// The particle step: one particle over (a chunk of) one forcing interval, all substeps in
// registers.
//
// SEM selects the rules of the reference path being replaced: SEM_HOST follows
// Particle::move (Particle.cpp:71-824), SEM_DEVICE follows the reference kernel
// (kernel.cu:153-368); the few places where they differ are marked. ARITH_REF reproduces the
// reference arithmetic (FP64 with float-rounded corner terms; compiled with -fmad=false so that
// no product is fused), ARITH_F32 interpolates in FP32 and keeps FP64 for positions, time
// weights and metric ratios.
#pragma once

#include "common.cuh"
#include "views.cuh"

namespace wb {

// Per-launch constants of one interval, computed by make_interval on the host (engine path)
// or by each thread from device memory (drop-in path, like kernel.cu:161-171).
struct IntervalParams {
    int t0, t1, direction;
    int rng;                  // WACOMM_B200_RNG_*
    int skip;                 // the interval lies before the restart checkpoint: no change
    double start, end, length;
    long long intervalKey;    // llround(min(start, end)) (Particle.cpp:523)
    double elapsed0;          // first elapsed of the interval after a restart clip
    double chunkEnd;          // substeps that start before this elapsed run in this launch
    int firstChunk, lastChunk;
    double kLower;            // -sW + 2
    double invKLower;         // 1 / kLower (FP32 step: depth factor of the random walk)
    // Survival test without a per-step exp: health = exp(-age/tau0) is below survprob for
    // age >= ageKillHi, above it for age <= ageKillLo, and evaluated exactly in between;
    // exp(-age/tau0) > 0 is certain for age < ageUnder.
    double ageKillLo, ageKillHi, ageUnder;
    double jibeFullStep;      // jibeStepProbability(hourly, dti)
};

// Interval bounds and restart clip (Particle.cpp:109-120 with NumericalHelpers.hpp:45-52 under
// the host rules; kernel.cu:161-171 under the device rules).
__host__ __device__ inline void make_interval(const wacomm_b200_config &cfg, const double *times,
                                              int nTimes, int timeIndex, int sW, int semantics,
                                              IntervalParams &P) {
    P.direction = cfg.trackingDirection;
    int next = timeIndex + P.direction;
    bool inside = next >= 0 && next < nTimes;
    P.start = times[timeIndex];
    P.end = inside ? times[next] : P.start + P.direction * cfg.deltat;
    P.length = fabs(P.end - P.start);
    P.t0 = timeIndex;
    P.t1 = inside ? next : timeIndex;
    P.intervalKey = llround(P.start < P.end ? P.start : P.end);
    P.skip = 0;
    P.elapsed0 = 0;
    double rc = cfg.restartCheckpoint;
    if (!isnan(rc)) {
        if (semantics == WACOMM_B200_SEMANTICS_HOST) {
            if (P.end > P.start) {
                if (P.end <= rc) P.skip = 1;
                else {
                    double a = P.end - P.start, b = rc - P.start;
                    b = b < 0.0 ? 0.0 : b;
                    P.elapsed0 = b < a ? b : a;
                }
            } else {
                if (P.end >= rc) P.skip = 1;
                else {
                    double a = P.start - P.end, b = P.start - rc;
                    b = b < 0.0 ? 0.0 : b;
                    P.elapsed0 = b < a ? b : a;
                }
            }
        } else {
            if ((P.direction > 0 && P.end <= rc) || (P.direction < 0 && P.end >= rc)) P.skip = 1;
            else P.elapsed0 = fmin(P.length, fmax(0.0, P.direction * (rc - P.start)));
        }
    }
    P.kLower = -sW + 2;
    P.invKLower = 1.0 / P.kLower;
    P.chunkEnd = INFINITY;
    P.firstChunk = 1;
    P.lastChunk = 1;
    P.rng = WACOMM_B200_RNG_REFERENCE;
    double tau0 = cfg.tau0;
    if (tau0 > 0 && isfinite(tau0)) {
        P.ageUnder = 700.0 * tau0;
        if (cfg.survprob > 0 && isfinite(cfg.survprob)) {
            double a = -tau0 * log(cfg.survprob);
            P.ageKillLo = a - 1e-9 * fabs(a) - 1e-300;
            P.ageKillHi = a + 1e-9 * fabs(a) + 1e-300;
        } else {
            // survprob <= 0 is never above exp(); NaN survprob never compares true
            P.ageKillLo = INFINITY;
            P.ageKillHi = INFINITY;
        }
    } else {
        P.ageUnder = -INFINITY;
        P.ageKillLo = -INFINITY;
        P.ageKillHi = INFINITY;
    }
    double hourly = cfg.leewayJibeProbabilityHourly, dt = cfg.dti;
    if (hourly <= 0 || dt <= 0) P.jibeFullStep = 0;
    else if (hourly >= 1) P.jibeFullStep = 1;
    else P.jibeFullStep = 1 - exp(log(1 - hourly) * dt / 3600);
}

struct ParticleState {
    uint64_t id;
    double k, j, i, health, age, time;
    int type, side;
};

// ------------------------------------------------------------------ interpolation pieces

// (float)interpolateTime(v0, v1, alpha) (NumericalHelpers.hpp:37-39, kernel.cu:71-74).
__device__ __forceinline__ float at_ref(float v0, float v1, double a) {
    return (float)((1.0 - a) * (double)v0 + a * (double)v1);
}
__device__ __forceinline__ float at_f32(float v0, float v1, float a) { return fmaf(a, v1 - v0, v0); }

// Bilinear corner weights in reference order: (j,i), (j+1,i), (j+1,i+1), (j,i+1).
struct Weights32 {
    float w1, w2, w3, w4;
};
__device__ __forceinline__ Weights32 weights32(double jF, double iF) {
    float fj = (float)jF, fi = (float)iF;
    return Weights32{(1.f - fi) * (1.f - fj), (1.f - fi) * fj, fi * fj, fi * (1.f - fj)};
}

// Float sum of four float-rounded corner terms c*(1-iF)*(1-jF) ... (Particle.cpp:271-277).
__device__ __forceinline__ float bilinear_ref(float c1, float c2, float c3, float c4, double jF,
                                              double iF) {
    float f1 = (float)((double)c1 * (1.0 - iF) * (1.0 - jF));
    float f2 = (float)((double)c2 * (1.0 - iF) * jF);
    float f3 = (float)((double)c3 * iF * jF);
    float f4 = (float)((double)c4 * iF * (1.0 - jF));
    return f1 + f2 + f3 + f4;
}

// Surface at a position: bilinear h (double) and zeta (float) (Particle.cpp:271-290;
// kernel.cu:197-198).
template <int ARITH, class View>
__device__ __forceinline__ void surface_at(const View &V, int jI, int iI, double jF, double iF,
                                           double alpha, double &hh, float &zz) {
    SurfPair s1 = V.surface(jI, iI), s2 = V.surface(jI + 1, iI);
    SurfPair s3 = V.surface(jI + 1, iI + 1), s4 = V.surface(jI, iI + 1);
    hh = s1.h * (1.0 - iF) * (1.0 - jF) + s2.h * (1.0 - iF) * jF + s3.h * iF * jF +
         s4.h * iF * (1.0 - jF);
    if (ARITH == ARITH_REF) {
        zz = bilinear_ref(at_ref(s1.z0, s1.z1, alpha), at_ref(s2.z0, s2.z1, alpha),
                          at_ref(s3.z0, s3.z1, alpha), at_ref(s4.z0, s4.z1, alpha), jF, iF);
    } else {
        float a = (float)alpha;
        Weights32 w = weights32(jF, iF);
        zz = at_f32(s1.z0, s1.z1, a) * w.w1 + at_f32(s2.z0, s2.z1, a) * w.w2 +
             at_f32(s3.z0, s3.z1, a) * w.w3 + at_f32(s4.z0, s4.z1, a) * w.w4;
    }
}

// hcMid of the host rules: one double chain of four h and four zeta terms (Particle.cpp:601-604).
template <class View>
__device__ __forceinline__ double hc_mid_host(const View &V, int jI, int iI, double jF, double iF,
                                              double alpha) {
    SurfPair s1 = V.surface(jI, iI), s2 = V.surface(jI + 1, iI);
    SurfPair s3 = V.surface(jI + 1, iI + 1), s4 = V.surface(jI, iI + 1);
    return s1.h * (1.0 - iF) * (1.0 - jF) + s2.h * (1.0 - iF) * jF + s3.h * iF * jF +
           s4.h * iF * (1.0 - jF) + (double)at_ref(s1.z0, s1.z1, alpha) * (1.0 - iF) * (1.0 - jF) +
           (double)at_ref(s2.z0, s2.z1, alpha) * (1.0 - iF) * jF +
           (double)at_ref(s3.z0, s3.z1, alpha) * iF * jF +
           (double)at_ref(s4.z0, s4.z1, alpha) * iF * (1.0 - jF);
}

// Vertical field blend: host rules sum eight float terms (Particle.cpp:464-474, 490-500);
// device rules blend two float bilinears in double (kernel.cu:258-259, 265-266).
template <int SEM>
__device__ __forceinline__ double trilinear_ref(float u1, float u2, float u3, float u4, float l1,
                                                float l2, float l3, float l4, double kF,
                                                double jF, double iF) {
    if (SEM == SEM_HOST) {
        float w1 = (float)((double)u1 * (1.0 - iF) * (1.0 - jF) * (1.0 - kF));
        float w2 = (float)((double)u2 * (1.0 - iF) * jF * (1.0 - kF));
        float w3 = (float)((double)u3 * iF * jF * (1.0 - kF));
        float w4 = (float)((double)u4 * iF * (1.0 - jF) * (1.0 - kF));
        float w5 = (float)((double)l1 * (1.0 - iF) * (1.0 - jF) * kF);
        float w6 = (float)((double)l2 * (1.0 - iF) * jF * kF);
        float w7 = (float)((double)l3 * iF * jF * kF);
        float w8 = (float)((double)l4 * iF * (1.0 - jF) * kF);
        return (double)(w1 + w2 + w3 + w4 + w5 + w6 + w7 + w8);
    } else {
        return (double)bilinear_ref(u1, u2, u3, u4, jF, iF) * (1.0 - kF) +
               (double)bilinear_ref(l1, l2, l3, l4, jF, iF) * kF;
    }
}

__device__ __forceinline__ int mem_level(int kI, int sW) {
    return kI > 0 ? 0 : (kI < -sW + 2 ? -sW + 2 : kI);
}

// Keys a substep draws from: the ordered prefix (seed, particle, interval) folded once per
// interval, then the substep.
struct DrawKeys {
    uint64_t prefix;     // ordered-splitmix64 prefix through the interval coordinate
    uint64_t philoxKey;  // particle id mixed with the run seed
};

// ------------------------------------------------------------------ advective velocity

// Ocean current plus leeway and Stokes at a fractional position and forcing weight
// (Particle.cpp:352-475; kernel.cu:206-260). kI must already be a valid memory level.
template <int SEM, int ARITH, class View>
__device__ __forceinline__ void advective_velocity(const wacomm_b200_config &cfg,
                                                   const IntervalParams &P, const View &V,
                                                   const ParticleState &p, int kI, double kF,
                                                   int jI, double jF, int iI, double iF,
                                                   double sa, double elapsed,
                                                   double physicalTime, double stepDt,
                                                   const DrawKeys &keys, float &uu, float &vv,
                                                   double &ww, int *err) {
    NodeUp c1 = V.up(kI, jI, iI), c2 = V.up(kI, jI + 1, iI);
    NodeUp c3 = V.up(kI, jI + 1, iI + 1), c4 = V.up(kI, jI, iI + 1);
    NodeLo l1 = V.lo(kI, jI, iI), l2 = V.lo(kI, jI + 1, iI);
    NodeLo l3 = V.lo(kI, jI + 1, iI + 1), l4 = V.lo(kI, jI, iI + 1);
    if (ARITH == ARITH_REF) {
        uu = bilinear_ref(at_ref(c1.u0, c1.u1, sa), at_ref(c2.u0, c2.u1, sa),
                          at_ref(c3.u0, c3.u1, sa), at_ref(c4.u0, c4.u1, sa), jF, iF);
        vv = bilinear_ref(at_ref(c1.v0, c1.v1, sa), at_ref(c2.v0, c2.v1, sa),
                          at_ref(c3.v0, c3.v1, sa), at_ref(c4.v0, c4.v1, sa), jF, iF);
    } else {
        float a = (float)sa;
        Weights32 w = weights32(jF, iF);
        uu = at_f32(c1.u0, c1.u1, a) * w.w1 + at_f32(c2.u0, c2.u1, a) * w.w2 +
             at_f32(c3.u0, c3.u1, a) * w.w3 + at_f32(c4.u0, c4.u1, a) * w.w4;
        vv = at_f32(c1.v0, c1.v1, a) * w.w1 + at_f32(c2.v0, c2.v1, a) * w.w2 +
             at_f32(c3.v0, c3.v1, a) * w.w3 + at_f32(c4.v0, c4.v1, a) * w.w4;
    }
    if (cfg.driftModel == 1 && p.type != 0) {
        if (SEM == SEM_HOST && (p.type < 0 || p.type > 22)) atomicOr(err, ERR_DRIFT_OBJECT);
        double windU = cfg.windU10, windV = cfg.windV10;
        EnvPair e1{}, e2{}, e3{}, e4{};
        bool env = V.hasWindU || V.hasWindV || V.hasStokes;
        if (env) {
            e1 = V.environment(jI, iI);
            e2 = V.environment(jI + 1, iI);
            e3 = V.environment(jI + 1, iI + 1);
            e4 = V.environment(jI, iI + 1);
        }
        // environmentAt: float corner sums per record, then the time blend
        // (Particle.cpp:384-395; kernel.cu:105-116)
        if (V.hasWindU) {
            float f = (float)((double)e1.wu0 * (1.0 - iF) * (1.0 - jF)) + (float)((double)e2.wu0 * (1.0 - iF) * jF) +
                      (float)((double)e3.wu0 * iF * jF) + (float)((double)e4.wu0 * iF * (1.0 - jF));
            float n = (float)((double)e1.wu1 * (1.0 - iF) * (1.0 - jF)) + (float)((double)e2.wu1 * (1.0 - iF) * jF) +
                      (float)((double)e3.wu1 * iF * jF) + (float)((double)e4.wu1 * iF * (1.0 - jF));
            windU = (1.0 - sa) * (double)f + sa * (double)n;
        }
        if (V.hasWindV) {
            float f = (float)((double)e1.wv0 * (1.0 - iF) * (1.0 - jF)) + (float)((double)e2.wv0 * (1.0 - iF) * jF) +
                      (float)((double)e3.wv0 * iF * jF) + (float)((double)e4.wv0 * iF * (1.0 - jF));
            float n = (float)((double)e1.wv1 * (1.0 - iF) * (1.0 - jF)) + (float)((double)e2.wv1 * (1.0 - iF) * jF) +
                      (float)((double)e3.wv1 * iF * jF) + (float)((double)e4.wv1 * iF * (1.0 - jF));
            windV = (1.0 - sa) * (double)f + sa * (double)n;
        }
        uint64_t substep = (uint64_t)floor(elapsed / cfg.dti);
        double longitude = V.lon(jI, iI) * (1.0 - iF) * (1.0 - jF) + V.lon(jI + 1, iI) * (1.0 - iF) * jF +
                           V.lon(jI + 1, iI + 1) * iF * jF + V.lon(jI, iI + 1) * iF * (1.0 - jF);
        double latitude = V.lat(jI, iI) * (1.0 - iF) * (1.0 - jF) + V.lat(jI + 1, iI) * (1.0 - iF) * jF +
                          V.lat(jI + 1, iI + 1) * iF * jF + V.lat(jI, iI + 1) * iF * (1.0 - jF);
        double stdDev = cfg.windErrorStdDev, corr = cfg.windErrorComponentCorrelation;
        double spatial = cfg.windErrorSpatialScale, temporal = cfg.windErrorTemporalScale;
        int region = calibration_region(cfg, longitude, latitude);
        if (region >= 0) {
            const wacomm_b200_calibration_region &g = cfg.observationalCalibrationRegions[region];
            stdDev = g.windErrorStdDev;
            corr = g.windErrorComponentCorrelation;
            spatial = g.windErrorSpatialScale;
            temporal = g.windErrorTemporalScale;
        }
        if (stdDev > 0) {
            double when = physicalTime + .5 * P.direction * stepDt;
            double first = forcing_error_normal(cfg.randomSeed, p.id, P.intervalKey, substep,
                                                WIND_U_COMPONENT, longitude, latitude, when,
                                                spatial, temporal);
            double second = forcing_error_normal(cfg.randomSeed, p.id, P.intervalKey, substep,
                                                 WIND_V_COMPONENT, longitude, latitude, when,
                                                 spatial, temporal);
            windU += stdDev * first;
            windV += stdDev * correlated_normal(first, second, corr);
        }
        double downwindNormal = 0, crosswindNormal = 0;
        if (cfg.leewayCoefficientEnsemble) {
            uint64_t ens = key_prefix(cfg.randomSeed, p.id, ENSEMBLE_INTERVAL, 0);
            downwindNormal = prefix_normal(ens, 0);
            crosswindNormal = prefix_normal(ens, 1);
            crosswindNormal = correlated_normal(downwindNormal, crosswindNormal,
                                                cfg.leewayResidualCorrelation);
        }
        Leeway lw = compute_leeway(p.type, windU, windV, p.side, downwindNormal, crosswindNormal);
        uu += (float)lw.u;
        vv += (float)lw.v;
        if (V.hasStokes) {
            // waveAt: double corner sums (Particle.cpp:446-453; kernel.cu:118-129)
            double fu = (double)e1.su0 * (1.0 - iF) * (1.0 - jF) + (double)e2.su0 * (1.0 - iF) * jF +
                        (double)e3.su0 * iF * jF + (double)e4.su0 * iF * (1.0 - jF);
            double nu = (double)e1.su1 * (1.0 - iF) * (1.0 - jF) + (double)e2.su1 * (1.0 - iF) * jF +
                        (double)e3.su1 * iF * jF + (double)e4.su1 * iF * (1.0 - jF);
            double fv = (double)e1.sv0 * (1.0 - iF) * (1.0 - jF) + (double)e2.sv0 * (1.0 - iF) * jF +
                        (double)e3.sv0 * iF * jF + (double)e4.sv0 * iF * (1.0 - jF);
            double nv = (double)e1.sv1 * (1.0 - iF) * (1.0 - jF) + (double)e2.sv1 * (1.0 - iF) * jF +
                        (double)e3.sv1 * iF * jF + (double)e4.sv1 * iF * (1.0 - jF);
            uu += (float)((1.0 - sa) * fu + sa * nu);
            vv += (float)((1.0 - sa) * fv + sa * nv);
        }
    }
    if (ARITH == ARITH_REF) {
        ww = trilinear_ref<SEM>(at_ref(c1.w0, c1.w1, sa), at_ref(c2.w0, c2.w1, sa),
                                at_ref(c3.w0, c3.w1, sa), at_ref(c4.w0, c4.w1, sa),
                                at_ref(l1.w0, l1.w1, sa), at_ref(l2.w0, l2.w1, sa),
                                at_ref(l3.w0, l3.w1, sa), at_ref(l4.w0, l4.w1, sa), kF, jF, iF);
    } else {
        float a = (float)sa, fk = (float)kF;
        Weights32 w = weights32(jF, iF);
        float up = at_f32(c1.w0, c1.w1, a) * w.w1 + at_f32(c2.w0, c2.w1, a) * w.w2 +
                   at_f32(c3.w0, c3.w1, a) * w.w3 + at_f32(c4.w0, c4.w1, a) * w.w4;
        float lo = at_f32(l1.w0, l1.w1, a) * w.w1 + at_f32(l2.w0, l2.w1, a) * w.w2 +
                   at_f32(l3.w0, l3.w1, a) * w.w3 + at_f32(l4.w0, l4.w1, a) * w.w4;
        ww = (double)(up * (1.f - fk) + lo * fk);
    }
}

// Vertical diffusivity at the particle (Particle.cpp:490-500; kernel.cu:265-266).
template <int SEM, int ARITH, class View>
__device__ __forceinline__ double akt_at(const View &V, int kI, double kF, int jI, double jF,
                                         int iI, double iF, double alpha) {
    NodeUp c1 = V.up(kI, jI, iI), c2 = V.up(kI, jI + 1, iI);
    NodeUp c3 = V.up(kI, jI + 1, iI + 1), c4 = V.up(kI, jI, iI + 1);
    NodeLo l1 = V.lo(kI, jI, iI), l2 = V.lo(kI, jI + 1, iI);
    NodeLo l3 = V.lo(kI, jI + 1, iI + 1), l4 = V.lo(kI, jI, iI + 1);
    if (ARITH == ARITH_REF) {
        return trilinear_ref<SEM>(at_ref(c1.a0, c1.a1, alpha), at_ref(c2.a0, c2.a1, alpha),
                                  at_ref(c3.a0, c3.a1, alpha), at_ref(c4.a0, c4.a1, alpha),
                                  at_ref(l1.a0, l1.a1, alpha), at_ref(l2.a0, l2.a1, alpha),
                                  at_ref(l3.a0, l3.a1, alpha), at_ref(l4.a0, l4.a1, alpha), kF,
                                  jF, iF);
    } else {
        float a = (float)alpha, fk = (float)kF;
        Weights32 w = weights32(jF, iF);
        float up = at_f32(c1.a0, c1.a1, a) * w.w1 + at_f32(c2.a0, c2.a1, a) * w.w2 +
                   at_f32(c3.a0, c3.a1, a) * w.w3 + at_f32(c4.a0, c4.a1, a) * w.w4;
        float lo = at_f32(l1.a0, l1.a1, a) * w.w1 + at_f32(l2.a0, l2.a1, a) * w.w2 +
                   at_f32(l3.a0, l3.a1, a) * w.w3 + at_f32(l4.a0, l4.a1, a) * w.w4;
        return (double)(up * (1.f - fk) + lo * fk);
    }
}

__device__ __forceinline__ void close_upper(const wacomm_b200_config &cfg, double &k, double &health,
                                            bool &lazy) {
    if (cfg.upperClosure == CLOSURE_CONSTRAINT) k = 0;
    else if (cfg.upperClosure == CLOSURE_KILL) { health = -1; lazy = false; }
    else if (cfg.upperClosure == CLOSURE_REFLECTION) k = -k;
}

__device__ __forceinline__ void close_lower(const wacomm_b200_config &cfg, double kLower, double &k,
                                            double &health, bool &lazy) {
    if (cfg.lowerClosure == CLOSURE_CONSTRAINT) k = kLower;
    else if (cfg.lowerClosure == CLOSURE_KILL) { health = -1; lazy = false; }
    else if (cfg.lowerClosure == CLOSURE_REFLECTION) k = 2.0 * kLower - k;
}

// ------------------------------------------------------------------ the interval loop

// Integrates particle p from `elapsed` while substeps start before min(length, chunkEnd).
// On return `elapsed` is where the next chunk resumes (>= length when the particle is done).
// Returns the number of substeps taken (particle-steps of this launch).
template <int SEM, int ARITH, class View>
__device__ int move_particle(const wacomm_b200_config &cfg, const IntervalParams &P,
                             const View &V, ParticleState &p, double &elapsed, int *err) {
    const int eta = V.g.eta, xi = V.g.xi, sW = V.g.sW;
    const double kLower = P.kLower, length = P.length;
    const int direction = P.direction;
    const double dir = (double)direction;
    const bool midpoint = cfg.integrator == INTEGRATOR_MIDPOINT;
    const bool diffuse = cfg.random && (dir > 0 || cfg.backwardDiffusion);
    bool lazy = false;  // true while health == exp(-age/tau0) is owed
    int steps = 0;

    if (P.firstChunk) {
        // Closures before the loop (Particle.cpp:134-176; kernel.cu:173-182)
        if (p.k > 0) close_upper(cfg, p.k, p.health, lazy);
        if (p.k < kLower) close_lower(cfg, kLower, p.k, p.health, lazy);
    }
    DrawKeys keys;
    keys.prefix = fold(fold(mix64(cfg.randomSeed), p.id), (uint64_t)P.intervalKey);
    keys.philoxKey = p.id ^ mix64(cfg.randomSeed);
    const double stop = P.chunkEnd < length ? P.chunkEnd : length;

    while (elapsed < stop) {
        double stepDt = SEM == SEM_HOST ? smin(cfg.dti, length - elapsed)
                                        : fmin(cfg.dti, length - elapsed);
        double physicalTime = P.start + direction * elapsed;
        if (direction > 0 && p.time > physicalTime) {
            // Not yet released: jump to the release time (Particle.cpp:211-215)
            elapsed = SEM == SEM_HOST ? smin(length, p.time - P.start)
                                      : fmin(length, p.time - P.start);
            continue;
        }
        bool dead;
        if (lazy)
            dead = p.age >= P.ageKillHi ||
                   (p.age > P.ageKillLo && exp(-p.age / cfg.tau0) < cfg.survprob);
        else
            dead = p.health < cfg.survprob;
        if (dead) {
            p.health = -1;
            lazy = false;
            elapsed = length;
            break;
        }
        double kc = ceil(p.k);
        int kI = to_index<SEM>(kc);
        int jI = to_index<SEM>(floor(p.j)), iI = to_index<SEM>(floor(p.i));
        double kF = kc - p.k, jF = p.j - jI, iF = p.i - iI;
        if (!valid_cell(jI, iI, eta, xi)) {
            p.health = -1;
            lazy = false;
            elapsed = length;
            break;
        }
        if (SEM == SEM_DEVICE && (kI > 0 || kI <= -sW + 1)) {
            p.health = -1;  // device-only level test (kernel.cu:195)
            lazy = false;
            elapsed = length;
            break;
        }
        steps++;
        double alpha = length == 0 ? 0 : (elapsed + 0.5 * stepDt) / length;
        double alphaStart = length == 0 ? 0 : elapsed / length;
        double hh;
        float zz;
        surface_at<ARITH>(V, jI, iI, jF, iF, alpha, hh, zz);
        double hc = hh + zz;
        if (hc <= cfg.shoreLimit && cfg.horizontalClosure == CLOSURE_KILL) {
            p.health = -1;
            lazy = false;
            if (SEM == SEM_DEVICE) {  // the host rules finish the step (Particle.cpp:311-319)
                elapsed = length;
                break;
            }
        }
        const int kM = mem_level(kI, sW);
        float uu, vv;
        double ww;
        advective_velocity<SEM, ARITH>(cfg, P, V, p, kM, kF, jI, jF, iI, iF,
                                       midpoint ? alphaStart : alpha, elapsed, physicalTime,
                                       stepDt, keys, uu, vv, ww, err);
        double dxleap = dir * uu * stepDt, dyleap = dir * vv * stepDt;
        double dzleap = dir * (cfg.sv + ww) * stepDt;
        double rx = 0, ry = 0, rz = 0;
        uint64_t substep = 0;
        uint64_t stepKey = 0;
        bool keyed = diffuse || (cfg.leewayJibeProbabilityHourly > 0 && p.type != 0);
        if (keyed) {
            substep = (uint64_t)floor(elapsed / cfg.dti);
            stepKey = fold(keys.prefix, substep);
        }
        if (diffuse) {
            // Stochastic leap (Particle.cpp:518-533; kernel.cu:269-276)
            double aa = akt_at<SEM, ARITH>(V, kM, kF, jI, jF, iI, iF, alpha);
            double sigmaDepth = cfg.sigma * (1 - p.k / kLower);
            double scale = sqrt(stepDt / cfg.dti);
            double n0, n1, n2;
            if (P.rng == WACOMM_B200_RNG_PHILOX) {
                float f0, f1, f2;
                philox_normals3(keys.philoxKey, P.intervalKey,
                                (uint64_t)__double_as_longlong(elapsed), f0, f1, f2);
                n0 = f0;
                n1 = f1;
                n2 = f2;
            } else {
                n0 = prefix_normal(stepKey, 0);
                n1 = prefix_normal(stepKey, 1);
                n2 = prefix_normal(stepKey, 2);
            }
            rx = sigmaDepth * n0 * scale;
            ry = sigmaDepth * n1 * scale;
            rz = sigmaDepth * n2 * aa * cfg.crid * scale;
        }
        double xleap = dxleap + rx, yleap = dyleap + ry, zleap = dzleap + rz;

        double2 md = V.cell_metric(jI, iI);
        double xdist = md.x, ydist = md.y;
        double zdist = hc * V.depth_interval(kM);

        if (midpoint) {
            // Explicit midpoint (Particle.cpp:585-641; kernel.cu:281-317)
            double kHalf = dir * (cfg.sv + ww) * 0.5 * stepDt;
            if (fabs(kHalf) > zdist) kHalf = sign_of(zdist, kHalf);
            double iMid = p.i + dir * uu * 0.5 * stepDt / xdist;
            double jMid = p.j + dir * vv * 0.5 * stepDt / ydist;
            double kMid = SEM == SEM_HOST ? smin(0.0, smax(kLower, p.k + kHalf / zdist))
                                          : fmin(0.0, fmax(kLower, p.k + kHalf / zdist));
            int iMI = to_index<SEM>(floor(iMid)), jMI = to_index<SEM>(floor(jMid));
            bool midValid = valid_cell(jMI, iMI, eta, xi);
            double hcMid = 0, iMF = 0, jMF = 0;
            if (midValid) {
                iMF = iMid - iMI;
                jMF = jMid - jMI;
                if (SEM == SEM_HOST && ARITH == ARITH_REF) {
                    hcMid = hc_mid_host(V, jMI, iMI, jMF, iMF, alpha);
                } else {
                    double hm;
                    float zm;
                    surface_at<ARITH>(V, jMI, iMI, jMF, iMF, alpha, hm, zm);
                    hcMid = hm + zm;
                }
                midValid = hcMid > cfg.shoreLimit && hcMid > 0;
            }
            double detX, detY, detZ;
            if (midValid) {
                double kmc = ceil(kMid);
                int kMI = mem_level(to_index<SEM>(kmc), sW);
                double kMF = kmc - kMid;
                float um, vm;
                double wm;
                advective_velocity<SEM, ARITH>(cfg, P, V, p, kMI, kMF, jMI, jMF, iMI, iMF, alpha,
                                               elapsed, physicalTime, stepDt, keys, um, vm, wm,
                                               err);
                double2 mm = V.cell_metric(jMI, iMI);
                double zdistMid = hcMid * V.depth_interval(kMI);
                detX = dir * um * stepDt * xdist / mm.x;
                detY = dir * vm * stepDt * ydist / mm.y;
                detZ = dir * (cfg.sv + wm) * stepDt * zdist / zdistMid;
            } else {
                float ue, ve;
                double we;
                advective_velocity<SEM, ARITH>(cfg, P, V, p, kM, kF, jI, jF, iI, iF, alpha, elapsed,
                                               physicalTime, stepDt, keys, ue, ve, we, err);
                detX = dir * ue * stepDt;
                detY = dir * ve * stepDt;
                detZ = dir * (cfg.sv + we) * stepDt;
            }
            if (SEM == SEM_HOST) {
                xleap = detX + rx;
                yleap = detY + ry;
                zleap = detZ + rz;
            } else {
                xleap += detX - dir * uu * stepDt;
                yleap += detY - dir * vv * stepDt;
                zleap += detZ - dir * (cfg.sv + ww) * stepDt;
            }
        }

        // Vertical cap, candidate position and vertical closures (Particle.cpp:644-704)
        if (fabs(zleap) > zdist) zleap = sign_of(zdist, zleap);
        double jdet = p.j + yleap / ydist;
        double idet = p.i + xleap / xdist;
        double kdet = p.k + zleap / zdist;
        if (kdet > 0.) close_upper(cfg, kdet, p.health, lazy);
        if (kdet < kLower) close_lower(cfg, kLower, kdet, p.health, lazy);

        // Horizontal landing and closures (Particle.cpp:706-791; kernel.cu:331-353)
        int jdetI = to_index<SEM>(floor(jdet)), idetI = to_index<SEM>(floor(idet));
        if (valid_cell(jdetI, idetI, eta, xi)) {
            double idetF = idet - idetI, jdetF = jdet - jdetI;
            double hd;
            float zd;
            surface_at<ARITH>(V, jdetI, idetI, jdetF, idetF, alpha, hd, zd);
            double hcdet = hd + zd;
            if (hcdet <= cfg.shoreLimit) {
                if (cfg.horizontalClosure == CLOSURE_CONSTRAINT) {
                    idet = p.i;
                    jdet = p.j;
                } else if (cfg.horizontalClosure == CLOSURE_KILL) {
                    p.health = -1;
                    lazy = false;
                } else if (cfg.horizontalClosure == CLOSURE_REFLECTION) {
                    idet = reflect_cell(p.i, iI, idet, idetI);
                    jdet = reflect_cell(p.j, jI, jdet, jdetI);
                }
            }
            p.i = idet;
            p.j = jdet;
            p.k = kdet;
        } else {
            if (cfg.horizontalClosure == CLOSURE_CONSTRAINT) {
                p.k = kdet;
            } else if (cfg.horizontalClosure == CLOSURE_KILL) {
                p.health = -1;
                lazy = false;
            } else if (cfg.horizontalClosure == CLOSURE_REFLECTION) {
                p.i = reflect_domain(idet, xi - 1);
                p.j = reflect_domain(jdet, eta - 1);
                p.k = kdet;
            }
        }

        // Age, decay and jibing (Particle.cpp:797-814; kernel.cu:354-364)
        bool alive = lazy ? (p.age < P.ageUnder || exp(-p.age / cfg.tau0) > 0) : p.health > 0;
        if (alive) {
            p.age = p.age + stepDt;
            lazy = true;
            if (cfg.leewayJibeProbabilityHourly > 0 && p.type != 0) {
                double probability = stepDt == cfg.dti
                                         ? P.jibeFullStep
                                         : jibe_step_probability(cfg.leewayJibeProbabilityHourly, stepDt);
                if (prefix_uniform(stepKey, JIBE_COMPONENT) < probability) p.side = -p.side;
            }
        }
        elapsed += stepDt;
    }
    if (lazy) p.health = exp(-p.age / cfg.tau0);
    return steps;
}

}  // namespace wb
