// Device building blocks of the particle step: random keys, Philox streams, the leeway model,
// closure helpers and reference-exact integer conversions. Shared by every kernel unit.
#pragma once

#include <cstdint>
#include <cfloat>
#include <cuda_runtime.h>

#include "wacomm_b200.h"

namespace wb {

constexpr int SEM_HOST = WACOMM_B200_SEMANTICS_HOST;
constexpr int SEM_DEVICE = WACOMM_B200_SEMANTICS_DEVICE;
constexpr int ARITH_REF = WACOMM_B200_ARITH_REFERENCE;
constexpr int ARITH_F32 = WACOMM_B200_ARITH_FP32;
constexpr int STORE_F32 = WACOMM_B200_STORAGE_FP32;
constexpr int STORE_F16 = WACOMM_B200_STORAGE_FP16;
constexpr int STORE_BF16 = WACOMM_B200_STORAGE_BF16;

// Compiled forms of the FP32 step (move_particle_fast's VARIANT): the branches a run can reach.
constexpr int VAR_LEAN = 0;     // deterministic passive tracking: no random walk, drift or jibing
constexpr int VAR_DIFFUSE = 1;  // random walk; no drifting objects, no jibing
constexpr int VAR_DRIFT = 2;    // leeway drift without wind-error fields, calibration regions or
                                // coefficient ensemble, with or without the random walk; no jibing
constexpr int VAR_FULL = 3;     // every branch

constexpr int CLOSURE_CONSTRAINT = 1;  // Config.hpp:201-203
constexpr int CLOSURE_KILL = 2;
constexpr int CLOSURE_REFLECTION = 3;
constexpr int INTEGRATOR_MIDPOINT = 2;  // Config.hpp:207

// Error bits raised by kernels into the context's status word.
constexpr int ERR_DRIFT_OBJECT = 1;
constexpr int ERR_SURROGATE_WAIT = 8;  // a surrogate kernel gave up on a bounded barrier wait

// Random-key coordinates of the drift model (DriftModel.hpp:110-114).
constexpr long long ENSEMBLE_INTERVAL = (-9223372036854775807LL - 1);
constexpr unsigned long long JIBE_COMPONENT = 0x4a494245ULL;
constexpr unsigned long long WIND_U_COMPONENT = 0x57494e4455ULL;
constexpr unsigned long long WIND_V_COMPONENT = 0x57494e4456ULL;

// ------------------------------------------------------------------ ordered SplitMix64 keys
// Scheme ordered-splitmix64-v2 (NumericalHelpers.hpp:84-120): the key folds seed, particle,
// interval, substep and component in that order through the SplitMix64 finaliser, so the
// (seed, particle, interval) prefix is computed once per interval and (substep) once per step.

__device__ __forceinline__ uint64_t mix64(uint64_t value) {
    value += 0x9e3779b97f4a7c15ULL;
    value = (value ^ (value >> 30)) * 0xbf58476d1ce4e5b9ULL;
    value = (value ^ (value >> 27)) * 0x94d049bb133111ebULL;
    return value ^ (value >> 31);
}

__device__ __forceinline__ uint64_t fold(uint64_t state, uint64_t coordinate) {
    return mix64(state ^ coordinate);
}

__device__ __forceinline__ double key_uniform(uint64_t key) {
    return (double)(key >> 11) * 0x1.0p-53;
}

// Uniform of component c under a prefix already folded through substep.
__device__ __forceinline__ double prefix_uniform(uint64_t prefix, uint64_t component) {
    return key_uniform(fold(prefix, component));
}

// Box-Muller normal of component c from uniforms 2c and 2c+1 (NumericalHelpers.hpp:114-120).
__device__ __forceinline__ double prefix_normal(uint64_t prefix, uint64_t component) {
    double u1 = fmax(prefix_uniform(prefix, component * 2), DBL_MIN);
    double u2 = prefix_uniform(prefix, component * 2 + 1);
    return sqrt(-2.0 * log(u1)) * cos(6.28318530717958647692 * u2);
}

__device__ __forceinline__ uint64_t key_prefix(uint64_t seed, uint64_t particle, long long interval,
                                               uint64_t substep) {
    return fold(fold(fold(mix64(seed), particle), (uint64_t)interval), substep);
}

__device__ __forceinline__ double full_normal(uint64_t seed, uint64_t particle, long long interval,
                                              uint64_t substep, uint64_t component) {
    return prefix_normal(key_prefix(seed, particle, interval, substep), component);
}

// Shared Earth-relative wind-error field (DriftModel.hpp:118-140).
__device__ __forceinline__ double forcing_error_normal(uint64_t seed, uint64_t particle,
                                                       long long interval, uint64_t substep,
                                                       uint64_t component, double longitude,
                                                       double latitude, double physicalTime,
                                                       double spatialScale, double temporalScale) {
    if (spatialScale <= 0 && temporalScale <= 0)
        return full_normal(seed, particle, interval, substep, component);
    uint64_t spatialKey = particle;
    if (spatialScale > 0) {
        const double earthRadius = 6371000.0;
        long long x = (long long)floor(earthRadius * longitude * cos(latitude) / spatialScale);
        long long y = (long long)floor(earthRadius * latitude / spatialScale);
        spatialKey = fold(mix64((uint64_t)x), (uint64_t)y);
    }
    long long timeKey = interval;
    uint64_t sampleKey = substep;
    if (temporalScale > 0) {
        timeKey = (long long)floor(physicalTime / temporalScale);
        sampleKey = 0;
    }
    return full_normal(seed, spatialKey, timeKey, sampleKey, component);
}

__device__ __forceinline__ double correlated_normal(double first, double independent,
                                                    double correlation) {
    return correlation * first + sqrt(1 - correlation * correlation) * independent;
}

// ------------------------------------------------------------------ Philox4x32-10 streams
// Counter-based generator (Salmon et al., SC'11) keyed on the stable 64-bit particle id and the
// run seed; the counter holds (substep, interval). Four 32-bit words give two Box-Muller pairs.

struct Philox4 {
    uint32_t x, y, z, w;
};

__device__ __forceinline__ Philox4 philox4x32_10(Philox4 ctr, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int round = 0; round < 10; round++) {
        uint32_t hi0 = __umulhi(0xD2511F53u, ctr.x), lo0 = 0xD2511F53u * ctr.x;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, ctr.z), lo1 = 0xCD9E8D57u * ctr.z;
        ctr = Philox4{hi1 ^ ctr.y ^ k0, lo1, hi0 ^ ctr.w ^ k1, lo0};
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return ctr;
}

// Three standard normals in single precision for (particle key, interval, step), the step named by
// any 64-bit value unique within the interval (the bits of its elapsed time).
__device__ __forceinline__ void philox_normals3(uint64_t key, long long interval, uint64_t step,
                                                float &n0, float &n1, float &n2) {
    Philox4 ctr{(uint32_t)step, (uint32_t)(step >> 32), (uint32_t)interval,
                (uint32_t)((uint64_t)interval >> 32)};
    Philox4 r = philox4x32_10(ctr, (uint32_t)key, (uint32_t)(key >> 32));
    const float scale = 2.3283064365386963e-10f;  // 2^-32; uniforms in (0,1]
    float u0 = ((float)r.x + 1.0f) * scale, u1 = (float)r.y * scale;
    float u2 = ((float)r.z + 1.0f) * scale, u3 = (float)r.w * scale;
    // radius sqrt(-2 ln u) as x rsqrt(x) (the hardware reciprocal square root, about 2 ulp),
    // with x kept off zero (u = 1 gives a radius of 1e-15 instead of 0 * inf)
    const float x0 = fmaxf(-2.0f * __logf(u0), 1e-30f), x2 = fmaxf(-2.0f * __logf(u2), 1e-30f);
    float rad0 = x0 * rsqrtf(x0), rad1 = x2 * rsqrtf(x2);
    // angles (2u - 1) pi in [-pi, pi), where the hardware sine and cosine are accurate to ~5e-7
    const float pi = 3.14159265358979f;
    float s0, c0, s1, c1;
    __sincosf(fmaf(2.0f, u1, -1.0f) * pi, &s0, &c0);
    __sincosf(fmaf(2.0f, u3, -1.0f) * pi, &s1, &c1);
    n0 = rad0 * c0;
    n1 = rad0 * s0;
    n2 = rad1 * c1;
}

// ------------------------------------------------------------------ drift objects
// Leeway regression coefficients per DriftObjectType id, in LeewayCoefficients order
// (DriftModel.hpp:46-56; values DriftModel.hpp:176-202).
#define WB_LEEWAY_CATALOGUE { \
    {0, 0, 0, 0, 0, 0, 0, 0, 0}, \
    {.0096, 0, .12, .0054, 0, .094, -.0054, 0, .094}, \
    {.0339, 0, .024, .0149, 0, .024, -.0149, 0, .024}, \
    {.0121, 0, .12, .0092, 0, .094, -.0092, 0, .094}, \
    {.0247, 0, .12, .0276, 0, .094, -.0276, 0, .094}, \
    {.0125, .0396, .0281, .0019, .0114, .0436, -.0019, -.0114, .0436}, \
    {.0048, 0, .083, .0015, 0, .067, -.0015, 0, .067}, \
    {.0171, .0112, .0393, .0136, -.033, .0171, -.0013, -.0265, .0162}, \
    {.01117, .102, .0304, .0004, .039, .0405, -.0004, -.039, .0405}, \
    {.0352, -.025, .061, .0062, -.03, .035, -.0045, -.002, .036}, \
    {.0088, 0, .025, .0018, 0, .024, -.0018, 0, .024}, \
    {.0116, .1112, .0412, .0041, 0, .0439, -.0041, 0, .0439}, \
    {.0193, 0, .083, .0051, 0, .067, -.0051, 0, .067}, \
    {.0315, 0, .022, .0129, 0, .022, -.0129, 0, .022}, \
    {.0165, 0, .031, .0039, 0, .029, -.0039, 0, .029}, \
    {.0654, 0, .03, .0219, 0, .028, -.0219, 0, .028}, \
    {.0187, 0, .083, .0209, 0, .067, -.0209, 0, .067}, \
    {.045, 0, .194, .0495, 0, .1842, -.0282, 0, .2495}, \
    {.0197, 0, .083, .0036, 0, .067, -.0036, 0, .067}, \
    {.0075, .0266, .0283, .0048, .0288, .0392, -.0045, -.0146, .0459}, \
    {.0107, .0447, .0655, .0041, .0115, .0413, -.0041, -.0115, .0413}, \
    {.0156, .083, .0153, .00078, .027, .0152, -.00078, -.027, .0152}, \
    {.0275, 0, .12, .005, 0, .094, -.005, 0, .094}, \
}

__constant__ static double c_leeway_catalogue[23][9] = WB_LEEWAY_CATALOGUE;
// The same rows in FP32 for the FP32 step, read through L1 (lanes of a warp may hold
// different objects; constant-bank reads of different addresses would serialize).
__device__ static const float c_leeway_catalogue_f32[23][9] = WB_LEEWAY_CATALOGUE;

struct Leeway {
    double u, v;
};

// computeLeeway (DriftModel.hpp:204-219) for catalogue row `type`; unknown rows give zero
// coefficients (the reference kernel's switch default).
__device__ __forceinline__ Leeway compute_leeway(int type, double windU, double windV, int side,
                                                 double downwindNormal, double crosswindNormal) {
    double speed = sqrt(windU * windU + windV * windV);
    if (speed < 1.0e-12 || side == 0) return Leeway{0, 0};
    const double *c = (type >= 0 && type <= 22) ? c_leeway_catalogue[type] : nullptr;
    double c0 = c ? c[0] : 0, c1 = c ? c[1] : 0, c2 = c ? c[2] : 0, c3 = c ? c[3] : 0;
    double c4 = c ? c[4] : 0, c5 = c ? c[5] : 0, c6 = c ? c[6] : 0, c7 = c ? c[7] : 0;
    double c8 = c ? c[8] : 0;
    double du = windU / speed, dv = windV / speed;
    double downwind = c0 * speed + c1 + c2 * downwindNormal;
    bool right = side == 1;
    double crosswind = (right ? c3 : c6) * speed + (right ? c4 : c7) + (right ? c5 : -c8) * crosswindNormal;
    return Leeway{downwind * du - crosswind * dv, downwind * dv + crosswind * du};
}

// DriftModel.hpp:95-108
__device__ __forceinline__ int calibration_region(const wacomm_b200_config &cfg, double lonRad,
                                                  double latRad) {
    const double radiansToDegrees = 57.2957795130823208768;
    double lon = lonRad * radiansToDegrees, lat = latRad * radiansToDegrees;
    for (uint32_t r = 0; r < cfg.observationalCalibrationRegionCount && r < 16; r++) {
        const wacomm_b200_calibration_region &g = cfg.observationalCalibrationRegions[r];
        if (lon >= g.west && lon <= g.east && lat >= g.south && lat <= g.north) return (int)r;
    }
    return -1;
}

// DriftModel.hpp:156-160
__device__ __forceinline__ double jibe_step_probability(double hourly, double seconds) {
    if (hourly <= 0 || seconds <= 0) return 0;
    if (hourly >= 1) return 1;
    return 1 - exp(log(1 - hourly) * seconds / 3600);
}

// ------------------------------------------------------------------ numerical helpers

// NumericalHelpers.hpp:62-65
__device__ __forceinline__ double reflect_cell(double oldCoordinate, int oldCell, double candidate,
                                               int candidateCell) {
    if (candidateCell < oldCell) return oldCell + fabs(oldCoordinate - candidate);
    // fmod(x, 1) is x - trunc(x) exactly (both are exact for every finite double)
    if (candidateCell > oldCell) return candidateCell - (candidate - trunc(candidate));
    return candidate;
}

// NumericalHelpers.hpp:67-74
__device__ __forceinline__ double reflect_domain(double coordinate, double maximum) {
    if (maximum <= 0) return 0;
    // fmod returns its argument when |coordinate| < 2 maximum (exact): the library call only for
    // positions more than a domain away
    const double period = 2.0 * maximum;
    double reflected = fabs(coordinate) < period ? coordinate : fmod(coordinate, period);
    if (reflected < 0) reflected += 2.0 * maximum;
    if (reflected >= maximum) reflected = 2.0 * maximum - reflected;
    if (reflected >= maximum) reflected = nextafter(maximum, 0.0);
    return reflected;
}

__device__ __forceinline__ bool valid_cell(int j, int i, int eta, int xi) {
    return j >= 0 && i >= 0 && j + 1 < eta && i + 1 < xi;
}

// Index of floor/ceil results. Host semantics reproduce x86-64 truncation (NaN and values out of
// int range become INT_MIN, which every cell and level test rejects); device semantics keep the
// GPU conversion of the reference kernel (NaN -> 0, out of range saturates).
template <int SEM>
__device__ __forceinline__ int to_index(double integral) {
    if (SEM == SEM_HOST) {
        if (!(integral >= -2147483648.0 && integral < 2147483648.0)) return (int)0x80000000u;
        return (int)integral;
    } else {
        return __double2int_rz(integral);
    }
}

__device__ __forceinline__ double sgn(double a) { return (double)((a > 0) - (a < 0)); }
__device__ __forceinline__ double sign_of(double a, double b) { return fabs(a) * sgn(b); }

// std::min / std::max argument order (NaN handling of the host semantics).
__device__ __forceinline__ double smin(double a, double b) { return b < a ? b : a; }
__device__ __forceinline__ double smax(double a, double b) { return a < b ? b : a; }

}  // namespace wb
