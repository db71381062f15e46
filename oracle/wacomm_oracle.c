/*
 * CPU oracle of the WaComM++ particle-move path -- TEST INFRASTRUCTURE ONLY (see the header).
 *
 * Arithmetic is written so that each rounding step of the reference is reproduced: values
 * the reference holds in float are held in float here, products are evaluated in the same
 * order, and the file is compiled with -ffp-contract=off so that no multiply-add is fused
 * (the reference's x86-64 Release build has none). With the same libm the host-semantics
 * move is bit-identical to the reference Particle::move (tests/test_oracle_vs_reference.py).
 */
#include "wacomm_oracle.h"

#include <float.h>
#include <stdio.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

_Static_assert(sizeof(wo_particle) == 64, "particle_data is 64 bytes");
_Static_assert(sizeof(wo_config) == 1248, "config_data is 1248 bytes");

/* ---------------------------------------------------------------- random keys */

/* SplitMix64 finaliser (NumericalHelpers.hpp:84-89). */
uint64_t wo_mix(uint64_t value) {
    value += 0x9e3779b97f4a7c15ULL;
    value = (value ^ (value >> 30)) * 0xbf58476d1ce4e5b9ULL;
    value = (value ^ (value >> 27)) * 0x94d049bb133111ebULL;
    return value ^ (value >> 31);
}

/* Ordered coordinate fold (NumericalHelpers.hpp:100-102). */
uint64_t wo_combine(uint64_t state, uint64_t coordinate) { return wo_mix(state ^ coordinate); }

/* Uniform on [0,1) with 53 bits from the folded key (NumericalHelpers.hpp:104-112). */
double wo_uniform(uint64_t seed, uint64_t particle, int64_t interval, uint64_t substep,
                  uint64_t component) {
    uint64_t key = wo_mix(seed);
    key = wo_combine(key, particle);
    key = wo_combine(key, (uint64_t)interval);
    key = wo_combine(key, substep);
    key = wo_combine(key, component);
    return (double)(key >> 11) * 0x1.0p-53;
}

/* Box-Muller from components 2c and 2c+1 (NumericalHelpers.hpp:114-120). */
double wo_normal(uint64_t seed, uint64_t particle, int64_t interval, uint64_t substep,
                 uint64_t component) {
    double u1 = wo_uniform(seed, particle, interval, substep, component * 2);
    if (u1 < DBL_MIN) u1 = DBL_MIN;
    double u2 = wo_uniform(seed, particle, interval, substep, component * 2 + 1);
    return sqrt(-2.0 * log(u1)) * cos(6.28318530717958647692 * u2);
}

/* ---------------------------------------------------------------- drift model */

#define WO_ENSEMBLE_INTERVAL ((int64_t)(-9223372036854775807LL - 1))
#define WO_SIDE_INTERVAL (WO_ENSEMBLE_INTERVAL + 1)
#define WO_SOURCE_INTERVAL (WO_ENSEMBLE_INTERVAL + 2)
#define WO_JIBE_COMPONENT 0x4a494245ULL
#define WO_WIND_U_COMPONENT 0x57494e4455ULL
#define WO_WIND_V_COMPONENT 0x57494e4456ULL

/* Shared Earth-relative wind-error field (DriftModel.hpp:118-140). */
double wo_forcing_error_normal(uint64_t seed, uint64_t particle, int64_t interval,
                               uint64_t substep, uint64_t component, double longitude,
                               double latitude, double physicalTime, double spatialScale,
                               double temporalScale) {
    if (spatialScale <= 0 && temporalScale <= 0)
        return wo_normal(seed, particle, interval, substep, component);
    uint64_t spatialKey = particle;
    if (spatialScale > 0) {
        const double earthRadius = 6371000.0;
        int64_t x = (int64_t)floor(earthRadius * longitude * cos(latitude) / spatialScale);
        int64_t y = (int64_t)floor(earthRadius * latitude / spatialScale);
        spatialKey = wo_combine(wo_mix((uint64_t)x), (uint64_t)y);
    }
    int64_t timeKey = interval;
    uint64_t sampleKey = substep;
    if (temporalScale > 0) {
        timeKey = (int64_t)floor(physicalTime / temporalScale);
        sampleKey = 0;
    }
    return wo_normal(seed, spatialKey, timeKey, sampleKey, component);
}

/* DriftModel.hpp:142-145. */
double wo_correlated_normal(double first, double independent, double correlation) {
    return correlation * first + sqrt(1 - correlation * correlation) * independent;
}

/* Hourly hazard to a per-step probability (DriftModel.hpp:156-160). */
double wo_jibe_step_probability(double hourly, double seconds) {
    if (hourly <= 0 || seconds <= 0) return 0;
    if (hourly >= 1) return 1;
    return 1 - exp(log(1 - hourly) * seconds / 3600);
}

/* Leeway catalogue, in the column order of LeewayCoefficients (DriftModel.hpp:46-56,
 * values DriftModel.hpp:176-202). Row index = DriftObjectType id. */
static const double wo_catalogue[23][9] = {
    {0, 0, 0, 0, 0, 0, 0, 0, 0},
    {.0096, 0, .12, .0054, 0, .094, -.0054, 0, .094},
    {.0339, 0, .024, .0149, 0, .024, -.0149, 0, .024},
    {.0121, 0, .12, .0092, 0, .094, -.0092, 0, .094},
    {.0247, 0, .12, .0276, 0, .094, -.0276, 0, .094},
    {.0125, .0396, .0281, .0019, .0114, .0436, -.0019, -.0114, .0436},
    {.0048, 0, .083, .0015, 0, .067, -.0015, 0, .067},
    {.0171, .0112, .0393, .0136, -.033, .0171, -.0013, -.0265, .0162},
    {.01117, .102, .0304, .0004, .039, .0405, -.0004, -.039, .0405},
    {.0352, -.025, .061, .0062, -.03, .035, -.0045, -.002, .036},
    {.0088, 0, .025, .0018, 0, .024, -.0018, 0, .024},
    {.0116, .1112, .0412, .0041, 0, .0439, -.0041, 0, .0439},
    {.0193, 0, .083, .0051, 0, .067, -.0051, 0, .067},
    {.0315, 0, .022, .0129, 0, .022, -.0129, 0, .022},
    {.0165, 0, .031, .0039, 0, .029, -.0039, 0, .029},
    {.0654, 0, .03, .0219, 0, .028, -.0219, 0, .028},
    {.0187, 0, .083, .0209, 0, .067, -.0209, 0, .067},
    {.045, 0, .194, .0495, 0, .1842, -.0282, 0, .2495},
    {.0197, 0, .083, .0036, 0, .067, -.0036, 0, .067},
    {.0075, .0266, .0283, .0048, .0288, .0392, -.0045, -.0146, .0459},
    {.0107, .0447, .0655, .0041, .0115, .0413, -.0041, -.0115, .0413},
    {.0156, .083, .0153, .00078, .027, .0152, -.00078, -.027, .0152},
    {.0275, 0, .12, .005, 0, .094, -.005, 0, .094},
};

int wo_drift_coefficients(int type, double out9[9]) {
    if (type < 0 || type > 22) {
        memset(out9, 0, 9 * sizeof(double));
        return -1;
    }
    memcpy(out9, wo_catalogue[type], 9 * sizeof(double));
    return 0;
}

/* Downwind/crosswind regression rotated into the wind frame (DriftModel.hpp:204-219). */
void wo_compute_leeway(const double c[9], double windU, double windV, int side,
                       double downwindNormal, double crosswindNormal, double outUV[2]) {
    double speed = sqrt(windU * windU + windV * windV);
    if (speed < 1.0e-12 || side == 0) {
        outUV[0] = 0;
        outUV[1] = 0;
        return;
    }
    double du = windU / speed, dv = windV / speed;
    double downwind = c[0] * speed + c[1] + c[2] * downwindNormal;
    int right = side == 1;
    double crosswind = (right ? c[3] : c[6]) * speed + (right ? c[4] : c[7]) +
                       (right ? c[5] : -c[8]) * crosswindNormal;
    outUV[0] = downwind * du - crosswind * dv;
    outUV[1] = downwind * dv + crosswind * du;
}

/* First closed lon/lat box containing the point (DriftModel.hpp:95-108). */
int wo_calibration_region(const wo_region *regions, uint32_t count, double lonRad,
                          double latRad) {
    const double radiansToDegrees = 57.2957795130823208768;
    double lon = lonRad * radiansToDegrees, lat = latRad * radiansToDegrees;
    for (uint32_t r = 0; r < count; r++)
        if (lon >= regions[r].west && lon <= regions[r].east && lat >= regions[r].south &&
            lat <= regions[r].north)
            return (int)r;
    return -1;
}

/* DriftModel.hpp:147-154. */
int wo_sample_drift_side(uint64_t seed, uint64_t particle, double rightProbability) {
    return wo_uniform(seed, particle, WO_SIDE_INTERVAL, 0, 0) < rightProbability ? 1 : -1;
}

/* ---------------------------------------------------------------- numerical helpers */

/* NumericalHelpers.hpp:45-52 (NaN = the interval lies before the checkpoint). */
double wo_restart_elapsed(double intervalStart, double intervalEnd, double checkpoint) {
    if (intervalEnd > intervalStart) {
        if (intervalEnd <= checkpoint) return NAN;
        double a = intervalEnd - intervalStart, b = checkpoint - intervalStart;
        if (b < 0.0) b = 0.0;
        return b < a ? b : a;
    }
    if (intervalEnd >= checkpoint) return NAN;
    double a = intervalStart - intervalEnd, b = intervalStart - checkpoint;
    if (b < 0.0) b = 0.0;
    return b < a ? b : a;
}

/* NumericalHelpers.hpp:62-65. */
double wo_reflect_cell(double oldCoordinate, int oldCell, double candidate, int candidateCell) {
    if (candidateCell < oldCell) return oldCell + fabs(oldCoordinate - candidate);
    if (candidateCell > oldCell) return candidateCell - fmod(candidate, 1.0);
    return candidate;
}

/* NumericalHelpers.hpp:67-74. */
double wo_reflect_domain(double coordinate, double maximum) {
    if (maximum <= 0) return 0;
    double reflected = fmod(coordinate, 2.0 * maximum);
    if (reflected < 0) reflected += 2.0 * maximum;
    if (reflected >= maximum) reflected = 2.0 * maximum - reflected;
    if (reflected >= maximum) reflected = nextafter(maximum, 0.0);
    return reflected;
}

static int valid_cell(int j, int i, int eta, int xi) {
    return j >= 0 && i >= 0 && j + 1 < eta && i + 1 < xi;
}

/* static_cast<int>(std::floor/ceil(x)) for finite in-range x; out-of-range values (undefined
 * in the reference) map to INT_MIN, which every cell and level check rejects. */
static int to_int(double x) {
    if (!(x >= -2147483648.0 && x < 2147483648.0)) return (int)0x80000000u;
    return (int)x;
}

static double dmin(double a, double b) { return b < a ? b : a; } /* std::min */
static double dmax(double a, double b) { return a < b ? b : a; } /* std::max */
static double sgn(double a) { return (double)((a > 0) - (a < 0)); }
static double sign_of(double a, double b) { return fabs(a) * sgn(b); } /* Particle.cpp:841 */

/* ---------------------------------------------------------------- particle move */

typedef struct interval_state {
    const wo_config *cfg;
    const wo_window *win;
    int t0, t1;            /* forcing records bracketing the interval */
    int direction;
    double start, end, length;
    int64_t intervalKey;   /* llround(min(start,end)) */
    size_t plane;          /* eta*xi */
} interval_state;

static size_t idx2(const interval_state *s, int j, int i) {
    return (size_t)j * (size_t)s->win->xi + (size_t)i;
}

/* Clamp a logical level for memory safety; in-range levels are unchanged. */
static int clamp_level(int k, int levels) {
    if (k > 0) return 0;
    if (k < -levels + 1) return -levels + 1;
    return k;
}

static float rec3(const interval_state *s, const float *f, int t, int j, int i) {
    return f[(size_t)t * s->plane + idx2(s, j, i)];
}

static float rec4(const interval_state *s, const float *f, int levels, int t, int k, int j,
                  int i) {
    k = clamp_level(k, levels);
    return f[((size_t)t * (size_t)levels + (size_t)(k + levels - 1)) * s->plane + idx2(s, j, i)];
}

/* (float)interpolateTime(f(t0), f(t1), alpha) (NumericalHelpers.hpp:37-39). */
static float at3(const interval_state *s, const float *f, int j, int i, double alpha) {
    double v0 = rec3(s, f, s->t0, j, i), v1 = rec3(s, f, s->t1, j, i);
    return (float)((1.0 - alpha) * v0 + alpha * v1);
}

static float at4(const interval_state *s, const float *f, int levels, int k, int j, int i,
                 double alpha) {
    double v0 = rec4(s, f, levels, s->t0, k, j, i), v1 = rec4(s, f, levels, s->t1, k, j, i);
    return (float)((1.0 - alpha) * v0 + alpha * v1);
}

/* Bilinear float sum of time-interpolated corners: zetaAt terms (Particle.cpp:271-277),
 * bilinear(float*) (kernel.cu:87-94). Each corner term is rounded to float. */
static float bilinear_t(const interval_state *s, const float *f, int j, int i, double jf,
                        double ifr, double alpha) {
    float f1 = (float)(at3(s, f, j, i, alpha) * (1.0 - ifr) * (1.0 - jf));
    float f2 = (float)(at3(s, f, j + 1, i, alpha) * (1.0 - ifr) * jf);
    float f3 = (float)(at3(s, f, j + 1, i + 1, alpha) * ifr * jf);
    float f4 = (float)(at3(s, f, j, i + 1, alpha) * ifr * (1.0 - jf));
    return f1 + f2 + f3 + f4;
}

static float bilinear_t4(const interval_state *s, const float *f, int levels, int k, int j,
                         int i, double jf, double ifr, double alpha) {
    float f1 = (float)(at4(s, f, levels, k, j, i, alpha) * (1.0 - ifr) * (1.0 - jf));
    float f2 = (float)(at4(s, f, levels, k, j + 1, i, alpha) * (1.0 - ifr) * jf);
    float f3 = (float)(at4(s, f, levels, k, j + 1, i + 1, alpha) * ifr * jf);
    float f4 = (float)(at4(s, f, levels, k, j, i + 1, alpha) * ifr * (1.0 - jf));
    return f1 + f2 + f3 + f4;
}

/* Bilinear of a double 2-D field (Particle.cpp:281-287, kernel.cu:82-85). */
static double bilinear_d(const interval_state *s, const double *f, int j, int i, double jf,
                         double ifr) {
    return f[idx2(s, j, i)] * (1.0 - ifr) * (1.0 - jf) + f[idx2(s, j + 1, i)] * (1.0 - ifr) * jf +
           f[idx2(s, j + 1, i + 1)] * ifr * jf + f[idx2(s, j, i + 1)] * ifr * (1.0 - jf);
}

/* Trilinear float sum of 8 corners (Particle.cpp:464-474 and 490-500). */
static float trilinear_f(const interval_state *s, const float *f, int levels, int kI, double kF,
                         int j, int i, double jf, double ifr, double alpha) {
    float w1 = (float)(at4(s, f, levels, kI, j, i, alpha) * (1.0 - ifr) * (1.0 - jf) * (1.0 - kF));
    float w2 = (float)(at4(s, f, levels, kI, j + 1, i, alpha) * (1.0 - ifr) * jf * (1.0 - kF));
    float w3 = (float)(at4(s, f, levels, kI, j + 1, i + 1, alpha) * ifr * jf * (1.0 - kF));
    float w4 = (float)(at4(s, f, levels, kI, j, i + 1, alpha) * ifr * (1.0 - jf) * (1.0 - kF));
    float w5 = (float)(at4(s, f, levels, kI - 1, j, i, alpha) * (1.0 - ifr) * (1.0 - jf) * kF);
    float w6 = (float)(at4(s, f, levels, kI - 1, j + 1, i, alpha) * (1.0 - ifr) * jf * kF);
    float w7 = (float)(at4(s, f, levels, kI - 1, j + 1, i + 1, alpha) * ifr * jf * kF);
    float w8 = (float)(at4(s, f, levels, kI - 1, j, i + 1, alpha) * ifr * (1.0 - jf) * kF);
    return w1 + w2 + w3 + w4 + w5 + w6 + w7 + w8;
}

/* Host metric (Particle.cpp:548-574): haversine along one grid axis with the cross
 * difference dropped; pow() as the reference writes it. */
static double host_metric(double dLat, double dLon, double latA, double latB) {
    double dLatLon = pow(sin(0.5 * dLat), 2) + pow(sin(0.5 * dLon), 2) * cos(latA) * cos(latB);
    return 2.0 * atan2(pow(dLatLon, .5), pow(1.0 - dLatLon, .5)) * 6371000.0;
}

/* Device metric (kernel.cu:145-149): full haversine between two nodes. */
static double device_distance(double lat0, double lon0, double lat1, double lon1) {
    double dLat = lat1 - lat0, dLon = lon1 - lon0;
    double value = sin(.5 * dLat) * sin(.5 * dLat) + sin(.5 * dLon) * sin(.5 * dLon) * cos(lat1) * cos(lat0);
    return 2.0 * atan2(sqrt(value), sqrt(1.0 - value)) * 6371000.0;
}

static void cell_metric(const interval_state *s, int semantics, int j, int i, double *xdist,
                        double *ydist) {
    const double *lat = s->win->latRad, *lon = s->win->lonRad;
    if (semantics == WO_SEMANTICS_HOST) {
        *ydist = host_metric(lat[idx2(s, j + 1, i)] - lat[idx2(s, j, i)], 0, lat[idx2(s, j + 1, i)],
                             lat[idx2(s, j, i)]);
        *xdist = host_metric(0, lon[idx2(s, j, i + 1)] - lon[idx2(s, j, i)], lat[idx2(s, j, i + 1)],
                             lat[idx2(s, j, i)]);
    } else {
        *ydist = device_distance(lat[idx2(s, j, i)], lon[idx2(s, j, i)], lat[idx2(s, j + 1, i)],
                                 lon[idx2(s, j + 1, i)]);
        *xdist = device_distance(lat[idx2(s, j, i)], lon[idx2(s, j, i)], lat[idx2(s, j, i + 1)],
                                 lon[idx2(s, j, i + 1)]);
    }
}

static double depth_interval(const interval_state *s, int kI) {
    int sW = s->win->sW;
    int index = kI + sW - 2;
    if (index < 0) index = 0;
    if (index > sW - 2) index = sW - 2;
    return s->win->depthIntervals[index];
}

/* Velocity at a fractional position and forcing weight: ocean current plus leeway and Stokes
 * (Particle.cpp:352-475 host; kernel.cu:206-260 device). The vertical component is a float
 * sum in host semantics and a double blend of two float bilinears in device semantics. */
/* Level used for memory access: valid levels are unchanged; an out-of-range level (reached only
 * by a dead particle when survprob <= -1, or by a NaN position, where the reference reads out of
 * bounds) is clamped into the grid so the oracle and the kernels read the same cells. */
static int mem_level(int kI, int sW) {
    if (kI > 0) return 0;
    if (kI < -sW + 2) return -sW + 2;
    return kI;
}

static int advective_velocity(const interval_state *s, int semantics, const wo_particle *p,
                              int kI, double kF, int jI, double jF, int iI, double iF,
                              double stageAlpha, double elapsed, double physicalTime,
                              double stepDt, float *uu, float *vv, double *ww) {
    const wo_config *cfg = s->cfg;
    const wo_window *win = s->win;
    kI = mem_level(kI, win->sW);
    *uu = bilinear_t4(s, win->u, win->sRho, kI, jI, iI, jF, iF, stageAlpha);
    *vv = bilinear_t4(s, win->v, win->sRho, kI, jI, iI, jF, iF, stageAlpha);
    if (cfg->driftModel == 1 && p->driftObjectType != 0) {
        double coeff[9];
        if (wo_drift_coefficients(p->driftObjectType, coeff) != 0 &&
            semantics == WO_SEMANTICS_HOST)
            return -1;
        double windU = cfg->windU10, windV = cfg->windV10;
        if (semantics == WO_SEMANTICS_HOST) {
            /* environmentAt (Particle.cpp:384-395): float corner sums, then interpolateTime */
            const float *fields[2] = {win->windU10, win->windV10};
            double values[2] = {cfg->windU10, cfg->windV10};
            for (int c = 0; c < 2; c++) {
                const float *f = fields[c];
                if (!f) continue;
                float f1 = (float)(rec3(s, f, s->t0, jI, iI) * (1 - iF) * (1 - jF));
                float f2 = (float)(rec3(s, f, s->t0, jI + 1, iI) * (1 - iF) * jF);
                float f3 = (float)(rec3(s, f, s->t0, jI + 1, iI + 1) * iF * jF);
                float f4 = (float)(rec3(s, f, s->t0, jI, iI + 1) * iF * (1 - jF));
                float n1 = (float)(rec3(s, f, s->t1, jI, iI) * (1 - iF) * (1 - jF));
                float n2 = (float)(rec3(s, f, s->t1, jI + 1, iI) * (1 - iF) * jF);
                float n3 = (float)(rec3(s, f, s->t1, jI + 1, iI + 1) * iF * jF);
                float n4 = (float)(rec3(s, f, s->t1, jI, iI + 1) * iF * (1 - jF));
                double first = f1 + f2 + f3 + f4, next = n1 + n2 + n3 + n4;
                values[c] = (1.0 - stageAlpha) * first + stageAlpha * next;
            }
            windU = values[0];
            windV = values[1];
        } else {
            /* environmentAt (kernel.cu:105-116) */
            const float *fields[2] = {win->windU10, win->windV10};
            double values[2] = {cfg->windU10, cfg->windV10};
            for (int c = 0; c < 2; c++) {
                const float *f = fields[c];
                if (!f) continue;
                float f1 = (float)(rec3(s, f, s->t0, jI, iI) * (1.0 - iF) * (1.0 - jF));
                float f2 = (float)(rec3(s, f, s->t0, jI + 1, iI) * (1.0 - iF) * jF);
                float f3 = (float)(rec3(s, f, s->t0, jI + 1, iI + 1) * iF * jF);
                float f4 = (float)(rec3(s, f, s->t0, jI, iI + 1) * iF * (1.0 - jF));
                float n1 = (float)(rec3(s, f, s->t1, jI, iI) * (1.0 - iF) * (1.0 - jF));
                float n2 = (float)(rec3(s, f, s->t1, jI + 1, iI) * (1.0 - iF) * jF);
                float n3 = (float)(rec3(s, f, s->t1, jI + 1, iI + 1) * iF * jF);
                float n4 = (float)(rec3(s, f, s->t1, jI, iI + 1) * iF * (1.0 - jF));
                values[c] = (1.0 - stageAlpha) * (float)(f1 + f2 + f3 + f4) +
                            stageAlpha * (float)(n1 + n2 + n3 + n4);
            }
            windU = values[0];
            windV = values[1];
        }
        uint64_t substep = (uint64_t)floor(elapsed / cfg->dti);
        double longitude = bilinear_d(s, win->lonRad, jI, iI, jF, iF);
        double latitude = bilinear_d(s, win->latRad, jI, iI, jF, iF);
        double stdDev = cfg->windErrorStdDev, corr = cfg->windErrorComponentCorrelation;
        double spatial = cfg->windErrorSpatialScale, temporal = cfg->windErrorTemporalScale;
        int region = wo_calibration_region(cfg->observationalCalibrationRegions,
                                           cfg->observationalCalibrationRegionCount, longitude,
                                           latitude);
        if (region >= 0) {
            const wo_region *r = &cfg->observationalCalibrationRegions[region];
            stdDev = r->windErrorStdDev;
            corr = r->windErrorComponentCorrelation;
            spatial = r->windErrorSpatialScale;
            temporal = r->windErrorTemporalScale;
        }
        if (stdDev > 0) {
            double when = physicalTime + .5 * s->direction * stepDt;
            double first = wo_forcing_error_normal(cfg->randomSeed, p->id, s->intervalKey, substep,
                                                   WO_WIND_U_COMPONENT, longitude, latitude, when,
                                                   spatial, temporal);
            double second = wo_forcing_error_normal(cfg->randomSeed, p->id, s->intervalKey,
                                                    substep, WO_WIND_V_COMPONENT, longitude,
                                                    latitude, when, spatial, temporal);
            windU += stdDev * first;
            windV += stdDev * wo_correlated_normal(first, second, corr);
        }
        double downwindNormal = 0, crosswindNormal = 0;
        if (cfg->leewayCoefficientEnsemble) {
            downwindNormal = wo_normal(cfg->randomSeed, p->id, WO_ENSEMBLE_INTERVAL, 0, 0);
            crosswindNormal = wo_normal(cfg->randomSeed, p->id, WO_ENSEMBLE_INTERVAL, 0, 1);
            crosswindNormal = wo_correlated_normal(downwindNormal, crosswindNormal,
                                                   cfg->leewayResidualCorrelation);
        }
        double leeway[2];
        wo_compute_leeway(coeff, windU, windV, p->driftSide, downwindNormal, crosswindNormal,
                          leeway);
        *uu += (float)leeway[0];
        *vv += (float)leeway[1];
        if (win->stokesU && win->stokesV) {
            /* waveAt (Particle.cpp:446-453, kernel.cu:118-129): double corner sums */
            const float *fields[2] = {win->stokesU, win->stokesV};
            float *out[2] = {uu, vv};
            for (int c = 0; c < 2; c++) {
                const float *f = fields[c];
                double first = rec3(s, f, s->t0, jI, iI) * (1.0 - iF) * (1.0 - jF) +
                               rec3(s, f, s->t0, jI + 1, iI) * (1.0 - iF) * jF +
                               rec3(s, f, s->t0, jI + 1, iI + 1) * iF * jF +
                               rec3(s, f, s->t0, jI, iI + 1) * iF * (1.0 - jF);
                double next = rec3(s, f, s->t1, jI, iI) * (1.0 - iF) * (1.0 - jF) +
                              rec3(s, f, s->t1, jI + 1, iI) * (1.0 - iF) * jF +
                              rec3(s, f, s->t1, jI + 1, iI + 1) * iF * jF +
                              rec3(s, f, s->t1, jI, iI + 1) * iF * (1.0 - jF);
                *out[c] += (float)((1.0 - stageAlpha) * first + stageAlpha * next);
            }
        }
    }
    if (semantics == WO_SEMANTICS_HOST) {
        *ww = trilinear_f(s, win->w, win->sW, kI, kF, jI, iI, jF, iF, stageAlpha);
    } else {
        *ww = (double)bilinear_t4(s, win->w, win->sW, kI, jI, iI, jF, iF, stageAlpha) * (1.0 - kF) +
              (double)bilinear_t4(s, win->w, win->sW, kI - 1, jI, iI, jF, iF, stageAlpha) * kF;
    }
    return 0;
}

static double zeta_h_mid_host(const interval_state *s, int jMI, int iMI, double jMF, double iMF,
                              double alpha) {
    /* hcMid (Particle.cpp:601-604): one double chain of 4 h and 4 zeta terms */
    const double *h = s->win->h;
    const float *z = s->win->zeta;
    return h[idx2(s, jMI, iMI)] * (1.0 - iMF) * (1.0 - jMF) +
           h[idx2(s, jMI + 1, iMI)] * (1.0 - iMF) * jMF +
           h[idx2(s, jMI + 1, iMI + 1)] * iMF * jMF + h[idx2(s, jMI, iMI + 1)] * iMF * (1.0 - jMF) +
           at3(s, z, jMI, iMI, alpha) * (1.0 - iMF) * (1.0 - jMF) +
           at3(s, z, jMI + 1, iMI, alpha) * (1.0 - iMF) * jMF +
           at3(s, z, jMI + 1, iMI + 1, alpha) * iMF * jMF +
           at3(s, z, jMI, iMI + 1, alpha) * iMF * (1.0 - jMF);
}

static void vertical_closure_upper(const wo_config *cfg, double *k, double *health) {
    if (cfg->upperClosure == WO_CLOSURE_CONSTRAINT) *k = 0;
    else if (cfg->upperClosure == WO_CLOSURE_KILL) *health = -1;
    else if (cfg->upperClosure == WO_CLOSURE_REFLECTION) *k = -*k;
}

static void vertical_closure_lower(const wo_config *cfg, double kLower, double *k,
                                   double *health) {
    if (cfg->lowerClosure == WO_CLOSURE_CONSTRAINT) *k = kLower;
    else if (cfg->lowerClosure == WO_CLOSURE_KILL) *health = -1;
    else if (cfg->lowerClosure == WO_CLOSURE_REFLECTION) *k = 2.0 * kLower - *k;
}

/* One particle over one interval. Host semantics: Particle.cpp:71-824; device semantics:
 * kernel.cu:153-368. Differences between the two are marked where they occur. */
static int move_one(const interval_state *base, int semantics, wo_particle *particle) {
    const wo_config *cfg = base->cfg;
    const wo_window *win = base->win;
    interval_state sv = *base;
    const interval_state *s = &sv;
    wo_particle p = *particle;
    int direction = s->direction;
    double length = s->length, elapsed = 0;

    if (!isnan(cfg->restartCheckpoint)) {
        if (semantics == WO_SEMANTICS_HOST) {
            elapsed = wo_restart_elapsed(s->start, s->end, cfg->restartCheckpoint);
            if (isnan(elapsed)) return 0;
        } else {
            if ((direction > 0 && s->end <= cfg->restartCheckpoint) ||
                (direction < 0 && s->end >= cfg->restartCheckpoint))
                return 0;
            elapsed = fmin(length, fmax(0.0, direction * (cfg->restartCheckpoint - s->start)));
        }
    }
    int sW = win->sW, eta = win->eta, xi = win->xi;
    double kLower = (double)(-sW + 2);
    if (p.k > 0) vertical_closure_upper(cfg, &p.k, &p.health);
    if (p.k < kLower) vertical_closure_lower(cfg, kLower, &p.k, &p.health);

    int midpoint = cfg->integrator == WO_MIDPOINT;
    double dir = (double)direction;
    while (elapsed < length) {
        double stepDt = semantics == WO_SEMANTICS_HOST ? dmin(cfg->dti, length - elapsed)
                                                        : fmin(cfg->dti, length - elapsed);
        double physicalTime = s->start + direction * elapsed;
        double alpha = length == 0 ? 0 : (elapsed + 0.5 * stepDt) / length;
        double alphaStart = length == 0 ? 0 : elapsed / length;
        if (direction > 0 && p.time > physicalTime) {
            elapsed = semantics == WO_SEMANTICS_HOST ? dmin(length, p.time - s->start)
                                                      : fmin(length, p.time - s->start);
            continue;
        }
        if (p.health < cfg->survprob) {
            p.health = -1;
            break;
        }
        double kc = ceil(p.k);
        int kI = to_int(kc), jI = to_int(floor(p.j)), iI = to_int(floor(p.i));
        double kF = kc - p.k, jF = p.j - jI, iF = p.i - iI;
        if (!valid_cell(jI, iI, eta, xi)) {
            p.health = -1;
            break;
        }
        if (semantics == WO_SEMANTICS_DEVICE && (kI > 0 || kI <= -sW + 1)) {
            p.health = -1; /* device-only level check (kernel.cu:195) */
            break;
        }
        float zz = bilinear_t(s, win->zeta, jI, iI, jF, iF, alpha);
        double hc = bilinear_d(s, win->h, jI, iI, jF, iF) + zz;
        if (hc <= cfg->shoreLimit && cfg->horizontalClosure == WO_CLOSURE_KILL) {
            p.health = -1;
            if (semantics == WO_SEMANTICS_DEVICE) break; /* the host path finishes the step */
        }

        float uu, vv;
        double ww;
        if (advective_velocity(s, semantics, &p, kI, kF, jI, jF, iI, iF,
                               midpoint ? alphaStart : alpha, elapsed, physicalTime, stepDt, &uu,
                               &vv, &ww) != 0)
            return -1;
        double aa;
        int kA = mem_level(kI, sW);
        if (semantics == WO_SEMANTICS_HOST)
            aa = trilinear_f(s, win->akt, sW, kA, kF, jI, iI, jF, iF, alpha);
        else
            aa = (double)bilinear_t4(s, win->akt, sW, kA, jI, iI, jF, iF, alpha) * (1.0 - kF) +
                 (double)bilinear_t4(s, win->akt, sW, kA - 1, jI, iI, jF, iF, alpha) * kF;

        double dxleap = dir * uu * stepDt, dyleap = dir * vv * stepDt;
        double dzleap = dir * (cfg->sv + ww) * stepDt;
        double rx = 0, ry = 0, rz = 0;
        if (cfg->random && (dir > 0 || cfg->backwardDiffusion)) {
            double sigmaDepth = cfg->sigma * (1 - p.k / kLower);
            uint64_t substep = (uint64_t)floor(elapsed / cfg->dti);
            double scale = sqrt(stepDt / cfg->dti);
            uint64_t seed = cfg->randomSeed;
            rx = sigmaDepth * wo_normal(seed, p.id, s->intervalKey, substep, 0) * scale;
            ry = sigmaDepth * wo_normal(seed, p.id, s->intervalKey, substep, 1) * scale;
            rz = sigmaDepth * wo_normal(seed, p.id, s->intervalKey, substep, 2) * aa * cfg->crid * scale;
        }
        double xleap = dxleap + rx, yleap = dyleap + ry, zleap = dzleap + rz;

        double xdist, ydist;
        cell_metric(s, semantics, jI, iI, &xdist, &ydist);
        double zdist = hc * depth_interval(s, kI);

        if (midpoint) {
            double kHalf = dir * (cfg->sv + ww) * 0.5 * stepDt;
            if (fabs(kHalf) > zdist) kHalf = sign_of(zdist, kHalf);
            double iMid = p.i + dir * uu * 0.5 * stepDt / xdist;
            double jMid = p.j + dir * vv * 0.5 * stepDt / ydist;
            double kMid = semantics == WO_SEMANTICS_HOST
                              ? dmin(0.0, dmax(kLower, p.k + kHalf / zdist))
                              : fmin(0.0, fmax(kLower, p.k + kHalf / zdist));
            int iMI = to_int(floor(iMid)), jMI = to_int(floor(jMid));
            int midValid = valid_cell(jMI, iMI, eta, xi);
            double hcMid = 0;
            double iMF = 0, jMF = 0;
            if (midValid) {
                iMF = iMid - iMI;
                jMF = jMid - jMI;
                if (semantics == WO_SEMANTICS_HOST)
                    hcMid = zeta_h_mid_host(s, jMI, iMI, jMF, iMF, alpha);
                else
                    hcMid = bilinear_d(s, win->h, jMI, iMI, jMF, iMF) +
                            bilinear_t(s, win->zeta, jMI, iMI, jMF, iMF, alpha);
                midValid = hcMid > cfg->shoreLimit && hcMid > 0;
            }
            double detX, detY, detZ;
            if (midValid) {
                double kmc = ceil(kMid);
                int kMI = to_int(kmc);
                double kMF = kmc - kMid;
                float um, vm;
                double wm;
                if (advective_velocity(s, semantics, &p, kMI, kMF, jMI, jMF, iMI, iMF, alpha,
                                       elapsed, physicalTime, stepDt, &um, &vm, &wm) != 0)
                    return -1;
                double xdistMid, ydistMid;
                cell_metric(s, semantics, jMI, iMI, &xdistMid, &ydistMid);
                double zdistMid = hcMid * depth_interval(s, kMI);
                detX = dir * um * stepDt * xdist / xdistMid;
                detY = dir * vm * stepDt * ydist / ydistMid;
                detZ = dir * (cfg->sv + wm) * stepDt * zdist / zdistMid;
            } else {
                float ue, ve;
                double we;
                if (advective_velocity(s, semantics, &p, kI, kF, jI, jF, iI, iF, alpha, elapsed,
                                       physicalTime, stepDt, &ue, &ve, &we) != 0)
                    return -1;
                detX = dir * ue * stepDt;
                detY = dir * ve * stepDt;
                detZ = dir * (cfg->sv + we) * stepDt;
            }
            if (semantics == WO_SEMANTICS_HOST) {
                xleap = detX + rx;
                yleap = detY + ry;
                zleap = detZ + rz;
            } else {
                /* kernel.cu:314-316 replaces the Euler part inside the accumulated leap */
                xleap += detX - dir * uu * stepDt;
                yleap += detY - dir * vv * stepDt;
                zleap += detZ - dir * (cfg->sv + ww) * stepDt;
            }
        }

        if (fabs(zleap) > zdist) zleap = sign_of(zdist, zleap);
        double jdet = p.j + yleap / ydist;
        double idet = p.i + xleap / xdist;
        double kdet = p.k + zleap / zdist;
        if (kdet > 0.) vertical_closure_upper(cfg, &kdet, &p.health);
        if (kdet < kLower) vertical_closure_lower(cfg, kLower, &kdet, &p.health);

        int jdetI = to_int(floor(jdet)), idetI = to_int(floor(idet));
        if (valid_cell(jdetI, idetI, eta, xi)) {
            double idetF = idet - idetI, jdetF = jdet - jdetI;
            float zzdet = bilinear_t(s, win->zeta, jdetI, idetI, jdetF, idetF, alpha);
            double hcdet = bilinear_d(s, win->h, jdetI, idetI, jdetF, idetF) + zzdet;
            if (hcdet <= cfg->shoreLimit) {
                if (cfg->horizontalClosure == WO_CLOSURE_CONSTRAINT) {
                    idet = p.i;
                    jdet = p.j;
                } else if (cfg->horizontalClosure == WO_CLOSURE_KILL) {
                    p.health = -1;
                } else if (cfg->horizontalClosure == WO_CLOSURE_REFLECTION) {
                    idet = wo_reflect_cell(p.i, iI, idet, idetI);
                    jdet = wo_reflect_cell(p.j, jI, jdet, jdetI);
                }
            }
            p.i = idet;
            p.j = jdet;
            p.k = kdet;
        } else {
            if (cfg->horizontalClosure == WO_CLOSURE_CONSTRAINT) {
                p.k = kdet;
            } else if (cfg->horizontalClosure == WO_CLOSURE_KILL) {
                p.health = -1;
            } else if (cfg->horizontalClosure == WO_CLOSURE_REFLECTION) {
                p.i = wo_reflect_domain(idet, xi - 1);
                p.j = wo_reflect_domain(jdet, eta - 1);
                p.k = kdet;
            }
        }

        if (p.health > 0) {
            p.age = p.age + stepDt;
            p.health = exp(-p.age / cfg->tau0);
            if (cfg->leewayJibeProbabilityHourly > 0 && p.driftObjectType != 0) {
                uint64_t substep = (uint64_t)floor(elapsed / cfg->dti);
                double probability = wo_jibe_step_probability(cfg->leewayJibeProbabilityHourly, stepDt);
                if (wo_uniform(cfg->randomSeed, p.id, s->intervalKey, substep, WO_JIBE_COMPONENT) <
                    probability)
                    p.driftSide = (int8_t)-p.driftSide;
            }
        }
        elapsed += stepDt;
    }
    *particle = p;
    return 0;
}

int wo_move_batch(const wo_config *config, wo_particle *particles, long n,
                  const wo_window *window, int timeIndex, int semantics, int threads) {
    interval_state s;
    memset(&s, 0, sizeof(s));
    s.cfg = config;
    s.win = window;
    s.direction = config->trackingDirection;
    s.t0 = timeIndex;
    int next = timeIndex + s.direction;
    s.start = window->times[timeIndex];
    s.end = (next >= 0 && next < window->T) ? window->times[next]
                                            : s.start + s.direction * config->deltat;
    s.length = fabs(s.end - s.start);
    s.t1 = (next >= 0 && next < window->T) ? next : timeIndex;
    s.intervalKey = (int64_t)llround(s.start < s.end ? s.start : s.end);
    s.plane = (size_t)window->eta * (size_t)window->xi;
    int status = 0;
#ifdef _OPENMP
    int team = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(team)
#else
    (void)threads;
#endif
    for (long idx = 0; idx < n; idx++) {
        if (move_one(&s, semantics, &particles[idx]) != 0) {
#pragma omp atomic write
            status = -1;
        }
    }
    return status;
}

/* ---------------------------------------------------------------- concentration */

void wo_concentration(const wo_particle *particles, long n, int concTimeIdx, int Tc, int sRho,
                      int eta, int xi, uint32_t *conc) {
    (void)Tc;
    size_t plane = (size_t)eta * (size_t)xi;
    for (long idx = 0; idx < n; idx++) {
        const wo_particle *p = &particles[idx];
        if (!(p->health > 0)) continue;
        double rk = round(p->k), rj = round(p->j), ri = round(p->i);
        if (!(rk > -2147483648.0 && rk < 2147483648.0 && rj > -2147483648.0 &&
              rj < 2147483648.0 && ri > -2147483648.0 && ri < 2147483648.0))
            continue;
        int k = (int)rk, j = (int)rj, i = (int)ri;
        if (j >= 0 && j < eta && i >= 0 && i < xi && k >= -sRho + 1 && k <= 0)
            conc[((size_t)concTimeIdx * sRho + (size_t)(k + sRho - 1)) * plane + (size_t)j * xi + i] += 1;
    }
}

/* The solver's float concentration output: the land cells of the particle grid (mask != 1,
 * Wacomm.cpp:188-196) get 1e37 in every level of the concentration time just evaluated
 * (Wacomm.cpp:724-737); counts elsewhere are the float grid Concentration::evaluate filled. */
void wo_concentration_mask(float *conc, int concTimeIdx, int sRho, int eta, int xi,
                           const double *mask) {
    size_t plane = (size_t)eta * (size_t)xi;
    for (int k = -sRho + 1; k <= 0; k++)
        for (int j = 0; j < eta; j++)
            for (int i = 0; i < xi; i++)
                if (mask[(size_t)j * xi + i] != 1)
                    conc[((size_t)concTimeIdx * sRho + (size_t)(k + sRho - 1)) * plane +
                         (size_t)j * xi + i] = 1e37f;
}

/* ---------------------------------------------------------------- emission schedule */

long wo_source_emission_times(int mode, double value, double sourceStart, double sourceEnd,
                              double intervalStart, double intervalEnd, double *out, long cap) {
    long count = 0;
    if (!isfinite(value) || value < 0 || !isfinite(sourceStart) || !isfinite(intervalStart) ||
        !isfinite(intervalEnd) || intervalEnd <= intervalStart)
        return -1;
    if (value == 0) return 0;
    if (mode == 2) { /* single_pulse */
        if (floor(value) != value) return -1;
        if (sourceStart >= intervalStart && sourceStart < intervalEnd) {
            for (long n = 0; n < (long)value; n++, count++)
                if (count < cap) out[count] = sourceStart;
        }
        return count;
    }
    if (mode == 1) { /* forcing_interval_batch */
        if (floor(value) != value) return -1;
        long long record = llround(intervalStart);
        if (record >= llround(sourceStart) && (sourceEnd < 0 || record <= llround(sourceEnd))) {
            for (long n = 0; n < (long)value; n++, count++)
                if (count < cap) out[count] = intervalStart;
        }
        return count;
    }
    double activeStart = dmax(intervalStart, sourceStart);
    double activeEnd = sourceEnd < 0 ? intervalEnd : dmin(intervalEnd, sourceEnd);
    if (activeEnd <= activeStart) return 0;
    double spacing = 3600.0 / value;
    long long first = (long long)ceil((activeStart - sourceStart) / spacing - 0.5);
    if (first < 0) first = 0;
    for (long long index = first;; index++) {
        double time = sourceStart + (index + 0.5) * spacing;
        if (time >= activeEnd) break;
        if (time >= activeStart) {
            if (count < cap) out[count] = time;
            count++;
        }
    }
    return count;
}

/* SourceEmission.hpp:20-23. */
double wo_source_position_offset(uint64_t seed, uint64_t particle, uint64_t component) {
    return 0.25 * wo_normal(seed, particle, WO_SOURCE_INTERVAL, 0, component);
}

/* Sources::emit (Sources.cpp:233-249): (time, source) pairs in source-major order, stably sorted
 * by time; each becomes a record through Source::emit (Source.cpp:25-45). */
typedef struct wo_release {
    double time;
    long order; /* position in the source-major list: the stable tie-break */
    int source;
} wo_release;

static int release_cmp(const void *a, const void *b) {
    const wo_release *x = (const wo_release *)a, *y = (const wo_release *)b;
    if (x->time < y->time) return -1;
    if (y->time < x->time) return 1;
    return (x->order > y->order) - (x->order < y->order);
}

long wo_sources_emit(const wo_config *config, const wo_source *sources, int n_sources,
                     double julian_start, double interval_start, double interval_end,
                     uint64_t first_id, wo_particle *out, long cap) {
    long total = 0;
    for (int s = 0; s < n_sources; s++) {
        const wo_source *src = &sources[s];
        if (src->mode != 1) continue; /* Source.cpp:18 */
        double start = src->start < 0 ? julian_start * 86400.0 : src->start * 86400.0;
        double end = src->end < 0 ? -1 : src->end * 86400.0;
        long c = wo_source_emission_times(src->emission_mode, src->emission_value, start, end,
                                          interval_start, interval_end, NULL, 0);
        if (c < 0) return -1;
        total += c;
    }
    wo_release *list = (wo_release *)malloc((size_t)(total > 0 ? total : 1) * sizeof(wo_release));
    double *times = NULL;
    long at = 0;
    for (int s = 0; s < n_sources; s++) {
        const wo_source *src = &sources[s];
        if (src->mode != 1) continue;
        double start = src->start < 0 ? julian_start * 86400.0 : src->start * 86400.0;
        double end = src->end < 0 ? -1 : src->end * 86400.0;
        long c = wo_source_emission_times(src->emission_mode, src->emission_value, start, end,
                                          interval_start, interval_end, NULL, 0);
        times = (double *)realloc(times, (size_t)(c > 0 ? c : 1) * sizeof(double));
        wo_source_emission_times(src->emission_mode, src->emission_value, start, end,
                                 interval_start, interval_end, times, c);
        for (long n = 0; n < c; n++, at++) {
            list[at].time = times[n];
            list[at].order = at;
            list[at].source = s;
        }
    }
    free(times);
    qsort(list, (size_t)total, sizeof(wo_release), release_cmp);
    for (long r = 0; r < total && r < cap; r++) {
        const wo_source *src = &sources[list[r].source];
        uint64_t id = first_id + (uint64_t)r;
        wo_particle p;
        memset(&p, 0, sizeof p);
        p.id = id;
        p.k = src->k;
        p.j = src->j;
        p.i = src->i;
        if (config->randomSources) {
            p.k = src->k + wo_source_position_offset(config->randomSeed, id, 0);
            p.j = src->j + wo_source_position_offset(config->randomSeed, id, 1);
            p.i = src->i + wo_source_position_offset(config->randomSeed, id, 2);
        }
        p.health = 1.0; /* Particle.cpp:30-44 */
        p.age = 0.0;
        p.time = list[r].time;
        p.driftObjectType = config->driftObjectType;
        p.driftSide = config->driftSide;
        if (config->leewayRandomSide)
            p.driftSide = (int8_t)wo_sample_drift_side(config->randomSeed, id,
                                                       config->leewayRightSideProbability);
        out[r] = p;
    }
    free(list);
    return total;
}

/* ---------------------------------------------------------------- kji <-> geo */

int wo_kji2deplatlon(int eta, int xi, int sW, const double *lon, const double *lat,
                     const double *h, const double *sWValues, double k, double j, double i,
                     double *dep, double *latOut, double *lonOut) {
    double kc = ceil(k);
    int kI = to_int(kc), jI = to_int(floor(j)), iI = to_int(floor(i));
    double kF = kc - k, jF = j - jI, iF = i - iI;
    if (!valid_cell(jI, iI, eta, xi) || kI > 0 || kI <= -sW + 1) {
        *lonOut = 1e37;
        *latOut = 1e37;
        *dep = 1e37;
        return -1;
    }
#define AT(f, jj, ii) (f)[(size_t)(jj) * (size_t)xi + (size_t)(ii)]
    double lon1 = AT(lon, jI, iI) * (1.0 - iF) * (1.0 - jF);
    double lon2 = AT(lon, jI + 1, iI) * (1.0 - iF) * jF;
    double lon3 = AT(lon, jI + 1, iI + 1) * iF * jF;
    double lon4 = AT(lon, jI, iI + 1) * iF * (1.0 - jF);
    *lonOut = lon1 + lon2 + lon3 + lon4;
    double lat1 = AT(lat, jI, iI) * (1.0 - iF) * (1.0 - jF);
    double lat2 = AT(lat, jI + 1, iI) * (1.0 - iF) * jF;
    double lat3 = AT(lat, jI + 1, iI + 1) * iF * jF;
    double lat4 = AT(lat, jI, iI + 1) * iF * (1.0 - jF);
    *latOut = lat1 + lat2 + lat3 + lat4;
    double h1 = AT(h, jI, iI) * (1.0 - iF) * (1.0 - jF);
    double h2 = AT(h, jI + 1, iI) * (1.0 - iF) * jF;
    double h3 = AT(h, jI + 1, iI + 1) * iF * jF;
    double h4 = AT(h, jI, iI + 1) * iF * (1.0 - jF);
    double hh = h1 + h2 + h3 + h4;
    double sUp = sWValues[kI + sW - 1], sLo = sWValues[kI - 1 + sW - 1];
    double aDep = fabs(fabs(hh * sLo) - fabs(hh * sUp));
    *dep = -(hh * fabs(sUp) + fabs(kF * aDep));
    return 0;
}

int wo_deplatlon2kji(int eta, int xi, int sW, const double *lon, const double *lat,
                     const double *h, const double *sWValues, double dep, double latIn,
                     double lonIn, double *kOut, double *jOut, double *iOut) {
    if (!isfinite(latIn) || !isfinite(lonIn)) return -1;
    const double tol = 1e-9;
    int found = 0;
    double jPos = 0, iPos = 0;
    for (int jC = 0; jC + 1 < eta && !found; jC++) {
        for (int iC = 0; iC + 1 < xi && !found; iC++) {
            double lon00 = AT(lon, jC, iC), lon10 = AT(lon, jC + 1, iC);
            double lon11 = AT(lon, jC + 1, iC + 1), lon01 = AT(lon, jC, iC + 1);
            double lat00 = AT(lat, jC, iC), lat10 = AT(lat, jC + 1, iC);
            double lat11 = AT(lat, jC + 1, iC + 1), lat01 = AT(lat, jC, iC + 1);
            double lonMin = dmin(dmin(lon00, lon10), dmin(lon11, lon01));
            double lonMax = dmax(dmax(lon00, lon10), dmax(lon11, lon01));
            double latMin = dmin(dmin(lat00, lat10), dmin(lat11, lat01));
            double latMax = dmax(dmax(lat00, lat10), dmax(lat11, lat01));
            double lonPad = tol * (lonMax - lonMin), latPad = tol * (latMax - latMin);
            if (lonIn < lonMin - lonPad || lonIn > lonMax + lonPad || latIn < latMin - latPad ||
                latIn > latMax + latPad)
                continue;
            double iF = 0.5, jF = 0.5;
            int converged = 0;
            for (int it = 0; it < 50; it++) {
                double rLon = lon00 * (1.0 - iF) * (1.0 - jF) + lon10 * (1.0 - iF) * jF +
                              lon11 * iF * jF + lon01 * iF * (1.0 - jF) - lonIn;
                double rLat = lat00 * (1.0 - iF) * (1.0 - jF) + lat10 * (1.0 - iF) * jF +
                              lat11 * iF * jF + lat01 * iF * (1.0 - jF) - latIn;
                double dLonDi = (lon01 - lon00) * (1.0 - jF) + (lon11 - lon10) * jF;
                double dLonDj = (lon10 - lon00) * (1.0 - iF) + (lon11 - lon01) * iF;
                double dLatDi = (lat01 - lat00) * (1.0 - jF) + (lat11 - lat10) * jF;
                double dLatDj = (lat10 - lat00) * (1.0 - iF) + (lat11 - lat01) * iF;
                double det = dLonDi * dLatDj - dLonDj * dLatDi;
                if (!isfinite(det) || det == 0) break;
                double stepI = (dLatDj * rLon - dLonDj * rLat) / det;
                double stepJ = (-dLatDi * rLon + dLonDi * rLat) / det;
                iF -= stepI;
                jF -= stepJ;
                if (!isfinite(iF) || !isfinite(jF)) break;
                if (fabs(stepI) < 1e-11 && fabs(stepJ) < 1e-11) {
                    converged = 1;
                    break;
                }
            }
            if (!converged || iF < -tol || iF > 1.0 + tol || jF < -tol || jF > 1.0 + tol) continue;
            if (fabs(iF) <= tol) iF = 0.0;
            else if (fabs(iF - 1.0) <= tol) iF = 1.0;
            if (fabs(jF) <= tol) jF = 0.0;
            else if (fabs(jF - 1.0) <= tol) jF = 1.0;
            if (!valid_cell(to_int(floor(jC + jF)), to_int(floor(iC + iF)), eta, xi)) continue;
            jPos = jC + jF;
            iPos = iC + iF;
            found = 1;
        }
    }
    if (!found) return -1;
    *jOut = jPos;
    *iOut = iPos;
    int jI = to_int(floor(jPos)), iI = to_int(floor(iPos));
    double jF = jPos - jI, iF = iPos - iI;
    dep = fabs(dep);
    double h1 = AT(h, jI, iI) * (1.0 - iF) * (1.0 - jF);
    double h2 = AT(h, jI + 1, iI) * (1.0 - iF) * jF;
    double h3 = AT(h, jI + 1, iI + 1) * iF * jF;
    double h4 = AT(h, jI, iI + 1) * iF * (1.0 - jF);
    double hh = h1 + h2 + h3 + h4;
    if (!isfinite(dep) || !isfinite(hh)) return -1;
    int kBottom = -sW + 2;
#define SW(k) sWValues[(k) + sW - 1]
    if (dep <= hh * fabs(SW(0))) {
        *kOut = 0;
    } else if (dep >= hh * fabs(SW(kBottom))) {
        *kOut = kBottom;
    } else {
        int kI = 0;
        while (kI - 1 > kBottom && dep >= hh * fabs(SW(kI - 1))) kI--;
        double upper = hh * fabs(SW(kI));
        double aDep = fabs(hh * fabs(SW(kI - 1)) - upper);
        double kF = (dep - upper) / aDep;
        *kOut = kI - kF;
    }
#undef SW
#undef AT
    return 0;
}

/* ------------------------------------------------------------------------------------------
 * Environmental regridding (EnvironmentalRegridder.cpp)
 * ------------------------------------------------------------------------------------------ */

/* nearLongitude / longitudeBranch (EnvironmentalRegridder.cpp:37-48) */
static double rg_near(double value, double reference) {
    while (value - reference > 180) value -= 360;
    while (value - reference < -180) value += 360;
    return value;
}

/* bilinear (EnvironmentalRegridder.cpp:50-52) */
static double rg_bilinear(double f00, double f10, double f01, double f11, double x, double y) {
    return (1 - x) * (1 - y) * f00 + x * (1 - y) * f10 + (1 - x) * y * f01 + x * y * f11;
}

/* bracket (EnvironmentalRegridder.cpp:14-28): the first interval of a strictly monotonic axis
 * that holds value within 1e-10. */
static int rg_bracket(const double *axis, int n, double value, int *lower, double *weight) {
    int increasing = axis[n - 1] > axis[0];
    for (int i = 1; i < n; i++)
        if ((increasing && axis[i] <= axis[i - 1]) || (!increasing && axis[i] >= axis[i - 1]))
            return WO_REGRID_GRID;
    double minimum = increasing ? axis[0] : axis[n - 1];
    double maximum = increasing ? axis[n - 1] : axis[0];
    if (value < minimum - 1.e-10 || value > maximum + 1.e-10) return WO_REGRID_OUTSIDE;
    for (int i = 0; i + 1 < n; i++) {
        if ((increasing && value >= axis[i] - 1.e-10 && value <= axis[i + 1] + 1.e-10) ||
            (!increasing && value <= axis[i] + 1.e-10 && value >= axis[i + 1] - 1.e-10)) {
            *lower = i;
            *weight = (value - axis[i]) / (axis[i + 1] - axis[i]);
            return 0;
        }
    }
    return WO_REGRID_OUTSIDE;
}

/* std::max(0.0, std::min(1.0, v)), signed zeros included */
static double rg_unit(double v) {
    double m = v < 1.0 ? v : 1.0;
    return 0.0 < m ? m : 0.0;
}

static int rg_fields_finite(int T, long plane, const float *src) {
    for (long n = 0; n < (long)T * plane; n++)
        if (!isfinite(src[n])) return WO_REGRID_FIELD;
    return 0;
}

int wo_regrid_geographic(int eta, int xi, const double *lon, const double *lat, int T,
                         const float *src, long nTarget, const double *tLon, const double *tLat,
                         float *out) {
    if (eta < 2 || xi < 2) return WO_REGRID_GRID;
    double *axisX = malloc(sizeof(double) * (size_t)xi);
    double *axisY = malloc(sizeof(double) * (size_t)eta);
    int rc = 0;
    for (int i = 0; i < xi; i++) axisX[i] = lon[i];
    for (int j = 0; j < eta; j++) axisY[j] = lat[(size_t)j * xi];
    for (int j = 0; j < eta && !rc; j++)
        for (int i = 0; i < xi && !rc; i++) {
            double x = lon[(size_t)j * xi + i], y = lat[(size_t)j * xi + i];
            if (!isfinite(x) || !isfinite(y) || fabs(x - axisX[i]) > 1.e-10 ||
                fabs(y - axisY[j]) > 1.e-10)
                rc = WO_REGRID_GRID;
        }
    /* unwrapLongitude (EnvironmentalRegridder.cpp:30-35) */
    for (int i = 1; i < xi && !rc; i++) {
        while (axisX[i] - axisX[i - 1] > 180) axisX[i] -= 360;
        while (axisX[i] - axisX[i - 1] < -180) axisX[i] += 360;
    }
    if (!rc && fabs(axisX[xi - 1] - axisX[0]) > 360 + 1.e-10) rc = WO_REGRID_GRID;
    const long plane = (long)eta * xi;
    if (!rc) rc = rg_fields_finite(T, plane, src);
    double center = .5 * (axisX[0] + axisX[xi - 1]);
    for (long n = 0; n < nTarget && !rc; n++) {
        if (!isfinite(tLon[n]) || !isfinite(tLat[n])) {
            rc = WO_REGRID_TARGET;
            break;
        }
        int xl = 0, yl = 0;
        double wx = 0, wy = 0;
        rc = rg_bracket(axisX, xi, rg_near(tLon[n], center), &xl, &wx);
        if (!rc) rc = rg_bracket(axisY, eta, tLat[n], &yl, &wy);
        if (rc) break;
        for (int t = 0; t < T; t++) {
            const float *s = src + (size_t)t * plane;
            double lower = s[(size_t)yl * xi + xl] * (1 - wx) + s[(size_t)yl * xi + xl + 1] * wx;
            double upper = s[(size_t)(yl + 1) * xi + xl] * (1 - wx) +
                           s[(size_t)(yl + 1) * xi + xl + 1] * wx;
            out[(size_t)t * nTarget + n] = (float)(lower * (1 - wy) + upper * wy);
        }
    }
    free(axisX);
    free(axisY);
    return rc;
}

/* CurvilinearCellIndex (EnvironmentalRegridder.cpp:170-236), cyclic longitude */
typedef struct rg_index {
    long cells;
    double *box;        /* [cells][4] minimumX, maximumX, minimumY, maximumY */
    long *binStart;     /* [bins + 1] */
    long *binCells;
    double minX, maxX, minY, maxY, reference;
    int binsX, binsY;
} rg_index;

static int rg_xbin(const rg_index *ix, double v) {
    if (ix->maxX == ix->minX) return 0;
    int b = (int)((v - ix->minX) / (ix->maxX - ix->minX) * ix->binsX);
    return b < 0 ? 0 : (b > ix->binsX - 1 ? ix->binsX - 1 : b);
}

static int rg_ybin(const rg_index *ix, double v) {
    if (ix->maxY == ix->minY) return 0;
    int b = (int)((v - ix->minY) / (ix->maxY - ix->minY) * ix->binsY);
    return b < 0 ? 0 : (b > ix->binsY - 1 ? ix->binsY - 1 : b);
}

static double rg_min4(double a, double b, double c, double d) {
    double l = b < a ? b : a, r = d < c ? d : c;  /* std::min(std::min(a,b),std::min(c,d)) */
    return r < l ? r : l;
}

static double rg_max4(double a, double b, double c, double d) {
    double l = a < b ? b : a, r = c < d ? d : c;  /* std::max(std::max(a,b),std::max(c,d)) */
    return l < r ? r : l;
}

static int rg_index_build(rg_index *ix, int eta, int xi, const double *lon, const double *lat) {
    memset(ix, 0, sizeof *ix);
    double reference = lon[0];
    if (!isfinite(reference)) return WO_REGRID_GRID;
    ix->cells = (long)(eta - 1) * (xi - 1);
    ix->box = malloc(sizeof(double) * 4 * (size_t)ix->cells);
    for (int j = 0; j + 1 < eta; j++)
        for (int i = 0; i + 1 < xi; i++) {
#define L(jj, ii) lon[(size_t)(jj) * xi + (ii)]
#define A(jj, ii) lat[(size_t)(jj) * xi + (ii)]
            double x00 = L(j, i), x10 = rg_near(L(j, i + 1), x00);
            double x01 = rg_near(L(j + 1, i), x00), x11 = rg_near(L(j + 1, i + 1), x00);
            double y00 = A(j, i), y10 = A(j, i + 1), y01 = A(j + 1, i), y11 = A(j + 1, i + 1);
#undef L
#undef A
            if (!isfinite(x00) || !isfinite(x10) || !isfinite(x01) || !isfinite(x11) ||
                !isfinite(y00) || !isfinite(y10) || !isfinite(y01) || !isfinite(y11))
                return WO_REGRID_GRID;
            double center = .25 * (x00 + x10 + x01 + x11);
            double shift = 360 * round((reference - center) / 360);
            double *b = ix->box + 4 * ((size_t)j * (xi - 1) + i);
            b[0] = rg_min4(x00, x10, x01, x11) + shift;
            b[1] = rg_max4(x00, x10, x01, x11) + shift;
            b[2] = rg_min4(y00, y10, y01, y11);
            b[3] = rg_max4(y00, y10, y01, y11);
        }
    ix->minX = ix->box[0];
    ix->maxX = ix->box[1];
    ix->minY = ix->box[2];
    ix->maxY = ix->box[3];
    for (long c = 0; c < ix->cells; c++) {
        const double *b = ix->box + 4 * c;
        ix->minX = b[0] < ix->minX ? b[0] : ix->minX;  /* std::min(minimumX, cell) */
        ix->maxX = ix->maxX < b[1] ? b[1] : ix->maxX;
        ix->minY = b[2] < ix->minY ? b[2] : ix->minY;
        ix->maxY = ix->maxY < b[3] ? b[3] : ix->maxY;
    }
    double width = ix->maxX - ix->minX, height = ix->maxY - ix->minY;
    width = width < 1.e-12 ? 1.e-12 : width;
    height = height < 1.e-12 ? 1.e-12 : height;
    double scale = sqrt((double)ix->cells);
    int bx = (int)round(scale * sqrt(width / height)), by = (int)round(scale * sqrt(height / width));
    bx = bx < 1 ? 1 : bx;
    by = by < 1 ? 1 : by;
    ix->binsX = bx < ix->cells ? bx : (int)ix->cells;
    ix->binsY = by < ix->cells ? by : (int)ix->cells;
    long bins = (long)ix->binsX * ix->binsY;
    ix->binStart = calloc((size_t)bins + 1, sizeof(long));
    for (int pass = 0; pass < 2; pass++) {
        long *fill = pass ? calloc((size_t)bins, sizeof(long)) : NULL;
        for (long c = 0; c < ix->cells; c++) {
            const double *b = ix->box + 4 * c;
            int i0 = rg_xbin(ix, b[0]), i1 = rg_xbin(ix, b[1]);
            int j0 = rg_ybin(ix, b[2]), j1 = rg_ybin(ix, b[3]);
            for (int jj = j0; jj <= j1; jj++)
                for (int ii = i0; ii <= i1; ii++) {
                    long bin = (long)jj * ix->binsX + ii;
                    if (pass) ix->binCells[ix->binStart[bin] + fill[bin]++] = c;
                    else ix->binStart[bin + 1]++;
                }
        }
        if (!pass) {
            for (long b = 0; b < bins; b++) ix->binStart[b + 1] += ix->binStart[b];
            ix->binCells = malloc(sizeof(long) * ((size_t)ix->binStart[bins] + 1));
        }
        free(fill);
    }
    ix->reference = reference;
    return 0;
}

static void rg_index_free(rg_index *ix) {
    free(ix->box);
    free(ix->binStart);
    free(ix->binCells);
}

int wo_regrid_curvilinear(int eta, int xi, const double *lon, const double *lat, int T,
                          const float *src, long nTarget, const double *tLon, const double *tLat,
                          float *out) {
    if (eta < 2 || xi < 2) return WO_REGRID_GRID;
    const long plane = (long)eta * xi;
    int rc = rg_fields_finite(T, plane, src);
    if (rc) return rc;
    rg_index ix;
    rc = rg_index_build(&ix, eta, xi, lon, lat);
    for (long n = 0; n < nTarget && !rc; n++) {
        double targetX = tLon[n], targetY = tLat[n];
        if (!isfinite(targetX) || !isfinite(targetY)) {
            rc = WO_REGRID_TARGET;
            break;
        }
        /* candidates(): the longitude is moved to the branch of the index reference first */
        targetX = rg_near(targetX, ix.reference);
        long first = 0, last = 0;
        if (!(targetX < ix.minX - 1.e-10 || targetX > ix.maxX + 1.e-10 ||
              targetY < ix.minY - 1.e-10 || targetY > ix.maxY + 1.e-10)) {
            long bin = (long)rg_ybin(&ix, targetY) * ix.binsX + rg_xbin(&ix, targetX);
            first = ix.binStart[bin];
            last = ix.binStart[bin + 1];
        }
        int foundJ = -1, foundI = -1;
        double foundX = 0, foundY = 0;
        for (long c = first; c < last; c++) {
            long cell = ix.binCells[c];
            int j = (int)(cell / (xi - 1)), i = (int)(cell % (xi - 1));
#define L(jj, ii) lon[(size_t)(jj) * xi + (ii)]
#define A(jj, ii) lat[(size_t)(jj) * xi + (ii)]
            double x00 = rg_near(L(j, i), targetX), x10 = rg_near(L(j, i + 1), targetX);
            double x01 = rg_near(L(j + 1, i), targetX), x11 = rg_near(L(j + 1, i + 1), targetX);
            double y00 = A(j, i), y10 = A(j, i + 1), y01 = A(j + 1, i), y11 = A(j + 1, i + 1);
#undef L
#undef A
            if (!isfinite(x00) || !isfinite(x10) || !isfinite(x01) || !isfinite(x11) ||
                !isfinite(y00) || !isfinite(y10) || !isfinite(y01) || !isfinite(y11)) {
                rc = WO_REGRID_GRID;
                break;
            }
            const double *b = ix.box + 4 * cell;
            if (targetX < b[0] - 1.e-10 || targetX > b[1] + 1.e-10 || targetY < b[2] - 1.e-10 ||
                targetY > b[3] + 1.e-10)
                continue;
            double x = .5, y = .5;
            for (int iteration = 0; iteration < 20; iteration++) {
                double mappedX = rg_bilinear(x00, x10, x01, x11, x, y);
                double mappedY = rg_bilinear(y00, y10, y01, y11, x, y);
                double dXdx = (1 - y) * (x10 - x00) + y * (x11 - x01);
                double dXdy = (1 - x) * (x01 - x00) + x * (x11 - x10);
                double dYdx = (1 - y) * (y10 - y00) + y * (y11 - y01);
                double dYdy = (1 - x) * (y01 - y00) + x * (y11 - y10);
                double determinant = dXdx * dYdy - dXdy * dYdx;
                if (fabs(determinant) < 1.e-14) break;
                double residualX = mappedX - targetX, residualY = mappedY - targetY;
                x -= (dYdy * residualX - dXdy * residualY) / determinant;
                y -= (-dYdx * residualX + dXdx * residualY) / determinant;
            }
            double residual = hypot(rg_bilinear(x00, x10, x01, x11, x, y) - targetX,
                                    rg_bilinear(y00, y10, y01, y11, x, y) - targetY);
            if (x >= -1.e-9 && x <= 1 + 1.e-9 && y >= -1.e-9 && y <= 1 + 1.e-9 &&
                residual < 1.e-8) {
                double d00 = (x10 - x00) * (y01 - y00) - (x01 - x00) * (y10 - y00);
                double d10 = (x10 - x00) * (y11 - y10) - (x11 - x10) * (y10 - y00);
                double d01 = (x11 - x01) * (y01 - y00) - (x01 - x00) * (y11 - y01);
                double d11 = (x11 - x01) * (y11 - y10) - (x11 - x10) * (y11 - y01);
                if (fabs(d00) < 1.e-14 || d00 * d10 <= 0 || d00 * d01 <= 0 || d00 * d11 <= 0) {
                    rc = WO_REGRID_FOLDED;
                    break;
                }
                foundJ = j;
                foundI = i;
                foundX = rg_unit(x);
                foundY = rg_unit(y);
                break;
            }
        }
        if (rc) break;
        if (foundJ < 0) {
            rc = WO_REGRID_OUTSIDE;
            break;
        }
        for (int t = 0; t < T; t++) {
            const float *s = src + (size_t)t * plane;
            size_t o = (size_t)foundJ * xi + foundI;
            out[(size_t)t * nTarget + n] =
                (float)rg_bilinear(s[o], s[o + 1], s[o + xi], s[o + xi + 1], foundX, foundY);
        }
    }
    rg_index_free(&ix);
    return rc;
}

int wo_align_times(int nSrc, const double *srcTimes, long plane, const float *src, int nDst,
                   const double *dstTimes, float *out) {
    if (nSrc < 1) return WO_REGRID_TIME;
    for (int s = 1; s < nSrc; s++)
        if (!(srcTimes[s] > srcTimes[s - 1])) return WO_REGRID_TIME;
    for (int d = 0; d < nDst; d++) {
        double t = dstTimes[d];
        int k0 = -1, k1 = -1;
        for (int s = 0; s < nSrc && k0 < 0; s++)
            if (fabs(t - srcTimes[s]) <= 1.e-6) k0 = k1 = s;
        for (int s = 0; s + 1 < nSrc && k0 < 0; s++)
            if (t > srcTimes[s] && t < srcTimes[s + 1]) {
                k0 = s;
                k1 = s + 1;
            }
        if (k0 < 0) return WO_REGRID_TIME;
        /* timeWeight (NumericalHelpers.hpp:30-33) */
        double alpha = 0.0;
        if (k1 != k0) {
            alpha = (t - srcTimes[k0]) / (srcTimes[k1] - srcTimes[k0]);
            alpha = rg_unit(alpha);
        }
        const float *a = src + (size_t)k0 * plane, *b = src + (size_t)k1 * plane;
        float *o = out + (size_t)d * plane;
        for (long n = 0; n < plane; n++)
            o[n] = k1 == k0 ? a[n] : (float)((1.0 - alpha) * a[n] + alpha * b[n]);
    }
    return 0;
}

/* ------------------------------------------------------------------------------------------
 * ROMS record normalization (OceanModelAdapters/ROMSAdapter.cpp)
 * ------------------------------------------------------------------------------------------ */

int wo_roms_normalize(int eta, int xi, int sRho, const double *maskRho, const double *maskU,
                      const double *maskV, const double *angle, const float *zeta, const float *u,
                      const float *v, const float *w, const float *akt, float *zetaOut,
                      float *uOut, float *vOut, float *wOut, float *aktOut) {
    const int xiU = xi - 1, etaV = eta - 1, sW = sRho + 1;
    const size_t plane = (size_t)eta * xi, planeU = (size_t)eta * xiU, planeV = (size_t)etaV * xi;
    /* grid checks (ROMSAdapter.cpp:139-147,148-160) */
    for (size_t n = 0; n < plane; n++) {
        if (maskRho[n] != 0.0 && maskRho[n] != 1.0) return WO_ROMS_MASK;
        if (angle && maskRho[n] > 0.0 && !isfinite(angle[n])) return WO_ROMS_ANGLE;
    }
    for (size_t n = 0; n < planeU; n++) {
        if (maskU[n] != 0.0 && maskU[n] != 1.0) return WO_ROMS_MASK;
        if (maskU[n] > 0.0)
            for (int k = 0; k < sRho; k++)
                if (!isfinite(u[k * planeU + n])) return WO_ROMS_FACE;
    }
    for (size_t n = 0; n < planeV; n++) {
        if (maskV[n] != 0.0 && maskV[n] != 1.0) return WO_ROMS_MASK;
        if (maskV[n] > 0.0)
            for (int k = 0; k < sRho; k++)
                if (!isfinite(v[k * planeV + n])) return WO_ROMS_FACE;
    }
    /* zeta (:254-265) */
    for (size_t n = 0; n < plane; n++)
        zetaOut[n] = (maskRho[n] == 0 || zeta[n] >= 1e+36f) ? 0.0f : zeta[n];
    /* uv2rho (:309-368) */
    for (int k = 0; k < sRho; k++)
        for (int j = 0; j < eta; j++)
            for (int i = 0; i < xi; i++) {
                float usum = 0.0f, vsum = 0.0f;
                int ucount = 0, vcount = 0;
                size_t o = k * plane + (size_t)j * xi + i;
                if (maskRho[(size_t)j * xi + i] > 0.0) {
                    if (i < xiU && maskU[(size_t)j * xiU + i] > 0.0) {
                        usum += u[k * planeU + (size_t)j * xiU + i];
                        ucount++;
                    }
                    if (i > 0 && i - 1 < xiU && maskU[(size_t)j * xiU + i - 1] > 0.0) {
                        usum += u[k * planeU + (size_t)j * xiU + i - 1];
                        ucount++;
                    }
                    if (j < etaV && maskV[(size_t)j * xi + i] > 0.0) {
                        vsum += v[k * planeV + (size_t)j * xi + i];
                        vcount++;
                    }
                    if (j > 0 && j - 1 < etaV && maskV[(size_t)(j - 1) * xi + i] > 0.0) {
                        vsum += v[k * planeV + (size_t)(j - 1) * xi + i];
                        vcount++;
                    }
                    uOut[o] = ucount > 0 ? usum / ucount : 0.0f;
                    vOut[o] = vcount > 0 ? vsum / vcount : 0.0f;
                } else {
                    uOut[o] = 0.0f;
                    vOut[o] = 0.0f;
                }
            }
    /* rotation to east/north (:273-302) */
    int invalid = 0;
    for (int k = 0; k < sRho; k++)
        for (size_t n = 0; n < plane; n++) {
            if (maskRho[n] <= 0.0) continue;
            double c = angle ? cos(angle[n]) : 1.0, s = angle ? sin(angle[n]) : 0.0;
            double gridU = uOut[k * plane + n], gridV = vOut[k * plane + n];
            double east = angle ? gridU * c - gridV * s : gridU;
            double north = angle ? gridU * s + gridV * c : gridV;
            if (!isfinite(east) || !isfinite(north) || fabs(east) > FLT_MAX || fabs(north) > FLT_MAX) {
                invalid = 1;
            } else {
                uOut[k * plane + n] = (float)east;
                vOut[k * plane + n] = (float)north;
            }
        }
    if (invalid) return WO_ROMS_VELOCITY;
    /* wakt2wakt (:431-462) */
    for (int k = 0; k < sW; k++)
        for (size_t n = 0; n < plane; n++) {
            int wet = maskRho[n] > 0.0;
            wOut[k * plane + n] = wet ? w[k * plane + n] : 0.0f;
            aktOut[k * plane + n] = wet ? akt[k * plane + n] : 0.0f;
        }
    return 0;
}

/* Particles::saveAsTxt / writeTxtHeader / writeTxtRecord (Particles.cpp:28-55). */
int wo_text_restart(const char *path, const wo_particle *records, size_t n) {
    FILE *f = fopen(path, "w");
    if (!f) return -1;
    int ok = fprintf(f, "\t%d\n", (int)n) > 0;
    for (size_t r = 0; ok && r < n; r++) {
        const wo_particle *p = records + r;
        ok = fprintf(f, "%llu %.17g %.17g %.17g %.17g %.17g %.17g %d %d\n",
                     (unsigned long long)p->id, p->i, p->j, p->k, p->health, p->age, p->time,
                     (int)p->driftObjectType, (int)p->driftSide) > 0;
    }
    if (fclose(f) != 0) ok = 0;
    return ok ? 0 : -1;
}
