// The FP32 particle step: the same algorithm as step.cuh with FP32 interpolation and metric,
// FP64 kept for the position accumulation, the closures and the interval clock.
//
// Differences from the reference arithmetic (all below the reference's own CPU/GPU snapshot
// tolerance once forcing is FP32, and stated per configuration in the parity tests):
//   * corner weights, time blends and the velocity/diffusivity sums are FP32 with fused
//     multiply-adds;
//   * cell sizes come from a per-cell table of reciprocals, so index increments are products
//     (u dt / dx) instead of double divisions, and the midpoint stage is written directly in
//     index units (u* dt / dx*, algebraically the reference's s u* dt dx/dx* / dx);
//   * the time weight uses a multiply by 1/length.
// Host and device rules keep their differences in closures, level checks and metric formula.
#pragma once

#include "step.cuh"

namespace wb {

struct FastExtras {
    const float2 *invMetric;     // [eta][xi] {1/xdist, 1/ydist}
    const float *depthIntervals; // [sW-1]
    const wacomm_b200_config *cfgDevice;  // device copy of the run parameters
};

template <int STORE>
struct FastView {
    PackedView<STORE> V;   // node layout: wind/Stokes pair, lon/lat (drift model)
    CellView<STORE> C;     // cell-column layout: velocity stencil and surface
    FastExtras X;
};

// Space-time weights of the 8 stencil values of one field: (1-a) w_c for record t0 and a w_c for
// record t1, corners (j,i), (j+1,i), (j+1,i+1), (j,i+1).
struct Weights8 {
    float p1, p2, p3, p4, q1, q2, q3, q4;
};

// The products run in pairs on the packed FP32x2 multiply of sm_100 (the same roundings).
__device__ __forceinline__ Weights8 weights8(float jF, float iF, float a) {
    const float oi = 1.f - iF, oj = 1.f - jF, b = 1.f - a;
    const float2 w12 = __fmul2_rn(make_float2(oi, oi), make_float2(oj, jF));
    const float2 w34 = __fmul2_rn(make_float2(iF, iF), make_float2(jF, oj));
    const float2 bb = make_float2(b, b), aa = make_float2(a, a);
    const float2 p12 = __fmul2_rn(bb, w12), p34 = __fmul2_rn(bb, w34);
    const float2 q12 = __fmul2_rn(aa, w12), q34 = __fmul2_rn(aa, w34);
    return Weights8{p12.x, p12.y, p34.x, p34.y, q12.x, q12.y, q34.x, q34.y};
}

// The 8 products summed as pairs of corners (c1, c2 | c3, c4) with the packed FP32x2 multiply
// and multiply-add of sm_100, record t0 and record t1 apart, then the four partial sums.
__device__ __forceinline__ float blend(const QuadPair &q, const Weights8 &w) {
    float2 x = __fmul2_rn(make_float2(q.t0.c1, q.t0.c2), make_float2(w.p1, w.p2));
    float2 y = __fmul2_rn(make_float2(q.t1.c1, q.t1.c2), make_float2(w.q1, w.q2));
    x = __ffma2_rn(make_float2(q.t0.c3, q.t0.c4), make_float2(w.p3, w.p4), x);
    y = __ffma2_rn(make_float2(q.t1.c3, q.t1.c4), make_float2(w.q3, w.q4), y);
    const float2 t = __fadd2_rn(x, y);
    return t.x + t.y;
}

// Bilinear h + zeta@t0 and zeta@t1 - zeta@t0 at a fractional position of a cell (FP32); the water
// column height at time weight a is s + a d.
struct SurfaceSums {
    float s, d;
    __device__ __forceinline__ float height(float a) const { return fmaf(a, d, s); }
};

// Corner weights in pairs {w1, w2}, {w3, w4} (packed FP32x2 multiplies).
__device__ __forceinline__ void corner_pairs(float jF, float iF, float2 &w12, float2 &w34) {
    const float oi = 1.f - iF, oj = 1.f - jF;
    w12 = __fmul2_rn(make_float2(oi, oi), make_float2(oj, jF));
    w34 = __fmul2_rn(make_float2(iF, iF), make_float2(jF, oj));
}

__device__ __forceinline__ SurfaceSums surface_from(const CellSurface &c, float jF, float iF) {
    float2 w12, w34;
    corner_pairs(jF, iF, w12, w34);
    float2 s = __fmul2_rn(make_float2(c.s0.x, c.s0.y), w12);
    float2 d = __fmul2_rn(make_float2(c.dz.x, c.dz.y), w12);
    s = __ffma2_rn(make_float2(c.s0.z, c.s0.w), w34, s);
    d = __ffma2_rn(make_float2(c.dz.z, c.dz.w), w34, d);
    return SurfaceSums{s.x + s.y, d.x + d.y};
}

template <int STORE>
__device__ __forceinline__ SurfaceSums surface_sums(const CellView<STORE> &C, int jI, int iI,
                                                    float jF, float iF) {
    return surface_from(C.surf(jI, iI), jF, iF);
}

// Water column height h + zeta at a fractional position of a cell (FP32).
template <int STORE>
__device__ __forceinline__ float column_height(const CellView<STORE> &C, int jI, int iI, float jF,
                                               float iF, float a) {
    return surface_sums(C, jI, iI, jF, iF).height(a);
}

// The velocity stencil of one cell and level at one time: u, v and the two w levels per corner.
struct StencilAt {
    Quad u, v, wUp, wLo;
};

// t0 + a (t1 - t0) per corner, two corners per packed FP32x2 add and multiply-add.
__device__ __forceinline__ Quad at_time(const QuadPair &q, float a) {
    const float2 a2 = make_float2(a, a);
    const float2 lo0 = make_float2(q.t0.c1, q.t0.c2), hi0 = make_float2(q.t0.c3, q.t0.c4);
    const float2 lo = __ffma2_rn(a2, __fadd2_rn(make_float2(q.t1.c1, q.t1.c2), make_float2(-lo0.x, -lo0.y)), lo0);
    const float2 hi = __ffma2_rn(a2, __fadd2_rn(make_float2(q.t1.c3, q.t1.c4), make_float2(-hi0.x, -hi0.y)), hi0);
    return Quad{lo.x, lo.y, hi.x, hi.y};
}

__device__ __forceinline__ float bilinear4(const Quad &q, float2 w12, float2 w34) {
    const float2 x = __ffma2_rn(make_float2(q.c3, q.c4), w34, __fmul2_rn(make_float2(q.c1, q.c2), w12));
    return x.x + x.y;
}

// Current (u, v, w) and, when wanted, AKT at a fractional position: one stencil read. With `keep`
// the stencil's corners blended to time weight aKeep are returned as well, for a second
// evaluation in the same cell and level without a second read.
template <int STORE, bool KEEP = false>
__device__ __forceinline__ void current_cell(const CellView<STORE> &C, int kI, float kF, int jI,
                                             float jF, int iI, float iF, float a, float aAkt,
                                             bool wantAkt, float &uu, float &vv, float &ww,
                                             float &aa, float aKeep = 0.f,
                                             StencilAt *keep = nullptr) {
    QuadPair u, v, wUp, aUp, wLo, aLo;
    if (wantAkt) C.stencil(kI, jI, iI, u, v, wUp, aUp, wLo, aLo);
    else C.stencil_w(kI, jI, iI, u, v, wUp, wLo);
    Weights8 w = weights8(jF, iF, a);
    uu = blend(u, w);
    vv = blend(v, w);
    float up = blend(wUp, w), lo = blend(wLo, w);
    ww = fmaf(lo - up, kF, up);
    if (wantAkt) {
        Weights8 wa = aAkt == a ? w : weights8(jF, iF, aAkt);
        float au = blend(aUp, wa), al = blend(aLo, wa);
        aa = fmaf(al - au, kF, au);
    }
    if (KEEP) {
        keep->u = at_time(u, aKeep);
        keep->v = at_time(v, aKeep);
        keep->wUp = at_time(wUp, aKeep);
        keep->wLo = at_time(wLo, aKeep);
    }
}

// Current (u, v, w) from a kept stencil at a fractional position of its cell and level.
__device__ __forceinline__ void current_kept(const StencilAt &k, float kF, float jF, float iF,
                                             float &uu, float &vv, float &ww) {
    float2 w12, w34;
    corner_pairs(jF, iF, w12, w34);
    uu = bilinear4(k.u, w12, w34);
    vv = bilinear4(k.v, w12, w34);
    const float up = bilinear4(k.wUp, w12, w34), lo = bilinear4(k.wLo, w12, w34);
    ww = fmaf(lo - up, kF, up);
}


// Leeway and Stokes velocity of a drifting object (the drift branch of advective_velocity) in FP32:
// wind and Stokes interpolated from the environment pair, the leeway regression of the object's
// catalogue row (computeLeeway, DriftModel.hpp:204-219) on the interpolated 10-m wind. The
// position-dependent parts (calibration regions, wind-error fields) and the coefficient ensemble
// exist only in the FULL form, run in FP64 there and only when the run configures them.
template <bool FULL, class View>
__device__ __forceinline__ void drift_velocity(const wacomm_b200_config &cfg, const IntervalParams &P,
                                            const View &V, uint64_t id, int type, int side,
                                            int jI, float jF, int iI, float iF, float a,
                                            double elapsed, double physicalTime, double stepDt,
                                            float &du, float &dv) {
    float windU = (float)cfg.windU10, windV = (float)cfg.windV10;
    EnvPair e1{}, e2{}, e3{}, e4{};
    if (V.hasWindU || V.hasWindV || V.hasStokes) {
        e1 = V.environment(jI, iI);
        e2 = V.environment(jI + 1, iI);
        e3 = V.environment(jI + 1, iI + 1);
        e4 = V.environment(jI, iI + 1);
    }
    const float w1 = (1.f - iF) * (1.f - jF), w2 = (1.f - iF) * jF, w3 = iF * jF, w4 = iF * (1.f - jF);
    if (V.hasWindU)
        windU = at_f32(e1.wu0 * w1 + e2.wu0 * w2 + e3.wu0 * w3 + e4.wu0 * w4,
                       e1.wu1 * w1 + e2.wu1 * w2 + e3.wu1 * w3 + e4.wu1 * w4, a);
    if (V.hasWindV)
        windV = at_f32(e1.wv0 * w1 + e2.wv0 * w2 + e3.wv0 * w3 + e4.wv0 * w4,
                       e1.wv1 * w1 + e2.wv1 * w2 + e3.wv1 * w3 + e4.wv1 * w4, a);
    if (FULL && (cfg.observationalCalibrationRegionCount > 0 || cfg.windErrorStdDev > 0)) {
        const double jd = jF, id_ = iF;
        double longitude = V.lon(jI, iI) * (1.0 - id_) * (1.0 - jd) + V.lon(jI + 1, iI) * (1.0 - id_) * jd +
                           V.lon(jI + 1, iI + 1) * id_ * jd + V.lon(jI, iI + 1) * id_ * (1.0 - jd);
        double latitude = V.lat(jI, iI) * (1.0 - id_) * (1.0 - jd) + V.lat(jI + 1, iI) * (1.0 - id_) * jd +
                          V.lat(jI + 1, iI + 1) * id_ * jd + V.lat(jI, iI + 1) * id_ * (1.0 - jd);
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
            uint64_t substep = (uint64_t)floor(elapsed / cfg.dti);
            double when = physicalTime + .5 * P.direction * stepDt;
            double first = forcing_error_normal(cfg.randomSeed, id, P.intervalKey, substep,
                                                WIND_U_COMPONENT, longitude, latitude, when,
                                                spatial, temporal);
            double second = forcing_error_normal(cfg.randomSeed, id, P.intervalKey, substep,
                                                 WIND_V_COMPONENT, longitude, latitude, when,
                                                 spatial, temporal);
            windU = (float)(windU + stdDev * first);
            windV = (float)(windV + stdDev * correlated_normal(first, second, corr));
        }
    }
    float dn = 0.f, cn = 0.f;
    if (FULL && cfg.leewayCoefficientEnsemble) {
        uint64_t ens = key_prefix(cfg.randomSeed, id, ENSEMBLE_INTERVAL, 0);
        double n0 = prefix_normal(ens, 0);
        dn = (float)n0;
        cn = (float)correlated_normal(n0, prefix_normal(ens, 1), cfg.leewayResidualCorrelation);
    }
    du = dv = 0.f;
    const float speed = sqrtf(windU * windU + windV * windV);
    if (speed >= 1.0e-12f && side != 0 && type >= 0 && type <= 22) {
        const float *c = c_leeway_catalogue_f32[type];
        const bool right = side == 1;
        const float rs = 1.0f / speed;
        const float ux = windU * rs, uy = windV * rs;
        const float downwind = __ldg(c + 0) * speed + __ldg(c + 1) + __ldg(c + 2) * dn;
        const float crosswind = right ? __ldg(c + 3) * speed + __ldg(c + 4) + __ldg(c + 5) * cn
                                      : __ldg(c + 6) * speed + __ldg(c + 7) - __ldg(c + 8) * cn;
        du = downwind * ux - crosswind * uy;
        dv = downwind * uy + crosswind * ux;
    }
    if (V.hasStokes) {
        du += at_f32(e1.su0 * w1 + e2.su0 * w2 + e3.su0 * w3 + e4.su0 * w4,
                     e1.su1 * w1 + e2.su1 * w2 + e3.su1 * w3 + e4.su1 * w4, a);
        dv += at_f32(e1.sv0 * w1 + e2.sv0 * w2 + e3.sv0 * w3 + e4.sv0 * w4,
                     e1.sv1 * w1 + e2.sv1 * w2 + e3.sv1 * w3 + e4.sv1 * w4, a);
    }
}

__device__ __forceinline__ float signf_of(float a, float b) {
    return fabsf(a) * (float)((b > 0.f) - (b < 0.f));
}

// VARIANT (VAR_*): the branches the run parameters can reach are compiled in, the rest out --
// fewer registers and a smaller instruction footprint for the common runs.
template <int SEM, int STORE, int VARIANT>
__device__ int move_particle_fast(const wacomm_b200_config &cfg, const IntervalParams &P,
                                  const FastView<STORE> &F, ParticleState &p, double &elapsed,
                                  int *err) {
    const PackedView<STORE> &V = F.V;
    const CellView<STORE> &C = F.C;
    const int eta = V.g.eta, xi = V.g.xi, sW = V.g.sW;
    const double kLower = P.kLower, length = P.length;
    const double invLength = length == 0 ? 0.0 : 1.0 / length;
    const int direction = P.direction;
    const float dirf = (float)direction;
    const float sv = (float)cfg.sv, shore = (float)cfg.shoreLimit;
    const bool midpoint = cfg.integrator == INTEGRATOR_MIDPOINT;
    constexpr bool canDiffuse = VARIANT != VAR_LEAN, canDrift = VARIANT >= VAR_DRIFT;
    constexpr bool full = VARIANT == VAR_FULL;
    const bool diffuse = canDiffuse && cfg.random && (direction > 0 || cfg.backwardDiffusion);
    const bool drift = canDrift && cfg.driftModel == 1 && p.type != 0;
    const bool jibe = full && cfg.leewayJibeProbabilityHourly > 0 && p.type != 0;
    if (drift && SEM == SEM_HOST && (p.type < 0 || p.type > 22)) atomicOr(err, ERR_DRIFT_OBJECT);
    bool lazy = false;
    int steps = 0;
    // Substeps left in which the lazy survival tests cannot change their outcome (age below
    // min(ageKillLo, ageUnder): neither dead nor without health), counted when the particle turns
    // lazy, two substeps short of the bound for rounding; skipped while it lasts and no closure
    // has ended the lazy tracking.
    const double ageSafe = fmin(P.ageKillLo, P.ageUnder);
    int youngLeft = 0;

    if (P.firstChunk) {
        if (p.k > 0) close_upper(cfg, p.k, p.health, lazy);
        if (p.k < kLower) close_lower(cfg, kLower, p.k, p.health, lazy);
    }
    const uint64_t prefix = fold(fold(mix64(cfg.randomSeed), p.id), (uint64_t)P.intervalKey);
    const uint64_t philoxKey = p.id ^ mix64(cfg.randomSeed);
    const double stop = P.chunkEnd < length ? P.chunkEnd : length;
    // surface sums, cell and fractional position of the previous step's destination, valid while
    // the particle still sits there: the next step starts from the same values
    constexpr bool keepStencil = VARIANT == VAR_LEAN;
    SurfaceSums carried{0.f, 0.f};
    int carriedJ = 0, carriedI = 0;
    float carriedJF = 0.f, carriedIF = 0.f;
    bool haveCarried = false;

    while (elapsed < stop) {
        double stepDt = fmin(cfg.dti, length - elapsed);
        double physicalTime = P.start + direction * elapsed;
        if (direction > 0 && p.time > physicalTime) {
            elapsed = fmin(length, p.time - P.start);
            continue;
        }
        if (!(lazy && youngLeft > 0)) {
            bool dead = lazy ? (p.age >= P.ageKillHi ||
                                (p.age > P.ageKillLo && exp(-p.age / cfg.tau0) < cfg.survprob))
                             : p.health < cfg.survprob;
            if (dead) {
                p.health = -1;
                lazy = false;
                elapsed = length;
                break;
            }
        }
        const double kc = ceil(p.k);
        const int kI = to_index<SEM>(kc);
        int jI, iI;
        float jF, iF;
        if (haveCarried) {
            jI = carriedJ;
            iI = carriedI;
            jF = carriedJF;
            iF = carriedIF;
        } else {
            const double fj0 = floor(p.j), fi0 = floor(p.i);
            jI = to_index<SEM>(fj0);
            iI = to_index<SEM>(fi0);
            jF = (float)(p.j - fj0);
            iF = (float)(p.i - fi0);
        }
        if (!valid_cell(jI, iI, eta, xi) || (SEM == SEM_DEVICE && (kI > 0 || kI <= -sW + 1))) {
            p.health = -1;
            lazy = false;
            elapsed = length;
            break;
        }
        steps++;
        const float kF = (float)(kc - p.k);
        const float dt = (float)stepDt;
        const float alpha = (float)((elapsed + 0.5 * stepDt) * invLength);
        const float alphaStart = (float)(elapsed * invLength);
        const SurfaceSums here = haveCarried ? carried : surface_sums(C, jI, iI, jF, iF);
        haveCarried = false;
        const float hc = here.height(alpha);
        if (hc <= shore && cfg.horizontalClosure == CLOSURE_KILL) {
            p.health = -1;
            lazy = false;
            if (SEM == SEM_DEVICE) {
                elapsed = length;
                break;
            }
        }
        const int kM = mem_level(kI, sW);
        const float sa = midpoint ? alphaStart : alpha;
        float uu, vv, ww, aa = 0.f;
        // the start stencil at the mid-stage time (midpoint rule; the lean form has the registers)
        StencilAt kept;
        if (keepStencil && midpoint)
            current_cell<STORE, true>(C, kM, kF, jI, jF, iI, iF, sa, alpha, diffuse, uu, vv, ww, aa,
                                      alpha, &kept);
        else
            current_cell(C, kM, kF, jI, jF, iI, iF, sa, alpha, diffuse, uu, vv, ww, aa);
        if (drift) {
            float du, dv;
            drift_velocity<full>(cfg, P, V, p.id, p.type, p.side, jI, jF, iI, iF, sa, elapsed,
                           physicalTime, stepDt, du, dv);
            uu += du;
            vv += dv;
        }
        // the substep index keys the reference draws and the jibe draw; Philox streams are keyed
        // on the step's elapsed time instead (unique per step, no division)
        uint64_t stepKey = 0;
        const bool philox = P.rng == WACOMM_B200_RNG_PHILOX;
        if ((diffuse && !philox) || jibe) stepKey = fold(prefix, (uint64_t)floor(elapsed / cfg.dti));
        float rx = 0.f, ry = 0.f, rz = 0.f;
        if (diffuse) {
            float sigmaDepth = (float)(cfg.sigma * (1 - p.k * P.invKLower));
            float scale = sqrtf(dt / (float)cfg.dti);
            float n0, n1, n2;
            if (philox) {
                philox_normals3(philoxKey, P.intervalKey, (uint64_t)__double_as_longlong(elapsed),
                                n0, n1, n2);
            } else {
                n0 = (float)prefix_normal(stepKey, 0);
                n1 = (float)prefix_normal(stepKey, 1);
                n2 = (float)prefix_normal(stepKey, 2);
            }
            const float2 rxy = __fmul2_rn(
                __fmul2_rn(make_float2(sigmaDepth, sigmaDepth), make_float2(n0, n1)),
                make_float2(scale, scale));
            rx = rxy.x;
            ry = rxy.y;
            rz = sigmaDepth * n2 * aa * (float)cfg.crid * scale;
        }
        const float2 inv = __ldg(F.X.invMetric + (size_t)jI * xi + iI);
        const float depthHere = __ldg(F.X.depthIntervals + (kM + sW - 2));
        const float zdist = hc * depthHere;
        const float rzdist = __frcp_rn(zdist);
        // index increments (i, j) and the vertical leap in metres
        float dI, dJ, zleap;
        if (midpoint) {
            float kHalf = dirf * (sv + ww) * 0.5f * dt;
            if (fabsf(kHalf) > zdist) kHalf = signf_of(zdist, kHalf);
            // (dirf u 0.5 dt) / dx for i and j as one packed FP32x2 chain (the same roundings)
            const float2 half = __fmul2_rn(
                __fmul2_rn(__fmul2_rn(make_float2(dirf * uu, dirf * vv), make_float2(0.5f, 0.5f)),
                           make_float2(dt, dt)),
                inv);
            double iMid = p.i + (double)half.x;
            double jMid = p.j + (double)half.y;
            double kMid = fmin(0.0, fmax(kLower, p.k + (double)(kHalf * rzdist)));
            double fim = floor(iMid), fjm = floor(jMid);
            int iMI = to_index<SEM>(fim), jMI = to_index<SEM>(fjm);
            bool midValid = valid_cell(jMI, iMI, eta, xi);
            float hcMid = 0.f, iMF = 0.f, jMF = 0.f;
            if (midValid) {
                iMF = (float)(iMid - fim);
                jMF = (float)(jMid - fjm);
                hcMid = column_height(C, jMI, iMI, jMF, iMF, alpha);
                midValid = hcMid > shore && hcMid > 0.f;
            }
            float detZ;
            if (midValid) {
                double kmc = ceil(kMid);
                int kMI = mem_level(to_index<SEM>(kmc), sW);
                float kMF = (float)(kmc - kMid);
                float um, vm, wm, unused;
                if (keepStencil && kMI == kM && jMI == jI && iMI == iI)
                    current_kept(kept, kMF, jMF, iMF, um, vm, wm);
                else
                    current_cell(C, kMI, kMF, jMI, jMF, iMI, iMF, alpha, alpha, false, um, vm, wm,
                                 unused);
                if (drift) {
                    float du, dv;
                    drift_velocity<full>(cfg, P, V, p.id, p.type, p.side, jMI, jMF, iMI, iMF, alpha,
                                   elapsed, physicalTime, stepDt, du, dv);
                    um += du;
                    vm += dv;
                }
                const bool sameCell = jMI == jI && iMI == iI;
                const float2 im = sameCell ? inv : __ldg(F.X.invMetric + (size_t)jMI * xi + iMI);
                float zdistMid =
                    hcMid * (kMI == kM ? depthHere : __ldg(F.X.depthIntervals + (kMI + sW - 2)));
                const float2 d = __fmul2_rn(
                    __fmul2_rn(make_float2(dirf * um, dirf * vm), make_float2(dt, dt)), im);
                dI = d.x;
                dJ = d.y;
                detZ = dirf * (sv + wm) * dt * zdist * __frcp_rn(zdistMid);
            } else {
                float ue, ve, we, unused;
                if (keepStencil) current_kept(kept, kF, jF, iF, ue, ve, we);
                else current_cell(C, kM, kF, jI, jF, iI, iF, alpha, alpha, false, ue, ve, we, unused);
                if (drift) {
                    float du, dv;
                    drift_velocity<full>(cfg, P, V, p.id, p.type, p.side, jI, jF, iI, iF, alpha, elapsed,
                                   physicalTime, stepDt, du, dv);
                    ue += du;
                    ve += dv;
                }
                const float2 d = __fmul2_rn(
                    __fmul2_rn(make_float2(dirf * ue, dirf * ve), make_float2(dt, dt)), inv);
                dI = d.x;
                dJ = d.y;
                detZ = dirf * (sv + we) * dt;
            }
            dI += rx * inv.x;
            dJ += ry * inv.y;
            zleap = detZ + rz;
        } else {
            dI = (dirf * uu * dt + rx) * inv.x;
            dJ = (dirf * vv * dt + ry) * inv.y;
            zleap = dirf * (sv + ww) * dt + rz;
        }
        if (fabsf(zleap) > zdist) zleap = signf_of(zdist, zleap);
        double jdet = p.j + (double)dJ;
        double idet = p.i + (double)dI;
        double kdet = p.k + (double)(zleap * rzdist);
        if (kdet > 0.) close_upper(cfg, kdet, p.health, lazy);
        if (kdet < kLower) close_lower(cfg, kLower, kdet, p.health, lazy);

        double fjd = floor(jdet), fid = floor(idet);
        int jdetI = to_index<SEM>(fjd), idetI = to_index<SEM>(fid);
        if (valid_cell(jdetI, idetI, eta, xi)) {
            const float jdF = (float)(jdet - fjd), idF = (float)(idet - fid);
            const SurfaceSums there = surface_sums(C, jdetI, idetI, jdF, idF);
            float hcdet = there.height(alpha);
            // the next step starts here unless a closure moves the particle
            carried = there;
            carriedJ = jdetI;
            carriedI = idetI;
            carriedJF = jdF;
            carriedIF = idF;
            haveCarried = hcdet > shore;
            if (hcdet <= shore) {
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
        bool alive;
        if (lazy && youngLeft > 0) {  // still lazy: no closure ended the tracking this substep
            alive = true;
            youngLeft--;
        } else {
            alive = lazy ? (p.age < P.ageUnder || exp(-p.age / cfg.tau0) > 0) : p.health > 0;
            if (alive && !lazy) {
                // FP32 and an approximate division: the two-substep margin covers their error
                const float n = floorf(__fdividef((float)(ageSafe - p.age), (float)cfg.dti)) - 2.f;
                youngLeft = n > 0.f ? (n < 1.0e9f ? (int)n : 1000000000) : 0;
            }
        }
        if (alive) {
            p.age = p.age + stepDt;
            lazy = true;
            if (jibe) {
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
