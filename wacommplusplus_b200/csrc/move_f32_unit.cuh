// FP32 move kernels (step_fast.cuh) for one rule set and one forcing storage: the instances of
// move_fast_kernel by launch shape and compiled form. Each move_f32_<rules>_<storage>.cu unit
// instantiates move_f32_unit for its pair, so the kernels build in parallel.
#pragma once

#include "engine.h"
#include "move_kernels.cuh"

namespace wb {

template <int STORE>
inline PackedView<STORE> typed_view(const PackedArgs &A) {
    PackedView<STORE> V;
    V.g = GridShape{A.eta, A.xi, A.sW, A.sRho};
    V.nodes = static_cast<const NodeRecord<STORE> *>(A.nodes);
    V.surf = A.surf;
    V.env = A.env;
    V.hasWindU = A.hasWindU;
    V.hasWindV = A.hasWindV;
    V.hasStokes = A.hasStokes;
    V.lonRad = A.lonRad;
    V.latRad = A.latRad;
    V.depthIntervals = A.depthIntervals;
    V.metric = A.metric;
    return V;
}

template <int STORE>
inline FastView<STORE> fast_view(const PackedArgs &A) {
    FastView<STORE> F;
    F.V = typed_view<STORE>(A);
    F.X.invMetric = A.invMetric;
    F.X.depthIntervals = A.depthIntervalsF;
    F.X.cfgDevice = A.cfgDevice;
    F.C.eta = A.eta;
    F.C.xi = A.xi;
    F.C.sW = A.sW;
    F.C.columns = static_cast<const CellQuad<STORE> *>(A.cells);
    F.C.surface = static_cast<const CellSurface *>(A.cellSurface);
    return F;
}

// The compiled form a run needs (VAR_*).
inline int fast_variant(const wacomm_b200_config &cfg, int direction) {
    const bool diffuse = cfg.random && (direction > 0 || cfg.backwardDiffusion);
    const bool drift = cfg.driftModel == 1, jibe = cfg.leewayJibeProbabilityHourly > 0;
    const bool plainDrift = cfg.observationalCalibrationRegionCount == 0 &&
                            !(cfg.windErrorStdDev > 0) && !cfg.leewayCoefficientEnsemble;
    if (jibe || (drift && !plainDrift)) return VAR_FULL;
    if (drift) return VAR_DRIFT;
    return diffuse ? VAR_DIFFUSE : VAR_LEAN;
}

// Shapes 1, 2 and 3 carry every form; shape 0 the full one. A negative shape picks by form: the
// lean form fits shape 3's 96 registers without spills and runs 4 % faster there (20 resident
// warps per SM instead of 16); the others spill at shape 3 and run at shape 2.
template <int SEM, int STORE>
cudaError_t move_f32_unit(int shape, const wacomm_b200_config &cfg, const IntervalParams &P,
                          const PackedArgs &A, const ParticleSoA &S, const MoveLaunch &L,
                          cudaStream_t stream) {
    FastView<STORE> F = fast_view<STORE>(A);
    const int variant = fast_variant(cfg, P.direction);
    if (shape < 0) shape = variant == VAR_LEAN ? 3 : 2;
    switch (shape) {
        case 0: return launch_move_fast<SEM, STORE, 0, VAR_FULL>(cfg, P, F, S, L, stream);
        case 3:
            switch (variant) {
                case VAR_LEAN: return launch_move_fast<SEM, STORE, 3, VAR_LEAN>(cfg, P, F, S, L, stream);
                case VAR_DIFFUSE: return launch_move_fast<SEM, STORE, 3, VAR_DIFFUSE>(cfg, P, F, S, L, stream);
                case VAR_DRIFT: return launch_move_fast<SEM, STORE, 3, VAR_DRIFT>(cfg, P, F, S, L, stream);
                default: return launch_move_fast<SEM, STORE, 3, VAR_FULL>(cfg, P, F, S, L, stream);
            }
        case 2:
            switch (variant) {
                case VAR_LEAN: return launch_move_fast<SEM, STORE, 2, VAR_LEAN>(cfg, P, F, S, L, stream);
                case VAR_DIFFUSE: return launch_move_fast<SEM, STORE, 2, VAR_DIFFUSE>(cfg, P, F, S, L, stream);
                case VAR_DRIFT: return launch_move_fast<SEM, STORE, 2, VAR_DRIFT>(cfg, P, F, S, L, stream);
                default: return launch_move_fast<SEM, STORE, 2, VAR_FULL>(cfg, P, F, S, L, stream);
            }
        default:
            switch (variant) {
                case VAR_LEAN: return launch_move_fast<SEM, STORE, 1, VAR_LEAN>(cfg, P, F, S, L, stream);
                case VAR_DIFFUSE: return launch_move_fast<SEM, STORE, 1, VAR_DIFFUSE>(cfg, P, F, S, L, stream);
                case VAR_DRIFT: return launch_move_fast<SEM, STORE, 1, VAR_DRIFT>(cfg, P, F, S, L, stream);
                default: return launch_move_fast<SEM, STORE, 1, VAR_FULL>(cfg, P, F, S, L, stream);
            }
    }
}

}  // namespace wb
