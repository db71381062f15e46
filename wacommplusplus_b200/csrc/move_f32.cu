// FP32 move kernels (step_fast.cuh) over FP32, FP16 or BF16 forcing storage; positions and
// closures stay FP64.
#include "engine.h"
#include "move_kernels.cuh"

namespace wb {

template <int STORE>
static PackedView<STORE> typed_view(const PackedArgs &A) {
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
static FastView<STORE> fast_view(const PackedArgs &A) {
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

template <int SEM, int STORE>
static cudaError_t by_shape(int shape, const wacomm_b200_config &cfg, const IntervalParams &P,
                            const PackedArgs &A, const ParticleSoA &S, const MoveLaunch &L,
                            cudaStream_t stream) {
    FastView<STORE> F = fast_view<STORE>(A);
    // deterministic passive tracking: no diffusion, no drifting objects, no jibing
    const bool lean = !(cfg.random && (P.direction > 0 || cfg.backwardDiffusion)) &&
                      cfg.driftModel != 1 && !(cfg.leewayJibeProbabilityHourly > 0);
    switch (shape) {
        case 0: return launch_move_fast<SEM, STORE, 0, false>(cfg, P, F, S, L, stream);
        case 2:
            return lean ? launch_move_fast<SEM, STORE, 2, true>(cfg, P, F, S, L, stream)
                        : launch_move_fast<SEM, STORE, 2, false>(cfg, P, F, S, L, stream);
        case 3: return launch_move_fast<SEM, STORE, 3, false>(cfg, P, F, S, L, stream);
        default:
            return lean ? launch_move_fast<SEM, STORE, 1, true>(cfg, P, F, S, L, stream)
                        : launch_move_fast<SEM, STORE, 1, false>(cfg, P, F, S, L, stream);
    }
}

template <int SEM>
static cudaError_t by_storage(int storage, int shape, const wacomm_b200_config &cfg,
                              const IntervalParams &P, const PackedArgs &A, const ParticleSoA &S,
                              const MoveLaunch &L, cudaStream_t stream) {
    switch (storage) {
        case STORE_F16: return by_shape<SEM, STORE_F16>(shape, cfg, P, A, S, L, stream);
        case STORE_BF16: return by_shape<SEM, STORE_BF16>(shape, cfg, P, A, S, L, stream);
        default: return by_shape<SEM, STORE_F32>(shape, cfg, P, A, S, L, stream);
    }
}

cudaError_t move_f32_dispatch(int semantics, int storage, int shape, const wacomm_b200_config &cfg,
                              const IntervalParams &P, const PackedArgs &A, const ParticleSoA &S,
                              const MoveLaunch &L, cudaStream_t stream) {
    if (semantics == SEM_HOST)
        return by_storage<SEM_HOST>(storage, shape, cfg, P, A, S, L, stream);
    return by_storage<SEM_DEVICE>(storage, shape, cfg, P, A, S, L, stream);
}

}  // namespace wb
