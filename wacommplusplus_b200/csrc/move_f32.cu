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
    return F;
}

template <int SEM>
static cudaError_t by_storage(int storage, const wacomm_b200_config &cfg, const IntervalParams &P,
                              const PackedArgs &A, const ParticleSoA &S, const MoveLaunch &L,
                              int blockSize, cudaStream_t stream) {
    switch (storage) {
        case STORE_F16:
            return launch_move_fast<SEM, STORE_F16>(cfg, P, fast_view<STORE_F16>(A), S, L,
                                                    blockSize, stream);
        case STORE_BF16:
            return launch_move_fast<SEM, STORE_BF16>(cfg, P, fast_view<STORE_BF16>(A), S, L,
                                                     blockSize, stream);
        default:
            return launch_move_fast<SEM, STORE_F32>(cfg, P, fast_view<STORE_F32>(A), S, L,
                                                    blockSize, stream);
    }
}

cudaError_t move_f32_dispatch(int semantics, int storage, const wacomm_b200_config &cfg,
                              const IntervalParams &P, const PackedArgs &A, const ParticleSoA &S,
                              const MoveLaunch &L, int blockSize, cudaStream_t stream) {
    if (semantics == SEM_HOST)
        return by_storage<SEM_HOST>(storage, cfg, P, A, S, L, blockSize, stream);
    return by_storage<SEM_DEVICE>(storage, cfg, P, A, S, L, blockSize, stream);
}

}  // namespace wb
