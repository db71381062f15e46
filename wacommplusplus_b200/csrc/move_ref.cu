// Move kernels in reference arithmetic (compiled with -fmad=false: every product and sum is
// rounded on its own, as in the reference's x86-64 Release build).
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

cudaError_t move_ref_dispatch(int semantics, const wacomm_b200_config &cfg,
                              const IntervalParams &P, const PackedArgs &A, const ParticleSoA &S,
                              const MoveLaunch &L, int blockSize, cudaStream_t stream) {
    PackedView<STORE_F32> V = typed_view<STORE_F32>(A);
    if (semantics == SEM_HOST)
        return launch_move_soa<SEM_HOST, ARITH_REF, STORE_F32>(cfg, P, V, S, L, blockSize, stream);
    return launch_move_soa<SEM_DEVICE, ARITH_REF, STORE_F32>(cfg, P, V, S, L, blockSize, stream);
}

}  // namespace wb
