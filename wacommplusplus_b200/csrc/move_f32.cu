// FP32 move kernels (step_fast.cuh) over FP32, FP16 or BF16 forcing storage; positions and
// closures stay FP64. The kernels live in the move_f32_<rules>_<storage>.cu units.
#include "engine.h"
#include "move_kernels.cuh"

namespace wb {

template <int SEM, int STORE>
cudaError_t move_f32_unit(int shape, const wacomm_b200_config &cfg, const IntervalParams &P,
                          const PackedArgs &A, const ParticleSoA &S, const MoveLaunch &L,
                          cudaStream_t stream);

template <int SEM>
static cudaError_t by_storage(int storage, int shape, const wacomm_b200_config &cfg,
                              const IntervalParams &P, const PackedArgs &A, const ParticleSoA &S,
                              const MoveLaunch &L, cudaStream_t stream) {
    switch (storage) {
        case STORE_F16: return move_f32_unit<SEM, STORE_F16>(shape, cfg, P, A, S, L, stream);
        case STORE_BF16: return move_f32_unit<SEM, STORE_BF16>(shape, cfg, P, A, S, L, stream);
        default: return move_f32_unit<SEM, STORE_F32>(shape, cfg, P, A, S, L, stream);
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
