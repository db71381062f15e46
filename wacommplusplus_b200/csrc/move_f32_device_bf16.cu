// The FP32 step's kernels for device rules over BF16 forcing storage.
#include "move_f32_unit.cuh"

namespace wb {
template cudaError_t move_f32_unit<SEM_DEVICE, STORE_BF16>(int, const wacomm_b200_config &,
                                                const IntervalParams &, const PackedArgs &,
                                                const ParticleSoA &, const MoveLaunch &,
                                                cudaStream_t);
}  // namespace wb
