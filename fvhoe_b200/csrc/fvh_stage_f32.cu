// FP32 stage runner: reconstruction, Riemann fluxes and detection in float32,
// the stage accumulation of the conserved state in float64. Compiled with
// FMA contraction enabled.
#include "fvh_stage.cuh"

namespace fvh {

int run_stage_f32(fvh_handle* h, const StageCall& c, cudaStream_t s) { return run_stage_any<float>(h, c, s); }

}  // namespace fvh
