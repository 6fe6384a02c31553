// FP32 ensemble kernels: reconstruction, Riemann fluxes and detection in
// float32, stage accumulation in float64 (compiled with fast math, like the
// FP32 stage runner).
#include "fvh_ensemble_launch.cuh"

namespace fvh {
namespace ens {

int launch_stage_f32(fvh_ensemble* e, int stage, int last, cudaStream_t s) {
  return launch_any<float>(e, stage, last, s);
}

int max_blocks_f32(int p, int variant, size_t* smem) { return max_blocks_any<float>(p, variant, smem); }

}  // namespace ens
}  // namespace fvh
