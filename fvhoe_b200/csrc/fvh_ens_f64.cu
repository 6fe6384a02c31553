// FP64 ensemble kernels (compiled with -fmad=false, like the FP64 stage
// runner, so an ensemble member equals the same problem run alone).
#include "fvh_ensemble_launch.cuh"

namespace fvh {
namespace ens {

int launch_stage_f64(fvh_ensemble* e, int stage, int last, cudaStream_t s) {
  return launch_any<double>(e, stage, last, s);
}

int max_blocks_f64(int p, int variant, size_t* smem) { return max_blocks_any<double>(p, variant, smem); }

}  // namespace ens
}  // namespace fvh
