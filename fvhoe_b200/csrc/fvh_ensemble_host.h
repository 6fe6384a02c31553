// Host side of the batched ensemble: the object behind fvh_ensemble_* (C ABI in
// include/fvh.h), shared by the API unit and the per-precision launch units.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "fvh.h"
#include "fvh_ensemble.cuh"

namespace fvh {
namespace ens {

// Tile shapes of the fluxes / detection / final phases the autotuner chooses from.
constexpr int kVariants = 3;
constexpr int kVariantTX[kVariants] = {16, 8, 16};
constexpr int kVariantTY[kVariants] = {32, 32, 64};

}  // namespace ens
}  // namespace fvh

struct fvh_ensemble {
  fvh_config cfg{};
  int nprob = 0;
  int p = 0;          // degree on both axes
  int r = 0;          // ceil(p / 2)
  int gw = 0;         // ghost width of the flux pass
  int gW = 0;         // ghost width of W
  size_t elem = 8;    // bytes of the compute type
  int sms = 0;        // multiprocessors of the device
  std::vector<int> nx, ny;
  std::vector<double> hx, hy;
  std::vector<fvh::ens::Problem> host;   // descriptors (host copy)
  fvh::ens::Problem* probs = nullptr;    // descriptors (device)
  int* prefix[fvh::ens::kVariants][4] = {};   // tile prefix sums per variant and phase (device)
  int ntiles[fvh::ens::kVariants][4] = {};
  std::vector<int> tiles_y[fvh::ens::kVariants][4];
  void* arena = nullptr;
  size_t arena_bytes = 0;
  fvh::ens::Barrier* bar = nullptr;
  unsigned int* active_count = nullptr;
  unsigned int wait_limit = 0;         // barrier polls before a wait gives up (0 = the default)
  int variant = 0;
  int blocks_per_sm = 0;               // 0 = as many as fit
  bool use_graph = true;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  cudaStream_t graph_stream = nullptr;  // stream the graph was captured on
  bool graph_failed = false;
  std::string graph_error;
  std::string err;
};

namespace fvh {
namespace ens {

// One stage launch (cooperative) of the ensemble kernel for the ensemble's
// precision, degree and current variant. Returns an FVH_ status.
int launch_stage_f64(fvh_ensemble* e, int stage, int last, cudaStream_t s);
int launch_stage_f32(fvh_ensemble* e, int stage, int last, cudaStream_t s);

// Resident blocks per SM of the kernel for (precision, degree, variant) and
// its dynamic shared memory; 0 when the variant does not fit.
int max_blocks_f64(int p, int variant, size_t* smem);
int max_blocks_f32(int p, int variant, size_t* smem);

}  // namespace ens
}  // namespace fvh
