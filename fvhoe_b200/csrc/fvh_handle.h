// Solver handle shared by the C ABI (fvh_api.cu) and the per-precision stage
// runners (fvh_stage_f64.cu, fvh_stage_f32.cu).
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "fvh.h"
#include "fvh_kernels.cuh"
#include "fvh_profile.h"

struct fvh_handle {
  fvh_config cfg;
  int nv = 5;
  int n[3] = {1, 1, 1};
  int p[3] = {0, 0, 0};
  int r[3] = {0, 0, 0};           // stencil radius ceil(p/2) per axis
  bool active[3] = {false, false, false};
  int ndim = 0;
  int gw = 0;                     // ghost width of the high-order flux pass
  int gW = 0;                     // ghost width of the primitive array W
  double cfl_h = 0.0;             // CFL * min(h)
  double neg_inv_h[3] = {0, 0, 0};
  fvh::Grid grid{};
  size_t elem = 8;                // bytes of the compute type

  // device memory owned by the handle
  void* bufA = nullptr;           // sweep scratch (ping)
  void* bufB = nullptr;           // sweep scratch (pong)
  size_t buf_elems = 0;
  void* W = nullptr;              // FV primitives of the stage input, gW ghosts
  void* Ws = nullptr;             // FV primitives of the candidate, 3 ghosts
  double* Us = nullptr;           // candidate state
  void* F[3] = {nullptr, nullptr, nullptr};      // face fluxes per axis
  float* theta[3] = {nullptr, nullptr, nullptr}; // convex face weights per axis
  float* conv = nullptr;                          // convex work arrays (3 padded boxes)
  uint8_t* trouble = nullptr;
  double* logs[3] = {nullptr, nullptr, nullptr};  // running trouble / NAD / PAD sums
  double* acc = nullptr;          // running k-sum of ssprk3 / rk4
  double* S[2] = {nullptr, nullptr};              // stage inputs
  fvh::Scalars* sc = nullptr;
  double* slab[3][2] = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};  // Dirichlet ghost values
  size_t slab_count[3][2] = {{0, 0}, {0, 0}, {0, 0}};
  fvh::Slabs slab_meta{};                 // host copy of the descriptor
  fvh::Slabs* slabs_dev = nullptr;        // device copy (grid.slabs points here)
  size_t scratch_bytes = 0;

  // learned troubled-cell predictor (optional)
  fvh_mlp* mlp = nullptr;         // attached network (not owned)
  uint8_t* pred = nullptr;        // predicted flags of the last prediction
  float pred_thr_logit = 0.0f;    // logit threshold
  int pred_interval = 1;          // stages between predictions (flags reused in between)
  long long pred_stage = 0;       // fused stages run since the predictor was attached
  bool last_stage_fused = false;  // the last stage ran the fused 2D kernels

  // host-resident state (fvh_step_host): device copy, two copy streams and
  // the per-chunk events that let one call's copy-in follow the previous
  // call's copy-out chunk by chunk
  static constexpr int kHostChunks = 16;
  double* host_state = nullptr;   // device copy of the host state
  cudaStream_t copy_in = nullptr, copy_out = nullptr;
  cudaEvent_t out_done[kHostChunks] = {};  // copy-out of chunk j finished
  cudaEvent_t in_done = nullptr, step_done = nullptr;
  bool out_pending = false;       // out_done events recorded by an earlier call
  int log_mode_next = 1;          // log mode of the next stage
  int next_stage = 0;             // fvh_stage: the stage the next call must run (0 = a new step)
  int stage_integrator = -1;      // fvh_stage: integrator and state of the step in progress
  const double* stage_state = nullptr;
  double log_divisor = 0.0;       // divisor applied by the next step's last stage (one-shot)
  fvh::Profiler* prof = nullptr;  // per-launch timing, when enabled
  fvh::KernelTotals prof_totals{};
  std::string err;
};

namespace fvh {

// Layout of the fused 2D path's primitive arrays (W with g = gW ghosts, W*
// with g = 3) on the handle's two active axes X (outer) and Y (inner): rows
// padded so that Y index 0 and the row stride fall on 16-byte boundaries
// (f2::make_v2_aligned computes the same numbers on the device side).
struct WLayout {
  int g, gy, sx, vs;
  size_t elems;  // per variable
};

inline WLayout fused_w_layout(const fvh_handle* h, int g) {
  int ax[3], na = 0;
  for (int a = 0; a < 3; ++a)
    if (h->active[a]) ax[na++] = a;
  const int nx = na == 2 ? h->n[ax[0]] : 1, ny = na == 2 ? h->n[ax[1]] : 1;
  const int al = 16 / (int)h->elem;
  WLayout l;
  l.g = g;
  l.gy = (g + al - 1) / al * al;
  l.sx = (l.gy + ny + g + al - 1) / al * al;
  l.vs = (nx + 2 * g) * l.sx;
  l.elems = (size_t)l.vs;
  return l;
}

struct StageCall {
  const double* stage_in;  // input state of this stage
  StageSpec spec;          // Runge-Kutta epilogue
  int first_stage;         // fixes the step's dt
  int has_target;
  double t;
  double target;
  int log_mode;            // 0 none, 1 overwrite, 2 add
  double log_div;          // > 0: divide the trouble-log sums by it after this stage
};

// Runs one stage on the stream; returns an FVH_ status.
int run_stage_f64(fvh_handle* h, const StageCall& c, cudaStream_t s);
int run_stage_f32(fvh_handle* h, const StageCall& c, cudaStream_t s);

// FV primitives of u over the interior (snapshot conversion).
int primitives_f64(fvh_handle* h, const double* u, double* w, int fv_average, cudaStream_t s);

// Predicted flags h->pred of the stage from h->W (fused 2D layout, after the
// primitive pass and its extrema reduction).
int mlp_predict_stage(fvh_handle* h, cudaStream_t s);

// Adds the stage's predicted / troubled / missed / false-alarm counts to the
// step's predictor statistics (after the detection).
int mlp_count_stage(fvh_handle* h, cudaStream_t s);

}  // namespace fvh
