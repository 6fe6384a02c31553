// Launch templates of the ensemble kernel, instantiated once per precision
// (fvh_ens_f64.cu with -fmad=false, fvh_ens_f32.cu with fast math).
#pragma once

#include <algorithm>

#include "fvh_ensemble_host.h"
#include "fvh_stage.cuh"

namespace fvh {
namespace ens {

// Resident blocks per SM on the current device, computed once per device (the
// first call sets the kernel's shared-memory limit; later calls, e.g. during a
// stream capture, only read the cache).
template <typename Tc, int P, int TX, int TY>
int max_blocks_t(size_t* smem) {
  using S = Smem<Tc, P, TX, TY>;
  *smem = (size_t)S::bytes;
  if (S::bytes > 227 * 1024) return 0;
  static int cache[64];  // blocks + 1 per device; 0 = not computed
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return 0;
  }
  if (cache[dev]) return cache[dev] - 1;
  auto kern = k_ens_stage<Tc, P, TX, TY>;
  if (cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, S::bytes) !=
      cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, 256, S::bytes) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  cache[dev] = blocks + 1;
  return blocks;
}

template <typename Tc, int P, int TX, int TY>
int launch_t(fvh_ensemble* e, int stage, int last, cudaStream_t s) {
  constexpr int R = (P + 1) / 2, RC = P / 2;
  constexpr int KC = 2 * RC + 1, KF = 2 * R + 1;
  size_t smem = 0;
  const int maxb = max_blocks_t<Tc, P, TX, TY>(&smem);
  if (maxb <= 0) {
    e->err = "ensemble tile variant does not fit on the device";
    return FVH_ERR_CONFIG;
  }
  const int bps = e->blocks_per_sm > 0 ? std::min(e->blocks_per_sm, maxb) : maxb;
  const fvh_config& cfg = e->cfg;
  Args<Tc, KC, KF> a{};
  a.probs = e->probs;
  a.nprob = e->nprob;
  for (int ph = 0; ph < 4; ++ph) {
    a.prefix[ph] = e->prefix[e->variant][ph];
    a.ntiles[ph] = e->ntiles[e->variant][ph];
  }
  a.stage = stage;
  a.last_stage = last;
  a.gW = e->gW;
  a.gw = e->gw;
  a.apost = cfg.a_posteriori ? 1 : 0;
  a.limiter = cfg.slope_limiter;
  a.use_fixed_dt = cfg.use_fixed_dt;
  a.fixed_dt = cfg.fixed_dt;
  a.crule = device_rule<Tc, KC>(centre_rule(P));
  a.trule = device_rule<Tc, KC>(transverse_rule(P));
  a.lrule = device_rule<Tc, KF>(left_face_rule(P));
  a.rrule = device_rule<Tc, KF>(right_face_rule(P));
  Phys<Tc> ph{};
  ph.gamma = (Tc)cfg.gamma;
  ph.gm1 = (Tc)(cfg.gamma - 1.0);
  ph.csq_floor = (Tc)cfg.csq_floor;
  ph.nv = 5;
  ph.riemann = cfg.riemann;
  ph.pad_ = 0;
  a.ph = ph;
  DetectSpec ds{};
  ds.nad_global = cfg.nad_global;
  ds.nad_relative = cfg.nad_relative;
  ds.nad_eps = cfg.nad_eps;
  ds.nad_var_mask = cfg.nad_var_mask;
  ds.sed = cfg.sed;
  ds.sed_eps = cfg.sed_eps;
  ds.pad_var = cfg.pad_var;
  ds.pad_lo = cfg.pad_lo;
  ds.pad_hi = cfg.pad_hi;
  ds.force_trouble = cfg.force_trouble;
  ds.log_mode = 0;
  a.ds = ds;
  a.bar = e->bar;
  a.wait_limit = e->wait_limit ? e->wait_limit : kDefaultWaitLimit;
  a.active_count = e->active_count;
  void* params[] = {&a};
  LaunchScope scope(KK_FINAL, 0.0, s);
  const cudaError_t err = cudaLaunchCooperativeKernel((const void*)k_ens_stage<Tc, P, TX, TY>,
                                                      dim3((unsigned)(bps * e->sms)), dim3(256), params, smem, s);
  if (err != cudaSuccess) {
    cudaGetLastError();
    e->err = std::string("ensemble stage launch: ") + cudaGetErrorString(err);
    return FVH_ERR_CUDA;
  }
  return FVH_OK;
}

// Dispatch over degree and variant.
template <typename Tc, int P>
int launch_p(fvh_ensemble* e, int stage, int last, cudaStream_t s) {
  switch (e->variant) {
    case 0: return launch_t<Tc, P, kVariantTX[0], kVariantTY[0]>(e, stage, last, s);
    case 1: return launch_t<Tc, P, kVariantTX[1], kVariantTY[1]>(e, stage, last, s);
    default: return launch_t<Tc, P, kVariantTX[2], kVariantTY[2]>(e, stage, last, s);
  }
}

template <typename Tc>
int launch_any(fvh_ensemble* e, int stage, int last, cudaStream_t s) {
  switch (e->p) {
    case 1: return launch_p<Tc, 1>(e, stage, last, s);
    case 2: return launch_p<Tc, 2>(e, stage, last, s);
    case 3: return launch_p<Tc, 3>(e, stage, last, s);
    case 4: return launch_p<Tc, 4>(e, stage, last, s);
    case 5: return launch_p<Tc, 5>(e, stage, last, s);
    case 6: return launch_p<Tc, 6>(e, stage, last, s);
    case 7: return launch_p<Tc, 7>(e, stage, last, s);
    case 8: return launch_p<Tc, 8>(e, stage, last, s);
  }
  e->err = "ensemble degree must be 1..8";
  return FVH_ERR_CONFIG;
}

template <typename Tc, int P>
int max_blocks_p(int variant, size_t* smem) {
  switch (variant) {
    case 0: return max_blocks_t<Tc, P, kVariantTX[0], kVariantTY[0]>(smem);
    case 1: return max_blocks_t<Tc, P, kVariantTX[1], kVariantTY[1]>(smem);
    default: return max_blocks_t<Tc, P, kVariantTX[2], kVariantTY[2]>(smem);
  }
}

template <typename Tc>
int max_blocks_any(int p, int variant, size_t* smem) {
  switch (p) {
    case 1: return max_blocks_p<Tc, 1>(variant, smem);
    case 2: return max_blocks_p<Tc, 2>(variant, smem);
    case 3: return max_blocks_p<Tc, 3>(variant, smem);
    case 4: return max_blocks_p<Tc, 4>(variant, smem);
    case 5: return max_blocks_p<Tc, 5>(variant, smem);
    case 6: return max_blocks_p<Tc, 6>(variant, smem);
    case 7: return max_blocks_p<Tc, 7>(variant, smem);
    case 8: return max_blocks_p<Tc, 8>(variant, smem);
  }
  return 0;
}

}  // namespace ens
}  // namespace fvh
