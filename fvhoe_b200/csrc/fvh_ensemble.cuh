// Batched ensemble of independent 2D problems: one persistent, cooperative
// launch per Runge-Kutta stage advances every active problem.
//
// The problems share every setting (degree, gamma, Riemann solver,
// boundaries, limiter, precision) except the grid. Each launch walks four
// phases over one work list of (problem, tile) entries:
//   1. primitives + CFL / extrema reductions   (tile2_primitives)
//   2. high-order fluxes + candidate u*          (tile2_fluxes)
//   3. a-posteriori detection                    (tile2_detect)
//   4. fallback, divergence, Runge-Kutta stage   (tile2_final)
// with a grid barrier between phases (each phase reads halos that other
// blocks wrote in the previous one) and one at the end, after which block 0
// resets the problems' reductions and, in the last stage, advances their times
// exactly as the single-problem stepper does (fvhoe/ode.py:11-22, 94-112):
// dt = min(CFL dt of stage 1, t_end - t), t += dt, active while t < t_end.
// Tiles of inactive problems are skipped. The tile functions are the ones of
// the one-problem fused path, so a problem advanced in the ensemble equals the
// same problem advanced alone, bit for bit in FP64.
//
// The barrier waits are bounded: a block that waits too long raises an abort
// flag that every block checks, and the host reports FVH_ERR_TIMEOUT. The
// launch is cooperative, so all blocks are resident and the barrier cannot
// deadlock on an unscheduled block.
#pragma once

#include "fvh_fused2d.cuh"

namespace fvh {
namespace ens {

// Per-problem descriptor (device memory).
struct Problem {
  f2::Geo g;
  double cx, cy;      // -1/h along X, Y
  double cfl_h;       // CFL * min(h)
  double t, t_end;    // time and target
  double dt_step;     // this step's dt (stage 1, clamped)
  int active;         // t < t_end
  int steps;          // steps taken
  double* u;          // state (5, nx, ny)
  double* s[2];       // stage inputs of stages 2.. (alternating)
  double* acc;        // Runge-Kutta accumulator
  double* us;         // candidate
  void* W;            // FV primitives, gW ghosts (compute type)
  void* F;            // X-face fluxes (5, nx+1, ny)
  void* G;            // Y-face fluxes (5, nx, ny+1)
  uint8_t* trouble;   // flags (nx, ny)
  Scalars* sc;        // stage reductions and counters
  int tiles_y[4];     // tiles along Y per phase (the fast tile index)
};

struct Barrier {
  unsigned int count;
  unsigned int gen;
  unsigned int abort;
  unsigned int timeouts;
};

template <typename Tc, int KC, int KF>
struct Args {
  Problem* probs;
  int nprob;
  const int* prefix[4];  // tile prefix sums per phase (nprob + 1 entries)
  int ntiles[4];
  int stage;             // 0, 1, 2 (SSP-RK3)
  int last_stage;
  int gW;                // ghost width of W
  int gw;                // ghost width of the flux pass (CFL box)
  int apost, limiter, use_fixed_dt;
  double fixed_dt;
  Rule<Tc, KC> crule, trule;
  Rule<Tc, KF> lrule, rrule;
  Phys<Tc> ph;
  DetectSpec ds;
  Barrier* bar;
  unsigned int wait_limit;  // polls a barrier wait makes before it gives up
  unsigned int* active_count;
};

// Default barrier wait bound: 2^24 polls (seconds with the back-off below).
constexpr unsigned int kDefaultWaitLimit = 1u << 24;

// Bounded grid barrier (all blocks resident: cooperative launch). Returns
// false when the wait gave up or another block aborted.
__device__ __forceinline__ bool grid_barrier(Barrier* b, unsigned int limit) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int* vgen = &b->gen;
    volatile unsigned int* vabort = &b->abort;
    const unsigned int g = *vgen;
    __threadfence();
    const unsigned int arrived = atomicAdd(&b->count, 1u) + 1u;
    int ok = 1;
    if (arrived == gridDim.x) {
      b->count = 0u;
      __threadfence();
      atomicAdd(&b->gen, 1u);
    } else {
      unsigned int i = 0;
      while (*vgen == g && *vabort == 0u && i < limit) {
        __nanosleep(64);
        ++i;
      }
      if (*vgen == g) {
        ok = 0;
        if (i >= limit) atomicAdd(&b->timeouts, 1u);
        atomicExch(&b->abort, 1u);
      }
    }
    __threadfence();
    s_ok = ok && (*vabort == 0u);
  }
  __syncthreads();
  return s_ok != 0;
}

// Problem owning global tile i of a phase (prefix has nprob + 1 entries).
__device__ __forceinline__ int find_problem(const int* __restrict__ prefix, int nprob, int i) {
  int lo = 0, hi = nprob;  // prefix[lo] <= i < prefix[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (prefix[mid] <= i)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

__device__ __forceinline__ const double* stage_input(const Problem* p, int stage) {
  return stage == 0 ? p->u : p->s[(stage - 1) & 1];
}

// Tile sizes: primitives always 16 x 32 outputs; fluxes / detection / final TX x TY.
constexpr int kPrimTX = 16, kPrimTY = 32;

template <typename Tc, int P, int TX, int TY>
struct Smem {
  static constexpr int R = (P + 1) / 2, RC = P / 2;
  using DP = f2::PrimsDims<Tc, P, kPrimTX, kPrimTY>;
  using DF = f2::FluxDims<P, TX, TY>;
  using DD = f2::PrimsDims<Tc, P, TX + 6, TY + 6>;
  using DE = f2::FinalDims<TX, TY>;
  static constexpr int prim = (DP::A + DP::B) * (int)sizeof(Tc);
  static constexpr int flux = DF::TOTAL * (int)sizeof(Tc);
  static constexpr int detect = (DD::A + DD::B) * (int)sizeof(Tc);
  static constexpr int fin = (DE::SP + DE::SF + DE::SG) * (int)sizeof(Tc) + DE::LIST;
  static constexpr int bytes = f2::Max<f2::Max<prim, flux>::value, f2::Max<detect, fin>::value>::value;
};

template <typename Tc, int P, int TX, int TY>
__global__ void __launch_bounds__(256)
    k_ens_stage(Args<Tc, 2 * (P / 2) + 1, 2 * ((P + 1) / 2) + 1> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int KC = 2 * (P / 2) + 1, KF = 2 * ((P + 1) / 2) + 1;
  const int stage = a.stage;
  // ---- phase 1: primitives over the gW-ghost box, CFL and extrema reductions
  for (int i = blockIdx.x; i < a.ntiles[0]; i += gridDim.x) {
    const int q = find_problem(a.prefix[0], a.nprob, i);
    const Problem* p = a.probs + q;
    if (!p->active) continue;
    const int li = i - a.prefix[0][q];
    const f2::Geo g = p->g;
    ReduceSpec rs{};
    rs.cfl = a.use_fixed_dt ? 0 : 1;
    rs.cfl_box = Region{{-a.gw, -a.gw, 0}, {g.nx + 2 * a.gw, g.ny + 2 * a.gw, 1}};
    rs.extrema = (a.apost && a.ds.nad_global) ? 1 : 0;
    rs.ext_box = Region{{-3, -3, 0}, {g.nx + 6, g.ny + 6, 1}};
    rs.ndim = 2.0;
    __syncthreads();  // the previous tile is done with shared memory
    f2::tile2_primitives<Tc, P, kPrimTX, kPrimTY, KC, true>(
        stage_input(p, stage), g, f2::make_v2((Tc*)p->W, g.nx, g.ny, a.gW), a.gW, a.crule, a.trule, a.ph, rs, p->sc,
        li % p->tiles_y[0], li / p->tiles_y[0], smem_raw);
  }
  if (!grid_barrier(a.bar, a.wait_limit)) return;
  // dt of the step (stage 1): the CFL dt clamped to the target
  if (stage == 0 && blockIdx.x == 0) {
    for (int q = threadIdx.x; q < a.nprob; q += blockDim.x) {
      Problem* p = a.probs + q;
      if (!p->active) continue;
      const double dt = a.use_fixed_dt ? a.fixed_dt : p->cfl_h / key_value(p->sc->cfl_key);
      p->dt_step = (p->t_end - p->t < dt) ? p->t_end - p->t : dt;
    }
  }
  // ---- phase 2: fluxes and the candidate
  for (int i = blockIdx.x; i < a.ntiles[1]; i += gridDim.x) {
    const int q = find_problem(a.prefix[1], a.nprob, i);
    const Problem* p = a.probs + q;
    if (!p->active) continue;
    const int li = i - a.prefix[1][q];
    const f2::Geo g = p->g;
    const double dt = a.use_fixed_dt ? a.fixed_dt : p->cfl_h / key_value(p->sc->cfl_key);
    const f2::V2<const Tc> Wc = f2::make_v2((const Tc*)p->W, g.nx, g.ny, a.gW);
    __syncthreads();
    f2::tile2_fluxes<Tc, P, TX, TY, KC, KF>(Wc, stage_input(p, stage), g, f2::make_v2((Tc*)p->F, g.nx + 1, g.ny, 0),
                                            f2::make_v2((Tc*)p->G, g.nx, g.ny + 1, 0), a.apost ? (Tc*)p->us : nullptr,
                                            a.crule, a.trule, a.lrule, a.rrule, a.ph, p->cx, p->cy, dt, nullptr, 1,
                                            a.limiter, li % p->tiles_y[1], li / p->tiles_y[1], smem_raw);
  }
  if (!grid_barrier(a.bar, a.wait_limit)) return;
  // ---- phase 3: a-posteriori detection
  if (a.apost) {
    for (int i = blockIdx.x; i < a.ntiles[2]; i += gridDim.x) {
      const int q = find_problem(a.prefix[2], a.nprob, i);
      const Problem* p = a.probs + q;
      if (!p->active) continue;
      const int li = i - a.prefix[2][q];
      const f2::Geo g = p->g;
      const f2::V2<const Tc> Wc = f2::make_v2((const Tc*)p->W, g.nx, g.ny, a.gW);
      __syncthreads();
      f2::tile2_detect<Tc, P, TX, TY, KC>((const Tc*)p->us, g, Wc, a.crule, a.trule, a.ph, a.ds, p->sc, p->trouble, nullptr,
                                          nullptr, nullptr, li % p->tiles_y[2], li / p->tiles_y[2], smem_raw);
    }
    if (!grid_barrier(a.bar, a.wait_limit)) return;
  }
  // ---- phase 4: fallback, divergence, Runge-Kutta combination
  for (int i = blockIdx.x; i < a.ntiles[3]; i += gridDim.x) {
    const int q = find_problem(a.prefix[3], a.nprob, i);
    const Problem* p = a.probs + q;
    if (!p->active) continue;
    const int li = i - a.prefix[3][q];
    const f2::Geo g = p->g;
    StageSpec st{};
    st.integrator = INT_SSPRK3;
    st.stage = stage;
    st.stage_in = stage_input(p, stage);
    st.u = p->u;
    st.acc = p->acc;
    st.next = p->s[stage & 1];
    const f2::V2<const Tc> Fc = f2::make_v2((const Tc*)p->F, g.nx + 1, g.ny, 0);
    const f2::V2<const Tc> Gc = f2::make_v2((const Tc*)p->G, g.nx, g.ny + 1, 0);
    __syncthreads();
    f2::tile2_final<Tc, TX, TY>(st.stage_in, g, Fc, Gc, p->trouble, nullptr, a.apost, 1, a.limiter, a.ph, p->cx, p->cy,
                                st, p->dt_step, p->sc, li % p->tiles_y[3], li / p->tiles_y[3], smem_raw);
  }
  if (!grid_barrier(a.bar, a.wait_limit)) return;
  // ---- end of stage: fresh reductions for the next stage; the last stage advances time
  if (blockIdx.x == 0) {
    unsigned int active = 0;
    for (int q = threadIdx.x; q < a.nprob; q += blockDim.x) {
      Problem* p = a.probs + q;
      Scalars* sc = p->sc;
      sc->cfl_key = 0ull;
      sc->troubled = 0u;
      for (int v = 0; v < 5; ++v) {
        sc->vmax_key[v] = 0ull;
        sc->vmin_key[v] = ~0ull;
      }
      if (a.last_stage && p->active) {
        p->t = p->t + p->dt_step;
        p->steps += 1;
        p->active = p->t < p->t_end ? 1 : 0;
      }
      active += p->active ? 1u : 0u;
    }
    if (a.last_stage) block_count_add(active, a.active_count);
  }
}

}  // namespace ens
}  // namespace fvh
