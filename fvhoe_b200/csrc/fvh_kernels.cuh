// Kernels of the per-stage update (generic N-D path).
//
// Every array is stored variable-major over an index box ("Region") in cell
// coordinates: element (v, i0, i1, i2) of a box with origin lo and extents n
// sits at ((v*n0 + i0-lo0)*n1 + i1-lo1)*n2 + i2-lo2. Axes are x, y, z in the
// reference's order (z contiguous); an inactive axis has extent 1.
//
// The stage is a sequence of passes, each a single launch over one box:
//   centre sweeps (the first one reads the conserved state through the
//   boundary index maps; the last one converts to primitives),
//   transverse sweeps (the last one also reduces the CFL speed and the
//   per-variable extrema), face reconstruction + Riemann solve, transverse
//   sweeps of the fluxes, the candidate update, troubled-cell detection,
//   the MUSCL fallback at troubled faces, and the flux divergence fused with
//   the Runge-Kutta stage combination.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "fvh_physics.cuh"

namespace fvh {

enum Bc : int { BC_PERIODIC = 0, BC_OUTFLOW = 1, BC_REFLECTIVE = 2, BC_FREE = 3 };

struct Region {
  int lo[3];
  int n[3];
};

struct Grid {
  int n[3];      // interior cells per axis
  int bc[3][2];  // Bc kinds at the low/high end of each axis
};

template <typename T, int K>
struct Rule {
  T w[K];
  int off;  // out[i] = sum_k w[k] * in[i + off + k]
};

__host__ __device__ __forceinline__ int64_t region_points(const Region& r) {
  return (int64_t)r.n[0] * r.n[1] * r.n[2];
}

__device__ __forceinline__ int64_t region_index(const Region& r, int v, int i0, int i1, int i2) {
  return (((int64_t)v * r.n[0] + (i0 - r.lo[0])) * r.n[1] + (i1 - r.lo[1])) * r.n[2] + (i2 - r.lo[2]);
}

__device__ __forceinline__ void region_point(const Region& r, int64_t idx, int& i0, int& i1, int& i2) {
  const int64_t q = idx / r.n[2];
  i2 = (int)(idx - q * r.n[2]) + r.lo[2];
  const int64_t q2 = q / r.n[1];
  i1 = (int)(q - q2 * r.n[1]) + r.lo[1];
  i0 = (int)q2 + r.lo[0];
}

// Ghost-cell source index along one axis (fvhoe/boundary_conditions.py:60-151):
// periodic copies the opposite interior, outflow and reflective mirror,
// free repeats the edge cell; `flip` reports a reflective mirror.
__device__ __forceinline__ int ghost_source(int i, int n, int lo_kind, int hi_kind, bool& flip) {
  if (i < 0) {
    if (lo_kind == BC_PERIODIC) return i + n;
    if (lo_kind == BC_FREE) return 0;
    flip = (lo_kind == BC_REFLECTIVE);
    return -1 - i;
  }
  if (i >= n) {
    if (hi_kind == BC_PERIODIC) return i - n;
    if (hi_kind == BC_FREE) return n - 1;
    flip = (hi_kind == BC_REFLECTIVE);
    return 2 * n - 1 - i;
  }
  return i;
}

// Reads all nv conserved variables at a (possibly ghost) cell. Reflective
// ghosts negate the momentum normal to the wall they mirror across.
template <typename Tc>
__device__ __forceinline__ void load_state(const double* __restrict__ u, const Grid& g, int nv, int i0, int i1,
                                           int i2, Tc* out) {
  bool f0 = false, f1 = false, f2 = false;
  const int j0 = ghost_source(i0, g.n[0], g.bc[0][0], g.bc[0][1], f0);
  const int j1 = ghost_source(i1, g.n[1], g.bc[1][0], g.bc[1][1], f1);
  const int j2 = ghost_source(i2, g.n[2], g.bc[2][0], g.bc[2][1], f2);
  const int64_t plane = (int64_t)g.n[0] * g.n[1] * g.n[2];
  const int64_t base = ((int64_t)j0 * g.n[1] + j1) * g.n[2] + j2;
  for (int v = 0; v < nv; ++v) {
    double x = u[v * plane + base];
    if ((v == 1 && f0) || (v == 2 && f1) || (v == 3 && f2)) x = -x;
    out[v] = (Tc)x;
  }
}

__device__ __forceinline__ void step_axis(int axis, int k, int& i0, int& i1, int& i2) {
  if (axis == 0) i0 += k;
  else if (axis == 1) i1 += k;
  else i2 += k;
}

// Kernels take the variable count NV as a template argument: NV = 5 keeps the
// per-point state in registers; NV = 0 means "known only at run time"
// (passive scalars), with arrays of kMaxVars and loops bounded by ph.nv.
template <int NV>
struct VarCount {
  static constexpr int kArray = NV > 0 ? NV : kMaxVars;
  template <typename T>
  __device__ __forceinline__ static int get(const Phys<T>& ph) {
    return NV > 0 ? NV : ph.nv;
  }
};

// ---------------------------------------------------------------------------
// Order-preserving 64-bit keys for atomic max/min of doubles.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long order_key(double x) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(x);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__host__ __device__ __forceinline__ double key_value(unsigned long long k) {
  const unsigned long long b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)b);
#else
  double d;
  __builtin_memcpy(&d, &b, sizeof(d));
  return d;
#endif
}

// Device-resident scalars of one stage.
struct Scalars {
  unsigned long long cfl_key;             // max CFL speed (order key)
  unsigned long long vmax_key[kMaxVars];  // per-variable extrema of w over the 3-ghost box
  unsigned long long vmin_key[kMaxVars];
  double dt_stage;                        // this stage's dt (CFL or fixed), used by the candidate
  double dt_step;                         // the step's dt after the target clamp
  unsigned int troubled;                  // troubled cells found this stage
  unsigned int nonfinite;                 // cells whose update is not finite
  unsigned int pad_[2];
};

// Reduction request for the last transverse sweep of the primitive pass.
struct ReduceSpec {
  int cfl;          // reduce the CFL speed over cfl_box
  Region cfl_box;
  int extrema;      // reduce per-variable max/min over ext_box
  Region ext_box;
  double ndim;      // number of active axes, as in ndim * c
};

template <typename T>
__device__ __forceinline__ bool in_box(const Region& r, int i0, int i1, int i2) {
  return i0 >= r.lo[0] && i0 < r.lo[0] + r.n[0] && i1 >= r.lo[1] && i1 < r.lo[1] + r.n[1] && i2 >= r.lo[2] &&
         i2 < r.lo[2] + r.n[2];
}

__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long x) {
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long y = __shfl_xor_sync(0xffffffffu, x, o);
    x = y > x ? y : x;
  }
  return x;
}
__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long x) {
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long y = __shfl_xor_sync(0xffffffffu, x, o);
    x = y < x ? y : x;
  }
  return x;
}

// ---------------------------------------------------------------------------
// Centre-interpolation sweep (fvhoe/fv.py:106-159, 175-197). FROM_STATE reads
// the conserved state through the ghost maps; TO_PRIMS converts the swept
// cell-centre values to primitives (fvhoe/hydro.py:146-170).
// ---------------------------------------------------------------------------
template <typename Tc, typename Tin, int NV, int K, bool FROM_STATE, bool TO_PRIMS>
__global__ void __launch_bounds__(256) k_centre_sweep(const Tin* __restrict__ in, Region rin, Tc* __restrict__ out,
                                                      Region rout, int axis, Rule<Tc, K> rule, Grid grid,
                                                      Phys<Tc> ph) {
  constexpr int NVA = VarCount<NV>::kArray;
  const int nv = VarCount<NV>::get(ph);
  const int64_t npts = region_points(rout);
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < npts;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int i0, i1, i2;
    region_point(rout, idx, i0, i1, i2);
    Tc acc[NVA];
    for (int v = 0; v < nv; ++v) acc[v] = Tc(0);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      int j0 = i0, j1 = i1, j2 = i2;
      step_axis(axis, rule.off + k, j0, j1, j2);
      Tc x[NVA];
      if constexpr (FROM_STATE) {
        load_state<Tc>(reinterpret_cast<const double*>(in), grid, nv, j0, j1, j2, x);
      } else {
        for (int v = 0; v < nv; ++v) x[v] = (Tc)in[region_index(rin, v, j0, j1, j2)];
      }
      for (int v = 0; v < nv; ++v) acc[v] = acc[v] + rule.w[k] * x[v];
    }
    if constexpr (TO_PRIMS) {
      Tc w[NVA];
      to_primitives(ph, nv, acc, w);
      for (int v = 0; v < nv; ++v) out[region_index(rout, v, i0, i1, i2)] = w[v];
    } else {
      for (int v = 0; v < nv; ++v) out[region_index(rout, v, i0, i1, i2)] = acc[v];
    }
  }
}

// ---------------------------------------------------------------------------
// Transverse-reconstruction sweep (fvhoe/fv.py:162-172, 200-224), optionally
// reducing the CFL speed (fvhoe/hydro.py:270-294) and the per-variable extrema
// used by global NAD (fvhoe/slope_limiting.py:165-170, 184-185).
// ---------------------------------------------------------------------------
template <typename Tc, int NV, int K, bool REDUCE>
__global__ void __launch_bounds__(256) k_transverse_sweep(const Tc* __restrict__ in, Region rin, Tc* __restrict__ out,
                                                          Region rout, int axis, Rule<Tc, K> rule, Phys<Tc> ph,
                                                          ReduceSpec rs, Scalars* __restrict__ sc) {
  constexpr int NVA = VarCount<NV>::kArray;
  const int nv = VarCount<NV>::get(ph);
  const int64_t npts = region_points(rout);
  unsigned long long cfl_key = 0ull;
  unsigned long long kmax[5], kmin[5];
  if constexpr (REDUCE) {
    for (int v = 0; v < 5; ++v) {
      kmax[v] = 0ull;
      kmin[v] = ~0ull;
    }
  }
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < npts;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int i0, i1, i2;
    region_point(rout, idx, i0, i1, i2);
    Tc acc[NVA];
    for (int v = 0; v < nv; ++v) acc[v] = Tc(0);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      int j0 = i0, j1 = i1, j2 = i2;
      step_axis(axis, rule.off + k, j0, j1, j2);
      for (int v = 0; v < nv; ++v) acc[v] = acc[v] + rule.w[k] * in[region_index(rin, v, j0, j1, j2)];
    }
    for (int v = 0; v < nv; ++v) out[region_index(rout, v, i0, i1, i2)] = acc[v];
    if constexpr (REDUCE) {
      if (rs.cfl && in_box<Tc>(rs.cfl_box, i0, i1, i2)) {
        const unsigned long long k = order_key((double)cfl_speed(ph, acc, (Tc)rs.ndim));
        cfl_key = k > cfl_key ? k : cfl_key;
      }
      if (rs.extrema && in_box<Tc>(rs.ext_box, i0, i1, i2)) {
        for (int v = 0; v < 5; ++v) {
          const unsigned long long k = order_key((double)acc[v]);
          kmax[v] = k > kmax[v] ? k : kmax[v];
          kmin[v] = k < kmin[v] ? k : kmin[v];
        }
      }
    }
  }
  if constexpr (REDUCE) {
    // warp, then block reduction in shared memory: one atomic per key and block
    __shared__ unsigned long long s_keys[8][11];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned long long c = warp_max_u64(cfl_key);
    if (lane == 0) s_keys[warp][0] = c;
    for (int v = 0; v < 5; ++v) {
      const unsigned long long a = warp_max_u64(kmax[v]);
      const unsigned long long b = warp_min_u64(kmin[v]);
      if (lane == 0) {
        s_keys[warp][1 + v] = a;
        s_keys[warp][6 + v] = b;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const int nw = blockDim.x >> 5;
      unsigned long long acc[11];
      for (int k = 0; k < 11; ++k) acc[k] = s_keys[0][k];
      for (int w = 1; w < nw; ++w) {
        for (int k = 0; k < 6; ++k) acc[k] = s_keys[w][k] > acc[k] ? s_keys[w][k] : acc[k];
        for (int k = 6; k < 11; ++k) acc[k] = s_keys[w][k] < acc[k] ? s_keys[w][k] : acc[k];
      }
      if (rs.cfl && acc[0]) atomicMax(&sc->cfl_key, acc[0]);
      if (rs.extrema) {
        for (int v = 0; v < 5; ++v) {
          if (acc[1 + v]) atomicMax(&sc->vmax_key[v], acc[1 + v]);
          if (acc[6 + v] != ~0ull) atomicMin(&sc->vmin_key[v], acc[6 + v]);
        }
      }
    }
  }
}

// Block-wide sum of a per-thread count with one atomic per block (blocks of
// at most 256 threads).
__device__ __forceinline__ void block_count_add(unsigned int count, unsigned int* dst) {
  __shared__ unsigned int s_count[8];
  for (int o = 16; o > 0; o >>= 1) count += __shfl_xor_sync(0xffffffffu, count, o);
  if ((threadIdx.x & 31) == 0) s_count[threadIdx.x >> 5] = count;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int total = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) total += s_count[w];
    if (total) atomicAdd(dst, total);
  }
}

// ---------------------------------------------------------------------------
// Face reconstruction along d and the Riemann solve (fvhoe/solver.py:522-607):
// face j lies between cells j-1 and j; the left state is cell j-1's right-face
// value, the right state is cell j's left-face value.
// ---------------------------------------------------------------------------
template <typename Tc, int NV, int K>
__global__ void __launch_bounds__(256) k_face_riemann(const Tc* __restrict__ in, Region rin, Tc* __restrict__ out,
                                                      Region rout, int d, Rule<Tc, K> left_rule,
                                                      Rule<Tc, K> right_rule, Phys<Tc> ph) {
  constexpr int NVA = VarCount<NV>::kArray;
  const int nv = VarCount<NV>::get(ph);
  const int64_t npts = region_points(rout);
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < npts;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int i0, i1, i2;
    region_point(rout, idx, i0, i1, i2);
    Tc wl[NVA], wr[NVA];
    for (int v = 0; v < nv; ++v) {
      wl[v] = Tc(0);
      wr[v] = Tc(0);
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
      int a0 = i0, a1 = i1, a2 = i2;
      step_axis(d, right_rule.off + k - 1, a0, a1, a2);  // cell j-1, right-face rule
      int b0 = i0, b1 = i1, b2 = i2;
      step_axis(d, left_rule.off + k, b0, b1, b2);  // cell j, left-face rule
      for (int v = 0; v < nv; ++v) {
        wl[v] = wl[v] + right_rule.w[k] * in[region_index(rin, v, a0, a1, a2)];
        wr[v] = wr[v] + left_rule.w[k] * in[region_index(rin, v, b0, b1, b2)];
      }
    }
    Tc f[NVA];
    riemann_flux<NVA>(ph, nv, wl, wr, d, f);
    for (int v = 0; v < nv; ++v) out[region_index(rout, v, i0, i1, i2)] = f[v];
  }
}

// ---------------------------------------------------------------------------
// Flux divergence, fvhoe/solver.py:734-751:
//   dudt = 0.0 + -(1/hx)(F[i+1]-F[i]) + -(1/hy)(G[j+1]-G[j]) + -(1/hz)(H[k+1]-H[k])
// ---------------------------------------------------------------------------
struct FluxSet {
  const void* f[3];  // per-axis face fluxes (nullptr for inactive axes)
  Region r[3];
  double neg_inv_h[3];  // -(1/h_d), rounded on the host as Python does
};

template <typename Tc>
__device__ __forceinline__ void divergence(const FluxSet& fs, int nv, int i0, int i1, int i2, Tc* dudt) {
  for (int v = 0; v < nv; ++v) dudt[v] = Tc(0);
  for (int d = 0; d < 3; ++d) {
    if (!fs.f[d]) continue;
    const Tc* F = reinterpret_cast<const Tc*>(fs.f[d]);
    int a0 = i0, a1 = i1, a2 = i2;
    step_axis(d, 1, a0, a1, a2);
    const Tc c = (Tc)fs.neg_inv_h[d];
    for (int v = 0; v < nv; ++v) {
      const Tc hi = (Tc)F[region_index(fs.r[d], v, a0, a1, a2)];
      const Tc lo = (Tc)F[region_index(fs.r[d], v, i0, i1, i2)];
      dudt[v] = dudt[v] + c * (hi - lo);
    }
  }
}

// Candidate state u* = u + dt L(F) (fvhoe/solver.py:677-678).
template <typename Tc, int NV>
__global__ void __launch_bounds__(256) k_candidate(const double* __restrict__ u, Region rint, FluxSet fs,
                                                   double* __restrict__ ustar, Phys<Tc> ph,
                                                   const Scalars* __restrict__ sc) {
  constexpr int NVA = VarCount<NV>::kArray;
  const int nv = VarCount<NV>::get(ph);
  const int64_t npts = region_points(rint);
  const double dt = sc->dt_stage;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < npts;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int i0, i1, i2;
    region_point(rint, idx, i0, i1, i2);
    Tc dudt[NVA];
    divergence<Tc>(fs, nv, i0, i1, i2, dudt);
    for (int v = 0; v < nv; ++v) {
      const int64_t o = region_index(rint, v, i0, i1, i2);
      ustar[o] = u[o] + dt * (double)dudt[v];
    }
  }
}

// ---------------------------------------------------------------------------
// Troubled-cell detection (fvhoe/slope_limiting.py:87-244).
// ---------------------------------------------------------------------------
struct DetectSpec {
  int nad_global;    // 1: range from the global extrema, 0: local box range
  int nad_relative;  // 1: relative tolerance, 0: absolute
  double nad_eps;
  int nad_var_mask;  // bit v set: variable v counts towards NAD
  int sed;
  double sed_eps;
  int pad_var;  // -1 when PAD is off; otherwise the primitive index of the last PAD key
  double pad_lo, pad_hi;
  int force_trouble;
  int active[3];
  int log_mode;  // 0: no logging, 1: overwrite the running sums, 2: add to them
};

template <typename Tc>
__global__ void __launch_bounds__(256) k_detect(const Tc* __restrict__ w, Region rw, const Tc* __restrict__ ws,
                                                Region rws, Region rint, DetectSpec ds, Scalars* __restrict__ sc,
                                                uint8_t* __restrict__ trouble, double* __restrict__ log_trouble,
                                                double* __restrict__ log_nad, double* __restrict__ log_pad) {
  const int64_t npts = region_points(rint);
  unsigned int count = 0;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < npts;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int i0, i1, i2;
    region_point(rint, idx, i0, i1, i2);
    const int r0 = ds.active[0], r1 = ds.active[1], r2 = ds.active[2];
    bool nad_any = false;
    Tc ind_min = Tc(0);
    Tc pad_ind = Tc(0);
    for (int v = 0; v < 5; ++v) {
      // 3^d box extrema of w (fvhoe/slope_limiting.py:145-162)
      Tc big = w[region_index(rw, v, i0, i1, i2)], small = big;
      for (int a = -r0; a <= r0; ++a)
        for (int b = -r1; b <= r1; ++b)
          for (int c = -r2; c <= r2; ++c) {
            const Tc x = w[region_index(rw, v, i0 + a, i1 + b, i2 + c)];
            big = np_maximum(big, x);
            small = np_minimum(small, x);
          }
      const Tc xs = ws[region_index(rws, v, i0, i1, i2)];
      Tc ind;
      bool tv;
      if (ds.nad_relative) {
        Tc range;
        if (ds.nad_global) {
          range = (Tc)(key_value(sc->vmax_key[v]) - key_value(sc->vmin_key[v]));
        } else {
          range = big - small;
        }
        ind = xs - small;
        ind = np_minimum(ind, big - xs);
        tv = ind < (Tc)(-ds.nad_eps) * range;
      } else {
        Tc lower, upper;
        if (ds.nad_global) {
          lower = (Tc)((1.0 - ds.nad_eps) * key_value(sc->vmin_key[v]));
          upper = (Tc)((1.0 + ds.nad_eps) * key_value(sc->vmax_key[v]));
        } else {
          lower = (Tc)(1.0 - ds.nad_eps) * small;
          upper = (Tc)(1.0 + ds.nad_eps) * big;
        }
        ind = np_minimum(xs - lower, upper - xs);
        tv = ind < Tc(0);
      }
      if (tv && ds.sed) {
        // smooth-extrema detector on w* (fvhoe/smooth_extrema_detection.py:8-95)
        Tc alpha = Tc(0);
        bool first = true;
        for (int a = 0; a < 3; ++a) {
          if (!ds.active[a]) continue;
          Tc line[7];
#pragma unroll
          for (int k = 0; k < 7; ++k) {
            int j0 = i0, j1 = i1, j2 = i2;
            step_axis(a, k - 3, j0, j1, j2);
            line[k] = ws[region_index(rws, v, j0, j1, j2)];
          }
          const Tc al = sed_alpha_line(line, (Tc)ds.sed_eps);
          alpha = first ? al : np_minimum(alpha, al);
          first = false;
        }
        tv = alpha < Tc(1);
      }
      if (!((ds.nad_var_mask >> v) & 1)) tv = false;
      nad_any = nad_any || tv;
      ind_min = (v == 0) ? ind : np_minimum(ind_min, ind);
      if (v == ds.pad_var) {
        pad_ind = xs - (Tc)ds.pad_lo;
        pad_ind = np_minimum(pad_ind, (Tc)ds.pad_hi - xs);
      }
    }
    const bool pad_trouble = pad_ind < Tc(0);
    bool t = pad_trouble || nad_any;
    if (ds.force_trouble) t = true;
    const int64_t o = region_index(rint, 0, i0, i1, i2);
    trouble[o] = t ? 1 : 0;
    count += t ? 1u : 0u;
    if (ds.log_mode) {
      const double lt = t ? 1.0 : 0.0;
      const double ln = nad_any ? -(double)ind_min : 0.0;
      const double lp = pad_trouble ? -(double)pad_ind : 0.0;
      if (ds.log_mode == 1) {
        log_trouble[o] = lt;
        log_nad[o] = ln;
        log_pad[o] = lp;
      } else {
        log_trouble[o] = log_trouble[o] + lt;
        log_nad[o] = log_nad[o] + ln;
        log_pad[o] = log_pad[o] + lp;
      }
    }
  }
  block_count_add(count, &sc->troubled);
}

// ---------------------------------------------------------------------------
// MUSCL fallback at troubled faces and the flux blend
// (fvhoe/solver.py:710-731, fvhoe/slope_limiting.py:24-84, 247-384).
// theta of face j = max(trouble[j-1], trouble[j]) with missing neighbours 0,
// or the convex weights when theta_in is given.
// ---------------------------------------------------------------------------
struct FallbackSpec {
  int d;             // face-normal axis
  int muscl;         // 1: slope-limited p=1 reconstruction along d, 0: first order
  int limiter;       // Limiter enum
  Region rflux;      // region of F_d
  Region rint;       // interior region
};

template <typename Tc, int NV>
__global__ void __launch_bounds__(256) k_fallback(const double* __restrict__ u, Grid grid, Tc* __restrict__ F,
                                                  const uint8_t* __restrict__ trouble, const float* __restrict__ theta_in,
                                                  FallbackSpec fb, Phys<Tc> ph) {
  constexpr int NVA = VarCount<NV>::kArray;
  const int nv = VarCount<NV>::get(ph);
  const int64_t npts = region_points(fb.rflux);
  const int d = fb.d;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < npts;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int i0, i1, i2;
    region_point(fb.rflux, idx, i0, i1, i2);
    Tc theta;
    if (theta_in) {
      theta = (Tc)theta_in[idx];
    } else {
      const int j = d == 0 ? i0 : (d == 1 ? i1 : i2);
      const int nd = grid.n[d];
      int a0 = i0, a1 = i1, a2 = i2;
      step_axis(d, -1, a0, a1, a2);
      const uint8_t tl = j >= 1 ? trouble[region_index(fb.rint, 0, a0, a1, a2)] : 0;
      const uint8_t tr = j < nd ? trouble[region_index(fb.rint, 0, i0, i1, i2)] : 0;
      theta = (tl || tr) ? Tc(1) : Tc(0);
    }
    if (!(theta > Tc(0))) continue;
    // primitives at cells j-2 .. j+1 along d (p=1 centre/transverse rules are identities)
    Tc w[4][NVA];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      int a0 = i0, a1 = i1, a2 = i2;
      step_axis(d, c - 2, a0, a1, a2);
      Tc uc[NVA];
      load_state<Tc>(u, grid, nv, a0, a1, a2, uc);
      to_primitives(ph, nv, uc, w[c]);
    }
    Tc wl[NVA], wr[NVA];
    for (int v = 0; v < nv; ++v) {
      if (fb.muscl && fb.limiter == LIMITER_NONE) {
        // unlimited p=1 face rules [1/4, 1, -1/4] and its mirror (fvhoe/stencils.py:44-46)
        wl[v] = ((Tc(0) + Tc(-0.25) * w[0][v]) + Tc(1) * w[1][v]) + Tc(0.25) * w[2][v];
        wr[v] = ((Tc(0) + Tc(0.25) * w[1][v]) + Tc(1) * w[2][v]) + Tc(-0.25) * w[3][v];
      } else if (fb.muscl) {
        const Tc sl = limited_slope(w[1][v] - w[0][v], w[2][v] - w[1][v], fb.limiter);
        const Tc sr = limited_slope(w[2][v] - w[1][v], w[3][v] - w[2][v], fb.limiter);
        wl[v] = w[1][v] + Tc(0.5) * sl;
        wr[v] = w[2][v] - Tc(0.5) * sr;
      } else {
        wl[v] = w[1][v];
        wr[v] = w[2][v];
      }
    }
    Tc flo[NVA];
    riemann_flux<NVA>(ph, nv, wl, wr, d, flo);
    for (int v = 0; v < nv; ++v) {
      const int64_t o = region_index(fb.rflux, v, i0, i1, i2);
      F[o] = (Tc(1) - theta) * F[o] + theta * flo[v];
    }
  }
}

// ---------------------------------------------------------------------------
// Flux divergence fused with the Runge-Kutta stage combination
// (fvhoe/ode.py:11-22, 245-298). Every term keeps the reference's association:
//   euler   s0: u = u + dt k
//   ssprk2  s0: s = u + dt k ;            s1: u = 0.5 u + 0.5 (s + dt k)
//   ssprk3  s0: a = k, s = u + dt k ;     s1: s' = (u + (0.25 dt) a) + (0.25 dt) k, a = a + k
//           s2: u = u + ((1/6) dt)(a + 4 k)
//   rk4     s0: a = k, s = u + (0.5 dt) k ; s1: a = a + 2k, s' = u + (0.5 dt) k
//           s2: a = a + 2k, s'' = u + dt k ; s3: u = u + ((1/6) dt)(a + k)
// Stage 0 also fixes the step's dt: min(dt_stage, target - t) when a target is
// set and closer than dt (fvhoe/ode.py:11-22).
// ---------------------------------------------------------------------------
enum Integrator : int { INT_EULER = 0, INT_SSPRK2 = 1, INT_SSPRK3 = 2, INT_RK4 = 3, INT_RHS = 4 };

struct StageSpec {
  int integrator;
  int stage;
  const double* stage_in;  // this stage's input state (u for stage 0)
  double* u;               // the solution, updated in place by the last stage
  double* acc;             // running k-sum (ssprk3 / rk4)
  double* next;            // next stage's input
  double* dudt_out;        // INT_RHS: dudt destination
};

template <typename Tc, int NV>
__global__ void __launch_bounds__(256) k_final(Region rint, FluxSet fs, Phys<Tc> ph, StageSpec st,
                                               Scalars* __restrict__ sc) {
  constexpr int NVA = VarCount<NV>::kArray;
  const int nv = VarCount<NV>::get(ph);
  const int64_t npts = region_points(rint);
  const double dt = sc->dt_step;
  unsigned int bad = 0;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < npts;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int i0, i1, i2;
    region_point(rint, idx, i0, i1, i2);
    Tc dudt_c[NVA];
    divergence<Tc>(fs, nv, i0, i1, i2, dudt_c);
    for (int v = 0; v < nv; ++v) {
      const int64_t o = region_index(rint, v, i0, i1, i2);
      const double k = (double)dudt_c[v];
      double res = 0.0;
      switch (st.integrator) {
        case INT_RHS:
          st.dudt_out[o] = k;
          res = k;
          break;
        case INT_EULER:
          res = st.u[o] + dt * k;
          st.u[o] = res;
          break;
        case INT_SSPRK2:
          if (st.stage == 0) {
            res = st.u[o] + dt * k;
            st.next[o] = res;
          } else {
            res = 0.5 * st.u[o] + 0.5 * (st.stage_in[o] + dt * k);
            st.u[o] = res;
          }
          break;
        case INT_SSPRK3:
          if (st.stage == 0) {
            st.acc[o] = k;
            res = st.u[o] + dt * k;
            st.next[o] = res;
          } else if (st.stage == 1) {
            const double a = st.acc[o];
            const double q = 0.25 * dt;
            res = (st.u[o] + q * a) + q * k;
            st.next[o] = res;
            st.acc[o] = a + k;
          } else {
            res = st.u[o] + ((1.0 / 6.0) * dt) * (st.acc[o] + 4.0 * k);
            st.u[o] = res;
          }
          break;
        case INT_RK4:
          if (st.stage == 0) {
            st.acc[o] = k;
            res = st.u[o] + (0.5 * dt) * k;
            st.next[o] = res;
          } else if (st.stage == 1) {
            st.acc[o] = st.acc[o] + 2.0 * k;
            res = st.u[o] + (0.5 * dt) * k;
            st.next[o] = res;
          } else if (st.stage == 2) {
            st.acc[o] = st.acc[o] + 2.0 * k;
            res = st.u[o] + dt * k;
            st.next[o] = res;
          } else {
            res = st.u[o] + ((1.0 / 6.0) * dt) * (st.acc[o] + k);
            st.u[o] = res;
          }
          break;
      }
      bad += isfinite(res) ? 0u : 1u;
    }
  }
  block_count_add(bad, &sc->nonfinite);
}

// ---------------------------------------------------------------------------
// Stage scalars: reset before a stage, finalize the CFL dt after the
// primitive pass (fvhoe/hydro.py:292, fvhoe/ode.py:11-22).
// ---------------------------------------------------------------------------
__global__ void k_reset_scalars(Scalars* sc, int reset_step);
__global__ void k_finalize_dt(Scalars* sc, double cfl_h, int use_fixed, double fixed_dt, int is_first_stage,
                              int has_target, double t, double target);

}  // namespace fvh
