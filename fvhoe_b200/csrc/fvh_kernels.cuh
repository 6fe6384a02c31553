// Kernels of the per-stage update (generic N-D path).
//
// Every array is stored variable-major over an index box ("Region") in cell
// coordinates: element (v, i0, i1, i2) of a box with origin lo and extents n
// sits at v*vs + (i0-lo0)*n1*n2 + (i1-lo1)*n2 + (i2-lo2). Axes are x, y, z in
// the reference's order (z contiguous); an inactive axis has extent 1.
// Offsets are 32-bit (the configuration check keeps every array below 2^31
// elements); a kernel forms one pointer per point and reaches its stencil
// taps and variables by constant strides.
//
// The stage is a sequence of passes, each a single launch over one box:
//   centre sweeps (the first one reads the conserved state through the
//   boundary index maps; the last one converts to primitives),
//   transverse sweeps (the last one also reduces the CFL speed and the
//   per-variable extrema), face reconstruction + Riemann solve, transverse
//   sweeps of the fluxes, the candidate update, troubled-cell detection,
//   pointwise primitives of the stage input, the MUSCL fallback at troubled
//   faces, and the flux divergence fused with the Runge-Kutta combination.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "fvh_physics.cuh"

namespace fvh {

enum Bc : int { BC_PERIODIC = 0, BC_OUTFLOW = 1, BC_REFLECTIVE = 2, BC_FREE = 3, BC_DIRICHLET = 4, BC_DMR_Y0 = 5 };

struct Region {
  int lo[3];
  int n[3];
};

// Ghost values of Dirichlet sides (boundary kinds "dirichlet" and "ic",
// fvhoe/boundary_conditions.py:18-55), given by the host: for axis a and side
// s an array (nv, E0, E1, E2) with E_a = depth[a] ghost layers along a and
// E_b = n_b + 2 pad[b] along the other axes (their ghost layers included).
// Element (v, i) of a ghost cell i: along a, i_a + depth[a] on the low side and
// i_a - n_a on the high side; along b, i_b + pad[b].
// A BC_DMR_Y0 low y side (the double-Mach-reflection wall) has no slab: its
// ghost cells take free or reflective values by the x index of their column
// (below dmr_split: free), fvhoe/boundary_conditions.py:374-395.
struct Slabs {
  int n[3];
  int bc[3][2];
  const double* p[3][2];  // nullptr unless that side is Dirichlet
  int depth[3];
  int pad[3];
  int dmr_split;
};

struct Grid {
  int n[3];      // interior cells per axis
  int bc[3][2];  // Bc kinds at the low/high end of each axis
  const Slabs* slabs;  // device copy when any side is Dirichlet, else nullptr
};

template <typename T, int K>
struct Rule {
  T w[K];
  int off;  // out[i] = sum_k w[k] * in[i + off + k]
};

__host__ __device__ __forceinline__ int64_t region_points(const Region& r) {
  return (int64_t)r.n[0] * r.n[1] * r.n[2];
}

// ---------------------------------------------------------------------------
// Division by a launch-constant divisor: q = (umulhi(n, m) + n) >> l with
// l = ceil(log2 d) and m = floor(2^32 (2^l - d) / d) + 1; exact for n < 2^31.
// ---------------------------------------------------------------------------
struct FastDiv {
  uint32_t m;
  uint32_t l;
};

inline FastDiv make_fastdiv(uint32_t d) {
  FastDiv f;
  uint32_t l = 0;
  while ((uint64_t(1) << l) < d) ++l;
  f.l = l;
  f.m = (uint32_t)(((uint64_t(1) << 32) * ((uint64_t(1) << l) - d)) / d + 1);
  return f;
}

__device__ __forceinline__ uint32_t fast_div(uint32_t n, const FastDiv& f) { return (__umulhi(n, f.m) + n) >> f.l; }

// An index box to iterate over, with its point count and dividers.
struct Box {
  int lo[3];
  int n[3];
  FastDiv d1, d2;
  uint32_t count;
};

inline Box make_box(const Region& r) {
  Box b;
  for (int a = 0; a < 3; ++a) {
    b.lo[a] = r.lo[a];
    b.n[a] = r.n[a];
  }
  b.d1 = make_fastdiv((uint32_t)r.n[1]);
  b.d2 = make_fastdiv((uint32_t)r.n[2]);
  b.count = (uint32_t)region_points(r);
  return b;
}

__device__ __forceinline__ void box_point(const Box& b, uint32_t idx, int& i0, int& i1, int& i2) {
  const uint32_t q = fast_div(idx, b.d2);
  i2 = (int)(idx - q * (uint32_t)b.n[2]) + b.lo[2];
  const uint32_t q2 = fast_div(q, b.d1);
  i1 = (int)(q - q2 * (uint32_t)b.n[1]) + b.lo[1];
  i0 = (int)q2 + b.lo[0];
}

#define FVH_FOR_POINTS(box, idx)                                                     \
  for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < (box).count; \
       idx += gridDim.x * blockDim.x)

// Strided view of a variable-major array stored over a Region.
template <typename T>
struct View {
  T* p;  // element (v = 0) at the region's origin
  int lo[3];
  int s0, s1;  // strides of axes 0 and 1; axis 2 is contiguous
  int vs;      // stride between variables
  __device__ __forceinline__ int at(int i0, int i1, int i2) const {
    return (i0 - lo[0]) * s0 + (i1 - lo[1]) * s1 + (i2 - lo[2]);
  }
  __device__ __forceinline__ int stride(int axis) const { return axis == 0 ? s0 : (axis == 1 ? s1 : 1); }
};

template <typename T>
inline View<T> make_view(T* p, const Region& r) {
  View<T> v;
  v.p = p;
  for (int a = 0; a < 3; ++a) v.lo[a] = r.lo[a];
  v.s1 = r.n[2];
  v.s0 = r.n[1] * r.n[2];
  v.vs = r.n[0] * r.n[1] * r.n[2];
  return v;
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

__device__ __forceinline__ int state_stride(const Grid& g, int axis) {
  return axis == 0 ? g.n[1] * g.n[2] : (axis == 1 ? g.n[2] : 1);
}

// Conserved state at a (possibly ghost) cell i when some side is Dirichlet.
// The reference fills the ghost slabs axis after axis, x then y then z, each
// slab spanning the others' ghost layers (fvhoe/boundary_conditions.py:306-402),
// so the last axis decides a corner: resolve z, then y, then x. A Dirichlet
// side returns its slab value at the coordinates mapped so far; a mirrored,
// periodic or free side maps its coordinate into the interior (the reflective
// sign flips apply to whatever value ends up copied).
template <typename Tc, typename Tin>
__device__ __forceinline__ void dirichlet_core(const Tin* __restrict__ u, const Slabs* __restrict__ sl, int nv,
                                               int i0, int i1, int i2, Tc* out) {
  int i[3] = {i0, i1, i2};
  bool flip[3] = {false, false, false};
  for (int a = 2; a >= 0; --a) {
    const int ia = i[a];
    const int na = sl->n[a];
    if (ia >= 0 && ia < na) continue;
    const int side = ia < 0 ? 0 : 1;
    if (sl->bc[a][side] == BC_DIRICHLET) {
      int e[3], k[3];
      for (int b = 0; b < 3; ++b) {
        e[b] = b == a ? sl->depth[b] : sl->n[b] + 2 * sl->pad[b];
        k[b] = b == a ? (side == 0 ? ia + sl->depth[b] : ia - na) : i[b] + sl->pad[b];
      }
      const double* p = sl->p[a][side];
      const int plane = e[0] * e[1] * e[2];
      const int o = (k[0] * e[1] + k[1]) * e[2] + k[2];
      for (int v = 0; v < nv; ++v) {
        double x = p[v * plane + o];
        if ((v == 1 && flip[0]) || (v == 2 && flip[1]) || (v == 3 && flip[2])) x = -x;
        out[v] = (Tc)x;
      }
      return;
    }
    // the double-Mach-reflection wall chooses by the column's x index, still
    // unmapped here because x is resolved last (it was filled first)
    int lo = sl->bc[a][0];
    if (lo == BC_DMR_Y0) lo = i[0] < sl->dmr_split ? BC_FREE : BC_REFLECTIVE;
    bool f = false;
    i[a] = ghost_source(ia, na, lo, sl->bc[a][1], f);
    flip[a] = f;
  }
  const int plane = sl->n[0] * sl->n[1] * sl->n[2];
  const int o = (i[0] * sl->n[1] + i[1]) * sl->n[2] + i[2];
  for (int v = 0; v < nv; ++v) {
    double x = (double)u[v * plane + o];
    if ((v == 1 && flip[0]) || (v == 2 && flip[1]) || (v == 3 && flip[2])) x = -x;
    out[v] = (Tc)x;
  }
}

// Out-of-line wrappers, so that kernels without Dirichlet sides pay only a
// uniform branch: any number of variables through a pointer, and the five
// variables of the fused 2D path returned by value (in registers).
template <typename Tc>
__device__ __noinline__ void load_state_dirichlet(const double* __restrict__ u, const Slabs* __restrict__ sl, int nv,
                                                  int i0, int i1, int i2, Tc* out) {
  dirichlet_core<Tc, double>(u, sl, nv, i0, i1, i2, out);
}

template <typename Tc>
struct State5 {
  Tc v[5];
};

template <typename Tc, typename Tin>
__device__ __noinline__ State5<Tc> load_state5_dirichlet(const Tin* __restrict__ u, const Slabs* __restrict__ sl,
                                                         int i0, int i1, int i2) {
  State5<Tc> s;
  dirichlet_core<Tc, Tin>(u, sl, 5, i0, i1, i2, s.v);
  return s;
}

// Reads nv conserved variables at a (possibly ghost) cell. Reflective ghosts
// negate the momentum normal to the wall they mirror across.
template <typename Tc>
__device__ __forceinline__ void load_state(const double* __restrict__ u, const Grid& g, int nv, int i0, int i1,
                                           int i2, Tc* out) {
  if (g.slabs) {
    load_state_dirichlet<Tc>(u, g.slabs, nv, i0, i1, i2, out);
    return;
  }
  bool f0 = false, f1 = false, f2 = false;
  const int j0 = ghost_source(i0, g.n[0], g.bc[0][0], g.bc[0][1], f0);
  const int j1 = ghost_source(i1, g.n[1], g.bc[1][0], g.bc[1][1], f1);
  const int j2 = ghost_source(i2, g.n[2], g.bc[2][0], g.bc[2][1], f2);
  const int plane = g.n[0] * g.n[1] * g.n[2];
  const int o = (j0 * g.n[1] + j1) * g.n[2] + j2;
  for (int v = 0; v < nv; ++v) {
    double x = u[v * plane + o];
    if ((v == 1 && f0) || (v == 2 && f1) || (v == 3 && f2)) x = -x;
    out[v] = (Tc)x;
  }
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
  unsigned int timeouts;                  // tile copies refused (misaligned) or whose bounded wait ran out, this step
  // learned-predictor counts, summed over the stages of a step
  unsigned int predicted;                 // cells the network flagged
  unsigned int judged;                    // cells the a-posteriori check flagged
  unsigned int missed;                    // judged, not predicted
  unsigned int false_alarm;               // predicted, not judged
  // faces whose flux the fused path revised, summed over the stages of a step:
  // by the final pass (troubled cells; with a predictor, only the misses) and
  // by the flux pass (faces of predicted cells)
  unsigned int revised_faces;
  unsigned int flux_fallback_faces;
  unsigned int fb_faces;  // length of this stage's fallback face list (fused 2D path)
};

// Reduction request for the last transverse sweep of the primitive pass.
struct ReduceSpec {
  int cfl;  // reduce the CFL speed over cfl_box
  Region cfl_box;
  int extrema;  // reduce per-variable max/min over ext_box
  Region ext_box;
  double ndim;  // number of active axes, as in ndim * c
};

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

// Block-wide sum of a per-thread count with one atomic per block (blocks of
// at most 256 threads).
__device__ __forceinline__ void block_count_add(unsigned int count, unsigned int* dst) {
  __shared__ unsigned int s_count[8];
  for (int o = 16; o > 0; o >>= 1) count += __shfl_xor_sync(0xffffffffu, count, o);
  __syncthreads();  // a previous call's reads of s_count are done
  if ((threadIdx.x & 31) == 0) s_count[threadIdx.x >> 5] = count;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int total = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) total += s_count[w];
    if (total) atomicAdd(dst, total);
  }
}

// ---------------------------------------------------------------------------
// Centre-interpolation sweep (fvhoe/fv.py:106-159, 175-197). FROM_STATE reads
// the conserved state through the ghost maps; TO_PRIMS converts the swept
// cell-centre values to primitives (fvhoe/hydro.py:146-170).
// ---------------------------------------------------------------------------
template <typename Tc, typename Tin, int NV, int K, bool FROM_STATE, bool TO_PRIMS>
__global__ void __launch_bounds__(256)
    k_centre_sweep(View<const Tin> in, const double* __restrict__ state, View<Tc> out, Box box, int axis,
                   Rule<Tc, K> rule, Grid grid, Phys<Tc> ph) {
  constexpr int NVA = VarCount<NV>::kArray;
  const int nv = VarCount<NV>::get(ph);
  const int plane = grid.n[0] * grid.n[1] * grid.n[2];
  FVH_FOR_POINTS(box, idx) {
    int i[3];
    box_point(box, idx, i[0], i[1], i[2]);
    Tc acc[NVA];
    for (int v = 0; v < nv; ++v) acc[v] = Tc(0);
    if constexpr (FROM_STATE) {
      if (grid.slabs) {
        // Dirichlet sides: every tap through the general ghost resolution
#pragma unroll
        for (int k = 0; k < K; ++k) {
          int t[3] = {i[0], i[1], i[2]};
          t[axis] += rule.off + k;
          Tc uc[NVA];
          load_state_dirichlet<Tc>(state, grid.slabs, nv, t[0], t[1], t[2], uc);
          for (int v = 0; v < nv; ++v) acc[v] = acc[v] + rule.w[k] * uc[v];
        }
      } else {
      // ghost maps of the two fixed coordinates, once per point
      bool fl[3] = {false, false, false};
      int base = 0;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        if (a == axis) continue;
        const int j = ghost_source(i[a], grid.n[a], grid.bc[a][0], grid.bc[a][1], fl[a]);
        base += j * state_stride(grid, a);
      }
      const int sa = state_stride(grid, axis);
      const int ia = axis == 0 ? i[0] : (axis == 1 ? i[1] : i[2]);
      const int na = axis == 0 ? grid.n[0] : (axis == 1 ? grid.n[1] : grid.n[2]);
      const int lo_kind = axis == 0 ? grid.bc[0][0] : (axis == 1 ? grid.bc[1][0] : grid.bc[2][0]);
      const int hi_kind = axis == 0 ? grid.bc[0][1] : (axis == 1 ? grid.bc[1][1] : grid.bc[2][1]);
#pragma unroll
      for (int k = 0; k < K; ++k) {
        bool fk = false;
        const int jk = ghost_source(ia + rule.off + k, na, lo_kind, hi_kind, fk);
        const double* q = state + base + jk * sa;
        for (int v = 0; v < nv; ++v) {
          double x = q[v * plane];
          const bool flip = (v == 1 && (axis == 0 ? fk : fl[0])) || (v == 2 && (axis == 1 ? fk : fl[1])) ||
                            (v == 3 && (axis == 2 ? fk : fl[2]));
          if (flip) x = -x;
          acc[v] = acc[v] + rule.w[k] * (Tc)x;
        }
      }
      }
    } else {
      const int sa = in.stride(axis);
      const Tin* q = in.p + in.at(i[0], i[1], i[2]) + rule.off * sa;
#pragma unroll
      for (int k = 0; k < K; ++k)
        for (int v = 0; v < nv; ++v) acc[v] = acc[v] + rule.w[k] * (Tc)q[v * in.vs + k * sa];
    }
    Tc* o = out.p + out.at(i[0], i[1], i[2]);
    if constexpr (TO_PRIMS) {
      Tc w[NVA];
      to_primitives(ph, nv, acc, w);
      for (int v = 0; v < nv; ++v) o[v * out.vs] = w[v];
    } else {
      for (int v = 0; v < nv; ++v) o[v * out.vs] = acc[v];
    }
  }
}

// ---------------------------------------------------------------------------
// Transverse-reconstruction sweep (fvhoe/fv.py:162-172, 200-224), optionally
// reducing the CFL speed (fvhoe/hydro.py:270-294) and the per-variable extrema
// used by global NAD (fvhoe/slope_limiting.py:165-170, 184-185).
// ---------------------------------------------------------------------------
template <typename Tc, int NV, int K, bool REDUCE>
__global__ void __launch_bounds__(256)
    k_transverse_sweep(View<const Tc> in, View<Tc> out, Box box, int axis, Rule<Tc, K> rule, Phys<Tc> ph,
                       ReduceSpec rs, Scalars* __restrict__ sc) {
  constexpr int NVA = VarCount<NV>::kArray;
  const int nv = VarCount<NV>::get(ph);
  unsigned long long cfl_key = 0ull;
  unsigned long long kmax[5], kmin[5];
  if constexpr (REDUCE) {
    for (int v = 0; v < 5; ++v) {
      kmax[v] = 0ull;
      kmin[v] = ~0ull;
    }
  }
  const int sa = in.stride(axis);
  FVH_FOR_POINTS(box, idx) {
    int i0, i1, i2;
    box_point(box, idx, i0, i1, i2);
    Tc acc[NVA];
    for (int v = 0; v < nv; ++v) acc[v] = Tc(0);
    const Tc* q = in.p + in.at(i0, i1, i2) + rule.off * sa;
#pragma unroll
    for (int k = 0; k < K; ++k)
      for (int v = 0; v < nv; ++v) acc[v] = acc[v] + rule.w[k] * q[v * in.vs + k * sa];
    Tc* o = out.p + out.at(i0, i1, i2);
    for (int v = 0; v < nv; ++v) o[v * out.vs] = acc[v];
    if constexpr (REDUCE) {
      if (rs.cfl && in_box(rs.cfl_box, i0, i1, i2)) {
        const unsigned long long k = order_key((double)cfl_speed(ph, acc, (Tc)rs.ndim));
        cfl_key = k > cfl_key ? k : cfl_key;
      }
      if (rs.extrema && in_box(rs.ext_box, i0, i1, i2)) {
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

// ---------------------------------------------------------------------------
// Face reconstruction along d and the Riemann solve (fvhoe/solver.py:522-607):
// face j lies between cells j-1 and j; the left state is cell j-1's right-face
// value, the right state is cell j's left-face value.
// ---------------------------------------------------------------------------
template <typename Tc, int NV, int K>
__global__ void __launch_bounds__(256)
    k_face_riemann(View<const Tc> in, View<Tc> out, Box box, int d, Rule<Tc, K> left_rule, Rule<Tc, K> right_rule,
                   Phys<Tc> ph) {
  constexpr int NVA = VarCount<NV>::kArray;
  const int nv = VarCount<NV>::get(ph);
  const int sd = in.stride(d);
  FVH_FOR_POINTS(box, idx) {
    int i0, i1, i2;
    box_point(box, idx, i0, i1, i2);
    const Tc* q = in.p + in.at(i0, i1, i2);
    const Tc* qa = q + (right_rule.off - 1) * sd;  // cell j-1, right-face rule
    const Tc* qb = q + left_rule.off * sd;         // cell j, left-face rule
    Tc wl[NVA], wr[NVA];
    for (int v = 0; v < nv; ++v) {
      wl[v] = Tc(0);
      wr[v] = Tc(0);
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
      for (int v = 0; v < nv; ++v) {
        wl[v] = wl[v] + right_rule.w[k] * qa[v * in.vs + k * sd];
        wr[v] = wr[v] + left_rule.w[k] * qb[v * in.vs + k * sd];
      }
    }
    Tc f[NVA];
    riemann_flux<NVA>(ph, nv, wl, wr, d, f);
    Tc* o = out.p + out.at(i0, i1, i2);
    for (int v = 0; v < nv; ++v) o[v * out.vs] = f[v];
  }
}

// ---------------------------------------------------------------------------
// Flux divergence, fvhoe/solver.py:734-751:
//   dudt = 0.0 + -(1/hx)(F[i+1]-F[i]) + -(1/hy)(G[j+1]-G[j]) + -(1/hz)(H[k+1]-H[k])
// ---------------------------------------------------------------------------
template <typename Tc>
struct FluxSet {
  View<const Tc> f[3];
  int has[3];
  double neg_inv_h[3];  // -(1/h_d), rounded on the host as Python does
};

template <typename Tc>
__device__ __forceinline__ void divergence(const FluxSet<Tc>& fs, int nv, int i0, int i1, int i2, Tc* dudt) {
  for (int v = 0; v < nv; ++v) dudt[v] = Tc(0);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (!fs.has[d]) continue;
    const View<const Tc>& F = fs.f[d];
    const Tc* q = F.p + F.at(i0, i1, i2);
    const int sd = F.stride(d);
    const Tc c = (Tc)fs.neg_inv_h[d];
    for (int v = 0; v < nv; ++v) dudt[v] = dudt[v] + c * (q[v * F.vs + sd] - q[v * F.vs]);
  }
}

// Candidate state u* = u + dt L(F) (fvhoe/solver.py:677-678), kept in float64.
template <typename Tc, int NV>
__global__ void __launch_bounds__(256) k_candidate(const double* __restrict__ u, View<double> ustar, Box box,
                                                   FluxSet<Tc> fs, Phys<Tc> ph, const Scalars* __restrict__ sc) {
  constexpr int NVA = VarCount<NV>::kArray;
  const int nv = VarCount<NV>::get(ph);
  const double dt = sc->dt_stage;
  FVH_FOR_POINTS(box, idx) {
    int i0, i1, i2;
    box_point(box, idx, i0, i1, i2);
    Tc dudt[NVA];
    divergence<Tc>(fs, nv, i0, i1, i2, dudt);
    const int o = ustar.at(i0, i1, i2);
    for (int v = 0; v < nv; ++v) ustar.p[v * ustar.vs + o] = u[v * ustar.vs + o] + dt * (double)dudt[v];
  }
}

// ---------------------------------------------------------------------------
// Troubled-cell detection (fvhoe/slope_limiting.py:87-244), for NDIM active axes.
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
  int axes[3];   // the active axes, ascending
  int log_mode;  // 0: no logging, 1: overwrite the running sums, 2: add to them
  double log_div;  // > 0: divide the sums by it afterwards (the step's last stage)
};

// Running trouble / NAD / PAD sums of log_troubles (fvhoe/solver.py:794-833):
// mode 1 overwrites them, mode 2 adds this stage's values; a positive log_div
// then divides them, the reset branch of log_troubles (:809-820) done here
// instead of in a separate pass over the arrays.
__device__ __forceinline__ void log_write(const DetectSpec& ds, int o, double lt, double ln, double lp,
                                          double* __restrict__ log_trouble, double* __restrict__ log_nad,
                                          double* __restrict__ log_pad) {
  double a = lt, b = ln, c = lp;
  if (ds.log_mode == 2) {
    a = log_trouble[o] + lt;
    b = log_nad[o] + ln;
    c = log_pad[o] + lp;
  }
  if (ds.log_div > 0.0) {
    a = a / ds.log_div;
    b = b / ds.log_div;
    c = c / ds.log_div;
  }
  log_trouble[o] = a;
  log_nad[o] = b;
  log_pad[o] = c;
}

// Whether the smooth-extrema detector's alpha along one line is below 1
// (fvhoe/smooth_extrema_detection.py:8-50). a[0..6] are the values at
// offsets -3..+3. The reference takes alpha = min over the cell and its two
// neighbours of min(alpha_L, alpha_R), with alpha_L clamped to 1 and alpha_R
// set to 1 where |dv| <= eps; alpha < 1 exactly when some alpha_L or alpha_R
// of the three positions is, so the scan stops at the first one found. Each
// alpha is the same quotient the reference forms.
template <typename T>
__device__ __forceinline__ bool sed_line_below_one(const T* a, T eps) {
  T du[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) du[k] = T(0.5) * (a[k + 2] - a[k]);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const T d2u = T(0.5) * (du[k + 2] - du[k]);
    T dv = T(0.5) * d2u;
    const bool small = fabs(dv) <= eps;
    if (small) dv = dv >= T(0) ? eps : -eps;
    const T vl = du[k] - du[k + 1];
    const T xl = dv < T(0) ? (vl > T(0) ? vl : T(0)) : (vl < T(0) ? vl : T(0));
    // alpha_L = -x_L / dv; a zero numerator gives a zero alpha without dividing
    if (xl == T(0) || -xl / dv < T(1)) return true;
    if (fabs(dv) > eps) {
      const T vr = du[k + 2] - du[k + 1];
      const T xr = dv > T(0) ? (vr > T(0) ? vr : T(0)) : (vr < T(0) ? vr : T(0));
      if (xr == T(0) || xr / dv < T(1)) return true;
    }
  }
  return false;
}

template <typename Tc, int NDIM>
__global__ void __launch_bounds__(256)
    k_detect(View<const Tc> w, View<const Tc> ws, Box box, DetectSpec ds, Scalars* __restrict__ sc,
             View<uint8_t> trouble, double* __restrict__ log_trouble, double* __restrict__ log_nad,
             double* __restrict__ log_pad) {
  int sw[3] = {0, 0, 0}, sws[3] = {0, 0, 0};
#pragma unroll
  for (int k = 0; k < NDIM; ++k) {
    sw[k] = w.stride(ds.axes[k]);
    sws[k] = ws.stride(ds.axes[k]);
  }
  // NAD bounds that do not depend on the cell
  Tc grange[5], glower[5], gupper[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    const double vmax = key_value(sc->vmax_key[v]);
    const double vmin = key_value(sc->vmin_key[v]);
    grange[v] = (Tc)(vmax - vmin);
    glower[v] = (Tc)((1.0 - ds.nad_eps) * vmin);
    gupper[v] = (Tc)((1.0 + ds.nad_eps) * vmax);
  }
  const Tc neg_eps = (Tc)(-ds.nad_eps);
  const Tc lo_fac = (Tc)(1.0 - ds.nad_eps), hi_fac = (Tc)(1.0 + ds.nad_eps);
  const Tc sed_eps = (Tc)ds.sed_eps;
  unsigned int count = 0;
  FVH_FOR_POINTS(box, idx) {
    int i0, i1, i2;
    box_point(box, idx, i0, i1, i2);
    const int ow = w.at(i0, i1, i2);
    const int ows = ws.at(i0, i1, i2);
    bool nad_any = false;
    Tc ind_min = Tc(0);
    Tc pad_ind = Tc(0);
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      // 3^d box extrema of w (fvhoe/slope_limiting.py:145-162)
      const Tc* pw = w.p + v * w.vs + ow;
      Tc big = pw[0], small = big;
#pragma unroll
      for (int a = -1; a <= 1; ++a)
#pragma unroll
        for (int b = (NDIM > 1 ? -1 : 0); b <= (NDIM > 1 ? 1 : 0); ++b)
#pragma unroll
          for (int c = (NDIM > 2 ? -1 : 0); c <= (NDIM > 2 ? 1 : 0); ++c) {
            const Tc x = pw[a * sw[0] + b * sw[1] + c * sw[2]];
            big = fmax(big, x);
            small = fmin(small, x);
          }
      const Tc* pws = ws.p + v * ws.vs + ows;
      const Tc xs = pws[0];
      Tc ind;
      bool tv;
      if (ds.nad_relative) {
        const Tc range = ds.nad_global ? grange[v] : big - small;
        ind = xs - small;
        ind = fmin(ind, big - xs);
        tv = ind < neg_eps * range;
      } else {
        const Tc lower = ds.nad_global ? glower[v] : lo_fac * small;
        const Tc upper = ds.nad_global ? gupper[v] : hi_fac * big;
        ind = fmin(xs - lower, upper - xs);
        tv = ind < Tc(0);
      }
      if (tv && ds.sed) {
        // smooth-extrema detector on w* (fvhoe/smooth_extrema_detection.py:8-95):
        // the flag survives only where alpha, the minimum over the axes, is below 1
        bool below = false;
#pragma unroll
        for (int k = 0; k < NDIM; ++k) {
          if (below) break;
          Tc line[7];
#pragma unroll
          for (int m = 0; m < 7; ++m) line[m] = pws[(m - 3) * sws[k]];
          below = sed_line_below_one(line, sed_eps);
        }
        tv = below;
      }
      if (!((ds.nad_var_mask >> v) & 1)) tv = false;
      nad_any = nad_any || tv;
      ind_min = (v == 0) ? ind : fmin(ind_min, ind);
      if (v == ds.pad_var) {
        pad_ind = xs - (Tc)ds.pad_lo;
        pad_ind = fmin(pad_ind, (Tc)ds.pad_hi - xs);
      }
    }
    const bool pad_trouble = pad_ind < Tc(0);
    bool t = pad_trouble || nad_any;
    if (ds.force_trouble) t = true;
    const int o = trouble.at(i0, i1, i2);
    trouble.p[o] = t ? 1 : 0;
    count += t ? 1u : 0u;
    if (ds.log_mode) {
      const double lt = t ? 1.0 : 0.0;
      const double ln = nad_any ? -(double)ind_min : 0.0;
      const double lp = pad_trouble ? -(double)pad_ind : 0.0;
      log_write(ds, o, lt, ln, lp, log_trouble, log_nad, log_pad);
    }
  }
  block_count_add(count, &sc->troubled);
}

// The same detection for three active axes, with the 3^3 box extrema from a
// sliding window: a thread owns one (i1, i2) column of the box and CH
// consecutive cells along axis 0, and per variable takes the 3x3 extrema of
// each plane once (9 loads), the box extrema of a cell being those of its
// three planes (9 (CH + 2) / CH loads per cell and variable instead of 27,
// at 80 registers for three blocks per SM). Minima
// and maxima do not depend on the order they are taken in, and every other
// quantity is formed as k_detect forms it, variable after variable, so the
// flags and logs are the same. Grid: x over the columns, y over the chunks.
template <typename Tc, int CH>
__global__ void __launch_bounds__(256, 3)
    k_detect3(View<const Tc> w, View<const Tc> ws, Box box, DetectSpec ds, Scalars* __restrict__ sc,
              View<uint8_t> trouble, double* __restrict__ log_trouble, double* __restrict__ log_nad,
              double* __restrict__ log_pad) {
  const int sw0 = w.stride(0), sw1 = w.stride(1), sw2 = w.stride(2);
  const int sws[3] = {ws.stride(0), ws.stride(1), ws.stride(2)};
  const Tc neg_eps = (Tc)(-ds.nad_eps);
  const Tc lo_fac = (Tc)(1.0 - ds.nad_eps), hi_fac = (Tc)(1.0 + ds.nad_eps);
  const Tc sed_eps = (Tc)ds.sed_eps;
  unsigned int count = 0;
  const uint32_t col = blockIdx.x * blockDim.x + threadIdx.x;
  const int x0 = box.lo[0] + (int)blockIdx.y * CH;
  const int ncell = min(CH, box.lo[0] + box.n[0] - x0);
  if (col < (uint32_t)box.n[1] * box.n[2] && ncell > 0) {
    const int i1 = box.lo[1] + (int)(col / (uint32_t)box.n[2]);
    const int i2 = box.lo[2] + (int)(col % (uint32_t)box.n[2]);
    Tc ind_min[CH], pad_ind[CH];
    unsigned int nad_bits = 0u;
#pragma unroll
    for (int c = 0; c < CH; ++c) {
      ind_min[c] = Tc(0);
      pad_ind[c] = Tc(0);
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      // the variable's global NAD bounds (formed as k_detect forms them)
      const double vmax = key_value(sc->vmax_key[v]);
      const double vmin = key_value(sc->vmin_key[v]);
      const Tc grange = (Tc)(vmax - vmin);
      const Tc glower = (Tc)((1.0 - ds.nad_eps) * vmin);
      const Tc gupper = (Tc)((1.0 + ds.nad_eps) * vmax);
      const Tc* pw = w.p + v * w.vs + w.at(x0, i1, i2);
      const Tc* pws0 = ws.p + v * ws.vs + ws.at(x0, i1, i2);
      // 3x3 extrema of the plane at offset a along axis 0 (centre first, as
      // the box loop of k_detect starts)
      auto plane = [&](int a, Tc& big, Tc& small) {
        const Tc* q = pw + a * sw0;
        big = q[0];
        small = big;
#pragma unroll
        for (int b = -1; b <= 1; ++b)
#pragma unroll
          for (int cc = -1; cc <= 1; ++cc) {
            const Tc x = q[b * sw1 + cc * sw2];
            big = fmax(big, x);
            small = fmin(small, x);
          }
      };
      Tc bm, sm, b0, s0, bp, sp;
      plane(-1, bm, sm);
      plane(0, b0, s0);
#pragma unroll
      for (int c = 0; c < CH; ++c) {
        if (c < ncell) {
          plane(c + 1, bp, sp);
          const Tc big = fmax(fmax(bm, b0), bp), small = fmin(fmin(sm, s0), sp);
          const Tc* pws = pws0 + c * sws[0];
          const Tc xs = pws[0];
          Tc ind;
          bool tv;
          if (ds.nad_relative) {
            const Tc range = ds.nad_global ? grange : big - small;
            ind = xs - small;
            ind = fmin(ind, big - xs);
            tv = ind < neg_eps * range;
          } else {
            const Tc lower = ds.nad_global ? glower : lo_fac * small;
            const Tc upper = ds.nad_global ? gupper : hi_fac * big;
            ind = fmin(xs - lower, upper - xs);
            tv = ind < Tc(0);
          }
          if (tv && ds.sed) {
            bool below = false;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
              if (below) break;
              Tc line[7];
#pragma unroll
              for (int m = 0; m < 7; ++m) line[m] = pws[(m - 3) * sws[k]];
              below = sed_line_below_one(line, sed_eps);
            }
            tv = below;
          }
          if (!((ds.nad_var_mask >> v) & 1)) tv = false;
          if (tv) nad_bits |= 1u << c;
          ind_min[c] = (v == 0) ? ind : fmin(ind_min[c], ind);
          if (v == ds.pad_var) {
            Tc pi = xs - (Tc)ds.pad_lo;
            pad_ind[c] = fmin(pi, (Tc)ds.pad_hi - xs);
          }
          bm = b0;
          sm = s0;
          b0 = bp;
          s0 = sp;
        }
      }
    }
#pragma unroll
    for (int c = 0; c < CH; ++c) {
      if (c < ncell) {
        const bool nad_any = (nad_bits >> c) & 1u;
        const bool pad_trouble = pad_ind[c] < Tc(0);
        bool t = pad_trouble || nad_any;
        if (ds.force_trouble) t = true;
        const int o = trouble.at(x0 + c, i1, i2);
        trouble.p[o] = t ? 1 : 0;
        count += t ? 1u : 0u;
        if (ds.log_mode) {
          const double lt = t ? 1.0 : 0.0;
          const double ln = nad_any ? -(double)ind_min[c] : 0.0;
          const double lp = pad_trouble ? -(double)pad_ind[c] : 0.0;
          log_write(ds, o, lt, ln, lp, log_trouble, log_nad, log_pad);
        }
      }
    }
  }
  block_count_add(count, &sc->troubled);
}

// ---------------------------------------------------------------------------
// Pointwise primitives of the stage input over the interior and 2 ghost
// cells: the fallback scheme's FV primitives, because its p = 1 centre and
// transverse rules are the identity (fvhoe/solver.py:712-717, 753-792).
// ---------------------------------------------------------------------------
template <typename Tc, int NV>
__global__ void __launch_bounds__(256) k_pointwise_primitives(const double* __restrict__ u, Grid grid, View<Tc> w1,
                                                              Box box, Phys<Tc> ph) {
  constexpr int NVA = VarCount<NV>::kArray;
  const int nv = VarCount<NV>::get(ph);
  FVH_FOR_POINTS(box, idx) {
    int i0, i1, i2;
    box_point(box, idx, i0, i1, i2);
    Tc uc[NVA], w[NVA];
    load_state<Tc>(u, grid, nv, i0, i1, i2, uc);
    to_primitives(ph, nv, uc, w);
    Tc* o = w1.p + w1.at(i0, i1, i2);
    for (int v = 0; v < nv; ++v) o[v * w1.vs] = w[v];
  }
}

// ---------------------------------------------------------------------------
// MUSCL fallback at troubled faces and the flux blend
// (fvhoe/solver.py:710-731, fvhoe/slope_limiting.py:24-84, 247-384).
// theta of face j = max(trouble[j-1], trouble[j]) with missing neighbours 0,
// or the convex weights when theta_in is given.
// ---------------------------------------------------------------------------
struct FallbackSpec {
  int d;        // face-normal axis
  int nd;       // interior cells along d
  int muscl;    // 1: slope-limited p=1 reconstruction along d, 0: first order
  int limiter;  // Limiter enum
};

template <typename Tc, int NV>
__global__ void __launch_bounds__(256)
    k_fallback(View<const Tc> w1, View<Tc> F, Box box, View<const uint8_t> trouble, const float* __restrict__ theta_in,
               FallbackSpec fb, Phys<Tc> ph) {
  constexpr int NVA = VarCount<NV>::kArray;
  const int nv = VarCount<NV>::get(ph);
  const int d = fb.d;
  const int st = trouble.stride(d);
  const int sw = w1.stride(d);
  FVH_FOR_POINTS(box, idx) {
    int i[3];
    box_point(box, idx, i[0], i[1], i[2]);
    Tc theta;
    if (theta_in) {
      theta = (Tc)theta_in[idx];
    } else {
      const int j = d == 0 ? i[0] : (d == 1 ? i[1] : i[2]);
      const int ot = trouble.at(i[0], i[1], i[2]);
      const uint8_t tl = j >= 1 ? trouble.p[ot - st] : 0;
      const uint8_t tr = j < fb.nd ? trouble.p[ot] : 0;
      theta = (tl || tr) ? Tc(1) : Tc(0);
    }
    if (!(theta > Tc(0))) continue;
    // primitives at cells j-2 .. j+1 along d
    const Tc* q = w1.p + w1.at(i[0], i[1], i[2]) - 2 * sw;
    Tc wl[NVA], wr[NVA];
    for (int v = 0; v < nv; ++v) {
      const Tc* qv = q + v * w1.vs;
      const Tc a0 = qv[0], a1 = qv[sw], a2 = qv[2 * sw], a3 = qv[3 * sw];
      if (fb.muscl && fb.limiter == LIMITER_NONE) {
        // unlimited p=1 face rules [1/4, 1, -1/4] and its mirror (fvhoe/stencils.py:44-46)
        wl[v] = ((Tc(0) + Tc(-0.25) * a0) + Tc(1) * a1) + Tc(0.25) * a2;
        wr[v] = ((Tc(0) + Tc(0.25) * a1) + Tc(1) * a2) + Tc(-0.25) * a3;
      } else if (fb.muscl) {
        const Tc sl = limited_slope(a1 - a0, a2 - a1, fb.limiter);
        const Tc sr = limited_slope(a2 - a1, a3 - a2, fb.limiter);
        wl[v] = a1 + Tc(0.5) * sl;
        wr[v] = a2 - Tc(0.5) * sr;
      } else {
        wl[v] = a1;
        wr[v] = a2;
      }
    }
    Tc flo[NVA];
    riemann_flux<NVA>(ph, nv, wl, wr, d, flo);
    Tc* o = F.p + F.at(i[0], i[1], i[2]);
    for (int v = 0; v < nv; ++v) o[v * F.vs] = (Tc(1) - theta) * o[v * F.vs] + theta * flo[v];
  }
}

// The same fallback without the pointwise pass and without idle lanes (the
// faces' own flags, no convex weights): a block takes 1024 faces at a time,
// gathers the faces next to a troubled cell into a shared list (one atomic
// per warp) and solves the list with whole warps, converting the four cells
// a face reads from the stage input as k_pointwise_primitives converts them.
// Every face value equals k_fallback's.
template <typename Tc, int NV>
__global__ void __launch_bounds__(256)
    k_fallback_direct(const double* __restrict__ u, Grid grid, View<Tc> F, Box box, View<const uint8_t> trouble,
                      FallbackSpec fb, Phys<Tc> ph) {
  constexpr int NVA = VarCount<NV>::kArray;
  constexpr int CHUNK = 1024;
  __shared__ uint32_t list[CHUNK];
  __shared__ int count;
  const int nv = VarCount<NV>::get(ph);
  const int d = fb.d;
  const int st = trouble.stride(d);
  const int lane = threadIdx.x & 31;
  for (uint32_t base = blockIdx.x * CHUNK; base < box.count; base += gridDim.x * CHUNK) {
    if (threadIdx.x == 0) count = 0;
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < CHUNK; k += blockDim.x) {
      const uint32_t idx = base + k;
      bool on = false;
      if (idx < box.count) {
        int i0, i1, i2;
        box_point(box, idx, i0, i1, i2);
        const int j = d == 0 ? i0 : (d == 1 ? i1 : i2);
        const int ot = trouble.at(i0, i1, i2);
        on = (j >= 1 && trouble.p[ot - st]) || (j < fb.nd && trouble.p[ot]);
      }
      const unsigned int ballot = __ballot_sync(0xffffffffu, on);
      int wbase = 0;
      if (lane == 0 && ballot) wbase = atomicAdd(&count, __popc(ballot));
      wbase = __shfl_sync(0xffffffffu, wbase, 0);
      if (on) list[wbase + __popc(ballot & ((1u << lane) - 1u))] = idx;
    }
    __syncthreads();
    const int n = count;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      int i[3];
      box_point(box, list[k], i[0], i[1], i[2]);
      // primitives at cells j-2 .. j+1 along d
      Tc a[4][NVA];
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        int c[3] = {i[0], i[1], i[2]};
        c[d] += m - 2;
        Tc uc[NVA];
        load_state<Tc>(u, grid, nv, c[0], c[1], c[2], uc);
        to_primitives(ph, nv, uc, a[m]);
      }
      Tc wl[NVA], wr[NVA];
      for (int v = 0; v < nv; ++v) {
        const Tc a0 = a[0][v], a1 = a[1][v], a2 = a[2][v], a3 = a[3][v];
        if (fb.muscl && fb.limiter == LIMITER_NONE) {
          wl[v] = ((Tc(0) + Tc(-0.25) * a0) + Tc(1) * a1) + Tc(0.25) * a2;
          wr[v] = ((Tc(0) + Tc(0.25) * a1) + Tc(1) * a2) + Tc(-0.25) * a3;
        } else if (fb.muscl) {
          const Tc sl = limited_slope(a1 - a0, a2 - a1, fb.limiter);
          const Tc sr = limited_slope(a2 - a1, a3 - a2, fb.limiter);
          wl[v] = a1 + Tc(0.5) * sl;
          wr[v] = a2 - Tc(0.5) * sr;
        } else {
          wl[v] = a1;
          wr[v] = a2;
        }
      }
      Tc flo[NVA];
      riemann_flux<NVA>(ph, nv, wl, wr, d, flo);
      Tc* o = F.p + F.at(i[0], i[1], i[2]);
      for (int v = 0; v < nv; ++v) o[v * F.vs] = (Tc(1) - Tc(1)) * o[v * F.vs] + Tc(1) * flo[v];
    }
    __syncthreads();  // the list is read before the next chunk resets it
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
__global__ void __launch_bounds__(256) k_final(Box box, View<double> state, FluxSet<Tc> fs, Phys<Tc> ph,
                                               StageSpec st, Scalars* __restrict__ sc) {
  constexpr int NVA = VarCount<NV>::kArray;
  const int nv = VarCount<NV>::get(ph);
  const double dt = sc->dt_step;
  unsigned int bad = 0;
  FVH_FOR_POINTS(box, idx) {
    int i0, i1, i2;
    box_point(box, idx, i0, i1, i2);
    Tc dudt_c[NVA];
    divergence<Tc>(fs, nv, i0, i1, i2, dudt_c);
    const int base = state.at(i0, i1, i2);
    for (int v = 0; v < nv; ++v) {
      const int o = base + v * state.vs;
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
          if (sizeof(Tc) == 4) {
            // FP32 form: the Shu-Osher stages (no k-sum), as the fused final pass
            if (st.stage == 0) {
              res = st.u[o] + dt * k;
              st.next[o] = res;
            } else if (st.stage == 1) {
              res = 0.75 * st.u[o] + 0.25 * (st.stage_in[o] + dt * k);
              st.next[o] = res;
            } else {
              res = (1.0 / 3.0) * st.u[o] + (2.0 / 3.0) * (st.stage_in[o] + dt * k);
              st.u[o] = res;
            }
          } else if (st.stage == 0) {
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
