// Fused 2D stage: five shared-memory-tiled launches per stage instead of the
// generic path's ~21 passes, for problems with two active axes, five
// variables and the same degree p (1..8) on both axes.
//
// The two active axes are called X (outer, strided) and Y (inner, contiguous);
// dX and dY are their physical axis ids (0, 1 or 2), which select the normal
// momentum component of each direction. Every per-point expression is the
// generic path's (and the reference's), evaluated in the same order, so the
// FP64 instantiation reproduces the reference bit for bit:
//   k2_primitives  W = FV primitives of the stage input on [-g, n+g)^2, with
//                  the CFL and per-variable extrema reductions
//                  (fvhoe/solver.py:753-792, fvhoe/hydro.py:270-294)
//   k2_fluxes      X- and Y-face high-order fluxes from W and the candidate
//                  u* = u + dt L(F) (fvhoe/solver.py:519-651, 677-678)
//   k2_primitives  on the candidate: W* over [-3, n+3)^2 (no reductions)
//   k2_detect_staged  troubled-cell detection from the W* and W tiles
//                  (fvhoe/slope_limiting.py:87-244); the batched ensemble's
//                  phase computes W* on each tile instead (tile2_detect)
//   k2_final       MUSCL fallback fluxes at troubled faces, the blend, the flux
//                  divergence and the Runge-Kutta combination
//                  (fvhoe/solver.py:710-751, fvhoe/ode.py:245-298); in FP64
//                  the fallback runs first in two launches of its own
//                  (k2_face_list, k2_face_solve) and k2_final streams the
//                  divergence and the combination alone
// Shared-memory arrays are variable-major: element (v, r, c) of an R x C tile
// sits at (v*R + r)*C + c.
#pragma once

#include "fvh_kernels.cuh"
#include "fvh_tma.cuh"

namespace fvh {
namespace f2 {

struct Geo {
  int nx, ny;          // interior cells along X and Y
  int bcx[2], bcy[2];  // Bc kinds at the low/high ends of X and Y
  int dx, dy;          // physical axis ids of X and Y
  int gmax;            // deepest ghost index any state load may reach
  const Slabs* slabs;  // Dirichlet ghost values (physical axes), or nullptr
};

// 2D view of a variable-major array over [-g, nx+g) x [-g, ny'+g). Row r of
// the array holds X index r - g; column c holds Y index c - gy (gy >= g: rows
// may start with padding, so that Y index 0 and every multiple of 16 bytes
// from it sit on 16-byte boundaries).
template <typename T>
struct V2 {
  T* p;
  int g;   // ghost cells on each side
  int sx;  // row stride (the padded Y extent)
  int vs;  // variable stride
  int gy;  // column of Y index 0
  __device__ __forceinline__ int at(int x, int y) const { return (x + g) * sx + (y + gy); }
  __host__ __device__ V2<const T> c() const { return V2<const T>{p, g, sx, vs, gy}; }
};

template <typename T>
__host__ __device__ inline V2<T> make_v2(T* p, int nx, int ny, int g) {
  V2<T> v;
  v.p = p;
  v.g = g;
  v.gy = g;
  v.sx = ny + 2 * g;
  v.vs = (nx + 2 * g) * (ny + 2 * g);
  return v;
}

// Rows padded to whole 16-byte vectors: gy and the row stride rounded up to
// multiples of al elements (16 bytes).
__host__ __device__ inline int round_up(int n, int al) { return (n + al - 1) / al * al; }

template <typename T>
__host__ __device__ inline V2<T> make_v2_aligned(T* p, int nx, int ny, int g) {
  constexpr int al = 16 / (int)sizeof(T);
  V2<T> v;
  v.p = p;
  v.g = g;
  v.gy = round_up(g, al);
  v.sx = round_up(v.gy + ny + g, al);
  v.vs = (nx + 2 * g) * v.sx;
  return v;
}

// Conserved state at a (possibly ghost) cell of the 2D grid, stored as Tin
// (double for the state, the compute type for the candidate). Coordinates of
// tile points that no output needs are clamped into the ghost range first.
template <typename Tc, typename Tin>
__device__ __forceinline__ void load_state2(const Tin* __restrict__ u, const Geo& g, int x, int y, Tc* out) {
  x = min(max(x, -g.gmax), g.nx + g.gmax - 1);
  y = min(max(y, -g.gmax), g.ny + g.gmax - 1);
  if (g.slabs) {
    int i[3] = {0, 0, 0};
    i[g.dx] = x;
    i[g.dy] = y;
    const State5<Tc> s = load_state5_dirichlet<Tc, Tin>(u, g.slabs, i[0], i[1], i[2]);
#pragma unroll
    for (int v = 0; v < 5; ++v) out[v] = s.v[v];
    return;
  }
  bool fx = false, fy = false;
  const int jx = ghost_source(x, g.nx, g.bcx[0], g.bcx[1], fx);
  const int jy = ghost_source(y, g.ny, g.bcy[0], g.bcy[1], fy);
  const int plane = g.nx * g.ny;
  const int o = jx * g.ny + jy;
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    double val = (double)u[v * plane + o];
    if ((v == 1 + g.dx && fx) || (v == 1 + g.dy && fy)) val = -val;
    out[v] = (Tc)val;
  }
}

// Fallback flux at a face from the pointwise primitives of the four cells
// around it: element e of variable v at base[v * vstride + e * estride], cells
// i-2, i-1 | i, i+1. MUSCL with the limiter (fvhoe/slope_limiting.py:24-53),
// the unlimited p=1 faces, or first order (muscl = 0).
template <typename Tc>
__device__ __forceinline__ void fallback_face_flux(const Tc* base, int vstride, int estride, int muscl, int limiter,
                                                   const Phys<Tc>& ph, int dir, Tc* flo) {
  Tc wl[5], wr[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    const Tc* pv = base + v * vstride;
    const Tc a0 = pv[0], a1 = pv[estride], a2 = pv[2 * estride], a3 = pv[3 * estride];
    if (muscl && limiter == LIMITER_NONE) {
      wl[v] = ((Tc(0) + Tc(-0.25) * a0) + Tc(1) * a1) + Tc(0.25) * a2;
      wr[v] = ((Tc(0) + Tc(0.25) * a1) + Tc(1) * a2) + Tc(-0.25) * a3;
    } else if (muscl) {
      const Tc sl = limited_slope(a1 - a0, a2 - a1, limiter);
      const Tc sr = limited_slope(a2 - a1, a3 - a2, limiter);
      wl[v] = a1 + Tc(0.5) * sl;
      wr[v] = a2 - Tc(0.5) * sr;
    } else {
      wl[v] = a1;
      wr[v] = a2;
    }
  }
  riemann_flux<5>(ph, 5, wl, wr, dir, flo);
}

// Pointwise primitives of the stage input on [x0-2, x0+TX+2) x [y0-2, y0+TY+2)
// into Pw ((TX+4) x (TY+4) per variable), the inputs of the fallback fluxes
// (p = 1 reconstruction is the identity, fvhoe/solver.py:710-732).
template <typename Tc, int TX, int TY>
__device__ __forceinline__ void pointwise_tile(const double* __restrict__ u, const Geo& g, int x0, int y0, Tc* Pw,
                                               const Phys<Tc>& ph) {
  constexpr int PX = TX + 4, PY = TY + 4;
  // tiles inside the grid read the state directly, the others through the ghost maps
  const bool inside = !g.slabs && x0 >= 2 && x0 + TX + 2 <= g.nx && y0 >= 2 && y0 + TY + 2 <= g.ny;
  const int plane = g.nx * g.ny;
  for (int i = threadIdx.x; i < PX * PY; i += blockDim.x) {
    const int r = i / PY, q = i - r * PY;
    Tc uc[5], w[5];
    if (inside) {
      const double* p = u + (x0 - 2 + r) * g.ny + y0 - 2 + q;
#pragma unroll
      for (int v = 0; v < 5; ++v) uc[v] = (Tc)p[v * plane];
    } else {
      load_state2<Tc>(u, g, x0 - 2 + r, y0 - 2 + q, uc);
    }
    to_primitives(ph, 5, uc, w);
#pragma unroll
    for (int v = 0; v < 5; ++v) Pw[(v * PX + r) * PY + q] = w[v];
  }
}

// 1 in every thread of the block when a[c] && !b[c] (b nullable) holds for a
// grid cell c of [x0-1, x0+TX] x [y0-1, y0+TY].
template <int TX, int TY>
__device__ __forceinline__ int tile_any(const uint8_t* __restrict__ a, const uint8_t* __restrict__ b, const Geo& g,
                                        int x0, int y0) {
  int local = 0;
  for (int i = threadIdx.x; i < (TX + 2) * (TY + 2); i += blockDim.x) {
    const int r = i / (TY + 2), q = i - r * (TY + 2);
    const int x = x0 - 1 + r, y = y0 - 1 + q;
    if (x >= 0 && x < g.nx && y >= 0 && y < g.ny) {
      const int o = x * g.ny + y;
      local |= (a[o] && !(b && b[o])) ? 1 : 0;
    }
  }
  return __syncthreads_or(local);
}

template <int a, int b>
struct Max {
  static constexpr int value = a > b ? a : b;
};

__host__ __device__ constexpr int up4(int n) { return (n + 3) / 4 * 4; }

// N (1, 2 or 4) consecutive elements at an address aligned to N elements, in
// as few 8- or 16-byte accesses as the type allows.
template <int N>
__device__ __forceinline__ void ldn(const float* p, float* o) {
  if constexpr (N == 4) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    o[0] = t.x, o[1] = t.y, o[2] = t.z, o[3] = t.w;
  } else if constexpr (N == 2) {
    const float2 t = *reinterpret_cast<const float2*>(p);
    o[0] = t.x, o[1] = t.y;
  } else {
    o[0] = p[0];
  }
}
template <int N>
__device__ __forceinline__ void ldn(const double* p, double* o) {
  if constexpr (N == 1) {
    o[0] = p[0];
  } else {
#pragma unroll
    for (int a = 0; a < N; a += 2) {
      const double2 t = *reinterpret_cast<const double2*>(p + a);
      o[a] = t.x, o[a + 1] = t.y;
    }
  }
}
template <int N>
__device__ __forceinline__ void stn(float* p, const float* o) {
  if constexpr (N == 4) {
    *reinterpret_cast<float4*>(p) = make_float4(o[0], o[1], o[2], o[3]);
  } else if constexpr (N == 2) {
    *reinterpret_cast<float2*>(p) = make_float2(o[0], o[1]);
  } else {
    p[0] = o[0];
  }
}
template <int N>
__device__ __forceinline__ void stn(double* p, const double* o) {
  if constexpr (N == 1) {
    p[0] = o[0];
  } else {
#pragma unroll
    for (int a = 0; a < N; a += 2) *reinterpret_cast<double2*>(p + a) = make_double2(o[a], o[a + 1]);
  }
}

// Output rows per thread of the sweeps along the strided axis (sweepv's M),
// as measured fastest on B200 (KH 2048^2 p=5 and 4096^2 p=7, both forms, all
// variants bit-identical): three in the FP64 primitive tiles, one in the FP32
// ones; in the flux tile two for the 7- and 9-tap rules of p >= 6, else one.
template <typename Tc>
constexpr int mrow_prims() {
  return sizeof(Tc) == 8 ? 3 : 1;
}
constexpr int mrow_flux(int kc) { return kc >= 7 ? 2 : 1; }

// One element from global to shared memory by an asynchronous copy (4 or 8
// bytes, cached in L1), and the wait for all of this thread's copies.
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* smem_dst, const T* gmem_src) {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "4- or 8-byte elements");
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"((uint32_t)__cvta_generic_to_shared(smem_dst)),
               "l"(gmem_src), "n"(sizeof(T))
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Elements per shared-memory vector: one 16-byte access (4 floats, 2 doubles).
template <typename Tc>
struct VecW {
  static constexpr int value = 16 / (int)sizeof(Tc);
};

// One stencil sweep over the five variable planes of a shared tile, VW
// consecutive outputs of a row per thread:
//   out(v, r, q) = sum_k w[k] in(v, r + k AR, OFF + q + k (1 - AR)),  r < NR, q < VW NG,
// each sum accumulated from k = 0 upwards as a one-output loop accumulates it,
// so every output is rounded exactly as before. AR = 1 puts the taps along the
// strided axis (one aligned vector, or two when OFF is not a multiple of VW,
// per tap), AR = 0 along the contiguous axis (one window of vectors per output
// group). Row strides IS and variable strides IVS are multiples of VW; outputs
// past the caller's column count land in the padding of the output rows.
// IN_LIM bounds the elements the sweep may read from `in`. epi(v, r, q, acc)
// stores the VW sums. M > 1 (AR = 1 only): each thread takes M consecutive
// output rows and reads each of their M + K - 1 input rows once (a sliding
// window along the strided axis), every output still summed from tap 0 up.
template <typename Tc, int VW, int K, int AR, int OFF, int NR, int NG, int IS, int IVS, int IN_LIM, int M = 1,
          typename Epi>
__device__ __forceinline__ void sweepv(const Tc* __restrict__ in, const Tc* __restrict__ w, Epi epi) {
  constexpr int S = OFF % VW, B0 = OFF - S;
  constexpr int NW = AR ? (S + 2 * VW - 1) / VW : (S + K + 2 * VW - 2) / VW;
  static_assert(IS % VW == 0 && IVS % VW == 0, "rows and planes must hold whole vectors");
  static_assert(4 * IVS + (NR - 1 + (AR ? K - 1 : 0)) * IS + B0 + VW * (NG - 1) + VW * NW <= IN_LIM,
                "sweep reads past its shared region");
  static_assert(M == 1 || AR == 1, "row blocking applies to sweeps along the strided axis");
  if constexpr (M > 1) {
    constexpr int NRM = (NR + M - 1) / M;
    for (int i = threadIdx.x; i < NRM * NG; i += blockDim.x) {
      const int r0 = (i / NG) * M, q = (i - (i / NG) * NG) * VW;
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        const Tc* src = in + v * IVS + B0 + q;
        Tc acc[M][VW];
#pragma unroll
        for (int m = 0; m < M; ++m)
#pragma unroll
          for (int j = 0; j < VW; ++j) acc[m][j] = Tc(0);
#pragma unroll
        for (int n = 0; n < M + K - 1; ++n) {
          const int row = min(r0 + n, NR - 1 + K - 1);  // rows past the last output's window feed no output
          Tc x[VW * NW];
#pragma unroll
          for (int u = 0; u < NW; ++u) ldn<VW>(src + row * IS + VW * u, x + VW * u);
#pragma unroll
          for (int m = 0; m < M; ++m) {
            const int k = n - m;
            if (k >= 0 && k < K) {
#pragma unroll
              for (int j = 0; j < VW; ++j) acc[m][j] = acc[m][j] + w[k] * x[S + j];
            }
          }
        }
#pragma unroll
        for (int m = 0; m < M; ++m)
          if (r0 + m < NR) epi(v, r0 + m, q, acc[m]);
      }
    }
    return;
  }
  for (int i = threadIdx.x; i < NR * NG; i += blockDim.x) {
    const int r = i / NG, q = (i - r * NG) * VW;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const Tc* src = in + v * IVS + r * IS + B0 + q;
      Tc acc[VW];
#pragma unroll
      for (int j = 0; j < VW; ++j) acc[j] = Tc(0);
      if constexpr (AR) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
          Tc x[VW * NW];
#pragma unroll
          for (int n = 0; n < NW; ++n) ldn<VW>(src + k * IS + VW * n, x + VW * n);
#pragma unroll
          for (int j = 0; j < VW; ++j) acc[j] = acc[j] + w[k] * x[S + j];
        }
      } else {
        Tc x[VW * NW];
#pragma unroll
        for (int n = 0; n < NW; ++n) ldn<VW>(src + VW * n, x + VW * n);
#pragma unroll
        for (int k = 0; k < K; ++k)
#pragma unroll
          for (int j = 0; j < VW; ++j) acc[j] = acc[j] + w[k] * x[S + j + k];
      }
      epi(v, r, q, acc);
    }
  }
}

// Tile dimensions of the primitive computation producing OX x OY outputs
// with degree P (centre / transverse rules of radius RC = P / 2) in the
// compute type Tc. Rows are padded to whole 16-byte vectors (LYS, PYS, OYS);
// PAD is slack after each buffer for the reads that feed padding outputs.
template <typename Tc, int P, int OX, int OY>
struct PrimsDims {
  static constexpr int VW = VecW<Tc>::value;
  static constexpr int RC = P / 2;
  static constexpr int LX = OX + 4 * RC, LY = OY + 4 * RC;  // loaded state
  static constexpr int CX = OX + 2 * RC;                    // after the X centre sweep: CX x LY
  static constexpr int PY = OY + 2 * RC;                    // after the Y centre sweep: CX x PY
  static constexpr int LYS = (LY + VW - 1) / VW * VW, PYS = (PY + VW - 1) / VW * VW, OYS = (OY + VW - 1) / VW * VW;
  static constexpr int PAD = 16;
  // WALK (rules of 5 or more taps, p >= 4): the loaded state is never stored,
  // its columns are swept along X as they arrive; with 3-tap rules the state
  // tile is staged in A first (measured faster there: the column walks leave
  // each thread a long chain of loads for little saved shared-memory work).
  static constexpr bool WALK = 2 * RC + 1 >= 5;
  // A: the staged state LX x LY (without WALK), after the Y centre sweep
  // CX x PY, after the Y transverse sweep OX x OY; B: after the X centre sweep
  // CX x LY, after the X transverse sweep OX x PY
  static constexpr int A = Max<Max<(WALK ? 0 : LX * LYS), CX * PYS>::value, OX * OYS>::value * 5 + PAD;
  static constexpr int B = Max<CX * LYS, OX * PYS>::value * 5 + PAD;
  // row segments per column in the X centre sweep: enough column segments
  // (five variables per column) for one per thread of a 256-thread block
  static constexpr int NS = (256 + 5 * LY - 1) / (5 * LY);
};

// X centre sweep of a tile straight from the state: a thread takes one
// variable of one column and SEG consecutive output rows, loads their
// SEG + KC - 1 state rows once, in order, into a register window, and stores
// each sum (accumulated from tap 0 upwards, as every sweep accumulates) into
// out, CX x LYS per variable. load(r, q, v): variable v of tile row r, column q.
template <typename Tc, int KC, int CX, int LY, int LYS, int NS, typename Load>
__device__ __forceinline__ void centre_x_columns(Tc* __restrict__ out, const Tc* __restrict__ w, Load load) {
  constexpr int SEG = (CX + NS - 1) / NS;
  for (int i = threadIdx.x; i < NS * 5 * LY; i += blockDim.x) {
    const int q = i % LY, rest = i / LY, v = rest % 5, r0 = (rest / 5) * SEG;
    Tc win[KC];
#pragma unroll
    for (int k = 0; k < KC - 1; ++k) win[k] = load(r0 + k, q, v);
#pragma unroll
    for (int m = 0; m < SEG; ++m) {
      if (r0 + m < CX) {
        win[KC - 1] = load(r0 + m + KC - 1, q, v);
        Tc acc = Tc(0);
#pragma unroll
        for (int k = 0; k < KC; ++k) acc = acc + w[k] * win[k];
        out[(v * CX + r0 + m) * LYS + q] = acc;
#pragma unroll
        for (int k = 0; k < KC - 1; ++k) win[k] = win[k + 1];
      }
    }
  }
}

// Variable v of the conserved state at a (possibly ghost) cell, as
// load_state2 gives it.
template <typename Tc, typename Tin>
__device__ __forceinline__ Tc load_var2(const Tin* __restrict__ u, const Geo& g, int x, int y, int v) {
  if (g.slabs) {
    Tc s[5];
    load_state2<Tc>(u, g, x, y, s);
    return s[v];
  }
  x = min(max(x, -g.gmax), g.nx + g.gmax - 1);
  y = min(max(y, -g.gmax), g.ny + g.gmax - 1);
  bool fx = false, fy = false;
  const int jx = ghost_source(x, g.nx, g.bcx[0], g.bcx[1], fx);
  const int jy = ghost_source(y, g.ny, g.bcy[0], g.bcy[1], fy);
  double val = (double)u[v * (g.nx * g.ny) + jx * g.ny + jy];
  if ((v == 1 + g.dx && fx) || (v == 1 + g.dy && fy)) val = -val;
  return (Tc)val;
}

// W on [x0, x0+OX) x [y0, y0+OY), computed in two shared buffers; the result
// is left in A as an OX x OY tile with row stride OYS. Rules: centre c and
// transverse t (KC taps). The sweeps run VW outputs per thread (sweepv), each
// output summed in the order of a one-output loop.
template <typename Tc, int P, int OX, int OY, int KC, typename Tin>
__device__ __forceinline__ void primitives_tile(const Tin* __restrict__ u, const Geo& g, int x0, int y0, Tc* A,
                                                Tc* B, const Rule<Tc, KC>& c, const Rule<Tc, KC>& t,
                                                const Phys<Tc>& ph) {
  using D = PrimsDims<Tc, P, OX, OY>;
  constexpr int RC = D::RC, VW = VecW<Tc>::value;
  const int nt = blockDim.x;
  // 1. the state with 2*RC ghosts around the tile, swept along X: B, CX x
  // LYS; staged in A first (3-tap rules) or swept as its columns arrive
  // (WALK). A tile whose loaded box lies inside the grid (most tiles) reads
  // the state directly; the others resolve every point through the ghost maps.
  const int lx0 = x0 - 2 * RC, ly0 = y0 - 2 * RC;
  const bool inside = !g.slabs && lx0 >= 0 && lx0 + D::LX <= g.nx && ly0 >= 0 && ly0 + D::LY <= g.ny;
  if constexpr (!D::WALK) {
    // the state tile staged in A (LX x LYS), then the X centre sweep into B
    if (inside) {
      const int plane = g.nx * g.ny;
      for (int i = threadIdx.x; i < D::LX * D::LY; i += nt) {
        const int r = i / D::LY, q = i - r * D::LY;
        const Tin* p = u + (lx0 + r) * g.ny + ly0 + q;
        Tin sv[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) sv[v] = p[v * plane];
#pragma unroll
        for (int v = 0; v < 5; ++v) A[(v * D::LX + r) * D::LYS + q] = (Tc)sv[v];
      }
    } else {
      for (int i = threadIdx.x; i < D::LX * D::LY; i += nt) {
        const int r = i / D::LY, q = i - r * D::LY;
        Tc sv[5];
        load_state2<Tc>(u, g, lx0 + r, ly0 + q, sv);
#pragma unroll
        for (int v = 0; v < 5; ++v) A[(v * D::LX + r) * D::LYS + q] = sv[v];
      }
    }
    __syncthreads();
    sweepv<Tc, VW, KC, 1, 0, D::CX, D::LYS / VW, D::LYS, D::LX * D::LYS, D::A, mrow_prims<Tc>()>(
        A, c.w, [&](int v, int r, int q, const Tc* acc) { stn<VW>(B + (v * D::CX + r) * D::LYS + q, acc); });
  } else if (inside) {
    const int plane = g.nx * g.ny;
    const Tin* base = u + lx0 * g.ny + ly0;
    centre_x_columns<Tc, KC, D::CX, D::LY, D::LYS, D::NS>(
        B, c.w, [&](int r, int q, int v) { return (Tc)base[v * plane + r * g.ny + q]; });
  } else if (!g.slabs) {
    // the ghost maps are separable: each tile row's and column's source
    // index and mirror flag (j << 1 | flip), resolved once into A (free until
    // the Y centre sweep), as load_state2 resolves them point by point
    int* const mx = reinterpret_cast<int*>(A);
    int* const my = mx + D::LX;
    for (int i = threadIdx.x; i < D::LX + D::LY; i += nt) {
      bool f = false;
      if (i < D::LX) {
        const int x = min(max(lx0 + i, -g.gmax), g.nx + g.gmax - 1);
        const int j = ghost_source(x, g.nx, g.bcx[0], g.bcx[1], f);
        mx[i] = (j << 1) | (f ? 1 : 0);
      } else {
        const int y = min(max(ly0 + i - D::LX, -g.gmax), g.ny + g.gmax - 1);
        const int j = ghost_source(y, g.ny, g.bcy[0], g.bcy[1], f);
        my[i - D::LX] = (j << 1) | (f ? 1 : 0);
      }
    }
    __syncthreads();
    const int plane = g.nx * g.ny;
    centre_x_columns<Tc, KC, D::CX, D::LY, D::LYS, D::NS>(B, c.w, [&](int r, int q, int v) {
      const int a = mx[r], b = my[q];
      double val = (double)u[v * plane + (a >> 1) * g.ny + (b >> 1)];
      if ((v == 1 + g.dx && (a & 1)) || (v == 1 + g.dy && (b & 1))) val = -val;
      return (Tc)val;
    });
  } else {
    centre_x_columns<Tc, KC, D::CX, D::LY, D::LYS, D::NS>(
        B, c.w, [&](int r, int q, int v) { return load_var2<Tc>(u, g, lx0 + r, ly0 + q, v); });
  }
  __syncthreads();
  // 2. centre sweep along Y, then primitives: A, CX x PYS
  {
    constexpr int NG = D::PYS / VW, NW = (KC + 2 * VW - 2) / VW;
    static_assert(4 * D::CX * D::LYS + (D::CX - 1) * D::LYS + VW * (NG - 1 + NW) <= D::B,
                  "centre sweep reads past its shared region");
    for (int i = threadIdx.x; i < D::CX * NG; i += nt) {
      const int r = i / NG, q = (i - r * NG) * VW;
      Tc acc[5][VW];
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        Tc x[VW * NW];
#pragma unroll
        for (int n = 0; n < NW; ++n) ldn<VW>(B + (v * D::CX + r) * D::LYS + q + VW * n, x + VW * n);
#pragma unroll
        for (int j = 0; j < VW; ++j) {
          acc[v][j] = Tc(0);
#pragma unroll
          for (int k = 0; k < KC; ++k) acc[v][j] = acc[v][j] + c.w[k] * x[j + k];
        }
      }
      Tc w[5][VW];
#pragma unroll
      for (int j = 0; j < VW; ++j) {
        Tc a5[5], w5[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) a5[v] = acc[v][j];
        to_primitives(ph, 5, a5, w5);
#pragma unroll
        for (int v = 0; v < 5; ++v) w[v][j] = w5[v];
      }
#pragma unroll
      for (int v = 0; v < 5; ++v) stn<VW>(A + (v * D::CX + r) * D::PYS + q, w[v]);
    }
  }
  __syncthreads();
  // 3. transverse sweep along X: B, OX x PYS
  sweepv<Tc, VW, KC, 1, 0, OX, D::PYS / VW, D::PYS, D::CX * D::PYS, D::A, mrow_prims<Tc>()>(
      A, t.w, [&](int v, int r, int q, const Tc* acc) { stn<VW>(B + (v * OX + r) * D::PYS + q, acc); });
  __syncthreads();
  // 4. transverse sweep along Y, into A as an OX x OYS tile
  sweepv<Tc, VW, KC, 0, 0, OX, D::OYS / VW, D::PYS, OX * D::PYS, D::B>(
      B, t.w, [&](int v, int r, int q, const Tc* acc) { stn<VW>(A + (v * OX + r) * D::OYS + q, acc); });
  __syncthreads();
}

__device__ __forceinline__ void reduce_keys_and_publish(unsigned long long cfl_key, const unsigned long long* kmax,
                                                        const unsigned long long* kmin, const ReduceSpec& rs,
                                                        Scalars* sc) {
  __shared__ unsigned long long s_keys[8][11];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned long long cm = warp_max_u64(cfl_key);
  if (lane == 0) s_keys[warp][0] = cm;
#pragma unroll
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
    unsigned long long acc[11];
    for (int k = 0; k < 11; ++k) acc[k] = s_keys[0][k];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
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

// ---------------------------------------------------------------------------
// k2_primitives: W over [-gw_out, n+gw_out)^2 in tiles of TX x TY outputs,
// with the CFL maximum and the per-variable extrema (REDUCE).
// ---------------------------------------------------------------------------
// Tile functions: the body of each kernel for the tile (bx, by) (bx along Y,
// by along X), so that one-problem launches (one tile per block) and the
// batched ensemble (blocks looping over the tiles of many problems) share it.
// Tin: double for the stage input, the compute type for the candidate
template <typename Tc, int P, int TX, int TY, int KC, bool REDUCE, typename Tin = double>
__device__ __forceinline__ void tile2_primitives(const Tin* __restrict__ u, Geo g, V2<Tc> W, int gw_out,
                                                 Rule<Tc, KC> c, Rule<Tc, KC> t, Phys<Tc> ph, ReduceSpec rs,
                                                 Scalars* __restrict__ sc, int bx, int by, unsigned char* smem_raw) {
  using D = PrimsDims<Tc, P, TX, TY>;
  Tc* A = reinterpret_cast<Tc*>(smem_raw);
  Tc* B = A + D::A;
  const int x0 = -gw_out + by * TX;
  const int y0 = -gw_out + bx * TY;
  primitives_tile<Tc, P, TX, TY, KC>(u, g, x0, y0, A, B, c, t, ph);
  unsigned long long cfl_key = 0ull, kmax[5], kmin[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    kmax[v] = 0ull;
    kmin[v] = ~0ull;
  }
  for (int i = threadIdx.x; i < TX * TY; i += blockDim.x) {
    const int r = i / TY, q = i - r * TY;
    const int x = x0 + r, y = y0 + q;
    if (x >= g.nx + gw_out || y >= g.ny + gw_out) continue;
    Tc w[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) w[v] = A[(v * TX + r) * D::OYS + q];
    Tc* o = W.p + W.at(x, y);
#pragma unroll
    for (int v = 0; v < 5; ++v) o[v * W.vs] = w[v];
    if constexpr (REDUCE) {
      // boxes in (X, Y, 0) coordinates
      if (rs.cfl && in_box(rs.cfl_box, x, y, 0)) {
        const unsigned long long k = order_key((double)cfl_speed(ph, w, (Tc)rs.ndim));
        cfl_key = k > cfl_key ? k : cfl_key;
      }
      if (rs.extrema && in_box(rs.ext_box, x, y, 0)) {
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          const unsigned long long k = order_key((double)w[v]);
          kmax[v] = k > kmax[v] ? k : kmax[v];
          kmin[v] = k < kmin[v] ? k : kmin[v];
        }
      }
    }
  }
  if constexpr (REDUCE) reduce_keys_and_publish(cfl_key, kmax, kmin, rs, sc);
}

template <typename Tc, int P, int TX, int TY, int KC, bool REDUCE, typename Tin = double>
__global__ void __launch_bounds__(256)
    k2_primitives(const Tin* __restrict__ u, Geo g, V2<Tc> W, int gw_out, Rule<Tc, KC> c, Rule<Tc, KC> t,
                  Phys<Tc> ph, ReduceSpec rs, Scalars* __restrict__ sc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  tile2_primitives<Tc, P, TX, TY, KC, REDUCE, Tin>(u, g, W, gw_out, c, t, ph, rs, sc, blockIdx.x, blockIdx.y,
                                                   smem_raw);
}

// ---------------------------------------------------------------------------
// k2_fluxes: high-order X- and Y-face fluxes of a TX x TY cell tile, and the
// candidate u* = u + dt L(F) of its cells.
// ---------------------------------------------------------------------------
// Shared memory of the flux tile: three regions, each reused once its tile is
// consumed, with rows padded to whole 16-byte vectors (4 elements):
//   region 0: W tile -> X-face Riemann fluxes -> Y-face Riemann fluxes (-> pointwise tile)
//   region 1: X centre sweep -> X face fluxes FX
//   region 2: Y centre sweep -> Y face fluxes GY
template <int P, int TX, int TY>
struct FluxDims {
  static_assert(TY % 4 == 0, "tile columns must hold whole vectors");
  static constexpr int R = (P + 1) / 2;  // face-rule radius
  static constexpr int RC = P / 2;       // centre / transverse radius
  static constexpr int KF = 2 * R + 1;
  static constexpr int H = Max<R + 1, 2 * RC>::value;  // W halo
  static constexpr int HY = up4(H);                    // W halo on the low Y side (aligned rows)
  static constexpr int WX = TX + 2 * H, WYS = up4(HY + TY + H);
  // X faces: centre sweep along Y on rows [x0-1-R, x0+TX+R], cols [y0-RC, y0+TY+RC)
  static constexpr int AXR = TX + 2 * R + 2, AXC = TY + 2 * RC, AXS = up4(AXC);
  // Riemann fluxes at faces x0..x0+TX on those cols (row stride AXS)
  static constexpr int BXR = TX + 1;
  // Y faces: centre sweep along X on rows [x0-RC, x0+TX+RC), cols [y0-1-R, y0+TY+R]
  static constexpr int AYR = TX + 2 * RC, AYC = TY + 2 * R + 2, AYS = up4(AYC);
  // Riemann fluxes at faces y0..y0+TY of those rows; the Y face fluxes GY (TX rows)
  static constexpr int BYR = TX + 2 * RC, BYS = up4(TY + 1), GYS = up4(TY + 1);
  static constexpr int PAD = 16;  // slack after each region for reads that feed padding outputs
  static constexpr int S0 =
      Max<Max<WX * WYS, BXR * AXS>::value, Max<BYR * BYS, (TX + 4) * (TY + 4)>::value>::value * 5 + PAD;
  static constexpr int S1 = Max<AXR * AXS, (TX + 1) * TY>::value * 5 + PAD;
  static constexpr int S2 = Max<AYR * AYS, TX * GYS>::value * 5 + PAD;
  static constexpr int TOTAL = S0 + S1 + S2;  // elements of the compute type
  // bytes after the three regions that a block with predicted flags needs: two
  // counters and the lists of the faces that take the fallback flux
  static constexpr int LIST = 16 + 2 * ((TX + 1) * TY + TX * (TY + 1));
  // resident blocks per SM that the shared memory allows (227 KB per SM, 128
  // bytes of alignment slack per block), at most 4 (FP32) or 3 (FP64): the
  // launch bounds give each thread the registers of that occupancy
  template <typename Tc>
  static constexpr int blocks() {
    constexpr int cap = sizeof(Tc) == 4 ? 4 : 3;
    constexpr int fit = (227 * 1024) / (TOTAL * (int)sizeof(Tc) + 128);
    return fit < cap ? fit : cap;
  }
};

// CHX, CHY: consecutive faces per thread in the two Riemann phases (sliding
// windows along X and Y); one in FP64, whose states take twice the registers,
// and fewer along Y for the 9-tap face rules when 4 blocks per SM leave 64
// registers (no register spills)
template <typename Tc, int P, int TX, int TY, int KC, int KF, int CHX = (sizeof(Tc) == 4 ? 3 : 1),
          int CHY = (sizeof(Tc) == 4 ? (KF >= 9 && FluxDims<P, TX, TY>::template blocks<Tc>() >= 4 ? 2 : 4) : 1)>
__device__ __forceinline__ void tile2_fluxes(V2<const Tc> W, const double* __restrict__ u, Geo g, V2<Tc> F, V2<Tc> G,
                                             Tc* __restrict__ ustar, Rule<Tc, KC> c, Rule<Tc, KC> t,
                                             Rule<Tc, KF> lrule, Rule<Tc, KF> rrule, Phys<Tc> ph, double cx,
                                             double cy, double dt, const uint8_t* __restrict__ pred, int muscl,
                                             int limiter, int bx, int by, unsigned char* smem_raw,
                                             const CUtensorMap* wmap = nullptr, uint64_t* bar = nullptr,
                                             unsigned int* tma_err = nullptr, unsigned int* fallback_count = nullptr) {
  using D = FluxDims<P, TX, TY>;
  constexpr int R = D::R, RC = D::RC, H = D::H, HY = D::HY, VW = VecW<Tc>::value;
  Tc* const S0 = reinterpret_cast<Tc*>(smem_raw);
  Tc* const S1 = S0 + D::S0;
  Tc* const S2 = S1 + D::S1;
  Tc* const Ws = S0;  // W tile, WX x WYS: element (r, c) is W(x0-H+r, y0-HY+c)
  Tc* const AX = S1;  // X centre sweep, AXR x AXS
  Tc* const AY = S2;  // Y centre sweep, AYR x AYS
  Tc* const BX = S0;  // X-face Riemann fluxes, BXR x AXS
  Tc* const FX = S1;  // X face fluxes, (TX+1) x TY
  Tc* const BY = S0;  // Y-face Riemann fluxes, BYR x BYS
  Tc* const GY = S2;  // Y face fluxes, TX x GYS
  const int nt = blockDim.x;
  const int x0 = by * TX, y0 = bx * TY;
  // W tile (W holds gW >= H ghosts). With a tensor map: one TMA box copy of
  // rows x0-H.. and columns y0-HY.. (16-byte aligned: y0, HY and W.gy are
  // multiples of 16 bytes), rows past the array read as zero and padding
  // columns as the zeros they were set to; those points feed no output.
  // Without: per-thread loads, points that no output needs clamped into
  // range, VW columns per access where W's rows are 16-byte aligned.
  if (wmap) {
    tma::stage_box(Ws, wmap, y0 - HY + W.gy, x0 - H + W.g, 0, (uint32_t)(5 * D::WX * D::WYS * sizeof(Tc)),
                   (int)sizeof(Tc), bar, tma_err);
  } else {
    constexpr int NG = D::WYS / VW;
    const bool vec = ((W.gy | W.sx | W.vs) & (VW - 1)) == 0 && (reinterpret_cast<uintptr_t>(W.p) & 15) == 0;
    for (int i = threadIdx.x; i < D::WX * NG; i += nt) {
      const int r = i / NG, cq = (i - r * NG) * VW;
      const int x = min(max(x0 - H + r, -W.g), g.nx + W.g - 1), y = y0 - HY + cq;
      Tc val[5][VW];
      if (vec && y >= -W.g && y + VW - 1 <= g.ny + W.g - 1) {
        const Tc* p = W.p + W.at(x, y);
#pragma unroll
        for (int v = 0; v < 5; ++v) ldn<VW>(p + v * W.vs, val[v]);
      } else {
#pragma unroll
        for (int j = 0; j < VW; ++j) {
          const Tc* p = W.p + W.at(x, min(max(y + j, -W.g), g.ny + W.g - 1));
#pragma unroll
          for (int v = 0; v < 5; ++v) val[v][j] = p[v * W.vs];
        }
      }
#pragma unroll
      for (int v = 0; v < 5; ++v) stn<VW>(Ws + (v * D::WX + r) * D::WYS + cq, val[v]);
    }
  }
  __syncthreads();
  // centre sweeps of both directions from the W tile
  // X faces: AX(r, q) at (x0-1-R+r, y0-RC+q), taps along Y
  sweepv<Tc, VW, KC, 0, HY - 2 * RC, D::AXR, D::AXS / VW, D::WYS, D::WX * D::WYS, D::S0 - (H - 1 - R) * D::WYS>(
      Ws + (H - 1 - R) * D::WYS, c.w,
      [&](int v, int r, int q, const Tc* acc) { stn<VW>(AX + (v * D::AXR + r) * D::AXS + q, acc); });
  // Y faces: AY(r, q) at (x0-RC+r, y0-1-R+q), taps along X
  sweepv<Tc, VW, KC, 1, HY - 1 - R, D::AYR, D::AYS / VW, D::WYS, D::WX * D::WYS, D::S0 - (H - 2 * RC) * D::WYS,
         mrow_flux(KC)>(
      Ws + (H - 2 * RC) * D::WYS, c.w,
      [&](int v, int r, int q, const Tc* acc) { stn<VW>(AY + (v * D::AYR + r) * D::AYS + q, acc); });
  __syncthreads();
  // ---- X faces: face f (x = x0+f) between cells x0+f-1 and x0+f; AX row of
  // cell x is x - (x0-1-R). Each thread takes one column q and CHX
  // consecutive faces, sliding along X: per variable, the rows f0 .. f0+CHX+KF-1
  // are read once into registers and feed all CHX faces (warps run along the
  // columns, so the scalar reads are conflict-free); every face state is
  // summed from tap 0 upwards, as a one-face loop sums it.
  {
    constexpr int NCH = (D::BXR + CHX - 1) / CHX;
    for (int i = threadIdx.x; i < NCH * D::AXC; i += nt) {
      const int ch = i / D::AXC, q = i - ch * D::AXC;
      const int f0 = ch * CHX;
      Tc wl[CHX][5], wr[CHX][5];
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        Tc x[CHX + KF];
#pragma unroll
        for (int n = 0; n < CHX + KF; ++n) x[n] = AX[(v * D::AXR + min(f0 + n, D::AXR - 1)) * D::AXS + q];
#pragma unroll
        for (int j = 0; j < CHX; ++j) {
          Tc a = Tc(0), b = Tc(0);
#pragma unroll
          for (int k = 0; k < KF; ++k) {
            a = a + rrule.w[k] * x[j + k];
            b = b + lrule.w[k] * x[j + 1 + k];
          }
          wl[j][v] = a;
          wr[j][v] = b;
        }
      }
#pragma unroll
      for (int j = 0; j < CHX; ++j) {
        if (f0 + j >= D::BXR) break;
        Tc fl[5];
        riemann_flux<5>(ph, 5, wl[j], wr[j], g.dx, fl);
#pragma unroll
        for (int v = 0; v < 5; ++v) BX[(v * D::BXR + f0 + j) * D::AXS + q] = fl[v];
      }
    }
  }
  __syncthreads();
  // X face fluxes: transverse sweep along Y -> FX and F (owned faces)
  sweepv<Tc, VW, KC, 0, 0, D::BXR, TY / VW, D::AXS, D::BXR * D::AXS, D::S0>(
      BX, t.w, [&](int v, int f, int q, const Tc* acc) {
        stn<VW>(FX + (v * (TX + 1) + f) * TY + q, acc);
        const int x = x0 + f;
        if ((f < TX || x == g.nx) && x <= g.nx) {
          Tc* o = F.p + F.at(x, y0 + q) + v * F.vs;
#pragma unroll
          for (int j = 0; j < VW; ++j)
            if (y0 + q + j < g.ny) o[j] = acc[j];
        }
      });
  __syncthreads();
  // ---- Y faces: face f (y = y0+f) between cells y0+f-1 and y0+f; AY column
  // of cell y is y - (y0-1-R). Each thread takes one row r and CHY consecutive
  // faces, sliding along Y: per variable the columns f0 .. f0+CHY+KF-1 are
  // read once (in the widest vectors that tile a chunk) and feed all CHY
  // faces, summed from tap 0 upwards.
  {
    constexpr int NCH = (TY + 1 + CHY - 1) / CHY;
    constexpr int LW = CHY % VW == 0 ? VW : (CHY % 2 == 0 ? 2 : 1);  // load width
    constexpr int NWY = (CHY + KF + LW - 1) / LW;  // loads covering columns f0 .. f0+CHY+KF-1
    static_assert(D::AYS % VW == 0 && D::BYS % VW == 0, "rows must hold whole vectors");
    static_assert(5 * D::AYR * D::AYS + (NCH - 1) * CHY + NWY * LW - D::AYS <= D::S2,
                  "Y-face reads past their shared region");
    static_assert((NCH - 1) * CHY + CHY <= D::BYS, "Y-face chunks must fit the padded rows");
    for (int i = threadIdx.x; i < D::BYR * NCH; i += nt) {
      const int r = i / NCH, f0 = (i - r * NCH) * CHY;
      Tc wl[CHY][5], wr[CHY][5];
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        Tc x[NWY * LW];
#pragma unroll
        for (int n = 0; n < NWY; ++n) ldn<LW>(AY + (v * D::AYR + r) * D::AYS + f0 + n * LW, x + n * LW);
#pragma unroll
        for (int j = 0; j < CHY; ++j) {
          Tc a = Tc(0), b = Tc(0);
#pragma unroll
          for (int k = 0; k < KF; ++k) {
            a = a + rrule.w[k] * x[j + k];
            b = b + lrule.w[k] * x[j + 1 + k];
          }
          wl[j][v] = a;
          wr[j][v] = b;
        }
      }
#pragma unroll
      for (int j = 0; j < CHY; ++j) {
        Tc fl[5];
        riemann_flux<5>(ph, 5, wl[j], wr[j], g.dy, fl);
#pragma unroll
        for (int v = 0; v < 5; ++v) BY[(v * D::BYR + r) * D::BYS + f0 + j] = fl[v];
      }
    }
  }
  __syncthreads();
  // Y face fluxes: transverse sweep along X -> GY and G (owned faces)
  sweepv<Tc, VW, KC, 1, 0, TX, D::GYS / VW, D::BYS, D::BYR * D::BYS, D::S0, mrow_flux(KC)>(
      BY, t.w, [&](int v, int r, int f, const Tc* acc) {
        stn<VW>(GY + (v * TX + r) * D::GYS + f, acc);
        const int x = x0 + r;
        if (x < g.nx) {
          Tc* o = G.p + G.at(x, y0 + f) + v * G.vs;
#pragma unroll
          for (int j = 0; j < VW; ++j) {
            // faces y0..y0+TY-1, and y0+TY when it is the last face of the grid;
            // columns past TY are padding
            const int fj = f + j, y = y0 + fj;
            if (fj <= TY && y <= g.ny && (fj < TY || y == g.ny)) o[j] = acc[j];
          }
        }
      });
  if (!ustar) return;
  __syncthreads();
  // candidate u* = u + dt (0 + cx (F[i+1]-F[i]) + cy (G[j+1]-G[j])), VW cells per thread
  {
    const int plane = g.nx * g.ny;
    for (int i = threadIdx.x; i < TX * (TY / VW); i += nt) {
      const int r = i / (TY / VW), q = (i - r * (TY / VW)) * VW;
      const int x = x0 + r;
      if (x >= g.nx) continue;
      const int o = x * g.ny + y0 + q;
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        Tc a[VW], b[VW], e[2 * VW];
        ldn<VW>(FX + (v * (TX + 1) + r) * TY + q, a);
        ldn<VW>(FX + (v * (TX + 1) + r + 1) * TY + q, b);
        ldn<VW>(GY + (v * TX + r) * D::GYS + q, e);
        ldn<VW>(GY + (v * TX + r) * D::GYS + q + VW, e + VW);
#pragma unroll
        for (int j = 0; j < VW; ++j) {
          if (y0 + q + j >= g.ny) continue;
          Tc d = Tc(0);
          d = d + (Tc)cx * (b[j] - a[j]);
          d = d + (Tc)cy * (e[j + 1] - e[j]);
          ustar[v * plane + o + j] = (Tc)(u[v * plane + o + j] + dt * (double)d);
        }
      }
    }
  }
  // predicted cells: their faces take the fallback flux now, blended as the
  // final pass would (the candidate above keeps the high-order fluxes). The
  // faces are gathered into two lists first so that whole warps solve them
  // (in place, a warp with one such face would run a full solve for it); the
  // lists take FluxDims::LIST bytes after the three regions, which a launch
  // that passes pred allocates.
  if (!pred || !tile_any<TX, TY>(pred, nullptr, g, x0, y0)) return;
  constexpr int PWX = TX + 4, PWY = TY + 4;
  static_assert(PWX * PWY * 5 <= D::S0, "pointwise tile must fit in region 0");
  Tc* Pw = Ws;
  int* nface = reinterpret_cast<int*>(smem_raw + (size_t)D::TOTAL * sizeof(Tc));
  uint16_t* xlist = reinterpret_cast<uint16_t*>(nface + 4);
  uint16_t* ylist = xlist + (TX + 1) * TY;
  if (threadIdx.x == 0) nface[0] = nface[1] = 0;
  pointwise_tile<Tc, TX, TY>(u, g, x0, y0, Pw, ph);
  __syncthreads();
  for (int i = threadIdx.x; i < (TX + 1) * TY; i += nt) {
    const int f = i / TY, q = i - f * TY;
    const int x = x0 + f, y = y0 + q;
    const bool owned = (f < TX || x == g.nx) && x <= g.nx && y < g.ny;
    if (!owned) continue;
    if (!((x >= 1 && pred[(x - 1) * g.ny + y]) || (x < g.nx && pred[x * g.ny + y]))) continue;
    xlist[atomicAdd(&nface[0], 1)] = (uint16_t)i;
  }
  for (int i = threadIdx.x; i < TX * (TY + 1); i += nt) {
    const int r = i / (TY + 1), f = i - r * (TY + 1);
    const int x = x0 + r, y = y0 + f;
    const bool owned = (f < TY || y == g.ny) && y <= g.ny && x < g.nx;
    if (!owned) continue;
    if (!((y >= 1 && pred[x * g.ny + y - 1]) || (y < g.ny && pred[x * g.ny + y]))) continue;
    ylist[atomicAdd(&nface[1], 1)] = (uint16_t)i;
  }
  __syncthreads();
  const int nxf = nface[0], nyf = nface[1];
  if (fallback_count && threadIdx.x == 0) atomicAdd(fallback_count, (unsigned int)(nxf + nyf));
  for (int k = threadIdx.x; k < nxf; k += nt) {
    const int i = xlist[k];
    const int f = i / TY, q = i - f * TY;
    Tc flo[5];
    fallback_face_flux<Tc>(Pw + f * PWY + q + 2, PWX * PWY, PWY, muscl, limiter, ph, g.dx, flo);
    Tc* o = F.p + F.at(x0 + f, y0 + q);
#pragma unroll
    for (int v = 0; v < 5; ++v) o[v * F.vs] = (Tc(1) - Tc(1)) * FX[(v * (TX + 1) + f) * TY + q] + Tc(1) * flo[v];
  }
  for (int k = threadIdx.x; k < nyf; k += nt) {
    const int i = ylist[k];
    const int r = i / (TY + 1), f = i - r * (TY + 1);
    Tc flo[5];
    fallback_face_flux<Tc>(Pw + (r + 2) * PWY + f, PWX * PWY, 1, muscl, limiter, ph, g.dy, flo);
    Tc* o = G.p + G.at(x0 + r, y0 + f);
#pragma unroll
    for (int v = 0; v < 5; ++v) o[v * G.vs] = (Tc(1) - Tc(1)) * GY[(v * TX + r) * D::GYS + f] + Tc(1) * flo[v];
  }
}

// The stage's time step: dt = CFL h / max speed or the fixed dt
// (fvhoe/hydro.py:270-294); the first stage of a step also fixes the step's dt,
// clamped so that t + dt does not pass the target (fvhoe/ode.py:11-22).
struct DtSpec {
  double cfl_h, fixed_dt, t, target;
  int use_fixed, first_stage, has_target, pad_;
};

template <typename Tc, int P, int TX, int TY, int KC, int KF>
__global__ void __launch_bounds__(256, FluxDims<P, TX, TY>::template blocks<Tc>())
    k2_fluxes(V2<const Tc> W, const double* __restrict__ u, Geo g, V2<Tc> F, V2<Tc> G, Tc* __restrict__ ustar,
              Rule<Tc, KC> c, Rule<Tc, KC> t, Rule<Tc, KF> lrule, Rule<Tc, KF> rrule, Phys<Tc> ph, double cx,
              double cy, Scalars* __restrict__ sc, DtSpec dts, const uint8_t* __restrict__ pred, int muscl,
              int limiter, const __grid_constant__ CUtensorMap wmap) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bar;  // before the dynamic block: the tiles start at align128(smem_raw)
  // every block derives dt from the reduced CFL key; block (0, 0) publishes it
  const double dt = dts.use_fixed ? dts.fixed_dt : dts.cfl_h / key_value(sc->cfl_key);
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
    sc->dt_stage = dt;
    if (dts.first_stage) {
      double d = dt;
      if (dts.has_target && dts.target - dts.t < d) d = dts.target - dts.t;
      sc->dt_step = d;
    }
  }
  tile2_fluxes<Tc, P, TX, TY, KC, KF>(W, u, g, F, G, ustar, c, t, lrule, rrule, ph, cx, cy, dt, pred, muscl, limiter,
                                      blockIdx.x, blockIdx.y, tma::align128(smem_raw), &wmap, &bar, &sc->timeouts,
                                      &sc->flux_fallback_faces);
}

// ---------------------------------------------------------------------------
// Detection: detect_cells (shared), tile2_detect (W* computed on the tile and
// its 3-cell ring, for the ensemble's persistent phase) and the staged form
// (W* precomputed over the grid, for the one-problem launches).
// ---------------------------------------------------------------------------
// W on [x0-1, x0+TX+1) x [y0-1, y0+TY+1) into Wt ((TX+2) x (TY+2) per variable)
// by per-thread loads, clamped into W's ghost range (points past it feed only
// cells outside the grid), for the 3x3 box extrema of detect_cells.
template <typename Tc, int TX, int TY>
__device__ __forceinline__ void stage_w_ring(Tc* __restrict__ Wt, const Geo& g, const V2<const Tc>& W, int x0,
                                             int y0) {
  constexpr int WX = TX + 2, WY = TY + 2;
  for (int i = threadIdx.x; i < WX * WY; i += blockDim.x) {
    const int r = i / WY, q = i - r * WY;
    const int x = min(x0 - 1 + r, g.nx + W.g - 1), y = min(y0 - 1 + q, g.ny + W.g - 1);
    const Tc* p = W.p + W.at(x, y);
#pragma unroll
    for (int v = 0; v < 5; ++v) Wt[(v * WX + r) * WY + q] = p[v * W.vs];
  }
}

// Troubled-cell detection of the tile's cells (fvhoe/slope_limiting.py:87-244)
// from W* on [x0-3, x0+TX+3) x [y0-3, y0+TY+3) in A (row stride OYS) and W on
// [x0-1, x0+TX+1) x [y0-1, y0+TY+1) in Wt (row stride WYS, variable stride
// (TX+2) WYS), both staged by the caller; the first read follows a barrier.
template <typename Tc, int TX, int TY, int OYS, int WYS>
__device__ __forceinline__ void detect_cells(const Tc* __restrict__ A, const Tc* __restrict__ Wt, const Geo& g,
                                             const DetectSpec& ds, Scalars* __restrict__ sc,
                                             uint8_t* __restrict__ trouble, double* __restrict__ log_trouble,
                                             double* __restrict__ log_nad, double* __restrict__ log_pad, int x0,
                                             int y0) {
  constexpr int OX = TX + 6;
  constexpr int WX = TX + 2, WY = WYS;
  __syncthreads();
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
  for (int i = threadIdx.x; i < TX * TY; i += blockDim.x) {
    const int r = i / TY, q = i - r * TY;
    const int x = x0 + r, y = y0 + q;
    if (x >= g.nx || y >= g.ny) continue;
    bool nad_any = false;
    Tc ind_min = Tc(0), pad_ind = Tc(0);
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const Tc* pw = Wt + (v * WX + r + 1) * WY + q + 1;
      Tc big = pw[0], small = big;
#pragma unroll
      for (int a = -1; a <= 1; ++a)
#pragma unroll
        for (int b = -1; b <= 1; ++b) {
          const Tc xv = pw[a * WY + b];
          big = fmax(big, xv);
          small = fmin(small, xv);
        }
      const Tc* ps = A + (v * OX + r + 3) * OYS + q + 3;
      const Tc xs = ps[0];
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
        Tc line[7];
#pragma unroll
        for (int m = 0; m < 7; ++m) line[m] = ps[(m - 3) * OYS];
        bool below = sed_line_below_one(line, sed_eps);
        if (!below) {
#pragma unroll
          for (int m = 0; m < 7; ++m) line[m] = ps[m - 3];
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
    bool tr = pad_trouble || nad_any;
    if (ds.force_trouble) tr = true;
    const int o = x * g.ny + y;
    trouble[o] = tr ? 1 : 0;
    count += tr ? 1u : 0u;
    if (ds.log_mode) {
      const double lt = tr ? 1.0 : 0.0;
      const double ln = nad_any ? -(double)ind_min : 0.0;
      const double lp = pad_trouble ? -(double)pad_ind : 0.0;
      log_write(ds, o, lt, ln, lp, log_trouble, log_nad, log_pad);
    }
  }
  block_count_add(count, &sc->troubled);
}

template <typename Tc, int P, int TX, int TY, int KC>
__device__ __forceinline__ void tile2_detect(const Tc* __restrict__ ustar, Geo g, V2<const Tc> W, Rule<Tc, KC> c,
                                             Rule<Tc, KC> t, Phys<Tc> ph, DetectSpec ds, Scalars* __restrict__ sc,
                                             uint8_t* __restrict__ trouble, double* __restrict__ log_trouble,
                                             double* __restrict__ log_nad, double* __restrict__ log_pad, int bx,
                                             int by, unsigned char* smem_raw) {
  constexpr int OX = TX + 6, OY = TY + 6;
  using D = PrimsDims<Tc, P, OX, OY>;
  Tc* A = reinterpret_cast<Tc*>(smem_raw);
  Tc* B = A + D::A;
  const int x0 = by * TX, y0 = bx * TY;
  primitives_tile<Tc, P, OX, OY, KC>(ustar, g, x0 - 3, y0 - 3, A, B, c, t, ph);
  // A now holds W* on [x0-3, x0+TX+3) x [y0-3, y0+TY+3); B is free for the W tile
  static_assert((TX + 2) * (TY + 2) * 5 <= D::B, "W tile must fit in the second buffer");
  stage_w_ring<Tc, TX, TY>(B, g, W, x0, y0);
  detect_cells<Tc, TX, TY, D::OYS, TY + 2>(A, B, g, ds, sc, trouble, log_trouble, log_nad, log_pad, x0, y0);
}


// Detection from a precomputed W*: the primitive kernel run on the candidate
// over the 3-ghost box (Wst) replaces the W* tile that tile2_detect computes
// on each tile plus its 3-cell ring; the cells and results are the same.
// Both tiles arrive by TMA box copies whose first column is rounded down to a
// 16-byte boundary (AL elements): the W* box starts at column y0-4 (Wst.gy is
// 4, so at array column y0, a multiple of AL) and is read from its second
// column on; the W box starts at W's column y0-1+gy rounded down, and is read
// from offset WOFF = (gy(gW) - 1) mod AL, with gW the ghost width of W for
// degree P with limiting, max(R+1, 2R, 3).
template <typename Tc, int P, int TX, int TY>
struct DetectStagedDims {
  static constexpr int AL = 16 / (int)sizeof(Tc);
  static constexpr int R = (P + 1) / 2;
  static constexpr int GW = Max<Max<R + 1, 2 * R>::value, 3>::value;
  static constexpr int GWY = (GW + AL - 1) / AL * AL;  // gy of W
  static constexpr int WOFF = (GWY - 1) % AL;
  static constexpr int OX = TX + 6, OYS = (TY + 7 + AL - 1) / AL * AL;      // W* box: columns y0-4 ..
  static constexpr int WX = TX + 2, WYS = (TY + 2 + WOFF + AL - 1) / AL * AL;  // W box
  static constexpr int BOXA = OX * OYS * 5, BOXB = WX * WYS * 5;  // elements of the two box copies
  static constexpr int A = (BOXA + 31) / 32 * 32;  // W* tile, rounded so that the W tile starts 128-byte aligned
  static constexpr int B = BOXB;                   // W tile
  static constexpr int TOTAL = A + B;              // elements of the compute type
};

template <typename Tc, int P, int TX, int TY>
__device__ __forceinline__ void tile2_detect_staged(V2<const Tc> Wst, Geo g, V2<const Tc> W, DetectSpec ds,
                                                    Scalars* __restrict__ sc, uint8_t* __restrict__ trouble,
                                                    double* __restrict__ log_trouble, double* __restrict__ log_nad,
                                                    double* __restrict__ log_pad, int bx, int by,
                                                    unsigned char* smem_raw, const CUtensorMap* wsmap,
                                                    const CUtensorMap* wmap, uint64_t* bars) {
  using D = DetectStagedDims<Tc, P, TX, TY>;
  Tc* A = reinterpret_cast<Tc*>(smem_raw);
  Tc* B = A + D::A;
  const int x0 = by * TX, y0 = bx * TY;
  // W* rows x0-3.. (array row x0), columns y0-4.. (array column y0); W rows
  // x0-1.. (array row x0-1+gW), columns y0-1+gy rounded down to AL
  const uint32_t bytes_a = (uint32_t)(D::BOXA * sizeof(Tc)), bytes_b = (uint32_t)(D::BOXB * sizeof(Tc));
  const int wcol = y0 - 1 + D::GWY - D::WOFF;  // the host checks W.gy == GWY
  if (threadIdx.x == 0) {
    tma::mbar_init(&bars[0], 1);
    tma::mbar_init(&bars[1], 1);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  int refused = 0;
  if (threadIdx.x == 0) {
    const int acol = y0 - 4 + Wst.gy;
    if (tma::copy_aligned(A, acol, (int)sizeof(Tc)) && tma::copy_aligned(B, wcol, (int)sizeof(Tc))) {
      tma::arrive_expect_tx(&bars[0], bytes_a);
      tma::load_3d(A, wsmap, acol, x0 - 3 + Wst.g, 0, &bars[0]);
      tma::arrive_expect_tx(&bars[1], bytes_b);
      tma::load_3d(B, wmap, wcol, x0 - 1 + W.g, 0, &bars[1]);
    } else {
      refused = 1;
      atomicAdd(&sc->timeouts, 1u);
    }
  }
  if (__syncthreads_or(refused)) return;  // nothing was copied: the host reports the error
  const bool ok = tma::wait_bounded(&bars[0], 0, tma::kWaitPolls) && tma::wait_bounded(&bars[1], 0, tma::kWaitPolls);
  if (__syncthreads_or(ok ? 0 : 1)) {
    // drain both copies before the block reads or leaves its shared memory
    tma::wait_bounded(&bars[0], 0, tma::kDrainPolls);
    tma::wait_bounded(&bars[1], 0, tma::kDrainPolls);
    if (threadIdx.x == 0) atomicAdd(&sc->timeouts, 1u);
  }
  detect_cells<Tc, TX, TY, D::OYS, D::WYS>(A + 1, B + D::WOFF, g, ds, sc, trouble, log_trouble, log_nad, log_pad, x0,
                                           y0);
}

template <typename Tc, int P, int TX, int TY>
__global__ void __launch_bounds__(256, 6)
    k2_detect_staged(V2<const Tc> Wst, Geo g, V2<const Tc> W, DetectSpec ds, Scalars* __restrict__ sc,
                     uint8_t* __restrict__ trouble, double* __restrict__ log_trouble, double* __restrict__ log_nad,
                     double* __restrict__ log_pad, const __grid_constant__ CUtensorMap wsmap,
                     const __grid_constant__ CUtensorMap wmap) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bars[2];  // before the dynamic block: the tiles start at align128(smem_raw)
  tile2_detect_staged<Tc, P, TX, TY>(Wst, g, W, ds, sc, trouble, log_trouble, log_nad, log_pad, blockIdx.x, blockIdx.y,
                                     tma::align128(smem_raw), &wsmap, &wmap, bars);
}

// ---------------------------------------------------------------------------
// k2_final: fallback fluxes at troubled faces of the tile (from pointwise
// primitives of the stage input with 2 ghosts), the blend with the
// high-order fluxes, the divergence and the Runge-Kutta combination.
// ---------------------------------------------------------------------------
// The Runge-Kutta combination of one cell's five variables at o + v*plane
// (fvhoe/ode.py:245-298; the expressions of k_final, evaluated in the same
// order) for integrator INTEG at stage STAGE. Every array the stage reads is
// loaded for all five variables before the first store, so a cell's loads are
// in flight together. SO: SSP-RK3 in the Shu-Osher form instead of the
// reference's k-sum form (the FP32 form: the same scheme, FP64 rounding apart,
// reading the stage input in place of the k-sum and writing no k-sum).
// pa / pb (variable stride ps): the cell's a and b operands already staged in
// shared memory, read there instead of from the arrays.
// Returns how many results are not finite.
template <int INTEG, int STAGE, bool SO = false>
__device__ __forceinline__ unsigned int rk_combine(const StageSpec& st, int o, int plane, double dt,
                                                   const double* k, const double* pa = nullptr,
                                                   const double* pb = nullptr, int ps = 0) {
  double a[5], b[5], res[5];
  if constexpr (INTEG == INT_RHS) {
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      st.dudt_out[o + v * plane] = k[v];
      res[v] = k[v];
    }
  } else if constexpr (INTEG == INT_EULER) {
#pragma unroll
    for (int v = 0; v < 5; ++v) a[v] = pa ? pa[v * ps] : st.u[o + v * plane];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      res[v] = a[v] + dt * k[v];
      st.u[o + v * plane] = res[v];
    }
  } else if constexpr (INTEG == INT_SSPRK2) {
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      a[v] = pa ? pa[v * ps] : st.u[o + v * plane];
      if constexpr (STAGE != 0) b[v] = pb ? pb[v * ps] : st.stage_in[o + v * plane];
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      if constexpr (STAGE == 0) {
        res[v] = a[v] + dt * k[v];
        st.next[o + v * plane] = res[v];
      } else {
        res[v] = 0.5 * a[v] + 0.5 * (b[v] + dt * k[v]);
        st.u[o + v * plane] = res[v];
      }
    }
  } else if constexpr (INTEG == INT_SSPRK3 && SO) {
    // u1 = u + dt k1; u2 = 3/4 u + 1/4 (u1 + dt k2); u3 = 1/3 u + 2/3 (u2 + dt k3)
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      a[v] = pa ? pa[v * ps] : st.u[o + v * plane];
      if constexpr (STAGE != 0) b[v] = pb ? pb[v * ps] : st.stage_in[o + v * plane];
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const int ov = o + v * plane;
      if constexpr (STAGE == 0) {
        res[v] = a[v] + dt * k[v];
        st.next[ov] = res[v];
      } else if constexpr (STAGE == 1) {
        res[v] = 0.75 * a[v] + 0.25 * (b[v] + dt * k[v]);
        st.next[ov] = res[v];
      } else {
        res[v] = (1.0 / 3.0) * a[v] + (2.0 / 3.0) * (b[v] + dt * k[v]);
        st.u[ov] = res[v];
      }
    }
  } else if constexpr (INTEG == INT_SSPRK3) {
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      a[v] = pa ? pa[v * ps] : st.u[o + v * plane];
      if constexpr (STAGE != 0) b[v] = pb ? pb[v * ps] : st.acc[o + v * plane];
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const int ov = o + v * plane;
      if constexpr (STAGE == 0) {
        st.acc[ov] = k[v];
        res[v] = a[v] + dt * k[v];
        st.next[ov] = res[v];
      } else if constexpr (STAGE == 1) {
        const double qd = 0.25 * dt;
        res[v] = (a[v] + qd * b[v]) + qd * k[v];
        st.next[ov] = res[v];
        st.acc[ov] = b[v] + k[v];
      } else {
        res[v] = a[v] + ((1.0 / 6.0) * dt) * (b[v] + 4.0 * k[v]);
        st.u[ov] = res[v];
      }
    }
  } else {  // INT_RK4
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      a[v] = pa ? pa[v * ps] : st.u[o + v * plane];
      if constexpr (STAGE != 0) b[v] = pb ? pb[v * ps] : st.acc[o + v * plane];
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const int ov = o + v * plane;
      if constexpr (STAGE == 0) {
        st.acc[ov] = k[v];
        res[v] = a[v] + (0.5 * dt) * k[v];
        st.next[ov] = res[v];
      } else if constexpr (STAGE == 1 || STAGE == 2) {
        st.acc[ov] = b[v] + 2.0 * k[v];
        res[v] = a[v] + (STAGE == 1 ? 0.5 * dt : dt) * k[v];
        st.next[ov] = res[v];
      } else {
        res[v] = a[v] + ((1.0 / 6.0) * dt) * (b[v] + k[v]);
        st.u[ov] = res[v];
      }
    }
  }
  unsigned int bad = 0;
#pragma unroll
  for (int v = 0; v < 5; ++v) bad += isfinite(res[v]) ? 0u : 1u;
  return bad;
}

// rk_combine for the integrator and stage named at run time (the batched ensemble)
template <bool SO>
__device__ __forceinline__ unsigned int rk_combine_rt(const StageSpec& st, int o, int plane, double dt,
                                                      const double* k) {
  switch (st.integrator) {
    case INT_RHS: return rk_combine<INT_RHS, 0>(st, o, plane, dt, k);
    case INT_EULER: return rk_combine<INT_EULER, 0>(st, o, plane, dt, k);
    case INT_SSPRK2:
      return st.stage == 0 ? rk_combine<INT_SSPRK2, 0>(st, o, plane, dt, k)
                           : rk_combine<INT_SSPRK2, 1>(st, o, plane, dt, k);
    case INT_SSPRK3:
      if (st.stage == 0) return rk_combine<INT_SSPRK3, 0, SO>(st, o, plane, dt, k);
      if (st.stage == 1) return rk_combine<INT_SSPRK3, 1, SO>(st, o, plane, dt, k);
      return rk_combine<INT_SSPRK3, 2, SO>(st, o, plane, dt, k);
    default:
      if (st.stage == 0) return rk_combine<INT_RK4, 0>(st, o, plane, dt, k);
      if (st.stage == 1) return rk_combine<INT_RK4, 1>(st, o, plane, dt, k);
      if (st.stage == 2) return rk_combine<INT_RK4, 2>(st, o, plane, dt, k);
      return rk_combine<INT_RK4, 3>(st, o, plane, dt, k);
  }
}

template <int TX, int TY>
struct FinalDims {
  static constexpr int PX = TX + 4, PY = TY + 4;
  static constexpr int SP = PX * PY * 5;
  static constexpr int SF = (TX + 1) * TY * 5;
  static constexpr int SG = TX * (TY + 1) * 5;
  static constexpr int NXF = (TX + 1) * TY, NYF = TX * (TY + 1);  // faces of the tile
  // bytes after the three tiles: two counters and the compacted fallback face lists
  static constexpr int LIST = 16 + 2 * (NXF + NYF);
  static_assert(NXF < 65536 && NYF < 65536, "face indices are 16-bit");
  // FP64 launches of a fixed integrator also stage the Runge-Kutta operands
  // of the tile's cells (two FP64 arrays, 5 variables each), after the lists
  static constexpr int LIST16 = (LIST + 15) / 16 * 16;
  static constexpr int RKOP = 2 * 5 * TX * TY;
  // FB: the fallback runs in the same launch (pointwise tile and face lists
  // after the two flux tiles); without it the launch holds the flux tiles only
  template <typename Tc>
  static constexpr size_t rk_offset(bool fb) {
    return fb ? (size_t)(SP + SF + SG) * sizeof(Tc) + LIST16 : ((size_t)(SF + SG) * sizeof(Tc) + 15) / 16 * 16;
  }
  template <typename Tc>
  static constexpr size_t bytes(bool rk_operands, bool fb = true) {
    return rk_operands ? rk_offset<Tc>(fb) + RKOP * sizeof(double)
                       : (fb ? (size_t)(SP + SF + SG) * sizeof(Tc) + LIST : (size_t)(SF + SG) * sizeof(Tc));
  }
};

// The arrays the Runge-Kutta combination of INTEG / STAGE reads besides the
// divergence (a: the step's initial state; b: the stage input or the k-sum;
// nullptr where it reads none), as rk_combine reads them.
template <int INTEG, int STAGE, bool SO>
__device__ __forceinline__ void rk_sources(const StageSpec& st, const double*& a, const double*& b) {
  a = INTEG == INT_RHS ? nullptr : st.u;
  b = nullptr;
  if constexpr (STAGE != 0) {
    if constexpr (INTEG == INT_SSPRK2 || (INTEG == INT_SSPRK3 && SO)) {
      b = st.stage_in;
    } else if constexpr (INTEG == INT_SSPRK3 || INTEG == INT_RK4) {
      b = st.acc;
    }
  }
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// RKI < 0: the integrator and stage are read from st at run time. FB: the
// fallback fluxes of the tile's troubled faces are solved here (the batched
// ensemble's phase); without it k2_face_solve has already written them into F
// and G, and this is the divergence and the Runge-Kutta combination alone.
template <typename Tc, int TX, int TY, int RKI = -1, int RKS = 0, bool FB = true>
__device__ __forceinline__ void tile2_final(const double* __restrict__ stage_in, Geo g, V2<const Tc> F,
                                            V2<const Tc> G, const uint8_t* __restrict__ trouble,
                                            const uint8_t* __restrict__ pred, int apost, int muscl, int limiter,
                                            Phys<Tc> ph, double cx, double cy, StageSpec st, double dt_step,
                                            Scalars* __restrict__ sc, int bx, int by, unsigned char* smem_raw) {
  using D = FinalDims<TX, TY>;
  Tc* FX = reinterpret_cast<Tc*>(smem_raw);
  Tc* GY = FX + D::SF;
  Tc* Pw = GY + D::SG;
  const int nt = blockDim.x;
  const int x0 = by * TX, y0 = bx * TY;
  // high-order fluxes of the tile's faces, copied by asynchronous
  // global-to-shared copies (cp.async): every element of both tiles is in
  // flight at once, no register holds it, and each thread waits for its own
  // copies before the first barrier
  for (int i = threadIdx.x; i < (TX + 1) * TY; i += nt) {
    const int f = i / TY, q = i - f * TY;
    const int x = min(x0 + f, g.nx), y = min(y0 + q, g.ny - 1);
    const Tc* p = F.p + F.at(x, y);
#pragma unroll
    for (int v = 0; v < 5; ++v) cp_async_elem(&FX[(v * (TX + 1) + f) * TY + q], p + v * F.vs);
  }
  for (int i = threadIdx.x; i < TX * (TY + 1); i += nt) {
    const int r = i / (TY + 1), f = i - r * (TY + 1);
    const int x = min(x0 + r, g.nx - 1), y = min(y0 + f, g.ny);
    const Tc* p = G.p + G.at(x, y);
#pragma unroll
    for (int v = 0; v < 5; ++v) cp_async_elem(&GY[(v * TX + r) * (TY + 1) + f], p + v * G.vs);
  }
  // FP64 launches of a fixed integrator without the fallback: the
  // Runge-Kutta operands of the tile's cells travel in a second copy group,
  // beside the flux tiles; each thread later reads only the cells it copied
  constexpr bool PRE = sizeof(Tc) == 8 && !FB && RKI >= 0 && RKI != INT_RHS;
  double* const RA = reinterpret_cast<double*>(smem_raw + D::template rk_offset<Tc>(FB));
  double* const RB = RA + 5 * TX * TY;
  const int plane = g.nx * g.ny;
  if constexpr (PRE) {
    cp_async_commit();
    const double *A, *B;
    rk_sources<RKI, RKS, false>(st, A, B);
    for (int i = threadIdx.x; i < TX * TY; i += nt) {
      const int r = i / TY, q = i - r * TY;
      const int x = x0 + r, y = y0 + q;
      if (x >= g.nx || y >= g.ny) continue;
      const int o = x * g.ny + y;
#pragma unroll
      for (int v = 0; v < 5; ++v) cp_async_elem(&RA[v * TX * TY + i], A + o + v * plane);
      if (B) {
#pragma unroll
        for (int v = 0; v < 5; ++v) cp_async_elem(&RB[v * TX * TY + i], B + o + v * plane);
      }
    }
    cp_async_commit();
    cp_async_wait_group<1>();  // the flux tiles
  } else {
    cp_async_wait_all();
  }
  // fallback at the faces of troubled cells; with predicted flags, faces next
  // to a predicted cell already hold their fallback flux (k2_fluxes) and only
  // the faces of missed cells are revised here. Revising face by face from the
  // stage input instead of the pointwise tile measured slower: misses touch
  // about one face in seven on KH, too many for scattered loads.
  if (FB && apost && tile_any<TX, TY>(trouble, pred, g, x0, y0)) {
    // the faces that take the fallback flux, gathered into two lists so that
    // whole warps solve them: solved in place, a warp holding one such face
    // among 32 would run the whole MUSCL + Riemann solve for it
    int* nface = reinterpret_cast<int*>(Pw + D::SP);
    uint16_t* xlist = reinterpret_cast<uint16_t*>(nface + 4);
    uint16_t* ylist = xlist + D::NXF;
    if (threadIdx.x == 0) nface[0] = nface[1] = 0;
    pointwise_tile<Tc, TX, TY>(stage_in, g, x0, y0, Pw, ph);
    __syncthreads();
    for (int i = threadIdx.x; i < D::NXF; i += nt) {
      const int f = i / TY, q = i - f * TY;
      const int x = x0 + f, y = y0 + q;
      if (x > g.nx || y >= g.ny) continue;
      const int ol = (x - 1) * g.ny + y, orr = x * g.ny + y;
      const bool tl = x >= 1 && trouble[ol], trr = x < g.nx && trouble[orr];
      if (!(tl || trr)) continue;
      if (pred && ((x >= 1 && pred[ol]) || (x < g.nx && pred[orr]))) continue;
      xlist[atomicAdd(&nface[0], 1)] = (uint16_t)i;
    }
    for (int i = threadIdx.x; i < D::NYF; i += nt) {
      const int r = i / (TY + 1), f = i - r * (TY + 1);
      const int x = x0 + r, y = y0 + f;
      if (x >= g.nx || y > g.ny) continue;
      const int ol = x * g.ny + y - 1, orr = x * g.ny + y;
      const bool tl = y >= 1 && trouble[ol], trr = y < g.ny && trouble[orr];
      if (!(tl || trr)) continue;
      if (pred && ((y >= 1 && pred[ol]) || (y < g.ny && pred[orr]))) continue;
      ylist[atomicAdd(&nface[1], 1)] = (uint16_t)i;
    }
    __syncthreads();
    // X faces
    const int nx_faces = nface[0], ny_faces = nface[1];
    if (threadIdx.x == 0) atomicAdd(&sc->revised_faces, (unsigned int)(nx_faces + ny_faces));
    for (int k = threadIdx.x; k < nx_faces; k += nt) {
      const int i = xlist[k];
      const int f = i / TY, q = i - f * TY;
      Tc flo[5];
      fallback_face_flux<Tc>(Pw + f * D::PY + q + 2, D::PX * D::PY, D::PY, muscl, limiter, ph, g.dx, flo);
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        Tc& fh = FX[(v * (TX + 1) + f) * TY + q];
        fh = (Tc(1) - Tc(1)) * fh + Tc(1) * flo[v];
      }
    }
    // Y faces
    for (int k = threadIdx.x; k < ny_faces; k += nt) {
      const int i = ylist[k];
      const int r = i / (TY + 1), f = i - r * (TY + 1);
      Tc flo[5];
      fallback_face_flux<Tc>(Pw + (r + 2) * D::PY + f, D::PX * D::PY, 1, muscl, limiter, ph, g.dy, flo);
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        Tc& fh = GY[(v * TX + r) * (TY + 1) + f];
        fh = (Tc(1) - Tc(1)) * fh + Tc(1) * flo[v];
      }
    }
  }
  if constexpr (PRE) cp_async_wait_all();
  __syncthreads();
  // divergence and the Runge-Kutta combination
  const double dt = (RKI >= 0 ? RKI : st.integrator) == INT_RHS ? 0.0 : dt_step;
  unsigned int bad = 0;
  for (int i = threadIdx.x; i < TX * TY; i += nt) {
    const int r = i / TY, q = i - r * TY;
    const int x = x0 + r, y = y0 + q;
    if (x >= g.nx || y >= g.ny) continue;
    double k[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      Tc dc = Tc(0);
      dc = dc + (Tc)cx * (FX[(v * (TX + 1) + r + 1) * TY + q] - FX[(v * (TX + 1) + r) * TY + q]);
      dc = dc + (Tc)cy * (GY[(v * TX + r) * (TY + 1) + q + 1] - GY[(v * TX + r) * (TY + 1) + q]);
      k[v] = (double)dc;
    }
    if constexpr (PRE) {
      bad += rk_combine<RKI, RKS, false>(st, x * g.ny + y, plane, dt, k, RA + i, RB + i, TX * TY);
    } else if constexpr (RKI >= 0) {
      bad += rk_combine<RKI, RKS, sizeof(Tc) == 4>(st, x * g.ny + y, plane, dt, k);
    } else {
      bad += rk_combine_rt<sizeof(Tc) == 4>(st, x * g.ny + y, plane, dt, k);
    }
  }
  block_count_add(bad, &sc->nonfinite);
}

// Fallback faces of a stage, as one list over the grid: every face with a
// troubled cell on either side (with predicted flags, only faces with no
// predicted neighbour: those already hold their fallback flux), as face ids
// (X faces x*ny + y, then Y faces (nx+1)*ny + x*(ny+1) + y). A block takes a
// 32 x 32 tile of each face grid, the X faces of rows x0 .. x0+31 (of nx+1)
// and the Y faces of columns y0 .. y0+31 (of ny+1), in FACE_ROUNDS rounds of
// 8 rows, counts them per warp and round, reserves its whole segment with one
// atomic and writes it in that order: neighbouring list entries are faces of
// one region, so the solves that read them share their cells in cache.
// Segments land in any order; the revised fluxes do not depend on it (every
// face is solved on its own). The count is fb_faces (zeroed by
// k_reset_scalars). One instantiation per compute type (the units of the two
// precisions each hold one).
constexpr int FACE_ROUNDS = 8;

__device__ __forceinline__ bool fallback_xface(const Geo& g, const uint8_t* __restrict__ trouble,
                                               const uint8_t* __restrict__ pred, int x, int y) {
  if (x > g.nx || y >= g.ny) return false;
  const int ol = (x - 1) * g.ny + y, orr = x * g.ny + y;
  const bool need = (x >= 1 && trouble[ol]) || (x < g.nx && trouble[orr]);
  return need && !(pred && ((x >= 1 && pred[ol]) || (x < g.nx && pred[orr])));
}

__device__ __forceinline__ bool fallback_yface(const Geo& g, const uint8_t* __restrict__ trouble,
                                               const uint8_t* __restrict__ pred, int x, int y) {
  if (x >= g.nx || y > g.ny) return false;
  const int ol = x * g.ny + y - 1, orr = x * g.ny + y;
  const bool need = (y >= 1 && trouble[ol]) || (y < g.ny && trouble[orr]);
  return need && !(pred && ((y >= 1 && pred[ol]) || (y < g.ny && pred[orr])));
}

template <typename Tc>
__global__ void __launch_bounds__(256) k2_face_list(Geo g, const uint8_t* __restrict__ trouble,
                                                    const uint8_t* __restrict__ pred, int* __restrict__ list,
                                                    Scalars* __restrict__ sc) {
  static_assert(FACE_ROUNDS == 8, "4 rounds of 8 rows of X faces, then 4 of Y faces");
  __shared__ int start[FACE_ROUNDS][8];  // per round and warp: its first list slot (then the block's base)
  __shared__ int block_base;
  const int nxf = (g.nx + 1) * g.ny;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int x0 = blockIdx.y * 32, y = blockIdx.x * 32 + lane;
  unsigned ballot[FACE_ROUNDS];
  int id[FACE_ROUNDS];
#pragma unroll
  for (int j = 0; j < FACE_ROUNDS; ++j) {
    const int x = x0 + (j & 3) * 8 + warp;
    const bool xf = j < 4;
    const bool need = xf ? fallback_xface(g, trouble, pred, x, y) : fallback_yface(g, trouble, pred, x, y);
    id[j] = xf ? x * g.ny + y : nxf + x * (g.ny + 1) + y;
    ballot[j] = __ballot_sync(0xffffffffu, need);
    if (lane == 0) start[j][warp] = __popc(ballot[j]);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int j = 0; j < FACE_ROUNDS; ++j)
      for (int w = 0; w < 8; ++w) {
        const int c = start[j][w];
        start[j][w] = run;
        run += c;
      }
    block_base = run ? (int)atomicAdd(&sc->fb_faces, (unsigned int)run) : 0;
  }
  __syncthreads();
  const unsigned below = (1u << lane) - 1u;
#pragma unroll
  for (int j = 0; j < FACE_ROUNDS; ++j)
    if ((ballot[j] >> lane) & 1u) list[block_base + start[j][warp] + __popc(ballot[j] & below)] = id[j];
}

// Fallback fluxes of the listed faces (fvhoe/solver.py:710-732), written over
// the high-order fluxes in F and G as (1-1)F + 1*F_low: per face, the
// pointwise primitives of the four cells i-2 .. i+1 along its axis (p = 1
// reconstruction is the identity), read from the stage input through the
// ghost maps, then MUSCL and the Riemann solve. Every thread holds a face, so
// the solves run at the occupancy of the launch instead of waiting on
// per-tile lists; each face appears once in the list, so no two threads write
// the same element. Four blocks per SM (64 registers in FP64, 92 bytes of
// spills) measured 4 % faster on the FP64 step than the unbounded 80 registers
// at 3 blocks.
template <typename Tc>
__global__ void __launch_bounds__(256, 4) k2_face_solve(const double* __restrict__ stage_in, Geo g, V2<Tc> F, V2<Tc> G,
                                                     const int* __restrict__ list, int muscl, int limiter,
                                                     Phys<Tc> ph, Scalars* __restrict__ sc) {
  const int n = (int)sc->fb_faces;
  const int nxf = (g.nx + 1) * g.ny;
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&sc->revised_faces, (unsigned int)n);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int id = list[k];
    const bool xface = id < nxf;
    int x, y;
    if (xface) {
      x = id / g.ny;
      y = id - x * g.ny;
    } else {
      const int j = id - nxf;
      x = j / (g.ny + 1);
      y = j - x * (g.ny + 1);
    }
    Tc cw[5][4];  // variable v of cell i-2+e at cw[v][e]
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      Tc uc[5], w[5];
      load_state2<Tc>(stage_in, g, xface ? x - 2 + e : x, xface ? y : y - 2 + e, uc);
      to_primitives(ph, 5, uc, w);
#pragma unroll
      for (int v = 0; v < 5; ++v) cw[v][e] = w[v];
    }
    Tc flo[5];
    fallback_face_flux<Tc>(&cw[0][0], 4, 1, muscl, limiter, ph, xface ? g.dx : g.dy, flo);
    Tc* o = xface ? F.p + F.at(x, y) : G.p + G.at(x, y);
    const int vs = xface ? F.vs : G.vs;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      Tc& fh = o[v * vs];
      fh = (Tc(1) - Tc(1)) * fh + Tc(1) * flo[v];
    }
  }
}

// RKI / RKS: the integrator and stage of the launch (one instantiation each).
// FB: the fallback fluxes are solved in this launch; without it they are
// already in F and G (k2_face_list + k2_face_solve).
template <typename Tc, int TX, int TY, int RKI, int RKS, bool FB>
__global__ void __launch_bounds__(256, sizeof(Tc) == 4 ? 5 : (FB ? 3 : 4))
    k2_final(const double* __restrict__ stage_in, Geo g, V2<const Tc> F, V2<const Tc> G,
             const uint8_t* __restrict__ trouble, const uint8_t* __restrict__ pred, int apost, int muscl, int limiter,
             Phys<Tc> ph, double cx, double cy, StageSpec st, Scalars* __restrict__ sc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  tile2_final<Tc, TX, TY, RKI, RKS, FB>(stage_in, g, F, G, trouble, pred, apost, muscl, limiter, ph, cx, cy, st,
                                        RKI == INT_RHS ? 0.0 : sc->dt_step, sc, blockIdx.x, blockIdx.y, smem_raw);
}

template <typename Tc, int TX, int TY>
using FinalKernel = void (*)(const double*, Geo, V2<const Tc>, V2<const Tc>, const uint8_t*, const uint8_t*, int,
                             int, int, Phys<Tc>, double, double, StageSpec, Scalars*);

// The k2_final instantiation of an integrator and stage.
template <typename Tc, int TX, int TY, bool FB>
FinalKernel<Tc, TX, TY> final_kernel(int integrator, int stage) {
  switch (integrator) {
    case INT_EULER: return k2_final<Tc, TX, TY, INT_EULER, 0, FB>;
    case INT_SSPRK2:
      return stage == 0 ? k2_final<Tc, TX, TY, INT_SSPRK2, 0, FB> : k2_final<Tc, TX, TY, INT_SSPRK2, 1, FB>;
    case INT_SSPRK3:
      if (stage == 0) return k2_final<Tc, TX, TY, INT_SSPRK3, 0, FB>;
      if (stage == 1) return k2_final<Tc, TX, TY, INT_SSPRK3, 1, FB>;
      return k2_final<Tc, TX, TY, INT_SSPRK3, 2, FB>;
    case INT_RK4:
      if (stage == 0) return k2_final<Tc, TX, TY, INT_RK4, 0, FB>;
      if (stage == 1) return k2_final<Tc, TX, TY, INT_RK4, 1, FB>;
      if (stage == 2) return k2_final<Tc, TX, TY, INT_RK4, 2, FB>;
      return k2_final<Tc, TX, TY, INT_RK4, 3, FB>;
    default: return k2_final<Tc, TX, TY, INT_RHS, 0, FB>;
  }
}

}  // namespace f2
}  // namespace fvh
