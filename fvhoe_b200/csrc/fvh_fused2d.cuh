// Fused 2D stage: four shared-memory-tiled kernels per stage instead of the
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
//   k2_detect      W* of u* on the tile plus 3 ghosts, then troubled-cell
//                  detection (fvhoe/slope_limiting.py:87-244)
//   k2_final       MUSCL fallback fluxes at troubled faces, the blend, the flux
//                  divergence and the Runge-Kutta combination
//                  (fvhoe/solver.py:710-751, fvhoe/ode.py:245-298)
// Shared-memory arrays are variable-major: element (v, r, c) of an R x C tile
// sits at (v*R + r)*C + c.
#pragma once

#include "fvh_kernels.cuh"

namespace fvh {
namespace f2 {

struct Geo {
  int nx, ny;          // interior cells along X and Y
  int bcx[2], bcy[2];  // Bc kinds at the low/high ends of X and Y
  int dx, dy;          // physical axis ids of X and Y
  int gmax;            // deepest ghost index any state load may reach
  const Slabs* slabs;  // Dirichlet ghost values (physical axes), or nullptr
};

// 2D view of a variable-major array over [-g, nx+g) x [-g, ny'+g).
template <typename T>
struct V2 {
  T* p;
  int g;   // ghost cells on each side
  int sx;  // row stride (the padded Y extent)
  int vs;  // variable stride
  __device__ __forceinline__ int at(int x, int y) const { return (x + g) * sx + (y + g); }
};

template <typename T>
__host__ __device__ inline V2<T> make_v2(T* p, int nx, int ny, int g) {
  V2<T> v;
  v.p = p;
  v.g = g;
  v.sx = ny + 2 * g;
  v.vs = (nx + 2 * g) * (ny + 2 * g);
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
  for (int i = threadIdx.x; i < PX * PY; i += blockDim.x) {
    const int r = i / PY, q = i - r * PY;
    Tc uc[5], w[5];
    load_state2<Tc>(u, g, x0 - 2 + r, y0 - 2 + q, uc);
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

// Tile dimensions of the primitive computation producing OX x OY outputs
// with degree P (centre / transverse rules of radius RC = P / 2).
template <int P, int OX, int OY>
struct PrimsDims {
  static constexpr int RC = P / 2;
  static constexpr int LX = OX + 4 * RC, LY = OY + 4 * RC;  // loaded state
  static constexpr int CX = OX + 2 * RC;                    // after the X centre sweep: CX x LY
  static constexpr int PY = OY + 2 * RC;                    // after the Y centre sweep: CX x PY
  // after the X transverse sweep: OX x PY; after the Y transverse sweep: OX x OY (in A)
  static constexpr int A = Max<Max<LX * LY, CX * PY>::value, OX * OY>::value * 5;
  static constexpr int B = Max<CX * LY, OX * PY>::value * 5;
};

// W on [x0, x0+OX) x [y0, y0+OY), computed in two shared buffers; the result
// is left in A as an OX x OY tile. Rules: centre c and transverse t (KC taps).
template <typename Tc, int P, int OX, int OY, int KC, typename Tin>
__device__ __forceinline__ void primitives_tile(const Tin* __restrict__ u, const Geo& g, int x0, int y0, Tc* A,
                                                Tc* B, const Rule<Tc, KC>& c, const Rule<Tc, KC>& t,
                                                const Phys<Tc>& ph) {
  using D = PrimsDims<P, OX, OY>;
  constexpr int RC = D::RC;
  const int nt = blockDim.x;
  // 1. state with 2*RC ghosts around the tile
  for (int i = threadIdx.x; i < D::LX * D::LY; i += nt) {
    const int r = i / D::LY, q = i - r * D::LY;
    Tc s[5];
    load_state2<Tc>(u, g, x0 - 2 * RC + r, y0 - 2 * RC + q, s);
#pragma unroll
    for (int v = 0; v < 5; ++v) A[(v * D::LX + r) * D::LY + q] = s[v];
  }
  __syncthreads();
  // 2. centre sweep along X
  for (int i = threadIdx.x; i < D::CX * D::LY; i += nt) {
    const int r = i / D::LY, q = i - r * D::LY;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      Tc acc = Tc(0);
#pragma unroll
      for (int k = 0; k < KC; ++k) acc = acc + c.w[k] * A[(v * D::LX + r + k) * D::LY + q];
      B[(v * D::CX + r) * D::LY + q] = acc;
    }
  }
  __syncthreads();
  // 3. centre sweep along Y, then primitives
  for (int i = threadIdx.x; i < D::CX * D::PY; i += nt) {
    const int r = i / D::PY, q = i - r * D::PY;
    Tc acc[5], w[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      acc[v] = Tc(0);
#pragma unroll
      for (int k = 0; k < KC; ++k) acc[v] = acc[v] + c.w[k] * B[(v * D::CX + r) * D::LY + q + k];
    }
    to_primitives(ph, 5, acc, w);
#pragma unroll
    for (int v = 0; v < 5; ++v) A[(v * D::CX + r) * D::PY + q] = w[v];
  }
  __syncthreads();
  // 4. transverse sweep along X
  for (int i = threadIdx.x; i < OX * D::PY; i += nt) {
    const int r = i / D::PY, q = i - r * D::PY;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      Tc acc = Tc(0);
#pragma unroll
      for (int k = 0; k < KC; ++k) acc = acc + t.w[k] * A[(v * D::CX + r + k) * D::PY + q];
      B[(v * OX + r) * D::PY + q] = acc;
    }
  }
  __syncthreads();
  // 5. transverse sweep along Y, into A as an OX x OY tile
  for (int i = threadIdx.x; i < OX * OY; i += nt) {
    const int r = i / OY, q = i - r * OY;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      Tc acc = Tc(0);
#pragma unroll
      for (int k = 0; k < KC; ++k) acc = acc + t.w[k] * B[(v * OX + r) * D::PY + q + k];
      A[(v * OX + r) * OY + q] = acc;
    }
  }
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
template <typename Tc, int P, int TX, int TY, int KC, bool REDUCE>
__device__ __forceinline__ void tile2_primitives(const double* __restrict__ u, Geo g, V2<Tc> W, int gw_out,
                                                 Rule<Tc, KC> c, Rule<Tc, KC> t, Phys<Tc> ph, ReduceSpec rs,
                                                 Scalars* __restrict__ sc, int bx, int by, unsigned char* smem_raw) {
  using D = PrimsDims<P, TX, TY>;
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
    for (int v = 0; v < 5; ++v) w[v] = A[(v * TX + r) * TY + q];
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

template <typename Tc, int P, int TX, int TY, int KC, bool REDUCE>
__global__ void __launch_bounds__(256)
    k2_primitives(const double* __restrict__ u, Geo g, V2<Tc> W, int gw_out, Rule<Tc, KC> c, Rule<Tc, KC> t,
                  Phys<Tc> ph, ReduceSpec rs, Scalars* __restrict__ sc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  tile2_primitives<Tc, P, TX, TY, KC, REDUCE>(u, g, W, gw_out, c, t, ph, rs, sc, blockIdx.x, blockIdx.y, smem_raw);
}

// ---------------------------------------------------------------------------
// k2_fluxes: high-order X- and Y-face fluxes of a TX x TY cell tile, and the
// candidate u* = u + dt L(F) of its cells.
// ---------------------------------------------------------------------------
template <int P, int TX, int TY>
struct FluxDims {
  static constexpr int R = (P + 1) / 2;  // face-rule radius
  static constexpr int RC = P / 2;       // centre / transverse radius
  static constexpr int KF = 2 * R + 1;
  static constexpr int H = Max<R + 1, 2 * RC>::value;  // W halo
  static constexpr int WX = TX + 2 * H, WY = TY + 2 * H;
  // X faces: centre sweep along Y on rows [x0-1-R, x0+TX+R], cols [y0-RC, y0+TY+RC)
  static constexpr int AXR = TX + 2 * R + 2, AXC = TY + 2 * RC;
  // Riemann fluxes at faces x0..x0+TX on those cols
  static constexpr int BXR = TX + 1, BXC = TY + 2 * RC;
  // Y faces: centre sweep along X on rows [x0-RC, x0+TX+RC), cols [y0-1-R, y0+TY+R]
  static constexpr int AYR = TX + 2 * RC, AYC = TY + 2 * R + 2;
  static constexpr int BYR = TX + 2 * RC, BYC = TY + 1;
  static constexpr int SW = WX * WY * 5;
  static constexpr int SA = Max<AXR * AXC, AYR * AYC>::value * 5;
  static constexpr int SB = Max<BXR * BXC, BYR * BYC>::value * 5;
  static constexpr int SF = (TX + 1) * TY * 5;
  static constexpr int SG = TX * (TY + 1) * 5;
};

template <typename Tc, int P, int TX, int TY, int KC, int KF>
__device__ __forceinline__ void tile2_fluxes(V2<const Tc> W, const double* __restrict__ u, Geo g, V2<Tc> F, V2<Tc> G,
                                             Tc* __restrict__ ustar, Rule<Tc, KC> c, Rule<Tc, KC> t,
                                             Rule<Tc, KF> lrule, Rule<Tc, KF> rrule, Phys<Tc> ph, double cx,
                                             double cy, double dt, const uint8_t* __restrict__ pred, int muscl,
                                             int limiter, int bx, int by, unsigned char* smem_raw) {
  using D = FluxDims<P, TX, TY>;
  constexpr int R = D::R, RC = D::RC, H = D::H;
  Tc* Ws = reinterpret_cast<Tc*>(smem_raw);
  Tc* A = Ws + D::SW;
  Tc* B = A + D::SA;
  Tc* FX = B + D::SB;
  Tc* GY = FX + D::SF;
  const int nt = blockDim.x;
  const int x0 = by * TX, y0 = bx * TY;
  // W tile with H ghosts (W holds gW >= H ghosts)
  for (int i = threadIdx.x; i < D::WX * D::WY; i += nt) {
    const int r = i / D::WY, q = i - r * D::WY;
    const int x = min(x0 - H + r, g.nx + W.g - 1), y = min(y0 - H + q, g.ny + W.g - 1);
    const Tc* p = W.p + W.at(x, y);
#pragma unroll
    for (int v = 0; v < 5; ++v) Ws[(v * D::WX + r) * D::WY + q] = p[v * W.vs];
  }
  __syncthreads();
  // ---- X faces
  // centre sweep along Y: A(r, q) at (x0-1-R+r, y0-RC+q)
  for (int i = threadIdx.x; i < D::AXR * D::AXC; i += nt) {
    const int r = i / D::AXC, q = i - r * D::AXC;
    const int wr = r + (H - 1 - R), wq = q + (H - RC) - RC;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      Tc acc = Tc(0);
#pragma unroll
      for (int k = 0; k < KC; ++k) acc = acc + c.w[k] * Ws[(v * D::WX + wr) * D::WY + wq + k];
      A[(v * D::AXR + r) * D::AXC + q] = acc;
    }
  }
  __syncthreads();
  // face f (x = x0+f) between cells x0+f-1 and x0+f; A row of cell x is x - (x0-1-R)
  for (int i = threadIdx.x; i < D::BXR * D::BXC; i += nt) {
    const int f = i / D::BXC, q = i - f * D::BXC;
    Tc wl[5], wr[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      wl[v] = Tc(0);
      wr[v] = Tc(0);
    }
#pragma unroll
    for (int k = 0; k < KF; ++k) {
      const int ra = f + k;      // cell x0+f-1, taps -R..R -> rows f .. f+2R
      const int rb = f + 1 + k;  // cell x0+f
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        wl[v] = wl[v] + rrule.w[k] * A[(v * D::AXR + ra) * D::AXC + q];
        wr[v] = wr[v] + lrule.w[k] * A[(v * D::AXR + rb) * D::AXC + q];
      }
    }
    Tc fl[5];
    riemann_flux<5>(ph, 5, wl, wr, g.dx, fl);
#pragma unroll
    for (int v = 0; v < 5; ++v) B[(v * D::BXR + f) * D::BXC + q] = fl[v];
  }
  __syncthreads();
  // transverse sweep along Y -> FX (TX+1) x TY
  for (int i = threadIdx.x; i < (TX + 1) * TY; i += nt) {
    const int f = i / TY, q = i - f * TY;
    const int x = x0 + f, y = y0 + q;
    Tc val[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      Tc acc = Tc(0);
#pragma unroll
      for (int k = 0; k < KC; ++k) acc = acc + t.w[k] * B[(v * D::BXR + f) * D::BXC + q + k];
      val[v] = acc;
      FX[(v * (TX + 1) + f) * TY + q] = acc;
    }
    const bool owned = (f < TX || x == g.nx) && x <= g.nx && y < g.ny;
    if (owned) {
      Tc* o = F.p + F.at(x, y);
#pragma unroll
      for (int v = 0; v < 5; ++v) o[v * F.vs] = val[v];
    }
  }
  __syncthreads();
  // ---- Y faces
  // centre sweep along X: A(r, q) at (x0-RC+r, y0-1-R+q)
  for (int i = threadIdx.x; i < D::AYR * D::AYC; i += nt) {
    const int r = i / D::AYC, q = i - r * D::AYC;
    const int wr = r + (H - RC) - RC, wq = q + (H - 1 - R);
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      Tc acc = Tc(0);
#pragma unroll
      for (int k = 0; k < KC; ++k) acc = acc + c.w[k] * Ws[(v * D::WX + wr + k) * D::WY + wq];
      A[(v * D::AYR + r) * D::AYC + q] = acc;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < D::BYR * D::BYC; i += nt) {
    const int r = i / D::BYC, f = i - r * D::BYC;
    Tc wl[5], wr[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      wl[v] = Tc(0);
      wr[v] = Tc(0);
    }
#pragma unroll
    for (int k = 0; k < KF; ++k) {
      const int qa = f + k, qb = f + 1 + k;
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        wl[v] = wl[v] + rrule.w[k] * A[(v * D::AYR + r) * D::AYC + qa];
        wr[v] = wr[v] + lrule.w[k] * A[(v * D::AYR + r) * D::AYC + qb];
      }
    }
    Tc fl[5];
    riemann_flux<5>(ph, 5, wl, wr, g.dy, fl);
#pragma unroll
    for (int v = 0; v < 5; ++v) B[(v * D::BYR + r) * D::BYC + f] = fl[v];
  }
  __syncthreads();
  // transverse sweep along X -> GY TX x (TY+1)
  for (int i = threadIdx.x; i < TX * (TY + 1); i += nt) {
    const int r = i / (TY + 1), f = i - r * (TY + 1);
    const int x = x0 + r, y = y0 + f;
    Tc val[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      Tc acc = Tc(0);
#pragma unroll
      for (int k = 0; k < KC; ++k) acc = acc + t.w[k] * B[(v * D::BYR + r + k) * D::BYC + f];
      val[v] = acc;
      GY[(v * TX + r) * (TY + 1) + f] = acc;
    }
    const bool owned = (f < TY || y == g.ny) && y <= g.ny && x < g.nx;
    if (owned) {
      Tc* o = G.p + G.at(x, y);
#pragma unroll
      for (int v = 0; v < 5; ++v) o[v * G.vs] = val[v];
    }
  }
  if (!ustar) return;
  __syncthreads();
  // candidate u* = u + dt (0 + cx (F[i+1]-F[i]) + cy (G[j+1]-G[j]))
  const int plane = g.nx * g.ny;
  for (int i = threadIdx.x; i < TX * TY; i += nt) {
    const int r = i / TY, q = i - r * TY;
    const int x = x0 + r, y = y0 + q;
    if (x >= g.nx || y >= g.ny) continue;
    const int o = x * g.ny + y;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      Tc d = Tc(0);
      d = d + (Tc)cx * (FX[(v * (TX + 1) + r + 1) * TY + q] - FX[(v * (TX + 1) + r) * TY + q]);
      d = d + (Tc)cy * (GY[(v * TX + r) * (TY + 1) + q + 1] - GY[(v * TX + r) * (TY + 1) + q]);
      ustar[v * plane + o] = (Tc)(u[v * plane + o] + dt * (double)d);
    }
  }
  // predicted cells: their faces take the fallback flux now, blended as the
  // final pass would (the candidate above keeps the high-order fluxes)
  if (!pred || !tile_any<TX, TY>(pred, nullptr, g, x0, y0)) return;
  constexpr int PWX = TX + 4, PWY = TY + 4;
  static_assert(PWX * PWY * 5 <= D::SW, "pointwise tile must fit in the W tile");
  Tc* Pw = Ws;
  pointwise_tile<Tc, TX, TY>(u, g, x0, y0, Pw, ph);
  __syncthreads();
  for (int i = threadIdx.x; i < (TX + 1) * TY; i += nt) {
    const int f = i / TY, q = i - f * TY;
    const int x = x0 + f, y = y0 + q;
    const bool owned = (f < TX || x == g.nx) && x <= g.nx && y < g.ny;
    if (!owned) continue;
    if (!((x >= 1 && pred[(x - 1) * g.ny + y]) || (x < g.nx && pred[x * g.ny + y]))) continue;
    Tc flo[5];
    fallback_face_flux<Tc>(Pw + f * PWY + q + 2, PWX * PWY, PWY, muscl, limiter, ph, g.dx, flo);
    Tc* o = F.p + F.at(x, y);
#pragma unroll
    for (int v = 0; v < 5; ++v) o[v * F.vs] = (Tc(1) - Tc(1)) * FX[(v * (TX + 1) + f) * TY + q] + Tc(1) * flo[v];
  }
  for (int i = threadIdx.x; i < TX * (TY + 1); i += nt) {
    const int r = i / (TY + 1), f = i - r * (TY + 1);
    const int x = x0 + r, y = y0 + f;
    const bool owned = (f < TY || y == g.ny) && y <= g.ny && x < g.nx;
    if (!owned) continue;
    if (!((y >= 1 && pred[x * g.ny + y - 1]) || (y < g.ny && pred[x * g.ny + y]))) continue;
    Tc flo[5];
    fallback_face_flux<Tc>(Pw + (r + 2) * PWY + f, PWX * PWY, 1, muscl, limiter, ph, g.dy, flo);
    Tc* o = G.p + G.at(x, y);
#pragma unroll
    for (int v = 0; v < 5; ++v) o[v * G.vs] = (Tc(1) - Tc(1)) * GY[(v * TX + r) * (TY + 1) + f] + Tc(1) * flo[v];
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
__global__ void __launch_bounds__(256)
    k2_fluxes(V2<const Tc> W, const double* __restrict__ u, Geo g, V2<Tc> F, V2<Tc> G, Tc* __restrict__ ustar,
              Rule<Tc, KC> c, Rule<Tc, KC> t, Rule<Tc, KF> lrule, Rule<Tc, KF> rrule, Phys<Tc> ph, double cx,
              double cy, Scalars* __restrict__ sc, DtSpec dts, const uint8_t* __restrict__ pred, int muscl,
              int limiter) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
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
                                      blockIdx.x, blockIdx.y, smem_raw);
}

// ---------------------------------------------------------------------------
// k2_detect: W* of u* on the tile and 3 ghosts, then the detection of the
// tile's cells against W (global, >= 3 ghosts).
// ---------------------------------------------------------------------------
template <typename Tc, int P, int TX, int TY, int KC>
__device__ __forceinline__ void tile2_detect(const Tc* __restrict__ ustar, Geo g, V2<const Tc> W, Rule<Tc, KC> c,
                                             Rule<Tc, KC> t, Phys<Tc> ph, DetectSpec ds, Scalars* __restrict__ sc,
                                             uint8_t* __restrict__ trouble, double* __restrict__ log_trouble,
                                             double* __restrict__ log_nad, double* __restrict__ log_pad, int bx,
                                             int by, unsigned char* smem_raw) {
  constexpr int OX = TX + 6, OY = TY + 6;
  using D = PrimsDims<P, OX, OY>;
  Tc* A = reinterpret_cast<Tc*>(smem_raw);
  Tc* B = A + D::A;
  const int x0 = by * TX, y0 = bx * TY;
  primitives_tile<Tc, P, OX, OY, KC>(ustar, g, x0 - 3, y0 - 3, A, B, c, t, ph);
  // A now holds W* on [x0-3, x0+TX+3) x [y0-3, y0+TY+3); B is free: stage W on
  // [x0-1, x0+TX+1) x [y0-1, y0+TY+1) there for the 3x3 box extrema
  constexpr int WX = TX + 2, WY = TY + 2;
  static_assert(WX * WY * 5 <= D::B, "W tile must fit in the second buffer");
  Tc* Wt = B;
  for (int i = threadIdx.x; i < WX * WY; i += blockDim.x) {
    const int r = i / WY, q = i - r * WY;
    const int x = min(x0 - 1 + r, g.nx + W.g - 1), y = min(y0 - 1 + q, g.ny + W.g - 1);
    const Tc* p = W.p + W.at(x, y);
#pragma unroll
    for (int v = 0; v < 5; ++v) Wt[(v * WX + r) * WY + q] = p[v * W.vs];
  }
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
      const Tc* ps = A + (v * OX + r + 3) * OY + q + 3;
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
        for (int m = 0; m < 7; ++m) line[m] = ps[(m - 3) * OY];
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
__global__ void __launch_bounds__(256)
    k2_detect(const Tc* __restrict__ ustar, Geo g, V2<const Tc> W, Rule<Tc, KC> c, Rule<Tc, KC> t, Phys<Tc> ph,
              DetectSpec ds, Scalars* __restrict__ sc, uint8_t* __restrict__ trouble, double* __restrict__ log_trouble,
              double* __restrict__ log_nad, double* __restrict__ log_pad) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  tile2_detect<Tc, P, TX, TY, KC>(ustar, g, W, c, t, ph, ds, sc, trouble, log_trouble, log_nad, log_pad, blockIdx.x,
                                  blockIdx.y, smem_raw);
}

// ---------------------------------------------------------------------------
// k2_final: fallback fluxes at troubled faces of the tile (from pointwise
// primitives of the stage input with 2 ghosts), the blend with the
// high-order fluxes, the divergence and the Runge-Kutta combination.
// ---------------------------------------------------------------------------
template <int TX, int TY>
struct FinalDims {
  static constexpr int PX = TX + 4, PY = TY + 4;
  static constexpr int SP = PX * PY * 5;
  static constexpr int SF = (TX + 1) * TY * 5;
  static constexpr int SG = TX * (TY + 1) * 5;
};

template <typename Tc, int TX, int TY>
__device__ __forceinline__ void tile2_final(const double* __restrict__ stage_in, Geo g, V2<const Tc> F,
                                            V2<const Tc> G, const uint8_t* __restrict__ trouble,
                                            const uint8_t* __restrict__ pred, int apost, int muscl, int limiter,
                                            Phys<Tc> ph, double cx, double cy, StageSpec st, double dt_step,
                                            Scalars* __restrict__ sc, int bx, int by, unsigned char* smem_raw) {
  using D = FinalDims<TX, TY>;
  Tc* Pw = reinterpret_cast<Tc*>(smem_raw);
  Tc* FX = Pw + D::SP;
  Tc* GY = FX + D::SF;
  const int nt = blockDim.x;
  const int x0 = by * TX, y0 = bx * TY;
  // high-order fluxes of the tile's faces
  for (int i = threadIdx.x; i < (TX + 1) * TY; i += nt) {
    const int f = i / TY, q = i - f * TY;
    const int x = min(x0 + f, g.nx), y = min(y0 + q, g.ny - 1);
    const Tc* p = F.p + F.at(x, y);
#pragma unroll
    for (int v = 0; v < 5; ++v) FX[(v * (TX + 1) + f) * TY + q] = p[v * F.vs];
  }
  for (int i = threadIdx.x; i < TX * (TY + 1); i += nt) {
    const int r = i / (TY + 1), f = i - r * (TY + 1);
    const int x = min(x0 + r, g.nx - 1), y = min(y0 + f, g.ny);
    const Tc* p = G.p + G.at(x, y);
#pragma unroll
    for (int v = 0; v < 5; ++v) GY[(v * TX + r) * (TY + 1) + f] = p[v * G.vs];
  }
  // fallback at the faces of troubled cells; with predicted flags, faces next
  // to a predicted cell already hold their fallback flux (k2_fluxes) and only
  // the faces of missed cells are revised here
  if (apost && tile_any<TX, TY>(trouble, pred, g, x0, y0)) {
    pointwise_tile<Tc, TX, TY>(stage_in, g, x0, y0, Pw, ph);
    __syncthreads();
    // X faces
    for (int i = threadIdx.x; i < (TX + 1) * TY; i += nt) {
      const int f = i / TY, q = i - f * TY;
      const int x = x0 + f, y = y0 + q;
      if (x > g.nx || y >= g.ny) continue;
      const int ol = (x - 1) * g.ny + y, orr = x * g.ny + y;
      const bool tl = x >= 1 && trouble[ol], trr = x < g.nx && trouble[orr];
      if (!(tl || trr)) continue;
      if (pred && ((x >= 1 && pred[ol]) || (x < g.nx && pred[orr]))) continue;
      Tc flo[5];
      fallback_face_flux<Tc>(Pw + f * D::PY + q + 2, D::PX * D::PY, D::PY, muscl, limiter, ph, g.dx, flo);
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        Tc& fh = FX[(v * (TX + 1) + f) * TY + q];
        fh = (Tc(1) - Tc(1)) * fh + Tc(1) * flo[v];
      }
    }
    // Y faces
    for (int i = threadIdx.x; i < TX * (TY + 1); i += nt) {
      const int r = i / (TY + 1), f = i - r * (TY + 1);
      const int x = x0 + r, y = y0 + f;
      if (x >= g.nx || y > g.ny) continue;
      const int ol = x * g.ny + y - 1, orr = x * g.ny + y;
      const bool tl = y >= 1 && trouble[ol], trr = y < g.ny && trouble[orr];
      if (!(tl || trr)) continue;
      if (pred && ((y >= 1 && pred[ol]) || (y < g.ny && pred[orr]))) continue;
      Tc flo[5];
      fallback_face_flux<Tc>(Pw + (r + 2) * D::PY + f, D::PX * D::PY, 1, muscl, limiter, ph, g.dy, flo);
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        Tc& fh = GY[(v * TX + r) * (TY + 1) + f];
        fh = (Tc(1) - Tc(1)) * fh + Tc(1) * flo[v];
      }
    }
  }
  __syncthreads();
  // divergence and the Runge-Kutta combination
  const double dt = st.integrator == INT_RHS ? 0.0 : dt_step;
  const int plane = g.nx * g.ny;
  unsigned int bad = 0;
  for (int i = threadIdx.x; i < TX * TY; i += nt) {
    const int r = i / TY, q = i - r * TY;
    const int x = x0 + r, y = y0 + q;
    if (x >= g.nx || y >= g.ny) continue;
    const int base = x * g.ny + y;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      Tc dc = Tc(0);
      dc = dc + (Tc)cx * (FX[(v * (TX + 1) + r + 1) * TY + q] - FX[(v * (TX + 1) + r) * TY + q]);
      dc = dc + (Tc)cy * (GY[(v * TX + r) * (TY + 1) + q + 1] - GY[(v * TX + r) * (TY + 1) + q]);
      const int o = base + v * plane;
      const double k = (double)dc;
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
            const double qd = 0.25 * dt;
            res = (st.u[o] + qd * a) + qd * k;
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

template <typename Tc, int TX, int TY>
__global__ void __launch_bounds__(256)
    k2_final(const double* __restrict__ stage_in, Geo g, V2<const Tc> F, V2<const Tc> G,
             const uint8_t* __restrict__ trouble, const uint8_t* __restrict__ pred, int apost, int muscl, int limiter,
             Phys<Tc> ph, double cx, double cy, StageSpec st, Scalars* __restrict__ sc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  tile2_final<Tc, TX, TY>(stage_in, g, F, G, trouble, pred, apost, muscl, limiter, ph, cx, cy, st,
                          st.integrator == INT_RHS ? 0.0 : sc->dt_step, sc, blockIdx.x, blockIdx.y, smem_raw);
}

}  // namespace f2
}  // namespace fvh
