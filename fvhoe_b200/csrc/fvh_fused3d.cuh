// Fused 3D primitive pass: the FV primitives of a conserved state over a
// ghost-padded box, one shared-memory tile per block, instead of the generic
// path's six sweep launches (three centre sweeps, the last converting to
// primitives, and three transverse sweeps; fvhoe/solver.py:753-792).
//
// For problems with three active axes, five variables, the same degree p on
// every axis and no Dirichlet sides. Every output is the generic path's value
// bit for bit: the sweeps run in the same axis order (centre x, y, z; the
// conversion; transverse x, y, z), every sum is accumulated from tap 0 upwards
// as a one-output loop accumulates it, and ghost cells are read through the
// same ghost maps (fvhoe/boundary_conditions.py:60-151). The output layout is
// the generic path's View over [-g, n+g)^3 (z contiguous), so the flux,
// detection and fallback passes read it unchanged.
//
// A tile of OX x OY x OZ outputs is computed variable by variable: the state
// tile with 2 RC ghost cells per side (RC = p / 2, the radius of the centre and
// transverse rules), the three centre sweeps into C (all five variables), the
// pointwise conversion in C, then per variable the three transverse sweeps,
// the last one writing W. The CFL and extrema reductions, which need all five
// primitives of a point, read the tile's W back after a block barrier.
#pragma once

#include "fvh_fused2d.cuh"

namespace fvh {
namespace f3 {

template <typename Tc, int P, int OX, int OY, int OZ>
struct Prims3Dims {
  static constexpr int RC = P / 2;
  static constexpr int LX = OX + 4 * RC, LY = OY + 4 * RC, LZ = OZ + 4 * RC;  // state tile
  static constexpr int CX = OX + 2 * RC, CY = OY + 2 * RC, CZ = OZ + 2 * RC;  // after the centre sweeps
  static constexpr int R1 = f2::Max<LX * LY * LZ, OX * CY * CZ>::value;     // state tile; transverse x
  static constexpr int R2 = f2::Max<CX * LY * LZ, OX * OY * CZ>::value;     // centre x; transverse y
  static constexpr int RC5 = 5 * CX * CY * CZ;                              // centre sweeps of all variables
  static constexpr int TOTAL = R1 + R2 + RC5;                               // elements of the compute type
};

// out(x, y, z) = sum_k w[k] in(x + k [AX = 0], y + k [AX = 1], z + k [AX = 2])
// over an NX x NY x NZ box; `in` has row strides ISX (x) and ISY (y), z
// contiguous; each sum accumulated from tap 0 upwards. Threads run along z.
template <typename Tc, int K, int AX, int NX, int NY, int NZ, int ISX, int ISY, typename Epi>
__device__ __forceinline__ void sweep3(const Tc* __restrict__ in, const Tc* __restrict__ w, Epi epi) {
  constexpr int ST = AX == 0 ? ISX : (AX == 1 ? ISY : 1);
  for (int i = threadIdx.x; i < NX * NY * NZ; i += blockDim.x) {
    const int x = i / (NY * NZ), rem = i - x * (NY * NZ), y = rem / NZ, z = rem - y * NZ;
    const Tc* p = in + x * ISX + y * ISY + z;
    Tc acc = Tc(0);
#pragma unroll
    for (int k = 0; k < K; ++k) acc = acc + w[k] * p[k * ST];
    epi(x, y, z, acc);
  }
}

// W over [-g, n+g)^3 (the generic View layout) in tiles of OX x OY x OZ
// outputs; block (bz, by, bx) = (blockIdx.x, blockIdx.y, blockIdx.z) covers
// outputs from (-g + bx OX, -g + by OY, -g + bz OZ). Tin: the stored type of
// the state (double). REDUCE: the CFL maximum over rs.cfl_box and the
// per-variable extrema over rs.ext_box.
template <typename Tc, int P, int OX, int OY, int OZ, int KC, bool REDUCE, typename Tin>
__global__ void __launch_bounds__(256)
    k3_primitives(const Tin* __restrict__ u, Grid grid, View<Tc> W, int g, Rule<Tc, KC> c, Rule<Tc, KC> t,
                  Phys<Tc> ph, ReduceSpec rs, Scalars* __restrict__ sc) {
  using D = Prims3Dims<Tc, P, OX, OY, OZ>;
  constexpr int RC = D::RC;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Tc* const R1 = reinterpret_cast<Tc*>(smem_raw);
  Tc* const R2 = R1 + D::R1;
  Tc* const C = R2 + D::R2;
  const int x0 = -g + (int)blockIdx.z * OX, y0 = -g + (int)blockIdx.y * OY, z0 = -g + (int)blockIdx.x * OZ;
  const int n0 = grid.n[0], n1 = grid.n[1], n2 = grid.n[2];
  const int gmax = g + 2 * RC;
  const int plane = n0 * n1 * n2;
  // ---- centre sweeps x, y, z of each variable into C
  for (int v = 0; v < 5; ++v) {
    // state tile with 2 RC ghost cells per side; points past the deepest
    // ghost cell any output needs are clamped into range (they feed no output)
    for (int i = threadIdx.x; i < D::LX * D::LY * D::LZ; i += blockDim.x) {
      const int r = i / (D::LY * D::LZ), rem = i - r * (D::LY * D::LZ), q = rem / D::LZ, s = rem - q * D::LZ;
      const int xi = min(max(x0 - 2 * RC + r, -gmax), n0 + gmax - 1);
      const int yi = min(max(y0 - 2 * RC + q, -gmax), n1 + gmax - 1);
      const int zi = min(max(z0 - 2 * RC + s, -gmax), n2 + gmax - 1);
      bool fx = false, fy = false, fz = false;
      const int jx = ghost_source(xi, n0, grid.bc[0][0], grid.bc[0][1], fx);
      const int jy = ghost_source(yi, n1, grid.bc[1][0], grid.bc[1][1], fy);
      const int jz = ghost_source(zi, n2, grid.bc[2][0], grid.bc[2][1], fz);
      double val = (double)u[v * plane + (jx * n1 + jy) * n2 + jz];
      if ((v == 1 && fx) || (v == 2 && fy) || (v == 3 && fz)) val = -val;
      R1[i] = (Tc)val;
    }
    __syncthreads();
    sweep3<Tc, KC, 0, D::CX, D::LY, D::LZ, D::LY * D::LZ, D::LZ>(
        R1, c.w, [&](int x, int y, int z, Tc a) { R2[(x * D::LY + y) * D::LZ + z] = a; });
    __syncthreads();
    sweep3<Tc, KC, 1, D::CX, D::CY, D::LZ, D::LY * D::LZ, D::LZ>(
        R2, c.w, [&](int x, int y, int z, Tc a) { R1[(x * D::CY + y) * D::LZ + z] = a; });
    __syncthreads();
    Tc* Cv = C + v * (D::CX * D::CY * D::CZ);
    sweep3<Tc, KC, 2, D::CX, D::CY, D::CZ, D::CY * D::LZ, D::LZ>(
        R1, c.w, [&](int x, int y, int z, Tc a) { Cv[(x * D::CY + y) * D::CZ + z] = a; });
    __syncthreads();
  }
  // ---- conserved -> primitive at every point of C
  constexpr int NC = D::CX * D::CY * D::CZ;
  for (int i = threadIdx.x; i < NC; i += blockDim.x) {
    Tc uc[5], w[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) uc[v] = C[v * NC + i];
    to_primitives(ph, 5, uc, w);
#pragma unroll
    for (int v = 0; v < 5; ++v) C[v * NC + i] = w[v];
  }
  __syncthreads();
  // ---- transverse sweeps x, y, z of each variable; the last writes W
  for (int v = 0; v < 5; ++v) {
    const Tc* Cv = C + v * NC;
    sweep3<Tc, KC, 0, OX, D::CY, D::CZ, D::CY * D::CZ, D::CZ>(
        Cv, t.w, [&](int x, int y, int z, Tc a) { R1[(x * D::CY + y) * D::CZ + z] = a; });
    __syncthreads();
    sweep3<Tc, KC, 1, OX, OY, D::CZ, D::CY * D::CZ, D::CZ>(
        R1, t.w, [&](int x, int y, int z, Tc a) { R2[(x * OY + y) * D::CZ + z] = a; });
    __syncthreads();
    Tc* Wv = W.p + v * W.vs;
    sweep3<Tc, KC, 2, OX, OY, OZ, OY * D::CZ, D::CZ>(R2, t.w, [&](int x, int y, int z, Tc a) {
      const int xi = x0 + x, yi = y0 + y, zi = z0 + z;
      if (xi < n0 + g && yi < n1 + g && zi < n2 + g) Wv[W.at(xi, yi, zi)] = a;
    });
    __syncthreads();
  }
  if constexpr (REDUCE) {
    // the block's own W outputs, visible to the block after the barrier above
    unsigned long long cfl_key = 0ull, kmax[5], kmin[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      kmax[v] = 0ull;
      kmin[v] = ~0ull;
    }
    for (int i = threadIdx.x; i < OX * OY * OZ; i += blockDim.x) {
      const int x = i / (OY * OZ), rem = i - x * (OY * OZ), y = rem / OZ, z = rem - y * OZ;
      const int xi = x0 + x, yi = y0 + y, zi = z0 + z;
      if (xi >= n0 + g || yi >= n1 + g || zi >= n2 + g) continue;
      Tc w[5];
      const Tc* p = W.p + W.at(xi, yi, zi);
#pragma unroll
      for (int v = 0; v < 5; ++v) w[v] = p[v * W.vs];
      if (rs.cfl && in_box(rs.cfl_box, xi, yi, zi)) {
        const unsigned long long k = order_key((double)cfl_speed(ph, w, (Tc)rs.ndim));
        cfl_key = k > cfl_key ? k : cfl_key;
      }
      if (rs.extrema && in_box(rs.ext_box, xi, yi, zi)) {
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          const unsigned long long k = order_key((double)w[v]);
          kmax[v] = k > kmax[v] ? k : kmax[v];
          kmin[v] = k < kmin[v] ? k : kmin[v];
        }
      }
    }
    f2::reduce_keys_and_publish(cfl_key, kmax, kmin, rs, sc);
  }
}

}  // namespace f3
}  // namespace fvh
