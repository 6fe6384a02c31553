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

namespace fvh {
namespace f3 {

// ---------------------------------------------------------------------------
// Fused 3D flux pass along one direction D (fvhoe/solver.py:519-651): the
// generic path's centre sweeps along (D+2)%3 then (D+1)%3, the face states
// along D with the Riemann solve, and the transverse sweeps along the other
// two axes in ascending order, for a tile of faces in one launch; every
// output bit for bit the generic value. The tile holds O[D] faces along D
// (face j between cells j-1 and j) and O[t] cells along the other axes.
// ---------------------------------------------------------------------------
template <typename Tc, int P, int D, int TX, int TY, int TZ>
struct Flux3Dims {
  static constexpr int R = (P + 1) / 2, RC = P / 2, KF = 2 * R + 1;
  static constexpr int T1 = (D + 2) % 3, T2 = (D + 1) % 3;            // centre sweep order
  static constexpr int TA = T1 < T2 ? T1 : T2, TB = T1 < T2 ? T2 : T1;  // transverse order
  static constexpr int O[3] = {TX, TY, TZ};
  // extent along axis a of: the W tile (L), after the first centre sweep (M),
  // after both (X, all variables), the faces (Y, all variables), after the
  // first transverse sweep (Q)
  static constexpr int ext_l(int a) { return a == D ? O[a] + 2 * R + 1 : O[a] + 4 * RC; }
  static constexpr int ext_m(int a) { return a == T1 ? O[a] + 2 * RC : ext_l(a); }
  static constexpr int ext_x(int a) { return a == D ? O[a] + 2 * R + 1 : O[a] + 2 * RC; }
  static constexpr int ext_y(int a) { return a == D ? O[a] : O[a] + 2 * RC; }
  static constexpr int ext_q(int a) { return a == TA ? O[a] : ext_y(a); }
  static constexpr int NL = ext_l(0) * ext_l(1) * ext_l(2), NM = ext_m(0) * ext_m(1) * ext_m(2);
  static constexpr int NX = ext_x(0) * ext_x(1) * ext_x(2), NY = ext_y(0) * ext_y(1) * ext_y(2);
  static constexpr int NQ = ext_q(0) * ext_q(1) * ext_q(2);
  static constexpr int RA = f2::Max<NL + NM, 5 * NY>::value;  // W tile + first sweep; then the face fluxes
  static constexpr int RX = f2::Max<5 * NX, NQ>::value;       // centre-swept tiles; then the first transverse sweep
  static constexpr int TOTAL = RA + RX;
};

// One sweep along axis AX between two z-contiguous boxes: out extents
// (E0, E1, E2); in extents are out's, grown by K-1 along AX.
template <typename Tc, int K, int AX, int E0, int E1, int E2, typename Epi>
__device__ __forceinline__ void sweep_box(const Tc* __restrict__ in, const Tc* __restrict__ w, Epi epi) {
  constexpr int I1 = E1 + (AX == 1 ? K - 1 : 0), I2 = E2 + (AX == 2 ? K - 1 : 0);
  sweep3<Tc, K, AX, E0, E1, E2, I1 * I2, I2>(in, w, epi);
}

template <typename Tc, int P, int D, int TX, int TY, int TZ, int KC, int KF>
__global__ void __launch_bounds__(256)
    k3_fluxes(View<const Tc> W, int gw, Grid grid, View<Tc> F, Rule<Tc, KC> c, Rule<Tc, KC> t, Rule<Tc, KF> lrule,
              Rule<Tc, KF> rrule, Phys<Tc> ph) {
  using Dm = Flux3Dims<Tc, P, D, TX, TY, TZ>;
  constexpr int R = Dm::R, RC = Dm::RC, T1 = Dm::T1, T2 = Dm::T2, TA = Dm::TA, TB = Dm::TB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Tc* const RA = reinterpret_cast<Tc*>(smem_raw);
  Tc* const RX = RA + Dm::RA;
  Tc* const L = RA;             // W tile of one variable
  Tc* const M = RA + Dm::NL;    // after the first centre sweep
  Tc* const Y = RA;             // face fluxes (all variables), after the W tiles are consumed
  Tc* const X = RX;             // after both centre sweeps (all variables)
  Tc* const Q = RX;             // first transverse sweep, after X is consumed
  // tile origin: faces along D, cells along the others
  const int o[3] = {(int)blockIdx.z * TX, (int)blockIdx.y * TY, (int)blockIdx.x * TZ};
  const int n[3] = {grid.n[0], grid.n[1], grid.n[2]};
  // W tile origin: cells o[D]-1-R along D, o[t]-2RC along the others
  int l0[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) l0[a] = a == D ? o[a] - 1 - R : o[a] - 2 * RC;
  constexpr int L0 = Dm::ext_l(0), L1 = Dm::ext_l(1), L2 = Dm::ext_l(2);
  constexpr int M0 = Dm::ext_m(0), M1 = Dm::ext_m(1), M2 = Dm::ext_m(2);
  constexpr int X0 = Dm::ext_x(0), X1 = Dm::ext_x(1), X2 = Dm::ext_x(2);
  constexpr int Y0 = Dm::ext_y(0), Y1 = Dm::ext_y(1), Y2 = Dm::ext_y(2);
  constexpr int Q0 = Dm::ext_q(0), Q1 = Dm::ext_q(1), Q2 = Dm::ext_q(2);
  for (int v = 0; v < 5; ++v) {
    // W tile; points past W's ghost range are clamped (they feed no output)
    const Tc* Wv = W.p + v * W.vs;
    for (int i = threadIdx.x; i < Dm::NL; i += blockDim.x) {
      const int a = i / (L1 * L2), rem = i - a * (L1 * L2), b = rem / L2, e = rem - b * L2;
      const int x = min(l0[0] + a, n[0] + gw - 1), y = min(l0[1] + b, n[1] + gw - 1), z = min(l0[2] + e, n[2] + gw - 1);
      L[i] = Wv[W.at(x, y, z)];
    }
    __syncthreads();
    sweep_box<Tc, KC, T1, M0, M1, M2>(L, c.w, [&](int a, int b, int e, Tc s) { M[(a * M1 + b) * M2 + e] = s; });
    __syncthreads();
    Tc* Xv = X + v * Dm::NX;
    sweep_box<Tc, KC, T2, X0, X1, X2>(M, c.w, [&](int a, int b, int e, Tc s) { Xv[(a * X1 + b) * X2 + e] = s; });
    __syncthreads();
  }
  // faces along D: face j of the tile between X cells j+R (right-face rule)
  // and j+R+1 (left-face rule), each sum from tap 0 upwards
  constexpr int SD = D == 0 ? X1 * X2 : (D == 1 ? X2 : 1);
  for (int i = threadIdx.x; i < Dm::NY; i += blockDim.x) {
    const int a = i / (Y1 * Y2), rem = i - a * (Y1 * Y2), b = rem / Y2, e = rem - b * Y2;
    const int base = (a * X1 + b) * X2 + e;  // X point of the face's first tap
    Tc wl[5], wr[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const Tc* q = X + v * Dm::NX + base;
      Tc sl = Tc(0), sr = Tc(0);
#pragma unroll
      for (int k = 0; k < KF; ++k) {
        sl = sl + rrule.w[k] * q[k * SD];
        sr = sr + lrule.w[k] * q[(k + 1) * SD];
      }
      wl[v] = sl;
      wr[v] = sr;
    }
    Tc f[5];
    riemann_flux<5>(ph, 5, wl, wr, D, f);
#pragma unroll
    for (int v = 0; v < 5; ++v) Y[v * Dm::NY + i] = f[v];
  }
  __syncthreads();
  // transverse sweeps along TA then TB; the last writes the owned faces of F
  for (int v = 0; v < 5; ++v) {
    sweep_box<Tc, KC, TA, Q0, Q1, Q2>(Y + v * Dm::NY, t.w,
                                      [&](int a, int b, int e, Tc s) { Q[(a * Q1 + b) * Q2 + e] = s; });
    __syncthreads();
    Tc* Fv = F.p + v * F.vs;
    sweep_box<Tc, KC, TB, TX, TY, TZ>(Q, t.w, [&](int a, int b, int e, Tc s) {
      const int x = o[0] + a, y = o[1] + b, z = o[2] + e;
      if (x < n[0] + (D == 0) && y < n[1] + (D == 1) && z < n[2] + (D == 2)) Fv[F.at(x, y, z)] = s;
    });
    __syncthreads();
  }
}

}  // namespace f3
}  // namespace fvh
