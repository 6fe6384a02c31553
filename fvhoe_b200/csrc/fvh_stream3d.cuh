// Streaming 3D primitive pass: the FV primitives of a conserved state over a
// ghost-padded box in one launch instead of the generic path's six sweeps
// (three centre sweeps, the last converting to primitives, three transverse
// sweeps; fvhoe/solver.py:753-792), for three active axes, five variables and
// the same degree p <= 3 on every axis without Dirichlet sides.
//
// Each block owns a y-z tile of OY x OZ outputs and slides along x over a
// chunk of output planes, so every state plane is read from memory once per
// tile instead of once per x tile, and the x-direction sweeps run on rings of
// planes kept in shared memory:
//   plane i of the state is loaded through registers (its loads in flight
//   while the plane before it is computed), sign-corrected and converted,
//   into a ring of 2RC+1 planes;
//   C(i) = C_z C_y C_x u at plane i (RC = p / 2, the centre rule's radius),
//   converted to primitives, into a ring of 2RC+1 planes;
//   W(i-RC) = T_z T_y T_x of the primitive ring, written to global memory.
// The sweeps along x and y run on whole 16-byte vectors along z (rows of the
// tiles are padded to whole vectors), the sweeps along z one point at a time.
// Every sum runs from tap 0 upwards in the generic path's axis order, and the
// ghost cells come through the same ghost maps (fvhoe/boundary_conditions.py:
// 60-151) with the reflective sign applied to the FP64 value before the
// conversion, so W equals the generic passes bit for bit. The output layout is
// the generic View over [-g, n+g)^3 (z contiguous).
#pragma once

#include "fvh_fused2d.cuh"

namespace fvh {
namespace s3 {

template <typename Tc, int P, int OY, int OZ, int NT = 256>
struct Stream3Dims {
  static constexpr int VW = 16 / (int)sizeof(Tc);  // elements per 16-byte shared-memory vector
  static constexpr int RC = P / 2;
  static constexpr int LY = OY + 4 * RC, LZ = OZ + 4 * RC;  // state plane tile
  static constexpr int CY = OY + 2 * RC, CZ = OZ + 2 * RC;  // after the centre sweeps
  static constexpr int CZS = (CZ + VW - 1) / VW * VW;       // primitive rows padded to whole vectors
  static_assert(OZ % VW == 0 && LZ % VW == 0, "tile rows must hold whole vectors");
  static constexpr int NU = 2 * RC + 1;  // state ring (the centre rule's planes)
  static constexpr int NP = 2 * RC + 1;  // primitive ring
  static constexpr int PL = LY * LZ, PCS = CY * CZS;
  // shared memory, in elements of the compute type: the state ring (NU x 5 x
  // PL); A, the x-swept plane (5 x LY x LZ), later the x-transverse plane
  // (5 x CY x CZS); B, the y-swept plane (5 x CY x LZ), later the y-transverse
  // plane (5 x OY x CZS); the primitive ring (NP x 5 x CY x CZS); then the
  // offsets and flip bits of the plane tile's y-z points
  static constexpr int U_ELEMS = NU * 5 * PL, A_ELEMS = 5 * PL, B_ELEMS = 5 * CY * LZ, R_ELEMS = NP * 5 * PCS;
  static_assert(5 * CY * CZS <= A_ELEMS && 5 * OY * CZS <= B_ELEMS, "transverse planes fit the swept ones");
  static constexpr int LOADS = (5 * PL + NT - 1) / NT;  // state values a thread stages per plane
  static constexpr int BYTES = (U_ELEMS + A_ELEMS + B_ELEMS + R_ELEMS) * (int)sizeof(Tc) + PL * 4 + PL + 16;
  // resident blocks the shared memory allows (at most 768 threads per SM), for
  // the launch bounds
  static constexpr int FIT = (228 * 1024) / (BYTES + 1024);
  static constexpr int CAP = 768 / NT;
  static constexpr int BLOCKS = FIT < 1 ? 1 : (FIT > CAP ? CAP : FIT);
};

__device__ __forceinline__ int ring(int i, int n) {
  const int r = i % n;
  return r < 0 ? r + n : r;
}


// W over [-g, n+g)^3 for a block's y-z tile (blockIdx.x along z, blockIdx.y
// along y) and its chunk of output planes along x (blockIdx.z). REDUCE: the
// CFL maximum over rs.cfl_box and the per-variable extrema over rs.ext_box.
template <typename Tc, int P, int OY, int OZ, int NT, int KC, bool REDUCE>
__global__ void __launch_bounds__(NT, (Stream3Dims<Tc, P, OY, OZ, NT>::BLOCKS))
    k3s_primitives(const double* __restrict__ u, Grid grid, View<Tc> W, int g, int chunk, Rule<Tc, KC> c,
                   Rule<Tc, KC> t, Phys<Tc> ph, ReduceSpec rs, Scalars* __restrict__ sc) {
  using D = Stream3Dims<Tc, P, OY, OZ, NT>;
  constexpr int RC = D::RC, LY = D::LY, LZ = D::LZ, CY = D::CY, CZ = D::CZ, CZS = D::CZS, PL = D::PL,
                PCS = D::PCS, NU = D::NU, NP = D::NP, VW = D::VW;
  extern __shared__ __align__(16) unsigned char smem[];
  Tc* const U = reinterpret_cast<Tc*>(smem);  // NU x 5 x PL: state planes, sign-corrected, converted
  Tc* const A = U + D::U_ELEMS;
  Tc* const B = A + D::A_ELEMS;
  Tc* const R = B + D::B_ELEMS;
  int* const off = reinterpret_cast<int*>(R + D::R_ELEMS);              // y-z source offset of each plane point
  unsigned char* const fl = reinterpret_cast<unsigned char*>(off + PL);  // bit 0: y mirror flips, bit 1: z
  const int n0 = grid.n[0], n1 = grid.n[1], n2 = grid.n[2];
  const int gmax = g + 2 * RC;
  const int plane = n0 * n1 * n2;
  const int y0 = -g + (int)blockIdx.y * OY, z0 = -g + (int)blockIdx.x * OZ;
  const int xb = -g + (int)blockIdx.z * chunk;
  const int xe = min(xb + chunk, n0 + g);
  // ghost maps of the tile's y-z points (the same for every plane); points
  // past the deepest ghost cell any output needs are clamped (they feed none)
  for (int e = threadIdx.x; e < PL; e += NT) {
    const int r = e / LZ, q = e - r * LZ;
    const int yi = min(max(y0 - 2 * RC + r, -gmax), n1 + gmax - 1);
    const int zi = min(max(z0 - 2 * RC + q, -gmax), n2 + gmax - 1);
    bool fy = false, fz = false;
    const int jy = ghost_source(yi, n1, grid.bc[1][0], grid.bc[1][1], fy);
    const int jz = ghost_source(zi, n2, grid.bc[2][0], grid.bc[2][1], fz);
    off[e] = jy * n2 + jz;
    fl[e] = (unsigned char)((fy ? 1 : 0) | (fz ? 2 : 0));
  }
  __syncthreads();
  // a state plane is staged through registers: the loads of plane xi are
  // issued early (fetch), and the values stored into the ring later (store),
  // each sign-corrected in FP64 (the reflective mirror flips) and converted
  double stage[D::LOADS];
  bool stage_fx = false;
  auto fetch = [&](int xi) {
    const int xc = min(max(xi, -gmax), n0 + gmax - 1);
    stage_fx = false;  // ghost_source only sets the flag
    const int jx = ghost_source(xc, n0, grid.bc[0][0], grid.bc[0][1], stage_fx);
    const double* src = u + (size_t)jx * n1 * n2;
#pragma unroll
    for (int m = 0; m < D::LOADS; ++m) {
      const int idx = threadIdx.x + NT * m;
      if (idx < 5 * PL) {
        const int v = idx / PL, e = idx - v * PL;
        stage[m] = src[(size_t)v * plane + off[e]];
      }
    }
  };
  auto store = [&](int xi) {
    Tc* dst = U + ring(xi, NU) * 5 * PL;
#pragma unroll
    for (int m = 0; m < D::LOADS; ++m) {
      const int idx = threadIdx.x + NT * m;
      if (idx < 5 * PL) {
        const int v = idx / PL, e = idx - v * PL;
        double d = stage[m];
        if ((v == 1 && stage_fx) || (v == 2 && (fl[e] & 1)) || (v == 3 && (fl[e] & 2))) d = -d;
        dst[idx] = (Tc)d;
      }
    }
  };
  for (int xi = xb - 2 * RC; xi <= xb; ++xi) {
    fetch(xi);
    store(xi);
  }
  unsigned long long cfl_key = 0ull, kmax[5], kmin[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    kmax[v] = 0ull;
    kmin[v] = ~0ull;
  }
  for (int i = xb - RC; i < xe + RC; ++i) {
    __syncthreads();  // state planes i-RC .. i+RC are in the ring
    const bool ahead = i + RC + 1 <= xe - 1 + 2 * RC;
    if (ahead) fetch(i + RC + 1);  // in flight while this plane is computed
    // centre sweep along x: A = sum_k c_k U(i-RC+k), whole vectors of the plane
    {
      int sk[KC];
#pragma unroll
      for (int k = 0; k < KC; ++k) sk[k] = ring(i - RC + k, NU) * 5 * PL;
      for (int iv = threadIdx.x; iv < 5 * PL / VW; iv += NT) {
        Tc acc[VW];
#pragma unroll
        for (int j = 0; j < VW; ++j) acc[j] = Tc(0);
#pragma unroll
        for (int k = 0; k < KC; ++k) {
          Tc x[VW];
          f2::ldn<VW>(U + sk[k] + iv * VW, x);
#pragma unroll
          for (int j = 0; j < VW; ++j) acc[j] = acc[j] + c.w[k] * x[j];
        }
        f2::stn<VW>(A + iv * VW, acc);
      }
    }
    __syncthreads();
    // plane i+RC+1 into the slot of plane i-RC, which the centre sweep above
    // was the last to read (the next iteration's first barrier orders it)
    if (ahead) store(i + RC + 1);
    // centre sweep along y: B (5 x CY x LZ), whole vectors along z
    {
      constexpr int LZV = LZ / VW;
      for (int it = threadIdx.x; it < 5 * CY * LZV; it += NT) {
        const int r = it / LZV, zq = it - r * LZV;
        const int v = r / CY, y = r - v * CY;
        const Tc* p = A + (v * LY + y) * LZ + zq * VW;
        Tc acc[VW];
#pragma unroll
        for (int j = 0; j < VW; ++j) acc[j] = Tc(0);
#pragma unroll
        for (int k = 0; k < KC; ++k) {
          Tc x[VW];
          f2::ldn<VW>(p + k * LZ, x);
#pragma unroll
          for (int j = 0; j < VW; ++j) acc[j] = acc[j] + c.w[k] * x[j];
        }
        f2::stn<VW>(B + r * LZ + zq * VW, acc);
      }
    }
    __syncthreads();
    // centre sweep along z and the conversion: primitive plane i into its ring
    // slot (rows of CZS; the padding columns are never written and feed only
    // padding outputs)
    {
      Tc* Ri = R + ring(i, NP) * 5 * PCS;
      for (int idx = threadIdx.x; idx < CY * CZ; idx += NT) {
        const int y = idx / CZ, z = idx - y * CZ;
        Tc uc[5], w[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          const Tc* p = B + (v * CY + y) * LZ + z;
          Tc acc = Tc(0);
#pragma unroll
          for (int k = 0; k < KC; ++k) acc = acc + c.w[k] * p[k];
          uc[v] = acc;
        }
        to_primitives(ph, 5, uc, w);
#pragma unroll
        for (int v = 0; v < 5; ++v) Ri[(v * CY + y) * CZS + z] = w[v];
      }
    }
    __syncthreads();
    const int xo = i - RC;
    if (xo < xb) continue;
    // transverse sweep along x over the primitive ring: A (5 x CY x CZS)
    {
      int rk[KC];
#pragma unroll
      for (int k = 0; k < KC; ++k) rk[k] = ring(xo - RC + k, NP) * 5 * PCS;
      for (int iv = threadIdx.x; iv < 5 * PCS / VW; iv += NT) {
        Tc acc[VW];
#pragma unroll
        for (int j = 0; j < VW; ++j) acc[j] = Tc(0);
#pragma unroll
        for (int k = 0; k < KC; ++k) {
          Tc x[VW];
          f2::ldn<VW>(R + rk[k] + iv * VW, x);
#pragma unroll
          for (int j = 0; j < VW; ++j) acc[j] = acc[j] + t.w[k] * x[j];
        }
        f2::stn<VW>(A + iv * VW, acc);
      }
    }
    __syncthreads();
    // transverse sweep along y: B (5 x OY x CZS), whole vectors along z
    {
      constexpr int CZV = CZS / VW;
      for (int it = threadIdx.x; it < 5 * OY * CZV; it += NT) {
        const int r = it / CZV, zq = it - r * CZV;
        const int v = r / OY, y = r - v * OY;
        const Tc* p = A + (v * CY + y) * CZS + zq * VW;
        Tc acc[VW];
#pragma unroll
        for (int j = 0; j < VW; ++j) acc[j] = Tc(0);
#pragma unroll
        for (int k = 0; k < KC; ++k) {
          Tc x[VW];
          f2::ldn<VW>(p + k * CZS, x);
#pragma unroll
          for (int j = 0; j < VW; ++j) acc[j] = acc[j] + t.w[k] * x[j];
        }
        f2::stn<VW>(B + r * CZS + zq * VW, acc);
      }
    }
    __syncthreads();
    // transverse sweep along z: W at output plane xo, and the reductions
    for (int idx = threadIdx.x; idx < OY * OZ; idx += NT) {
      const int y = idx / OZ, z = idx - y * OZ;
      const int yi = y0 + y, zi = z0 + z;
      if (yi >= n1 + g || zi >= n2 + g) continue;
      Tc w[5];
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        const Tc* p = B + (v * OY + y) * CZS + z;
        Tc acc = Tc(0);
#pragma unroll
        for (int k = 0; k < KC; ++k) acc = acc + t.w[k] * p[k];
        w[v] = acc;
      }
      Tc* o = W.p + W.at(xo, yi, zi);
#pragma unroll
      for (int v = 0; v < 5; ++v) o[v * W.vs] = w[v];
      if constexpr (REDUCE) {
        if (rs.cfl && in_box(rs.cfl_box, xo, yi, zi)) {
          const unsigned long long k = order_key((double)cfl_speed(ph, w, (Tc)rs.ndim));
          cfl_key = k > cfl_key ? k : cfl_key;
        }
        if (rs.extrema && in_box(rs.ext_box, xo, yi, zi)) {
#pragma unroll
          for (int v = 0; v < 5; ++v) {
            const unsigned long long k = order_key((double)w[v]);
            kmax[v] = k > kmax[v] ? k : kmax[v];
            kmin[v] = k < kmin[v] ? k : kmin[v];
          }
        }
      }
    }
  }
  if constexpr (REDUCE) f2::reduce_keys_and_publish(cfl_key, kmax, kmin, rs, sc);
}

}  // namespace s3
// ---------------------------------------------------------------------------
// Two consecutive sweeps of five variables in one launch: out = S2(S1(in)),
// S1 along axis A1 with rule r1 (K1 taps), S2 along A2 with r2 (K2 taps),
// every sum from tap 0 upwards and the intermediate rounded to Tc, as two
// sweep launches with a stored intermediate compute them. A block owns a tile
// of T0 x T1 x T2 outputs (axis 2 contiguous, no halo on the unswept axis):
// it loads the input tile with its halos, sweeps it along A1 into a second
// shared tile and sweeps that along A2 into the output, one point per thread
// and pass. Input points past the input region (only partial tiles reach
// them) are clamped into it; they feed only outputs past the box, which are
// not stored.
// ---------------------------------------------------------------------------
template <int A1, int A2, int K1, int K2, int T0, int T1, int T2>
struct PairDims {
  static constexpr int N0 = T0 + (A1 == 0 ? K1 - 1 : 0) + (A2 == 0 ? K2 - 1 : 0);
  static constexpr int N1 = T1 + (A1 == 1 ? K1 - 1 : 0) + (A2 == 1 ? K2 - 1 : 0);
  static constexpr int N2 = T2 + (A1 == 2 ? K1 - 1 : 0) + (A2 == 2 ? K2 - 1 : 0);
  static constexpr int M0 = T0 + (A2 == 0 ? K2 - 1 : 0);  // after the first sweep
  static constexpr int M1 = T1 + (A2 == 1 ? K2 - 1 : 0);
  static constexpr int M2 = T2 + (A2 == 2 ? K2 - 1 : 0);
  static constexpr int NP = N0 * N1 * N2, MP = M0 * M1 * M2;
  template <typename Tc>
  static constexpr int bytes() {
    return 5 * (NP + MP) * (int)sizeof(Tc);
  }
};

template <typename Tc, int A1, int A2, int K1, int K2, int T0, int T1, int T2, int MINB>
__global__ void __launch_bounds__(256, MINB)
    k_sweep_pair(View<const Tc> in, Region rin, View<Tc> out, Box box, Rule<Tc, K1> r1, Rule<Tc, K2> r2) {
  static_assert(A1 != A2, "two different axes");
  using D = PairDims<A1, A2, K1, K2, T0, T1, T2>;
  constexpr int N1 = D::N1, N2 = D::N2, M1 = D::M1, M2 = D::M2;
  extern __shared__ __align__(16) unsigned char pair_smem[];
  Tc* const S = reinterpret_cast<Tc*>(pair_smem);  // 5 x N0 x N1 x N2
  Tc* const Mid = S + 5 * D::NP;                   // 5 x M0 x M1 x M2
  const int o0 = box.lo[0] + (int)blockIdx.z * T0, o1 = box.lo[1] + (int)blockIdx.y * T1,
            o2 = box.lo[2] + (int)blockIdx.x * T2;
  // input origin: the output origin moved by each sweep's first tap
  const int i0 = o0 + (A1 == 0 ? r1.off : 0) + (A2 == 0 ? r2.off : 0);
  const int i1 = o1 + (A1 == 1 ? r1.off : 0) + (A2 == 1 ? r2.off : 0);
  const int i2 = o2 + (A1 == 2 ? r1.off : 0) + (A2 == 2 ? r2.off : 0);
  for (int idx = threadIdx.x; idx < D::NP; idx += 256) {
    const int p0 = idx / (N1 * N2), rem = idx - p0 * (N1 * N2), p1 = rem / N2, p2 = rem - p1 * N2;
    const int g0 = min(i0 + p0, rin.lo[0] + rin.n[0] - 1), g1 = min(i1 + p1, rin.lo[1] + rin.n[1] - 1),
              g2 = min(i2 + p2, rin.lo[2] + rin.n[2] - 1);
    const Tc* q = in.p + in.at(g0, g1, g2);
#pragma unroll
    for (int v = 0; v < 5; ++v) S[v * D::NP + idx] = q[v * in.vs];
  }
  __syncthreads();
  constexpr int SA1 = A1 == 0 ? N1 * N2 : (A1 == 1 ? N2 : 1);  // stride of A1 in S
  for (int idx = threadIdx.x; idx < D::MP; idx += 256) {
    const int m0 = idx / (M1 * M2), rem = idx - m0 * (M1 * M2), m1 = rem / M2, m2 = rem - m1 * M2;
    const int src = (m0 * N1 + m1) * N2 + m2;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const Tc* q = S + v * D::NP + src;
      Tc acc = Tc(0);
#pragma unroll
      for (int k = 0; k < K1; ++k) acc = acc + r1.w[k] * q[k * SA1];
      Mid[v * D::MP + idx] = acc;
    }
  }
  __syncthreads();
  constexpr int SA2 = A2 == 0 ? M1 * M2 : (A2 == 1 ? M2 : 1);  // stride of A2 in Mid
  for (int idx = threadIdx.x; idx < T0 * T1 * T2; idx += 256) {
    const int t0 = idx / (T1 * T2), rem = idx - t0 * (T1 * T2), t1 = rem / T2, t2 = rem - t1 * T2;
    const int x0 = o0 + t0, x1 = o1 + t1, x2 = o2 + t2;
    if (x0 >= box.lo[0] + box.n[0] || x1 >= box.lo[1] + box.n[1] || x2 >= box.lo[2] + box.n[2]) continue;
    const int src = (t0 * M1 + t1) * M2 + t2;
    Tc* o = out.p + out.at(x0, x1, x2);
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const Tc* q = Mid + v * D::MP + src;
      Tc acc = Tc(0);
#pragma unroll
      for (int k = 0; k < K2; ++k) acc = acc + r2.w[k] * q[k * SA2];
      o[v * out.vs] = acc;
    }
  }
}

}  // namespace fvh
