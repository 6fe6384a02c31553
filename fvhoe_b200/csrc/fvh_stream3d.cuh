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
//   plane i of the state arrives by asynchronous copies (cp.async, raw FP64)
//   into a ring of 2RC+2 planes (one plane ahead of its use);
//   C(i) = C_z C_y C_x u at plane i (RC = p / 2, the centre rule's radius),
//   converted to primitives, into a ring of 2RC+1 planes;
//   W(i-RC) = T_z T_y T_x of the primitive ring, written to global memory.
// Every sum runs from tap 0 upwards in the generic path's axis order, and the
// ghost cells come through the same ghost maps (fvhoe/boundary_conditions.py:
// 60-151) with the reflective sign applied to the FP64 value before the
// conversion, so W equals the generic passes bit for bit. The output layout is
// the generic View over [-g, n+g)^3 (z contiguous).
#pragma once

#include "fvh_fused2d.cuh"

namespace fvh {
namespace s3 {

template <typename Tc, int P, int OY, int OZ>
struct Stream3Dims {
  static constexpr int RC = P / 2;
  static constexpr int LY = OY + 4 * RC, LZ = OZ + 4 * RC;  // state plane tile
  static constexpr int CY = OY + 2 * RC, CZ = OZ + 2 * RC;  // after the centre sweeps
  static constexpr int NU = 2 * RC + 2;                     // state ring (one plane ahead)
  static constexpr int NP = 2 * RC + 1;                     // primitive ring
  static constexpr int PL = LY * LZ, PC = CY * CZ;
  // bytes: state ring (FP64), x-swept plane A (5 LY LZ), y-swept plane B
  // (5 CY LZ), primitive ring (NP x 5 CY CZ), offsets and flip bits of the
  // plane tile's y-z points
  static constexpr int U_BYTES = NU * 5 * PL * 8;
  static constexpr int A_ELEMS = 5 * PL, B_ELEMS = 5 * CY * LZ, R_ELEMS = NP * 5 * PC;
  static constexpr int BYTES = U_BYTES + (A_ELEMS + B_ELEMS + R_ELEMS) * (int)sizeof(Tc) + PL * 4 + PL + 16;
};

__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gmem_src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(smem_dst)),
               "l"(gmem_src)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ int ring(int i, int n) {
  const int r = i % n;
  return r < 0 ? r + n : r;
}


// W over [-g, n+g)^3 for a block's y-z tile (blockIdx.x along z, blockIdx.y
// along y) and its chunk of output planes along x (blockIdx.z). REDUCE: the
// CFL maximum over rs.cfl_box and the per-variable extrema over rs.ext_box.
template <typename Tc, int P, int OY, int OZ, int KC, bool REDUCE>
__global__ void __launch_bounds__(256)
    k3s_primitives(const double* __restrict__ u, Grid grid, View<Tc> W, int g, int chunk, Rule<Tc, KC> c,
                   Rule<Tc, KC> t, Phys<Tc> ph, ReduceSpec rs, Scalars* __restrict__ sc) {
  using D = Stream3Dims<Tc, P, OY, OZ>;
  constexpr int RC = D::RC, LZ = D::LZ, CY = D::CY, CZ = D::CZ, PL = D::PL, PC = D::PC, NU = D::NU,
                NP = D::NP;
  extern __shared__ __align__(16) unsigned char smem[];
  double* const U = reinterpret_cast<double*>(smem);  // NU x 5 x PL
  Tc* const A = reinterpret_cast<Tc*>(smem + D::U_BYTES);
  Tc* const B = A + D::A_ELEMS;
  Tc* const R = B + D::B_ELEMS;
  int* const off = reinterpret_cast<int*>(R + D::R_ELEMS);              // y-z source offset of each plane point
  unsigned char* const fl = reinterpret_cast<unsigned char*>(off + PL);  // bit 0: y mirror flips, bit 1: z
  __shared__ int xflip[NU];
  const int n0 = grid.n[0], n1 = grid.n[1], n2 = grid.n[2];
  const int gmax = g + 2 * RC;
  const int plane = n0 * n1 * n2;
  const int y0 = -g + (int)blockIdx.y * OY, z0 = -g + (int)blockIdx.x * OZ;
  const int xb = -g + (int)blockIdx.z * chunk;
  const int xe = min(xb + chunk, n0 + g);
  // ghost maps of the tile's y-z points (the same for every plane); points
  // past the deepest ghost cell any output needs are clamped (they feed none)
  for (int e = threadIdx.x; e < PL; e += blockDim.x) {
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
  // asynchronous copies of state plane xi into its ring slot
  auto issue = [&](int xi) {
    const int xc = min(max(xi, -gmax), n0 + gmax - 1);
    bool fx = false;
    const int jx = ghost_source(xc, n0, grid.bc[0][0], grid.bc[0][1], fx);
    const int slot = ring(xi, NU);
    if (threadIdx.x == 0) xflip[slot] = fx ? 1 : 0;
    double* dst = U + slot * 5 * PL;
    const double* src = u + (size_t)jx * n1 * n2;
    for (int idx = threadIdx.x; idx < 5 * PL; idx += blockDim.x) {
      const int v = idx / PL, e = idx - v * PL;
      cp_async8(dst + idx, src + (size_t)v * plane + off[e]);
    }
  };
  for (int xi = xb - 2 * RC; xi <= xb; ++xi) issue(xi);
  unsigned long long cfl_key = 0ull, kmax[5], kmin[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    kmax[v] = 0ull;
    kmin[v] = ~0ull;
  }
  for (int i = xb - RC; i < xe + RC; ++i) {
    cp_async_wait();
    __syncthreads();  // state planes i-RC .. i+RC and their flip flags are in place
    if (i + RC + 1 <= xe - 1 + 2 * RC) issue(i + RC + 1);  // its slot held plane i-RC-1, no longer read
    // centre sweep along x (the state, sign-corrected in FP64, then converted)
    for (int idx = threadIdx.x; idx < 5 * PL; idx += blockDim.x) {
      const int v = idx / PL, e = idx - v * PL;
      const bool fyz = (v == 2 && (fl[e] & 1)) || (v == 3 && (fl[e] & 2));
      Tc acc = Tc(0);
#pragma unroll
      for (int k = 0; k < KC; ++k) {
        const int slot = ring(i - RC + k, NU);
        double d = U[slot * 5 * PL + idx];
        if (fyz || (v == 1 && xflip[slot])) d = -d;
        acc = acc + c.w[k] * (Tc)d;
      }
      A[idx] = acc;
    }
    __syncthreads();
    // centre sweep along y: B (5 x CY x LZ)
    for (int idx = threadIdx.x; idx < 5 * CY * LZ; idx += blockDim.x) {
      const int v = idx / (CY * LZ), rem = idx - v * (CY * LZ), y = rem / LZ, z = rem - y * LZ;
      const Tc* p = A + v * PL + y * LZ + z;
      Tc acc = Tc(0);
#pragma unroll
      for (int k = 0; k < KC; ++k) acc = acc + c.w[k] * p[k * LZ];
      B[idx] = acc;
    }
    __syncthreads();
    // centre sweep along z and the conversion: primitive plane i into its ring slot
    {
      Tc* Ri = R + ring(i, NP) * 5 * PC;
      for (int idx = threadIdx.x; idx < PC; idx += blockDim.x) {
        const int y = idx / CZ, z = idx - y * CZ;
        Tc uc[5], w[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          const Tc* p = B + v * (CY * LZ) + y * LZ + z;
          Tc acc = Tc(0);
#pragma unroll
          for (int k = 0; k < KC; ++k) acc = acc + c.w[k] * p[k];
          uc[v] = acc;
        }
        to_primitives(ph, 5, uc, w);
#pragma unroll
        for (int v = 0; v < 5; ++v) Ri[v * PC + idx] = w[v];
      }
    }
    __syncthreads();
    const int xo = i - RC;
    if (xo < xb) continue;
    // transverse sweep along x over the primitive ring: A (5 x CY x CZ)
    for (int idx = threadIdx.x; idx < 5 * PC; idx += blockDim.x) {
      Tc acc = Tc(0);
#pragma unroll
      for (int k = 0; k < KC; ++k) acc = acc + t.w[k] * R[ring(xo - RC + k, NP) * 5 * PC + idx];
      A[idx] = acc;
    }
    __syncthreads();
    // transverse sweep along y: B (5 x OY x CZ)
    for (int idx = threadIdx.x; idx < 5 * OY * CZ; idx += blockDim.x) {
      const int v = idx / (OY * CZ), rem = idx - v * (OY * CZ), y = rem / CZ, z = rem - y * CZ;
      const Tc* p = A + v * PC + y * CZ + z;
      Tc acc = Tc(0);
#pragma unroll
      for (int k = 0; k < KC; ++k) acc = acc + t.w[k] * p[k * CZ];
      B[idx] = acc;
    }
    __syncthreads();
    // transverse sweep along z: W at output plane xo, and the reductions
    for (int idx = threadIdx.x; idx < OY * OZ; idx += blockDim.x) {
      const int y = idx / OZ, z = idx - y * OZ;
      const int yi = y0 + y, zi = z0 + z;
      if (yi >= n1 + g || zi >= n2 + g) continue;
      Tc w[5];
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        const Tc* p = B + v * (OY * CZ) + y * CZ + z;
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
  cp_async_wait();
  if constexpr (REDUCE) f2::reduce_keys_and_publish(cfl_key, kmax, kmin, rs, sc);
}

}  // namespace s3
}  // namespace fvh
