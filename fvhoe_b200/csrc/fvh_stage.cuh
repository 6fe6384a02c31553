// Host orchestration of one stage of the per-stage update, templated on the
// compute type. Included once by fvh_stage_f64.cu (built with -fmad=false,
// bit-exact with the reference) and once by fvh_stage_f32.cu.
//
// Pass sequence of one stage (fvhoe/solver.py:429-454):
//   1. W  = FV primitives of the stage input with gW ghosts, plus the CFL
//           maximum over the gw-ghost box and the per-variable extrema over
//           the 3-ghost box                  (solver.py:491-517, 686)
//   2. dt = CFL h / max, or fixed_dt; stage 0 also clamps to the target
//   3. per active axis d: centre sweeps along the other axes, face states +
//      Riemann solve along d, transverse sweeps          (solver.py:519-651)
//   4. a-posteriori limiting (solver.py:653-732): candidate u*, W* of u*,
//      detection, convex weights, MUSCL fallback + blend at troubled faces
//   5. flux divergence + Runge-Kutta stage combination   (solver.py:734-751)
#pragma once

#include <algorithm>
#include <cstdio>
#include <string>

#include "fvh_fused2d.cuh"
#include "fvh_stream3d.cuh"
#include "fvh_handle.h"
#include "fvh_profile.h"

namespace fvh {

// ---------------------------------------------------------------------------
// stencil rules (fvhoe/stencils.py:25-255), stored as exact rationals; the
// float64 weight is the correctly rounded quotient, as the reference's `a / b`
// literals evaluate. Centre and transverse rules of odd p equal the rule of
// p - 1 (their extra end taps are zero), so only even degrees are stored.
// ---------------------------------------------------------------------------
struct HostRule {
  int K = 1;
  int off = 0;
  double w[9] = {1, 0, 0, 0, 0, 0, 0, 0, 0};
};

inline HostRule make_rule(long long den, const long long* num, int K) {
  HostRule r;
  r.K = K;
  r.off = -(K - 1) / 2;
  for (int k = 0; k < K; ++k) r.w[k] = (double)num[k] / (double)den;
  return r;
}

inline HostRule left_face_rule(int p) {
  static const long long den[9] = {1, 4, 6, 24, 60, 120, 420, 1680, 2520};
  static const long long num[9][9] = {
      {1},
      {1, 4, -1},
      {2, 5, -1},
      {-1, 10, 20, -6, 1},
      {-3, 27, 47, -13, 2},
      {1, -10, 59, 94, -31, 8, -1},
      {4, -38, 214, 319, -101, 25, -3},
      {-3, 34, -194, 898, 1276, -446, 142, -30, 3},
      {-5, 55, -305, 1375, 1879, -641, 199, -41, 4},
  };
  const int K = 2 * ((p + 1) / 2) + 1;
  return make_rule(den[p], num[p], K);
}

inline HostRule right_face_rule(int p) {
  HostRule l = left_face_rule(p);
  HostRule r = l;
  for (int k = 0; k < l.K; ++k) r.w[k] = l.w[l.K - 1 - k];
  return r;
}

inline HostRule centre_rule(int p) {
  static const long long den[5] = {1, 24, 1920, 107520, 10321920};
  static const long long num[5][9] = {
      {1},
      {-1, 26, -1},
      {9, -116, 2134, -116, 9},
      {-75, 954, -7621, 121004, -7621, 954, -75},
      {1225, -17000, 125884, -800216, 11702134, -800216, 125884, -17000, 1225},
  };
  const int e = p / 2;
  return make_rule(den[e], num[e], 2 * e + 1);
}

inline HostRule transverse_rule(int p) {
  static const long long den[5] = {1, 24, 5760, 967680, 464486400};
  static const long long num[5][9] = {
      {1},
      {1, 22, 1},
      {-17, 308, 5178, 308, -17},
      {367, -5058, 57249, 862564, 57249, -5058, 367},
      {-27859, 399032, -3207892, 29039624, 412080590, 29039624, -3207892, 399032, -27859},
  };
  const int e = p / 2;
  return make_rule(den[e], num[e], 2 * e + 1);
}

template <typename Tc, int K>
inline Rule<Tc, K> device_rule(const HostRule& hr) {
  Rule<Tc, K> r;
  for (int k = 0; k < K; ++k) r.w[k] = (Tc)hr.w[k];
  r.off = hr.off;
  return r;
}

inline unsigned blocks_for(int64_t n, int threads = 256) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > (1 << 22)) b = 1 << 22;
  return (unsigned)b;
}

// bytes of nv variables of `elem` bytes over r, with r grown by `grow` cells along `axis`
inline double region_bytes(const Region& r, int nv, size_t elem, int axis = -1, int grow = 0) {
  double pts = 1.0;
  for (int a = 0; a < 3; ++a) pts *= (double)(r.n[a] + (a == axis ? grow : 0));
  return pts * nv * (double)elem;
}

inline Region interior_region(const fvh_handle* h) {
  Region r;
  for (int a = 0; a < 3; ++a) {
    r.lo[a] = 0;
    r.n[a] = h->n[a];
  }
  return r;
}

// Box [-g, n+g) on the active axes, interior extent elsewhere.
inline Region padded_region(const fvh_handle* h, int g) {
  Region r;
  for (int a = 0; a < 3; ++a) {
    const int ga = h->active[a] ? g : 0;
    r.lo[a] = -ga;
    r.n[a] = h->n[a] + 2 * ga;
  }
  return r;
}

inline Region face_region(const fvh_handle* h, int d) {
  Region r = interior_region(h);
  r.n[d] += 1;
  return r;
}

inline int set_cuda_error(fvh_handle* h, const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return FVH_OK;
  h->err = std::string(what) + ": " + cudaGetErrorString(e);
  return FVH_ERR_CUDA;
}

inline int fail_config(fvh_handle* h, const char* what) {
  h->err = what;
  return FVH_ERR_CONFIG;
}

template <typename Tc>
inline Phys<Tc> make_phys(const fvh_handle* h) {
  Phys<Tc> ph;
  ph.gamma = (Tc)h->cfg.gamma;
  ph.gm1 = (Tc)(h->cfg.gamma - 1.0);
  ph.csq_floor = (Tc)h->cfg.csq_floor;
  ph.nv = h->nv;
  ph.riemann = h->cfg.riemann;
  ph.pad_ = 0;
  return ph;
}

// ---------------------------------------------------------------------------
// launch helpers: dispatch the tap count K to a compile-time constant
// ---------------------------------------------------------------------------
template <typename Tc, int NV, int K>
void launch_centre_k(bool from_state, bool to_prims, const void* in, Region rin, Tc* out, Region rout, int axis,
                     const HostRule& hr, const Grid& g, const Phys<Tc>& ph, cudaStream_t s) {
  const Rule<Tc, K> rule = device_rule<Tc, K>(hr);
  const Box box = make_box(rout);
  const View<Tc> vo = make_view(out, rout);
  const unsigned nb = blocks_for(region_points(rout));
  LaunchScope scope(KK_CENTRE,
                    region_bytes(rout, ph.nv, from_state ? sizeof(double) : sizeof(Tc), axis, K - 1) +
                        region_bytes(rout, ph.nv, sizeof(Tc)),
                    s);
  if (from_state) {
    const View<const double> none = make_view((const double*)nullptr, rout);
    if (to_prims)
      k_centre_sweep<Tc, double, NV, K, true, true>
          <<<nb, 256, 0, s>>>(none, (const double*)in, vo, box, axis, rule, g, ph);
    else
      k_centre_sweep<Tc, double, NV, K, true, false>
          <<<nb, 256, 0, s>>>(none, (const double*)in, vo, box, axis, rule, g, ph);
  } else {
    const View<const Tc> vi = make_view((const Tc*)in, rin);
    if (to_prims)
      k_centre_sweep<Tc, Tc, NV, K, false, true><<<nb, 256, 0, s>>>(vi, nullptr, vo, box, axis, rule, g, ph);
    else
      k_centre_sweep<Tc, Tc, NV, K, false, false><<<nb, 256, 0, s>>>(vi, nullptr, vo, box, axis, rule, g, ph);
  }
}

template <typename Tc, int NV>
void launch_centre(bool from_state, bool to_prims, const void* in, Region rin, Tc* out, Region rout, int axis,
                   const HostRule& hr, const Grid& g, const Phys<Tc>& ph, cudaStream_t s) {
  switch (hr.K) {
    case 1: launch_centre_k<Tc, NV, 1>(from_state, to_prims, in, rin, out, rout, axis, hr, g, ph, s); break;
    case 3: launch_centre_k<Tc, NV, 3>(from_state, to_prims, in, rin, out, rout, axis, hr, g, ph, s); break;
    case 5: launch_centre_k<Tc, NV, 5>(from_state, to_prims, in, rin, out, rout, axis, hr, g, ph, s); break;
    case 7: launch_centre_k<Tc, NV, 7>(from_state, to_prims, in, rin, out, rout, axis, hr, g, ph, s); break;
    case 9: launch_centre_k<Tc, NV, 9>(from_state, to_prims, in, rin, out, rout, axis, hr, g, ph, s); break;
  }
}

template <typename Tc, int NV, int K>
void launch_transverse_k(bool reduce, const Tc* in, Region rin, Tc* out, Region rout, int axis, const HostRule& hr,
                         const Phys<Tc>& ph, const ReduceSpec& rs, Scalars* sc, cudaStream_t s) {
  const Rule<Tc, K> rule = device_rule<Tc, K>(hr);
  const Box box = make_box(rout);
  const View<const Tc> vi = make_view(in, rin);
  const View<Tc> vo = make_view(out, rout);
  // reducing sweeps use a bounded, grid-stride grid so each block folds many points
  const unsigned nb = reduce ? std::min(blocks_for(region_points(rout)), 148u * 8u) : blocks_for(region_points(rout));
  LaunchScope scope(KK_TRANSVERSE,
                    region_bytes(rout, ph.nv, sizeof(Tc), axis, K - 1) + region_bytes(rout, ph.nv, sizeof(Tc)), s);
  if (reduce)
    k_transverse_sweep<Tc, NV, K, true><<<nb, 256, 0, s>>>(vi, vo, box, axis, rule, ph, rs, sc);
  else
    k_transverse_sweep<Tc, NV, K, false><<<nb, 256, 0, s>>>(vi, vo, box, axis, rule, ph, rs, sc);
}

template <typename Tc, int NV>
void launch_transverse(bool reduce, const Tc* in, Region rin, Tc* out, Region rout, int axis, const HostRule& hr,
                       const Phys<Tc>& ph, const ReduceSpec& rs, Scalars* sc, cudaStream_t s) {
  switch (hr.K) {
    case 1: launch_transverse_k<Tc, NV, 1>(reduce, in, rin, out, rout, axis, hr, ph, rs, sc, s); break;
    case 3: launch_transverse_k<Tc, NV, 3>(reduce, in, rin, out, rout, axis, hr, ph, rs, sc, s); break;
    case 5: launch_transverse_k<Tc, NV, 5>(reduce, in, rin, out, rout, axis, hr, ph, rs, sc, s); break;
    case 7: launch_transverse_k<Tc, NV, 7>(reduce, in, rin, out, rout, axis, hr, ph, rs, sc, s); break;
    case 9: launch_transverse_k<Tc, NV, 9>(reduce, in, rin, out, rout, axis, hr, ph, rs, sc, s); break;
  }
}

template <typename Tc, int NV, int K>
void launch_face_k(const Tc* in, Region rin, Tc* out, Region rout, int d, const HostRule& l, const HostRule& r,
                   const Phys<Tc>& ph, cudaStream_t s) {
  LaunchScope scope(KK_FACE, region_bytes(rout, ph.nv, sizeof(Tc), d, K) + region_bytes(rout, ph.nv, sizeof(Tc)), s);
  k_face_riemann<Tc, NV, K><<<blocks_for(region_points(rout)), 256, 0, s>>>(
      make_view(in, rin), make_view(out, rout), make_box(rout), d, device_rule<Tc, K>(l), device_rule<Tc, K>(r), ph);
}

template <typename Tc, int NV>
void launch_face(const Tc* in, Region rin, Tc* out, Region rout, int d, const HostRule& l, const HostRule& r,
                 const Phys<Tc>& ph, cudaStream_t s) {
  switch (l.K) {
    case 1: launch_face_k<Tc, NV, 1>(in, rin, out, rout, d, l, r, ph, s); break;
    case 3: launch_face_k<Tc, NV, 3>(in, rin, out, rout, d, l, r, ph, s); break;
    case 5: launch_face_k<Tc, NV, 5>(in, rin, out, rout, d, l, r, ph, s); break;
    case 7: launch_face_k<Tc, NV, 7>(in, rin, out, rout, d, l, r, ph, s); break;
    case 9: launch_face_k<Tc, NV, 9>(in, rin, out, rout, d, l, r, ph, s); break;
  }
}

// ---------------------------------------------------------------------------
// FV primitives with g ghost cells (fvhoe/solver.py:753-792):
// ghost-fill u with g + 2r cells through the index maps, centre sweeps along
// x, y, z (the last converts to primitives), transverse sweeps along x, y, z
// (the last writes dst and performs the requested reductions).
// With fv_average = false only the centre sweeps run, with g + r ghosts.
// ---------------------------------------------------------------------------
template <typename Tc, int NV>
int primitive_pass(fvh_handle* h, const double* state, int g, Tc* dst, const ReduceSpec& rs, bool reduce,
                   bool fv_average, cudaStream_t s) {
  const Phys<Tc> ph = make_phys<Tc>(h);
  int axes[3], na = 0;
  for (int a = 0; a < 3; ++a)
    if (h->active[a]) axes[na++] = a;
  Region cur;
  const int grow = fv_average ? 2 : 1;
  for (int a = 0; a < 3; ++a) {
    const int ga = h->active[a] ? g + grow * h->r[a] : 0;
    cur.lo[a] = -ga;
    cur.n[a] = h->n[a] + 2 * ga;
  }
  Tc* bufs[2] = {(Tc*)h->bufA, (Tc*)h->bufB};
  int which = 0;
  const void* src = state;
  Region rsrc = cur;
  for (int q = 0; q < na; ++q) {
    const int a = axes[q];
    Region out = cur;
    const int ga = fv_average ? g + h->r[a] : g;
    out.lo[a] = -ga;
    out.n[a] = h->n[a] + 2 * ga;
    const bool last = (q == na - 1);
    Tc* o = (last && !fv_average) ? dst : bufs[which];
    if (o != dst && (size_t)h->nv * (size_t)region_points(out) > h->buf_elems)
      return fail_config(h, "primitive pass: a sweep box exceeds the scratch buffers");
    launch_centre<Tc, NV>(q == 0, last, src, rsrc, o, out, a, centre_rule(h->p[a]), h->grid, ph, s);
    src = o;
    rsrc = out;
    cur = out;
    which ^= 1;
  }
  if (fv_average) {
    for (int q = 0; q < na; ++q) {
      const int a = axes[q];
      Region out = cur;
      out.lo[a] = -g;
      out.n[a] = h->n[a] + 2 * g;
      const bool last = (q == na - 1);
      Tc* o = last ? dst : bufs[which];
      if (o != dst && (size_t)h->nv * (size_t)region_points(out) > h->buf_elems)
        return fail_config(h, "primitive pass: a sweep box exceeds the scratch buffers");
      launch_transverse<Tc, NV>(last && reduce, (const Tc*)src, rsrc, o, out, a, transverse_rule(h->p[a]), ph, rs,
                                h->sc, s);
      src = o;
      rsrc = out;
      cur = out;
      which ^= 1;
    }
  }
  return set_cuda_error(h, "primitive pass");
}

// ---------------------------------------------------------------------------
// Two consecutive sweeps in one launch (k_sweep_pair, fvh_stream3d.cuh) for
// the flux passes: FP32, three active axes, five variables, the same degree
// p <= 3 on every axis, unless the generic kernels are asked for; tiles of
// 4 x 8 x 32 outputs. On Sedov 256^3 it took the FP32 step from 18.2 to 17.7 ms;
// in FP64 (tiles of 2 x 8 x 32) it measured 30.64 against 30.52 ms.
// ---------------------------------------------------------------------------
template <typename Tc>
inline bool sweep_pair_eligible(const fvh_handle* h) {
  return sizeof(Tc) == 4 && h->cfg.kernel_path != FVH_PATH_GENERIC && h->ndim == 3 && h->nv == 5 &&
         h->p[0] == h->p[1] && h->p[1] == h->p[2] && h->p[0] <= 3;
}

template <typename Tc, int A1, int A2, int K>
void launch_pair_k(const Tc* in, const Region& rin, Tc* out, const Region& rout, const HostRule& h1,
                   const HostRule& h2, int kind, cudaStream_t s) {
  constexpr int T0 = sizeof(Tc) == 4 ? 4 : 2, T1 = 8, T2 = 32;
  using D = PairDims<A1, A2, K, K, T0, T1, T2>;
  constexpr int bytes = D::template bytes<Tc>();
  constexpr int fit = (228 * 1024) / (bytes + 1024);
  constexpr int minb = fit < 1 ? 1 : (fit > 4 ? 4 : fit);
  auto kern = k_sweep_pair<Tc, A1, A2, K, K, T0, T1, T2, minb>;
  cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  const dim3 grid((rout.n[2] + T2 - 1) / T2, (rout.n[1] + T1 - 1) / T1, (rout.n[0] + T0 - 1) / T0);
  LaunchScope scope(kind, 2.0 * region_bytes(rout, 5, sizeof(Tc)), s);
  kern<<<grid, 256, bytes, s>>>(make_view(in, rin), rin, make_view(out, rout), make_box(rout),
                                device_rule<Tc, K>(h1), device_rule<Tc, K>(h2));
}

template <typename Tc, int A1, int A2>
void launch_pair_axes(const Tc* in, const Region& rin, Tc* out, const Region& rout, const HostRule& h1,
                      const HostRule& h2, int kind, cudaStream_t s) {
  if (h1.K == 1)
    launch_pair_k<Tc, A1, A2, 1>(in, rin, out, rout, h1, h2, kind, s);
  else
    launch_pair_k<Tc, A1, A2, 3>(in, rin, out, rout, h1, h2, kind, s);
}

// out = sweep along a2 of (sweep along a1 of in); the (a1, a2) pairs the flux
// passes take
template <typename Tc>
void launch_pair(const Tc* in, const Region& rin, Tc* out, const Region& rout, int a1, int a2, const HostRule& h1,
                 const HostRule& h2, int kind, cudaStream_t s) {
  const int key = a1 * 3 + a2;
  switch (key) {
    case 2 * 3 + 1: launch_pair_axes<Tc, 2, 1>(in, rin, out, rout, h1, h2, kind, s); break;
    case 0 * 3 + 2: launch_pair_axes<Tc, 0, 2>(in, rin, out, rout, h1, h2, kind, s); break;
    case 1 * 3 + 0: launch_pair_axes<Tc, 1, 0>(in, rin, out, rout, h1, h2, kind, s); break;
    case 1 * 3 + 2: launch_pair_axes<Tc, 1, 2>(in, rin, out, rout, h1, h2, kind, s); break;
    case 0 * 3 + 1: launch_pair_axes<Tc, 0, 1>(in, rin, out, rout, h1, h2, kind, s); break;
    default: break;
  }
}

// ---------------------------------------------------------------------------
// High-order face fluxes along d from W (fvhoe/solver.py:519-651).
// ---------------------------------------------------------------------------
template <typename Tc, int NV>
int flux_pass(fvh_handle* h, const Tc* W, Region rW, int d, Tc* Fd, cudaStream_t s) {
  const Phys<Tc> ph = make_phys<Tc>(h);
  Tc* bufs[2] = {(Tc*)h->bufA, (Tc*)h->bufB};
  int which = 0;
  // restrict the source box to what the faces of the interior need
  Region cur = rW;
  cur.lo[d] = -(h->r[d] + 1);
  cur.n[d] = h->n[d] + 2 * (h->r[d] + 1);
  for (int t = 0; t < 3; ++t) {
    if (t == d || !h->active[t]) continue;
    cur.lo[t] = -2 * h->r[t];
    cur.n[t] = h->n[t] + 4 * h->r[t];
  }
  const Tc* src = W;
  Region rsrc = rW;
  // centre sweeps along (d+2)%3 then (d+1)%3 (fvhoe/solver.py:523-568)
  const int order[2] = {(d + 2) % 3, (d + 1) % 3};
  const bool pair = sweep_pair_eligible<Tc>(h) && NV == 5;
  if (pair) {
    Region out = cur;
    for (int q = 0; q < 2; ++q) {
      out.lo[order[q]] = -h->r[order[q]];
      out.n[order[q]] = h->n[order[q]] + 2 * h->r[order[q]];
    }
    Tc* o = bufs[which];
    launch_pair<Tc>(src, rsrc, o, out, order[0], order[1], centre_rule(h->p[order[0]]),
                    centre_rule(h->p[order[1]]), KK_CENTRE, s);
    src = o;
    rsrc = out;
    cur = out;
    which ^= 1;
  }
  for (int q = 0; q < 2 && !pair; ++q) {
    const int t = order[q];
    if (!h->active[t]) continue;
    Region out = cur;
    out.lo[t] = -h->r[t];
    out.n[t] = h->n[t] + 2 * h->r[t];
    Tc* o = bufs[which];
    launch_centre<Tc, NV>(false, false, src, rsrc, o, out, t, centre_rule(h->p[t]), h->grid, ph, s);
    src = o;
    rsrc = out;
    cur = out;
    which ^= 1;
  }
  // face states along d and the Riemann solve
  int others[2], no = 0;
  for (int t = 0; t < 3; ++t)
    if (t != d && h->active[t]) others[no++] = t;
  Region rf = cur;
  rf.lo[d] = 0;
  rf.n[d] = h->n[d] + 1;
  for (int t = 0; t < 3; ++t)
    if (t != d && !h->active[t]) {
      rf.lo[t] = 0;
      rf.n[t] = 1;
    }
  Tc* o = (no == 0) ? Fd : bufs[which];
  launch_face<Tc, NV>(src, rsrc, o, rf, d, left_face_rule(h->p[d]), right_face_rule(h->p[d]), ph, s);
  src = o;
  rsrc = rf;
  which ^= 1;
  // transverse sweeps along the other axes in ascending order (solver.py:629-648)
  Region c2 = rf;
  if (pair && no == 2) {
    Region out = c2;
    for (int q = 0; q < 2; ++q) {
      out.lo[others[q]] = 0;
      out.n[others[q]] = h->n[others[q]];
    }
    launch_pair<Tc>(src, rsrc, Fd, out, others[0], others[1], transverse_rule(h->p[others[0]]),
                    transverse_rule(h->p[others[1]]), KK_TRANSVERSE, s);
    return set_cuda_error(h, "flux pass");
  }
  for (int q = 0; q < no; ++q) {
    const int t = others[q];
    Region out = c2;
    out.lo[t] = 0;
    out.n[t] = h->n[t];
    Tc* dst = (q == no - 1) ? Fd : bufs[which];
    ReduceSpec none{};
    launch_transverse<Tc, NV>(false, src, rsrc, dst, out, t, transverse_rule(h->p[t]), ph, none, h->sc, s);
    src = dst;
    rsrc = out;
    c2 = out;
    which ^= 1;
  }
  return set_cuda_error(h, "flux pass");
}

// ---------------------------------------------------------------------------
// Convex face weights (fvhoe/slope_limiting.py:281-363, 387-442): applied as
// the reference's sequence of shifted maxima on a trouble array padded by 2
// zero cells on the active axes. (The reference's periodic wrap of this
// padding writes an empty slice unless all three axes are active, so the
// padding stays zero in 1D and 2D.)
// ---------------------------------------------------------------------------
int convex_weights(fvh_handle* h, cudaStream_t s);

// Three active axes take the sliding-window kernel (k_detect3, the same flags
// and logs) unless the generic kernels are asked for.
template <int NDIM, typename Tc>
void launch_detect(const fvh_handle* h, const View<const Tc>& w, const View<const Tc>& ws, const Box& box,
                   const DetectSpec& ds, const View<uint8_t>& tr, cudaStream_t s) {
  if (NDIM == 3 && h->cfg.kernel_path != FVH_PATH_GENERIC) {
    // cells per thread along x, measured fastest on Sedov 256^3 at 3 blocks per SM
    constexpr int CH = sizeof(Tc) == 4 ? 2 : 4;
    const dim3 grid((unsigned)(((size_t)box.n[1] * box.n[2] + 255) / 256), (unsigned)((box.n[0] + CH - 1) / CH));
    k_detect3<Tc, CH><<<grid, 256, 0, s>>>(w, ws, box, ds, h->sc, tr, h->logs[0], h->logs[1], h->logs[2]);
    return;
  }
  k_detect<Tc, NDIM><<<blocks_for(box.count), 256, 0, s>>>(w, ws, box, ds, h->sc, tr, h->logs[0], h->logs[1],
                                                           h->logs[2]);
}

// ---------------------------------------------------------------------------
// streaming 3D primitive pass (fvh_stream3d.cuh): three active axes, five
// variables, the same degree p <= 3 on every axis, no Dirichlet sides; the six
// sweeps of a primitive pass in one launch, bit for bit the same W. On Sedov
// 256^3 its two launches per stage take 7.4 ms per step against 9.2 ms of
// generic sweeps in FP32, and 13.0 against 14.4 in FP64.
// ---------------------------------------------------------------------------
inline bool stream3d_eligible(const fvh_handle* h) {
  return h->cfg.kernel_path != FVH_PATH_GENERIC && h->ndim == 3 && h->nv == 5 && !h->grid.slabs &&
         h->p[0] == h->p[1] && h->p[1] == h->p[2] && h->p[0] <= 3;
}

template <typename Tc>
struct Stream3Tiles;
template <>
struct Stream3Tiles<float> {
  static constexpr int OY = 8, OZ = 32, NT = 256;
};
template <>
struct Stream3Tiles<double> {
  static constexpr int OY = 8, OZ = 16, NT = 256;
};

template <typename Tc, int P, bool REDUCE>
int stream3d_p(fvh_handle* h, const double* state, int g, Tc* dst, const ReduceSpec& rs, cudaStream_t s) {
  using T = Stream3Tiles<Tc>;
  constexpr int KC = 2 * (P / 2) + 1;
  using D = s3::Stream3Dims<Tc, P, T::OY, T::OZ, T::NT>;
  auto kern = s3::k3s_primitives<Tc, P, T::OY, T::OZ, T::NT, KC, REDUCE>;
  cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, D::BYTES);
  const Region rW = padded_region(h, g);
  const int ty = (rW.n[1] + T::OY - 1) / T::OY, tz = (rW.n[2] + T::OZ - 1) / T::OZ;
  // enough x chunks for about four waves of blocks; each chunk re-reads 3 RC planes
  int blocks_per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, (const void*)kern, T::NT, D::BYTES);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->cfg.device);
  const int want = std::max(1, 4 * sms * std::max(blocks_per_sm, 1) / (ty * tz));
  const int chunk = std::max(16, (rW.n[0] + want - 1) / want);
  const dim3 grid(tz, ty, (rW.n[0] + chunk - 1) / chunk);
  const double pts = (double)region_points(rW);
  LaunchScope scope(KK_CENTRE, (double)h->n[0] * h->n[1] * h->n[2] * 5 * 8.0 + pts * 5 * sizeof(Tc), s);
  kern<<<grid, T::NT, D::BYTES, s>>>(state, h->grid, make_view(dst, rW), g, chunk, device_rule<Tc, KC>(centre_rule(P)),
                                   device_rule<Tc, KC>(transverse_rule(P)), make_phys<Tc>(h), rs, h->sc);
  return set_cuda_error(h, "streaming 3D primitives");
}

template <typename Tc, bool REDUCE>
int stream3d(fvh_handle* h, const double* state, int g, Tc* dst, const ReduceSpec& rs, cudaStream_t s) {
  switch (h->p[0]) {
    case 0: return stream3d_p<Tc, 0, REDUCE>(h, state, g, dst, rs, s);
    case 1: return stream3d_p<Tc, 1, REDUCE>(h, state, g, dst, rs, s);
    case 2: return stream3d_p<Tc, 2, REDUCE>(h, state, g, dst, rs, s);
    default: return stream3d_p<Tc, 3, REDUCE>(h, state, g, dst, rs, s);
  }
}

// ---------------------------------------------------------------------------
// one stage
// ---------------------------------------------------------------------------
template <typename Tc, int NV>
int run_stage_t(fvh_handle* h, const StageCall& c, cudaStream_t s) {
  const Phys<Tc> ph = make_phys<Tc>(h);
  const fvh_config& cfg = h->cfg;
  const bool apost = cfg.a_posteriori != 0;
  int st;
  {
    LaunchScope scope(KK_SMALL, 0.0, s);
    k_reset_scalars<<<1, 32, 0, s>>>(h->sc, c.first_stage);
  }
  // 1. FV primitives of the stage input
  ReduceSpec rs{};
  rs.cfl = cfg.use_fixed_dt ? 0 : 1;
  rs.cfl_box = padded_region(h, h->gw);
  rs.extrema = (apost && cfg.nad_global) ? 1 : 0;
  rs.ext_box = padded_region(h, 3);
  rs.ndim = (double)h->ndim;
  const Region rW = padded_region(h, h->gW);
  const bool stream3 = stream3d_eligible(h);
  if (stream3) {
    if ((st = stream3d<Tc, true>(h, c.stage_in, h->gW, (Tc*)h->W, rs, s))) return st;
  } else if ((st = primitive_pass<Tc, NV>(h, c.stage_in, h->gW, (Tc*)h->W, rs, true, true, s))) {
    return st;
  }
  // 2. dt
  {
    LaunchScope scope(KK_SMALL, 0.0, s);
    k_finalize_dt<<<1, 1, 0, s>>>(h->sc, h->cfl_h, cfg.use_fixed_dt, cfg.fixed_dt, c.first_stage, c.has_target,
                                  c.t, c.target);
  }
  // 3. high-order fluxes
  FluxSet<Tc> fs{};
  for (int d = 0; d < 3; ++d) {
    if (!h->active[d]) continue;
    if ((st = flux_pass<Tc, NV>(h, (const Tc*)h->W, rW, d, (Tc*)h->F[d], s))) return st;
    fs.f[d] = make_view((const Tc*)h->F[d], face_region(h, d));
    fs.has[d] = 1;
    fs.neg_inv_h[d] = h->neg_inv_h[d];
  }
  const Region rint = interior_region(h);
  const Box bint = make_box(rint);
  double flux_bytes = 0.0;
  for (int d = 0; d < 3; ++d)
    if (h->active[d]) flux_bytes += region_bytes(face_region(h, d), h->nv, sizeof(Tc));
  const double state_bytes = region_bytes(rint, h->nv, sizeof(double));
  // 4. a-posteriori limiting
  if (apost) {
    {
      LaunchScope scope(KK_CANDIDATE, 2 * state_bytes + flux_bytes, s);
      k_candidate<Tc, NV><<<blocks_for(bint.count), 256, 0, s>>>(c.stage_in, make_view(h->Us, rint), bint, fs, ph,
                                                                 h->sc);
    }
    if ((st = set_cuda_error(h, "candidate"))) return st;
    ReduceSpec none{};
    if (stream3) {
      if ((st = stream3d<Tc, false>(h, h->Us, 3, (Tc*)h->Ws, none, s))) return st;
    } else if ((st = primitive_pass<Tc, NV>(h, h->Us, 3, (Tc*)h->Ws, none, false, true, s))) {
      return st;
    }
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
    int na = 0;
    for (int a = 0; a < 3; ++a)
      if (h->active[a]) ds.axes[na++] = a;
    ds.log_mode = cfg.log_troubles ? c.log_mode : 0;
    ds.log_div = ds.log_mode ? c.log_div : 0.0;
    {
      const double log_bytes = ds.log_mode ? 3.0 * (ds.log_mode == 2 ? 2 : 1) * region_bytes(rint, 1, 8) : 0.0;
      LaunchScope scope(KK_DETECT,
                        region_bytes(padded_region(h, 1), 5, sizeof(Tc)) + region_bytes(padded_region(h, 3), 5,
                                                                                         sizeof(Tc)) +
                            region_bytes(rint, 1, 1) + log_bytes,
                        s);
      const View<const Tc> vw = make_view((const Tc*)h->W, rW);
      const View<const Tc> vws = make_view((const Tc*)h->Ws, padded_region(h, 3));
      const View<uint8_t> vtr = make_view(h->trouble, rint);
      if (h->ndim == 1)
        launch_detect<1>(h, vw, vws, bint, ds, vtr, s);
      else if (h->ndim == 2)
        launch_detect<2>(h, vw, vws, bint, ds, vtr, s);
      else
        launch_detect<3>(h, vw, vws, bint, ds, vtr, s);
    }
    if ((st = set_cuda_error(h, "detect"))) return st;
    if (cfg.convex) {
      if ((st = convex_weights(h, s))) return st;
    }
    // without convex weights (and unless the generic kernels are asked for),
    // one compacting kernel per direction solves the faces of troubled cells
    // from the stage input
    if (!cfg.convex && cfg.kernel_path != FVH_PATH_GENERIC) {
      for (int d = 0; d < 3; ++d) {
        if (!h->active[d]) continue;
        FallbackSpec fb{};
        fb.d = d;
        fb.nd = h->n[d];
        fb.muscl = h->p[d] > 0 ? 1 : 0;
        fb.limiter = cfg.slope_limiter;
        const Region rf = face_region(h, d);
        LaunchScope scope(KK_FALLBACK, region_bytes(rint, 1, 1), s);
        const Box bf = make_box(rf);
        k_fallback_direct<Tc, NV><<<blocks_for(bf.count, 1024), 256, 0, s>>>(
            c.stage_in, h->grid, make_view((Tc*)h->F[d], rf), bf, make_view((const uint8_t*)h->trouble, rint), fb,
            ph);
      }
      if ((st = set_cuda_error(h, "fallback"))) return st;
    } else {
      // primitives of the stage input with 2 ghosts, into W (no longer needed)
      const Region r1 = padded_region(h, 2);
      {
        LaunchScope scope(KK_FALLBACK, state_bytes + region_bytes(r1, h->nv, sizeof(Tc)), s);
        const Box b1 = make_box(r1);
        k_pointwise_primitives<Tc, NV><<<blocks_for(b1.count), 256, 0, s>>>(c.stage_in, h->grid,
                                                                            make_view((Tc*)h->W, r1), b1, ph);
      }
      for (int d = 0; d < 3; ++d) {
        if (!h->active[d]) continue;
        FallbackSpec fb{};
        fb.d = d;
        fb.nd = h->n[d];
        fb.muscl = h->p[d] > 0 ? 1 : 0;
        fb.limiter = cfg.slope_limiter;
        const Region rf = face_region(h, d);
        {
          LaunchScope scope(KK_FALLBACK,
                            region_bytes(rint, 1, 1) + region_bytes(r1, h->nv, sizeof(Tc)) +
                                2 * region_bytes(rf, h->nv, sizeof(Tc)),
                            s);
          const Box bf = make_box(rf);
          k_fallback<Tc, NV><<<blocks_for(bf.count), 256, 0, s>>>(
              make_view((const Tc*)h->W, r1), make_view((Tc*)h->F[d], rf), bf,
              make_view((const uint8_t*)h->trouble, rint), cfg.convex ? h->theta[d] : nullptr, fb, ph);
        }
        if ((st = set_cuda_error(h, "fallback"))) return st;
      }
    }
  }
  // 5. divergence + Runge-Kutta combination
  {
    // state arrays read and written by the Runge-Kutta combination of this stage
    int arrays = 1;
    switch (c.spec.integrator) {
      case INT_EULER: arrays = 2; break;
      case INT_SSPRK2: arrays = c.spec.stage == 0 ? 2 : 3; break;
      // FP32: the Shu-Osher stages read u (and the stage input) and write one array
      case INT_SSPRK3: arrays = sizeof(Tc) == 4 ? (c.spec.stage == 0 ? 2 : 3) : (c.spec.stage == 1 ? 4 : 3); break;
      case INT_RK4: arrays = c.spec.stage == 0 ? 3 : (c.spec.stage == 3 ? 3 : 4); break;
      default: arrays = 1; break;
    }
    LaunchScope scope(KK_FINAL, flux_bytes + arrays * state_bytes, s);
    k_final<Tc, NV><<<blocks_for(bint.count), 256, 0, s>>>(bint, make_view((double*)nullptr, rint), fs, ph, c.spec,
                                                           h->sc);
  }
  return set_cuda_error(h, "final");
}

// ---------------------------------------------------------------------------
// fused 2D stage (fvh_fused2d.cuh)
// ---------------------------------------------------------------------------
// Tile shapes (rows along X x columns along the contiguous Y) per precision.
template <typename Tc>
struct FusedTiles;
template <>
struct FusedTiles<float> {
  static constexpr int PX = 32, PY = 32;  // primitives of the stage input
  static constexpr int SX = 24, SY = 32;  // primitives of the candidate (W* over the 3-ghost box; 4 blocks/SM)
  static constexpr int FX = 16, FY = 32;  // fluxes
  static constexpr int DX = 16, DY = 32;  // detection
  static constexpr int EX = 16, EY = 32;  // fallback + final
};
template <>
struct FusedTiles<double> {
  static constexpr int PX = 16, PY = 32;
  static constexpr int SX = 16, SY = 32;
  static constexpr int FX = 8, FY = 32;
  static constexpr int DX = 8, DY = 32;
  static constexpr int EX = 8, EY = 32;
};

// Eligible: two active axes, five variables, the same degree 1..8 on both,
// simple face broadcast.
inline bool fused2d_eligible(const fvh_handle* h) {
  if (h->ndim != 2 || h->nv != 5 || h->cfg.convex) return false;
  int ax[2], na = 0;
  for (int a = 0; a < 3; ++a)
    if (h->active[a]) ax[na++] = a;
  return h->p[ax[0]] == h->p[ax[1]] && h->p[ax[0]] >= 1 && h->p[ax[0]] <= 8;
}

inline void set_smem(const void* kernel, size_t bytes) {
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <typename Tc, int P>
int run_stage_fused2d(fvh_handle* h, const StageCall& c, cudaStream_t s) {
  using T = FusedTiles<Tc>;
  constexpr int R = (P + 1) / 2, RC = P / 2;
  constexpr int KC = 2 * RC + 1, KF = 2 * R + 1;
  const Phys<Tc> ph = make_phys<Tc>(h);
  const fvh_config& cfg = h->cfg;
  const bool apost = cfg.a_posteriori != 0;
  int ax[2], na = 0;
  for (int a = 0; a < 3; ++a)
    if (h->active[a]) ax[na++] = a;
  f2::Geo g;
  g.nx = h->n[ax[0]];
  g.ny = h->n[ax[1]];
  g.bcx[0] = cfg.bc[ax[0]][0];
  g.bcx[1] = cfg.bc[ax[0]][1];
  g.bcy[0] = cfg.bc[ax[1]][0];
  g.bcy[1] = cfg.bc[ax[1]][1];
  g.dx = ax[0];
  g.dy = ax[1];
  g.gmax = h->gW + 2 * h->r[ax[0]];
  g.slabs = h->grid.slabs;
  const Rule<Tc, KC> crule = device_rule<Tc, KC>(centre_rule(P));
  const Rule<Tc, KC> trule = device_rule<Tc, KC>(transverse_rule(P));
  const Rule<Tc, KF> lrule = device_rule<Tc, KF>(left_face_rule(P));
  const Rule<Tc, KF> rrule = device_rule<Tc, KF>(right_face_rule(P));
  const double cx = h->neg_inv_h[ax[0]], cy = h->neg_inv_h[ax[1]];
  const double cells = (double)g.nx * g.ny;
  int st;
  {
    LaunchScope scope(KK_SMALL, 0.0, s);
    k_reset_scalars<<<1, 32, 0, s>>>(h->sc, c.first_stage);
  }
  // 1. W with gW ghosts + reductions
  {
    using D = f2::PrimsDims<Tc, P, T::PX, T::PY>;
    const size_t smem = (size_t)(D::A + D::B) * sizeof(Tc);
    auto kern = f2::k2_primitives<Tc, P, T::PX, T::PY, KC, true>;
    set_smem((const void*)kern, smem);
    ReduceSpec rs{};
    rs.cfl = cfg.use_fixed_dt ? 0 : 1;
    rs.cfl_box = Region{{-h->gw, -h->gw, 0}, {g.nx + 2 * h->gw, g.ny + 2 * h->gw, 1}};
    rs.extrema = (apost && cfg.nad_global) ? 1 : 0;
    rs.ext_box = Region{{-3, -3, 0}, {g.nx + 6, g.ny + 6, 1}};
    rs.ndim = 2.0;
    const int gw = h->gW;
    const dim3 grid((g.ny + 2 * gw + T::PY - 1) / T::PY, (g.nx + 2 * gw + T::PX - 1) / T::PX);
    LaunchScope scope(KK_CENTRE, cells * 5 * (8.0 + sizeof(Tc)), s);
    kern<<<grid, 256, smem, s>>>(c.stage_in, g, f2::make_v2_aligned((Tc*)h->W, g.nx, g.ny, gw), gw, crule, trule, ph,
                                 rs, h->sc);
  }
  if ((st = set_cuda_error(h, "fused primitives"))) return st;
  // the stage's dt is derived (and published) by the flux kernel
  f2::DtSpec dts{};
  dts.cfl_h = h->cfl_h;
  dts.fixed_dt = cfg.fixed_dt;
  dts.t = c.t;
  dts.target = c.target;
  dts.use_fixed = cfg.use_fixed_dt;
  dts.first_stage = c.first_stage;
  dts.has_target = c.has_target;
  // learned predictor: flags from W and the extrema just reduced, refreshed
  // every pred_interval stages and reused in between
  const uint8_t* pred = nullptr;
  if (h->mlp && apost) {
    if (h->pred_stage % h->pred_interval == 0 && (st = mlp_predict_stage(h, s))) return st;
    ++h->pred_stage;
    pred = h->pred;
  }
  const f2::V2<Tc> F = f2::make_v2((Tc*)h->F[ax[0]], g.nx + 1, g.ny, 0);
  const f2::V2<Tc> G = f2::make_v2((Tc*)h->F[ax[1]], g.nx, g.ny + 1, 0);
  // 2. fluxes (+ candidate)
  {
    using D = f2::FluxDims<P, T::FX, T::FY>;
    // 128 spare bytes: the kernel starts its tiles at the first 128-byte boundary (TMA destination)
    const size_t smem = (size_t)D::TOTAL * sizeof(Tc) + (pred ? D::LIST : 0) + 128;
    auto kern = f2::k2_fluxes<Tc, P, T::FX, T::FY, KC, KF>;
    set_smem((const void*)kern, smem);
    const dim3 grid((g.ny + T::FY - 1) / T::FY, (g.nx + T::FX - 1) / T::FX);
    // W in, F and G out; with limiting, the state in and the candidate (compute type) out
    const f2::V2<const Tc> Wc = f2::make_v2_aligned((const Tc*)h->W, g.nx, g.ny, h->gW);
    // the W tile of every block arrives by one TMA box copy
    CUtensorMap wmap;
    const char* why = nullptr;
    if (!encode_tensor_map_3d(&wmap, Wc.p, (int)sizeof(Tc), Wc.sx, g.nx + 2 * Wc.g, 5, Wc.sx, Wc.vs, D::WYS, D::WX, 5,
                              &why))
      return fail_config(h, why);
    LaunchScope scope(KK_FACE, cells * 5 * (3.0 * sizeof(Tc) + (apost ? 8.0 + sizeof(Tc) : 0.0)), s);
    kern<<<grid, 256, smem, s>>>(Wc, c.stage_in, g, F, G, apost ? (Tc*)h->Us : nullptr, crule, trule, lrule, rrule, ph,
                                 cx, cy, h->sc, dts, pred, 1, cfg.slope_limiter, wmap);
  }
  if ((st = set_cuda_error(h, "fused fluxes"))) return st;
  // 3. W* + detection
  if (apost) {
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
    ds.log_mode = cfg.log_troubles ? c.log_mode : 0;
    ds.log_div = ds.log_mode ? c.log_div : 0.0;
    // W* of the candidate over its 3-ghost box, once per cell: the primitive
    // kernel on u* (no reductions)
    const f2::V2<Tc> Wst = f2::make_v2_aligned((Tc*)h->Ws, g.nx, g.ny, 3);
    {
      using DP = f2::PrimsDims<Tc, P, T::SX, T::SY>;
      const size_t smemp = (size_t)(DP::A + DP::B) * sizeof(Tc);
      auto kp = f2::k2_primitives<Tc, P, T::SX, T::SY, KC, false, Tc>;
      set_smem((const void*)kp, smemp);
      const dim3 gp((g.ny + 6 + T::SY - 1) / T::SY, (g.nx + 6 + T::SX - 1) / T::SX);
      LaunchScope scope(KK_CENTRE, cells * 5 * 2.0 * sizeof(Tc), s);
      kp<<<gp, 256, smemp, s>>>((const Tc*)h->Us, g, Wst, 3, crule, trule, ph, ReduceSpec{}, h->sc);
      if ((st = set_cuda_error(h, "fused candidate primitives"))) return st;
    }
    using D = f2::DetectStagedDims<Tc, P, T::DX, T::DY>;
    const size_t smem = (size_t)D::TOTAL * sizeof(Tc) + 128;  // + the alignment slack of the TMA destination
    auto kern = f2::k2_detect_staged<Tc, P, T::DX, T::DY>;
    set_smem((const void*)kern, smem);
    const dim3 grid((g.ny + T::DY - 1) / T::DY, (g.nx + T::DX - 1) / T::DX);
    const f2::V2<const Tc> Wc = f2::make_v2_aligned((const Tc*)h->W, g.nx, g.ny, h->gW);
    // both tiles of every block arrive by TMA box copies (column offsets fixed by P)
    if (Wc.gy != D::GWY || Wst.gy != 4 || Wst.g != 3) return fail_config(h, "detection tile layout mismatch");
    CUtensorMap wsmap, wmap;
    const char* why = nullptr;
    if (!encode_tensor_map_3d(&wsmap, Wst.p, (int)sizeof(Tc), Wst.sx, g.nx + 6, 5, Wst.sx, Wst.vs, D::OYS, D::OX, 5,
                              &why) ||
        !encode_tensor_map_3d(&wmap, Wc.p, (int)sizeof(Tc), Wc.sx, g.nx + 2 * Wc.g, 5, Wc.sx, Wc.vs, D::WYS, D::WX, 5,
                              &why))
      return fail_config(h, why);
    // W* and W in (compute type), flags out, trouble-log sums in and out
    LaunchScope scope(KK_DETECT, cells * (10.0 * sizeof(Tc) + 1 + (ds.log_mode ? 48.0 : 0.0)), s);
    kern<<<grid, 256, smem, s>>>(Wst.c(), g, Wc, ds, h->sc, h->trouble, h->logs[0], h->logs[1], h->logs[2], wsmap,
                                 wmap);
    if ((st = set_cuda_error(h, "fused detect"))) return st;
  }
  if (pred && (st = mlp_count_stage(h, s))) return st;
  // 4. FP64: fallback fluxes of the troubled faces, written over F and G by
  // their own launches: the list of those faces (in the sweep scratch, unused
  // by this path) and its solves. FP32 solves them inside the final pass,
  // from a pointwise tile per troubled tile (measured faster there; the FP64
  // final pass holds 3 blocks per SM with the fallback and waits on it).
  constexpr bool split = sizeof(Tc) == 8;
  if (apost && split) {
    const int64_t faces = (int64_t)(g.nx + 1) * g.ny + (int64_t)g.nx * (g.ny + 1);
    if ((size_t)faces * sizeof(int) > h->buf_elems * sizeof(double)) return fail_config(h, "face list exceeds scratch");
    {
      LaunchScope scope(KK_FALLBACK, cells * 1.0, s);  // the flags
      // 32 x 32 tiles of the (nx+1) x ny X faces and the nx x (ny+1) Y faces
      const dim3 tiles((unsigned)(g.ny + 1 + 31) / 32, (unsigned)(g.nx + 1 + 31) / 32);
      f2::k2_face_list<Tc><<<tiles, 256, 0, s>>>(g, h->trouble, pred, (int*)h->bufA, h->sc);
      if ((st = set_cuda_error(h, "fused fallback list"))) return st;
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->cfg.device);
    // the listed faces' states and fluxes: a fraction of the grid, counted as none
    LaunchScope scope(KK_FALLBACK, 0.0, s);
    f2::k2_face_solve<Tc><<<(unsigned)(sms * 8), 256, 0, s>>>(c.stage_in, g, F, G, (const int*)h->bufA, 1,
                                                                 cfg.slope_limiter, ph, h->sc);
    if ((st = set_cuda_error(h, "fused fallback solve"))) return st;
  }
  // 5. (FP32: fallback +) divergence + Runge-Kutta
  {
    using D = f2::FinalDims<T::EX, T::EY>;
    // FP64 launches of a stepper stage also stage the Runge-Kutta operands
    const size_t smem = D::template bytes<Tc>(sizeof(Tc) == 8 && split && c.spec.integrator != INT_RHS, !split);
    auto kern = f2::final_kernel<Tc, T::EX, T::EY, !split>(c.spec.integrator, c.spec.stage);
    set_smem((const void*)kern, smem);
    const dim3 grid((g.ny + T::EY - 1) / T::EY, (g.nx + T::EX - 1) / T::EX);
    int arrays = 1;
    switch (c.spec.integrator) {
      case INT_EULER: arrays = 2; break;
      case INT_SSPRK2: arrays = c.spec.stage == 0 ? 2 : 3; break;
      // FP32: the Shu-Osher stages read u (and the stage input) and write one array
      case INT_SSPRK3: arrays = sizeof(Tc) == 4 ? (c.spec.stage == 0 ? 2 : 3) : (c.spec.stage == 1 ? 4 : 3); break;
      case INT_RK4: arrays = c.spec.stage == 0 ? 3 : (c.spec.stage == 3 ? 3 : 4); break;
      default: arrays = 1; break;
    }
    LaunchScope scope(KK_FINAL, cells * (5 * 2.0 * sizeof(Tc) + arrays * 40.0 + (apost && !split ? 41.0 : 0.0)), s);
    kern<<<grid, 256, smem, s>>>(c.stage_in, g, F.c(), G.c(), h->trouble, pred, apost ? 1 : 0, 1, cfg.slope_limiter, ph,
                                 cx, cy, c.spec, h->sc);
  }
  return set_cuda_error(h, "fused final");
}

template <typename Tc>
int run_stage_any(fvh_handle* h, const StageCall& c, cudaStream_t s) {
  h->last_stage_fused = h->cfg.kernel_path != FVH_PATH_GENERIC && fused2d_eligible(h);
  if (h->last_stage_fused) {
    int p = 0;
    for (int a = 0; a < 3; ++a)
      if (h->active[a]) p = h->p[a];
    switch (p) {
      case 1: return run_stage_fused2d<Tc, 1>(h, c, s);
      case 2: return run_stage_fused2d<Tc, 2>(h, c, s);
      case 3: return run_stage_fused2d<Tc, 3>(h, c, s);
      case 4: return run_stage_fused2d<Tc, 4>(h, c, s);
      case 5: return run_stage_fused2d<Tc, 5>(h, c, s);
      case 6: return run_stage_fused2d<Tc, 6>(h, c, s);
      case 7: return run_stage_fused2d<Tc, 7>(h, c, s);
      case 8: return run_stage_fused2d<Tc, 8>(h, c, s);
    }
  }
  if (h->nv == 5) return run_stage_t<Tc, 5>(h, c, s);
  return run_stage_t<Tc, 0>(h, c, s);
}

}  // namespace fvh
