// Per-point physics of the Euler update: primitive/conservative conversion,
// sound speed, physical fluxes, the Riemann solvers, MUSCL slopes and the
// smooth-extrema detector.
//
// Every expression keeps the association order of the reference NumPy code
// (jpalafou/FVHOE, files cited per function). In the FP64 "exact" build these
// functions are compiled with -fmad=false, so each product and sum rounds on
// its own exactly as NumPy does, and results match the reference bit for bit.
// The FP32 build compiles the same code with contraction enabled.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace fvh {

constexpr int kMaxVars = 16;  // 5 hydro variables + up to 11 passive scalars

enum Riemann : int { RIEMANN_HLLC = 0, RIEMANN_LLF = 1, RIEMANN_UPWIND = 2 };
enum Limiter : int { LIMITER_MINMOD = 0, LIMITER_MONCEN = 1, LIMITER_NONE = 2 };

// Physics constants shared by the per-point routines.
template <typename T>
struct Phys {
  T gamma;      // specific heat ratio
  T gm1;        // gamma - 1, rounded once on the host like Python's (gamma - 1)
  T csq_floor;  // floor on c^2
  int nv;       // number of variables (>= 5)
  int riemann;  // Riemann enum
  int pad_;
};

// NumPy's maximum/minimum propagate NaN; comparisons below keep that.
template <typename T>
__device__ __forceinline__ T np_maximum(T a, T b) {
  return (a != a) ? a : ((b != b) ? b : (a >= b ? a : b));
}
template <typename T>
__device__ __forceinline__ T np_minimum(T a, T b) {
  return (a != a) ? a : ((b != b) ? b : (a <= b ? a : b));
}

// conservatives -> primitives, fvhoe/hydro.py:146-170.
// v = m / rho ; P = (gamma - 1) * (E - 0.5 * ((mx vx + my vy) + mz vz))
template <typename T>
__device__ __forceinline__ void to_primitives(const Phys<T>& ph, int nv, const T* u, T* w) {
  const T rho = u[0];
  w[0] = rho;
  w[1] = u[1] / rho;
  w[2] = u[2] / rho;
  w[3] = u[3] / rho;
  T ke = u[1] * w[1];
  ke = ke + u[2] * w[2];
  ke = ke + u[3] * w[3];
  w[4] = ph.gm1 * (u[4] - T(0.5) * ke);
  for (int v = 5; v < nv; ++v) w[v] = u[v] / rho;
}

// primitives -> conservatives, fvhoe/hydro.py:173-196.
template <typename T>
__device__ __forceinline__ void to_conservatives(const Phys<T>& ph, int nv, const T* w, T* u) {
  const T rho = w[0];
  u[0] = rho;
  u[1] = rho * w[1];
  u[2] = rho * w[2];
  u[3] = rho * w[3];
  T ke = u[1] * w[1];
  ke = ke + u[2] * w[2];
  ke = ke + u[3] * w[3];
  u[4] = w[4] / ph.gm1 + T(0.5) * ke;
  for (int v = 5; v < nv; ++v) u[v] = rho * w[v];
}

// sqrt(gamma P / rho) with c^2 floored, fvhoe/hydro.py:199-210.
template <typename T>
__device__ __forceinline__ T sound_speed(const Phys<T>& ph, T rho, T P) {
  const T csq = ph.gamma * P / rho;
  return sqrt(csq > ph.csq_floor ? csq : ph.csq_floor);
}

// CFL signal speed sum_d |v_d| + ndim c, fvhoe/hydro.py:290-292.
template <typename T>
__device__ __forceinline__ T cfl_speed(const Phys<T>& ph, const T* w, T ndim) {
  const T c = sound_speed(ph, w[0], w[4]);
  T s = fabs(w[1]) + fabs(w[2]);
  s = s + fabs(w[3]);
  return s + ndim * c;
}

// Component 1 + d of a per-point array, selected without a run-time index so
// the array stays in registers.
template <typename T>
__device__ __forceinline__ T normal_component(const T* w, int d) {
  return d == 0 ? w[1] : (d == 1 ? w[2] : w[3]);
}

// Physical Euler flux along axis d (0..2), fvhoe/hydro.py:213-246.
template <typename T>
__device__ __forceinline__ void physical_flux(int nv, const T* w, const T* u, int d, bool with_pressure, T* f) {
  const T v = normal_component(w, d);
  f[0] = v * w[0];
#pragma unroll
  for (int k = 1; k < 4; ++k) {
    f[k] = v * u[k];
    if (with_pressure && k - 1 == d) f[k] = f[k] + w[4];
  }
  f[4] = v * u[4];
  if (with_pressure) f[4] = f[4] + v * w[4];
  for (int k = 5; k < nv; ++k) f[k] = v * u[k];
}

// Interface flux between left state wl and right state wr (primitives) along d.
//   HLLC ("David variation"): fvhoe/riemann_solvers.py:91-197
//   LLF:                      fvhoe/riemann_solvers.py:48-88
//   advection upwinding:      fvhoe/riemann_solvers.py:13-45
// NVA is the register-array length (the variable count, or kMaxVars when the
// count is only known at run time); nv is the count itself.
template <int NVA, typename T>
__device__ __forceinline__ void riemann_flux(const Phys<T>& ph, int nv, const T* wl, const T* wr, int d, T* out) {
  T ul[NVA], ur[NVA];
  to_conservatives(ph, nv, wl, ul);
  to_conservatives(ph, nv, wr, ur);
  if (ph.riemann == RIEMANN_UPWIND) {
    T fl[NVA], fr[NVA];
    physical_flux(nv, wl, ul, d, false, fl);
    physical_flux(nv, wr, ur, d, false, fr);
    const T v = normal_component(wl, d);
    for (int k = 0; k < nv; ++k) out[k] = v > T(0) ? fl[k] : (v < T(0) ? fr[k] : T(0));
    return;
  }
  if (ph.riemann == RIEMANN_LLF) {
    T fl[NVA], fr[NVA];
    physical_flux(nv, wl, ul, d, true, fl);
    physical_flux(nv, wr, ur, d, true, fr);
    const T sl = fabs(normal_component(wl, d)) + sound_speed(ph, wl[0], wl[4]);
    const T sr = fabs(normal_component(wr, d)) + sound_speed(ph, wr[0], wr[4]);
    const T half_smax = T(0.5) * np_maximum(sl, sr);
    for (int k = 0; k < nv; ++k) out[k] = T(0.5) * (fl[k] + fr[k]) - half_smax * (ur[k] - ul[k]);
    return;
  }
  const T cl = sound_speed(ph, wl[0], wl[4]);
  const T cr = sound_speed(ph, wr[0], wr[4]);
  const T cmax = np_maximum(cl, cr);
  const T vl = normal_component(wl, d), vr = normal_component(wr, d);
  const T rl = wl[0], rr = wr[0];
  const T pl = wl[4], pr = wr[4];
  const T el = ul[4], er = ur[4];
  const T s_l = np_minimum(vl, vr) - cmax;
  const T s_r = np_maximum(vl, vr) + cmax;
  const T rcl = rl * (vl - s_l);
  const T rcr = rr * (s_r - vr);
  const T den = rcl + rcr;
  const T v_star = (((rcl * vl + rcr * vr) + pl) - pr) / den;
  const T p_star = ((rcl * pr + rcr * pl) + (rcl * rcr) * (vl - vr)) / den;
  T r_g, v_g, p_g, e_g;
  if (s_l > T(0)) {
    r_g = rl; v_g = vl; p_g = pl; e_g = el;
  } else if (v_star > T(0)) {
    const T dl = s_l - v_star;
    r_g = rl * (s_l - vl) / dl;
    e_g = (((s_l - vl) * el - pl * vl) + p_star * v_star) / dl;
    v_g = v_star; p_g = p_star;
  } else if (s_r > T(0)) {
    const T dr = s_r - v_star;
    r_g = rr * (s_r - vr) / dr;
    e_g = (((s_r - vr) * er - pr * vr) + p_star * v_star) / dr;
    v_g = v_star; p_g = p_star;
  } else {
    r_g = rr; v_g = vr; p_g = pr; e_g = er;
  }
  const T mass = r_g * v_g;
  out[0] = mass;
#pragma unroll
  for (int t = 0; t < 3; ++t) {
    if (t == d) {
      out[1 + t] = mass * v_g + p_g;
    } else {
      const T up = v_g > T(0) ? wl[1 + t] : (v_g < T(0) ? wr[1 + t] : T(0));
      out[1 + t] = mass * up;
    }
  }
  out[4] = v_g * (e_g + p_g);
  for (int k = 5; k < nv; ++k) {
    const T up = v_g > T(0) ? wl[k] : (v_g < T(0) ? wr[k] : T(0));
    out[k] = mass * up;
  }
}

// Limited slope from left/right differences, fvhoe/slope_limiting.py:40-84.
template <typename T>
__device__ __forceinline__ T limited_slope(T dl, T dr, int limiter) {
  if (limiter == LIMITER_MINMOD) {
    const T den = dl > T(0) ? (dl > T(1e-16) ? dl : T(1e-16)) : (dl < T(-1e-16) ? dl : T(-1e-16));
    T ratio = dr / den;
    ratio = ratio < T(1) ? ratio : T(1);
    return (ratio > T(0) ? ratio : T(0)) * dl;
  }
  if (limiter == LIMITER_MONCEN) {
    const T dc = T(0.5) * (dl + dr);
    T s = np_minimum(fabs(T(2) * dl), fabs(T(2) * dr));
    const T sgn = dc > T(0) ? T(1) : (dc < T(0) ? T(-1) : (dc == T(0) ? T(0) : dc));
    s = sgn * np_minimum(s, fabs(dc));
    return dl * dr >= T(0) ? s : T(0);
  }
  return T(0.5) * (dl + dr);
}

// Smooth-extrema detector along one line, fvhoe/smooth_extrema_detection.py:8-50.
// a[0..6] are the values at offsets -3..+3 around the cell; returns the
// first-neighbour minimum of alpha at the centre.
template <typename T>
__device__ __forceinline__ T sed_alpha_line(const T* a, T eps) {
  T du[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) du[k] = T(0.5) * (a[k + 2] - a[k]);
  T alpha[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const T d2u = T(0.5) * (du[k + 2] - du[k]);
    T dv = T(0.5) * d2u;
    if (fabs(dv) <= eps) dv = dv >= T(0) ? eps : -eps;
    const T vl = du[k] - du[k + 1];
    const T xl = dv < T(0) ? (vl > T(0) ? vl : T(0)) : (vl < T(0) ? vl : T(0));
    T al = -xl / dv;
    al = al < T(1) ? al : T(1);
    const T vr = du[k + 2] - du[k + 1];
    const T xr = dv > T(0) ? (vr > T(0) ? vr : T(0)) : (vr < T(0) ? vr : T(0));
    T ar = xr / dv;
    if (fabs(dv) <= eps) ar = T(1);
    ar = ar < al ? ar : al;
    alpha[k] = np_minimum(al, ar);
  }
  return np_minimum(np_minimum(alpha[2], alpha[1]), alpha[0]);
}

}  // namespace fvh
