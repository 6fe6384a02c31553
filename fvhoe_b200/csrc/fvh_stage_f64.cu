// FP64 stage runner. This translation unit is compiled with -fmad=false so
// that every product and sum rounds separately, in the reference's order.
// It also holds the precision-independent kernels (stage scalars, convex face
// weights, trouble-log arithmetic).
#include "fvh_stage.cuh"

namespace fvh {

__global__ void k_reset_scalars(Scalars* sc, int reset_step) {
  const int t = threadIdx.x;
  if (t == 0) {
    sc->cfl_key = 0ull;
    sc->troubled = 0u;
    sc->fb_faces = 0u;
    if (reset_step) {
      sc->nonfinite = 0u;
      sc->timeouts = 0u;
      sc->predicted = 0u;
      sc->judged = 0u;
      sc->missed = 0u;
      sc->false_alarm = 0u;
      sc->revised_faces = 0u;
      sc->flux_fallback_faces = 0u;
    }
  }
  for (int v = t; v < kMaxVars; v += blockDim.x) {
    sc->vmax_key[v] = 0ull;
    sc->vmin_key[v] = ~0ull;
  }
}

// dt = CFL h / max speed (fvhoe/hydro.py:292), or the fixed dt; the first
// stage of a step also applies the target clamp (fvhoe/ode.py:11-22).
__global__ void k_finalize_dt(Scalars* sc, double cfl_h, int use_fixed, double fixed_dt, int is_first_stage,
                              int has_target, double t, double target) {
  const double dt = use_fixed ? fixed_dt : cfl_h / key_value(sc->cfl_key);
  sc->dt_stage = dt;
  if (is_first_stage) {
    double d = dt;
    if (has_target && target - t < d) d = target - t;
    sc->dt_step = d;
  }
}

__global__ void k_convex_init(View<const uint8_t> trouble, Region rint, Box pad, float* __restrict__ th) {
  FVH_FOR_POINTS(pad, idx) {
    int i0, i1, i2;
    box_point(pad, idx, i0, i1, i2);
    const bool inside = i0 >= 0 && i0 < rint.n[0] && i1 >= 0 && i1 < rint.n[1] && i2 >= 0 && i2 < rint.n[2];
    th[idx] = inside ? (float)trouble.p[trouble.at(i0, i1, i2)] : 0.0f;
  }
}

// One statement "theta[target] = max(coef * src[target + shift], theta[target])"
// of the reference's convex broadcast; src_is_theta turns src into (src > 0).
__global__ void k_convex_step(View<const float> src, const float* __restrict__ prev, float* __restrict__ out, Box pad,
                              int s0, int s1, int s2, float coef, int src_is_theta) {
  FVH_FOR_POINTS(pad, idx) {
    int i0, i1, i2;
    box_point(pad, idx, i0, i1, i2);
    const int j0 = i0 + s0, j1 = i1 + s1, j2 = i2 + s2;
    float v = prev[idx];
    if (j0 >= pad.lo[0] && j0 < pad.lo[0] + pad.n[0] && j1 >= pad.lo[1] && j1 < pad.lo[1] + pad.n[1] &&
        j2 >= pad.lo[2] && j2 < pad.lo[2] + pad.n[2]) {
      float x = src.p[src.at(j0, j1, j2)];
      if (src_is_theta) x = x > 0.0f ? 1.0f : 0.0f;
      const float c = coef * x;
      v = c > v ? c : v;
    }
    out[idx] = v;
  }
}

// Face weight = max(theta of the two cells sharing the face).
__global__ void k_convex_faces(View<const float> th, float* __restrict__ theta, Box faces, int d) {
  const int sd = th.stride(d);
  FVH_FOR_POINTS(faces, idx) {
    int i0, i1, i2;
    box_point(faces, idx, i0, i1, i2);
    const int o = th.at(i0, i1, i2);
    const float x = th.p[o];
    const float y = th.p[o - sd];
    theta[idx] = x > y ? x : y;
  }
}

int convex_weights(fvh_handle* h, cudaStream_t s) {
  const Region rpad = padded_region(h, 2);
  const Region rint = interior_region(h);
  const Box pad = make_box(rpad);
  const unsigned nb = blocks_for(pad.count);
  // conv holds three padded arrays: the trouble flags and two theta buffers
  const int64_t np = region_points(rpad);
  float* t0 = h->conv;
  float* th_a = h->conv + np;
  float* th_b = h->conv + 2 * np;
  {
    LaunchScope scope(KK_SMALL, 0.0, s);
    k_convex_init<<<nb, 256, 0, s>>>(make_view((const uint8_t*)h->trouble, rint), rint, pad, t0);
  }
  cudaMemcpyAsync(th_a, t0, sizeof(float) * np, cudaMemcpyDeviceToDevice, s);
  int ax[3], na = 0;
  for (int a = 0; a < 3; ++a)
    if (h->active[a]) ax[na++] = a;
  struct Stmt {
    int s[2];
    float coef;
    int theta_src;
  };
  // statement lists of fvhoe/slope_limiting.py:394-405 (1D) and :418-440 (2D)
  static const Stmt one_d[4] = {{{+1, 0}, 0.75f, 0}, {{-1, 0}, 0.75f, 0}, {{+1, 0}, 0.25f, 1}, {{-1, 0}, 0.25f, 1}};
  static const Stmt two_d[12] = {
      {{0, +1}, 0.75f, 0}, {{0, -1}, 0.75f, 0}, {{+1, 0}, 0.75f, 0}, {{-1, 0}, 0.75f, 0},
      {{+1, +1}, 0.5f, 0}, {{+1, -1}, 0.5f, 0}, {{-1, +1}, 0.5f, 0}, {{-1, -1}, 0.5f, 0},
      {{0, +1}, 0.25f, 1}, {{0, -1}, 0.25f, 1}, {{+1, 0}, 0.25f, 1}, {{-1, 0}, 0.25f, 1},
  };
  const Stmt* list = na == 1 ? one_d : two_d;
  const int count = na == 1 ? 4 : 12;
  float* cur = th_a;
  float* nxt = th_b;
  for (int i = 0; i < count; ++i) {
    int sh[3] = {0, 0, 0};
    sh[ax[0]] = list[i].s[0];
    if (na == 2) sh[ax[1]] = list[i].s[1];
    const float* src = list[i].theta_src ? cur : t0;
    {
      LaunchScope scope(KK_SMALL, 0.0, s);
      k_convex_step<<<nb, 256, 0, s>>>(make_view(src, rpad), cur, nxt, pad, sh[0], sh[1], sh[2], list[i].coef,
                                       list[i].theta_src);
    }
    float* tmp = cur;
    cur = nxt;
    nxt = tmp;
  }
  for (int q = 0; q < na; ++q) {
    const int d = ax[q];
    const Box bf = make_box(face_region(h, d));
    LaunchScope scope(KK_SMALL, 0.0, s);
    k_convex_faces<<<blocks_for(bf.count), 256, 0, s>>>(make_view((const float*)cur, rpad), h->theta[d], bf, d);
  }
  return set_cuda_error(h, "convex weights");
}

int run_stage_f64(fvh_handle* h, const StageCall& c, cudaStream_t s) { return run_stage_any<double>(h, c, s); }

int primitives_f64(fvh_handle* h, const double* u, double* w, int fv_average, cudaStream_t s) {
  ReduceSpec none{};
  if (h->nv == 5) return primitive_pass<double, 5>(h, u, 0, w, none, false, fv_average != 0, s);
  return primitive_pass<double, 0>(h, u, 0, w, none, false, fv_average != 0, s);
}

}  // namespace fvh
