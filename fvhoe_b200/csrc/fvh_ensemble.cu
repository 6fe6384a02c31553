// C ABI of the batched ensemble (include/fvh.h): set-up, stepping through a
// captured CUDA graph, status, and the autotuner that chooses the tile shape
// and the resident blocks per SM of the persistent stage kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "fvh_ensemble_host.h"
#include "fvh_handle.h"

namespace fvh {
int configure_handle(fvh_handle* h, const fvh_config* cfg, std::string& msg);
int check_device_visible(const fvh_config* cfg, std::string& msg);
}

using namespace fvh;

namespace {

thread_local std::string g_ens_error;

int fail(fvh_ensemble* e, int code, const std::string& msg) {
  if (e)
    e->err = msg;
  else
    g_ens_error = msg;
  return code;
}

int cuda_fail(fvh_ensemble* e, const char* what, cudaError_t err) {
  cudaGetLastError();
  return fail(e, FVH_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(err));
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

int ceil_div(int a, int b) { return (a + b - 1) / b; }

void release(fvh_ensemble* e) {
  cudaSetDevice(e->cfg.device);
  if (e->graph_exec) cudaGraphExecDestroy(e->graph_exec);
  if (e->graph) cudaGraphDestroy(e->graph);
  if (e->graph_stream) cudaStreamDestroy(e->graph_stream);
  for (int v = 0; v < ens::kVariants; ++v)
    for (int ph = 0; ph < 4; ++ph)
      if (e->prefix[v][ph]) cudaFree(e->prefix[v][ph]);
  if (e->probs) cudaFree(e->probs);
  if (e->arena) cudaFree(e->arena);
  if (e->bar) cudaFree(e->bar);
  if (e->active_count) cudaFree(e->active_count);
}

void drop_graph(fvh_ensemble* e) {
  if (e->graph_exec) cudaGraphExecDestroy(e->graph_exec);
  if (e->graph) cudaGraphDestroy(e->graph);
  e->graph_exec = nullptr;
  e->graph = nullptr;
}

// Tile counts of every problem for the current variant into the descriptors.
void set_variant_tiles(fvh_ensemble* e) {
  for (int q = 0; q < e->nprob; ++q)
    for (int ph = 0; ph < 4; ++ph) e->host[q].tiles_y[ph] = e->tiles_y[e->variant][ph][q];
}

int upload(fvh_ensemble* e, cudaStream_t s) {
  set_variant_tiles(e);
  const cudaError_t err = cudaMemcpyAsync(e->probs, e->host.data(), sizeof(ens::Problem) * e->nprob,
                                          cudaMemcpyHostToDevice, s);
  if (err != cudaSuccess) return cuda_fail(e, "descriptor upload", err);
  return cudaStreamSynchronize(s) == cudaSuccess ? FVH_OK : cuda_fail(e, "descriptor upload", cudaGetLastError());
}

int launch_stage(fvh_ensemble* e, int stage, int last, cudaStream_t s) {
  return e->elem == sizeof(float) ? ens::launch_stage_f32(e, stage, last, s) : ens::launch_stage_f64(e, stage, last, s);
}

// One SSP-RK3 step of every active problem on stream s (no synchronisation).
int issue_step(fvh_ensemble* e, cudaStream_t s) {
  cudaError_t err = cudaMemsetAsync(e->active_count, 0, sizeof(unsigned int), s);
  if (err != cudaSuccess) return cuda_fail(e, "active counter", err);
  for (int k = 0; k < 3; ++k)
    if (int st = launch_stage(e, k, k == 2, s)) return st;
  return FVH_OK;
}

// Captures one step into a graph on the private stream.
int capture(fvh_ensemble* e) {
  drop_graph(e);
  // occupancy and shared-memory limits are set up outside the capture
  size_t smem = 0;
  const int maxb = e->elem == sizeof(float) ? ens::max_blocks_f32(e->p, e->variant, &smem)
                                            : ens::max_blocks_f64(e->p, e->variant, &smem);
  if (maxb <= 0) return fail(e, FVH_ERR_CONFIG, "this tile variant does not fit for this degree and precision");
  cudaError_t err = cudaStreamBeginCapture(e->graph_stream, cudaStreamCaptureModeThreadLocal);
  if (err != cudaSuccess) return cuda_fail(e, "begin capture", err);
  const int st = issue_step(e, e->graph_stream);
  cudaGraph_t g = nullptr;
  err = cudaStreamEndCapture(e->graph_stream, &g);
  if (st) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  if (err != cudaSuccess) return cuda_fail(e, "end capture", err);
  e->graph = g;
  err = cudaGraphInstantiate(&e->graph_exec, g, 0);
  if (err != cudaSuccess) {
    e->graph_exec = nullptr;
    return cuda_fail(e, "graph instantiate", err);
  }
  return FVH_OK;
}

int check_barrier(fvh_ensemble* e, cudaStream_t s) {
  ens::Barrier b{};
  cudaError_t err = cudaMemcpyAsync(&b, e->bar, sizeof(b), cudaMemcpyDeviceToHost, s);
  if (err == cudaSuccess) err = cudaStreamSynchronize(s);
  if (err != cudaSuccess) return cuda_fail(e, "barrier state", err);
  if (b.abort || b.timeouts) return fail(e, FVH_ERR_TIMEOUT, "an ensemble grid barrier wait ran out");
  return FVH_OK;
}

}  // namespace

extern "C" {

int fvh_ensemble_create(const fvh_config* cfg, int nprob, const int* nx, const int* ny, const double* hx,
                        const double* hy, fvh_ensemble** out) {
  if (!out) return FVH_ERR_ARG;
  *out = nullptr;
  if (!cfg || !nx || !ny || !hx || !hy || nprob <= 0) return fail(nullptr, FVH_ERR_ARG, "null or empty arguments");
  fvh_ensemble* e = new (std::nothrow) fvh_ensemble();
  if (!e) return fail(nullptr, FVH_ERR_CONFIG, "out of host memory");
  e->cfg = *cfg;
  e->cfg.kernel_path = FVH_PATH_FUSED2D;
  e->nprob = nprob;
  // every member must be a valid fused 2D problem on axes x and y
  for (int q = 0; q < nprob; ++q) {
    fvh_config c = e->cfg;
    c.n[0] = nx[q];
    c.n[1] = ny[q];
    c.n[2] = 1;
    c.p[2] = 0;
    c.h[0] = hx[q];
    c.h[1] = hy[q];
    fvh_handle tmp;
    std::string msg;
    if (int st = fvh::configure_handle(&tmp, &c, msg)) {
      delete e;
      return fail(nullptr, st, "problem " + std::to_string(q) + ": " + msg);
    }
    for (int a = 0; a < 2; ++a)
      for (int side = 0; side < 2; ++side)
        if (c.bc[a][side] == FVH_BC_DIRICHLET || c.bc[a][side] == FVH_BC_DMR_Y0) {
          delete e;
          return fail(nullptr, FVH_ERR_CONFIG,
                      "ensemble members cannot have Dirichlet or double-Mach-reflection boundaries");
        }
    if (!tmp.active[0] || !tmp.active[1]) {
      delete e;
      return fail(nullptr, FVH_ERR_CONFIG, "ensemble members must have two active axes (x and y)");
    }
    if (q == 0) {
      e->p = tmp.p[0];
      e->r = tmp.r[0];
      e->gw = tmp.gw;
      e->gW = tmp.gW;
      e->elem = tmp.elem;
    }
    e->nx.push_back(nx[q]);
    e->ny.push_back(ny[q]);
    e->hx.push_back(hx[q]);
    e->hy.push_back(hy[q]);
  }
  {
    std::string msg;
    if (int st = fvh::check_device_visible(&e->cfg, msg)) {
      delete e;
      return fail(nullptr, st, msg);
    }
  }
  if (cudaSetDevice(e->cfg.device) != cudaSuccess) {
    delete e;
    return fail(nullptr, FVH_ERR_CUDA, "cudaSetDevice failed");
  }
  cudaDeviceGetAttribute(&e->sms, cudaDevAttrMultiProcessorCount, e->cfg.device);
  int coop = 0;
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, e->cfg.device);
  if (!coop) {
    delete e;
    return fail(nullptr, FVH_ERR_CONFIG, "the device does not support cooperative launches");
  }
  // arena: all states first (one contiguous block), then per-problem scratch
  const size_t s = e->elem;
  std::vector<size_t> off_u(nprob), off_rest(nprob);
  size_t bytes = 0;
  for (int q = 0; q < nprob; ++q) {
    off_u[q] = bytes;
    bytes += align256((size_t)5 * nx[q] * ny[q] * 8);
  }
  const size_t states_bytes = bytes;
  for (int q = 0; q < nprob; ++q) {
    const size_t cells = (size_t)nx[q] * ny[q];
    const size_t wbox = (size_t)(nx[q] + 2 * e->gW) * (ny[q] + 2 * e->gW);
    off_rest[q] = bytes;
    bytes += 4 * align256(5 * cells * 8);                       // s0, s1, acc, us
    bytes += align256(5 * wbox * s);                            // W
    bytes += align256((size_t)5 * (nx[q] + 1) * ny[q] * s);     // F
    bytes += align256((size_t)5 * nx[q] * (ny[q] + 1) * s);     // G
    bytes += align256(cells);                                   // trouble
    bytes += align256(sizeof(Scalars));                         // reductions
  }
  e->arena_bytes = bytes;
  cudaError_t err = cudaMalloc(&e->arena, bytes);
  if (err == cudaSuccess) err = cudaMalloc(&e->probs, sizeof(ens::Problem) * nprob);
  if (err == cudaSuccess) err = cudaMalloc(&e->bar, sizeof(ens::Barrier));
  if (err == cudaSuccess) err = cudaMalloc(&e->active_count, sizeof(unsigned int));
  if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&e->graph_stream, cudaStreamNonBlocking);
  if (err != cudaSuccess) {
    const int st = cuda_fail(nullptr, "ensemble allocation", err);
    release(e);
    delete e;
    return st;
  }
  cudaMemset(e->arena, 0, bytes);
  cudaMemset(e->bar, 0, sizeof(ens::Barrier));
  (void)states_bytes;
  // descriptors
  e->host.resize(nprob);
  unsigned char* base = static_cast<unsigned char*>(e->arena);
  for (int q = 0; q < nprob; ++q) {
    ens::Problem& p = e->host[q];
    p = ens::Problem{};
    p.g.nx = nx[q];
    p.g.ny = ny[q];
    p.g.bcx[0] = e->cfg.bc[0][0];
    p.g.bcx[1] = e->cfg.bc[0][1];
    p.g.bcy[0] = e->cfg.bc[1][0];
    p.g.bcy[1] = e->cfg.bc[1][1];
    p.g.dx = 0;
    p.g.dy = 1;
    p.g.gmax = e->gW + 2 * e->r;
    // the host arithmetic of fvh_create: CFL * min(h) and -(1 / h) in float64
    const double hmin = std::min(hx[q], std::min(hy[q], e->cfg.h[2]));
    p.cfl_h = e->cfg.cfl * hmin;
    p.cx = -(1.0 / hx[q]);
    p.cy = -(1.0 / hy[q]);
    p.t = 0.0;
    p.t_end = 0.0;
    p.active = 0;
    const size_t cells = (size_t)nx[q] * ny[q];
    const size_t wbox = (size_t)(nx[q] + 2 * e->gW) * (ny[q] + 2 * e->gW);
    p.u = reinterpret_cast<double*>(base + off_u[q]);
    size_t o = off_rest[q];
    p.s[0] = reinterpret_cast<double*>(base + o);
    o += align256(5 * cells * 8);
    p.s[1] = reinterpret_cast<double*>(base + o);
    o += align256(5 * cells * 8);
    p.acc = reinterpret_cast<double*>(base + o);
    o += align256(5 * cells * 8);
    p.us = reinterpret_cast<double*>(base + o);
    o += align256(5 * cells * 8);
    p.W = base + o;
    o += align256(5 * wbox * s);
    p.F = base + o;
    o += align256((size_t)5 * (nx[q] + 1) * ny[q] * s);
    p.G = base + o;
    o += align256((size_t)5 * nx[q] * (ny[q] + 1) * s);
    p.trouble = reinterpret_cast<uint8_t*>(base + o);
    o += align256(cells);
    p.sc = reinterpret_cast<Scalars*>(base + o);
  }
  // the reductions start empty: keys at their identities
  {
    std::vector<Scalars> init(1);
    Scalars& sc = init[0];
    std::memset(&sc, 0, sizeof(sc));
    for (int v = 0; v < kMaxVars; ++v) sc.vmin_key[v] = ~0ull;
    for (int q = 0; q < nprob; ++q) cudaMemcpy(e->host[q].sc, &sc, sizeof(sc), cudaMemcpyHostToDevice);
  }
  // tile prefix sums of every variant
  for (int v = 0; v < ens::kVariants; ++v) {
    for (int ph = 0; ph < 4; ++ph) {
      std::vector<int> prefix(nprob + 1, 0);
      e->tiles_y[v][ph].resize(nprob);
      for (int q = 0; q < nprob; ++q) {
        int ty, tx;
        if (ph == 0) {
          ty = ceil_div(ny[q] + 2 * e->gW, ens::kPrimTY);
          tx = ceil_div(nx[q] + 2 * e->gW, ens::kPrimTX);
        } else {
          ty = ceil_div(ny[q], ens::kVariantTY[v]);
          tx = ceil_div(nx[q], ens::kVariantTX[v]);
        }
        e->tiles_y[v][ph][q] = ty;
        const long long next = (long long)prefix[q] + (long long)tx * ty;
        if (next >= (1ll << 31)) {
          release(e);
          delete e;
          return fail(nullptr, FVH_ERR_CONFIG, "too many tiles in the ensemble");
        }
        prefix[q + 1] = (int)next;
      }
      e->ntiles[v][ph] = prefix[nprob];
      err = cudaMalloc(&e->prefix[v][ph], sizeof(int) * (nprob + 1));
      if (err == cudaSuccess)
        err = cudaMemcpy(e->prefix[v][ph], prefix.data(), sizeof(int) * (nprob + 1), cudaMemcpyHostToDevice);
      if (err != cudaSuccess) {
        const int st = cuda_fail(nullptr, "tile tables", err);
        release(e);
        delete e;
        return st;
      }
    }
  }
  e->variant = e->elem == sizeof(float) ? 0 : 1;
  if (int st = upload(e, nullptr)) {
    g_ens_error = e->err;
    release(e);
    delete e;
    return st;
  }
  *out = e;
  return FVH_OK;
}

int fvh_ensemble_destroy(fvh_ensemble* e) {
  if (!e) return FVH_OK;
  release(e);
  delete e;
  return FVH_OK;
}

const char* fvh_ensemble_last_error(const fvh_ensemble* e) { return e ? e->err.c_str() : g_ens_error.c_str(); }

size_t fvh_ensemble_bytes(const fvh_ensemble* e) { return e ? e->arena_bytes : 0; }

double* fvh_ensemble_state(fvh_ensemble* e, int q) {
  if (!e || q < 0 || q >= e->nprob) return nullptr;
  return e->host[q].u;
}

int fvh_ensemble_load(fvh_ensemble* e, int q, const double* src, void* stream) {
  if (!e) return FVH_ERR_ARG;
  if (q < 0 || q >= e->nprob || !src) return fail(e, FVH_ERR_ARG, "bad member index or null source");
  if (cudaSetDevice(e->cfg.device) != cudaSuccess) return cuda_fail(e, "cudaSetDevice", cudaGetLastError());
  const size_t bytes = (size_t)5 * e->nx[q] * e->ny[q] * sizeof(double);
  const cudaError_t err = cudaMemcpyAsync(e->host[q].u, src, bytes, cudaMemcpyDefault, (cudaStream_t)stream);
  return err == cudaSuccess ? FVH_OK : cuda_fail(e, "state load", err);
}

int fvh_ensemble_store(fvh_ensemble* e, int q, double* dst, void* stream) {
  if (!e) return FVH_ERR_ARG;
  if (q < 0 || q >= e->nprob || !dst) return fail(e, FVH_ERR_ARG, "bad member index or null destination");
  if (cudaSetDevice(e->cfg.device) != cudaSuccess) return cuda_fail(e, "cudaSetDevice", cudaGetLastError());
  const size_t bytes = (size_t)5 * e->nx[q] * e->ny[q] * sizeof(double);
  cudaError_t err = cudaMemcpyAsync(dst, e->host[q].u, bytes, cudaMemcpyDefault, (cudaStream_t)stream);
  if (err == cudaSuccess) err = cudaStreamSynchronize((cudaStream_t)stream);
  return err == cudaSuccess ? FVH_OK : cuda_fail(e, "state store", err);
}

int fvh_ensemble_reset(fvh_ensemble* e, double t0, double t_end, void* stream) {
  if (!e) return FVH_ERR_ARG;
  if (cudaSetDevice(e->cfg.device) != cudaSuccess) return cuda_fail(e, "cudaSetDevice", cudaGetLastError());
  cudaStream_t s = (cudaStream_t)stream;
  for (auto& p : e->host) {
    p.t = t0;
    p.t_end = t_end;
    p.active = t0 < t_end ? 1 : 0;
    p.steps = 0;
    p.dt_step = 0.0;
  }
  cudaError_t err = cudaMemsetAsync(e->bar, 0, sizeof(ens::Barrier), s);
  if (err != cudaSuccess) return cuda_fail(e, "barrier reset", err);
  for (auto& p : e->host) {
    err = cudaMemsetAsync(&p.sc->nonfinite, 0, sizeof(unsigned int), s);
    if (err != cudaSuccess) return cuda_fail(e, "counter reset", err);
  }
  return upload(e, s);
}

int fvh_ensemble_configure(fvh_ensemble* e, int variant, int blocks_per_sm, int use_graph) {
  if (!e) return FVH_ERR_ARG;
  if (variant < 0 || variant >= ens::kVariants) return fail(e, FVH_ERR_ARG, "unknown tile variant");
  if (cudaSetDevice(e->cfg.device) != cudaSuccess) return cuda_fail(e, "cudaSetDevice", cudaGetLastError());
  size_t smem = 0;
  const int maxb = e->elem == sizeof(float) ? ens::max_blocks_f32(e->p, variant, &smem)
                                            : ens::max_blocks_f64(e->p, variant, &smem);
  if (maxb <= 0) return fail(e, FVH_ERR_CONFIG, "this tile variant does not fit for this degree and precision");
  // host descriptors may hold times newer than the host copy: read them back first
  cudaError_t err = cudaMemcpy(e->host.data(), e->probs, sizeof(ens::Problem) * e->nprob, cudaMemcpyDeviceToHost);
  if (err != cudaSuccess) return cuda_fail(e, "descriptor read", err);
  e->variant = variant;
  e->blocks_per_sm = blocks_per_sm < 0 ? 0 : blocks_per_sm;
  e->use_graph = use_graph != 0;
  drop_graph(e);
  return upload(e, nullptr);
}

int fvh_ensemble_set_wait_limit(fvh_ensemble* e, unsigned int polls) {
  if (!e) return FVH_ERR_ARG;
  if (polls == e->wait_limit) return FVH_OK;
  e->wait_limit = polls;
  drop_graph(e);  // a captured step holds the old bound in its kernel arguments
  return FVH_OK;
}

int fvh_ensemble_variant_info(fvh_ensemble* e, int variant, int* tx, int* ty, int* max_blocks_per_sm,
                              size_t* smem_bytes) {
  if (!e || variant < 0 || variant >= ens::kVariants) return FVH_ERR_ARG;
  if (cudaSetDevice(e->cfg.device) != cudaSuccess) return cuda_fail(e, "cudaSetDevice", cudaGetLastError());
  size_t smem = 0;
  const int maxb = e->elem == sizeof(float) ? ens::max_blocks_f32(e->p, variant, &smem)
                                            : ens::max_blocks_f64(e->p, variant, &smem);
  if (tx) *tx = ens::kVariantTX[variant];
  if (ty) *ty = ens::kVariantTY[variant];
  if (max_blocks_per_sm) *max_blocks_per_sm = maxb;
  if (smem_bytes) *smem_bytes = smem;
  return FVH_OK;
}

int fvh_ensemble_step(fvh_ensemble* e, int nsteps, void* stream) {
  if (!e || nsteps < 0) return FVH_ERR_ARG;
  if (cudaSetDevice(e->cfg.device) != cudaSuccess) return cuda_fail(e, "cudaSetDevice", cudaGetLastError());
  cudaStream_t s = (cudaStream_t)stream;
  if (nsteps == 0) return FVH_OK;
  if (e->use_graph && !e->graph_failed) {
    if (!e->graph_exec) {
      if (int st = capture(e)) {
        // cooperative launches that cannot be captured fall back to direct launches
        e->graph_failed = true;
        e->graph_error = e->err;
      }
    }
  }
  if (e->use_graph && !e->graph_failed && e->graph_exec) {
    cudaEvent_t in = nullptr, done = nullptr;
    cudaError_t err = cudaEventCreateWithFlags(&in, cudaEventDisableTiming);
    if (err == cudaSuccess) err = cudaEventCreateWithFlags(&done, cudaEventDisableTiming);
    if (err == cudaSuccess) err = cudaEventRecord(in, s);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(e->graph_stream, in, 0);
    for (int i = 0; i < nsteps && err == cudaSuccess; ++i) {
      err = cudaGraphLaunch(e->graph_exec, e->graph_stream);
      launch_counter().fetch_add(3, std::memory_order_relaxed);
    }
    if (err == cudaSuccess) err = cudaEventRecord(done, e->graph_stream);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(s, done, 0);
    if (in) cudaEventDestroy(in);
    if (done) cudaEventDestroy(done);
    if (err != cudaSuccess) return cuda_fail(e, "graph launch", err);
    return FVH_OK;
  }
  for (int i = 0; i < nsteps; ++i)
    if (int st = issue_step(e, s)) return st;
  return FVH_OK;
}

int fvh_ensemble_status(fvh_ensemble* e, double* t, int* steps, int* active, unsigned int* nonfinite,
                        void* stream) {
  if (!e) return FVH_ERR_ARG;
  if (cudaSetDevice(e->cfg.device) != cudaSuccess) return cuda_fail(e, "cudaSetDevice", cudaGetLastError());
  cudaStream_t s = (cudaStream_t)stream;
  if (int st = check_barrier(e, s)) return st;
  std::vector<ens::Problem> d(e->nprob);
  cudaError_t err = cudaMemcpyAsync(d.data(), e->probs, sizeof(ens::Problem) * e->nprob, cudaMemcpyDeviceToHost, s);
  if (err == cudaSuccess) err = cudaStreamSynchronize(s);
  if (err != cudaSuccess) return cuda_fail(e, "status read", err);
  int nact = 0;
  unsigned int bad = 0;
  for (int q = 0; q < e->nprob; ++q) {
    if (t) t[q] = d[q].t;
    if (steps) steps[q] = d[q].steps;
    nact += d[q].active;
    if (nonfinite) {
      unsigned int nf = 0;
      err = cudaMemcpy(&nf, &d[q].sc->nonfinite, sizeof(nf), cudaMemcpyDeviceToHost);
      if (err != cudaSuccess) return cuda_fail(e, "counter read", err);
      bad += nf;
    }
  }
  if (active) *active = nact;
  if (nonfinite) *nonfinite = bad;
  return FVH_OK;
}

int fvh_ensemble_graph_info(const fvh_ensemble* e, int* in_use, const char** error) {
  if (!e) return FVH_ERR_ARG;
  if (in_use) *in_use = (e->use_graph && !e->graph_failed && e->graph_exec) ? 1 : 0;
  if (error) *error = e->graph_error.c_str();
  return FVH_OK;
}

int fvh_ensemble_autotune(fvh_ensemble* e, int steps, int* variant_out, int* blocks_out, double* ms_out,
                          void* stream) {
  if (!e || steps <= 0) return FVH_ERR_ARG;
  if (cudaSetDevice(e->cfg.device) != cudaSuccess) return cuda_fail(e, "cudaSetDevice", cudaGetLastError());
  cudaStream_t s = (cudaStream_t)stream;
  // the trials advance the problems: keep the states and descriptors to put back
  size_t states = 0;
  for (int q = 0; q < e->nprob; ++q) states += align256((size_t)5 * e->nx[q] * e->ny[q] * 8);
  void* backup = nullptr;
  cudaError_t err = cudaMalloc(&backup, states);
  if (err != cudaSuccess) return cuda_fail(e, "autotune backup", err);
  err = cudaMemcpyAsync(backup, e->host[0].u, states, cudaMemcpyDeviceToDevice, s);
  std::vector<ens::Problem> saved(e->nprob);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(saved.data(), e->probs, sizeof(ens::Problem) * e->nprob, cudaMemcpyDeviceToHost, s);
  if (err == cudaSuccess) err = cudaStreamSynchronize(s);
  if (err != cudaSuccess) {
    cudaFree(backup);
    return cuda_fail(e, "autotune backup", err);
  }
  const bool graph = e->use_graph;
  double best = 1e300;
  int best_v = e->variant, best_b = e->blocks_per_sm;
  cudaEvent_t a = nullptr, b = nullptr;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  int status = FVH_OK;
  for (int v = 0; v < ens::kVariants && status == FVH_OK; ++v) {
    size_t smem = 0;
    const int maxb = e->elem == sizeof(float) ? ens::max_blocks_f32(e->p, v, &smem)
                                              : ens::max_blocks_f64(e->p, v, &smem);
    if (maxb <= 0) continue;
    const int cands[2] = {maxb, maxb > 1 ? maxb - 1 : 0};
    for (int c = 0; c < 2 && status == FVH_OK; ++c) {
      if (cands[c] <= 0) continue;
      e->host = saved;
      if ((status = fvh_ensemble_configure(e, v, cands[c], 0))) break;
      e->host = saved;
      if ((status = upload(e, s))) break;
      // one untimed step, then the timed ones
      if ((status = fvh_ensemble_step(e, 1, stream))) break;
      cudaEventRecord(a, s);
      if ((status = fvh_ensemble_step(e, steps, stream))) break;
      cudaEventRecord(b, s);
      cudaEventSynchronize(b);
      if ((status = check_barrier(e, s))) break;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, a, b);
      if (ms < best) {
        best = ms;
        best_v = v;
        best_b = cands[c];
      }
      // put the states back for the next trial
      err = cudaMemcpyAsync(e->host[0].u, backup, states, cudaMemcpyDeviceToDevice, s);
      if (err != cudaSuccess) status = cuda_fail(e, "autotune restore", err);
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  err = cudaMemcpyAsync(e->host[0].u, backup, states, cudaMemcpyDeviceToDevice, s);
  cudaStreamSynchronize(s);
  cudaFree(backup);
  if (status) return status;
  if (err != cudaSuccess) return cuda_fail(e, "autotune restore", err);
  e->host = saved;
  if ((status = fvh_ensemble_configure(e, best_v, best_b, graph ? 1 : 0))) return status;
  e->host = saved;
  if ((status = upload(e, s))) return status;
  if (variant_out) *variant_out = best_v;
  if (blocks_out) *blocks_out = best_b;
  if (ms_out) *ms_out = best / steps;
  return FVH_OK;
}

}  // extern "C"
