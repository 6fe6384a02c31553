// C ABI of the per-stage update (declarations and reference citations in
// include/fvh.h): configuration checks, scratch allocation, and the stage
// sequences of the Runge-Kutta integrators.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include <cudaTypedefs.h>

#include "fvh_handle.h"
#include "fvh_tma.cuh"

namespace fvh {

bool encode_tensor_map_3d(CUtensorMap* map, const void* base, int elem, int cols, int rows, int nv, int sx, int vs,
                          int box_cols, int box_rows, int box_vars, const char** why) {
  // the driver's encoder, reached through the runtime (no link against libcuda)
  static PFN_cuTensorMapEncodeTiled_v12000 encode = [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      fn = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }();
  if (!encode) {
    *why = "cuTensorMapEncodeTiled is not available from the driver";
    return false;
  }
  const cuuint64_t dims[3] = {(cuuint64_t)cols, (cuuint64_t)rows, (cuuint64_t)nv};
  const cuuint64_t strides[2] = {(cuuint64_t)sx * elem, (cuuint64_t)vs * elem};
  const cuuint32_t box[3] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows, (cuuint32_t)box_vars};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = encode(map, elem == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
                            const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    *why = "cuTensorMapEncodeTiled refused the tile map";
    return false;
  }
  return true;
}

Profiler::~Profiler() {
  for (auto& p : used_) {
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  for (auto& p : pool_) {
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
}

void Profiler::record_begin(int kind, double bytes, cudaStream_t s) {
  Pair p;
  if (!pool_.empty()) {
    p = pool_.back();
    pool_.pop_back();
  } else {
    cudaEventCreate(&p.a);
    cudaEventCreate(&p.b);
  }
  p.kind = kind;
  p.bytes = bytes;
  cudaEventRecord(p.a, s);
  open_.push_back(used_.size());
  used_.push_back(p);
}

void Profiler::record_end(cudaStream_t s) {
  if (open_.empty()) return;
  cudaEventRecord(used_[open_.back()].b, s);
  open_.pop_back();
}

int Profiler::collect(KernelTotals& t) {
  if (!open_.empty()) return FVH_ERR_CUDA;  // a scope is still open
  for (auto& p : used_) {
    if (cudaEventSynchronize(p.b) != cudaSuccess) return FVH_ERR_CUDA;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, p.a, p.b) != cudaSuccess) return FVH_ERR_CUDA;
    t.ms[p.kind] += ms;
    t.bytes[p.kind] += p.bytes;
    t.launches[p.kind] += 1;
    pool_.push_back(p);
  }
  used_.clear();
  return FVH_OK;
}

Profiler*& active_profiler() {
  thread_local Profiler* p = nullptr;
  return p;
}

std::atomic<uint64_t>& launch_counter() {
  static std::atomic<uint64_t> n{0};
  return n;
}

}  // namespace fvh

namespace {

// Makes h's profiler (if enabled) the calling thread's for the scope.
struct ProfilerBinding {
  explicit ProfilerBinding(fvh_handle* h) { fvh::active_profiler() = h->prof; }
  ~ProfilerBinding() { fvh::active_profiler() = nullptr; }
};

thread_local std::string g_create_error;

int fail(fvh_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

int ceil_half(int p) { return (p + 1) / 2; }

// Validates cfg and fills the derived geometry of h. Mirrors the checks the
// reference makes implicitly: an axis is active unless it has one cell and
// p = 0 (fvhoe/solver.py:244-254); the ghost width of the flux pass is
// max(ceil(p/2) + 1, 2 ceil(p/2)) (fvhoe/solver.py:492-493); mirrored and
// periodic ghost fills read no further than the interior.
int configure(fvh_handle* h, const fvh_config* cfg, std::string& msg) {
  if (cfg->abi_version != FVH_ABI_VERSION) {
    msg = "abi_version mismatch";
    return FVH_ERR_CONFIG;
  }
  if (cfg->nvars < 5 || cfg->nvars > fvh::kMaxVars) {
    msg = "nvars must be in [5, 16]";
    return FVH_ERR_CONFIG;
  }
  h->cfg = *cfg;
  h->nv = cfg->nvars;
  int pmax = 0;
  h->ndim = 0;
  for (int a = 0; a < 3; ++a) {
    if (cfg->n[a] < 1) {
      msg = "n must be >= 1 on every axis";
      return FVH_ERR_CONFIG;
    }
    if (cfg->p[a] < 0 || cfg->p[a] > 8) {
      msg = "p must be in [0, 8]";
      return FVH_ERR_CONFIG;
    }
    h->n[a] = cfg->n[a];
    h->p[a] = cfg->p[a];
    h->r[a] = ceil_half(cfg->p[a]);
    h->active[a] = !(cfg->n[a] == 1 && cfg->p[a] == 0);
    if (h->active[a]) {
      h->ndim += 1;
      if (cfg->p[a] > pmax) pmax = cfg->p[a];
    }
    if (!(cfg->h[a] > 0.0)) {
      msg = "cell widths must be positive";
      return FVH_ERR_CONFIG;
    }
  }
  if (h->ndim == 0) {
    msg = "no active axis";
    return FVH_ERR_CONFIG;
  }
  const int rmax = ceil_half(pmax);
  h->gw = std::max(rmax + 1, 2 * rmax);
  h->gW = cfg->a_posteriori ? std::max(h->gw, 3) : h->gw;
  for (int a = 0; a < 3; ++a) {
    if (!h->active[a]) continue;
    for (int side = 0; side < 2; ++side) {
      const int k = cfg->bc[a][side];
      if (k < FVH_BC_PERIODIC || k > FVH_BC_DMR_Y0) {
        msg = "unsupported boundary kind";
        return FVH_ERR_CONFIG;
      }
      if (k == FVH_BC_DMR_Y0 && !(a == 1 && side == 0)) {
        msg = "the double-Mach-reflection boundary is defined on the low y side only";
        return FVH_ERR_CONFIG;
      }
    }
    if (cfg->bc[a][1] == FVH_BC_PERIODIC && cfg->bc[a][0] != FVH_BC_PERIODIC) {
      msg = "a periodic high boundary needs a periodic low boundary";
      return FVH_ERR_CONFIG;
    }
    const int ghosts = h->gW + 2 * h->r[a];
    for (int side = 0; side < 2; ++side) {
      // mirrored and periodic ghosts copy interior cells; free and Dirichlet ones do not
      const int k = cfg->bc[a][side];
      if (k != FVH_BC_FREE && k != FVH_BC_DIRICHLET && ghosts > cfg->n[a]) {
        msg = "axis " + std::string(1, "xyz"[a]) + " has " + std::to_string(cfg->n[a]) +
              " cells, fewer than the " + std::to_string(ghosts) + " ghost cells this degree needs";
        return FVH_ERR_CONFIG;
      }
    }
    h->grid.bc[a][0] = cfg->bc[a][0];
    h->grid.bc[a][1] = cfg->bc[a][1];
  }
  for (int a = 0; a < 3; ++a) {
    h->grid.n[a] = cfg->n[a];
    if (!h->active[a]) {
      h->grid.bc[a][0] = FVH_BC_FREE;
      h->grid.bc[a][1] = FVH_BC_FREE;
    }
  }
  if (cfg->riemann < 0 || cfg->riemann > 2) {
    msg = "unknown Riemann solver";
    return FVH_ERR_CONFIG;
  }
  if (cfg->slope_limiter < 0 || cfg->slope_limiter > 2) {
    msg = "unknown slope limiter";
    return FVH_ERR_CONFIG;
  }
  if (cfg->precision != FVH_PREC_FP64 && cfg->precision != FVH_PREC_FP32) {
    msg = "unknown precision mode";
    return FVH_ERR_CONFIG;
  }
  if (cfg->a_posteriori && cfg->convex && h->ndim > 2) {
    msg = "3D convex broadcast not implemented";
    return FVH_ERR_CONFIG;
  }
  if (cfg->kernel_path < FVH_PATH_AUTO || cfg->kernel_path > FVH_PATH_FUSED2D) {
    msg = "unknown kernel path";
    return FVH_ERR_CONFIG;
  }
  if (cfg->kernel_path == FVH_PATH_FUSED2D) {
    int na = 0, p0 = -1;
    bool same = true;
    for (int a = 0; a < 3; ++a) {
      if (!(cfg->n[a] == 1 && cfg->p[a] == 0)) {
        ++na;
        if (p0 < 0) p0 = cfg->p[a];
        same = same && cfg->p[a] == p0;
      }
    }
    if (na != 2 || cfg->nvars != 5 || (cfg->a_posteriori && cfg->convex) || !same || p0 < 1) {
      msg = "the fused 2D kernels need two active axes, five variables, equal p in 1..8, no convex weights";
      return FVH_ERR_CONFIG;
    }
  }
  if (cfg->pad_var < -1 || cfg->pad_var > 4) {
    msg = "pad_var must be -1 or a primitive index in [0, 4]";
    return FVH_ERR_CONFIG;
  }
  if (!(cfg->gamma > 1.0)) {
    msg = "gamma must exceed 1";
    return FVH_ERR_CONFIG;
  }
  // Python evaluates CFL * min(h) and -(1 / h) in float64; so does the host here.
  const double hmin = std::min(cfg->h[0], std::min(cfg->h[1], cfg->h[2]));
  h->cfl_h = cfg->cfl * hmin;
  for (int a = 0; a < 3; ++a) h->neg_inv_h[a] = -(1.0 / cfg->h[a]);
  h->elem = cfg->precision == FVH_PREC_FP32 ? sizeof(float) : sizeof(double);
  // kernels address arrays with 32-bit offsets: the largest (the state
  // ghost-filled by gW + 2r cells on every active axis, all variables) must
  // stay below 2^31 elements
  double largest = (double)h->nv;
  for (int a = 0; a < 3; ++a) largest *= (double)(h->n[a] + (h->active[a] ? 2 * (h->gW + 2 * h->r[a]) : 0));
  if (largest >= 2147483648.0) {
    msg = "grid too large: a sweep buffer would exceed 2^31 elements";
    return FVH_ERR_CONFIG;
  }
  return FVH_OK;
}

// cfg->device must name a visible CUDA device.
int check_device(const fvh_config* cfg, std::string& msg) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess) {
    cudaGetLastError();
    count = 0;
  }
  if (cfg->device < 0 || cfg->device >= count) {
    msg = "device " + std::to_string(cfg->device) + " is not a visible CUDA device (" + std::to_string(count) +
          " visible)";
    return FVH_ERR_CONFIG;
  }
  return FVH_OK;
}

// Each entry point selects the handle's device first: this library carries its
// own CUDA runtime, whose current device is independent of the caller's.
int use_device(fvh_handle* h) {
  const cudaError_t e = cudaSetDevice(h->cfg.device);
  if (e != cudaSuccess) {
    h->err = std::string("cudaSetDevice: ") + cudaGetErrorString(e);
    return FVH_ERR_CUDA;
  }
  return FVH_OK;
}

int64_t box(const fvh_handle* h, int g) {
  int64_t n = 1;
  for (int a = 0; a < 3; ++a) n *= h->n[a] + (h->active[a] ? 2 * g : 0);
  return n;
}

int alloc(fvh_handle* h, void** p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  const cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    h->err = std::string("cudaMalloc of ") + std::to_string(bytes) + " bytes: " + cudaGetErrorString(e);
    return FVH_ERR_CUDA;
  }
  h->scratch_bytes += bytes;
  return FVH_OK;
}

void release(fvh_handle* h) {
  cudaSetDevice(h->cfg.device);
  delete h->prof;
  h->prof = nullptr;
  if (h->copy_out) cudaStreamSynchronize(h->copy_out);
  if (h->copy_in) cudaStreamSynchronize(h->copy_in);
  for (cudaEvent_t& e : h->out_done)
    if (e) cudaEventDestroy(e);
  if (h->in_done) cudaEventDestroy(h->in_done);
  if (h->step_done) cudaEventDestroy(h->step_done);
  if (h->copy_in) cudaStreamDestroy(h->copy_in);
  if (h->copy_out) cudaStreamDestroy(h->copy_out);
  if (h->host_state) cudaFree(h->host_state);
  void* ptrs[] = {h->bufA, h->bufB, h->W,        h->Ws,       h->Us,       h->F[0],     h->F[1],
                  h->F[2], h->trouble, h->logs[0], h->logs[1], h->logs[2], h->acc,      h->S[0],
                  h->S[1], h->theta[0], h->theta[1], h->theta[2], h->conv, h->sc, h->pred, h->slabs_dev,
                  h->slab[0][0], h->slab[0][1], h->slab[1][0], h->slab[1][1], h->slab[2][0], h->slab[2][1]};
  for (void* p : ptrs)
    if (p) cudaFree(p);
}

int allocate(fvh_handle* h) {
  const size_t nv = (size_t)h->nv;
  const size_t el = h->elem;
  int64_t ncell = (int64_t)h->n[0] * h->n[1] * h->n[2];
  // largest sweep box: the state ghost-filled by gW + 2r on each active axis
  int64_t big = 1;
  for (int a = 0; a < 3; ++a) big *= h->n[a] + (h->active[a] ? 2 * (h->gW + 2 * h->r[a]) : 0);
  h->buf_elems = nv * (size_t)big;
  int st;
  // double-sized even in FP32 mode: the snapshot conversion always runs in FP64
  if ((st = alloc(h, &h->bufA, h->buf_elems * sizeof(double)))) return st;
  if ((st = alloc(h, &h->bufB, h->buf_elems * sizeof(double)))) return st;
  // W and W* hold either the generic path's boxes or the fused 2D path's padded rows
  const bool two_d = h->ndim == 2;
  const size_t w_elems = std::max((size_t)box(h, h->gW), two_d ? fvh::fused_w_layout(h, h->gW).elems : 0);
  const size_t ws_elems = std::max((size_t)box(h, 3), two_d ? fvh::fused_w_layout(h, 3).elems : 0);
  if ((st = alloc(h, &h->W, nv * w_elems * el))) return st;
  cudaMemset(h->W, 0, nv * w_elems * el);  // padding columns that tile copies read stay zero
  for (int d = 0; d < 3; ++d) {
    if (!h->active[d]) continue;
    const size_t faces = (size_t)ncell / h->n[d] * (h->n[d] + 1);
    if ((st = alloc(h, &h->F[d], nv * faces * el))) return st;
  }
  if (h->cfg.a_posteriori) {
    if ((st = alloc(h, &h->Ws, nv * ws_elems * el))) return st;
    cudaMemset(h->Ws, 0, nv * ws_elems * el);
    if ((st = alloc(h, (void**)&h->Us, nv * (size_t)ncell * sizeof(double)))) return st;
    if ((st = alloc(h, (void**)&h->trouble, (size_t)ncell))) return st;
    if (h->cfg.log_troubles) {
      for (int i = 0; i < 3; ++i) {
        if ((st = alloc(h, (void**)&h->logs[i], (size_t)ncell * sizeof(double)))) return st;
        cudaMemset(h->logs[i], 0, (size_t)ncell * sizeof(double));
      }
    }
    if (h->cfg.convex) {
      for (int d = 0; d < 3; ++d) {
        if (!h->active[d]) continue;
        const size_t faces = (size_t)ncell / h->n[d] * (h->n[d] + 1);
        if ((st = alloc(h, (void**)&h->theta[d], faces * sizeof(float)))) return st;
      }
      if ((st = alloc(h, (void**)&h->conv, 3 * (size_t)box(h, 2) * sizeof(float)))) return st;
    }
  }
  const size_t state = nv * (size_t)ncell * sizeof(double);
  if ((st = alloc(h, (void**)&h->acc, state))) return st;
  if ((st = alloc(h, (void**)&h->S[0], state))) return st;
  if ((st = alloc(h, (void**)&h->S[1], state))) return st;
  if ((st = alloc(h, (void**)&h->sc, sizeof(fvh::Scalars)))) return st;
  cudaMemset(h->sc, 0, sizeof(fvh::Scalars));
  // Dirichlet sides: ghost-value arrays (zero until the caller uploads) and their
  // descriptor, which the double-Mach-reflection wall also needs (its split)
  bool dirichlet = h->active[1] && h->cfg.bc[1][0] == FVH_BC_DMR_Y0;
  fvh::Slabs& m = h->slab_meta;
  m.dmr_split = h->cfg.dmr_split;
  for (int a = 0; a < 3; ++a) {
    m.n[a] = h->n[a];
    m.depth[a] = h->active[a] ? h->gW + 2 * h->r[a] : 0;
    m.pad[a] = m.depth[a];
    for (int side = 0; side < 2; ++side) m.bc[a][side] = h->grid.bc[a][side];
  }
  for (int a = 0; a < 3; ++a) {
    if (!h->active[a]) continue;
    for (int side = 0; side < 2; ++side) {
      if (h->cfg.bc[a][side] != FVH_BC_DIRICHLET) continue;
      size_t count = nv * (size_t)m.depth[a];
      for (int b = 0; b < 3; ++b)
        if (b != a) count *= (size_t)(h->n[b] + 2 * m.pad[b]);
      if ((st = alloc(h, (void**)&h->slab[a][side], count * sizeof(double)))) return st;
      cudaMemset(h->slab[a][side], 0, count * sizeof(double));
      h->slab_count[a][side] = count;
      m.p[a][side] = h->slab[a][side];
      dirichlet = true;
    }
  }
  if (dirichlet) {
    if ((st = alloc(h, (void**)&h->slabs_dev, sizeof(fvh::Slabs)))) return st;
    cudaMemcpy(h->slabs_dev, &m, sizeof(fvh::Slabs), cudaMemcpyHostToDevice);
    h->grid.slabs = h->slabs_dev;
  }
  const cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    h->err = std::string("initialising scratch: ") + cudaGetErrorString(e);
    return FVH_ERR_CUDA;
  }
  return FVH_OK;
}

}  // namespace

namespace fvh {
// Configuration checks shared with the handle-free entry point (fvh_noalloc.cu):
// the geometry and kinds of cfg (no CUDA call), and the device ordinal.
int configure_handle(fvh_handle* h, const fvh_config* cfg, std::string& msg) { return configure(h, cfg, msg); }
int check_device_visible(const fvh_config* cfg, std::string& msg) { return check_device(cfg, msg); }
}  // namespace fvh

namespace {

int run_stage(fvh_handle* h, const fvh::StageCall& c, cudaStream_t s) {
  ProfilerBinding bind(h);
  return h->cfg.precision == FVH_PREC_FP32 ? fvh::run_stage_f32(h, c, s) : fvh::run_stage_f64(h, c, s);
}

int next_log_mode(fvh_handle* h) {
  const int m = h->log_mode_next;
  h->log_mode_next = 2;
  return m;
}

// The dt read-back of fvh_step / fvh_rhs / fvh_step_host. The same copy brings
// the step's non-finite count, so a call that reads dt also reports a failed
// update: FVH_ERR_NONFINITE when the update wrote NaN/Inf values, when dt is
// not finite, or when a CFL dt is not positive (an infinite signal speed);
// *dt_out is written in every case.
int read_dt(fvh_handle* h, cudaStream_t s, double* dt_out) {
  if (!dt_out) return FVH_OK;
  fvh::Scalars host{};
  cudaError_t e = cudaMemcpyAsync(&host, h->sc, sizeof(host), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    h->err = std::string("reading dt: ") + cudaGetErrorString(e);
    return FVH_ERR_CUDA;
  }
  *dt_out = host.dt_step;
  if (host.timeouts)
    return fail(h, FVH_ERR_TIMEOUT,
                std::to_string(host.timeouts) +
                    " tile copies were refused (misaligned) or did not complete within their bounded waits");
  if (host.nonfinite)
    return fail(h, FVH_ERR_NONFINITE,
                "the update wrote " + std::to_string(host.nonfinite) + " non-finite values");
  if (!std::isfinite(host.dt_step) || !std::isfinite(host.dt_stage))
    return fail(h, FVH_ERR_NONFINITE, "the time step is not finite");
  if (!h->cfg.use_fixed_dt && !(host.dt_stage > 0.0))
    return fail(h, FVH_ERR_NONFINITE, "the CFL time step is not positive (infinite signal speed)");
  return FVH_OK;
}

// Device copy, copy streams and events of fvh_step_host, made on its first
// call; all or nothing, so a failed set-up is retried by the next call.
int host_path_init(fvh_handle* h) {
  if (h->host_state) return FVH_OK;
  cudaStream_t in = nullptr, out = nullptr;
  cudaEvent_t ev[fvh_handle::kHostChunks + 2] = {};
  cudaError_t e = cudaStreamCreateWithFlags(&in, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&out, cudaStreamNonBlocking);
  for (int j = 0; j < fvh_handle::kHostChunks + 2 && e == cudaSuccess; ++j)
    e = cudaEventCreateWithFlags(&ev[j], cudaEventDisableTiming);
  double* state = nullptr;
  int st = FVH_OK;
  if (e == cudaSuccess)
    st = alloc(h, (void**)&state, (size_t)h->nv * h->n[0] * h->n[1] * h->n[2] * sizeof(double));
  if (e != cudaSuccess || st != FVH_OK) {
    for (cudaEvent_t x : ev)
      if (x) cudaEventDestroy(x);
    if (in) cudaStreamDestroy(in);
    if (out) cudaStreamDestroy(out);
    if (e != cudaSuccess) return fail(h, FVH_ERR_CUDA, std::string("host path set-up: ") + cudaGetErrorString(e));
    return st;
  }
  h->copy_in = in;
  h->copy_out = out;
  for (int j = 0; j < fvh_handle::kHostChunks; ++j) h->out_done[j] = ev[j];
  h->in_done = ev[fvh_handle::kHostChunks];
  h->step_done = ev[fvh_handle::kHostChunks + 1];
  h->host_state = state;
  return FVH_OK;
}

__global__ void k_divide(double* a, int64_t n, double by) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    a[i] = a[i] / by;
}

}  // namespace

extern "C" {

void fvh_config_default(fvh_config* c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->abi_version = FVH_ABI_VERSION;
  c->nvars = 5;
  for (int a = 0; a < 3; ++a) {
    c->n[a] = 1;
    c->p[a] = 0;
    c->h[a] = 1.0;
    c->bc[a][0] = FVH_BC_PERIODIC;
    c->bc[a][1] = FVH_BC_PERIODIC;
  }
  c->gamma = 5.0 / 3.0;
  c->cfl = 0.8;
  c->csq_floor = 1e-10;
  c->riemann = FVH_RIEMANN_HLLC;
  c->slope_limiter = FVH_LIMITER_MINMOD;
  c->nad_eps = 1e-2;
  c->nad_global = 1;
  c->nad_relative = 1;
  c->nad_var_mask = 0x1f;
  c->pad_var = 4;
  c->pad_lo = 0.0;
  c->pad_hi = INFINITY;
  c->sed = 1;
  c->sed_eps = 1e-10;
  c->precision = FVH_PREC_FP64;
  c->log_troubles = 1;
}

int fvh_create(const fvh_config* cfg, fvh_handle** out) {
  if (!cfg || !out) {
    g_create_error = "null argument";
    return FVH_ERR_ARG;
  }
  *out = nullptr;
  fvh_handle* h = new (std::nothrow) fvh_handle();
  if (!h) {
    g_create_error = "out of host memory";
    return FVH_ERR_CONFIG;
  }
  std::string msg;
  int st = configure(h, cfg, msg);
  if (!st) st = check_device(cfg, msg);
  if (st) {
    g_create_error = msg;
    delete h;
    return st;
  }
  st = use_device(h);
  if (!st) st = allocate(h);
  if (st) {
    g_create_error = h->err;
    release(h);
    delete h;
    return st;
  }
  *out = h;
  return FVH_OK;
}

int fvh_destroy(fvh_handle* h) {
  if (!h) return FVH_OK;
  release(h);
  delete h;
  return FVH_OK;
}

const char* fvh_last_error(const fvh_handle* h) {
  if (!h) return g_create_error.c_str();
  return h->err.c_str();
}

size_t fvh_scratch_bytes(const fvh_handle* h) { return h ? h->scratch_bytes : 0; }

int fvh_rhs(fvh_handle* h, const double* u, double* dudt, double* dt_out, void* stream) {
  if (!h) return FVH_ERR_ARG;
  if (!u || !dudt) return fail(h, FVH_ERR_ARG, "null array");
  if (int st0 = use_device(h)) return st0;
  cudaStream_t s = (cudaStream_t)stream;
  fvh::StageCall c{};
  c.stage_in = u;
  c.spec.integrator = fvh::INT_RHS;
  c.spec.stage = 0;
  c.spec.stage_in = u;
  c.spec.dudt_out = dudt;
  c.first_stage = 1;
  c.has_target = 0;
  c.log_mode = next_log_mode(h);
  int st = run_stage(h, c, s);
  if (st) return st;
  return read_dt(h, s, dt_out);
}

namespace {

int stage_count(int integrator) {
  switch (integrator) {
    case FVH_INT_EULER: return 1;
    case FVH_INT_SSPRK2: return 2;
    case FVH_INT_SSPRK3: return 3;
    case FVH_INT_RK4: return 4;
    default: return 0;
  }
}

// Stage k of a step of u. Stage inputs: u, then alternating S[0], S[1]; the
// last stage writes u.
int step_stage(fvh_handle* h, double* u, int integrator, int k, int stages, double t, int has_target,
               double target, cudaStream_t s) {
  fvh::StageCall c{};
  const double* in = k == 0 ? u : h->S[(k - 1) & 1];
  if (stages == 1) {
    // A one-stage step writes u in place, while the final pass of a troubled
    // tile reads its stage input in a halo of cells that neighbouring blocks
    // update: the stage reads a copy of u instead.
    const size_t bytes = (size_t)h->nv * h->n[0] * h->n[1] * h->n[2] * sizeof(double);
    if (cudaMemcpyAsync(h->S[1], u, bytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
      return fail(h, FVH_ERR_CUDA, std::string("stage input copy: ") + cudaGetErrorString(cudaGetLastError()));
    in = h->S[1];
  }
  c.stage_in = in;
  c.spec.integrator = integrator;  // FVH_INT_* and fvh::Integrator share values
  c.spec.stage = k;
  c.spec.stage_in = in;
  c.spec.u = u;
  c.spec.acc = h->acc;
  c.spec.next = h->S[k & 1];
  c.first_stage = k == 0;
  c.has_target = has_target;
  c.t = t;
  c.target = target;
  c.log_mode = next_log_mode(h);
  c.log_div = k == stages - 1 ? h->log_divisor : 0.0;
  const int st = run_stage(h, c, s);
  if (st || k == stages - 1) h->log_divisor = 0.0;
  return st;
}

}  // namespace

int fvh_step(fvh_handle* h, double* u, int integrator, double t, int has_target, double target, double* dt_out,
             void* stream) {
  if (!h) return FVH_ERR_ARG;
  if (!u) return fail(h, FVH_ERR_ARG, "null array");
  const int stages = stage_count(integrator);
  if (!stages) return fail(h, FVH_ERR_ARG, "unknown integrator");
  if (int st0 = use_device(h)) return st0;
  cudaStream_t s = (cudaStream_t)stream;
  h->next_stage = 0;
  for (int k = 0; k < stages; ++k)
    if (int st = step_stage(h, u, integrator, k, stages, t, has_target, target, s)) return st;
  return read_dt(h, s, dt_out);
}

int fvh_stage(fvh_handle* h, double* u, int integrator, int k, double t, int has_target, double target,
              double* dt_out, void* stream) {
  if (!h) return FVH_ERR_ARG;
  if (!u) return fail(h, FVH_ERR_ARG, "null array");
  const int stages = stage_count(integrator);
  if (!stages) return fail(h, FVH_ERR_ARG, "unknown integrator");
  if (k < 0 || k >= stages) return fail(h, FVH_ERR_ARG, "stage index out of range for this integrator");
  if (k != 0 && (k != h->next_stage || integrator != h->stage_integrator || u != h->stage_state))
    return fail(h, FVH_ERR_ARG,
                "stage " + std::to_string(k) + " must follow stage " + std::to_string(k - 1) +
                    " of the same integrator and state");
  if (int st0 = use_device(h)) return st0;
  cudaStream_t s = (cudaStream_t)stream;
  h->next_stage = 0;
  if (int st = step_stage(h, u, integrator, k, stages, t, has_target, target, s)) return st;
  h->next_stage = k + 1 < stages ? k + 1 : 0;
  h->stage_integrator = integrator;
  h->stage_state = u;
  return read_dt(h, s, dt_out);
}

int fvh_step_host(fvh_handle* h, double* u_host, int integrator, double t, int has_target, double target,
                  double* dt_out, void* stream) {
  if (!h) return FVH_ERR_ARG;
  if (!u_host) return fail(h, FVH_ERR_ARG, "null array");
  if (int st0 = use_device(h)) return st0;
  if (int st0 = host_path_init(h)) return st0;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t count = (size_t)h->nv * h->n[0] * h->n[1] * h->n[2];
  constexpr int NC = fvh_handle::kHostChunks;
  auto chunk = [&](int j, size_t& off, size_t& len) {
    off = count * j / NC;
    len = count * (j + 1) / NC - off;
  };
  cudaError_t e = cudaSuccess;
  // copy-in: chunk j waits only for chunk j of the previous call's copy-out
  for (int j = 0; j < NC && e == cudaSuccess; ++j) {
    size_t off, len;
    chunk(j, off, len);
    if (h->out_pending) e = cudaStreamWaitEvent(h->copy_in, h->out_done[j], 0);
    if (e == cudaSuccess && len)
      e = cudaMemcpyAsync(h->host_state + off, u_host + off, len * sizeof(double), cudaMemcpyHostToDevice,
                          h->copy_in);
  }
  if (e == cudaSuccess) e = cudaEventRecord(h->in_done, h->copy_in);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(s, h->in_done, 0);
  if (e != cudaSuccess) return fail(h, FVH_ERR_CUDA, std::string("copy-in: ") + cudaGetErrorString(e));
  if (int st = fvh_step(h, h->host_state, integrator, t, has_target, target, nullptr, stream)) return st;
  // copy-out on its own stream, chunk by chunk, each chunk's completion recorded
  e = cudaEventRecord(h->step_done, s);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(h->copy_out, h->step_done, 0);
  for (int j = 0; j < NC && e == cudaSuccess; ++j) {
    size_t off, len;
    chunk(j, off, len);
    if (len)
      e = cudaMemcpyAsync(u_host + off, h->host_state + off, len * sizeof(double), cudaMemcpyDeviceToHost,
                          h->copy_out);
    if (e == cudaSuccess) e = cudaEventRecord(h->out_done[j], h->copy_out);
  }
  if (e != cudaSuccess) return fail(h, FVH_ERR_CUDA, std::string("copy-out: ") + cudaGetErrorString(e));
  h->out_pending = true;
  return read_dt(h, s, dt_out);
}

int fvh_host_sync(fvh_handle* h) {
  if (!h) return FVH_ERR_ARG;
  if (!h->copy_out) return FVH_OK;
  if (int st0 = use_device(h)) return st0;
  const cudaError_t e = cudaStreamSynchronize(h->copy_out);
  if (e != cudaSuccess) return fail(h, FVH_ERR_CUDA, std::string("copy-out: ") + cudaGetErrorString(e));
  return FVH_OK;
}

int fvh_primitives(fvh_handle* h, const double* u, double* w, int fv_average, void* stream) {
  if (!h) return FVH_ERR_ARG;
  if (!u || !w) return fail(h, FVH_ERR_ARG, "null array");
  if (int st0 = use_device(h)) return st0;
  ProfilerBinding bind(h);
  return fvh::primitives_f64(h, u, w, fv_average, (cudaStream_t)stream);
}

int fvh_trouble_flags(fvh_handle* h, uint8_t* flags, void* stream) {
  if (!h) return FVH_ERR_ARG;
  if (!flags) return fail(h, FVH_ERR_ARG, "null array");
  if (!h->trouble) return fail(h, FVH_ERR_CONFIG, "a-posteriori limiting is off");
  if (int st0 = use_device(h)) return st0;
  const size_t n = (size_t)h->n[0] * h->n[1] * h->n[2];
  const cudaError_t e = cudaMemcpyAsync(flags, h->trouble, n, cudaMemcpyDeviceToDevice, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(h, FVH_ERR_CUDA, cudaGetErrorString(e));
  return FVH_OK;
}

int fvh_trouble_log(fvh_handle* h, double divide_by, double* trouble, double* nad_mag, double* pad_mag,
                    void* stream) {
  if (!h) return FVH_ERR_ARG;
  if (!h->logs[0]) return fail(h, FVH_ERR_CONFIG, "trouble logging is off");
  if (int st0 = use_device(h)) return st0;
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t n = (int64_t)h->n[0] * h->n[1] * h->n[2];
  if (divide_by > 0.0) {
    ProfilerBinding bind(h);
    for (int i = 0; i < 3; ++i) {
      fvh::LaunchScope scope(fvh::KK_SMALL, 2.0 * n * sizeof(double), s);
      k_divide<<<(unsigned)std::min<int64_t>((n + 255) / 256, 1 << 20), 256, 0, s>>>(h->logs[i], n, divide_by);
    }
  }
  double* dst[3] = {trouble, nad_mag, pad_mag};
  for (int i = 0; i < 3; ++i) {
    if (!dst[i]) continue;
    const cudaError_t e = cudaMemcpyAsync(dst[i], h->logs[i], n * sizeof(double), cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return fail(h, FVH_ERR_CUDA, cudaGetErrorString(e));
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(h, FVH_ERR_CUDA, cudaGetErrorString(e));
  return FVH_OK;
}

int fvh_set_log_divisor(fvh_handle* h, double divisor) {
  if (!h) return FVH_ERR_ARG;
  if (!(divisor >= 0.0)) return fail(h, FVH_ERR_ARG, "the divisor must be >= 0");
  h->log_divisor = divisor;
  return FVH_OK;
}

int fvh_set_log_mode(fvh_handle* h, int mode) {
  if (!h) return FVH_ERR_ARG;
  if (mode != 1 && mode != 2) return fail(h, FVH_ERR_ARG, "log mode must be 1 or 2");
  h->log_mode_next = mode;
  return FVH_OK;
}

int fvh_get_stats(fvh_handle* h, fvh_stats* out, void* stream) {
  if (!h || !out) return FVH_ERR_ARG;
  if (int st0 = use_device(h)) return st0;
  fvh::Scalars host{};
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(&host, h->sc, sizeof(host), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(h, FVH_ERR_CUDA, cudaGetErrorString(e));
  out->dt_stage = host.dt_stage;
  out->dt_step = host.dt_step;
  out->troubled = host.troubled;
  out->nonfinite = host.nonfinite;
  return FVH_OK;
}

int fvh_boundary_layout(fvh_handle* h, int axis, int side, int* depth, int* ext, size_t* count) {
  if (!h) return FVH_ERR_ARG;
  if (axis < 0 || axis > 2 || side < 0 || side > 1) return fail(h, FVH_ERR_ARG, "axis must be 0..2, side 0..1");
  if (!h->slab[axis][side]) return fail(h, FVH_ERR_CONFIG, "that side is not a Dirichlet boundary");
  const fvh::Slabs& m = h->slab_meta;
  if (depth) *depth = m.depth[axis];
  if (ext)
    for (int b = 0; b < 3; ++b) ext[b] = b == axis ? m.depth[b] : h->n[b] + 2 * m.pad[b];
  if (count) *count = h->slab_count[axis][side];
  return FVH_OK;
}

int fvh_set_boundary_values(fvh_handle* h, int axis, int side, const double* values, void* stream) {
  if (!h) return FVH_ERR_ARG;
  if (axis < 0 || axis > 2 || side < 0 || side > 1 || !values)
    return fail(h, FVH_ERR_ARG, "axis must be 0..2, side 0..1, values non-null");
  if (!h->slab[axis][side]) return fail(h, FVH_ERR_CONFIG, "that side is not a Dirichlet boundary");
  if (int st0 = use_device(h)) return st0;
  const cudaError_t e = cudaMemcpyAsync(h->slab[axis][side], values, h->slab_count[axis][side] * sizeof(double),
                                        cudaMemcpyDefault, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(h, FVH_ERR_CUDA, cudaGetErrorString(e));
  return FVH_OK;
}

int fvh_get_pred_stats(fvh_handle* h, fvh_pred_stats* out, void* stream) {
  if (!h || !out) return FVH_ERR_ARG;
  if (int st0 = use_device(h)) return st0;
  fvh::Scalars host{};
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(&host, h->sc, sizeof(host), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(h, FVH_ERR_CUDA, cudaGetErrorString(e));
  out->predicted = host.predicted;
  out->troubled = host.judged;
  out->missed = host.missed;
  out->false_alarm = host.false_alarm;
  out->revised_faces = host.revised_faces;
  out->flux_fallback_faces = host.flux_fallback_faces;
  return FVH_OK;
}

int fvh_pred_flags(fvh_handle* h, uint8_t* flags, void* stream) {
  if (!h) return FVH_ERR_ARG;
  if (!flags) return fail(h, FVH_ERR_ARG, "null array");
  if (!h->pred) return fail(h, FVH_ERR_CONFIG, "no predictor was attached");
  if (int st0 = use_device(h)) return st0;
  const size_t n = (size_t)h->n[0] * h->n[1] * h->n[2];
  const cudaError_t e = cudaMemcpyAsync(flags, h->pred, n, cudaMemcpyDeviceToDevice, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(h, FVH_ERR_CUDA, cudaGetErrorString(e));
  return FVH_OK;
}

uint64_t fvh_kernel_launches(void) { return fvh::launch_counter().load(); }

int fvh_profile_enable(fvh_handle* h, int on) {
  if (!h) return FVH_ERR_ARG;
  if (int st0 = use_device(h)) return st0;
  if (on && !h->prof) h->prof = new (std::nothrow) fvh::Profiler();
  if (!on) {
    delete h->prof;
    h->prof = nullptr;
    h->prof_totals = fvh::KernelTotals{};
  }
  return FVH_OK;
}

int fvh_profile_read(fvh_handle* h, double* ms, double* bytes, uint64_t* launches, void* stream) {
  if (!h) return FVH_ERR_ARG;
  if (!h->prof) return fail(h, FVH_ERR_CONFIG, "profiling is off");
  if (int st0 = use_device(h)) return st0;
  const cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) return fail(h, FVH_ERR_CUDA, cudaGetErrorString(e));
  if (h->prof->collect(h->prof_totals)) return fail(h, FVH_ERR_CUDA, "reading profiling events");
  for (int k = 0; k < fvh::KK_COUNT; ++k) {
    if (ms) ms[k] = h->prof_totals.ms[k];
    if (bytes) bytes[k] = h->prof_totals.bytes[k];
    if (launches) launches[k] = h->prof_totals.launches[k];
  }
  h->prof_totals = fvh::KernelTotals{};
  return FVH_OK;
}

}  // extern "C"
