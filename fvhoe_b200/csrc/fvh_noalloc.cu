// Allocation-free variant of fvh_primitives (declared in include/fvh.h).
//
// Some callers cannot allocate device memory at the moment they need this
// conversion: a host application that owns the device's memory pool and
// forbids outside allocations, or a simulation that has already committed the
// whole device to its state and must not fail later on an out-of-memory
// cudaMalloc. For them, fvh_primitives_noalloc runs the same primitive pass as
// fvh_primitives without a handle, taking its two sweep buffers from the
// static device array below instead of from fvh_create's allocations.
//
// Limits and sharing rules:
//  - The array holds kNoAllocScratchDoubles doubles (16 MiB) on every GPU that
//    loads this library, until the process exits. Grids whose sweep boxes do
//    not fit (see fvh_primitives_noalloc_max_doubles) are refused.
//  - Every call shares the array and leaves its last contents behind. The
//    primitive pass writes every scratch element before reading it, so nothing
//    needs clearing between calls; but two calls whose work overlaps on the GPU
//    (different streams, or different host threads) race on the array.
//  - The first call on a device resolves the array's device address with
//    cudaGetSymbolAddress, with that device current; make that first call
//    before any stream capture. The address is kept for the life of the
//    process: after cudaDeviceReset (which also frees every handle's memory)
//    the module may load at another address, so this library must not be
//    used across a device reset.
//  - Every refusal (null arguments, configuration, boundary kinds, device
//    ordinal, grid size) is decided on the host before any CUDA call, and
//    before the state pointers are used.
//
// Compiled with -fmad=false like the FP64 stage runner, so the results equal
// fvh_primitives (and the reference) bit for bit.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "fvh_stage.cuh"

namespace {

constexpr size_t kNoAllocScratchDoubles = size_t(2) << 20;  // 2 Mi doubles = 16 MiB
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

std::mutex g_setup_mutex;
double* g_scratch_address[kMaxDevices] = {};

thread_local char g_noalloc_error[256] = "";

int set_error(int code, const char* msg) {
  std::snprintf(g_noalloc_error, sizeof(g_noalloc_error), "%s", msg);
  return code;
}

// Device address of the static scratch on `device`, resolved once per device
// with that device current.
int scratch_address(int device, double** out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_address[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      cudaGetLastError();
      std::snprintf(g_noalloc_error, sizeof(g_noalloc_error), "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
      return FVH_ERR_CUDA;
    }
    g_scratch_address[device] = static_cast<double*>(p);
  }
  *out = g_scratch_address[device];
  return FVH_OK;
}

}  // namespace

namespace fvh {
int configure_handle(fvh_handle* h, const fvh_config* cfg, std::string& msg);
int check_device_visible(const fvh_config* cfg, std::string& msg);
}

extern "C" {

size_t fvh_primitives_noalloc_max_doubles(void) { return kNoAllocScratchDoubles / 2; }

const char* fvh_primitives_noalloc_error(void) { return g_noalloc_error; }

int fvh_primitives_noalloc(const fvh_config* cfg, const double* u, double* w, int fv_average, void* stream) {
  if (!cfg) return set_error(FVH_ERR_ARG, "null configuration");
  fvh_handle h;  // host-side geometry only; no device memory behind it
  std::string msg;
  const int st = fvh::configure_handle(&h, cfg, msg);
  if (st) return set_error(st, msg.c_str());
  if (h.cfg.device < 0 || h.cfg.device >= kMaxDevices)
    return set_error(FVH_ERR_CONFIG, "device ordinal out of range [0, 64)");
  for (int a = 0; a < 3; ++a)
    for (int side = 0; side < 2; ++side)
      if (h.active[a] && (cfg->bc[a][side] == FVH_BC_DIRICHLET || cfg->bc[a][side] == FVH_BC_DMR_Y0))
        return set_error(FVH_ERR_CONFIG,
                         "Dirichlet and double-Mach-reflection boundaries need a handle (fvh_primitives)");
  // per-buffer requirement: the state ghost-filled by 2r on each active axis
  size_t need = (size_t)h.nv;
  for (int a = 0; a < 3; ++a) need *= (size_t)(h.n[a] + (h.active[a] ? 4 * h.r[a] : 0));
  const size_t limit = kNoAllocScratchDoubles / 2;
  if (need > limit) {
    std::snprintf(g_noalloc_error, sizeof(g_noalloc_error),
                  "grid too large for the allocation-free conversion: each of its two sweep buffers needs %zu "
                  "doubles, the static scratch holds %zu per buffer",
                  need, limit);
    return FVH_ERR_CONFIG;
  }
  if (!u || !w) return set_error(FVH_ERR_ARG, "null state or output array");
  if (int sd = fvh::check_device_visible(cfg, msg)) return set_error(sd, msg.c_str());
  cudaError_t e = cudaSetDevice(h.cfg.device);
  if (e != cudaSuccess) return set_error(FVH_ERR_CUDA, cudaGetErrorString(e));
  double* base = nullptr;
  if (int s2 = scratch_address(h.cfg.device, &base)) return s2;
  h.bufA = base;
  h.bufB = base + limit;
  h.buf_elems = limit;
  const int r = fvh::primitives_f64(&h, u, w, fv_average, (cudaStream_t)stream);
  h.bufA = h.bufB = nullptr;  // not owned
  if (r) return set_error(r, h.err.c_str());
  g_noalloc_error[0] = '\0';
  return FVH_OK;
}

}  // extern "C"
