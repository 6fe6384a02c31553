// Optional per-kernel timing of the stage runners.
//
// Every launch in the library goes through a LaunchScope: it counts the
// launch and, when the calling thread has an active Profiler, records a CUDA
// event pair around it together with the kernel kind and the bytes the launch
// must move (each input element read once, each output element written once).
// Profiler::collect synchronises and folds the pairs into per-kind totals.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <vector>

namespace fvh {

enum KernelKind : int {
  KK_CENTRE = 0,     // centre-interpolation sweep (incl. ghost fill / primitives)
  KK_TRANSVERSE,     // transverse-reconstruction sweep (incl. reductions)
  KK_FACE,           // face states + Riemann solve
  KK_CANDIDATE,      // candidate update u*
  KK_DETECT,         // troubled-cell detection
  KK_FALLBACK,       // MUSCL fallback + blend
  KK_FINAL,          // divergence + Runge-Kutta combination
  KK_SMALL,          // scalars, convex weights, log arithmetic
  KK_PREDICT,        // learned troubled-cell predictor
  KK_COUNT
};

struct KernelTotals {
  double ms[KK_COUNT];
  double bytes[KK_COUNT];
  uint64_t launches[KK_COUNT];
};

class Profiler {
 public:
  ~Profiler();
  void record_begin(int kind, double bytes, cudaStream_t s);
  void record_end(cudaStream_t s);
  // Synchronises, adds the recorded pairs to `totals` and recycles the events.
  int collect(KernelTotals& totals);

 private:
  struct Pair {
    cudaEvent_t a, b;
    int kind;
    double bytes;
  };
  std::vector<Pair> used_;
  std::vector<Pair> pool_;
  std::vector<size_t> open_;  // indices into used_ of the scopes still open (nested scopes allowed)
};

// Profiler of the calling thread (nullptr when profiling is off).
Profiler*& active_profiler();
// Total kernel launches issued by this library in the process.
std::atomic<uint64_t>& launch_counter();

struct LaunchScope {
  cudaStream_t s;
  bool on;
  LaunchScope(int kind, double bytes, cudaStream_t stream) : s(stream), on(active_profiler() != nullptr) {
    launch_counter().fetch_add(1, std::memory_order_relaxed);
    if (on) active_profiler()->record_begin(kind, bytes, s);
  }
  ~LaunchScope() {
    if (on) active_profiler()->record_end(s);
  }
};

}  // namespace fvh
