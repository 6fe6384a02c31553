// Tile staging through the Tensor Memory Accelerator (sm_100a): one thread
// issues a 3D bulk tensor copy of a (variables x rows x columns) box of a
// variable-major array from this GPU's global memory into shared memory, and
// the block waits on an mbarrier for its bytes. No cluster multicast is used.
//
// Rules the callers keep (checked on the host where they can be):
//  - the array's base is 16-byte aligned, its row and variable strides are
//    multiples of 16 bytes, and the box's inner extent is a multiple of 16
//    bytes (cuTensorMapEncodeTiled refuses the map otherwise);
//  - the box's innermost start coordinate times the element size is a
//    multiple of 16 bytes (nothing checks this before the copy runs, so every
//    caller derives it from 16-byte aligned quantities only);
//  - a load may start at or run past the array's end on the outer axes: those
//    elements read as zero;
//  - the shared-memory destination is 128-byte aligned: kernels round their
//    dynamic shared memory up to it at run time (align128), since static
//    shared variables placed before it (their mbarriers) shift its start.
// Each copy checks the destination's and the inner coordinate's alignment
// before it is issued; a copy that fails the check is not issued, counts into
// an error word and is not waited for.
// Waits are bounded (2^20 polls): a wait that runs out counts into an error
// word, then the block waits again (2^22 polls) for the copy it issued, so that the copy does
// not land in shared memory after the block has moved on or exited.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace fvh {
namespace tma {

constexpr uint32_t kWaitPolls = 1u << 20, kDrainPolls = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool wait_bounded(uint64_t* bar, uint32_t parity, uint32_t max_polls) {
  for (uint32_t i = 0; i < max_polls; ++i)
    if (try_wait(bar, parity)) return true;
  return false;
}

// Box (c0, c1, c2) of a 3D tensor map (c0 innermost) into shared memory at dst,
// completing on bar.
__device__ __forceinline__ void load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}

// The first 128-byte boundary at or after p (dynamic shared memory requests
// carry 128 spare bytes for it).
__device__ __forceinline__ unsigned char* align128(unsigned char* p) {
  return p + ((128u - (smem_u32(p) & 127u)) & 127u);
}

// Whether a box copy to dst starting at inner coordinate c0 (elements of
// elem bytes) meets the alignment rules above.
__device__ __forceinline__ bool copy_aligned(const void* dst, int c0, int elem) {
  return (smem_u32(dst) & 127u) == 0 && ((long long)c0 * elem) % 16 == 0;
}

// Whole block: stages the box at (c0, c1, c2) of map into dst (bytes = the
// box's size) through bar, which this call initialises (one use per barrier
// and kernel). Returns false in every thread when the copy was refused for
// its alignment or its wait ran out (the error word is raised once per block).
__device__ __forceinline__ bool stage_box(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint32_t bytes,
                                          int elem, uint64_t* bar, unsigned int* err) {
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  int refused = 0;
  if (threadIdx.x == 0) {
    if (copy_aligned(dst, c0, elem)) {
      arrive_expect_tx(bar, bytes);
      load_3d(dst, map, c0, c1, c2, bar);
    } else {
      refused = 1;
      atomicAdd(err, 1u);
    }
  }
  if (__syncthreads_or(refused)) return false;
  const bool ok = wait_bounded(bar, 0, kWaitPolls);
  const bool all_ok = __syncthreads_or(ok ? 0 : 1) == 0;
  if (!all_ok) {
    wait_bounded(bar, 0, kDrainPolls);  // drain: the copy must land before the block moves on
    if (threadIdx.x == 0) atomicAdd(err, 1u);
    __syncthreads();
  }
  return all_ok;
}

}  // namespace tma

// Host: a 3D tiled tensor map over a variable-major array of nv planes of
// rows x cols elements of elem bytes (row stride sx elements, plane stride vs
// elements), box (box_cols, box_rows, box_vars). Returns false (with a
// message) when the driver refuses it. Defined in fvh_api.cu.
bool encode_tensor_map_3d(CUtensorMap* map, const void* base, int elem, int cols, int rows, int nv, int sx, int vs,
                          int box_cols, int box_rows, int box_vars, const char** why);

}  // namespace fvh
