// Thin wrappers over the sm_100a tensor-core instructions used by the learned
// troubled-cell predictor: tcgen05.mma (kind::f16, BF16 x BF16 -> FP32, one
// CTA), TMEM allocation and loads, mbarrier completion tracking.
//
// Operand tiles live in shared memory in the K-major, non-swizzled canonical
// layout: 8-row x 8-element core matrices of 128 contiguous bytes (row r of a
// core matrix at byte 16 r), core matrices of consecutive 8-row groups 128 B
// apart (stride byte offset), core matrices of consecutive 8-element K chunks
// (rows/8) * 128 B apart (leading byte offset). One MMA consumes K = 16.
// The accumulator of an M = 128 MMA occupies TMEM lanes 0..127 (row m in lane
// m) and N consecutive 32-bit columns; warp w of the CTA reads lanes
// 32w..32w+31 with tcgen05.ld.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace fvh {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Byte offset of element (row, k) in a K-major canonical tile with `rows` rows.
__device__ __forceinline__ uint32_t kmajor_offset(int row, int k, int rows) {
  return (uint32_t)((((k >> 3) * (rows >> 3) + (row >> 3)) << 7) + ((row & 7) << 4) + ((k & 7) << 1));
}

// Shared-memory matrix descriptor: start address, leading / stride byte
// offsets (all >> 4), version 1, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Descriptor of the K slice [16 j, 16 j + 16) of a K-major tile with `rows` rows.
__device__ __forceinline__ uint64_t kslice_desc(uint32_t tile_saddr, int rows, int j) {
  const uint32_t chunk = (uint32_t)(rows >> 3) << 7;  // bytes between K chunks
  return smem_desc(tile_saddr + 2u * (uint32_t)j * chunk, chunk, 128u);
}

// Instruction descriptor: BF16 A and B, FP32 accumulator, both K-major, M = 128.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Makes this thread's generic-proxy shared-memory writes visible to the tensor cores.
__device__ __forceinline__ void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
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

// Waits for the given phase parity with a bounded number of polls; returns
// false (and leaves the decision to the caller) when the bound is reached.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t max_polls = 1u << 26) {
  for (uint32_t i = 0; i < max_polls; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// TMEM allocation: executed by one whole warp; the base address is written to *dst.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive FP32 accumulator columns of this thread's lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* out) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) out[i] = __uint_as_float(r[i]);
}

}  // namespace tc
}  // namespace fvh
