// Learned troubled-cell predictor: a 100 -> 64 -> 64 -> 1 GELU network over
// the 5x5 neighbourhood of (rho, v_X, v_Y, P) around each cell of a 2D grid.
//
// Features (computed from the stage's FV primitives W): for each variable v
// and offset (a, b) in [-2, 2]^2, d = W_v(x+a, y+b) - W_v(x, y) and
//   f = sign(d) log1p(|d| / (eps R_v)) / log1p(1 / eps),   eps = 1e-5,
// where R_v is the variable's global range over the stage (the same extrema the
// global NAD test uses); index v*25 + (a+2)*5 + (b+2); 12 zero columns pad the
// row to K = 112.
//
// Layers run on the tensor cores (tcgen05.mma, BF16 operands, FP32
// accumulators in TMEM) in tiles of 128 rows, one row per thread, so thread t
// owns TMEM lane t. Parameters are kept in FP32 (W1[64][100] and W2[64][64]
// stored output-major, then b1, b2, w3[64], b3); the kernels read BF16 images
// of the weight matrices in the shared-memory operand layout.
#pragma once

#include <cuda_bf16.h>

#include "fvh_tc.cuh"

namespace fvh {
namespace mlp {

constexpr int kIn = 100;       // features
constexpr int kInPad = 112;    // K of the first layer, a multiple of 16
constexpr int kHidden = 64;
constexpr int kRows = 128;     // rows per tile (MMA M)
constexpr float kEps = 1e-5f;  // feature compression scale

// FP32 parameter offsets
constexpr int kW1 = 0;
constexpr int kB1 = kW1 + kHidden * kIn;
constexpr int kW2 = kB1 + kHidden;
constexpr int kB2 = kW2 + kHidden * kHidden;
constexpr int kW3 = kB2 + kHidden;
constexpr int kB3 = kW3 + kHidden;
constexpr int kParams = kB3 + 1;

// BF16 weight images (bytes)
constexpr int kImgB1 = kHidden * kInPad * 2;    // W1 as N = 64 x K = 112
constexpr int kImgB2 = kHidden * kHidden * 2;   // W2 as N = j x K = i (forward)
constexpr int kImgB2t = kHidden * kHidden * 2;  // W2 as N = i x K = j (backward)
constexpr int kImgBytes = kImgB1 + kImgB2 + kImgB2t;

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * __expf(-0.5f * x * x);
  return cdf + x * pdf;
}

__device__ __forceinline__ void store_bf16(unsigned char* tile, uint32_t off, float v) {
  *reinterpret_cast<__nv_bfloat16*>(tile + off) = __float2bfloat16_rn(v);
}
__device__ __forceinline__ float load_bf16(const unsigned char* tile, uint32_t off) {
  return __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(tile + off));
}

// Feature vector of the cell at offset o of a 2D primitive array (row stride
// sx, variable stride vs); vid = primitive indices of (rho, v_X, v_Y, P),
// inv_s[v] = 1 / (eps R_v).
template <typename Tw>
__device__ __forceinline__ void cell_features(const Tw* __restrict__ W, int sx, int vs, int o, const int* vid,
                                              const float* inv_s, float* f) {
  const float norm = 1.0f / log1pf(1.0f / kEps);
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    const Tw* base = W + vid[v] * vs + o;
    const Tw c = base[0];
#pragma unroll
    for (int a = -2; a <= 2; ++a)
#pragma unroll
      for (int b = -2; b <= 2; ++b) {
        const float d = (float)(base[a * sx + b] - c);  // difference in the precision of W
        const float m = log1pf(fabsf(d) * inv_s[v]) * norm;
        f[v * 25 + (a + 2) * 5 + (b + 2)] = d < 0.0f ? -m : m;
      }
  }
}

}  // namespace mlp
}  // namespace fvh
