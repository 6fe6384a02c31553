// Learned troubled-cell predictor: a 100 -> 64 -> 64 -> 1 network with GELU
// (tanh form) activations over the 5x5 neighbourhood of (rho, v_X, v_Y, P)
// around each cell of a 2D grid.
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

// GELU in its tanh form, 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3)))
// (Hendrycks & Gimpel, "Gaussian Error Linear Units", 2016), with the
// hardware tanh approximation (tanh.approx.f32, absolute error near 2^-11,
// below the BF16 rounding of the activations).
__device__ __forceinline__ float tanh_approx(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
constexpr float kGeluC = 0.7978845608028654f;  // sqrt(2 / pi)
constexpr float kGeluA = 0.044715f;
__device__ __forceinline__ float gelu(float x) {
  const float t = tanh_approx(kGeluC * fmaf(kGeluA * x, x * x, x));
  return 0.5f * x * (1.0f + t);
}
// 2 gelu(x), rounded exactly as gelu(x) and doubled (the inference kernel keeps
// doubled activations: a power-of-two scale that BF16 and FP32 carry exactly)
__device__ __forceinline__ float gelu2(float x) {
  const float t = tanh_approx(kGeluC * fmaf(kGeluA * x, x * x, x));
  return x * (1.0f + t);
}
__device__ __forceinline__ float gelu_grad(float x) {
  const float t = tanh_approx(kGeluC * fmaf(kGeluA * x, x * x, x));
  return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * kGeluC * fmaf(3.0f * kGeluA, x * x, 1.0f);
}

__device__ __forceinline__ void store_bf16(unsigned char* tile, uint32_t off, float v) {
  *reinterpret_cast<__nv_bfloat16*>(tile + off) = __float2bfloat16_rn(v);
}
__device__ __forceinline__ float load_bf16(const unsigned char* tile, uint32_t off) {
  return __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(tile + off));
}
// Eight floats as eight BF16 values (round to nearest even), first at the lowest address.
__device__ __forceinline__ uint4 pack_bf16x8(const float* v) {
  uint4 q;
  uint32_t* w = reinterpret_cast<uint32_t*>(&q);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    w[i] = *reinterpret_cast<const uint32_t*>(&h);
  }
  return q;
}

// Features [8 C, 8 C + 8) of the cell at offset o of a 2D primitive array (row
// stride sx, variable stride vs), packed as BF16; vid = primitive indices of
// (rho, v_X, v_Y, P), inv_s[v] = 1 / (eps R_v). Feature k = v*25 + (a+2)*5 +
// (b+2) is sign(d) ln(1 + |d| inv_s) / ln(1 + 1/eps) with d = w(x+a, y+b) -
// w(x, y) taken in the precision of W; k >= 100 is zero.
template <typename Tw, int C>
__device__ __forceinline__ uint4 feature_chunk(const Tw* __restrict__ W, int sx, int vs, int o, const int* vid,
                                               const float* inv_s) {
  constexpr float kNorm2 = 0.060205946838836726f;  // ln 2 / ln(1 + 1e5): log2 scaled to the normalised log
  float f[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int k = 8 * C + i;
    if (k >= kIn) {
      f[i] = 0.0f;
      continue;
    }
    const int v = k / 25, a = (k % 25) / 5 - 2, b = (k % 5) - 2;
    const Tw* base = W + vid[v] * vs + o;
    const float d = (float)(base[a * sx + b] - base[0]);
    const float m = __log2f(fmaf(fabsf(d), inv_s[v], 1.0f)) * kNorm2;
    f[i] = d < 0.0f ? -m : m;
  }
  return pack_bf16x8(f);
}

// All 14 chunks of a cell's feature row, handed to store(c, chunk).
template <typename Tw, int C = 0, typename Store>
__device__ __forceinline__ void feature_row(const Tw* __restrict__ W, int sx, int vs, int o, const int* vid,
                                            const float* inv_s, Store&& store) {
  if constexpr (C < kInPad / 8) {
    store(C, feature_chunk<Tw, C>(W, sx, vs, o, vid, inv_s));
    feature_row<Tw, C + 1>(W, sx, vs, o, vid, inv_s, store);
  }
}

}  // namespace mlp
}  // namespace fvh
