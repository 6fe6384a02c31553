// Learned troubled-cell predictor: tensor-core kernels (tcgen05) for
// inference and training, the feature extraction, and their C ABI
// (include/fvh.h). See fvh_mlp.cuh for the network and feature definitions.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>
#include <random>
#include <string>
#include <vector>

#include "fvh_handle.h"
#include "fvh_mlp.cuh"

using namespace fvh;
using namespace fvh::mlp;

struct fvh_mlp {
  int device = 0;
  float* params = nullptr;  // FP32 master parameters
  float* grads = nullptr;
  float* m = nullptr;       // Adam moments
  float* v = nullptr;
  unsigned char* img = nullptr;  // BF16 weight images
  float* loss = nullptr;         // device loss sum
  unsigned int* err = nullptr;   // device error counter (bounded waits that gave up)
  int step = 0;
  std::string errmsg;
};

namespace {

thread_local std::string g_mlp_error;

// inference tile: features (the first layer's operand, then the second's), images, FP32 vectors
constexpr int kPredictSmem = kRows * kInPad * 2 + kImgB1 + kImgB2 + 256 * 4;

// Training tile layout (bytes of dynamic shared memory). Operands of the
// forward GEMMs (rows = samples), of dh1 = dz2 W2, and of the weight-gradient
// GEMMs, which contract over the 128 samples of the tile:
//   dW1^T (128 x 64) += X^T (128 features x 128 samples) . dz1^T (64 x 128)
//   dW2^T (128 x 64) += h1^T (128 x 128 samples)         . dz2^T (64 x 128)
// Feature row 112 of X^T and unit row 64 of h1^T are all ones, so the same
// products also accumulate the bias gradients sum_q dz1 and sum_q dz2.
namespace tl {
constexpr int XA = 0;                          // X, 128 x 112
constexpr int XT = XA + kRows * kInPad * 2;    // X^T, 128 x 128
constexpr int H1 = XT + kRows * kRows * 2;     // h1, 128 x 64
constexpr int H1T = H1 + kRows * kHidden * 2;  // h1^T, 128 x 128
constexpr int DZ2 = H1T + kRows * kRows * 2;   // dz2, 128 x 64
constexpr int DZ2T = DZ2 + kRows * kHidden * 2;  // dz2^T, 64 x 128
constexpr int DZ1T = DZ2T + kHidden * kRows * 2; // dz1^T, 64 x 128
constexpr int IMG = DZ1T + kHidden * kRows * 2;  // B1, B2, B2t images
constexpr int PB = IMG + kImgBytes;             // b1, b2, w3, b3 (FP32)
constexpr int GW3 = PB + 256 * 4;               // w3 gradient partials [64][128] (FP32)
constexpr int BYTES = GW3 + kHidden * kRows * 4;
constexpr int kOnesX = kInPad;  // row of ones in X^T
constexpr int kOnesH = kHidden; // row of ones in h1^T
}  // namespace tl
constexpr int kTrainSmem = tl::BYTES;
static_assert(kTrainSmem <= 227 * 1024, "training tile exceeds shared memory");

// TMEM columns of the training kernel
constexpr int kColD1 = 0, kColD2 = 64, kColDH = 128, kColGW1 = 192, kColGW2 = 256, kTrainCols = 512;

// Issues D (+)= A (128 x K) B^T (N x K) over K/16 slices (thread 0 only).
__device__ __forceinline__ void issue_gemm(uint32_t tmem_d, const void* a, const void* b, int K, int N,
                                           bool accumulate) {
  const uint32_t idesc = tc::idesc_bf16_f32(N);
  const uint32_t as = tc::smem_u32(a), bs = tc::smem_u32(b);
  for (int j = 0; j < K / 16; ++j)
    tc::mma_bf16(tmem_d, tc::kslice_desc(as, kRows, j), tc::kslice_desc(bs, N, j), idesc,
                 (accumulate || j > 0) ? 1u : 0u);
}

// All threads: publish shared-memory operands and pass the barrier; thread 0
// then issues through the tensor-core proxy.
__device__ __forceinline__ bool publish_operands() {
  tc::fence_smem_to_async();
  tc::fence_before_sync();
  __syncthreads();
  if (threadIdx.x != 0) return false;
  tc::fence_after_sync();
  return true;
}

// All threads: wait (bounded) for the GEMMs committed to bar. Returns false in
// every thread of the block when any thread gave up; the caller then stops
// issuing and releases TMEM (the error counter tells the host).
//
// Give-up path: a commit whose wait ran out may still be executing, and its
// MMAs write TMEM and its completion arrives on `bar` in this CTA's shared
// memory. Releasing TMEM (or ending the CTA, which hands its shared memory to
// the next CTA) before they land would let them write memory that is no
// longer this CTA's. So on a give-up every thread first drains: it waits
// again, with a 16x longer bound, for the same phase. Once that phase has
// completed no MMA of this CTA is in flight (each commit tracks all MMAs the
// thread issued before it, and nothing is issued after a give-up), and the
// release is safe. If the drain runs out too, the block still releases and
// returns, so the kernel ends instead of hanging, and the second count tells
// the host that the last commit never completed.
__device__ __forceinline__ bool wait_gemms(uint64_t* bar, uint32_t& phase, unsigned int* err) {
  const bool ok = tc::mbar_wait_bounded(bar, phase, 1u << 22);
  if (!ok) atomicAdd(err, 1u);
  const bool all_ok = __syncthreads_or(ok ? 0 : 1) == 0;
  if (!all_ok) {
    const bool drained = tc::mbar_wait_bounded(bar, phase, 1u << 26);
    if (!drained && threadIdx.x == 0) atomicAdd(err, 1u);
    __syncthreads();
  }
  phase ^= 1u;
  tc::fence_after_sync();
  return all_ok;
}

__device__ __forceinline__ bool run_gemm(uint32_t tmem_d, const void* a, const void* b, int K, int N, uint64_t* bar,
                                         uint32_t& phase, unsigned int* err) {
  if (publish_operands()) {
    issue_gemm(tmem_d, a, b, K, N, false);
    tc::mma_commit(bar);
  }
  return wait_gemms(bar, phase, err);
}

// 64 accumulator columns of this thread's row, starting at column col.
__device__ __forceinline__ void load_row64(uint32_t tmem_base, int col, float* out) {
  const uint32_t lane = (uint32_t)(threadIdx.x & ~31) << 16;
#pragma unroll
  for (int c = 0; c < 4; ++c) tc::tmem_ld16(tmem_base + lane + (uint32_t)(col + 16 * c), out + 16 * c);
}

__device__ __forceinline__ void copy_bytes(unsigned char* dst, const unsigned char* src, int bytes) {
  const uint4* s = reinterpret_cast<const uint4*>(src);
  uint4* d = reinterpret_cast<uint4*>(dst);
  for (int i = threadIdx.x; i < bytes / 16; i += blockDim.x) d[i] = s[i];
}

__device__ __forceinline__ void block_tmem_setup(uint32_t* tmem_slot, uint64_t* bar, uint32_t ncols = 128) {
  if (threadIdx.x == 0) tc::mbar_init(bar, 1);
  if (threadIdx.x < 32) tc::tmem_alloc(tmem_slot, ncols);
  tc::fence_smem_to_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
}

__device__ __forceinline__ void block_tmem_release(uint32_t tmem_base, uint32_t ncols = 128) {
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (threadIdx.x < 32) tc::tmem_dealloc(tmem_base, ncols);
}

// ---------------------------------------------------------------------------
// Inference inside a stage: prediction flags of every interior cell from the
// stage's FV primitives W (2D view with g ghosts).
// ---------------------------------------------------------------------------
template <typename Tw>
__global__ void __launch_bounds__(128, 4)
    k_mlp_predict(const Tw* __restrict__ W, int g, int gy, int sx, int vs, int nx, int ny, int4 vid4,
                  const Scalars* __restrict__ sc,
                  const unsigned char* __restrict__ img, const float* __restrict__ params, float thr_logit,
                  uint8_t* __restrict__ pred, unsigned int* __restrict__ err) {
  extern __shared__ __align__(128) unsigned char sm[];
  unsigned char* A = sm;
  // h1 reuses the feature tile: the first GEMM has completed when it is written,
  // and the second has completed before the next tile's features are
  unsigned char* A2 = A;
  unsigned char* B1 = A + kRows * kInPad * 2;
  unsigned char* B2 = B1 + kImgB1;
  float* pb = reinterpret_cast<float*>(B2 + kImgB2);  // b1, b2, w3, b3
  __shared__ uint64_t bar;
  __shared__ uint32_t tmem_slot;
  copy_bytes(B1, img, kImgB1 + kImgB2);
  // the hidden layers carry doubled activations (gelu2): the second layer's
  // accumulator is halved in its bias FMA and w3 is stored halved, so every
  // value equals the plain forward pass bit for bit
  for (int i = threadIdx.x; i < kHidden; i += blockDim.x) {
    pb[i] = params[kB1 + i];
    pb[64 + i] = params[kB2 + i];
    pb[128 + i] = 0.5f * params[kW3 + i];
  }
  if (threadIdx.x == 0) pb[192] = params[kB3];
  block_tmem_setup(&tmem_slot, &bar);
  const uint32_t tb = tmem_slot;
  const int vid[4] = {vid4.x, vid4.y, vid4.z, vid4.w};
  float inv_s[4];
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    const double range = key_value(sc->vmax_key[vid[v]]) - key_value(sc->vmin_key[vid[v]]);
    inv_s[v] = (float)(1.0 / ((double)kEps * (range > 0.0 ? range : 1.0)));
  }
  const int ncell = nx * ny;
  const int r = threadIdx.x;
  const uint32_t lane = (uint32_t)(threadIdx.x & ~31) << 16;
  uint32_t phase = 0;
  for (int tile = blockIdx.x; tile * kRows < ncell; tile += gridDim.x) {
    const int cell = tile * kRows + r;
    const bool valid = cell < ncell;
    // features straight into the operand tile, one 16-byte row of a core matrix per chunk
    if (valid) {
      const int x = cell / ny, y = cell - (cell / ny) * ny;
      feature_row<Tw>(W, sx, vs, (x + g) * sx + (y + gy), vid, inv_s, [&](int c, uint4 q) {
        *reinterpret_cast<uint4*>(A + tc::kmajor_offset(r, 8 * c, kRows)) = q;
      });
    } else {
#pragma unroll
      for (int c = 0; c < kInPad / 8; ++c)
        *reinterpret_cast<uint4*>(A + tc::kmajor_offset(r, 8 * c, kRows)) = make_uint4(0u, 0u, 0u, 0u);
    }
    if (!run_gemm(tb, A, B1, kInPad, kHidden, &bar, phase, err)) break;
#pragma unroll
    for (int c = 0; c < kHidden / 16; ++c) {
      float h[16];
      tc::tmem_ld16(tb + lane + (uint32_t)(16 * c), h);
#pragma unroll
      for (int j = 0; j < 16; ++j) h[j] = gelu2(h[j] + pb[16 * c + j]);
      *reinterpret_cast<uint4*>(A2 + tc::kmajor_offset(r, 16 * c, kRows)) = pack_bf16x8(h);
      *reinterpret_cast<uint4*>(A2 + tc::kmajor_offset(r, 16 * c + 8, kRows)) = pack_bf16x8(h + 8);
    }
    if (!run_gemm(tb + 64, A2, B2, kHidden, kHidden, &bar, phase, err)) break;
    float logit = pb[192];
#pragma unroll
    for (int c = 0; c < kHidden / 16; ++c) {
      float h[16];
      tc::tmem_ld16(tb + lane + (uint32_t)(64 + 16 * c), h);
#pragma unroll
      for (int j = 0; j < 16; ++j)
        logit = fmaf(gelu2(fmaf(h[j], 0.5f, pb[64 + 16 * c + j])), pb[128 + 16 * c + j], logit);
    }
    if (valid) pred[cell] = logit > thr_logit ? 1 : 0;
    tc::fence_before_sync();
    __syncthreads();
  }
  block_tmem_release(tb);
}

// ---------------------------------------------------------------------------
// Training (and evaluation) over rows of stored features X (n x 112 BF16,
// row-major) with labels y: forward through both layers on the tensor cores,
// binary cross-entropy with pos_weight averaged with inv_batch, backward with
// dh1 = dz2 W2 on the tensor cores, weight gradients accumulated in FP32 into
// grads. With grads == nullptr only the forward runs (logits written when
// logits != nullptr).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128)
    k_mlp_train(const __nv_bfloat16* __restrict__ X, const uint8_t* __restrict__ y, int n, float pos_weight,
                float inv_batch, const unsigned char* __restrict__ img, const float* __restrict__ params,
                float* __restrict__ grads, float* __restrict__ loss_sum, float* __restrict__ logits,
                unsigned int* __restrict__ err) {
  extern __shared__ __align__(128) unsigned char sm[];
  unsigned char* XA = sm + tl::XA;
  unsigned char* XT = sm + tl::XT;
  unsigned char* H1 = sm + tl::H1;
  unsigned char* H1T = sm + tl::H1T;
  unsigned char* DZ2 = sm + tl::DZ2;
  unsigned char* DZ2T = sm + tl::DZ2T;
  unsigned char* DZ1T = sm + tl::DZ1T;
  unsigned char* B1 = sm + tl::IMG;
  unsigned char* B2 = B1 + kImgB1;
  unsigned char* B2t = B2 + kImgB2;
  float* pb = reinterpret_cast<float*>(sm + tl::PB);     // b1, b2, w3, b3
  float* gw3 = reinterpret_cast<float*>(sm + tl::GW3);   // [64][128] partials of the w3 gradient
  __shared__ uint64_t bar;
  __shared__ uint32_t tmem_slot;
  const bool train = grads != nullptr;
  copy_bytes(B1, img, kImgBytes);
  for (int i = threadIdx.x; i < kHidden; i += blockDim.x) {
    pb[i] = params[kB1 + i];
    pb[64 + i] = params[kB2 + i];
    pb[128 + i] = params[kW3 + i];
  }
  if (threadIdx.x == 0) pb[192] = params[kB3];
  if (train) {
    // transposed tiles: zero, with the rows of ones that carry the bias sums
    const __nv_bfloat16 one = __float2bfloat16_rn(1.0f), zero = __float2bfloat16_rn(0.0f);
    for (int e = threadIdx.x; e < kRows * kRows; e += blockDim.x) {
      const int row = e / kRows, q = e - (e / kRows) * kRows;
      *reinterpret_cast<__nv_bfloat16*>(XT + tc::kmajor_offset(row, q, kRows)) = row == tl::kOnesX ? one : zero;
      *reinterpret_cast<__nv_bfloat16*>(H1T + tc::kmajor_offset(row, q, kRows)) = row == tl::kOnesH ? one : zero;
    }
    for (int e = threadIdx.x; e < kHidden * kRows; e += blockDim.x) gw3[e] = 0.0f;
  }
  block_tmem_setup(&tmem_slot, &bar, kTrainCols);
  const uint32_t tb = tmem_slot;
  const int r = threadIdx.x;
  uint32_t phase = 0;
  float loss_local = 0.0f, gb3 = 0.0f;
  bool accumulated = false, failed = false;
  for (int tile = blockIdx.x; tile * kRows < n; tile += gridDim.x) {
    const int s = tile * kRows + r;
    const bool valid = s < n;
    // X row -> canonical tile (16-byte chunks of 8 features) and its transpose
    const uint4* xr = reinterpret_cast<const uint4*>(X + (size_t)(valid ? s : 0) * kInPad);
#pragma unroll
    for (int c = 0; c < kInPad / 8; ++c) {
      const uint4 q = valid ? xr[c] : make_uint4(0u, 0u, 0u, 0u);
      *reinterpret_cast<uint4*>(XA + tc::kmajor_offset(r, 8 * c, kRows)) = q;
      if (train) {
        const unsigned short* e = reinterpret_cast<const unsigned short*>(&q);
#pragma unroll
        for (int k = 0; k < 8; ++k)
          *reinterpret_cast<unsigned short*>(XT + tc::kmajor_offset(8 * c + k, r, kRows)) = e[k];
      }
    }
    const float label = valid ? (float)y[s] : 0.0f;
    if (!run_gemm(tb + kColD1, XA, B1, kInPad, kHidden, &bar, phase, err)) {
      failed = true;
      break;
    }
    float h[kHidden];
    load_row64(tb, kColD1, h);
#pragma unroll
    for (int j = 0; j < kHidden; ++j) {
      const float a = gelu(h[j] + pb[j]);
      store_bf16(H1, tc::kmajor_offset(r, j, kRows), a);
      if (train) store_bf16(H1T, tc::kmajor_offset(j, r, kRows), a);
    }
    if (!run_gemm(tb + kColD2, H1, B2, kHidden, kHidden, &bar, phase, err)) {
      failed = true;
      break;
    }
    load_row64(tb, kColD2, h);
    float logit = pb[192];
#pragma unroll
    for (int j = 0; j < kHidden; ++j) logit += gelu(h[j] + pb[64 + j]) * pb[128 + j];
    if (logits && valid) logits[s] = logit;
    // BCE with logits and pos_weight: L = -(pw y log s(x) + (1 - y) log(1 - s(x)))
    const float sp = log1pf(__expf(-fabsf(logit))) + fmaxf(-logit, 0.0f);  // softplus(-x)
    const float lw = 1.0f + (pos_weight - 1.0f) * label;
    if (valid) loss_local += (1.0f - label) * logit + lw * sp;
    if (train) {
      const float sig = 1.0f / (1.0f + __expf(-logit));
      const float dlogit = valid ? (sig * (pos_weight * label + 1.0f - label) - pos_weight * label) * inv_batch : 0.0f;
      gb3 += dlogit;
      // output-layer gradient partials and dz2 = dlogit w3 gelu'(z2)
#pragma unroll
      for (int j = 0; j < kHidden; ++j) {
        const float z = h[j] + pb[64 + j];
        gw3[j * kRows + r] += gelu(z) * dlogit;
        const float dz = dlogit * pb[128 + j] * gelu_grad(z);
        store_bf16(DZ2, tc::kmajor_offset(r, j, kRows), dz);
        store_bf16(DZ2T, tc::kmajor_offset(j, r, kHidden), dz);
      }
      // dh1 = dz2 W2, then dz1 = dh1 gelu'(z1) with z1 read back from TMEM
      if (!run_gemm(tb + kColDH, DZ2, B2t, kHidden, kHidden, &bar, phase, err)) {
        failed = true;
        break;
      }
      float z1[kHidden];
      load_row64(tb, kColDH, h);
      load_row64(tb, kColD1, z1);
#pragma unroll
      for (int j = 0; j < kHidden; ++j)
        store_bf16(DZ1T, tc::kmajor_offset(j, r, kHidden), h[j] * gelu_grad(z1[j] + pb[j]));
      // weight (and bias) gradients of the tile, accumulated in TMEM
      if (publish_operands()) {
        issue_gemm(tb + kColGW1, XT, DZ1T, kRows, kHidden, accumulated);
        issue_gemm(tb + kColGW2, H1T, DZ2T, kRows, kHidden, accumulated);
        tc::mma_commit(&bar);
      }
      if (!wait_gemms(&bar, phase, err)) {
        failed = true;
        break;
      }
      accumulated = true;
    }
    tc::fence_before_sync();
    __syncthreads();
  }
  if (loss_sum) {
    for (int o = 16; o > 0; o >>= 1) loss_local += __shfl_xor_sync(0xffffffffu, loss_local, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss_sum, loss_local);
  }
  if (train && accumulated && !failed) {
    // lane r of the accumulators: dW1^T row r (feature r, or b1 at the ones
    // row) and dW2^T row r (unit r, or b2 at the ones row)
    float g[kHidden];
    load_row64(tb, kColGW1, g);
    if (r < kIn) {
#pragma unroll
      for (int j = 0; j < kHidden; ++j) atomicAdd(&grads[kW1 + j * kIn + r], g[j]);
    } else if (r == tl::kOnesX) {
#pragma unroll
      for (int j = 0; j < kHidden; ++j) atomicAdd(&grads[kB1 + j], g[j]);
    }
    load_row64(tb, kColGW2, g);
    if (r < kHidden) {
#pragma unroll
      for (int j = 0; j < kHidden; ++j) atomicAdd(&grads[kW2 + j * kHidden + r], g[j]);
    } else if (r == tl::kOnesH) {
#pragma unroll
      for (int j = 0; j < kHidden; ++j) atomicAdd(&grads[kB2 + j], g[j]);
    }
    __syncthreads();
    if (r < kHidden) {
      float a = 0.0f;
      for (int q = 0; q < kRows; ++q) a += gw3[r * kRows + q];
      atomicAdd(&grads[kW3 + r], a);
    }
    for (int o = 16; o > 0; o >>= 1) gb3 += __shfl_xor_sync(0xffffffffu, gb3, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&grads[kB3], gb3);
  }
  block_tmem_release(tb, kTrainCols);
}

// Adam on the FP32 parameters; clears the gradients.
__global__ void k_mlp_adam(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                           int n, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    g[i] = 0.0f;
  }
}

// BF16 operand images of W1 (N = 64 x K = 112), W2 (N = j x K = i) and its
// transpose (N = i x K = j), in the K-major canonical layout of 64-row tiles.
__global__ void k_mlp_pack(const float* __restrict__ p, unsigned char* __restrict__ img) {
  unsigned char* b1 = img;
  unsigned char* b2 = img + kImgB1;
  unsigned char* b2t = b2 + kImgB2;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < kHidden * kInPad; e += gridDim.x * blockDim.x) {
    const int j = e / kInPad, k = e - (e / kInPad) * kInPad;
    store_bf16(b1, tc::kmajor_offset(j, k, kHidden), k < kIn ? p[kW1 + j * kIn + k] : 0.0f);
  }
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < kHidden * kHidden; e += gridDim.x * blockDim.x) {
    const int j = e / kHidden, i = e - (e / kHidden) * kHidden;
    const float w = p[kW2 + j * kHidden + i];
    store_bf16(b2, tc::kmajor_offset(j, i, kHidden), w);
    store_bf16(b2t, tc::kmajor_offset(i, j, kHidden), w);
  }
}

// Features and labels of every interior cell from a handle's last stage.
template <typename Tw>
__global__ void k_mlp_features(const Tw* __restrict__ W, int g, int gy, int sx, int vs, int nx, int ny, int4 vid4,
                               const Scalars* __restrict__ sc, const uint8_t* __restrict__ trouble,
                               __nv_bfloat16* __restrict__ X, uint8_t* __restrict__ y) {
  const int vid[4] = {vid4.x, vid4.y, vid4.z, vid4.w};
  float inv_s[4];
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    const double range = key_value(sc->vmax_key[vid[v]]) - key_value(sc->vmin_key[vid[v]]);
    inv_s[v] = (float)(1.0 / ((double)kEps * (range > 0.0 ? range : 1.0)));
  }
  for (int cell = blockIdx.x * blockDim.x + threadIdx.x; cell < nx * ny; cell += gridDim.x * blockDim.x) {
    const int x = cell / ny, yy = cell - (cell / ny) * ny;
    uint4* row = reinterpret_cast<uint4*>(X + (size_t)cell * kInPad);
    feature_row<Tw>(W, sx, vs, (x + g) * sx + (yy + gy), vid, inv_s, [&](int c, uint4 q) { row[c] = q; });
    y[cell] = trouble[cell];
  }
}

// Predicted / troubled / missed / false-alarm counts of one stage.
__global__ void k_pred_counts(const uint8_t* __restrict__ trouble, const uint8_t* __restrict__ pred, int n,
                              Scalars* __restrict__ sc) {
  unsigned int np = 0, nt = 0, nm = 0, nf = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const bool t = trouble[i] != 0, p = pred[i] != 0;
    np += p;
    nt += t;
    nm += t && !p;
    nf += p && !t;
  }
  block_count_add(np, &sc->predicted);
  block_count_add(nt, &sc->judged);
  block_count_add(nm, &sc->missed);
  block_count_add(nf, &sc->false_alarm);
}

int fail_mlp(fvh_mlp* m, int code, const std::string& msg) {
  if (m) m->errmsg = msg;
  g_mlp_error = msg;
  return code;
}

int mlp_sync_error(fvh_mlp* m, const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail_mlp(m, FVH_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return FVH_OK;
}

int pack(fvh_mlp* m, cudaStream_t s) {
  k_mlp_pack<<<32, 256, 0, s>>>(m->params, m->img);
  return mlp_sync_error(m, "pack");
}

// 2D geometry of a handle: active axes, ghost width of W, primitive ids
bool handle_2d(const fvh_handle* h, int* ax) {
  int na = 0;
  for (int a = 0; a < 3; ++a)
    if (h->active[a]) {
      if (na < 2) ax[na] = a;
      ++na;
    }
  return na == 2;
}

}  // namespace

namespace fvh {

// Prediction flags for the fused 2D stage (called by the stage runners).
int mlp_predict_stage(fvh_handle* h, cudaStream_t s) {
  fvh_mlp* m = h->mlp;
  int ax[2];
  handle_2d(h, ax);
  const int nx = h->n[ax[0]], ny = h->n[ax[1]];
  const int4 vid = make_int4(0, 1 + ax[0], 1 + ax[1], 4);
  const int tiles = (nx * ny + kRows - 1) / kRows;
  const int grid = tiles < 148 * 4 ? tiles : 148 * 4;  // 4 CTAs per SM: shared memory and TMEM both allow it
  const WLayout lay = fused_w_layout(h, h->gW);
  LaunchScope scope(KK_PREDICT, (double)nx * ny * (4 * h->elem + 1), s);
  if (h->elem == sizeof(float)) {
    cudaFuncSetAttribute(k_mlp_predict<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, kPredictSmem);
    k_mlp_predict<float><<<grid, kRows, kPredictSmem, s>>>((const float*)h->W, lay.g, lay.gy, lay.sx, lay.vs, nx, ny,
                                                          vid, h->sc, m->img,
                                                          m->params, h->pred_thr_logit, h->pred, m->err);
  } else {
    cudaFuncSetAttribute(k_mlp_predict<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, kPredictSmem);
    k_mlp_predict<double><<<grid, kRows, kPredictSmem, s>>>((const double*)h->W, lay.g, lay.gy, lay.sx, lay.vs, nx,
                                                           ny, vid, h->sc, m->img,
                                                           m->params, h->pred_thr_logit, h->pred, m->err);
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    h->err = std::string("predictor: ") + cudaGetErrorString(e);
    return FVH_ERR_CUDA;
  }
  return FVH_OK;
}

int mlp_count_stage(fvh_handle* h, cudaStream_t s) {
  const int n = h->n[0] * h->n[1] * h->n[2];
  const int grid = (n + 4095) / 4096 < 148 * 8 ? (n + 4095) / 4096 : 148 * 8;
  LaunchScope scope(KK_SMALL, 2.0 * n, s);
  k_pred_counts<<<grid, 256, 0, s>>>(h->trouble, h->pred, n, h->sc);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    h->err = std::string("predictor counts: ") + cudaGetErrorString(e);
    return FVH_ERR_CUDA;
  }
  return FVH_OK;
}

}  // namespace fvh

extern "C" {

size_t fvh_mlp_param_count(void) { return (size_t)kParams; }

int fvh_mlp_create(int device, uint64_t seed, fvh_mlp** out) {
  if (!out) return FVH_ERR_ARG;
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return fail_mlp(nullptr, FVH_ERR_CONFIG, "invalid device");
  }
  fvh_mlp* m = new (std::nothrow) fvh_mlp();
  if (!m) return fail_mlp(nullptr, FVH_ERR_CONFIG, "out of host memory");
  m->device = device;
  const size_t pb = kParams * sizeof(float);
  if (cudaMalloc(&m->params, pb) != cudaSuccess || cudaMalloc(&m->grads, pb) != cudaSuccess ||
      cudaMalloc(&m->m, pb) != cudaSuccess || cudaMalloc(&m->v, pb) != cudaSuccess ||
      cudaMalloc(&m->img, kImgBytes) != cudaSuccess || cudaMalloc(&m->loss, sizeof(float)) != cudaSuccess ||
      cudaMalloc(&m->err, sizeof(unsigned int)) != cudaSuccess) {
    cudaGetLastError();
    fvh_mlp_destroy(m);
    return fail_mlp(nullptr, FVH_ERR_CUDA, "cudaMalloc failed");
  }
  // He-style initialisation from the seed; zero biases
  std::vector<float> host(kParams, 0.0f);
  std::mt19937_64 rng(seed);
  std::normal_distribution<float> nd(0.0f, 1.0f);
  for (int i = 0; i < kHidden * kIn; ++i) host[kW1 + i] = nd(rng) * std::sqrt(2.0f / kIn);
  for (int i = 0; i < kHidden * kHidden; ++i) host[kW2 + i] = nd(rng) * std::sqrt(2.0f / kHidden);
  for (int i = 0; i < kHidden; ++i) host[kW3 + i] = nd(rng) * std::sqrt(1.0f / kHidden);
  cudaMemcpy(m->params, host.data(), pb, cudaMemcpyHostToDevice);
  cudaMemset(m->grads, 0, pb);
  cudaMemset(m->m, 0, pb);
  cudaMemset(m->v, 0, pb);
  cudaMemset(m->err, 0, sizeof(unsigned int));
  int st = pack(m, nullptr);
  if (!st && cudaDeviceSynchronize() != cudaSuccess) st = mlp_sync_error(m, "init");
  if (st) {
    fvh_mlp_destroy(m);
    return st;
  }
  *out = m;
  return FVH_OK;
}

int fvh_mlp_destroy(fvh_mlp* m) {
  if (!m) return FVH_OK;
  cudaSetDevice(m->device);
  void* ptrs[] = {m->params, m->grads, m->m, m->v, m->img, m->loss, m->err};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  delete m;
  return FVH_OK;
}

const char* fvh_mlp_last_error(const fvh_mlp* m) { return m ? m->errmsg.c_str() : g_mlp_error.c_str(); }

int fvh_mlp_get_params(fvh_mlp* m, float* host, size_t n) {
  if (!m || !host || n != (size_t)kParams) return FVH_ERR_ARG;
  cudaSetDevice(m->device);
  if (cudaMemcpy(host, m->params, n * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
    return mlp_sync_error(m, "get_params");
  return FVH_OK;
}

int fvh_mlp_set_params(fvh_mlp* m, const float* host, size_t n) {
  if (!m || !host || n != (size_t)kParams) return FVH_ERR_ARG;
  cudaSetDevice(m->device);
  if (cudaMemcpy(m->params, host, n * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
    return mlp_sync_error(m, "set_params");
  cudaMemset(m->m, 0, n * sizeof(float));
  cudaMemset(m->v, 0, n * sizeof(float));
  m->step = 0;
  int st = pack(m, nullptr);
  if (!st && cudaDeviceSynchronize() != cudaSuccess) st = mlp_sync_error(m, "set_params");
  return st;
}

int fvh_mlp_features(fvh_handle* h, uint16_t* X, uint8_t* y, void* stream) {
  if (!h || !X || !y) return FVH_ERR_ARG;
  int ax[2];
  if (!handle_2d(h, ax) || !h->last_stage_fused || !h->cfg.a_posteriori || !h->cfg.nad_global) {
    h->err = "features need a 2D a-posteriori (global NAD) handle whose last stage ran the fused 2D kernels";
    return FVH_ERR_CONFIG;
  }
  if (cudaSetDevice(h->cfg.device) != cudaSuccess) return FVH_ERR_CUDA;
  const int nx = h->n[ax[0]], ny = h->n[ax[1]];
  const int4 vid = make_int4(0, 1 + ax[0], 1 + ax[1], 4);
  cudaStream_t s = (cudaStream_t)stream;
  const int grid = (nx * ny + 255) / 256 < 4096 ? (nx * ny + 255) / 256 : 4096;
  const WLayout lay = fused_w_layout(h, h->gW);
  if (h->elem == sizeof(float))
    k_mlp_features<float><<<grid, 256, 0, s>>>((const float*)h->W, lay.g, lay.gy, lay.sx, lay.vs, nx, ny, vid, h->sc,
                                               h->trouble, reinterpret_cast<__nv_bfloat16*>(X), y);
  else
    k_mlp_features<double><<<grid, 256, 0, s>>>((const double*)h->W, lay.g, lay.gy, lay.sx, lay.vs, nx, ny, vid,
                                                h->sc, h->trouble, reinterpret_cast<__nv_bfloat16*>(X), y);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    h->err = std::string("features: ") + cudaGetErrorString(e);
    return FVH_ERR_CUDA;
  }
  return FVH_OK;
}

// Gradients (added to the internal gradient buffer, or written to grads_out
// when given) and the summed loss of n rows, without an update.
static int run_train_kernel(fvh_mlp* m, const uint16_t* X, const uint8_t* y, int n, float pos_weight,
                            float inv_batch, float* grads, float* logits, cudaStream_t s) {
  cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrainSmem);
  const int tiles = (n + kRows - 1) / kRows;
  const int grid = tiles < 148 ? tiles : 148;
  k_mlp_train<<<grid, kRows, kTrainSmem, s>>>(reinterpret_cast<const __nv_bfloat16*>(X), y, n, pos_weight, inv_batch,
                                              m->img, m->params, grads, m->loss, logits, m->err);
  return mlp_sync_error(m, "train kernel");
}

int fvh_mlp_train_step(fvh_mlp* m, const uint16_t* X, const uint8_t* y, int n, float lr, float pos_weight,
                       float* loss_out, void* stream) {
  if (!m || !X || !y || n <= 0) return FVH_ERR_ARG;
  cudaSetDevice(m->device);
  cudaStream_t s = (cudaStream_t)stream;
  cudaMemsetAsync(m->loss, 0, sizeof(float), s);
  int st = run_train_kernel(m, X, y, n, pos_weight, 1.0f / (float)n, m->grads, nullptr, s);
  if (st) return st;
  m->step += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - std::pow(b1, (float)m->step), c2 = 1.0f - std::pow(b2, (float)m->step);
  k_mlp_adam<<<(kParams + 255) / 256, 256, 0, s>>>(m->params, m->grads, m->m, m->v, kParams, lr, b1, b2, 1e-8f, c1,
                                                   c2);
  if ((st = mlp_sync_error(m, "adam"))) return st;
  if ((st = pack(m, s))) return st;
  if (loss_out) {
    float l = 0.0f;
    if (cudaMemcpyAsync(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return mlp_sync_error(m, "loss");
    *loss_out = l / (float)n;
  }
  return FVH_OK;
}

int fvh_mlp_gradients(fvh_mlp* m, const uint16_t* X, const uint8_t* y, int n, float pos_weight, float* grads_out,
                      float* loss_out, void* stream) {
  if (!m || !X || !y || !grads_out || n <= 0) return FVH_ERR_ARG;
  cudaSetDevice(m->device);
  cudaStream_t s = (cudaStream_t)stream;
  cudaMemsetAsync(m->loss, 0, sizeof(float), s);
  cudaMemsetAsync(grads_out, 0, kParams * sizeof(float), s);
  int st = run_train_kernel(m, X, y, n, pos_weight, 1.0f / (float)n, grads_out, nullptr, s);
  if (st) return st;
  if (loss_out) {
    float l = 0.0f;
    cudaMemcpyAsync(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return mlp_sync_error(m, "loss");
    *loss_out = l / (float)n;
  }
  return FVH_OK;
}

int fvh_mlp_logits(fvh_mlp* m, const uint16_t* X, int n, float* logits, void* stream) {
  if (!m || !X || !logits || n <= 0) return FVH_ERR_ARG;
  cudaSetDevice(m->device);
  cudaStream_t s = (cudaStream_t)stream;
  // labels are not read without gradients; X doubles as a harmless label pointer
  return run_train_kernel(m, X, reinterpret_cast<const uint8_t*>(X), n, 1.0f, 1.0f, nullptr, logits, s);
}

unsigned int fvh_mlp_errors(fvh_mlp* m) {
  if (!m) return 0;
  unsigned int e = 0;
  cudaSetDevice(m->device);
  cudaMemcpy(&e, m->err, sizeof(e), cudaMemcpyDeviceToHost);
  return e;
}

int fvh_set_predictor(fvh_handle* h, fvh_mlp* m, float threshold) {
  if (!h) return FVH_ERR_ARG;
  if (!m) {
    h->mlp = nullptr;
    return FVH_OK;
  }
  int ax[2];
  if (!handle_2d(h, ax) || !h->cfg.a_posteriori || !h->cfg.nad_global || h->nv != 5 || h->cfg.convex ||
      h->cfg.kernel_path == FVH_PATH_GENERIC || h->p[ax[0]] != h->p[ax[1]] || h->p[ax[0]] < 1) {
    h->err = "the predictor needs the fused 2D path with a-posteriori limiting and global NAD";
    return FVH_ERR_CONFIG;
  }
  if (m->device != h->cfg.device) {
    h->err = "predictor and solver live on different devices";
    return FVH_ERR_CONFIG;
  }
  if (!(threshold > 0.0f && threshold < 1.0f)) {
    h->err = "threshold must be a probability in (0, 1)";
    return FVH_ERR_ARG;
  }
  if (cudaSetDevice(h->cfg.device) != cudaSuccess) return FVH_ERR_CUDA;
  if (!h->pred) {
    const size_t n = (size_t)h->n[0] * h->n[1] * h->n[2];
    if (cudaMalloc(&h->pred, n) != cudaSuccess) {
      cudaGetLastError();
      h->err = "cudaMalloc of the prediction flags failed";
      return FVH_ERR_CUDA;
    }
    cudaMemset(h->pred, 0, n);
    h->scratch_bytes += n;
  }
  h->mlp = m;
  h->pred_thr_logit = std::log(threshold / (1.0f - threshold));
  h->pred_stage = 0;
  return FVH_OK;
}

int fvh_set_predictor_interval(fvh_handle* h, int stages) {
  if (!h) return FVH_ERR_ARG;
  if (stages < 1) {
    h->err = "the prediction interval is a positive number of stages";
    return FVH_ERR_ARG;
  }
  h->pred_interval = stages;
  h->pred_stage = 0;
  return FVH_OK;
}

}  // extern "C"
