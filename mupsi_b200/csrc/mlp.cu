// Surrogate-mean MLP on the tcgen05 tensor cores: inference, a fused
// forward+backward gradient kernel, minibatch gathering and Adam.
//
// The network (include/mupsi_gpu.h, mupsi_mlp_desc): Fourier features of
// p - center (48 sin/cos pairs), four 64-wide ReLU layers, a linear output.
// One CTA of 128 threads owns a tile of 128 points: thread b is point b and
// TMEM lane b. Every layer is an M = 128 BF16 MMA with an FP32 accumulator in
// TMEM; a thread reads its row back (tcgen05.ld), adds the bias, applies the
// ReLU and stores the BF16 activations into the next layer's operand tile.
//
// Backward, per layer with pre-activation gradient dz (128 x 64, BF16):
//   dW += dz^T H   (M = 128 over the 64 outputs, the upper half unused; K = the
//                   128 points; H carries an extra column of ones, so the same
//                   product yields the bias gradient)
//   dh  = dz W     (M = 128 points, K = 64)
// Both read dz and H from the same tiles the forward pass uses: dz^T and H as
// MN-major operands. The weight gradients accumulate in TMEM across all tiles
// a CTA processes and are added to global memory once at the end.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>

#include "core.cuh"
#include "host.h"
#include "tc.cuh"

namespace mupsi {
namespace {

constexpr int kFreq = 48;
constexpr int kFeat = 96;    // sin/cos features
constexpr int kFeatP = 112;  // + a column of ones + padding to a core-matrix multiple
constexpr int kHid = 64;
constexpr int kHidP = 80;    // + ones + padding
constexpr int kRows = 128;   // points per tile

// parameter vector (mupsi_mlp_desc.params): W1[64][96], b1, (W_l, b_l) l = 2..4, w5, b5
constexpr int kOffW5 = 18688;
constexpr int kOffB5 = 18752;
MD int offW(int l) { return l == 0 ? 0 : 6208 + 4160 * (l - 1); }
MD int offB(int l) { return l == 0 ? 6144 : 6208 + 4160 * (l - 1) + 4096; }

struct MlpConst {
  float B[kFreq * 3];
  float c[3];
  float ys;
};

// ---- shared-memory layout (bytes) ----
// W1 [64x96], W2..W4 [64x64], K-major (both kernels)
MD uint32_t sW(int l) { return l == 0 ? 0u : l == 1 ? 12288u : l == 2 ? 20480u : 28672u; }
// gradient kernel: H0 [128x112], H1..H3 [128x80] K-major; dz [128x64] K-major + 2 KB slack
// (the MN-major view of dz as an M = 128 operand reads up to 1 KB past its end)
MD uint32_t sH(int l) { return l == 0 ? 36864u : l == 1 ? 65536u : l == 2 ? 86016u : 106496u; }
constexpr uint32_t kSDZ = 126976;
constexpr uint32_t kSF = 145408;  // floats
constexpr uint32_t kGradSmem = kSF + 1024 + 256 + 256 + 64 + 64;
// inference kernel: one activation tile [128x96] (K 96, then 64)
constexpr uint32_t kIX = 36864;
constexpr uint32_t kIF = kIX + 128 * 96 * 2;
constexpr uint32_t kInferSmem = kIF + 1024 + 256 + 64 + 64;

MD int wK(int l) { return l == 0 ? kFeat : kHid; }                         // K of layer l's product
MD int hP(int l) { return l == 0 ? kFeatP : kHidP; }                       // row stride of H_l; N of its dW
MD uint32_t dwCol(int l) { return l == 0 ? 64u : 96u + 80u * (uint32_t)l; }  // TMEM columns of dW1..dW4

MD uint16_t bf16_bits(float x) {
  __nv_bfloat16 h = __float2bfloat16_rn(x);
  return *reinterpret_cast<uint16_t*>(&h);
}
MD float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
MD uint32_t pack2(float a, float b) { return (uint32_t)bf16_bits(a) | ((uint32_t)bf16_bits(b) << 16); }
MD uint4 pack8(const float* v) {
  return make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]), pack2(v[6], v[7]));
}

// Stage the layer weights as BF16 K-major tiles [64 x K].
MD void stage_weights(unsigned char* sm, const float* __restrict__ params) {
  for (int l = 0; l < 4; ++l) {
    const int K = wK(l);
    const float* W = params + offW(l);
    for (int idx = threadIdx.x; idx < 64 * K; idx += blockDim.x) {
      const int j = idx / K, i = idx - j * K;
      *reinterpret_cast<uint16_t*>(sm + sW(l) + tc::kmajor_off(j, i, K)) = bf16_bits(W[idx]);
    }
  }
}

// Fourier features of x = p - center (phases u_f = B_f . x in FP32) into row b
// of a K-major tile with row stride K: sin in columns 0..47, cos in 48..95.
MD void store_features(unsigned char* sm, uint32_t base, int b, int K, const MlpConst& mc, float x0, float x1,
                       float x2) {
#pragma unroll 1
  for (int g = 0; g < 6; ++g) {
    float s[8], c[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int f = 8 * g + q;
      const float u = mc.B[3 * f] * x0 + (mc.B[3 * f + 1] * x1 + mc.B[3 * f + 2] * x2);
      sincosf(u, &s[q], &c[q]);
    }
    *reinterpret_cast<uint4*>(sm + base + tc::kmajor_off(b, 8 * g, K)) = pack8(s);
    *reinterpret_cast<uint4*>(sm + base + tc::kmajor_off(b, 48 + 8 * g, K)) = pack8(c);
  }
}

// The ones column (element 0 of group g; 0 for padding rows) and a zero group after it.
MD void store_ones(unsigned char* sm, uint32_t base, int b, int K, int g, bool valid) {
  *reinterpret_cast<uint4*>(sm + base + tc::kmajor_off(b, 8 * g, K)) = make_uint4(valid ? 0x3F80u : 0u, 0u, 0u, 0u);
  *reinterpret_cast<uint4*>(sm + base + tc::kmajor_off(b, 8 * g + 8, K)) = make_uint4(0u, 0u, 0u, 0u);
}

// Forward product of layer l: D[0..64) = H_l[:, :K] W_l^T.
MD void issue_forward(uint32_t tmem, uint32_t sbase, uint32_t h_off, int h_stride, uint32_t w_off, int K) {
  const uint32_t id = tc::idesc_bf16(128, 64, false, false);
  const uint32_t sbo_h = (uint32_t)(h_stride / 8) * 128, sbo_w = (uint32_t)(K / 8) * 128;
  for (int ks = 0; ks < K / 16; ++ks) {
    const uint64_t a = tc::sdesc(sbase + h_off + ks * 256, 128, sbo_h);
    const uint64_t b = tc::sdesc(sbase + w_off + ks * 256, 128, sbo_w);
    tc::mma_bf16(tmem, a, b, id, ks > 0);
  }
}

// Wait for the MMAs committed to mbar; every thread learns whether any timed out.
MD bool wait_mma(uint32_t mbar, uint32_t& phase) {
  const bool ok = tc::mbar_wait(mbar, phase);
  phase ^= 1u;
  return __syncthreads_and(ok ? 1 : 0) != 0;
}

// ---------------------------------------------------------------- gradient
__global__ void __launch_bounds__(128, 1) k_mlp_grad(const float* __restrict__ params, MlpConst mc,
                                                     const float* __restrict__ P, const float* __restrict__ T,
                                                     int64_t n, float inv_n, float* __restrict__ grad,
                                                     float* __restrict__ loss, int* err) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  float* bias = reinterpret_cast<float*>(sm + kSF);  // [4][64]
  float* w5f = bias + 256;                           // BF16-rounded output weights
  float* dw5 = w5f + 64;                             // output-layer gradient accumulators
  float* misc = dw5 + 64;                            // [0] b5, [1] db5, [2] loss
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(misc + 14);
  uint64_t* mbar_p = reinterpret_cast<uint64_t*>(misc + 16);
  const uint32_t sbase = tc::smem_u32(sm);
  const uint32_t mbar = tc::smem_u32(mbar_p);

  stage_weights(sm, params);
  for (int i = tid; i < 256; i += 128) bias[i] = params[offB(i >> 6) + (i & 63)];
  if (tid < 64) {
    w5f[tid] = bf16_round(params[kOffW5 + tid]);
    dw5[tid] = 0.0f;
  }
  if (tid == 0) {
    misc[0] = params[kOffB5];
    misc[1] = 0.0f;
    misc[2] = 0.0f;
    tc::mbar_init(mbar, 1);
  }
  if (warp == 0) tc::tmem_alloc(tc::smem_u32(tmem_slot), 512);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t tlane = tmem + ((uint32_t)(32 * warp) << 16);
  uint32_t phase = 0;
  bool any = false, failed = false;
  float loss_acc = 0.0f;

  for (int64_t tile = blockIdx.x; tile * kRows < n && !failed; tile += gridDim.x) {
    const int64_t row = tile * kRows + tid;
    const bool valid = row < n;
    float x0 = 0.0f, x1 = 0.0f, x2 = 0.0f, tgt = 0.0f;
    if (valid) {
      x0 = P[3 * row] - mc.c[0];
      x1 = P[3 * row + 1] - mc.c[1];
      x2 = P[3 * row + 2] - mc.c[2];
      tgt = T[row];
    }
    store_features(sm, sH(0), tid, kFeatP, mc, x0, x1, x2);
    store_ones(sm, sH(0), tid, kFeatP, 12, valid);
    uint64_t mask[4];
    float y = 0.0f;
    // ---- forward
    for (int l = 0; l < 4 && !failed; ++l) {
      tc::fence_proxy_async();
      tc::fence_before();
      __syncthreads();
      if (tid == 0) {
        tc::fence_after();
        issue_forward(tmem, sbase, sH(l), hP(l), sW(l), wK(l));
        tc::commit(mbar);
      }
      if (!wait_mma(mbar, phase)) {
        failed = true;
        break;
      }
      tc::fence_after();
      uint64_t m = 0;
      if (l < 3) {
        for (int c = 0; c < 4; ++c) {
          float z[16];
          tc::tmem_ld16(tlane + 16 * c, z);
          tc::tmem_wait_ld();
          float h[16];
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            const float v = z[q] + bias[64 * l + 16 * c + q];
            if (v > 0.0f) m |= 1ull << (16 * c + q);
            h[q] = v > 0.0f ? v : 0.0f;
          }
          *reinterpret_cast<uint4*>(sm + sH(l + 1) + tc::kmajor_off(tid, 16 * c, kHidP)) = pack8(h);
          *reinterpret_cast<uint4*>(sm + sH(l + 1) + tc::kmajor_off(tid, 16 * c + 8, kHidP)) = pack8(h + 8);
        }
        store_ones(sm, sH(l + 1), tid, kHidP, 8, valid);
      } else {
        for (int c = 0; c < 4; ++c) {
          float z[16];
          tc::tmem_ld16(tlane + 16 * c, z);
          tc::tmem_wait_ld();
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            const float v = z[q] + bias[192 + 16 * c + q];
            if (v > 0.0f) m |= 1ull << (16 * c + q);
            y = y + w5f[16 * c + q] * bf16_round(v > 0.0f ? v : 0.0f);
          }
        }
        y = y + misc[0];
      }
      mask[l] = m;
    }
    if (failed) break;
    // ---- output layer (CUDA cores)
    const float r = valid ? y - tgt / mc.ys : 0.0f;
    loss_acc += r * r;
    const float dy = 2.0f * r * inv_n;
    {
      float s = dy;
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) atomicAdd(&misc[1], s);
    }
    for (int c = 0; c < 4; ++c) {
      float z[16];
      tc::tmem_ld16(tlane + 16 * c, z);  // z4 is still in D
      tc::tmem_wait_ld();
      float d[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const int j = 16 * c + q;
        const float v = z[q] + bias[192 + j];
        float s = dy * bf16_round(v > 0.0f ? v : 0.0f);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) atomicAdd(&dw5[j], s);
        const float dh = dy * w5f[j];
        d[q] = ((mask[3] >> j) & 1ull) ? dh : 0.0f;
      }
      *reinterpret_cast<uint4*>(sm + kSDZ + tc::kmajor_off(tid, 16 * c, kHid)) = pack8(d);
      *reinterpret_cast<uint4*>(sm + kSDZ + tc::kmajor_off(tid, 16 * c + 8, kHid)) = pack8(d + 8);
    }
    // ---- backward through the hidden layers: l = 3..0 is W_{l+1} with input H_l
    for (int l = 3; l >= 0 && !failed; --l) {
      tc::fence_proxy_async();
      tc::fence_before();
      __syncthreads();
      if (tid == 0) {
        tc::fence_after();
        const uint32_t sbo_h = (uint32_t)(hP(l) / 8) * 128;
        const uint32_t id_w = tc::idesc_bf16(128, hP(l), true, true);
        for (int ks = 0; ks < kRows / 16; ++ks) {
          const uint64_t a = tc::sdesc(sbase + kSDZ + ks * 2048, 1024, 128);        // dz^T, MN-major
          const uint64_t b = tc::sdesc(sbase + sH(l) + ks * 2 * sbo_h, sbo_h, 128);  // H_l, MN-major
          tc::mma_bf16(tmem + dwCol(l), a, b, id_w, (any || ks > 0) ? 1u : 0u);
        }
        if (l > 0) {
          const uint32_t id_h = tc::idesc_bf16(128, 64, false, true);
          for (int ks = 0; ks < kHid / 16; ++ks) {
            const uint64_t a = tc::sdesc(sbase + kSDZ + ks * 256, 128, 1024);     // dz, K-major
            const uint64_t b = tc::sdesc(sbase + sW(l) + ks * 2048, 1024, 128);  // W_{l+1}, MN-major
            tc::mma_bf16(tmem, a, b, id_h, ks > 0);
          }
        }
        tc::commit(mbar);
      }
      if (!wait_mma(mbar, phase)) {
        failed = true;
        break;
      }
      tc::fence_after();
      if (l > 0) {
        for (int c = 0; c < 4; ++c) {
          float dh[16];
          tc::tmem_ld16(tlane + 16 * c, dh);
          tc::tmem_wait_ld();
#pragma unroll
          for (int q = 0; q < 16; ++q)
            if (!((mask[l - 1] >> (16 * c + q)) & 1ull)) dh[q] = 0.0f;
          *reinterpret_cast<uint4*>(sm + kSDZ + tc::kmajor_off(tid, 16 * c, kHid)) = pack8(dh);
          *reinterpret_cast<uint4*>(sm + kSDZ + tc::kmajor_off(tid, 16 * c + 8, kHid)) = pack8(dh + 8);
        }
      }
    }
    any = true;
  }
  // ---- weight and bias gradients out of TMEM (rows 0..63: warps 0 and 1)
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  if (any && !failed && warp < 2) {
    const int j = 32 * warp + lane;
    for (int l = 0; l < 4; ++l) {
      const int K = wK(l);
      for (int c = 0; c < hP(l) / 16; ++c) {
        float v[16];
        tc::tmem_ld16(tlane + dwCol(l) + 16 * c, v);
        tc::tmem_wait_ld();
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          const int i = 16 * c + q;
          if (i < K)
            atomicAdd(&grad[offW(l) + j * K + i], v[q]);
          else if (i == K)
            atomicAdd(&grad[offB(l) + j], v[q]);
        }
      }
    }
  }
  {
    float s = loss_acc;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) atomicAdd(&misc[2], s);
  }
  tc::fence_before();
  __syncthreads();
  if (!failed) {
    if (tid < 64) atomicAdd(&grad[kOffW5 + tid], dw5[tid]);
    if (tid == 0) {
      atomicAdd(&grad[kOffB5], misc[1]);
      atomicAdd(loss, misc[2]);
    }
  } else if (tid == 0) {
    atomicOr(err, 1);
  }
  if (warp == 0) tc::tmem_dealloc(tmem, 512);
}

// ---------------------------------------------------------------- inference
// Points p_i at P + i * pstride; n points, or *n_dev points when n_dev is set
// (a count another kernel wrote, at most n).
__global__ void __launch_bounds__(128) k_mlp_infer(const float* __restrict__ params, MlpConst mc,
                                                   const float* __restrict__ P, int pstride, int64_t n,
                                                   const uint32_t* __restrict__ n_dev, float* __restrict__ out,
                                                   int* err) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const int tid = threadIdx.x, warp = tid >> 5;
  if (n_dev) n = min(n, (int64_t)*n_dev);
  if ((int64_t)blockIdx.x * kRows >= n) return;  // no tile for this CTA
  float* bias = reinterpret_cast<float*>(sm + kIF);
  float* w5f = bias + 256;
  float* misc = w5f + 64;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(misc + 6);
  uint64_t* mbar_p = reinterpret_cast<uint64_t*>(misc + 8);
  const uint32_t sbase = tc::smem_u32(sm);
  const uint32_t mbar = tc::smem_u32(mbar_p);
  stage_weights(sm, params);
  for (int i = tid; i < 256; i += 128) bias[i] = params[offB(i >> 6) + (i & 63)];
  if (tid < 64) w5f[tid] = bf16_round(params[kOffW5 + tid]);
  if (tid == 0) {
    misc[0] = params[kOffB5];
    tc::mbar_init(mbar, 1);
  }
  if (warp == 0) tc::tmem_alloc(tc::smem_u32(tmem_slot), 64);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t tlane = tmem + ((uint32_t)(32 * warp) << 16);
  uint32_t phase = 0;
  bool failed = false;
  for (int64_t tile = blockIdx.x; tile * kRows < n && !failed; tile += gridDim.x) {
    const int64_t row = tile * kRows + tid;
    const bool valid = row < n;
    float x0 = 0.0f, x1 = 0.0f, x2 = 0.0f;
    if (valid) {
      x0 = P[pstride * row] - mc.c[0];
      x1 = P[pstride * row + 1] - mc.c[1];
      x2 = P[pstride * row + 2] - mc.c[2];
    }
    store_features(sm, kIX, tid, kFeat, mc, x0, x1, x2);
    float y = 0.0f;
    for (int l = 0; l < 4; ++l) {
      tc::fence_proxy_async();
      tc::fence_before();
      __syncthreads();
      if (tid == 0) {
        tc::fence_after();
        issue_forward(tmem, sbase, kIX, wK(l), sW(l), wK(l));
        tc::commit(mbar);
      }
      if (!wait_mma(mbar, phase)) {
        failed = true;
        break;
      }
      tc::fence_after();
      for (int c = 0; c < 4; ++c) {
        float z[16];
        tc::tmem_ld16(tlane + 16 * c, z);
        tc::tmem_wait_ld();
        if (l < 3) {
          float h[16];
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            const float v = z[q] + bias[64 * l + 16 * c + q];
            h[q] = v > 0.0f ? v : 0.0f;
          }
          *reinterpret_cast<uint4*>(sm + kIX + tc::kmajor_off(tid, 16 * c, kHid)) = pack8(h);
          *reinterpret_cast<uint4*>(sm + kIX + tc::kmajor_off(tid, 16 * c + 8, kHid)) = pack8(h + 8);
        } else {
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            const float v = z[q] + bias[192 + 16 * c + q];
            y = y + w5f[16 * c + q] * bf16_round(v > 0.0f ? v : 0.0f);
          }
        }
      }
    }
    if (failed) break;
    if (valid) out[row] = mc.ys * (y + misc[0]);
  }
  tc::fence_before();
  __syncthreads();
  if (failed && tid == 0) atomicOr(err, 1);
  if (warp == 0) tc::tmem_dealloc(tmem, 64);
}

// ---------------------------------------------------------------- training
MD uint64_t splitmix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Minibatch of `batch` points drawn with replacement from the n.
__global__ void k_mlp_gather(uint64_t seed, int64_t step, int64_t n, const float* __restrict__ P,
                             const float* __restrict__ T, int batch, float* __restrict__ bp, float* __restrict__ bt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < batch; i += gridDim.x * blockDim.x) {
    const uint64_t h = splitmix(seed ^ splitmix((uint64_t)step * 0x100000001B3ull + (uint64_t)i));
    const int64_t j = (int64_t)__umul64hi(h, (uint64_t)n);
    bp[3 * i] = P[3 * j];
    bp[3 * i + 1] = P[3 * j + 1];
    bp[3 * i + 2] = P[3 * j + 2];
    bt[i] = T[j];
  }
}

// Adam (bias-corrected) on the FP32 master parameters; clears the gradient.
__global__ void k_mlp_adam(float* __restrict__ w, float* __restrict__ g, float* __restrict__ m,
                           float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    g[i] = 0.0f;
  }
}

}  // namespace
}  // namespace mupsi

using namespace mupsi;

struct mupsi_mlp {
  MlpConst mc;
  float* params = nullptr;  // FP32 master
  float* grad = nullptr;
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  float* loss = nullptr;    // per-step losses of the last train call (device)
  int64_t loss_cap = 0;
  float* batch = nullptr;   // minibatch points + targets
  int64_t batch_cap = 0;
  int* err = nullptr;
  int64_t adam_t = 0;
  ~mupsi_mlp() {
    for (void* p : {(void*)params, (void*)grad, (void*)adam_m, (void*)adam_v, (void*)loss, (void*)batch, (void*)err})
      if (p) cudaFree(p);
  }
};

namespace mupsi {
namespace {

int mlp_check_err(mupsi_mlp* m, cudaStream_t st) {
  int h = 0;
  MUPSI_CUDA(cudaMemcpyAsync(&h, m->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  MUPSI_CUDA(cudaStreamSynchronize(st));
  if (h) {
    cudaMemsetAsync(m->err, 0, sizeof(int), st);
    return fail(MUPSI_ERR_DEVICE_LIMIT, "tensor-core MMA completion wait timed out");
  }
  return MUPSI_OK;
}

std::mutex g_attr_mu;
bool g_attr_set[64] = {};

int mlp_kernel_attrs() {
  int dev = 0;
  MUPSI_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(g_attr_mu);
  if (dev >= 0 && dev < 64 && !g_attr_set[dev]) {
    MUPSI_CUDA(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGradSmem));
    MUPSI_CUDA(cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInferSmem));
    g_attr_set[dev] = true;
  }
  return MUPSI_OK;
}

int mlp_launch_grad(mupsi_mlp* m, int64_t n, const float* p, const float* t, float* grad, float* loss,
                    cudaStream_t st) {
  if (int e = mlp_kernel_attrs()) return e;
  const int64_t tiles = (n + kRows - 1) / kRows;
  const int grid = (int)std::min<int64_t>(tiles, num_sms());
  k_mlp_grad<<<grid, 128, kGradSmem, st>>>(m->params, m->mc, p, t, n, 1.0f / (float)n, grad, loss, m->err);
  count_launch();
  MUPSI_CUDA(cudaGetLastError());
  return MUPSI_OK;
}

}  // namespace

int mlp_infer_device(mupsi_mlp* m, int64_t n, const float* p, int pstride, const uint32_t* n_dev, float* out,
                     cudaStream_t st) {
  if (n <= 0) return MUPSI_OK;
  if (int e = mlp_kernel_attrs()) return e;
  const int64_t tiles = (n + kRows - 1) / kRows;
  const int grid = (int)std::min<int64_t>(tiles, (int64_t)num_sms() * 3);
  k_mlp_infer<<<grid, 128, kInferSmem, st>>>(m->params, m->mc, p, pstride, n, n_dev, out, m->err);
  count_launch();
  MUPSI_CUDA(cudaGetLastError());
  return MUPSI_OK;
}

}  // namespace mupsi

extern "C" {

int mupsi_gpu_mlp_create(const mupsi_mlp_desc* d, mupsi_mlp** out) {
  clear_error();
  if (!d || !out || !d->params) return fail(MUPSI_ERR_INVALID, "null argument");
  *out = nullptr;
  if (!(d->y_scale > 0.0f) || !std::isfinite(d->y_scale)) return fail(MUPSI_ERR_INVALID, "y_scale must be positive");
  std::unique_ptr<mupsi_mlp> m(new mupsi_mlp);
  std::memcpy(m->mc.B, d->fourier, sizeof m->mc.B);
  std::memcpy(m->mc.c, d->center, sizeof m->mc.c);
  m->mc.ys = d->y_scale;
  const size_t bytes = MUPSI_MLP_PARAMS * sizeof(float);
  MUPSI_CUDA(cudaMalloc((void**)&m->params, bytes));
  MUPSI_CUDA(cudaMalloc((void**)&m->grad, bytes));
  MUPSI_CUDA(cudaMalloc((void**)&m->adam_m, bytes));
  MUPSI_CUDA(cudaMalloc((void**)&m->adam_v, bytes));
  MUPSI_CUDA(cudaMalloc((void**)&m->err, sizeof(int)));
  MUPSI_CUDA(cudaMemcpy(m->params, d->params, bytes, cudaMemcpyHostToDevice));
  MUPSI_CUDA(cudaMemset(m->grad, 0, bytes));
  MUPSI_CUDA(cudaMemset(m->adam_m, 0, bytes));
  MUPSI_CUDA(cudaMemset(m->adam_v, 0, bytes));
  MUPSI_CUDA(cudaMemset(m->err, 0, sizeof(int)));
  *out = m.release();
  return MUPSI_OK;
}

int mupsi_gpu_mlp_destroy(mupsi_mlp* m) {
  clear_error();
  if (m) {
    cudaDeviceSynchronize();
    delete m;
  }
  return MUPSI_OK;
}

int mupsi_gpu_mlp_get_params(mupsi_mlp* m, float* out) {
  clear_error();
  if (!m || !out) return fail(MUPSI_ERR_INVALID, "null argument");
  MUPSI_CUDA(cudaDeviceSynchronize());
  MUPSI_CUDA(cudaMemcpy(out, m->params, MUPSI_MLP_PARAMS * sizeof(float), cudaMemcpyDeviceToHost));
  return MUPSI_OK;
}

int mupsi_gpu_mlp_infer(mupsi_mlp* m, int64_t n, const float* p, float* out, mupsi_mem mem, void* stream) {
  clear_error();
  if (!m || n < 0) return fail(MUPSI_ERR_INVALID, "bad argument");
  if (n == 0) return MUPSI_OK;
  if (!p || !out) return fail(MUPSI_ERR_INVALID, "null buffer");
  cudaStream_t st = resolve_stream(stream);
  Staged<float> dp(st), dout(st);
  MUPSI_CUDA(dp.in(p, n * 3, mem));
  MUPSI_CUDA(dout.out(out, n, mem));
  if (int e = mlp_infer_device(m, n, dp.ptr, 3, nullptr, dout.ptr, st)) return e;
  MUPSI_CUDA(dout.finish());
  return mlp_check_err(m, st);
}

int mupsi_gpu_mlp_grad(mupsi_mlp* m, int64_t n, const float* p, const float* t, float* grad_out, float* loss_out,
                       mupsi_mem mem, void* stream) {
  clear_error();
  if (!m || n <= 0 || !p || !t || !grad_out || !loss_out) return fail(MUPSI_ERR_INVALID, "bad argument");
  cudaStream_t st = resolve_stream(stream);
  Staged<float> dp(st), dt(st);
  MUPSI_CUDA(dp.in(p, n * 3, mem));
  MUPSI_CUDA(dt.in(t, n, mem));
  float* g = nullptr;
  MUPSI_CUDA(cudaMallocAsync((void**)&g, (MUPSI_MLP_PARAMS + 1) * sizeof(float), st));
  MUPSI_CUDA(cudaMemsetAsync(g, 0, (MUPSI_MLP_PARAMS + 1) * sizeof(float), st));
  int rc = mlp_launch_grad(m, n, dp.ptr, dt.ptr, g, g + MUPSI_MLP_PARAMS, st);
  std::unique_ptr<float[]> h(new float[MUPSI_MLP_PARAMS + 1]);
  if (rc == MUPSI_OK)
    MUPSI_CUDA(cudaMemcpyAsync(h.get(), g, (MUPSI_MLP_PARAMS + 1) * sizeof(float), cudaMemcpyDeviceToHost, st));
  MUPSI_CUDA(cudaFreeAsync(g, st));
  if (int e = mlp_check_err(m, st)) return e;
  if (rc) return rc;
  std::memcpy(grad_out, h.get(), MUPSI_MLP_PARAMS * sizeof(float));
  *loss_out = h[MUPSI_MLP_PARAMS] / (float)n;
  return MUPSI_OK;
}

int mupsi_gpu_mlp_train(mupsi_mlp* m, int64_t n, const float* p, const float* t, const mupsi_mlp_train_args* a,
                        float* loss_out, mupsi_mem mem, void* stream) {
  clear_error();
  if (!m || !a || n <= 0 || !p || !t) return fail(MUPSI_ERR_INVALID, "bad argument");
  if (a->steps < 0 || a->batch <= 0 || a->batch > (1 << 24)) return fail(MUPSI_ERR_INVALID, "bad steps or batch");
  cudaStream_t st = resolve_stream(stream);
  Staged<float> dp(st), dt(st);
  MUPSI_CUDA(dp.in(p, n * 3, mem));
  MUPSI_CUDA(dt.in(t, n, mem));
  if (a->batch > m->batch_cap) {
    MUPSI_CUDA(cudaStreamSynchronize(st));
    if (m->batch) cudaFree(m->batch);
    m->batch = nullptr;
    MUPSI_CUDA(cudaMalloc((void**)&m->batch, (size_t)a->batch * 4 * sizeof(float)));
    m->batch_cap = a->batch;
  }
  if (a->steps > m->loss_cap) {
    MUPSI_CUDA(cudaStreamSynchronize(st));
    if (m->loss) cudaFree(m->loss);
    m->loss = nullptr;
    MUPSI_CUDA(cudaMalloc((void**)&m->loss, (size_t)std::max(1, a->steps) * sizeof(float)));
    m->loss_cap = a->steps;
  }
  if (a->steps > 0) MUPSI_CUDA(cudaMemsetAsync(m->loss, 0, (size_t)a->steps * sizeof(float), st));
  float* bp = m->batch;
  float* bt = m->batch + 3 * (size_t)a->batch;
  MUPSI_CUDA(cudaMemsetAsync(m->grad, 0, MUPSI_MLP_PARAMS * sizeof(float), st));
  const double pi = 3.14159265358979323846;
  for (int s = 0; s < a->steps; ++s) {
    k_mlp_gather<<<(a->batch + 255) / 256, 256, 0, st>>>(a->seed, s, n, dp.ptr, dt.ptr, a->batch, bp, bt);
    if (int e = mlp_launch_grad(m, a->batch, bp, bt, m->grad, m->loss + s, st)) return e;
    const double frac = a->steps > 1 ? (double)s / (double)(a->steps - 1) : 1.0;
    const float lr = (float)(a->lr_final + 0.5 * (a->lr - a->lr_final) * (1.0 + std::cos(pi * frac)));
    m->adam_t++;
    const float c1 = (float)(1.0 - std::pow((double)a->beta1, (double)m->adam_t));
    const float c2 = (float)(1.0 - std::pow((double)a->beta2, (double)m->adam_t));
    k_mlp_adam<<<(MUPSI_MLP_PARAMS + 255) / 256, 256, 0, st>>>(m->params, m->grad, m->adam_m, m->adam_v,
                                                              MUPSI_MLP_PARAMS, lr, a->beta1, a->beta2, a->eps, c1, c2);
    count_launch(2);
  }
  MUPSI_CUDA(cudaGetLastError());
  if (int e = mlp_check_err(m, st)) return e;
  if (loss_out && a->steps > 0) {
    MUPSI_CUDA(cudaMemcpy(loss_out, m->loss, (size_t)a->steps * sizeof(float), cudaMemcpyDeviceToHost));
    const float inv = 1.0f / (float)a->batch;
    for (int s = 0; s < a->steps; ++s) loss_out[s] *= inv;
  }
  return MUPSI_OK;
}

}  // extern "C"
