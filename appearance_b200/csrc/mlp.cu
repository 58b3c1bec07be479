// Radiance cache: a small MLP that predicts the outgoing radiance of a path
// vertex from its position, direction and material, trained online on the
// radiance the tracer itself measures at path suffixes (include/appearance_cuda.h,
// "radiance cache").  The reference has no radiance cache; this is new.
//
// Network: 144 encoded inputs -> 4 hidden layers of 64 (ReLU) -> 3 outputs
// (exp), no biases; FP16 weights and activations, FP32 accumulation, FP32
// master weights updated by Adam.  Encoding (143 features + 1 zero pad):
// position normalised to the scene box with sin/cos of 12 octaves per axis
// (72), direction as two 32-bin one-blobs of its spherical angles (64),
// roughness, diffuse albedo (3), specular albedo (3).
//
// Inference (k_rc_infer) runs on the 5th-generation tensor cores: one CTA of
// 128 threads holds all weights in shared memory in the K-major core-matrix
// layout, encodes 128 queries into shared memory, and for each layer one
// thread issues tcgen05.mma (M=128, N=64 or 16, K=16 per instruction) with the
// FP32 accumulator in tensor memory; every warp reads its 32 rows back with
// tcgen05.ld, applies ReLU, rounds to FP16 and writes the next layer's
// operand.  Training (k_rc_forward_backward, k_rc_weight_grad, k_rc_adam) runs
// on the CUDA cores in FP32 on the same FP16-rounded weights and activations:
// 2^16 samples per step is a few GFLOP, small beside the frame.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/appearance_cuda.h"
#include "dev_common.cuh"

namespace ap {
namespace {

constexpr int kIn = 144, kHid = 64, kOut = 3, kOutPad = 16;
// FP32 master parameters, row-major [out][in]
constexpr int kOffW0 = 0;
constexpr int kOffW1 = kOffW0 + kHid * kIn;
constexpr int kOffW2 = kOffW1 + kHid * kHid;
constexpr int kOffW3 = kOffW2 + kHid * kHid;
constexpr int kOffW4 = kOffW3 + kHid * kHid;
constexpr int kNumParams = kOffW4 + kOut * kHid;  // 21696
static_assert(kNumParams == AP_RC_NUM_PARAMS, "parameter count");
// FP16 operands for the tensor cores, K-major core matrices (8 rows x 8 halves,
// 128 bytes each; core matrix (i, j) of an R x K operand at (i * K/8 + j) * 128
// bytes).  W4 is padded to 16 rows (rows 3..15 zero).
constexpr int kPackW0 = 0;
constexpr int kPackW1 = kPackW0 + kHid * kIn;
constexpr int kPackW2 = kPackW1 + kHid * kHid;
constexpr int kPackW3 = kPackW2 + kHid * kHid;
constexpr int kPackW4 = kPackW3 + kHid * kHid;
constexpr int kPackHalves = kPackW4 + kOutPad * kHid;  // 22528 halves = 45056 bytes
constexpr int kTile = 128;                             // queries per CTA tile (MMA M)
constexpr int kSmemWeights = kPackHalves * 2;
constexpr int kSmemAct = kTile * kIn * 2;              // 36864: A0, then the two hidden buffers
constexpr int kSmemInfer = kSmemWeights + kSmemAct + 16;
constexpr int kQueryFloats = 16;

__host__ __device__ inline int core_offset(int row, int k, int K) {
  return ((row >> 3) * (K >> 3) + (k >> 3)) * 64 + (row & 7) * 8 + (k & 7);
}

struct RcBounds {
  float lo[3], inv[3];
};

// Query record (16 floats): position, roughness, direction (unit, outgoing),
// 0, diffuse albedo, specular albedo, 0, 0.
APD void rc_encode(const float* q, const RcBounds& b, float* f) {
  const float kPi = 3.14159265358979323846f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float x = (q[a] - b.lo[a]) * b.inv[a];
    float scale = kPi;
#pragma unroll
    for (int o = 0; o < 12; ++o) {
      float s, c;
      dm::sincos_(x * scale, &s, &c);
      f[a * 24 + 2 * o] = s;
      f[a * 24 + 2 * o + 1] = c;
      scale = scale * 2.0f;
    }
  }
  float th = dm::acos_(dm::clamp(q[6], -1.0f, 1.0f)) * (1.0f / kPi);
  float ph = dm::atan2_(q[5], q[4]) * (0.5f / kPi) + 0.5f;
#pragma unroll
  for (int i = 0; i < 32; ++i) {
    float cth = (th - ((float)i + 0.5f) * (1.0f / 32.0f)) * 32.0f;
    float cph = (ph - ((float)i + 0.5f) * (1.0f / 32.0f)) * 32.0f;
    f[72 + i] = dm::exp_(-0.5f * cth * cth);
    f[104 + i] = dm::exp_(-0.5f * cph * cph);
  }
  f[136] = q[3];
  f[137] = q[8];
  f[138] = q[9];
  f[139] = q[10];
  f[140] = q[11];
  f[141] = q[12];
  f[142] = q[13];
  f[143] = 0.0f;
}

APD float h16(float x) { return __half2float(__float2half_rn(x)); }

// ---- tensor-core inference -------------------------------------------------

APD uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, K-major without swizzle: start address,
// leading byte offset (between the two K-adjacent core matrices of one MMA),
// stride byte offset (between 8-row groups), descriptor version 1.
APD uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor, kind::f16: FP32 accumulator, FP16 A and B, both K-major.
__host__ __device__ constexpr uint32_t mma_idesc(int M, int N) {
  return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

APD void mma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

APD void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// Waits for phase `parity` of the mbarrier with an iteration limit; returns false on timeout.
APD bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (int it = 0; it < (1 << 22); ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

APD void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Writes 8 consecutive features of one row (k0 a multiple of 8) as one 16-byte store.
APD void store_row8(__half* base, int row, int k0, int K, const float* v) {
  __align__(16) __half h[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) h[i] = __float2half_rn(v[i]);
  *reinterpret_cast<uint4*>(base + core_offset(row, k0, K)) = *reinterpret_cast<const uint4*>(h);
}

// One layer of a 128-row tile: thread 0 issues the K/16 MMAs and commits them
// to the mbarrier; every warp then reads its 32 accumulator rows (N columns)
// from tensor memory.  Hidden layers write fp16(relu(.)) as the next layer's
// A operand; the last writes exp() of the 3 outputs.  Returns false (on every
// thread) when the MMA completion wait timed out.
template <int K, int N, bool kLast>
APD bool rc_layer(uint32_t tmem, uint32_t bar, uint32_t& phase, uint32_t a_base, uint32_t b_base, __half* dst, int t,
                  uint32_t row, uint32_t n, float* out) {
  if (t == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    constexpr uint32_t sbo = (uint32_t)(K / 8) * 128;
#pragma unroll
    for (int ks = 0; ks < K / 16; ++ks)
      mma_f16(tmem, smem_desc(a_base + ks * 256, 128, sbo), smem_desc(b_base + ks * 256, 128, sbo), mma_idesc(kTile, N),
              ks > 0 ? 1u : 0u);
    mma_commit(bar);
  }
  const bool bad = !mbar_wait(bar, phase);
  phase ^= 1u;
  if (__syncthreads_or(bad)) return false;
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t taddr = tmem + ((uint32_t)((t >> 5) * 32) << 16);
  float v[N];
#pragma unroll
  for (int c = 0; c < N; c += 16) tmem_ld16(taddr + c, v + c);
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
  if (!kLast) {
#pragma unroll
    for (int k = 0; k < N; k += 8) {
      float r[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) r[i] = fmaxf(v[k + i], 0.0f);
      store_row8(dst, t, k, N, r);
    }
  } else if (row < n) {
#pragma unroll
    for (int c = 0; c < kOut; ++c) out[3 * (size_t)row + c] = dm::exp_(v[c]);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();
  return true;
}

__global__ void __launch_bounds__(kTile, 1) k_rc_infer(const uint4* __restrict__ packed, const float4* __restrict__ queries,
                                                       uint32_t n, RcBounds bounds, float* __restrict__ out,
                                                       uint32_t* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __half* w = reinterpret_cast<__half*>(smem);
  __half* act = reinterpret_cast<__half*>(smem + kSmemWeights);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kSmemWeights + kSmemAct);
  uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(smem + kSmemWeights + kSmemAct + 8);
  const int t = threadIdx.x, warp = t >> 5;
  for (int i = t; i < kSmemWeights / 16; i += kTile) reinterpret_cast<uint4*>(smem)[i] = packed[i];
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_holder)),
                 "r"(64));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_holder;
  const uint32_t bar_a = smem_u32(bar);
  const uint32_t act_a = smem_u32(act), w_a = smem_u32(w);
  __half* h0 = act;                   // hidden buffers alias A0: its MMA has completed when they are written
  __half* h1 = act + kTile * kHid;
  const uint32_t h0_a = act_a, h1_a = act_a + kTile * kHid * 2;
  uint32_t phase = 0;
  bool ok = true;
  const uint32_t tiles = (n + kTile - 1) / kTile;
  for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
    const uint32_t row = tile * kTile + t;
    {  // encode this thread's query into row t of A0 (128 x 144)
      float q[kQueryFloats], f[kIn];
      if (row < n) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          float4 v = queries[4 * (size_t)row + i];
          q[4 * i] = v.x; q[4 * i + 1] = v.y; q[4 * i + 2] = v.z; q[4 * i + 3] = v.w;
        }
        rc_encode(q, bounds, f);
      } else {
#pragma unroll
        for (int i = 0; i < kIn; ++i) f[i] = 0.0f;
      }
#pragma unroll
      for (int k = 0; k < kIn; k += 8) store_row8(act, t, k, kIn, f + k);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    ok = rc_layer<kIn, kHid, false>(tmem, bar_a, phase, act_a, w_a + kPackW0 * 2, h0, t, row, n, out) &&
         rc_layer<kHid, kHid, false>(tmem, bar_a, phase, h0_a, w_a + kPackW1 * 2, h1, t, row, n, out) &&
         rc_layer<kHid, kHid, false>(tmem, bar_a, phase, h1_a, w_a + kPackW2 * 2, h0, t, row, n, out) &&
         rc_layer<kHid, kHid, false>(tmem, bar_a, phase, h0_a, w_a + kPackW3 * 2, h1, t, row, n, out) &&
         rc_layer<kHid, kOutPad, true>(tmem, bar_a, phase, h1_a, w_a + kPackW4 * 2, nullptr, t, row, n, out);
  }
  if (!ok && t == 0) atomicExch(err, 1u);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(64));
}

// ---- training (CUDA cores, FP32 on FP16-rounded weights and activations) ----

// Per sample: h0 = encode (FP16-rounded), h_{l+1} = fp16(relu(W_l h_l)) for
// l = 0..3, y = W4 h4, prediction exp(y).  Relative L2 loss (the prediction in
// the denominator held constant), averaged over samples and channels:
//   L = mean (exp(y) - t)^2 / (exp(y)^2 + 0.01).
// Backward: d4 = dL/dy, d_l = (W_{l+1}^T d_{l+1}) * [h_{l+1} > 0].  Stores
// h_l and d_l for the weight gradients dW_l = sum_s d_l h_l^T.
__global__ void __launch_bounds__(128) k_rc_forward_backward(const float* __restrict__ wf, const float4* __restrict__ queries,
                                                             const float* __restrict__ targets, const uint32_t* __restrict__ n_dev,
                                                             uint32_t cap, RcBounds bounds, float* __restrict__ h,
                                                             float* __restrict__ d, float* __restrict__ loss_sum) {
  extern __shared__ float sw[];
  const uint32_t n = min(*n_dev, cap);
  if (blockIdx.x * blockDim.x >= n) return;
  for (int i = threadIdx.x; i < kNumParams; i += blockDim.x) sw[i] = wf[i];
  __syncthreads();
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  float loss = 0.0f;
  if (s < n) {
    float* hs = h + (size_t)s * (kIn + 4 * kHid);  // h0 (144) then h1..h4 (64 each)
    float* ds = d + (size_t)s * (4 * kHid + kOut);  // d0..d3 (64 each) then d4 (3)
    float q[kQueryFloats], f[kIn];
    for (int i = 0; i < 4; ++i) {
      float4 v = queries[4 * (size_t)s + i];
      q[4 * i] = v.x; q[4 * i + 1] = v.y; q[4 * i + 2] = v.z; q[4 * i + 3] = v.w;
    }
    rc_encode(q, bounds, f);
    for (int i = 0; i < kIn; ++i) hs[i] = h16(f[i]);
    const float* prev = hs;
    int K = kIn;
    const int woff[4] = {kOffW0, kOffW1, kOffW2, kOffW3};
    for (int l = 0; l < 4; ++l) {
      float* cur = hs + kIn + l * kHid;
      for (int o = 0; o < kHid; ++o) {
        const float* wr = sw + woff[l] + o * K;
        float z = 0.0f;
        for (int i = 0; i < K; ++i) z = fmaf(wr[i], prev[i], z);
        cur[o] = h16(fmaxf(z, 0.0f));
      }
      prev = cur;
      K = kHid;
    }
    float y[kOut], dy[kOut];
    const float inv_count = 1.0f / (3.0f * (float)n);
    for (int c = 0; c < kOut; ++c) {
      const float* wr = sw + kOffW4 + c * kHid;
      float z = 0.0f;
      for (int i = 0; i < kHid; ++i) z = fmaf(wr[i], prev[i], z);
      y[c] = z;
      float p = dm::exp_(z), tg = targets[3 * (size_t)s + c];
      float den = p * p + 0.01f;
      loss += (p - tg) * (p - tg) / den;
      dy[c] = 2.0f * (p - tg) / den * p * inv_count;  // through exp
      ds[4 * kHid + c] = dy[c];
    }
    // d3 = (W4^T dy) * [h4 > 0]
    float g[kHid];
    const float* h4 = hs + kIn + 3 * kHid;
    for (int i = 0; i < kHid; ++i) {
      float a = 0.0f;
      for (int c = 0; c < kOut; ++c) a = fmaf(sw[kOffW4 + c * kHid + i], dy[c], a);
      g[i] = h4[i] > 0.0f ? a : 0.0f;
      ds[3 * kHid + i] = g[i];
    }
    const int wnext[3] = {kOffW3, kOffW2, kOffW1};
    for (int l = 2; l >= 0; --l) {  // d_l = (W_{l+1}^T d_{l+1}) * [h_{l+1} > 0]
      const float* hl1 = hs + kIn + l * kHid;
      const float* dn = ds + (l + 1) * kHid;
      const float* W = sw + wnext[2 - l];
      for (int i = 0; i < kHid; ++i) {
        float a = 0.0f;
        for (int o = 0; o < kHid; ++o) a = fmaf(W[o * kHid + i], dn[o], a);
        ds[l * kHid + i] = hl1[i] > 0.0f ? a : 0.0f;
      }
    }
    (void)y;
  }
  // block sum of the loss
  for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss_sum, loss);
}

// dW_l[o][i] += sum over a chunk of samples of d_l[s][o] * h_l[s][i].
__global__ void __launch_bounds__(256) k_rc_weight_grad(const float* __restrict__ h, const float* __restrict__ d,
                                                        const uint32_t* __restrict__ n_dev, uint32_t cap, int layer,
                                                        uint32_t chunk, float* __restrict__ grad) {
  __shared__ float sd[32][kHid];
  __shared__ float sh[32][kIn];
  const uint32_t n = min(*n_dev, cap);
  if (blockIdx.x * chunk >= n) return;
  const int K = layer == 0 ? kIn : kHid, O = layer == 4 ? kOut : kHid;
  const int hoff = layer == 0 ? 0 : kIn + (layer - 1) * kHid;
  const int doff = layer == 4 ? 4 * kHid : layer * kHid;
  const int goff = layer == 0 ? kOffW0 : (layer == 1 ? kOffW1 : (layer == 2 ? kOffW2 : (layer == 3 ? kOffW3 : kOffW4)));
  const uint32_t s0 = blockIdx.x * chunk, s1 = min(n, s0 + chunk);
  constexpr int kPer = (kHid * kIn + 255) / 256;
  float acc[kPer];
  for (int e = 0; e < kPer; ++e) acc[e] = 0.0f;
  for (uint32_t sb = s0; sb < s1; sb += 32) {
    const uint32_t m = min(32u, s1 - sb);
    __syncthreads();
    for (int idx = threadIdx.x; idx < 32 * K; idx += 256) {
      int r = idx / K, c = idx % K;
      sh[r][c] = (uint32_t)r < m ? h[(size_t)(sb + r) * (kIn + 4 * kHid) + hoff + c] : 0.0f;
    }
    for (int idx = threadIdx.x; idx < 32 * O; idx += 256) {
      int r = idx / O, c = idx % O;
      sd[r][c] = (uint32_t)r < m ? d[(size_t)(sb + r) * (4 * kHid + kOut) + doff + c] : 0.0f;
    }
    __syncthreads();
    for (int e = 0; e < kPer; ++e) {
      int idx = threadIdx.x + e * 256;
      if (idx >= O * K) break;
      int o = idx / K, i = idx % K;
      float a = acc[e];
      for (int r = 0; r < 32; ++r) a = fmaf(sd[r][o], sh[r][i], a);
      acc[e] = a;
    }
  }
  for (int e = 0; e < kPer; ++e) {
    int idx = threadIdx.x + e * 256;
    if (idx >= O * K) break;
    atomicAdd(&grad[goff + idx], acc[e]);
  }
}

// Adam on the FP32 master weights, then the FP16-rounded FP32 copy used by
// training and the packed FP16 tensor-core operands.
__global__ void k_rc_adam(float* __restrict__ master, float* __restrict__ m1, float* __restrict__ m2,
                          const float* __restrict__ grad, float lr, float b1, float b2, float eps, float c1, float c2,
                          int update, float* __restrict__ wf, __half* __restrict__ packed) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kNumParams) return;
  float w = master[p];
  if (update) {
    const float g = grad[p];
    const float a = b1 * m1[p] + (1.0f - b1) * g;
    const float b = b2 * m2[p] + (1.0f - b2) * g * g;
    m1[p] = a;
    m2[p] = b;
    w = w - lr * (a / c1) / (sqrtf(b / c2) + eps);
    master[p] = w;
  }
  const __half hw = __float2half_rn(w);
  wf[p] = __half2float(hw);
  int row, k, K, base;
  if (p < kOffW1) { row = p / kIn; k = p % kIn; K = kIn; base = kPackW0; }
  else if (p < kOffW4) { int q = p - kOffW1; int l = q / (kHid * kHid); q %= kHid * kHid; row = q / kHid; k = q % kHid; K = kHid; base = kPackW1 + l * kHid * kHid; }
  else { int q = p - kOffW4; row = q / kHid; k = q % kHid; K = kHid; base = kPackW4; }
  packed[base + core_offset(row, k, K)] = hw;
}

struct Cache {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  RcBounds bounds{};
  float *master = nullptr, *m1 = nullptr, *m2 = nullptr, *grad = nullptr, *wf = nullptr, *loss = nullptr;
  uint32_t* count = nullptr;  // sample count of host-submitted batches
  __half* packed = nullptr;
  uint32_t* err = nullptr;
  int step = 0;
  // batch buffers
  float *h = nullptr, *d = nullptr, *targets = nullptr;
  float4* queries = nullptr;
  float* out = nullptr;
  uint32_t cap = 0;
  std::string msg;
};

int cfail(Cache* c, int code, const std::string& m) {
  if (c) c->msg = m;
  return code;
}

int cuda_ok(Cache* c, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return AP_OK;
  return cfail(c, e == cudaErrorMemoryAllocation ? AP_E_OOM : AP_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int ensure_batch(Cache* c, uint32_t n) {
  if (n <= c->cap) return AP_OK;
  cudaFree(c->h); cudaFree(c->d); cudaFree(c->targets); cudaFree(c->queries); cudaFree(c->out);
  c->h = c->d = c->targets = c->out = nullptr;
  c->queries = nullptr;
  c->cap = 0;
  int rc;
  if ((rc = cuda_ok(c, cudaMalloc(&c->h, (size_t)n * (kIn + 4 * kHid) * 4), "batch")) ||
      (rc = cuda_ok(c, cudaMalloc(&c->d, (size_t)n * (4 * kHid + kOut) * 4), "batch")) ||
      (rc = cuda_ok(c, cudaMalloc(&c->targets, (size_t)n * 12), "batch")) ||
      (rc = cuda_ok(c, cudaMalloc(&c->queries, (size_t)n * 64), "batch")) ||
      (rc = cuda_ok(c, cudaMalloc(&c->out, (size_t)n * 12), "batch")))
    return rc;
  c->cap = n;
  return AP_OK;
}

// Refreshes the FP16 copies from the master weights (no update).
void repack(Cache* c) {
  k_rc_adam<<<(kNumParams + 255) / 256, 256, 0, c->stream>>>(c->master, c->m1, c->m2, c->grad, 0.0f, 0.9f, 0.999f, 1e-8f,
                                                               1.0f, 1.0f, 0, c->wf, c->packed);
}

}  // namespace

// Entry points used by the frame (device pointers, the caller's stream).
int rc_infer_device(void* cp, const float4* queries, uint32_t n, float* out, cudaStream_t st) {
  Cache* c = static_cast<Cache*>(cp);
  if (n == 0) return AP_OK;
  const int tiles = (int)((n + kTile - 1) / kTile);
  const int grid = tiles < 2 * c->num_sms ? tiles : 2 * c->num_sms;
  k_rc_infer<<<grid, kTile, kSmemInfer, st>>>(reinterpret_cast<const uint4*>(c->packed), queries, n, c->bounds, out, c->err);
  return cuda_ok(c, cudaGetLastError(), "radiance cache inference");
}

// Training step on at most `cap` samples; the sample count is read from device
// memory (n_dev), so a batch assembled on the device needs no host round trip.
int rc_train_device(void* cp, const float4* queries, const float* targets, const uint32_t* n_dev, uint32_t cap, float lr,
                    int update, cudaStream_t st) {
  Cache* c = static_cast<Cache*>(cp);
  if (cap == 0) return AP_OK;
  int rc = ensure_batch(c, cap);
  if (rc) return rc;
  cudaMemsetAsync(c->grad, 0, kNumParams * 4, st);
  cudaMemsetAsync(c->loss, 0, 4, st);
  k_rc_forward_backward<<<(cap + 127) / 128, 128, kNumParams * 4, st>>>(c->wf, queries, targets, n_dev, cap, c->bounds,
                                                                       c->h, c->d, c->loss);
  const uint32_t chunk = 1024;
  for (int l = 0; l < 5; ++l)
    k_rc_weight_grad<<<(cap + chunk - 1) / chunk, 256, 0, st>>>(c->h, c->d, n_dev, cap, l, chunk, c->grad);
  if (update) {
    c->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - (float)std::pow(0.9, c->step), c2 = 1.0f - (float)std::pow(0.999, c->step);
    k_rc_adam<<<(kNumParams + 255) / 256, 256, 0, st>>>(c->master, c->m1, c->m2, c->grad, lr, b1, b2, 1e-8f, c1, c2, 1,
                                                        c->wf, c->packed);
  }
  return cuda_ok(c, cudaGetLastError(), "radiance cache training");
}

}  // namespace ap

using ap::Cache;

extern "C" {

void* ap_rc_create(int device, const float* scene_lo, const float* scene_hi, uint32_t seed, int* err) {
  if (err) *err = AP_OK;
  int n = 0;
  if (!scene_lo || !scene_hi || cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
    cudaGetLastError();
    if (err) *err = scene_lo && scene_hi ? AP_E_CUDA : AP_E_INVALID;
    return nullptr;
  }
  cudaSetDevice(device);
  Cache* c = new Cache;
  c->device = device;
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
  for (int a = 0; a < 3; ++a) {
    c->bounds.lo[a] = scene_lo[a];
    float ext = scene_hi[a] - scene_lo[a];
    c->bounds.inv[a] = ext > 0.0f ? 1.0f / ext : 0.0f;
  }
  int rc = AP_OK;
  if ((rc = ap::cuda_ok(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "stream")) ||
      (rc = ap::cuda_ok(c, cudaMalloc(&c->master, ap::kNumParams * 4), "params")) ||
      (rc = ap::cuda_ok(c, cudaMalloc(&c->m1, ap::kNumParams * 4), "params")) ||
      (rc = ap::cuda_ok(c, cudaMalloc(&c->m2, ap::kNumParams * 4), "params")) ||
      (rc = ap::cuda_ok(c, cudaMalloc(&c->grad, ap::kNumParams * 4), "params")) ||
      (rc = ap::cuda_ok(c, cudaMalloc(&c->wf, ap::kNumParams * 4), "params")) ||
      (rc = ap::cuda_ok(c, cudaMalloc(&c->loss, 4), "params")) ||
      (rc = ap::cuda_ok(c, cudaMalloc(&c->err, 4), "params")) ||
      (rc = ap::cuda_ok(c, cudaMalloc(&c->count, 4), "params")) ||
      (rc = ap::cuda_ok(c, cudaMalloc(&c->packed, ap::kPackHalves * 2), "params")) ||
      (rc = ap::cuda_ok(c, cudaFuncSetAttribute(ap::k_rc_infer, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                ap::kSmemInfer), "smem")) ||
      (rc = ap::cuda_ok(c, cudaFuncSetAttribute(ap::k_rc_forward_backward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                ap::kNumParams * 4), "smem"))) {
    if (err) *err = rc;
    ap_rc_destroy(c);
    return nullptr;
  }
  // He-uniform initialisation from a seeded LCG (host), FP32 master weights
  std::vector<float> w(ap::kNumParams);
  uint64_t st = 0x9E3779B97F4A7C15ull ^ ((uint64_t)seed * 0xD1B54A32D192ED03ull);
  auto uni = [&]() {
    st = st * 6364136223846793005ull + 1442695040888963407ull;
    return (float)((st >> 40) * (1.0 / 16777216.0)) * 2.0f - 1.0f;
  };
  const int fan_in[5] = {ap::kIn, ap::kHid, ap::kHid, ap::kHid, ap::kHid};
  const int off[6] = {ap::kOffW0, ap::kOffW1, ap::kOffW2, ap::kOffW3, ap::kOffW4, ap::kNumParams};
  for (int l = 0; l < 5; ++l) {
    float bound = std::sqrt(6.0f / (float)fan_in[l]) * (l == 4 ? 0.1f : 1.0f);
    for (int p = off[l]; p < off[l + 1]; ++p) w[p] = uni() * bound;
  }
  ap_rc_set_params(c, w.data(), ap::kNumParams);
  cudaMemset(c->err, 0, 4);
  return c;
}

void ap_rc_destroy(void* cp) {
  Cache* c = static_cast<Cache*>(cp);
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  void* ptrs[] = {c->master, c->m1, c->m2, c->grad, c->wf, c->loss, c->err, c->count, c->packed, c->h, c->d, c->targets,
                  c->queries, c->out};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

const char* ap_rc_last_error(const void* cp) {
  const Cache* c = static_cast<const Cache*>(cp);
  return c ? c->msg.c_str() : "null cache";
}

int ap_rc_set_params(void* cp, const float* params, uint32_t count) {
  Cache* c = static_cast<Cache*>(cp);
  if (!c || !params || count != ap::kNumParams) return ap::cfail(c, AP_E_INVALID, "parameter count");
  cudaSetDevice(c->device);
  int rc;
  if ((rc = ap::cuda_ok(c, cudaMemcpy(c->master, params, ap::kNumParams * 4, cudaMemcpyHostToDevice), "params")))
    return rc;
  cudaMemsetAsync(c->m1, 0, ap::kNumParams * 4, c->stream);
  cudaMemsetAsync(c->m2, 0, ap::kNumParams * 4, c->stream);
  cudaMemsetAsync(c->packed, 0, ap::kPackHalves * 2, c->stream);
  c->step = 0;
  ap::repack(c);
  return ap::cuda_ok(c, cudaStreamSynchronize(c->stream), "params");
}

int ap_rc_get_params(void* cp, float* params, uint32_t count) {
  Cache* c = static_cast<Cache*>(cp);
  if (!c || !params || count != ap::kNumParams) return ap::cfail(c, AP_E_INVALID, "parameter count");
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  return ap::cuda_ok(c, cudaMemcpy(params, c->master, ap::kNumParams * 4, cudaMemcpyDeviceToHost), "params");
}

int ap_rc_infer(void* cp, const float* queries, uint32_t n, float* out_rgb) {
  Cache* c = static_cast<Cache*>(cp);
  if (!c || (n && (!queries || !out_rgb))) return ap::cfail(c, AP_E_INVALID, "null buffer");
  if (n == 0) return AP_OK;
  cudaSetDevice(c->device);
  int rc = ap::ensure_batch(c, n);
  if (rc) return rc;
  cudaMemcpyAsync(c->queries, queries, (size_t)n * 64, cudaMemcpyHostToDevice, c->stream);
  if ((rc = ap::rc_infer_device(c, c->queries, n, c->out, c->stream))) return rc;
  cudaMemcpyAsync(out_rgb, c->out, (size_t)n * 12, cudaMemcpyDeviceToHost, c->stream);
  uint32_t e = 0;
  cudaMemcpyAsync(&e, c->err, 4, cudaMemcpyDeviceToHost, c->stream);
  if ((rc = ap::cuda_ok(c, cudaStreamSynchronize(c->stream), "radiance cache inference"))) return rc;
  if (e) return ap::cfail(c, AP_E_TIMEOUT, "radiance cache inference: tensor-core wait timed out");
  return AP_OK;
}

int ap_rc_train(void* cp, const float* queries, const float* targets, uint32_t n, float lr, int update, float* loss,
                float* grad_out) {
  Cache* c = static_cast<Cache*>(cp);
  if (!c || (n && (!queries || !targets))) return ap::cfail(c, AP_E_INVALID, "null buffer");
  if (n == 0) return AP_OK;
  cudaSetDevice(c->device);
  int rc = ap::ensure_batch(c, n);
  if (rc) return rc;
  cudaMemcpyAsync(c->queries, queries, (size_t)n * 64, cudaMemcpyHostToDevice, c->stream);
  cudaMemcpyAsync(c->targets, targets, (size_t)n * 12, cudaMemcpyHostToDevice, c->stream);
  cudaMemcpyAsync(c->count, &n, 4, cudaMemcpyHostToDevice, c->stream);
  if ((rc = ap::rc_train_device(c, c->queries, c->targets, c->count, n, lr, update, c->stream))) return rc;
  float l = 0.0f;
  cudaMemcpyAsync(&l, c->loss, 4, cudaMemcpyDeviceToHost, c->stream);
  if (grad_out) cudaMemcpyAsync(grad_out, c->grad, ap::kNumParams * 4, cudaMemcpyDeviceToHost, c->stream);
  if ((rc = ap::cuda_ok(c, cudaStreamSynchronize(c->stream), "radiance cache training"))) return rc;
  if (loss) *loss = l / (3.0f * (float)n);
  return AP_OK;
}

}  // extern "C"
