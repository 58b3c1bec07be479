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
// 256 threads (two per query row) holds all weights in shared memory in the
// K-major core-matrix layout, encodes 128 queries into shared memory, and for
// each layer one thread issues tcgen05.mma (M=128, N=64 or 16, K=16 per
// instruction) with the FP32 accumulator in tensor memory; the warps read
// their rows back with tcgen05.ld (each thread half of a row's columns),
// apply ReLU, round to FP16 and write the next layer's operand.  Training (k_rc_train_tc) runs forward and backward on the tensor
// cores in one kernel per step, tile by tile with the weight-gradient sums in
// tensor memory, one gradient row per CTA; k_rc_grad_sum adds the rows in a
// fixed order and k_rc_adam updates the FP32 master weights and repacks the
// FP16 operands (forward and transposed).
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/appearance_cuda.h"
#include "dev_common.cuh"
#include "device_scope.h"

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
// Transposed copies for the backward pass (W_l^T as the B operand of
// dH_l = dZ_l W_l: rows = the layer's inputs, K = its outputs), W1..W4; W4^T's
// K is padded to 16 (outputs 3..15 zero).
constexpr int kPackT1 = kPackHalves;
constexpr int kPackT4 = kPackT1 + 3 * kHid * kHid;
constexpr int kPackTHalves = 3 * kHid * kHid + kHid * kOutPad;  // 13312 halves = 26624 bytes
constexpr int kPackAllHalves = kPackHalves + kPackTHalves;
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
// 0, diffuse albedo, specular albedo, 0, 0.  The 144 features go to
// sink(k, value).  Octave o of each position axis is sin/cos(2^o pi x), by the
// double-angle recurrence from o = 0.  Each one-blob bin i holds
// exp(-0.5 c_i^2), c_i = (v - (i + 0.5)/32) * 32; only the 13 bins around the
// peak are evaluated (written after zeroing all 32): farther bins are below
// half the smallest FP16 subnormal, so their FP16 value is 0 either way.  The
// elementary functions are the deterministic ones the oracle's encoding uses,
// so the FP16 features match it bit for bit (hardware-rate functions flip
// enough FP16 roundings to move the weight gradients by ~1e-3).
// The two threads of a query row share its encoding, balanced by their
// elementary functions: rc_encode_part<0> writes the x and y position
// features and the polar-angle one-blob (two sincos, one acos, 13 exps),
// rc_encode_part<1> the z position features, the azimuth one-blob and the
// material tail (one sincos, one atan2, 13 exps); rc_encode writes all of them.
template <class Sink>
APD void rc_encode_axis(const float* q, const RcBounds& b, int a, Sink& sink) {
  const float kPi = 3.14159265358979323846f;
  const float x = (q[a] - b.lo[a]) * b.inv[a];
  float s, c;
  dm::sincos_(x * kPi, &s, &c);
#pragma unroll
  for (int o = 0; o < 12; ++o) {
    sink(a * 24 + 2 * o, s);
    sink(a * 24 + 2 * o + 1, c);
    const float s2 = 2.0f * s * c, c2 = 1.0f - 2.0f * s * s;
    s = s2;
    c = c2;
  }
}

// One-blob j of the direction: 0 the polar angle / pi, 1 the azimuth / (2 pi) + 1/2.
template <int j, class Sink>
APD void rc_encode_blob(const float* q, Sink& sink) {
  const float kPi = 3.14159265358979323846f;
  const float v = j == 0 ? dm::acos_(dm::clamp(q[6], -1.0f, 1.0f)) * (1.0f / kPi)
                         : dm::atan2_(q[5], q[4]) * (0.5f / kPi) + 0.5f;
#pragma unroll
  for (int i = 0; i < 32; ++i) sink(72 + 32 * j + i, 0.0f);
  const int b0 = min(max((int)floorf(v * 32.0f), 0), 31);
#pragma unroll
  for (int w = -6; w <= 6; ++w) {
    const int i = b0 + w;
    if (i < 0 || i > 31) continue;
    const float ci = (v - ((float)i + 0.5f) * (1.0f / 32.0f)) * 32.0f;
    sink(72 + 32 * j + i, dm::exp_(-0.5f * ci * ci));
  }
}

template <int kPart, class Sink>
APD void rc_encode_part(const float* q, const RcBounds& b, Sink sink) {
  if (kPart == 0) {
    rc_encode_axis(q, b, 0, sink);
    rc_encode_axis(q, b, 1, sink);
    rc_encode_blob<0>(q, sink);
    return;
  }
  rc_encode_axis(q, b, 2, sink);
  rc_encode_blob<1>(q, sink);
  sink(136, q[3]);
  sink(137, q[8]);
  sink(138, q[9]);
  sink(139, q[10]);
  sink(140, q[11]);
  sink(141, q[12]);
  sink(142, q[13]);
  sink(143, 0.0f);
}

template <class Sink>
APD void rc_encode(const float* q, const RcBounds& b, Sink sink) {
  rc_encode_part<0>(q, b, sink);
  rc_encode_part<1>(q, b, sink);
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
APD bool mbar_wait(uint32_t bar, uint32_t parity, int limit = 1 << 22) {
  for (int it = 0; it < limit; ++it) {
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

// Self-test of the bounded wait, with no tensor-core work: a barrier that
// nothing arrives on must give up after `limit` tries and say so (out[0] = 0);
// one that the thread itself arrived on must complete (out[1] = 1).
__global__ void k_wait_selftest(int limit, uint32_t* out) {
  __shared__ __align__(8) uint64_t bar[2];
  if (threadIdx.x != 0) return;
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar[0])));
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar[1])));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  out[0] = mbar_wait(smem_u32(&bar[0]), 0u, limit) ? 1u : 0u;
  uint64_t state;
  asm volatile("mbarrier.arrive.shared::cta.b64 %0, [%1];" : "=l"(state) : "r"(smem_u32(&bar[1])) : "memory");
  out[1] = mbar_wait(smem_u32(&bar[1]), 0u, limit) ? 1u : 0u;
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
// Two threads share each query row: `half` 0 takes the first half of a hidden
// layer's columns (and the outputs), half 1 the second; their warps read the
// same tensor-memory lane quarter.
template <int K, int N, bool kLast>
APD bool rc_layer(uint32_t tmem, uint32_t bar, uint32_t& phase, uint32_t a_base, uint32_t b_base, __half* dst, int tid,
                  int t, int half, uint32_t row, uint32_t n, float* out) {
  if (tid == 0) {
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
  const uint32_t taddr = tmem + ((uint32_t)(((tid >> 5) & 3) * 32) << 16);
  if (!kLast) {
    constexpr int kCols = N / 2;
    float v[kCols];
#pragma unroll
    for (int c = 0; c < kCols; c += 16) tmem_ld16(taddr + half * kCols + c, v + c);
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < kCols; k += 8) {
      float r[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) r[i] = fmaxf(v[k + i], 0.0f);
      store_row8(dst, t, half * kCols + k, N, r);
    }
  } else if (half == 0) {
    float v[16];
    tmem_ld16(taddr, v);
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    if (row < n)
#pragma unroll
      for (int c = 0; c < kOut; ++c) out[3 * (size_t)row + c] = dm::exp_(v[c]);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();
  return true;
}

__global__ void __launch_bounds__(2 * kTile, 1) k_rc_infer(const uint4* __restrict__ packed, const float4* __restrict__ queries,
                                                       uint32_t n, RcBounds bounds, float* __restrict__ out,
                                                       uint32_t* __restrict__ err, const uint32_t* __restrict__ n_dev) {
  if (n_dev) n = min(n, *n_dev);  // a query count produced on the device (at most n)
  extern __shared__ __align__(1024) unsigned char smem[];
  __half* w = reinterpret_cast<__half*>(smem);
  __half* act = reinterpret_cast<__half*>(smem + kSmemWeights);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kSmemWeights + kSmemAct);
  uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(smem + kSmemWeights + kSmemAct + 8);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int t = tid & (kTile - 1), half = tid >> 7;  // the query row, and which half of it
  for (int i = tid; i < kSmemWeights / 16; i += 2 * kTile) reinterpret_cast<uint4*>(smem)[i] = packed[i];
  if (tid == 0) {
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
      float q[kQueryFloats];
      if (row < n) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          float4 v = queries[4 * (size_t)row + i];
          q[4 * i] = v.x; q[4 * i + 1] = v.y; q[4 * i + 2] = v.z; q[4 * i + 3] = v.w;
        }
        auto sink = [&](int k, float x) { act[core_offset(t, k, kIn)] = __float2half_rn(x); };
        if (half == 0) rc_encode_part<0>(q, bounds, sink);
        else rc_encode_part<1>(q, bounds, sink);
      } else if (half == 0) {
#pragma unroll
        for (int k = 0; k < kIn; k += 8) *reinterpret_cast<uint4*>(act + core_offset(t, k, kIn)) = make_uint4(0, 0, 0, 0);
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    ok = rc_layer<kIn, kHid, false>(tmem, bar_a, phase, act_a, w_a + kPackW0 * 2, h0, tid, t, half, row, n, out) &&
         rc_layer<kHid, kHid, false>(tmem, bar_a, phase, h0_a, w_a + kPackW1 * 2, h1, tid, t, half, row, n, out) &&
         rc_layer<kHid, kHid, false>(tmem, bar_a, phase, h1_a, w_a + kPackW2 * 2, h0, tid, t, half, row, n, out) &&
         rc_layer<kHid, kHid, false>(tmem, bar_a, phase, h0_a, w_a + kPackW3 * 2, h1, tid, t, half, row, n, out) &&
         rc_layer<kHid, kOutPad, true>(tmem, bar_a, phase, h1_a, w_a + kPackW4 * 2, nullptr, tid, t, half, row, n, out);
  }
  if (!ok && tid == 0) atomicExch(err, 1u);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(64));
}

// ---- training on the tensor cores -------------------------------------------
//
// k_rc_train_tc: one CTA of 256 threads (two per sample row) takes whole
// 128-sample tiles.  Per tile it runs the forward layers as k_rc_infer does,
// keeping each hidden activation (the next layer's operand) and its
// transpose (an operand of the weight gradient), then the loss and its
// gradient per sample, then the backward layers:
//   dH_l = dZ_l W_l       M = 128 samples, N = the layer's inputs, K = its
//                         outputs (B = the packed W_l^T);
//   dW_l += dZ_l^T H_l    M = 128 rows, N = the layer's inputs, K = the tile's
//                         128 samples;
//   dZ_{l-1} = dH_l * [H_l > 0].
// Tensor-core operands are FP16.  A gradient value x enters as two FP16
// numbers, hi = fp16(x) and lo = fp16(x - hi), about 21 significant bits
// together: dH_l takes two MMAs (hi, then lo, into one accumulator), and the
// A operand of dW_l stacks the 64 outputs' hi rows over their lo rows, the two
// halves of the sum being added when it is read out.  The activations H_l are
// FP16 values already (the model rounds them).  So the products and their
// FP32 sums keep the precision of an FP32 backward pass.  The weight-gradient
// sums stay in tensor memory over all of the CTA's tiles and are stored to the
// CTA's own gradient row at the end; k_rc_grad_sum adds the rows in a fixed
// order, so a step's gradient is reproducible bit for bit.  The per-sample loss
// gradient enters without the mean's 1 / (3n), which is applied to the sums
// (the FP16 operands stay clear of underflow); a value beyond the FP16 range
// (65504) is clamped there.
constexpr int kTrainR = kPackAllHalves * 2;           // A0, H_l ping-pong, dY and dZ rows, H0^T
constexpr int kTrainHT = kTrainR + kTile * kIn * 2;   // H1^T .. H4^T, kHid x kTile each
constexpr int kTrainHTBytes = kHid * kTile * 2;
constexpr int kTrainDZT = kTrainHT + 4 * kTrainHTBytes;  // [dZ^T hi; dZ^T lo], 128 x kTile
constexpr int kTrainBar = kTrainDZT + 2 * kHid * kTile * 2;
constexpr int kSmemTrain = kTrainBar + 16;
static_assert(kSmemTrain <= 227 * 1024, "training shared memory");
// tensor-memory columns: the layer accumulator, then the weight-gradient sums
constexpr uint32_t kColLayer = 0, kColDW4 = 64, kColDW3 = 128, kColDW2 = 192, kColDW1 = 256, kColDW0 = 320;

APD void split_half(float x, __half* hi, __half* lo) {
  x = fminf(fmaxf(x, -65504.0f), 65504.0f);
  const __half h = __float2half_rn(x);
  *hi = h;
  *lo = __float2half_rn(x - __half2float(h));
}

// `steps` MMAs of K = 16 over K-major operands (stride byte offsets sbo_a,
// sbo_b between 8-row groups); the first overwrites the accumulator unless acc.
APD void mma_steps(uint32_t d, uint32_t a, uint32_t sbo_a, uint32_t b, uint32_t sbo_b, int steps, uint32_t idesc,
                   bool acc) {
  for (int ks = 0; ks < steps; ++ks)
    mma_f16(d, smem_desc(a + ks * 256, 128, sbo_a), smem_desc(b + ks * 256, 128, sbo_b), idesc,
            (acc || ks > 0) ? 1u : 0u);
}

// Shared-memory operands written by all threads, handed to the tensor core.
APD void operands_ready() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Thread 0 commits the MMAs it issued; all wait for them (bounded).  Returns
// false on every thread when the wait ran out.
APD bool mmas_done(uint32_t bar, uint32_t& phase, int t) {
  if (t == 0) mma_commit(bar);
  const bool bad = !mbar_wait(bar, phase);
  phase ^= 1u;
  const bool any_bad = __syncthreads_or(bad);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  return !any_bad;
}

// Two threads share each sample row: `half` 0 takes the first 32 columns of
// a 64-wide layer, half 1 the other 32 (their warps read the same tensor-
// memory lane quarter).
constexpr int kTrainThreads = 2 * kTile;
constexpr int kHalfCols = kHid / 2;

// This thread's 32 columns of the layer accumulator, in its row.
APD void layer_row(uint32_t lane_addr, int half, float* v) {
#pragma unroll
  for (int c = 0; c < kHalfCols; c += 16) tmem_ld16(lane_addr + kColLayer + half * kHalfCols + c, v + c);
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

APD void store_row8h(__half* base, int row, int k0, int K, const __half* h) {
  *reinterpret_cast<uint4*>(base + core_offset(row, k0, K)) = *reinterpret_cast<const uint4*>(h);
}

// Forward epilogue of a hidden layer: H = fp16(relu(acc)) as the next layer's
// A operand (row t of `next`) and into column t of its transpose `ht`.
APD void train_fwd_epilogue(uint32_t lane_addr, __half* next, __half* ht, int t, int half) {
  float v[kHalfCols];
  layer_row(lane_addr, half, v);
#pragma unroll
  for (int k = 0; k < kHalfCols; k += 8) {
    __align__(16) __half h[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      h[i] = __float2half_rn(fmaxf(v[k + i], 0.0f));
      ht[core_offset(half * kHalfCols + k + i, t, kTile)] = h[i];
    }
    store_row8h(next, t, half * kHalfCols + k, kHid, h);
  }
}

// Backward epilogue: dZ = dH * [H > 0] from the layer accumulator and the
// mask of ht (H's transpose); hi / lo rows into dz_hi / dz_lo (when given) and
// columns into [dZ^T hi; dZ^T lo].
APD void train_bwd_epilogue(uint32_t lane_addr, const __half* ht, __half* dz_hi, __half* dz_lo, __half* dzt, int t,
                               int half) {
  float v[kHalfCols];
  layer_row(lane_addr, half, v);
#pragma unroll
  for (int k0 = 0; k0 < kHalfCols; k0 += 8) {
    const int k = half * kHalfCols + k0;
    __align__(16) __half hi[8];
    __align__(16) __half lo[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int c = k + i;
      const float x = __half2float(ht[core_offset(c, t, kTile)]) > 0.0f ? v[k0 + i] : 0.0f;
      split_half(x, &hi[i], &lo[i]);
      dzt[core_offset(c, t, kTile)] = hi[i];
      dzt[core_offset(kHid + c, t, kTile)] = lo[i];
    }
    if (dz_hi) {
      store_row8h(dz_hi, t, k, kHid, hi);
      store_row8h(dz_lo, t, k, kHid, lo);
    }
  }
}

__global__ void __launch_bounds__(kTrainThreads, 1) k_rc_train_tc(const uint4* __restrict__ packed,
                                                          const float4* __restrict__ queries,
                                                          const float* __restrict__ targets,
                                                          const uint32_t* __restrict__ n_dev, uint32_t cap,
                                                          RcBounds bounds, float* __restrict__ parts,
                                                          float* __restrict__ loss_parts, uint32_t* __restrict__ err) {
  const uint32_t n = min(*n_dev, cap);
  extern __shared__ __align__(1024) unsigned char smem[];
  const int tid = threadIdx.x, warp = tid >> 5;
  const int t = tid & (kTile - 1), half = tid >> 7;  // the sample row, and which half of it
  for (int i = tid; i < kPackAllHalves / 8; i += kTrainThreads) reinterpret_cast<uint4*>(smem)[i] = packed[i];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kTrainBar);
  uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(smem + kTrainBar + 8);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_holder)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_holder;
  const uint32_t lane_addr = tmem + ((uint32_t)((warp & 3) * 32) << 16);
  const uint32_t bar_a = smem_u32(bar);
  const uint32_t w_a = smem_u32(smem), r_a = smem_u32(smem + kTrainR), dzt_a = smem_u32(smem + kTrainDZT);
  __half* r = reinterpret_cast<__half*>(smem + kTrainR);
  __half* p0 = r;                // H1, H3, dZ hi rows
  __half* p1 = r + kTile * kHid;  // H2, H4, dZ lo rows
  __half* dzt = reinterpret_cast<__half*>(smem + kTrainDZT);
  __half* ht[4];
  uint32_t ht_a[4];
  for (int l = 0; l < 4; ++l) {
    ht[l] = reinterpret_cast<__half*>(smem + kTrainHT + l * kTrainHTBytes);
    ht_a[l] = smem_u32(ht[l]);
  }
  const uint32_t p0_a = r_a, p1_a = r_a + kTile * kHid * 2;
  const uint32_t sbo64 = (kHid / 8) * 128, sbo144 = (kIn / 8) * 128, sbo16 = (kOutPad / 8) * 128,
                 sbo_s = (kTile / 8) * 128;
  const uint32_t id64 = mma_idesc(kTile, kHid), id16 = mma_idesc(kTile, kOutPad), id144 = mma_idesc(kTile, kIn);
  const uint32_t wt_a[5] = {0u, w_a + kPackT1 * 2, w_a + (kPackT1 + kHid * kHid) * 2,
                            w_a + (kPackT1 + 2 * kHid * kHid) * 2, w_a + kPackT4 * 2};
  uint32_t phase = 0;
  bool ok = true, first = true;
  float loss = 0.0f;
  const uint32_t tiles = (n + kTile - 1) / kTile;
  for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
    const uint32_t row = tile * kTile + t;
    float q[kQueryFloats];
    if (row < n) {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const float4 v = queries[4 * (size_t)row + i];
        q[4 * i] = v.x; q[4 * i + 1] = v.y; q[4 * i + 2] = v.z; q[4 * i + 3] = v.w;
      }
      auto sink = [&](int k, float x) { r[core_offset(t, k, kIn)] = __float2half_rn(x); };
      if (half == 0) rc_encode_part<0>(q, bounds, sink);
      else rc_encode_part<1>(q, bounds, sink);
    } else if (half == 0) {
#pragma unroll
      for (int k = 0; k < kIn; k += 8) *reinterpret_cast<uint4*>(r + core_offset(t, k, kIn)) = make_uint4(0, 0, 0, 0);
    }
    // forward: H1 .. H4
    operands_ready();
    if (tid == 0) mma_steps(tmem + kColLayer, r_a, sbo144, w_a + kPackW0 * 2, sbo144, kIn / 16, id64, false);
    if (!(ok = mmas_done(bar_a, phase, tid))) break;
    train_fwd_epilogue(lane_addr, p0, ht[0], t, half);
    operands_ready();
    if (tid == 0) mma_steps(tmem + kColLayer, p0_a, sbo64, w_a + kPackW1 * 2, sbo64, kHid / 16, id64, false);
    if (!(ok = mmas_done(bar_a, phase, tid))) break;
    train_fwd_epilogue(lane_addr, p1, ht[1], t, half);
    operands_ready();
    if (tid == 0) mma_steps(tmem + kColLayer, p1_a, sbo64, w_a + kPackW2 * 2, sbo64, kHid / 16, id64, false);
    if (!(ok = mmas_done(bar_a, phase, tid))) break;
    train_fwd_epilogue(lane_addr, p0, ht[2], t, half);
    operands_ready();
    if (tid == 0) mma_steps(tmem + kColLayer, p0_a, sbo64, w_a + kPackW3 * 2, sbo64, kHid / 16, id64, false);
    if (!(ok = mmas_done(bar_a, phase, tid))) break;
    train_fwd_epilogue(lane_addr, p1, ht[3], t, half);
    operands_ready();
    if (tid == 0) mma_steps(tmem + kColLayer, p1_a, sbo64, w_a + kPackW4 * 2, sbo64, kHid / 16, id16, false);
    if (!(ok = mmas_done(bar_a, phase, tid))) break;
    // output layer: loss and its gradient per sample (without the 1 / (3n))
    for (int i = tid; i < 2 * kHid * kTile / 8; i += kTrainThreads) reinterpret_cast<uint4*>(dzt)[i] = make_uint4(0, 0, 0, 0);
    __syncthreads();
    if (half == 0) {
      float v[16];
      tmem_ld16(lane_addr + kColLayer, v);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      __align__(16) __half hi[16];
      __align__(16) __half lo[16];
#pragma unroll
      for (int c = 0; c < 16; ++c) {
        hi[c] = __float2half_rn(0.0f);
        lo[c] = hi[c];
      }
      if (row < n) {
#pragma unroll
        for (int c = 0; c < kOut; ++c) {
          const float p = dm::exp_(v[c]), tg = targets[3 * (size_t)row + c];
          const float den = p * p + 0.01f;
          loss += (p - tg) * (p - tg) / den;
          split_half(2.0f * (p - tg) / den * p, &hi[c], &lo[c]);
        }
      }
      store_row8h(p0, t, 0, kOutPad, hi);      // dY hi rows: [128 x 16]
      store_row8h(p0, t, 8, kOutPad, hi + 8);
      __half* dy_lo = p0 + kTile * kOutPad;    // dY lo rows
      store_row8h(dy_lo, t, 0, kOutPad, lo);
      store_row8h(dy_lo, t, 8, kOutPad, lo + 8);
#pragma unroll
      for (int c = 0; c < kOut; ++c) {
        dzt[core_offset(c, t, kTile)] = hi[c];
        dzt[core_offset(kHid + c, t, kTile)] = lo[c];
      }
    }
    // backward: layer 4, then 3 .. 1
    operands_ready();
    if (tid == 0) {
      mma_steps(tmem + kColDW4, dzt_a, sbo_s, ht_a[3], sbo_s, kTile / 16, id64, !first);
      mma_steps(tmem + kColLayer, p0_a, sbo16, wt_a[4], sbo16, 1, id64, false);
      mma_steps(tmem + kColLayer, p0_a + kTile * kOutPad * 2, sbo16, wt_a[4], sbo16, 1, id64, true);
    }
    if (!(ok = mmas_done(bar_a, phase, tid))) break;
    train_bwd_epilogue(lane_addr, ht[3], p0, p1, dzt, t, half);  // dZ3
    const uint32_t dw_col[4] = {kColDW0, kColDW1, kColDW2, kColDW3};
    for (int l = 3; l >= 1; --l) {
      operands_ready();
      if (tid == 0) {
        mma_steps(tmem + dw_col[l], dzt_a, sbo_s, ht_a[l - 1], sbo_s, kTile / 16, id64, !first);
        mma_steps(tmem + kColLayer, p0_a, sbo64, wt_a[l], sbo64, kHid / 16, id64, false);
        mma_steps(tmem + kColLayer, p1_a, sbo64, wt_a[l], sbo64, kHid / 16, id64, true);
      }
      if (!(ok = mmas_done(bar_a, phase, tid))) break;
      // dZ_{l-1}; the last one (dZ0) only as the weight-gradient operand
      train_bwd_epilogue(lane_addr, ht[l - 1], l > 1 ? p0 : nullptr, l > 1 ? p1 : nullptr, dzt, t, half);
    }
    if (!ok) break;
    // H0^T (the encoding, re-computed) for dW0 = dZ0^T H0
    if (row < n) {
      auto sink = [&](int k, float x) { r[core_offset(k, t, kTile)] = __float2half_rn(x); };
      if (half == 0) rc_encode_part<0>(q, bounds, sink);
      else rc_encode_part<1>(q, bounds, sink);
    } else if (half == 0) {
      for (int k = 0; k < kIn; ++k) r[core_offset(k, t, kTile)] = __float2half_rn(0.0f);
    }
    operands_ready();
    if (tid == 0) mma_steps(tmem + kColDW0, dzt_a, sbo_s, r_a, sbo_s, kTile / 16, id144, !first);
    if (!(ok = mmas_done(bar_a, phase, tid))) break;
    first = false;
  }
  // weight-gradient sums -> this CTA's gradient row: rows 0..63 (hi) plus
  // rows 64..127 (lo); k_rc_grad_sum adds the CTAs' rows in a fixed order
  float* row = parts + (size_t)blockIdx.x * kNumParams;
  if (!(ok && !first))
    for (int p = tid; p < kNumParams; p += kTrainThreads) row[p] = 0.0f;
  if (ok && !first) {
    float* lo_rows = reinterpret_cast<float*>(smem + kTrainR) + half * kHid * 16;  // 64 rows x 16 columns per half
    const int out_rows[5] = {kHid, kHid, kHid, kHid, kOut};
    const int width[5] = {kIn, kHid, kHid, kHid, kHid};
    const int woff[5] = {kOffW0, kOffW1, kOffW2, kOffW3, kOffW4};
    const uint32_t col[5] = {kColDW0, kColDW1, kColDW2, kColDW3, kColDW4};
    const float inv_count = 1.0f / (3.0f * (float)n);
    for (int l = 0; l < 5; ++l)
      for (int cc = 0; cc < width[l]; cc += 32) {
        const int c0 = cc + 16 * half;  // each half reads its own 16 columns
        const bool mine = c0 < width[l];
        float v[16];
        if (mine) {
          tmem_ld16(lane_addr + col[l] + c0, v);
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          if (t >= kHid)
            for (int i = 0; i < 16; ++i) lo_rows[(t - kHid) * 16 + i] = v[i];
        }
        __syncthreads();
        if (mine && t < out_rows[l])
          for (int i = 0; i < 16; ++i) row[woff[l] + t * width[l] + c0 + i] = (v[i] + lo_rows[t * 16 + i]) * inv_count;
        __syncthreads();
      }
  }
  __shared__ float s_loss[kTrainThreads / 32];
  for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
  if ((tid & 31) == 0) s_loss[warp] = loss;
  __syncthreads();
  if (tid == 0) {
    float l = 0.0f;
    for (int w = 0; w < kTrainThreads / 32; ++w) l += s_loss[w];
    loss_parts[blockIdx.x] = l;
  }
  if (!ok && tid == 0) atomicExch(err, 1u);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
}

// Gradient and loss of a training step: the sum of the CTAs' rows in a fixed
// order (row r to group r % 8, each group in row order, then the groups in
// order), so a step's gradient does not depend on which CTA finished first.
constexpr int kSumParams = 32, kSumGroups = 8;
__global__ void k_rc_grad_sum(const float* __restrict__ parts, int rows, float* __restrict__ grad,
                              const float* __restrict__ loss_parts, float* __restrict__ loss) {
  __shared__ float s[kSumGroups][kSumParams];
  const int pl = threadIdx.x % kSumParams, g = threadIdx.x / kSumParams;
  const int p = blockIdx.x * kSumParams + pl;
  float acc = 0.0f;
  if (p < kNumParams)
    for (int r = g; r < rows; r += kSumGroups) acc += parts[(size_t)r * kNumParams + p];
  s[g][pl] = acc;
  __syncthreads();
  if (g == 0 && p < kNumParams) {
    float t = 0.0f;
    for (int k = 0; k < kSumGroups; ++k) t += s[k][pl];
    grad[p] = t;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    float l = 0.0f;
    for (int r = 0; r < rows; ++r) l += loss_parts[r];
    *loss = l;
  }
}

// Adam on the FP32 master weights, then the packed FP16 tensor-core operands
// (forward, and transposed for the backward pass).
__global__ void k_rc_adam(float* __restrict__ master, float* __restrict__ m1, float* __restrict__ m2,
                          const float* __restrict__ grad, float lr, float b1, float b2, float eps, float c1, float c2,
                          int update, __half* __restrict__ packed) {
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
  int row, k, K, base;
  if (p < kOffW1) { row = p / kIn; k = p % kIn; K = kIn; base = kPackW0; }
  else if (p < kOffW4) { int q = p - kOffW1; int l = q / (kHid * kHid); q %= kHid * kHid; row = q / kHid; k = q % kHid; K = kHid; base = kPackW1 + l * kHid * kHid; }
  else { int q = p - kOffW4; row = q / kHid; k = q % kHid; K = kHid; base = kPackW4; }
  packed[base + core_offset(row, k, K)] = hw;
  if (p >= kOffW1 && p < kOffW4) {  // W_l^T: row = input k, K index = output row
    const int l = (p - kOffW1) / (kHid * kHid);
    packed[kPackT1 + l * kHid * kHid + core_offset(k, row, kHid)] = hw;
  } else if (p >= kOffW4) {
    packed[kPackT4 + core_offset(k, row, kOutPad)] = hw;
  }
}

struct Cache {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  RcBounds bounds{};
  float *master = nullptr, *m1 = nullptr, *m2 = nullptr, *grad = nullptr, *loss = nullptr;
  float *parts = nullptr, *loss_parts = nullptr;  // per-CTA gradient rows and losses of a training step
  uint32_t* count = nullptr;  // sample count of host-submitted batches
  __half* packed = nullptr;
  uint32_t* err = nullptr;
  int step = 0;
  // batch buffers
  float* targets = nullptr;
  float4* queries = nullptr;
  float* out = nullptr;
  uint32_t cap = 0;
  std::string msg;
  int pending = 0;  // first error of a frame-driven call (rc_infer_device / rc_train_device)
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
  cudaFree(c->targets); cudaFree(c->queries); cudaFree(c->out);
  c->targets = c->out = nullptr;
  c->queries = nullptr;
  c->cap = 0;
  int rc;
  if ((rc = cuda_ok(c, cudaMalloc(&c->targets, (size_t)n * 12), "batch")) ||
      (rc = cuda_ok(c, cudaMalloc(&c->queries, (size_t)n * 64), "batch")) ||
      (rc = cuda_ok(c, cudaMalloc(&c->out, (size_t)n * 12), "batch")))
    return rc;
  c->cap = n;
  return AP_OK;
}

// Refreshes the FP16 copies from the master weights (no update).
void repack(Cache* c) {
  k_rc_adam<<<(kNumParams + 255) / 256, 256, 0, c->stream>>>(c->master, c->m1, c->m2, c->grad, 0.0f, 0.9f, 0.999f, 1e-8f,
                                                               1.0f, 1.0f, 0, c->packed);
}

}  // namespace

// Entry points used by the frame (device pointers, the caller's stream).
int rc_infer_device(void* cp, const float4* queries, uint32_t n, float* out, cudaStream_t st, const uint32_t* n_dev) {
  Cache* c = static_cast<Cache*>(cp);
  if (n == 0) return AP_OK;
  const int tiles = (int)((n + kTile - 1) / kTile);
  const int grid = tiles < 2 * c->num_sms ? tiles : 2 * c->num_sms;
  k_rc_infer<<<grid, 2 * kTile, kSmemInfer, st>>>(reinterpret_cast<const uint4*>(c->packed), queries, n, c->bounds, out, c->err,
                                               n_dev);
  const int rc = cuda_ok(c, cudaGetLastError(), "radiance cache inference");
  if (rc && !c->pending) c->pending = rc;
  return rc;
}

// After the caller's stream has drained: the first error of the frame-driven
// calls since the last check, or AP_E_TIMEOUT when an inference tile's
// tensor-core wait ran out of its bound; clears both.
int rc_take_status(void* cp, std::string* msg) {
  Cache* c = static_cast<Cache*>(cp);
  uint32_t e = 0;
  cudaMemcpy(&e, c->err, 4, cudaMemcpyDeviceToHost);
  int rc = c->pending;
  if (!rc && e) rc = cfail(c, AP_E_TIMEOUT, "inference: tensor-core wait timed out");
  if (rc && msg) *msg = c->msg;
  if (e) cudaMemset(c->err, 0, 4);
  c->pending = 0;
  return rc;
}

// Training step on at most `cap` samples; the sample count is read from device
// memory (n_dev), so a batch assembled on the device needs no host round trip.
int rc_train_device(void* cp, const float4* queries, const float* targets, const uint32_t* n_dev, uint32_t cap, float lr,
                    int update, cudaStream_t st) {
  Cache* c = static_cast<Cache*>(cp);
  if (cap == 0) return AP_OK;
  int rc = ensure_batch(c, cap);
  if (rc) {
    if (!c->pending) c->pending = rc;
    return rc;
  }
  const int tiles = (int)((cap + kTile - 1) / kTile);
  const int grid = tiles < c->num_sms ? tiles : c->num_sms;
  k_rc_train_tc<<<grid, kTrainThreads, kSmemTrain, st>>>(reinterpret_cast<const uint4*>(c->packed), queries, targets, n_dev,
                                                  cap, c->bounds, c->parts, c->loss_parts, c->err);
  k_rc_grad_sum<<<(kNumParams + kSumParams - 1) / kSumParams, kSumParams * kSumGroups, 0, st>>>(
      c->parts, grid, c->grad, c->loss_parts, c->loss);
  if (update) {
    c->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - (float)std::pow(0.9, c->step), c2 = 1.0f - (float)std::pow(0.999, c->step);
    k_rc_adam<<<(kNumParams + 255) / 256, 256, 0, st>>>(c->master, c->m1, c->m2, c->grad, lr, b1, b2, 1e-8f, c1, c2, 1,
                                                        c->packed);
  }
  rc = cuda_ok(c, cudaGetLastError(), "radiance cache training");
  if (rc && !c->pending) c->pending = rc;
  return rc;
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
  ap::DeviceScope device_scope(device);
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
      (rc = ap::cuda_ok(c, cudaMalloc(&c->loss, 4), "params")) ||
      (rc = ap::cuda_ok(c, cudaMalloc(&c->parts, (size_t)c->num_sms * ap::kNumParams * 4), "gradient rows")) ||
      (rc = ap::cuda_ok(c, cudaMalloc(&c->loss_parts, (size_t)c->num_sms * 4), "gradient rows")) ||
      (rc = ap::cuda_ok(c, cudaMalloc(&c->err, 4), "params")) ||
      (rc = ap::cuda_ok(c, cudaMalloc(&c->count, 4), "params")) ||
      (rc = ap::cuda_ok(c, cudaMalloc(&c->packed, ap::kPackAllHalves * 2), "params")) ||
      (rc = ap::cuda_ok(c, cudaFuncSetAttribute(ap::k_rc_infer, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                ap::kSmemInfer), "smem")) ||
      (rc = ap::cuda_ok(c, cudaFuncSetAttribute(ap::k_rc_train_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                ap::kSmemTrain), "smem"))) {
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
  ap::DeviceScope device_scope(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  void* ptrs[] = {c->master, c->m1, c->m2, c->grad, c->loss, c->parts, c->loss_parts, c->err, c->count, c->packed,
                  c->targets, c->queries, c->out};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

const char* ap_rc_last_error(const void* cp) {
  const Cache* c = static_cast<const Cache*>(cp);
  return c ? c->msg.c_str() : "null cache";
}

int ap_rc_wait_selftest(int device, int limit, uint32_t* out2) {
  if (!out2 || limit <= 0 || limit > (1 << 22)) return AP_E_INVALID;
  ap::DeviceScope device_scope(device);
  if (device_scope.status() != cudaSuccess) return AP_E_CUDA;
  uint32_t* d = nullptr;
  if (cudaMalloc(&d, 8) != cudaSuccess) return AP_E_OOM;
  cudaMemset(d, 0xff, 8);
  ap::k_wait_selftest<<<1, 32>>>(limit, d);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(out2, d, 8, cudaMemcpyDeviceToHost);
  cudaFree(d);
  return e == cudaSuccess ? AP_OK : AP_E_CUDA;
}

int ap_rc_set_params(void* cp, const float* params, uint32_t count) {
  Cache* c = static_cast<Cache*>(cp);
  if (!c || !params || count != ap::kNumParams) return ap::cfail(c, AP_E_INVALID, "parameter count");
  ap::DeviceScope device_scope(c->device);
  int rc;
  if ((rc = ap::cuda_ok(c, cudaMemcpy(c->master, params, ap::kNumParams * 4, cudaMemcpyHostToDevice), "params")))
    return rc;
  cudaMemsetAsync(c->m1, 0, ap::kNumParams * 4, c->stream);
  cudaMemsetAsync(c->m2, 0, ap::kNumParams * 4, c->stream);
  cudaMemsetAsync(c->packed, 0, ap::kPackAllHalves * 2, c->stream);
  c->step = 0;
  ap::repack(c);
  return ap::cuda_ok(c, cudaStreamSynchronize(c->stream), "params");
}

int ap_rc_get_params(void* cp, float* params, uint32_t count) {
  Cache* c = static_cast<Cache*>(cp);
  if (!c || !params || count != ap::kNumParams) return ap::cfail(c, AP_E_INVALID, "parameter count");
  ap::DeviceScope device_scope(c->device);
  cudaStreamSynchronize(c->stream);
  return ap::cuda_ok(c, cudaMemcpy(params, c->master, ap::kNumParams * 4, cudaMemcpyDeviceToHost), "params");
}

int ap_rc_infer(void* cp, const float* queries, uint32_t n, float* out_rgb) {
  Cache* c = static_cast<Cache*>(cp);
  if (!c || (n && (!queries || !out_rgb))) return ap::cfail(c, AP_E_INVALID, "null buffer");
  if (n == 0) return AP_OK;
  ap::DeviceScope device_scope(c->device);
  int rc = ap::ensure_batch(c, n);
  if (rc) return rc;
  cudaMemcpyAsync(c->queries, queries, (size_t)n * 64, cudaMemcpyHostToDevice, c->stream);
  if ((rc = ap::rc_infer_device(c, c->queries, n, c->out, c->stream, nullptr))) return rc;
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
  ap::DeviceScope device_scope(c->device);
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
