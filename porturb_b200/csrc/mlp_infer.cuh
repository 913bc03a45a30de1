// Tensor-core inference of the learned WENO weights.
//
// The network maps a stencil normalised to its local range (the reference's
// normalize convention, dynamics_rk.h:42-53, WenoLimiter.h:85-96) to the five
// nonlinear weights of the left edge; the right edge uses the mirrored stencil
// (the right-edge weights of a stencil are the left-edge weights of its mirror
// image, WenoLimiter.h:383-387 vs 406-410):
//
//   x(9) -> relu(W1 bf(x) + b1) -> bf -> relu(W2 h1 + b2) -> bf -> W3 h2 + b3 -> softmax
//
// bf() rounds to bfloat16; weights are used rounded to bfloat16, biases and
// accumulation are FP32.  One warp evaluates 32 stencils and their mirrors
// (64 rows, four 16-row tiles) with mma.sync m16n8k16 BF16 -> FP32; each
// layer's accumulator fragment is the next layer's A-operand fragment after a
// fused relu + bfloat16 conversion, so activations never leave registers.
#pragma once

#include <cuda_bf16.h>

#include <cstdint>

namespace pu {
namespace mlp {
constexpr int NIN = 9, NH = 32, NOUT = 5;
constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + NH * NIN;
constexpr int OFF_W2 = OFF_B1 + NH;
constexpr int OFF_B2 = OFF_W2 + NH * NH;
constexpr int OFF_W3 = OFF_B2 + NH;
constexpr int OFF_B3 = OFF_W3 + NOUT * NH;
constexpr int NPARAM = OFF_B3 + NOUT;   // 1541
constexpr int FRAG_WORDS = 38;          // per lane: 28 bf16x2 operand words + 10 FP32 bias values
constexpr int FRAG_BYTES = 32 * FRAG_WORDS * 4;
// Per-warp shared memory: 64 input rows of 16 bf16 (2 KB), then the logits
// column by column with a 68-float stride (5 x 68 floats), bank-conflict
// free for the fragment-layout stores and the per-lane reads.
constexpr int LOGIT_STRIDE = 68;
constexpr int WARP_SMEM_BYTES = 64 * 32 + 5 * LOGIT_STRIDE * 4;

__host__ __device__ inline bool is_bias(int p) {
  return (p >= OFF_B1 && p < OFF_W2) || (p >= OFF_B2 && p < OFF_W3) || p >= OFF_B3;
}
}  // namespace mlp

__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// (s - min) / (max - min); all zeros when the range is <= 1e-20 (the
// reference's normalize keeps scale = 1 there, WenoLimiter.h:85-96).
// Returns the largest normalised jump between neighbouring entries.
__device__ __forceinline__ float normalize9(const float (&s)[9], float (&x)[9]) {
  float mn = s[0], mx = s[0];
#pragma unroll
  for (int m = 1; m < 9; m++) {
    mn = fminf(mn, s[m]);
    mx = fmaxf(mx, s[m]);
  }
  const float rng = mx - mn;
  const float r = rng > 1e-20f ? 1.f / rng : 0.f;
#pragma unroll
  for (int m = 0; m < 9; m++) x[m] = (s[m] - mn) * r;
  float jmp = 0.f;
#pragma unroll
  for (int m = 0; m < 8; m++) jmp = fmaxf(jmp, fabsf(x[m + 1] - x[m]));
  return jmp;
}

__device__ __forceinline__ uint32_t bf16_bits(float x) {
  __nv_bfloat16 b = __float2bfloat16_rn(x);
  return uint32_t(*reinterpret_cast<unsigned short *>(&b));
}

// Per-lane operand fragments of mma.m16n8k16 (B is K x N, K = layer input,
// N = layer output), word layout: w1[4][2], w2[2][4][2], w3[2][2] (bfloat16
// pairs, lower k in the low half), then b2[4][2], b3[2] as FP32 bits.
static __global__ void k_mlp_frags(const float *__restrict__ theta, uint32_t *__restrict__ frags) {
  using namespace mlp;
  const int lane = threadIdx.x;
  if (lane >= 32) return;
  const int g = lane >> 2, t = lane & 3;
  // Input columns 9 and 10 are constant 1: W1's columns there carry the
  // layer-1 bias split into a bfloat16 pair (b1 = hi + lo to about 2^-17).
  auto W1 = [&](int o, int i) {
    if (i < NIN) return theta[OFF_W1 + o * NIN + i];
    const float b = theta[OFF_B1 + o], hi = __bfloat162float(__float2bfloat16_rn(b));
    return i == NIN ? hi : (i == NIN + 1 ? b - hi : 0.f);
  };
  auto W2 = [&](int o, int i) { return theta[OFF_W2 + o * NH + i]; };
  auto W3 = [&](int o, int i) { return o < NOUT ? theta[OFF_W3 + o * NH + i] : 0.f; };
  auto pk = [](float lo, float hi) { return bf16_bits(lo) | (bf16_bits(hi) << 16); };
  uint32_t *f = frags + lane * FRAG_WORDS;
  int w = 0;
  for (int n = 0; n < 4; n++) {
    f[w++] = pk(W1(8 * n + g, 2 * t), W1(8 * n + g, 2 * t + 1));
    f[w++] = pk(W1(8 * n + g, 2 * t + 8), W1(8 * n + g, 2 * t + 9));
  }
  for (int s = 0; s < 2; s++)
    for (int n = 0; n < 4; n++) {
      f[w++] = pk(W2(8 * n + g, 16 * s + 2 * t), W2(8 * n + g, 16 * s + 2 * t + 1));
      f[w++] = pk(W2(8 * n + g, 16 * s + 2 * t + 8), W2(8 * n + g, 16 * s + 2 * t + 9));
    }
  for (int s = 0; s < 2; s++) {
    f[w++] = pk(W3(g, 16 * s + 2 * t), W3(g, 16 * s + 2 * t + 1));
    f[w++] = pk(W3(g, 16 * s + 2 * t + 8), W3(g, 16 * s + 2 * t + 9));
  }
  for (int n = 0; n < 4; n++) {
    f[w++] = __float_as_uint(theta[OFF_B2 + 8 * n + 2 * t]);
    f[w++] = __float_as_uint(theta[OFF_B2 + 8 * n + 2 * t + 1]);
  }
  f[w++] = __float_as_uint(2 * t < NOUT ? theta[OFF_B3 + 2 * t] : 0.f);
  f[w++] = __float_as_uint(2 * t + 1 < NOUT ? theta[OFF_B3 + 2 * t + 1] : 0.f);
}

// One lane's operand fragments, held in registers for the life of a kernel.
struct MlpLane {
  uint32_t w1[4][2], w2[2][4][2], w3[2][2];
  float b2[4][2], b3[2];
};

__device__ __forceinline__ void load_lane(const uint32_t *__restrict__ frags, MlpLane &L) {
  const uint32_t *f = frags + (threadIdx.x & 31) * mlp::FRAG_WORDS;
  int w = 0;
#pragma unroll
  for (int n = 0; n < 4; n++) {
    L.w1[n][0] = __ldg(f + w++);
    L.w1[n][1] = __ldg(f + w++);
  }
#pragma unroll
  for (int s = 0; s < 2; s++)
#pragma unroll
    for (int n = 0; n < 4; n++) {
      L.w2[s][n][0] = __ldg(f + w++);
      L.w2[s][n][1] = __ldg(f + w++);
    }
#pragma unroll
  for (int s = 0; s < 2; s++) {
    L.w3[s][0] = __ldg(f + w++);
    L.w3[s][1] = __ldg(f + w++);
  }
#pragma unroll
  for (int n = 0; n < 4; n++) {
    L.b2[n][0] = __uint_as_float(__ldg(f + w++));
    L.b2[n][1] = __uint_as_float(__ldg(f + w++));
  }
  L.b3[0] = __uint_as_float(__ldg(f + w++));
  L.b3[1] = __uint_as_float(__ldg(f + w++));
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2],
                                         const float (&c)[4]) {
  asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%10,%11,%12,%13};\n"
      : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]), "f"(c[0]), "f"(c[1]), "f"(c[2]),
        "f"(c[3]));
}

// relu, then round to a bfloat16 pair: low half <- lo, high half <- hi.
__device__ __forceinline__ uint32_t relu_bf16x2(float lo, float hi) {
  uint32_t r;
  asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}
__device__ __forceinline__ uint32_t bf16x2(float lo, float hi) {
  uint32_t r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}

// Input fragment k-step s of the next layer from output n-tiles 2s, 2s+1.
__device__ __forceinline__ void acc_to_a(const float (&d)[4][4], int s, uint32_t (&a)[4]) {
  a[0] = relu_bf16x2(d[2 * s][0], d[2 * s][1]);
  a[1] = relu_bf16x2(d[2 * s][2], d[2 * s][3]);
  a[2] = relu_bf16x2(d[2 * s + 1][0], d[2 * s + 1][1]);
  a[3] = relu_bf16x2(d[2 * s + 1][2], d[2 * s + 1][3]);
}

// One warp evaluates the network on the 32 normalised stencils held by its
// lanes and on their mirror images.  sW: per-warp scratch of WARP_SMEM_BYTES
// (16-byte aligned).  Input row r occupies 16-byte chunks 2r and 2r+1 with
// the halves swapped when bit 2 of r is set, so the row stores and the
// ldmatrix phases hit 8 distinct bank groups.  Returns each lane's left-edge
// weights and the right-edge weights of its stencil.  All 32 lanes must call it.
__device__ __forceinline__ int row_chunk(int r, int half) { return 2 * r + (half ^ ((r >> 2) & 1)); }

__device__ __forceinline__ void mlp_warp_weights(const MlpLane &L, uint32_t *sW, const float (&x)[9], float (&wl)[5],
                                                 float (&wr)[5]) {
  using mlp::LOGIT_STRIDE;
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  uint4 *rows = reinterpret_cast<uint4 *>(sW);
  float *sZ = reinterpret_cast<float *>(sW + 64 * 8);   // [5][LOGIT_STRIDE]
  const uint32_t one = 0x3F80u;   // bfloat16 1.0 in input column 10 (column 9 is the high half of word 4)
  rows[row_chunk(lane, 0)] =
      make_uint4(bf16x2(x[0], x[1]), bf16x2(x[2], x[3]), bf16x2(x[4], x[5]), bf16x2(x[6], x[7]));
  rows[row_chunk(lane, 1)] = make_uint4(bf16x2(x[8], 1.f), one, 0u, 0u);
  rows[row_chunk(32 + lane, 0)] =
      make_uint4(bf16x2(x[8], x[7]), bf16x2(x[6], x[5]), bf16x2(x[4], x[3]), bf16x2(x[2], x[1]));
  rows[row_chunk(32 + lane, 1)] = make_uint4(bf16x2(x[0], 1.f), one, 0u, 0u);
  __syncwarp();
#pragma unroll 1
  for (int T = 0; T < 4; T++) {
    uint32_t a[4];
    const uint4 *src = rows + row_chunk(16 * T + (lane & 15), lane >> 4);
    const unsigned addr = static_cast<unsigned>(__cvta_generic_to_shared(src));
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3])
                 : "r"(addr)
                 : "memory");
    float d1[4][4];
#pragma unroll
    for (int n = 0; n < 4; n++) {
      const float c[4] = {0.f, 0.f, 0.f, 0.f};
      mma_bf16(d1[n], a, L.w1[n], c);
    }
    uint32_t a2[2][4];
    acc_to_a(d1, 0, a2[0]);
    acc_to_a(d1, 1, a2[1]);
    float d2[4][4];
#pragma unroll
    for (int n = 0; n < 4; n++) {
      const float c[4] = {L.b2[n][0], L.b2[n][1], L.b2[n][0], L.b2[n][1]};
      mma_bf16(d2[n], a2[0], L.w2[0][n], c);
      mma_bf16(d2[n], a2[1], L.w2[1][n], d2[n]);
    }
    uint32_t a3[2][4];
    acc_to_a(d2, 0, a3[0]);
    acc_to_a(d2, 1, a3[1]);
    float d3[4];
    {
      const float c[4] = {L.b3[0], L.b3[1], L.b3[0], L.b3[1]};
      mma_bf16(d3, a3[0], L.w3[0], c);
      mma_bf16(d3, a3[1], L.w3[1], d3);
    }
    const int r0 = 16 * T + g, r1 = r0 + 8;
    if (2 * t < 5) {
      sZ[2 * t * LOGIT_STRIDE + r0] = d3[0];
      sZ[2 * t * LOGIT_STRIDE + r1] = d3[2];
    }
    if (2 * t + 1 < 5) {
      sZ[(2 * t + 1) * LOGIT_STRIDE + r0] = d3[1];
      sZ[(2 * t + 1) * LOGIT_STRIDE + r1] = d3[3];
    }
  }
  __syncwarp();
  float zl[5], zr[5];
#pragma unroll
  for (int k = 0; k < 5; k++) {
    zl[k] = sZ[k * LOGIT_STRIDE + lane];
    zr[k] = sZ[k * LOGIT_STRIDE + 32 + lane];
  }
  __syncwarp();   // the scratch is free for the next call
  float ml = zl[0], mr = zr[0];
#pragma unroll
  for (int k = 1; k < 5; k++) {
    ml = fmaxf(ml, zl[k]);
    mr = fmaxf(mr, zr[k]);
  }
  float sl = 0.f, sr = 0.f;
#pragma unroll
  for (int k = 0; k < 5; k++) {
    zl[k] = __expf(zl[k] - ml);
    zr[k] = __expf(zr[k] - mr);
    sl += zl[k];
    sr += zr[k];
  }
  const float il = __frcp_rn(sl), ir = __frcp_rn(sr);
#pragma unroll
  for (int k = 0; k < 5; k++) {
    wl[k] = zl[k] * il;
    wr[4 - k] = zr[k] * ir;   // the mirror's left weights, reversed, are the right-edge weights
  }
}

}  // namespace pu
