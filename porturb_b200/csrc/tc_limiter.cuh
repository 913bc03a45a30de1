// The linear part of the order-9 limiter on the 5th-generation tensor cores.
//
// Of the limiter's ~310 FP32 operations per stencil, about 85 are linear
// forms of the 8 stencil differences d_0..d_7: the LDL^T factors of the five
// smoothness indicators (TV_k = sum_i D_ki y_ki^2, y_k = L_k^T d_k..k+3;
// folded here as z_ki = sqrt(D_ki) y_ki so that TV_k = sum_i z_ki^2) and the
// ten edge forms lin_L[k], lin_R[k] (edge value = s_4 + sum_k w_k lin[k]).
// For a block of 128 stencils these are one product D[128 x 32] =
// A[128 x 8] * C[32 x 8]^T (20 z's, 10 lin's, 2 zero columns): a
// tcgen05.mma of kind tf32 with M = 128, N = 32, K = 8, accumulator in TMEM.
// FP32 accuracy comes from the usual three-term split: A = A_hi + A_lo and
// C = C_hi + C_lo in TF32 (cvt.rna), D = A_hi C_hi + A_hi C_lo + A_lo C_hi
// (the dropped A_lo C_lo is below 2^-22 relative), products exact in the
// FP32 accumulator.  Each thread then reads its stencil's row with one
// tcgen05.ld (32x32b.x32: warp w of the block reads TMEM lanes 32w..32w+31).
//
// Shared-memory operands are K-major without swizzle: 8-row core matrices of
// 16-byte rows (4 TF32), the two K halves of a core matrix LBO = 128 B apart,
// successive 8-row groups SBO = 256 B apart (the canonical layout
// ((8,n),2):((1,SBO),LBO) in 16-byte units).  Descriptor and instruction
// fields as the sm_100 UMMA descriptors define them.
#pragma once

#include <cstdint>

#include "weno9.cuh"

namespace pu {
namespace tc {

constexpr int TC_M = 128, TC_N = 32, TC_K = 8;
constexpr uint32_t TC_LBO = 128, TC_SBO = 256;
constexpr int TC_A_WORDS = TC_M * TC_K, TC_B_WORDS = TC_N * TC_K;   // 32-bit words per operand copy

// Word index of element (row, k) in the K-major core-matrix layout.
__host__ __device__ constexpr int kmajor_word(int row, int k) {
  return (row / 8) * int(TC_SBO / 4) + (k / 4) * int(TC_LBO / 4) + (row % 8) * 4 + (k % 4);
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint32_t tf32_bits(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// hi + lo = x to about 2^-22 relative, both TF32.
__device__ __forceinline__ void tf32_split(float x, uint32_t &hi, uint32_t &lo) {
  hi = tf32_bits(x);
  lo = tf32_bits(x - __uint_as_float(hi));
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
  uint64_t d = uint64_t((saddr >> 4) & 0x3FFFu);
  d |= uint64_t((TC_LBO >> 4) & 0x3FFFu) << 16;
  d |= uint64_t((TC_SBO >> 4) & 0x3FFFu) << 32;
  d |= uint64_t(1) << 46;   // descriptor version 1; base offset 0, no swizzle
  return d;
}

// D = F32, A = B = TF32, both K-major, N = 32, M = 128.
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(TC_N >> 3) << 17) | (uint32_t(TC_M >> 4) << 24);

// accumulate = 0: D = A C^T; 1: D += A C^T.  No output lane is disabled.
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %3, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %4, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(accumulate), "r"(IDESC), "r"(z));
}

__device__ __forceinline__ void commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for phase `parity` of the barrier: at most 20 ms by the GPU's
// nanosecond timer (and at most 2^26 polls, in case the timer stood still);
// false if it did not come.  Polls with test_wait (no suspension of the
// waiting threads).
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  uint64_t t0, t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  for (int it = 0; it < (1 << 26); it++) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (ok) return true;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    if (t - t0 > 20000000ull) return false;
  }
  return false;
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Warp-collective TMEM allocation of `cols` columns; the address goes to *dst (shared).
__device__ __forceinline__ void tmem_alloc(uint32_t dst_saddr, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_saddr), "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

// This warp's 32 lanes x 32 columns from TMEM address taddr (lane field set
// by the caller), one row per thread.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// A taken from tensor memory (the "TS" form): lanes are rows, 8 columns of
// TF32 per operand copy; same descriptor for C, same accumulator.
__device__ __forceinline__ void mma_tf32_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b, uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %3, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %4, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(d_tmem),
      "r"(a_tmem), "l"(b), "r"(accumulate), "r"(IDESC), "r"(z));
}

// This warp's lanes, 16 columns from taddr: one row of 16 values per thread.
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16};" ::"r"(taddr),
      "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
      "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
      : "memory");
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// One stencil's differences split into TF32 hi (values 0..7) and lo (8..15).
__device__ __forceinline__ void split_row(const float (&s)[9], uint32_t (&v)[16]) {
#pragma unroll
  for (int m = 0; m < 8; m++) tf32_split(s[m + 1] - s[m], v[m], v[8 + m]);
}

// Coefficient q of output n (0..31) over difference k (0..7), FP64.
__device__ inline double coef(int n, int k) {
  using namespace pu_weno9;
  if (n < 20) {
    const int s = n / 4, i = n % 4, j = k - s;   // z_si over d_{s+j}
    if (j < i || j > 3) return 0.0;
    return sqrt(TV_D[s][i]) * TV_L[s][j][i];
  }
  if (n < 30) {
    const int s = (n - 20) % 5, m = k - s;
    if (m < 0 || m > 3) return 0.0;
    return n < 25 ? LIN_L[s][m] : LIN_R[s][m];
  }
  return 0.0;
}

// Fills the C operand (hi, lo) in shared memory: all threads of the block.
__device__ inline void fill_coefs(uint32_t *bhi, uint32_t *blo) {
  for (int e = threadIdx.x; e < TC_N * TC_K; e += blockDim.x) {
    const int n = e / TC_K, k = e % TC_K;
    uint32_t hi, lo;
    tf32_split(float(coef(n, k)), hi, lo);
    bhi[kmajor_word(n, k)] = hi;
    blo[kmajor_word(n, k)] = lo;
  }
}

// Writes one stencil's differences (hi, lo) into row `row` of the A operand.
__device__ __forceinline__ void stage_row(const float (&s)[9], int row, uint32_t *ahi, uint32_t *alo) {
  uint32_t h[8], l[8];
#pragma unroll
  for (int m = 0; m < 8; m++) tf32_split(s[m + 1] - s[m], h[m], l[m]);
#pragma unroll
  for (int c = 0; c < 2; c++) {
    const int w = kmajor_word(row, 4 * c);
    *reinterpret_cast<uint4 *>(ahi + w) = make_uint4(h[4 * c], h[4 * c + 1], h[4 * c + 2], h[4 * c + 3]);
    *reinterpret_cast<uint4 *>(alo + w) = make_uint4(l[4 * c], l[4 * c + 1], l[4 * c + 2], l[4 * c + 3]);
  }
}

// The three MMAs of one block of 128 rows into the accumulator at TMEM address taddr.
__device__ __forceinline__ void issue(uint32_t taddr, const uint32_t *ahi, const uint32_t *alo, const uint32_t *bhi,
                                      const uint32_t *blo) {
  const uint64_t ah = smem_desc(smem_addr(ahi)), al = smem_desc(smem_addr(alo));
  const uint64_t bh = smem_desc(smem_addr(bhi)), bl = smem_desc(smem_addr(blo));
  mma_tf32(taddr, al, bh, 0u);
  mma_tf32(taddr, ah, bl, 1u);
  mma_tf32(taddr, ah, bh, 1u);
}

// Edge value from the linear forms of one edge and the shared reciprocals,
// as weno9_edge does from the differences.
template <bool LEFT>
__device__ __forceinline__ float edge_from_lin(const float (&lin)[5], float s4, const float (&rk)[5], bool do_map) {
  using namespace pu_weno9;
  float w[5];
#pragma unroll
  for (int k = 0; k < 5; k++) w[k] = float(LEFT ? IDEAL_L[k] : IDEAL_R[k]) * rk[k];
  normalize5(w);
  float r = 1.f;
  if (do_map) {
#pragma unroll
    for (int k = 0; k < 5; k++) {
      const float dk = float(LEFT ? IDEAL_L[k] : IDEAL_R[k]);
      const float t = w[k] - dk, t2 = t * t, t6 = t2 * t2 * t2;
      const float u = fmaf(-w[k], w[k], w[k]), u3 = u * u * u;
      w[k] = fmaf(t6 * t, fast_rcp(fmaf(2000.f, u3, t6)), dk);
    }
    r = fast_rcp(w[0] + w[1] + w[2] + w[3] + w[4]);
  }
  float acc = 0.f;
#pragma unroll
  for (int k = 0; k < 5; k++) acc = fmaf(w[k], lin[k], acc);
  return fmaf(acc, r, s4);
}

// The nonlinear rest of the limiter from one TMEM row (z's and lin's).
__device__ __forceinline__ void edges_from_row(const uint32_t (&r)[32], float s4, float &qL, float &qR, bool do_map,
                                               bool imm_L, bool imm_R) {
  float tv[5], lL[5], lR[5];
#pragma unroll
  for (int k = 0; k < 5; k++) {
    const float z0 = __uint_as_float(r[4 * k]), z1 = __uint_as_float(r[4 * k + 1]);
    const float z2 = __uint_as_float(r[4 * k + 2]), z3 = __uint_as_float(r[4 * k + 3]);
    tv[k] = fmaf(z0, z0, fmaf(z1, z1, fmaf(z2, z2, z3 * z3)));
    lL[k] = __uint_as_float(r[20 + k]);
    lR[k] = __uint_as_float(r[25 + k]);
  }
  convexify5(tv);
  if (imm_L || imm_R) {
    const float mx = fmaxf(fmaxf(fmaxf(fmaxf(tv[0], tv[1]), tv[2]), tv[3]), tv[4]);
    if (imm_L) tv[4] = mx;
    if (imm_R) tv[0] = mx;
  }
  float rk[5];
#pragma unroll
  for (int k = 0; k < 5; k++) rk[k] = fast_rcp(fmaf(tv[k], tv[k], 1.e-20f));
  qL = edge_from_lin<true>(lL, s4, rk, do_map);
  qR = edge_from_lin<false>(lR, s4, rk, do_map);
}

}  // namespace tc
}  // namespace pu
