// Training and checking of the learned WENO weights (the network and its
// tensor-core inference are in mlp_infer.cuh).  The plain limiter's weights
// are the training targets and the fallback.  Contents:
//   k_harvest         -- sample stencils of a state and their plain weights
//   k_mlp_prepare     -- bfloat16-rounded copy of the FP32 master parameters
//   k_mlp_fwd_bwd     -- forward + backward of a batch tile, per-block gradient
//   k_mlp_reduce      -- deterministic sum of the per-block gradients
//   k_adam            -- Adam update of the FP32 master parameters
//   k_mlp_eval        -- forward only (SIMT), for checks
//   k_mlp_eval_mma    -- tensor-core forward of a stencil list, for checks
#pragma once

#include <cstdint>

#include "dycore_kernels.cuh"
#include "mlp_infer.cuh"

namespace pu {
namespace mlp {
constexpr int TB = 256;                 // samples per training block
constexpr int TBP = TB + 1;             // padded stride of the per-sample tiles
}  // namespace mlp

// ---------------------------------------------------------------------------
// Harvest: n samples of (normalised stencil, plain left-edge weights) from the
// state s.  Each sample draws a field, a direction and a cell from a
// counter-based generator; stencils touching immersed cells, or reaching the
// z walls, are redrawn (the dycore never uses the learned weights there).
// ---------------------------------------------------------------------------
template <class R, int NTR>
__global__ void k_harvest(const Grid<R> G, const R *__restrict__ s, long n, unsigned long long seed, long offset,
                          float *__restrict__ xs, float *__restrict__ ts) {
  const long q = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (q >= n) return;
  constexpr int F = 6 + NTR;
  const int nx = G.nx, ny = G.ny, nz = G.nz;
  const int ndir = G.sim2d ? 2 : 3;
  float st[9];
  for (int attempt = 0; attempt < 64; attempt++) {
    unsigned long long r = splitmix64(seed * 0x100000001B3ull + (unsigned long long)(offset + q) * 64 + attempt);
    const int f = int((r & 0xFFFF) % F);
    int dir = int(((r >> 16) & 0xFF) % ndir);
    if (G.sim2d && dir == 1) dir = 2;
    const int i = int(((r >> 24) & 0xFFFFF) % nx);
    const int j = int(((r >> 44) & 0xFFFFF) % ny);
    unsigned long long r2 = splitmix64(r);
    int k = int(r2 % nz);
    if (dir == 2) {
      if (nz < 2 * HS + 3) continue;
      k = HS + 1 + int(r2 % (nz - 2 * HS - 2));
    }
    if ((dir == 0 && G.bc_x != BC_PERIODIC) || (dir == 1 && G.bc_y != BC_PERIODIC)) {
      // precursor boundaries: keep the stencil inside the domain
      if (dir == 0 && (i < HS || i >= nx - HS)) continue;
      if (dir == 1 && (j < HS || j >= ny - HS)) continue;
    }
    bool ok = true;
    for (int m = 0; m < 9 && ok; m++) {
      int ii = i, jj = j, kk = k;
      if (dir == 0) ii = wrapi(i + m - 4, nx);
      else if (dir == 1) jj = wrapi(j + m - 4, ny);
      else kk = k + m - 4;
      const size_t idx = (size_t(kk) * ny + jj) * nx + ii;
      if (G.flags && (__ldg(G.flags + idx) & (FLAG_IMM | FLAG_ANY10))) ok = false;
      R w[F];
      prims<R, NTR>(G, s, idx, kk, w);
      st[m] = float(w[f]);
    }
    if (ok) break;
  }
  float x[9], wt[5];
  normalize9(st, x);
  weno9_left_weights(st, wt);
#pragma unroll
  for (int m = 0; m < 9; m++) xs[q * 9 + m] = x[m];
#pragma unroll
  for (int k = 0; k < 5; k++) ts[q * 5 + k] = wt[k];
}

// ---------------------------------------------------------------------------
// Training.
// ---------------------------------------------------------------------------
static __global__ void k_mlp_prepare(const float *__restrict__ theta, float *__restrict__ wq) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < mlp::NPARAM) wq[p] = mlp::is_bias(p) ? theta[p] : bf16_round(theta[p]);
}

// Sample index of batch slot q at step `step`, uniform over the dataset.
__device__ __forceinline__ long batch_sample(unsigned long long seed, long step, long q, long ndata) {
  return long(splitmix64(seed ^ (0xA24BAED4963EE407ull * (unsigned long long)(step + 1)) ^ (unsigned long long)q) %
              (unsigned long long)ndata);
}

// Forward and backward of TB samples per block; writes the block's gradient
// sum (NPARAM values) and loss sum to partial[blockIdx.x].
static __global__ void __launch_bounds__(mlp::TB) k_mlp_fwd_bwd(const float *__restrict__ wq, const float *__restrict__ xs,
                                                         const float *__restrict__ ts, long ndata, long step,
                                                         unsigned long long seed, int batch, int sequential,
                                                         float *__restrict__ partial) {
  using namespace mlp;
  extern __shared__ __align__(16) float sm[];
  float *W = sm;                       // NPARAM (bf16-rounded weights, FP32 biases)
  float *sx = W + ((NPARAM + 3) / 4) * 4;  // [NIN][TBP]
  float *s1 = sx + NIN * TBP;          // h1 [NH][TBP]
  float *s2 = s1 + NH * TBP;           // h2
  float *g1 = s2 + NH * TBP;           // da1
  float *g2 = g1 + NH * TBP;           // da2
  float *gz = g2 + NH * TBP;           // dz [NOUT][TBP]
  float *sl = gz + NOUT * TBP;         // loss [TB]
  const int tid = threadIdx.x;
  for (int p = tid; p < NPARAM; p += TB) W[p] = wq[p];
  __syncthreads();
  const long qb = long(blockIdx.x) * TB + tid;
  const bool live = qb < batch;
  float x[NIN], h1[NH], h2[NH], z[NOUT], t[NOUT];
  unsigned m1 = 0, m2 = 0;
  if (live) {
    const long smp = sequential ? qb : batch_sample(seed, step, qb, ndata);
#pragma unroll
    for (int m = 0; m < NIN; m++) x[m] = bf16_round(xs[smp * NIN + m]);
#pragma unroll
    for (int k = 0; k < NOUT; k++) t[k] = ts[smp * NOUT + k];
  } else {
#pragma unroll
    for (int m = 0; m < NIN; m++) x[m] = 0.f;
#pragma unroll
    for (int k = 0; k < NOUT; k++) t[k] = 0.f;
  }
#pragma unroll
  for (int u = 0; u < NH; u++) {
    float a = W[OFF_B1 + u];
#pragma unroll
    for (int m = 0; m < NIN; m++) a = fmaf(W[OFF_W1 + u * NIN + m], x[m], a);
    if (a > 0.f) m1 |= 1u << u;
    h1[u] = bf16_round(fmaxf(a, 0.f));
  }
#pragma unroll
  for (int u = 0; u < NH; u++) {
    float a = W[OFF_B2 + u];
#pragma unroll
    for (int v = 0; v < NH; v++) a = fmaf(W[OFF_W2 + u * NH + v], h1[v], a);
    if (a > 0.f) m2 |= 1u << u;
    h2[u] = bf16_round(fmaxf(a, 0.f));
  }
  float zmax = -3.0e38f;
#pragma unroll
  for (int k = 0; k < NOUT; k++) {
    float a = W[OFF_B3 + k];
#pragma unroll
    for (int u = 0; u < NH; u++) a = fmaf(W[OFF_W3 + k * NH + u], h2[u], a);
    z[k] = a;
    zmax = fmaxf(zmax, a);
  }
  float se = 0.f;
#pragma unroll
  for (int k = 0; k < NOUT; k++) {
    z[k] = expf(z[k] - zmax);
    se += z[k];
  }
  float loss = 0.f;
  const float inv_b = 1.f / float(batch);
#pragma unroll
  for (int k = 0; k < NOUT; k++) {
    const float p = z[k] / se;
    if (live && t[k] > 0.f) loss -= t[k] * logf(fmaxf(p, 1e-30f));
    z[k] = live ? (p - t[k]) * inv_b : 0.f;   // dz
  }
  // Store the tiles for the gradient reduction.
#pragma unroll
  for (int m = 0; m < NIN; m++) sx[m * TBP + tid] = x[m];
#pragma unroll
  for (int u = 0; u < NH; u++) {
    s1[u * TBP + tid] = h1[u];
    s2[u * TBP + tid] = h2[u];
  }
#pragma unroll
  for (int k = 0; k < NOUT; k++) gz[k * TBP + tid] = z[k];
  // da2 = (W3^T dz) * [a2 > 0], da1 = (W2^T da2) * [a1 > 0]
  float d2[NH];
#pragma unroll
  for (int u = 0; u < NH; u++) {
    float a = 0.f;
#pragma unroll
    for (int k = 0; k < NOUT; k++) a = fmaf(W[OFF_W3 + k * NH + u], z[k], a);
    d2[u] = ((m2 >> u) & 1u) ? a : 0.f;
    g2[u * TBP + tid] = d2[u];
  }
#pragma unroll
  for (int v = 0; v < NH; v++) {
    float a = 0.f;
#pragma unroll
    for (int u = 0; u < NH; u++) a = fmaf(W[OFF_W2 + u * NH + v], d2[u], a);
    g1[v * TBP + tid] = ((m1 >> v) & 1u) ? a : 0.f;
  }
  sl[tid] = loss;
  __syncthreads();
  // Gradient of every parameter summed over the block's samples.
  float *out = partial + size_t(blockIdx.x) * (NPARAM + 1);
  for (int p = tid; p < NPARAM; p += TB) {
    const float *a, *b;   // gradient = sum_s a[s] * b[s]  (b null: sum_s a[s])
    if (p < OFF_B1) { a = g1 + (p / NIN) * TBP; b = sx + (p % NIN) * TBP; }
    else if (p < OFF_W2) { a = g1 + (p - OFF_B1) * TBP; b = nullptr; }
    else if (p < OFF_B2) { const int q = p - OFF_W2; a = g2 + (q / NH) * TBP; b = s1 + (q % NH) * TBP; }
    else if (p < OFF_W3) { a = g2 + (p - OFF_B2) * TBP; b = nullptr; }
    else if (p < OFF_B3) { const int q = p - OFF_W3; a = gz + (q / NH) * TBP; b = s2 + (q % NH) * TBP; }
    else { a = gz + (p - OFF_B3) * TBP; b = nullptr; }
    float acc = 0.f;
    if (b) {
      for (int s = 0; s < TB; s++) acc = fmaf(a[s], b[s], acc);
    } else {
      for (int s = 0; s < TB; s++) acc += a[s];
    }
    out[p] = acc;
  }
  if (tid == 0) {
    float L = 0.f;
    for (int s = 0; s < TB; s++) L += sl[s];
    out[NPARAM] = L;
  }
}

inline size_t mlp_train_smem_bytes() {
  using namespace mlp;
  return sizeof(float) * (size_t((NPARAM + 3) / 4) * 4 + size_t(NIN + 4 * NH + NOUT) * TBP + TB);
}

// grad[p] = sum over blocks of partial[b][p] (fixed order: deterministic).
static __global__ void k_mlp_reduce(const float *__restrict__ partial, int nblocks, float *__restrict__ grad) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p > mlp::NPARAM) return;
  double acc = 0.0;
  for (int b = 0; b < nblocks; b++) acc += partial[size_t(b) * (mlp::NPARAM + 1) + p];
  grad[p] = float(acc);
}

static __global__ void k_adam(float *__restrict__ theta, float *__restrict__ m, float *__restrict__ v,
                       const float *__restrict__ grad, float lr, float b1, float b2, float eps, float bc1, float bc2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= mlp::NPARAM) return;
  const float g = grad[p];
  const float mm = b1 * m[p] + (1.f - b1) * g;
  const float vv = b2 * v[p] + (1.f - b2) * g * g;
  m[p] = mm;
  v[p] = vv;
  theta[p] -= lr * (mm / bc1) / (sqrtf(vv / bc2) + eps);
}

// Forward only, one sample per thread (checks and statistics).
static __global__ void __launch_bounds__(256) k_mlp_eval(const float *__restrict__ wq, const float *__restrict__ xs, long n,
                                                  float *__restrict__ out) {
  using namespace mlp;
  __shared__ float W[NPARAM];
  for (int p = threadIdx.x; p < NPARAM; p += blockDim.x) W[p] = wq[p];
  __syncthreads();
  const long q = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (q >= n) return;
  float x[NIN], h1[NH], h2[NH], z[NOUT];
#pragma unroll
  for (int m = 0; m < NIN; m++) x[m] = bf16_round(xs[q * NIN + m]);
#pragma unroll
  for (int u = 0; u < NH; u++) {
    float a = W[OFF_B1 + u];
#pragma unroll
    for (int m = 0; m < NIN; m++) a = fmaf(W[OFF_W1 + u * NIN + m], x[m], a);
    h1[u] = bf16_round(fmaxf(a, 0.f));
  }
#pragma unroll
  for (int u = 0; u < NH; u++) {
    float a = W[OFF_B2 + u];
#pragma unroll
    for (int v = 0; v < NH; v++) a = fmaf(W[OFF_W2 + u * NH + v], h1[v], a);
    h2[u] = bf16_round(fmaxf(a, 0.f));
  }
  float zmax = -3.0e38f, se = 0.f;
#pragma unroll
  for (int k = 0; k < NOUT; k++) {
    float a = W[OFF_B3 + k];
#pragma unroll
    for (int u = 0; u < NH; u++) a = fmaf(W[OFF_W3 + k * NH + u], h2[u], a);
    z[k] = a;
    zmax = fmaxf(zmax, a);
  }
#pragma unroll
  for (int k = 0; k < NOUT; k++) {
    z[k] = expf(z[k] - zmax);
    se += z[k];
  }
#pragma unroll
  for (int k = 0; k < NOUT; k++) out[q * NOUT + k] = z[k] / se;
}

// Test entry: tensor-core evaluation of n stencils (already normalised),
// returning the left weights and the mirrored-stencil (right-edge) weights.
static __global__ void __launch_bounds__(128) k_mlp_eval_mma(const uint32_t *__restrict__ frags, const float *__restrict__ xs,
                                                      long n, float *__restrict__ wl_out, float *__restrict__ wr_out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t *sW = reinterpret_cast<uint32_t *>(smem_raw + warp * mlp::WARP_SMEM_BYTES);
  MlpLane L;
  load_lane(frags, L);
  const long q = (long(blockIdx.x) * (blockDim.x >> 5) + warp) * 32 + lane;
  float x[9], wl[5], wr[5];
#pragma unroll
  for (int m = 0; m < 9; m++) x[m] = q < n ? xs[q * 9 + m] : 0.f;
  mlp_warp_weights(L, sW, x, wl, wr);
  if (q < n) {
#pragma unroll
    for (int k = 0; k < 5; k++) {
      wl_out[q * 5 + k] = wl[k];
      wr_out[q * 5 + k] = wr[k];
    }
  }
}

}  // namespace pu
