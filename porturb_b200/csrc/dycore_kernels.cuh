// Kernels of the B200 dycore (order-9 WENO finite volume, SSPRK3).
//
// Storage: the resident state is structure-of-arrays, one (nz,ny,nx) array
// per prognostic with no halos, in the stencil type R (float or double):
//   q0 = rho - rho_h(k)             (density perturbation)
//   q1..q3 = rho*u, rho*v, rho*w
//   q4 = rho*theta - rho_h*theta_h(k)
//   q5.. = tracer densities rho*q (the reference's tracers array)
// rho_h, theta_h are the hydrostatic cell profiles (hy_dens_cells,
// hy_theta_cells, dynamics_rk.h:961-1008).  Storing perturbations keeps FP32
// state at the precision of the fluctuations rather than of the background.
// Halos are never stored: periodic wraps, precursor clamps and wall values are
// applied while tiles are loaded.
//
// Per SSPRK3 stage two kernels run:
//   k_xy : one (x,y) tile of one level: primitive perturbation fields of the
//          tile plus 5-cell halos into shared memory, WENO edges in x and y
//          (dynamics_rk.h:572-607), upwind Riemann fluxes (:640-684) and their
//          x/y divergence, written to the tendency buffer txy.
//   k_z  : one column per thread marching up a chunk of levels with a 9-plane
//          ring of primitive fields in shared memory: WENO edges in z
//          (:608-625), wall/periodic face states (:891-908), Riemann fluxes
//          (:685-706), the z divergence added to txy, gravity and Coriolis
//          (:710-722), the SSPRK3 stage combination (:308-360), positivity
//          clip and immersed relaxation (:429-469).
#pragma once

#include <cstdint>
#include <type_traits>

#include "mlp_infer.cuh"
#include "tma.cuh"
#include "weno9.cuh"

namespace pu {

// Packed FP32 limiter (two stencils per FFMA2/FADD2/FMUL2) in the plain x/y
// kernel; 0 keeps the scalar limiter (results are identical).
#ifndef PU_PACKED_LIMITER
#define PU_PACKED_LIMITER 1
#endif
// The same in the z march, on pairs of fields of the cell (weno_all): under
// the 128-register cap of PU_Z_MIN_BLOCKS it fits without spills (126
// registers; uncapped it took ~165 and lost the time to occupancy) and takes
// k_z from 1.055 to 0.919 ms on the 256x256x128 boundary layer.
#ifndef PU_PACKED_Z
#define PU_PACKED_Z 1
#endif
// Minimum resident blocks per SM requested for the plain FP32 x/y kernel: 4
// (64 registers) keeps 32 warps per SM with the packed limiter (measured on
// the 256x256x128 boundary layer: 1.80 ms per launch against 2.05 ms uncapped
// and 1.87 ms with the scalar limiter).
#ifndef PU_XY_MIN_BLOCKS
#define PU_XY_MIN_BLOCKS 4
#endif
// Minimum resident blocks per SM requested for the plain z march: 4 blocks
// of 128 threads (at most 128 registers) measured 0.4 % faster than no cap.
#ifndef PU_Z_MIN_BLOCKS
#define PU_Z_MIN_BLOCKS 4
#endif
// Minimum resident blocks per SM requested for the learned stencil kernels
// (caps their registers: the network's operand fragments stay in registers).
#ifndef PU_LEARNED_XY_MIN_BLOCKS
#define PU_LEARNED_XY_MIN_BLOCKS 2
#endif
// Minimum resident blocks per SM requested for the tiled z kernel k_zt
// (256 threads: 4 blocks cap it at 64 registers, as the x/y kernel).
#ifndef PU_ZT_MIN_BLOCKS
#define PU_ZT_MIN_BLOCKS 4
#endif
#ifndef PU_LEARNED_Z_MIN_BLOCKS
#define PU_LEARNED_Z_MIN_BLOCKS 3
#endif

constexpr int HS = 4;
constexpr int BC_PERIODIC = 0, BC_PRECURSOR = 1, BC_WALL = 2;
constexpr unsigned FLAG_IMM = 1u, FLAG_ANY10 = 2u;
// Bits of the device error word (Grid::err): a non-finite state, a tile copy
// (TMA) that did not complete within its wait limit.
constexpr int ERR_NONFINITE = 1, ERR_TMA = 2;
constexpr int iR = 0, iU = 1, iV = 2, iW = 3, iT = 4, iP = 5;

template <class R>
struct Grid {
  int nx, ny, nz;
  size_t N, NP;                 // nx*ny*nz and nx*ny
  R rdx, rdy, rdz;
  int bc_x, bc_y, bc_z;
  int sim2d, weno_all, enable_gravity;
  R grav, fcor, gamma;
  R pc[5];                      // C(gamma, n), n = 1..5: the series of pow1pm1
  int pser;                     // gamma in [1, 5/3]: pow1pm1 may use the series
  unsigned tracer_positive;     // bit t: tracer t is positive definite
  // Level tables.  Cell tables have nz+2*HS entries (index k+HS); edge tables nz+1.
  const R *rho_h, *theta_h;     // hy_dens_cells, hy_theta_cells
  const R *rt_inv;              // 1 / (rho_h*theta_h)
  const R *p0_h;                // C0*(rho_h*theta_h)^gamma
  const R *dp_h;                // p0_h - hy_pressure_cells
  const R *rho_e, *theta_e;     // hy_dens_edges, hy_theta_edges
  const R *rt_target;           // immersed relaxation target of q4 (index k)
  const uint8_t *flags;         // FLAG_IMM | FLAG_ANY10 per cell, or null
  const R *imm_mult;            // immersed_proportion^power / tau per cell, or null
  int *err;                     // bit 0: a non-finite value was written
  // Decomposed tiles (k_xy with DECOMP): the stage input's raw state beyond
  // the tile's x and y edges, received from the neighbouring tiles, as slabs
  // [S][nz][ny][HALO_W] (x: hxl below i = 0, hxr from i = nx) and
  // [S][nz][HALO_W][nx] (y), with their immersed flags ([nz][ny][HALO_W],
  // [nz][HALO_W][nx]).  gx0/gx1/gy0/gy1: the tile's low/high x/y edge is the
  // global domain edge (precursor conditions apply only there; 1 for an
  // undecomposed domain).
  const R *hxl, *hxr, *hyl, *hyr;
  const uint8_t *fxl, *fxr, *fyl, *fyr;
  int gx0, gx1, gy0, gy1;
  // First level of a k_xy launch (blockIdx.z counts from it) and first z
  // chunk of a k_zt launch: a stage can run the immersed kernels on the
  // levels that need them and the plain ones above.  First column and row of
  // a k_xy launch (blockIdx.x, .y count tiles from them): a decomposed tile
  // can run its interior tiles while its halos cross, its edge tiles after.
  int k_first, c_first, i_first, j_first;
  // Learned WENO weights (kernels instantiated with LEARNED only).
  const uint32_t *ml_frags;     // per-lane operand fragments of the network
  unsigned long long *ml_counts;  // [0] stencils given learned weights, [1] limiter fallbacks
  float ml_jump;                // largest normalised neighbour jump given learned weights
};

__device__ __forceinline__ int wrapi(int i, int n) {
  if (unsigned(i) < unsigned(n)) return i;   // inside: no division
  i %= n;
  return i < 0 ? i + n : i;
}
__device__ __forceinline__ int clampi(int i, int n) { return i < 0 ? 0 : (i >= n ? n - 1 : i); }

__device__ __forceinline__ float pu_log1p(float x) { return log1pf(x); }
__device__ __forceinline__ double pu_log1p(double x) { return log1p(x); }
__device__ __forceinline__ float pu_expm1(float x) { return expm1f(x); }
__device__ __forceinline__ double pu_expm1(double x) { return expm1(x); }

// (1+x)^gamma - 1, the pressure perturbation relative to the column's
// C0 (rho theta)_h^gamma.  In FP32 and for |x| <= 1/16 (every cell of the
// boundary-layer, bubble and urban cases) the binomial series to x^5,
// sum C(gamma,n) x^n by Horner (coefficients G.pc): the first omitted term is
// below 5e-9 of the result for gamma in [1, 5/3], under the FP32 rounding.
// Otherwise, and in FP64, expm1(gamma log1p(x)).
template <class R>
__device__ __forceinline__ R pow1pm1(const Grid<R> &G, R x) {
  if constexpr (std::is_same<R, float>::value) {
    if (G.pser && fabsf(x) <= 0.0625f)
      return fmaf(fmaf(fmaf(fmaf(G.pc[4], x, G.pc[3]), x, G.pc[2]), x, G.pc[1]), x, G.pc[0]) * x;
  }
  return pu_expm1(G.gamma * pu_log1p(x));
}

template <class R, int NTR>
__device__ __forceinline__ void load_cell(const Grid<R> &G, const R *__restrict__ s, size_t idx, R (&q)[5 + NTR]) {
#pragma unroll
  for (int v = 0; v < 5 + NTR; v++) q[v] = __ldg(s + v * G.N + idx);
}

// Primitive perturbation fields of one cell (dynamics_rk.h:550-558) from its
// S raw fields q at level k: rho', u, v, w, theta', p', tracer mixing
// ratios.  theta' and p' are formed from the perturbation storage without
// cancellation:
//   theta' = (q4 - theta_h q0)/rho,   p' = P0_h*((1 + q4/(rho theta)_h)^gamma - 1) + (P0_h - p_h).
template <class R, int NTR>
__device__ __forceinline__ void prims_of(const Grid<R> &G, const R (&q)[5 + NTR], int k, R (&w)[6 + NTR]) {
  const int kh = k + HS;
  R rho = __ldg(G.rho_h + kh) + q[0];
  R rr = R(1) / rho;
  w[0] = q[0];
  w[1] = q[1] * rr;
  w[2] = q[2] * rr;
  w[3] = q[3] * rr;
  w[4] = (q[4] - __ldg(G.theta_h + kh) * q[0]) * rr;
  w[5] = fma(__ldg(G.p0_h + kh), pow1pm1(G, q[4] * __ldg(G.rt_inv + kh)), __ldg(G.dp_h + kh));
#pragma unroll
  for (int t = 0; t < NTR; t++) w[6 + t] = q[5 + t] * rr;
}

// The same from a state whose S fields lie N elements apart (the resident
// arrays, N = nz*ny*nx, or a halo slab).
template <class R, int NTR>
__device__ __forceinline__ void prims_s(const Grid<R> &G, const R *__restrict__ s, size_t N, size_t idx, int k,
                                        R (&w)[6 + NTR]) {
  R q[5 + NTR];
#pragma unroll
  for (int v = 0; v < 5 + NTR; v++) q[v] = __ldg(s + v * N + idx);
  prims_of<R, NTR>(G, q, k, w);
}

template <class R, int NTR>
__device__ __forceinline__ void prims(const Grid<R> &G, const R *__restrict__ s, size_t idx, int k, R (&w)[6 + NTR]) {
  prims_s<R, NTR>(G, s, G.N, idx, k, w);
}

// Width of the halo a decomposed tile receives from each neighbour: the
// order-9 stencils of cells -1 and n reach 5 cells beyond the tile.
constexpr int HALO_W = 5;

// Where the state and the immersed flags of cell (gi, gj) of level k come
// from in a decomposed tile: the tile's own arrays, the receive slab beyond
// an x or a y edge, or -- at a global precursor edge, for the state only --
// the nearest tile cell (halo_boundary_conditions, dynamics_rk.h:745-790;
// the immersed halos are exchanged periodically, :1026-1032).  Cells beyond
// both an x and a y edge, and cells more than HALO_W beyond an edge, are only
// read by stencils of cells outside the tile, whose results are discarded;
// they read the nearest valid cell.
template <class R>
__device__ __forceinline__ void tile_source(const Grid<R> &G, const R *sin, int gi, int gj, int k, const R *&src,
                                            size_t &fs, size_t &q, const uint8_t *&fl) {
  const int nx = G.nx, ny = G.ny;
  // A 2-D domain (ny == 1) has no y halo: rows beyond it belong to stencils
  // of rows outside the domain and read row 0, as the periodic wrap does.
  const bool ox = gi < 0 || gi >= nx, oy = !G.sim2d && (gj < 0 || gj >= ny);
  if (ox && !oy) {
    const int col = gi < 0 ? gi + HALO_W : min(gi - nx, HALO_W - 1);
    const size_t e = (size_t(k) * ny + gj) * HALO_W + col;
    fl = (gi < 0 ? G.fxl : G.fxr) ? (gi < 0 ? G.fxl : G.fxr) + e : nullptr;
    if (G.bc_x == BC_PRECURSOR && (gi < 0 ? G.gx0 : G.gx1)) {
      src = sin;
      fs = G.N;
      q = size_t(k) * G.NP + size_t(gj) * nx + clampi(gi, nx);
    } else {
      src = gi < 0 ? G.hxl : G.hxr;
      fs = size_t(G.nz) * ny * HALO_W;
      q = e;
    }
  } else if (oy && !ox) {
    const int row = gj < 0 ? gj + HALO_W : min(gj - ny, HALO_W - 1);
    const size_t e = (size_t(k) * HALO_W + row) * nx + gi;
    fl = (gj < 0 ? G.fyl : G.fyr) ? (gj < 0 ? G.fyl : G.fyr) + e : nullptr;
    if (G.bc_y == BC_PRECURSOR && (gj < 0 ? G.gy0 : G.gy1)) {
      src = sin;
      fs = G.N;
      q = size_t(k) * G.NP + size_t(clampi(gj, ny)) * nx + gi;
    } else {
      src = gj < 0 ? G.hyl : G.hyr;
      fs = size_t(G.nz) * HALO_W * nx;
      q = e;
    }
  } else {
    src = sin;
    fs = G.N;
    q = size_t(k) * G.NP + size_t(clampi(gj, ny)) * nx + clampi(gi, nx);
    fl = G.flags ? G.flags + q : nullptr;
  }
}

// Copies a bx x by box of each of bz stacked planes between two arrays of
// planes (x fastest): dst[(p*dyn + dj0 + j)*dxn + di0 + i] =
// src[(p*syn + sj0 + j)*sxn + si0 + i].  Halo slabs of decomposed tiles are
// packed, assembled and cropped with it (fields are stacked planes too).
template <class T>
__global__ void k_box(const T *__restrict__ src, int sxn, int syn, int si0, int sj0, T *__restrict__ dst, int dxn,
                      int dyn, int di0, int dj0, int bx, int by, int bz) {
  const size_t n = size_t(bx) * by * bz;
  for (size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x) {
    const int i = int(e % bx), j = int((e / bx) % by);
    const size_t p = e / (size_t(bx) * by);
    dst[(p * dyn + dj0 + j) * size_t(dxn) + di0 + i] = src[(p * syn + sj0 + j) * size_t(sxn) + si0 + i];
  }
}

// Upwind Riemann flux across one face (dynamics_rk.h:640-706): acoustic
// upwinding of mass flux and pressure with a constant sound speed of 350 m/s,
// advective upwinding of everything else.  L and Rt are the edge states of
// the left and right cells (perturbation fields); hr, ht the hydrostatic
// density and potential temperature at the face; idN the normal velocity.
template <class R, int NTR>
__device__ __forceinline__ void riemann(const R (&L)[6 + NTR], const R (&Rt)[6 + NTR], R hr, R ht, int idN,
                                        R (&flux)[5 + NTR]) {
  const R cs = R(350.), r_cs = R(1.) / R(350.);
  R rL = L[iR] + hr, rR = Rt[iR] + hr;
  R ruL = L[idN] * rL, ruR = Rt[idN] * rR;
  R pL = L[iP], pR = Rt[iP];
  R p_upw = R(0.5) * (pL + pR - cs * (ruR - ruL));
  R ru_upw = R(0.5) * (ruL + ruR - (pR - pL) * r_cs);
  const bool up = ru_upw > R(0);
  flux[iR] = ru_upw;
  flux[iU] = ru_upw * (up ? L[iU] : Rt[iU]);
  flux[iV] = ru_upw * (up ? L[iV] : Rt[iV]);
  flux[iW] = ru_upw * (up ? L[iW] : Rt[iW]);
  flux[iT] = ru_upw * ((up ? L[iT] : Rt[iT]) + ht);
  flux[idN] += p_upw;
#pragma unroll
  for (int t = 0; t < NTR; t++) flux[5 + t] = ru_upw * (up ? L[6 + t] : Rt[6 + t]);
}

template <class R, int NTR, int TX, int TY, bool IMM, bool LEARNED = false>
struct XYShape {
  static constexpr int F = 6 + NTR, S = 5 + NTR, NT = TX * TY;
  static constexpr int HX = TX + 10, HY = TY + 10;       // tile plus 5-cell halos
  static constexpr int EXN = TY * (TX + 2), EYN = (TY + 2) * TX;
  static constexpr int EN = EXN > EYN ? EXN : EYN;
  static constexpr int FXN = TY * (TX + 1), FYN = (TY + 1) * TX;
  static constexpr int FN = FXN > FYN ? FXN : FYN;
  // Edges of the y lines' halo cells, taken during the x phase (packed path).
  static constexpr int YON = 2 * F * TX;
  // Immersed domains: the flag byte of every tile and halo cell, then the
  // stencil masks of the x lines ([TY][TX+2]) and the y lines ([TY+2][TX]).
  static constexpr size_t MB = (size_t(HY) * HX + 15) / 16 * 16;
  static constexpr size_t MASKB = (size_t(2) * (TY * (TX + 2) + (TY + 2) * TX) + 15) / 16 * 16;
  // Learned mode: per-warp network scratch and two fallback counters; the
  // fallback queue (16-bit stencil indices) lives in the flux buffer, which
  // is idle while edges are reconstructed.
  static constexpr size_t learned_bytes = LEARNED ? size_t(NT / 32) * mlp::WARP_SMEM_BYTES + 16 : 0;
  static constexpr size_t layout_bytes = sizeof(R) * (size_t(F) * HY * HX + 2 * size_t(F) * EN + size_t(S) * FN + YON) +
                                         (IMM ? MB + MASKB : 0) + learned_bytes;
  static constexpr size_t bytes = layout_bytes;
  // TMA staging of the 16x16 tile (FP32, the TMA instantiation): the raw
  // stage input of the tile's cross -- the 16x16 interior, 5 rows above and
  // below, 5 columns left and right, the latter in 8-column boxes -- lands in
  // the edge and flux buffers, idle until the primitive fields are formed;
  // one mbarrier after the layout.  That kernel rounds its dynamic shared
  // memory up to 128 bytes (PAD).
  static constexpr size_t PAD = 128;
  static constexpr size_t al(size_t b) { return (b + 127) / 128 * 128; }
  static constexpr size_t h_bytes = sizeof(R) * size_t(F) * HY * HX;
  static constexpr size_t st_in = al(h_bytes);                      // [S][16][16]
  static constexpr size_t st_top = al(st_in + sizeof(R) * S * 256);  // [S][5][16]
  static constexpr size_t st_bot = al(st_top + sizeof(R) * S * 80);  // [S][5][16]
  static constexpr size_t st_west = al(st_bot + sizeof(R) * S * 80); // [S][16][8]
  static constexpr size_t st_east = al(st_west + sizeof(R) * S * 128);
  static constexpr size_t stage_end = st_east + sizeof(R) * S * 128;
  static constexpr size_t yo_off = h_bytes + sizeof(R) * (2 * size_t(F) * EN + size_t(S) * FN);
  static constexpr bool TMA_FITS = TX == 16 && TY == 16 && sizeof(R) == 4 && !LEARNED && stage_end <= yo_off;
  static constexpr size_t bar_off = al(layout_bytes);
  static constexpr size_t tma_bytes = bar_off + 16 + PAD;
  static_assert(!LEARNED || size_t(F) * EN * 2 <= sizeof(R) * S * FN, "fallback queue exceeds the flux buffer");
  static_assert(NT % 32 == 0, "whole warps");
};

// Tensor maps of one k_xy launch (TMA staging, 16x16 tiles): the stage input
// with the boxes (16, 16, 1, S) interior, (16, 5, 1, S) halo rows and
// (8, 16, 1, S) halo columns.
struct XyMaps {
  CUtensorMap in, ns, ew;
};

// Edge reconstruction of `total` stencils with learned weights by the NT
// threads of a block.  Every warp walks the stencil list in lock step (one
// stencil per lane), so the network is always evaluated by full warps.
// Stencils with an immersed cell within reach, or a normalised neighbour jump
// above G.ml_jump, go to a queue and are then reconstructed by the plain
// limiter, again by all threads.  load(it, s, imm, any10) fetches stencil it
// (with the immersed modifications applied), store(it, qL, qR) writes its
// edges.  Returns the number of fallbacks.
template <int NT, class Load, class Store>
__device__ __forceinline__ int recon_learned(const Grid<float> &G, uint32_t *sW, uint16_t *queue, int *qn, int total,
                                             Load load, Store store) {
  const int tid = threadIdx.x, lane = tid & 31;
  MlpLane L;
  load_lane(G.ml_frags, L);
  for (int base = tid & ~31; base < total; base += NT) {
    const int it = base + lane;
    const bool valid = it < total;
    float s[9];
    unsigned imm;
    bool any10;
    load(valid ? it : base, s, imm, any10);
    float x[9], wl[5], wr[5];
    const float jmp = normalize9(s, x);
    mlp_warp_weights(L, sW, x, wl, wr);
    const bool fb = valid && (any10 || imm != 0u || jmp > G.ml_jump);
    if (valid && !fb) {
      float qL, qR;
      edges_from_weights(s, wl, wr, qL, qR);
      store(it, qL, qR);
    }
    const unsigned m = __ballot_sync(0xffffffffu, fb);
    if (m) {
      int pos = 0;
      if (lane == 0) pos = atomicAdd(qn, __popc(m));
      pos = __shfl_sync(0xffffffffu, pos, 0);
      if (fb) queue[pos + __popc(m & ((1u << lane) - 1u))] = uint16_t(it);
    }
  }
  __syncthreads();
  const int nq = *qn;
  for (int q = tid; q < nq; q += NT) {
    const int it = queue[q];
    float s[9];
    unsigned imm;
    bool any10;
    load(it, s, imm, any10);
    float qL, qR;
    weno9_edges(s, qL, qR, !any10, (imm >> 3) & 1u, (imm >> 5) & 1u);
    store(it, qL, qR);
  }
  return nq;
}

// Reconstruction of a tile's lines of faces with the packed FP32 limiter
// (weno_all).  There are F x LINES lines of W+2 cells (positions 0..W+1,
// cells -1..W); the faces of a line read both edges of the W inner cells, the
// right edge of position 0 and the left edge of position W+1.  Inner cells go
// two per thread and iteration (weno9_edges2, recon_packed_inner); the two
// halo cells of a line go together through the one-edge form
// (weno9_outer_edges2, recon_outer_pair), which skips the two edges nobody
// reads.  Per stencil and edge the bits are those of weno9_edges.
// POS_MAJOR: consecutive threads take consecutive lines at one position (y),
// else consecutive positions of one line (x).
// mask(line, pos, imm, any10) gives a position's immersed bits (the same for
// all fields), vals(f, line, pos, s, imm) a field's stencil with the immersed
// modification applied; load(f, line, pos, s, imm, any10) is the two
// together; store(f, line, pos, qL, qR), store_outer(f, line, qR of position
// 0, qL of position W+1).
template <int NT, int F, int LINES, int W, bool POS_MAJOR, class Mask, class Vals, class Store>
__device__ __forceinline__ void recon_packed_inner(Mask mask, Vals vals, Store store) {
  constexpr int N_IN = F * LINES * W;
  auto coords = [](int it, int &f, int &line, int &pos) {
    f = it / (LINES * W);
    const int q = it % (LINES * W);
    line = POS_MAJOR ? q % LINES : q / W;
    pos = (POS_MAJOR ? q / LINES : q % W) + 1;
  };
  if constexpr (NT == LINES * W) {
    // One position per thread: walk its fields in pairs (the same pairs as
    // below, where stencil it+NT is the next field of stencil it).
    int f0, line, pos;
    coords(threadIdx.x, f0, line, pos);
    unsigned im;
    bool ax;
    mask(line, pos, im, ax);
    const bool il = ((im >> 3) & 1u) != 0, ir = ((im >> 5) & 1u) != 0;
#pragma unroll 1
    for (int f = 0; f + 1 < F; f += 2) {
      float a[9], b[9];
      vals(f, line, pos, a, im);
      vals(f + 1, line, pos, b, im);
      float2 s2[9], qL, qR;
#pragma unroll
      for (int m = 0; m < 9; m++) s2[m] = make_float2(a[m], b[m]);
      weno9_edges2(s2, qL, qR, bool2{!ax, !ax}, bool2{il, il}, bool2{ir, ir});
      store(f, line, pos, qL.x, qR.x);
      store(f + 1, line, pos, qL.y, qR.y);
    }
    if constexpr (F % 2 == 1) {
      // The odd field alone through the scalar limiter (the same bits): a
      // packed pair with an idle lane would cost the FMA pipe as much as two.
      float a[9], qL, qR;
      vals(F - 1, line, pos, a, im);
      weno9_edges(a, qL, qR, !ax, il, ir);
      store(F - 1, line, pos, qL, qR);
    }
  } else {
    for (int it = threadIdx.x; it < N_IN; it += 2 * NT) {
      const int it2 = it + NT;
      const bool two = it2 < N_IN;
      int fa, la, pa, fb, lb, pb;
      coords(it, fa, la, pa);
      float a[9], b[9];
      unsigned ia, ib;
      bool xa, xb;
      mask(la, pa, ia, xa);
      vals(fa, la, pa, a, ia);
      if (two) {
        coords(it2, fb, lb, pb);
        mask(lb, pb, ib, xb);
        vals(fb, lb, pb, b, ib);
      } else {
#pragma unroll
        for (int m = 0; m < 9; m++) b[m] = a[m];
        ib = ia;
        xb = xa;
        fb = fa, lb = la, pb = pa;
      }
      float2 s2[9], qL, qR;
#pragma unroll
      for (int m = 0; m < 9; m++) s2[m] = make_float2(a[m], b[m]);
      weno9_edges2(s2, qL, qR, bool2{!xa, !xb}, bool2{((ia >> 3) & 1u) != 0, ((ib >> 3) & 1u) != 0},
                   bool2{((ia >> 5) & 1u) != 0, ((ib >> 5) & 1u) != 0});
      store(fa, la, pa, qL.x, qR.x);
      if (two) store(fb, lb, pb, qL.y, qR.y);
    }
  }
}

template <int W, class Load, class StoreOuter>
__device__ __forceinline__ void recon_outer_pair(int f, int line, Load load, StoreOuter store_outer) {
  float a[9], b[9];
  unsigned ia, ib;
  bool xa, xb;
  load(f, line, 0, a, ia, xa);
  load(f, line, W + 1, b, ib, xb);
  float2 s2[9];
#pragma unroll
  for (int m = 0; m < 9; m++) s2[m] = make_float2(a[m], b[m]);
  const float2 q = weno9_outer_edges2(s2, bool2{!xa, !xb}, bool2{((ia >> 3) & 1u) != 0, ((ib >> 3) & 1u) != 0},
                                      bool2{((ia >> 5) & 1u) != 0, ((ib >> 5) & 1u) != 0});
  store_outer(f, line, q.x, q.y);
}

// x/y fluxes and their divergence for one (x,y) tile of one level.
// LEARNED (FP32, weno_all only): edges from the network's weights, with the
// plain limiter as the fallback.
// TMA (16x16 FP32 tiles of an undecomposed plain domain): a tile that lies
// whole in the domain takes its cross from TMA copies (maps: tensor maps of
// sin), the halo rows and columns wrapping periodically box by box; tiles at
// a precursor edge, partial tiles and halo boxes that would straddle the
// domain's edge are loaded by the threads.
template <class R, int NTR, int TX, int TY, bool IMM, bool LEARNED = false, bool DECOMP = false, bool TMA = false>
__global__ void __launch_bounds__(TX *TY, LEARNED ? PU_LEARNED_XY_MIN_BLOCKS : (sizeof(R) == 4 ? PU_XY_MIN_BLOCKS : 1)) k_xy(const Grid<R> G, const R *__restrict__ sin, R *__restrict__ txy, const __grid_constant__ XyMaps maps) {
  using Sh = XYShape<R, NTR, TX, TY, IMM, LEARNED>;
  constexpr int F = Sh::F, S = Sh::S, NT = Sh::NT, HX = Sh::HX, HY = Sh::HY, EN = Sh::EN, FN = Sh::FN;
  static_assert(!TMA || (Sh::TMA_FITS && !DECOMP && !IMM), "TMA staging: 16x16 FP32 tiles, plain domains");
  extern __shared__ __align__(16) unsigned char smem_xy[];
  unsigned char *smem_raw = TMA ? smem_xy + ((128u - (tma::saddr(smem_xy) & 127u)) & 127u) : smem_xy;
  R *H = reinterpret_cast<R *>(smem_raw);
  R *EL = H + F * HY * HX;
  R *ER = EL + F * EN;
  R *FL = ER + F * EN;
  R *YO = FL + S * FN;                                       // [2][F][TX] y halo-cell edges
  uint8_t *M = reinterpret_cast<uint8_t *>(YO + Sh::YON);
  uint16_t *MX = reinterpret_cast<uint16_t *>(M + Sh::MB);  // [TY][TX+2] x-stencil masks (immersed only)
  uint16_t *MY = MX + TY * (TX + 2);                          // [TY+2][TX] y-stencil masks
  unsigned char *lrn = reinterpret_cast<unsigned char *>(YO + Sh::YON) + (IMM ? Sh::MB + Sh::MASKB : 0);
  int *qn = reinterpret_cast<int *>(lrn);                    // [2] fallback counts (x, y)
  uint32_t *sW = reinterpret_cast<uint32_t *>(lrn + 16) + (threadIdx.x >> 5) * (mlp::WARP_SMEM_BYTES / 4);
  uint16_t *queue = reinterpret_cast<uint16_t *>(FL);

  const int tid = threadIdx.x;
  const int i0 = G.i_first + int(blockIdx.x) * TX, j0 = G.j_first + int(blockIdx.y) * TY,
            k = G.k_first + int(blockIdx.z);
  const int nx = G.nx, ny = G.ny;
  const size_t plane = size_t(k) * G.NP;
  const bool sim2d = G.sim2d != 0;
  if (LEARNED && tid < 2) qn[tid] = 0;

  // 0. TMA staging of the tile's cross (block-uniform decision).  Box origins:
  // the interior at (i0, j0); the 5 rows above at j0-5 (ny-5 for the first
  // tile row), below at j0+16 (0 for the last); the 8 columns left at i0-8
  // (nx-8), right at i0+16 (0).  Every x origin is a multiple of 8.
  bool staged = false;
  if constexpr (TMA) {
    if (!sim2d && i0 + TX <= nx && j0 + TY <= ny) {
      const bool px = G.bc_x != BC_PRECURSOR, py = G.bc_y != BC_PRECURSOR;
      const int xw = i0 > 0 ? i0 - 8 : (px ? nx - 8 : -1);
      const int xe = i0 + TX < nx ? (i0 + TX + 8 <= nx ? i0 + TX : -1) : (px ? 0 : -1);
      const int yn = j0 > 0 ? j0 - 5 : (py ? ny - 5 : -1);
      const int ys = j0 + TY < ny ? (j0 + TY + 5 <= ny ? j0 + TY : -1) : (py ? 0 : -1);
      staged = xw >= 0 && xe >= 0 && yn >= 0 && ys >= 0;
      if (staged) {
        uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw + Sh::bar_off);
        if (tid == 0) {
          tma::mbar_init(bar);
          tma::mbar_expect(bar, uint32_t(sizeof(R) * S * (256 + 80 + 80 + 128 + 128)));
          tma::load_4d(smem_raw + Sh::st_in, &maps.in, i0, j0, k, 0, bar);
          tma::load_4d(smem_raw + Sh::st_top, &maps.ns, i0, yn, k, 0, bar);
          tma::load_4d(smem_raw + Sh::st_bot, &maps.ns, i0, ys, k, 0, bar);
          tma::load_4d(smem_raw + Sh::st_west, &maps.ew, xw, j0, k, 0, bar);
          tma::load_4d(smem_raw + Sh::st_east, &maps.ew, xe, j0, k, 0, bar);
        }
        __syncthreads();
        if (!__syncthreads_and(tma::mbar_wait(bar, 0))) {
          // The copies did not complete: report it, give them a last bounded
          // wait, and give up the tile.
          if (tid == 0) atomicOr(G.err, ERR_TMA);
          tma::mbar_wait(bar, 0);
          return;
        }
      }
    }
  }

  // 1. Primitive fields of the tile, its x halo rows and its y halo columns.
  constexpr int NA = TY * HX, NB = 10 * TX;
  for (int it = tid; it < NA + (sim2d ? 0 : NB); it += NT) {
    int r, c;
    if (it < NA) {
      r = 5 + it / HX;
      c = it % HX;
    } else {
      int b = it - NA, rr = b / TX;
      c = 5 + b % TX;
      r = rr < 5 ? rr : rr + TY;
    }
    const int gi = i0 - 5 + c, gj = j0 - 5 + r;
    R w[F];
    if (TMA && staged) {
      // The cell's place in the staged boxes ([S][rows][cols]).
      const R *src;
      int fstride;
      if (r < 5) {
        src = reinterpret_cast<const R *>(smem_raw + Sh::st_top) + r * 16 + (c - 5);
        fstride = 80;
      } else if (r >= 5 + TY) {
        src = reinterpret_cast<const R *>(smem_raw + Sh::st_bot) + (r - 5 - TY) * 16 + (c - 5);
        fstride = 80;
      } else if (c < 5) {
        src = reinterpret_cast<const R *>(smem_raw + Sh::st_west) + (r - 5) * 8 + (c + 3);
        fstride = 128;
      } else if (c >= 5 + TX) {
        src = reinterpret_cast<const R *>(smem_raw + Sh::st_east) + (r - 5) * 8 + (c - 5 - TX);
        fstride = 128;
      } else {
        src = reinterpret_cast<const R *>(smem_raw + Sh::st_in) + (r - 5) * 16 + (c - 5);
        fstride = 256;
      }
      R q[S];
#pragma unroll
      for (int s2 = 0; s2 < S; s2++) q[s2] = src[s2 * fstride];
      prims_of<R, NTR>(G, q, k, w);
    } else if constexpr (DECOMP) {
      const R *src;
      size_t fs, q;
      const uint8_t *fl;
      tile_source(G, sin, gi, gj, k, src, fs, q, fl);
      prims_s<R, NTR>(G, src, fs, q, k, w);
      if (IMM) M[r * HX + c] = fl ? __ldg(fl) : uint8_t(0);
    } else {
      const int vi = G.bc_x == BC_PRECURSOR ? clampi(gi, nx) : wrapi(gi, nx);
      const int vj = G.bc_y == BC_PRECURSOR ? clampi(gj, ny) : wrapi(gj, ny);
      prims<R, NTR>(G, sin, plane + size_t(vj) * nx + vi, k, w);
      if (IMM) M[r * HX + c] = __ldg(G.flags + plane + size_t(wrapi(gj, ny)) * nx + wrapi(gi, nx));
    }
#pragma unroll
    for (int f = 0; f < F; f++) H[(f * HY + r) * HX + c] = w[f];
  }
  __syncthreads();
  if (IMM) {
    // 1b. The stencil mask of every x and y stencil position, once for all
    // fields: bits 0-8 the immersed flags of the stencil's cells, bit 9 an
    // immersed cell within 10 of its centre.
    constexpr int NXM = TY * (TX + 2), NYM = (TY + 2) * TX;
    for (int it = tid; it < NXM + (sim2d ? 0 : NYM); it += NT) {
      const uint8_t *m0;
      int step;
      if (it < NXM) {
        m0 = M + (5 + it / (TX + 2)) * HX + it % (TX + 2);
        step = 1;
      } else {
        const int q = it - NXM;
        m0 = M + (q / TX) * HX + 5 + q % TX;
        step = HX;
      }
      unsigned e = (m0[4 * step] & FLAG_ANY10) ? 0x200u : 0u;
#pragma unroll
      for (int m = 0; m < 9; m++) e |= (unsigned(m0[m * step]) & FLAG_IMM) << m;
      if (it < NXM) MX[it] = uint16_t(e);
      else MY[it - NXM] = uint16_t(e);
    }
    __syncthreads();
  }

  // 2. x edges of cells -1..TX of every tile row (position c = cell + 1).
  auto mask_xc = [&](int r, int c, unsigned &imm, bool &any10) {
    imm = 0;
    any10 = false;
    if (IMM) {
      const unsigned e = MX[r * (TX + 2) + c];
      imm = e & 0x1ffu;
      any10 = (e & 0x200u) != 0;
    }
  };
  auto vals_xc = [&](int f, int r, int c, R (&s)[9], unsigned imm) {
    const R *row = H + (f * HY + 5 + r) * HX + c;
#pragma unroll
    for (int m = 0; m < 9; m++) s[m] = row[m];
    if (IMM && (f == iV || f == iW || f == iP)) der0_modify(s, imm);
  };
  auto load_xc = [&](int f, int r, int c, R (&s)[9], unsigned &imm, bool &any10) {
    mask_xc(r, c, imm, any10);
    vals_xc(f, r, c, s, imm);
  };
  auto store_xc = [&](int f, int r, int c, R qL, R qR) {
    EL[f * EN + r * (TX + 2) + c] = qL;
    ER[f * EN + r * (TX + 2) + c] = qR;
  };
  auto load_x = [&](int it, R (&s)[9], unsigned &imm, bool &any10) {
    const int f = it / Sh::EXN, rem = it % Sh::EXN;
    load_xc(f, rem / (TX + 2), rem % (TX + 2), s, imm, any10);
  };
  // y stencil of cell rr-1 of tile column cc (position rr = 0..TY+1).
  auto mask_yc = [&](int cc, int rr, unsigned &imm, bool &any10) {
    imm = 0;
    any10 = false;
    if (IMM) {
      const unsigned e = MY[rr * TX + cc];
      imm = e & 0x1ffu;
      any10 = (e & 0x200u) != 0;
    }
  };
  auto vals_yc = [&](int f, int cc, int rr, R (&s)[9], unsigned imm) {
    const R *col = H + (f * HY + rr) * HX + 5 + cc;
#pragma unroll
    for (int m = 0; m < 9; m++) s[m] = col[m * HX];
    if (IMM && (f == iU || f == iW || f == iP)) der0_modify(s, imm);
  };
  auto load_yc = [&](int f, int cc, int rr, R (&s)[9], unsigned &imm, bool &any10) {
    mask_yc(cc, rr, imm, any10);
    vals_yc(f, cc, rr, s, imm);
  };
  auto store_x = [&](int it, R qL, R qR) {
    const int f = it / Sh::EXN, rem = it % Sh::EXN;
    EL[f * EN + rem] = qL;
    ER[f * EN + rem] = qR;
  };
  int n_fb = 0;
  bool packed = false;
  if constexpr (std::is_same<R, float>::value && PU_PACKED_LIMITER && !LEARNED) {
    packed = G.weno_all != 0;
    if (packed) {
      recon_packed_inner<NT, F, TY, TX, false>(mask_xc, vals_xc, store_xc);
      // Halo pairs of the x lines, and already those of the y lines (kept in
      // YO until the y phase), so that every thread takes one pair here and
      // the y phase is the inner rounds alone.
      const int nxo = F * TY, nyo = sim2d ? 0 : F * TX;
      for (int p = tid; p < nxo + nyo; p += NT) {
        if (p < nxo) {
          recon_outer_pair<TX>(p / TY, p % TY, load_xc, [&](int f, int r, R qR0, R qL1) {
            ER[f * EN + r * (TX + 2)] = qR0;
            EL[f * EN + r * (TX + 2) + TX + 1] = qL1;
          });
        } else {
          const int q = p - nxo;
          recon_outer_pair<TY>(q / TX, q % TX, load_yc, [&](int f, int cc, R qR0, R qL1) {
            YO[f * TX + cc] = qR0;
            YO[(F + f) * TX + cc] = qL1;
          });
        }
      }
    }
  }
  if constexpr (LEARNED) {
    n_fb += recon_learned<NT>(G, sW, queue, qn, F * Sh::EXN, load_x, store_x);
  } else if (!packed) {
    for (int it = tid; it < F * Sh::EXN; it += NT) {
      R s[9];
      unsigned imm;
      bool any10;
      load_x(it, s, imm, any10);
      R qL, qR;
      if (!any10 && !G.weno_all) linear9_edges(s, qL, qR);
      else weno9_edges(s, qL, qR, !any10, (imm >> 3) & 1u, (imm >> 5) & 1u);
      store_x(it, qL, qR);
    }
  }
  __syncthreads();

  // 3. Riemann fluxes on x faces 0..TX (face fi between cells fi-1 and fi).
  const R hr = __ldg(G.rho_h + k + HS), ht = __ldg(G.theta_h + k + HS);
  for (int it = tid; it < Sh::FXN; it += NT) {
    const int r = it / (TX + 1), fi = it % (TX + 1);
    const int cl = r * (TX + 2) + fi, cr = cl + 1;
    R L[F], Rt[F];
#pragma unroll
    for (int f = 0; f < F; f++) {
      L[f] = ER[f * EN + cl];
      Rt[f] = EL[f * EN + cr];
    }
    if (G.bc_x == BC_PRECURSOR) {  // edge_exchange precursor mirror (dynamics_rk.h:864-875)
      const int gf = i0 + fi;
#pragma unroll
      for (int f = 0; f < F; f++) {
        if (gf == 0 && G.gx0) L[f] = Rt[f];
        if (gf == nx && G.gx1) Rt[f] = L[f];
      }
    }
    R fl[S];
    riemann<R, NTR>(L, Rt, hr, ht, iU, fl);
#pragma unroll
    for (int s = 0; s < S; s++) FL[s * FN + it] = fl[s];
  }
  __syncthreads();

  // 4. x divergence of this thread's cell.
  const int r = tid / TX, c = tid % TX;
  R tend[S];
#pragma unroll
  for (int s = 0; s < S; s++) tend[s] = -(FL[s * FN + r * (TX + 1) + c + 1] - FL[s * FN + r * (TX + 1) + c]) * G.rdx;

  if (!sim2d) {
    // 5. y edges of cells -1..TY of every tile column.
    auto load_y = [&](int it, R (&s)[9], unsigned &imm, bool &any10) {
      const int f = it / Sh::EYN, rem = it % Sh::EYN;
      load_yc(f, rem % TX, rem / TX, s, imm, any10);
    };
    auto store_y = [&](int it, R qL, R qR) {
      const int f = it / Sh::EYN, rem = it % Sh::EYN;
      EL[f * EN + rem] = qL;
      ER[f * EN + rem] = qR;
    };
    if constexpr (LEARNED) {
      __syncthreads();   // step 4 has read the flux buffer that holds the queue
      n_fb += recon_learned<NT>(G, sW, queue, qn + 1, F * Sh::EYN, load_y, store_y);
    } else if (packed) {
      if constexpr (std::is_same<R, float>::value) {
        recon_packed_inner<NT, F, TX, TY, true>(mask_yc, vals_yc, [&](int f, int cc, int rr, R qL, R qR) {
          EL[f * EN + rr * TX + cc] = qL;
          ER[f * EN + rr * TX + cc] = qR;
        });
        for (int p = tid; p < F * TX; p += NT) {   // the halo-cell edges taken in the x phase
          const int f = p / TX, cc = p % TX;
          ER[f * EN + cc] = YO[p];
          EL[f * EN + (TY + 1) * TX + cc] = YO[F * TX + p];
        }
      }
    } else {
      for (int it = tid; it < F * Sh::EYN; it += NT) {
        R s[9];
        unsigned imm;
        bool any10;
        load_y(it, s, imm, any10);
        R qL, qR;
        if (!any10 && !G.weno_all) linear9_edges(s, qL, qR);
        else weno9_edges(s, qL, qR, !any10, (imm >> 3) & 1u, (imm >> 5) & 1u);
        store_y(it, qL, qR);
      }
    }
    __syncthreads();
    // 6. Riemann fluxes on y faces 0..TY.
    for (int it = tid; it < Sh::FYN; it += NT) {
      const int fj = it / TX, cc = it % TX;
      const int cl = fj * TX + cc, cr = cl + TX;
      R L[F], Rt[F];
#pragma unroll
      for (int f = 0; f < F; f++) {
        L[f] = ER[f * EN + cl];
        Rt[f] = EL[f * EN + cr];
      }
      if (G.bc_y == BC_PRECURSOR) {
        const int gf = j0 + fj;
#pragma unroll
        for (int f = 0; f < F; f++) {
          if (gf == 0 && G.gy0) L[f] = Rt[f];
          if (gf == ny && G.gy1) Rt[f] = L[f];
        }
      }
      R fl[S];
      riemann<R, NTR>(L, Rt, hr, ht, iV, fl);
#pragma unroll
      for (int s = 0; s < S; s++) FL[s * FN + it] = fl[s];
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < S; s++) tend[s] -= (FL[s * FN + (r + 1) * TX + c] - FL[s * FN + r * TX + c]) * G.rdy;
  }
  if (LEARNED && tid == 0) {
    const int total = F * (Sh::EXN + (sim2d ? 0 : Sh::EYN));
    atomicAdd(G.ml_counts, (unsigned long long)(total - n_fb));
    atomicAdd(G.ml_counts + 1, (unsigned long long)n_fb);
  }

  const int gi = i0 + c, gj = j0 + r;
  if (gi < nx && gj < ny) {
    const size_t idx = plane + size_t(gj) * nx + gi;
#pragma unroll
    for (int s = 0; s < S; s++) txy[s * G.N + idx] = tend[s];
  }
}

// Immersed relaxation toward the hydrostatic state and positivity of
// positive-definite tracers (enforce_immersed_boundaries, dynamics_rk.h:429-469)
// on one cell's perturbation state.
template <class R, int NTR, bool IMM>
__device__ __forceinline__ void enforce_cell(const Grid<R> &G, R (&q)[5 + NTR], size_t idx, int k) {
  if (IMM) {
    const R mult = __ldg(G.imm_mult + idx);
    q[0] = q[0] + (R(0) - q[0]) * mult;
    q[1] = q[1] + (R(0) - q[1]) * mult;
    q[2] = q[2] + (R(0) - q[2]) * mult;
    q[3] = q[3] + (R(0) - q[3]) * mult;
    q[4] = q[4] + (__ldg(G.rt_target + k) - q[4]) * mult;
#pragma unroll
    for (int t = 0; t < NTR; t++) q[5 + t] = q[5 + t] + (R(0) - q[5 + t]) * mult;
  }
#pragma unroll
  for (int t = 0; t < NTR; t++)
    if ((G.tracer_positive >> t) & 1u) q[5 + t] = fmax(R(0), q[5 + t]);
}

template <class R, int NTR, int TX, int TY, bool LEARNED = false>
struct ZShape {
  static constexpr int F = 6 + NTR, NT = TX * TY;
  // 9-plane ring of primitive fields, left edges of the current cell, right
  // edges of the current and the previous cell; all thread-private columns.
  // Learned mode adds per-warp network scratch and a per-warp fallback queue
  // of up to F*32 entries.
  static constexpr size_t learned_bytes = LEARNED ? size_t(NT / 32) * (mlp::WARP_SMEM_BYTES + F * 32 * 4) : 0;
  static constexpr size_t bytes = sizeof(R) * (9 + 3) * size_t(F) * NT + learned_bytes;
};

// Raw state of one cell (S values) for a later conversion to primitive fields.
// The end of one cell's stage in both z kernels: tend = txy - dF/dz plus
// gravity and Coriolis, the combination a_n*sn + (1-a_n)*sin + a_dt*tend
// (sn null: sin + a_dt*tend), n_enforce applications of the immersed and
// positivity enforcement, the store and the finite check.  dF is the flux
// difference F(k+1/2) - F(k-1/2); qn(s) gives field s of sn and is called
// only when sn is set.
template <class R, int NTR, bool IMM, class Qn>
__device__ __forceinline__ void finish_cell(const Grid<R> &G, const R (&qin)[5 + NTR], const R (&tx)[5 + NTR],
                                            Qn qn, const R (&dF)[5 + NTR], bool have_sn, R a_n, R a_dt,
                                            int n_enforce, size_t idx, int k, R *sout) {
  constexpr int S = 5 + NTR;
  R tend[S], out[S];
#pragma unroll
  for (int s = 0; s < S; s++) tend[s] = tx[s] - dF[s] * G.rdz;
  if (G.sim2d) tend[iV] = R(0);
  if (G.enable_gravity) tend[iW] += -G.grav * qin[iR];
  if (G.fcor != R(0) && !G.sim2d) {
    tend[iU] += G.fcor * qin[iV];
    tend[iV] -= G.fcor * qin[iU];
  }
  if (have_sn) {
#pragma unroll
    for (int s = 0; s < S; s++) out[s] = qin[s] + fma(a_n, qn(s) - qin[s], a_dt * tend[s]);
  } else {
#pragma unroll
    for (int s = 0; s < S; s++) out[s] = qin[s] + a_dt * tend[s];
  }
  for (int e = 0; e < n_enforce; e++) enforce_cell<R, NTR, IMM>(G, out, idx, k);
  bool bad = false;
#pragma unroll
  for (int s = 0; s < S; s++) {
    bad |= !isfinite(out[s]);
    sout[s * G.N + idx] = out[s];
  }
  if (bad) atomicOr(G.err, ERR_NONFINITE);
}

// z fluxes, their divergence, sources and the SSPRK3 stage combination
// a_n*sn + (1-a_n)*sin + a_dt*tend, evaluated as
//   out = sin + (a_n*(sn - sin) + a_dt*tend),   tend = txy - dFz/dz + sources
// (sn null: out = sin + a_dt*tend), followed by n_enforce applications of the
// immersed/positivity enforcement.  The weights 1/3 and 2/3 of the last stage
// are inexact in FP32 and their sum is 1 + 6e-8: the direct form would scale
// the stored state by that factor every step (a drift of ~1e-5 over 200
// steps); in this form the weight error only touches the per-step change.
// One thread per column marches up levels k0..k1-1 of its chunk.  The raw
// state of the plane entering the ring is loaded one step ahead, and the
// inputs of the cell being finalised are loaded before the reconstruction, so
// global-load latency overlaps the limiter work.  The field loop is not
// unrolled: one inlined limiter keeps the kernel small.
// LEARNED (FP32, weno_all only, every block full: nx % TX == ny % TY == 0):
// each warp evaluates the network for its 32 columns field by field; stencils
// near walls or immersed cells, or with a normalised neighbour jump above
// G.ml_jump, are queued per warp and reconstructed by the plain limiter after
// the level's field loop, by all lanes of the warp.
template <class R, int NTR, int TX, int TY, bool IMM, bool LEARNED = false>
__global__ void __launch_bounds__(TX *TY, LEARNED ? PU_LEARNED_Z_MIN_BLOCKS : (sizeof(R) == 4 ? PU_Z_MIN_BLOCKS : 1)) k_z(const Grid<R> G, const R *__restrict__ sin, const R *sn, R *sout,
                                              const R *__restrict__ txy, R a_n, R a_dt, int n_enforce,
                                              int kchunk) {
  constexpr int F = 6 + NTR, S = 5 + NTR, NT = TX * TY;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R *ring = reinterpret_cast<R *>(smem_raw);   // [9][F][NT]
  R *eL = ring + 9 * F * NT;                     // [F][NT]
  R *eR = eL + F * NT;                           // [2][F][NT]
  uint32_t *sW = reinterpret_cast<uint32_t *>(eR + 2 * F * NT) +
                 (threadIdx.x >> 5) * ((mlp::WARP_SMEM_BYTES + F * 32 * 4) / 4);
  uint32_t *wq = sW + mlp::WARP_SMEM_BYTES / 4;  // per-warp fallback queue
  unsigned long long n_learned = 0, n_fallback = 0;
  const int tid = threadIdx.x;
  const int i = blockIdx.x * TX + tid % TX, j = blockIdx.y * TY + tid / TX;
  if (i >= G.nx || j >= G.ny) return;            // no block-wide synchronisation below
  const int nz = G.nz;
  const int k0 = blockIdx.z * kchunk, k1 = min(nz, k0 + kchunk);
  const bool wall = G.bc_z == BC_WALL;
  const size_t col = size_t(j) * G.nx + i, NP = G.NP;

  auto slot_of = [](int p) { return (p % 9 + 9) % 9; };
  // Level whose state feeds plane p (wall halos replicate the boundary cell,
  // periodic halos wrap; :780-797).
  auto src_level = [&](int p) { return (p >= 0 && p < nz) ? p : (wall ? clampi(p, nz) : wrapi(p, nz)); };
  auto store_plane = [&](int p, const R (&q)[S]) {
    R w[F];
    prims_of<R, NTR>(G, q, src_level(p), w);
    if (wall && (p < 0 || p >= nz)) {
      w[iW] = R(0);
      w[iT] = R(0);
    }
    R *dst = ring + slot_of(p) * F * NT + tid;
#pragma unroll
    for (int f = 0; f < F; f++) dst[f * NT] = w[f];
  };
  // Immersed bits of the z stencil of canonical cell cc: levels beyond the
  // domain count as immersed (the z halos of the proportion are 1, :1031-1034).
  auto stencil_flags = [&](int cc) {
    unsigned imm = 0;
#pragma unroll
    for (int m = 0; m < 9; m++) {
      const int p = cc - 4 + m;
      unsigned b = (p < 0 || p >= nz) ? 1u : (IMM ? (unsigned(__ldg(G.flags + size_t(p) * NP + col)) & FLAG_IMM) : 0u);
      imm |= b << m;
    }
    return imm;
  };

  const int cstart = (wall && k0 == 0) ? 0 : k0 - 1;
  {
    R q[S];
    for (int p = cstart - 4; p <= cstart + 3; p++) {
      load_cell<R, NTR>(G, sin, size_t(src_level(p)) * NP + col, q);
      store_plane(p, q);
    }
  }
  R qnext[S];   // raw state of plane c+4, loaded one step ahead
  load_cell<R, NTR>(G, sin, size_t(src_level(cstart + 4)) * NP + col, qnext);

  R Fp[S];
#pragma unroll
  for (int s = 0; s < S; s++) Fp[s] = R(0);
  int par = 0;   // eR double-buffer index of the current cell
  unsigned imm_prev = 0;
  int cc_prev = -1000;   // canonical cell whose stencil flags imm_prev holds

  for (int c = cstart; c <= k1; c++) {
    store_plane(c + 4, qnext);
    if (c < k1) load_cell<R, NTR>(G, sin, size_t(src_level(c + 5)) * NP + col, qnext);
    // Inputs of cell c-1 (finalised below), loaded before the reconstruction.
    const bool fin = c > cstart && c - 1 >= k0;
    R qin[S], qn[S], tx[S];
    if (fin) {
      const size_t idx = size_t(c - 1) * NP + col;
#pragma unroll
      for (int s = 0; s < S; s++) {
        qin[s] = sin[s * G.N + idx];
        tx[s] = txy[s * G.N + idx];
        qn[s] = sn ? sn[s * G.N + idx] : R(0);
      }
    }
    const bool have_cell = !(wall && c >= nz);
    R *eRc = eR + par * F * NT + tid, *eRp = eR + (par ^ 1) * F * NT + tid;
    if (have_cell) {
      const int cc = wall ? c : wrapi(c, nz);
      // Stencil flags of cc: one level beyond the previous cell's, one new
      // flag; else (the first cell, a periodic wrap) all nine.
      if (cc == cc_prev + 1) {
        const int p = cc + 4;
        const unsigned b =
            (p < 0 || p >= nz) ? 1u : (IMM ? (unsigned(__ldg(G.flags + size_t(p) * NP + col)) & FLAG_IMM) : 0u);
        imm_prev = (imm_prev >> 1) | (b << 8);
      } else {
        imm_prev = stencil_flags(cc);
      }
      cc_prev = cc;
      const unsigned imm = imm_prev;
      const bool any10 = IMM && (__ldg(G.flags + size_t(cc) * NP + col) & FLAG_ANY10);
      int sl[9];
#pragma unroll
      for (int m = 0; m < 9; m++) sl[m] = slot_of(c - 4 + m) * F * NT + tid;
      if constexpr (LEARNED) {
        const int lane = tid & 31;
        MlpLane L;
        load_lane(G.ml_frags, L);
        int cnt = 0;   // queued stencils of this warp (the same in every lane)
#pragma unroll 1
        for (int f = 0; f < F; f++) {
          float s[9], x[9], wl[5], wr[5];
#pragma unroll
          for (int m = 0; m < 9; m++) s[m] = ring[sl[m] + f * NT];
          const float jmp = normalize9(s, x);
          mlp_warp_weights(L, sW, x, wl, wr);
          const bool fb = any10 || imm != 0u || jmp > G.ml_jump;
          if (!fb) {
            float qL, qR;
            edges_from_weights(s, wl, wr, qL, qR);
            eL[f * NT + tid] = qL;
            eRc[f * NT] = qR;
          }
          const unsigned mk = __ballot_sync(0xffffffffu, fb);
          if (fb)
            wq[cnt + __popc(mk & ((1u << lane) - 1u))] =
                unsigned(f) | (unsigned(lane) << 4) | (imm << 9) | (unsigned(any10) << 18);
          cnt += __popc(mk);
        }
        __syncwarp();
        for (int q = lane; q < cnt; q += 32) {
          const unsigned e = wq[q];
          const int f = int(e & 15u), t2 = (tid & ~31) + int((e >> 4) & 31u);
          const unsigned im = (e >> 9) & 511u;
          float s[9];
#pragma unroll
          for (int m = 0; m < 9; m++) s[m] = ring[sl[m] - tid + t2 + f * NT];
          if (f == iU || f == iV || f == iP) der0_modify(s, im);
          float qL, qR;
          weno9_edges(s, qL, qR, ((e >> 18) & 1u) == 0u, (im >> 3) & 1u, (im >> 5) & 1u);
          eL[f * NT + t2] = qL;
          eR[par * F * NT + f * NT + t2] = qR;
        }
        __syncwarp();
        n_learned += unsigned(F * 32 - cnt);
        n_fallback += unsigned(cnt);
      } else {
        auto one_field = [&](int f) {
          R s[9];
#pragma unroll
          for (int m = 0; m < 9; m++) s[m] = ring[sl[m] + f * NT];
          if (f == iU || f == iV || f == iP) der0_modify(s, imm);
          R qL, qR;
          if (!any10 && !G.weno_all) linear9_edges(s, qL, qR);
          else weno9_edges(s, qL, qR, !any10, (imm >> 3) & 1u, (imm >> 5) & 1u);
          eL[f * NT + tid] = qL;
          eRc[f * NT] = qR;
        };
        bool done = false;
        if constexpr (std::is_same<R, float>::value && PU_PACKED_Z) {
          if (G.weno_all) {   // pairs of fields through the packed limiter
#pragma unroll 1
            for (int f = 0; f + 1 < F; f += 2) {
              float a[9], b[9];
#pragma unroll
              for (int m = 0; m < 9; m++) {
                a[m] = ring[sl[m] + f * NT];
                b[m] = ring[sl[m] + (f + 1) * NT];
              }
              if (f == iU || f == iV || f == iP) der0_modify(a, imm);
              if (f + 1 == iU || f + 1 == iV || f + 1 == iP) der0_modify(b, imm);
              float2 s2[9], qL, qR;
#pragma unroll
              for (int m = 0; m < 9; m++) s2[m] = make_float2(a[m], b[m]);
              const bool il = (imm >> 3) & 1u, ir = (imm >> 5) & 1u;
              weno9_edges2(s2, qL, qR, bool2{!any10, !any10}, bool2{il, il}, bool2{ir, ir});
              eL[f * NT + tid] = qL.x;
              eL[(f + 1) * NT + tid] = qL.y;
              eRc[f * NT] = qR.x;
              eRc[(f + 1) * NT] = qR.y;
            }
            if (F & 1) one_field(F - 1);
            done = true;
          }
        }
        if (!done) {
#pragma unroll 1
          for (int f = 0; f < F; f++) one_field(f);
        }
      }
    }
    if (c > cstart || (wall && c == 0)) {
      // Face c between cells c-1 and c (edge_exchange z, :891-908).
      R Lf[F], Rf[F];
      if (wall && c == 0) {
#pragma unroll
        for (int f = 0; f < F; f++) Lf[f] = Rf[f] = eL[f * NT + tid];
        Lf[iW] = Rf[iW] = Lf[iT] = Rf[iT] = R(0);
      } else if (wall && c == nz) {
#pragma unroll
        for (int f = 0; f < F; f++) Lf[f] = Rf[f] = eRp[f * NT];
        Lf[iW] = Rf[iW] = Lf[iT] = Rf[iT] = R(0);
      } else {
#pragma unroll
        for (int f = 0; f < F; f++) {
          Lf[f] = eRp[f * NT];
          Rf[f] = eL[f * NT + tid];
        }
      }
      R Fc[S];
      riemann<R, NTR>(Lf, Rf, __ldg(G.rho_e + c), __ldg(G.theta_e + c), iW, Fc);
      if (fin) {
        R dF[S];
#pragma unroll
        for (int s = 0; s < S; s++) dF[s] = Fc[s] - Fp[s];
        finish_cell<R, NTR, IMM>(G, qin, tx, [&](int s) { return qn[s]; }, dF, sn != nullptr, a_n, a_dt,
                                 n_enforce, size_t(c - 1) * NP + col, c - 1, sout);
      }
#pragma unroll
      for (int s = 0; s < S; s++) Fp[s] = Fc[s];
    }
    par ^= 1;
  }
  if (LEARNED && (tid & 31) == 0) {
    atomicAdd(G.ml_counts, n_learned);
    atomicAdd(G.ml_counts + 1, n_fallback);
  }
}

// Shared memory of k_zt: primitive fields of the tile's columns at levels
// k0-5 .. k0+TZ+4 and the left/right z edges of the cells at levels
// k0-1 .. k0+TZ.
//
// With TMA staging, the raw stage input of levels k0-5 .. k0+TZ+4
// ([S][HZ][TX], x fastest) lands in the edge buffers, which are idle until
// the primitive fields have been formed from it; when they fit beside four
// blocks per SM, the cell inputs of the finalisation -- the stage input, the
// step's initial state and the x/y tendency of levels k0 .. k0+TZ-1
// ([S][TZ][TX] each) -- land in buffers of their own, copied while the block
// reconstructs.  Two mbarriers complete the copies.
template <int NTR, int TX, int TZ, bool IMM = false>
struct ZTShape {
  static constexpr int F = 6 + NTR, S = 5 + NTR, NT = TX * TZ, HZ = TZ + 10;
  static constexpr int EN = (TZ + 2) * TX;
  static constexpr size_t al(size_t b) { return (b + 127) / 128 * 128; }
  // Immersed domains add one flag byte per level and column (bit 0 immersed,
  // bit 1 an immersed cell within 10).
  static constexpr size_t base_bytes = sizeof(float) * (size_t(F) * HZ * TX + 2 * size_t(F) * EN) +
                                       (IMM ? (size_t(HZ) * TX + 15) / 16 * 16 : 0);
  static constexpr size_t bytes = base_bytes;
  // The TMA instantiation rounds the start of its dynamic shared memory up to
  // 128 bytes (the alignment of the TMA destinations): PAD bytes more.
  static constexpr size_t PAD = 128;
  // TMA staging (byte offsets from the start of shared memory).
  static constexpr size_t el_off = sizeof(float) * size_t(F) * HZ * TX;
  static constexpr size_t raw_off = al(el_off);
  static constexpr size_t raw_bytes = sizeof(float) * size_t(S) * HZ * TX;
  static constexpr size_t cell_bytes = sizeof(float) * size_t(S) * TZ * TX;
  static_assert(raw_off + raw_bytes <= el_off + sizeof(float) * 2 * size_t(F) * EN, "raw tile exceeds the edge buffers");
  static constexpr size_t cells_off = al(base_bytes);
  static constexpr size_t bar_off = cells_off + 3 * cell_bytes;
  static constexpr size_t tma_bytes_prefetch = bar_off + 16;
  // Four blocks per SM share 228 KB (1 KB of it reserved per block).
  static constexpr bool PREFETCH = 4 * (tma_bytes_prefetch + PAD + 1024) <= 228 * 1024;
  static constexpr size_t tma_bar_off = PREFETCH ? bar_off : al(base_bytes);
  static constexpr size_t tma_bytes = tma_bar_off + 16 + PAD;
};

// Tensor maps of one k_zt launch (TMA staging): the stage input with the
// halo box (TX, 1, TZ+10, S) and with the cell box (TX, 1, TZ, S), the step's
// initial state and the x/y tendency with the cell box.
struct ZtMaps {
  CUtensorMap raw, qin, sn, txy;
};

// The z operator and the stage combination of k_z on a tile of TX columns of
// one row by TZ levels, with the work spread over the block instead of
// marched: the same results bit for bit (the same primitive fields, face
// states, limiter bits per stencil, Riemann fluxes and combination).  The
// primitive fields of levels k0-5 .. k0+TZ+4 go to shared memory; the z edges
// of the TZ inner cells of each column come from the packed limiter two
// stencils per thread, the two cells that close a column (k0-1: right edge,
// k0+TZ: left edge) from its one-edge form; then each thread takes the
// Riemann fluxes through the two faces of its cell and finalises it.  FP32
// with weno_all (IMM: domains with immersed cells, whose level flags go to
// shared memory with the fields); every other form keeps the march.
//
// TMA: the raw tile and the finalisation's cell inputs come from TMA copies
// (maps: tensor maps of sin, sn and txy); rows the halo box does not hold
// (the wrapped levels of a periodic z) and, when the cell buffers do not
// fit, the cell inputs are read per thread as without it.  Columns beyond
// the domain read zero there instead of the last column; their results are
// discarded either way.
template <int NTR, int TX, int TZ, bool IMM, bool TMA = false>
__global__ void __launch_bounds__(TX *TZ, PU_ZT_MIN_BLOCKS) k_zt(const Grid<float> G, const float *__restrict__ sin,
                                                               const float *sn, float *sout,
                                                               const float *__restrict__ txy, float a_n, float a_dt,
                                                               int n_enforce, const __grid_constant__ ZtMaps maps) {
  using R = float;
  using Sh = ZTShape<NTR, TX, TZ, IMM>;
  constexpr int F = Sh::F, S = Sh::S, NT = Sh::NT, HZ = Sh::HZ;
  extern __shared__ __align__(16) unsigned char smem_zt[];
  unsigned char *smem_raw = TMA ? smem_zt + ((128u - (tma::saddr(smem_zt) & 127u)) & 127u) : smem_zt;
  R *H = reinterpret_cast<R *>(smem_raw);   // [F][HZ][TX]
  R *EL = H + F * HZ * TX;                   // [F][TZ+2][TX]
  R *ER = EL + F * Sh::EN;
  uint8_t *M = reinterpret_cast<uint8_t *>(ER + F * Sh::EN);   // [HZ][TX], immersed domains
  R *RAW = reinterpret_cast<R *>(smem_raw + Sh::raw_off);     // [S][HZ][TX] (TMA), in the edge buffers
  R *QIN = reinterpret_cast<R *>(smem_raw + Sh::cells_off);   // [S][TZ][TX] (TMA with PREFETCH)
  R *SN = QIN + S * TZ * TX;
  R *TXY = SN + S * TZ * TX;
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw + Sh::tma_bar_off);
  const int tid = threadIdx.x;
  const int i0 = blockIdx.x * TX, j = blockIdx.y, k0 = (G.c_first + int(blockIdx.z)) * TZ;
  const int nx = G.nx, nz = G.nz;
  const bool wall = G.bc_z == BC_WALL;
  const size_t NP = G.NP, row = size_t(j) * nx;
  constexpr bool pref = Sh::PREFETCH && TMA;
  // Level whose state feeds level p (wall halos replicate the boundary cell,
  // periodic halos wrap; dynamics_rk.h:780-797).
  auto src_level = [&](int p) { return (p >= 0 && p < nz) ? p : (wall ? clampi(p, nz) : wrapi(p, nz)); };

  if constexpr (TMA) {
    if (tid == 0) {
      tma::mbar_init(bar);
      tma::mbar_init(bar + 1);
      tma::mbar_expect(bar, uint32_t(Sh::raw_bytes));
      tma::load_4d(RAW, &maps.raw, i0, j, k0 - 5, 0, bar);
      if (pref) {
        tma::mbar_expect(bar + 1, uint32_t(Sh::cell_bytes) * (sn ? 3u : 2u));
        tma::load_4d(QIN, &maps.qin, i0, j, k0, 0, bar + 1);
        tma::load_4d(TXY, &maps.txy, i0, j, k0, 0, bar + 1);
        if (sn) tma::load_4d(SN, &maps.sn, i0, j, k0, 0, bar + 1);
      }
    }
    __syncthreads();
    if (!__syncthreads_and(tma::mbar_wait(bar, 0))) {
      // The copy did not complete: report it, give the copies in flight a
      // last bounded wait, and give up the tile.
      if (tid == 0) atomicOr(G.err, ERR_TMA);
      tma::mbar_wait(bar, 0);
      if (pref) tma::mbar_wait(bar + 1, 0);
      return;
    }
  }

  // 1. Primitive fields of levels k0-5 .. k0+TZ+4.  Columns beyond the domain
  // read its last column; their results are discarded.
  for (int it = tid; it < HZ * TX; it += NT) {
    const int r = it / TX, c = it % TX;
    const int p = k0 - 5 + r, lv = src_level(p);
    const size_t col = row + min(i0 + c, nx - 1);
    R q[S], w[F];
    const int rr = lv - (k0 - 5);   // the halo box's row of level lv
    if (TMA && rr >= 0 && rr < HZ) {
#pragma unroll
      for (int s2 = 0; s2 < S; s2++) q[s2] = RAW[(s2 * HZ + rr) * TX + c];
    } else {
      load_cell<R, NTR>(G, sin, size_t(lv) * NP + col, q);
    }
    prims_of<R, NTR>(G, q, lv, w);
    if (wall && (p < 0 || p >= nz)) {
      w[iW] = R(0);
      w[iT] = R(0);
    }
#pragma unroll
    for (int f = 0; f < F; f++) H[(f * HZ + r) * TX + c] = w[f];
    if (IMM) {
      uint8_t fl = 0;
      if (p >= 0 && p < nz) {
        const uint8_t g = __ldg(G.flags + size_t(p) * NP + col);
        fl = uint8_t(((g & FLAG_IMM) ? 1 : 0) | ((g & FLAG_ANY10) ? 2 : 0));
      }
      M[r * TX + c] = fl;
    }
  }
  __syncthreads();

  // 2. z edges of the cells at positions q = 0 .. TZ+1 (level k0-1+q).  The
  // immersed bits of a stencil are the levels around its canonical cell cc
  // (wrapped in periodic z) that lie beyond the domain (the z halos of the
  // proportion are 1, dynamics_rk.h:1031-1034: bits 0..3-cc below, bits
  // nz+4-cc..8 above) or, with IMM, hold an immersed cell.
  auto mask = [&](int c, int q, unsigned &imm, bool &any10) {
    const int L = k0 - 1 + q;
    // A cell beyond the domain is read in periodic z only (in a wall domain
    // no face reads it).
    const bool inside = L >= 0 && L < nz;
    const int cc = inside ? L : wrapi(L, nz);
    imm = 0;
    any10 = false;
    if (cc < 4) imm |= (1u << (4 - cc)) - 1u;
    if (cc > nz - 5) imm |= 0x1ffu & ~((1u << (nz + 4 - cc)) - 1u);
    if (IMM) {
      if (inside) {
#pragma unroll
        for (int m = 0; m < 9; m++) imm |= (unsigned(M[(q + m) * TX + c]) & 1u) << m;
        any10 = (M[(q + 4) * TX + c] & 2u) != 0;
      } else {
        const size_t col = row + min(i0 + c, nx - 1);
#pragma unroll
        for (int m = 0; m < 9; m++) {
          const int p = cc - 4 + m;
          if (p >= 0 && p < nz) imm |= ((__ldg(G.flags + size_t(p) * NP + col) & FLAG_IMM) ? 1u : 0u) << m;
        }
        any10 = (__ldg(G.flags + size_t(cc) * NP + col) & FLAG_ANY10) != 0;
      }
    }
  };
  auto vals = [&](int f, int c, int q, R (&s)[9], unsigned imm) {
    const R *colh = H + (f * HZ + q) * TX + c;
#pragma unroll
    for (int m = 0; m < 9; m++) s[m] = colh[m * TX];
    if (f == iU || f == iV || f == iP) der0_modify(s, imm);
  };
  auto load = [&](int f, int c, int q, R (&s)[9], unsigned &imm, bool &any10) {
    mask(c, q, imm, any10);
    vals(f, c, q, s, imm);
  };
  recon_packed_inner<NT, F, TX, TZ, true>(mask, vals, [&](int f, int c, int q, R qL, R qR) {
    EL[(f * (TZ + 2) + q) * TX + c] = qL;
    ER[(f * (TZ + 2) + q) * TX + c] = qR;
  });
  for (int pr = tid; pr < F * TX; pr += NT)
    recon_outer_pair<TZ>(pr / TX, pr % TX, load, [&](int f, int c, R qR0, R qL1) {
      ER[(f * (TZ + 2)) * TX + c] = qR0;
      EL[(f * (TZ + 2) + TZ + 1) * TX + c] = qL1;
    });
  __syncthreads();

  // The cell inputs of the finalisation, copied while the block reconstructed.
  if (pref && !__syncthreads_and(tma::mbar_wait(bar + 1, 0))) {
    if (tid == 0) atomicOr(G.err, ERR_TMA);
    tma::mbar_wait(bar + 1, 0);
    return;
  }

  // 3. Each thread takes the Riemann fluxes through the two faces of its
  // cell (face k0+fz lies between the cells at positions fz and fz+1;
  // edge_exchange z, dynamics_rk.h:891-908) -- each inner face is computed
  // by the two cells beside it, with the same bits, which spares a block
  // barrier -- then the divergence, sources, stage combination and
  // enforcement of the cell.
  const int c = tid % TX, kz = tid / TX, k = k0 + kz, gi = i0 + c;
  if (gi >= nx || k >= nz) return;
  auto face_flux = [&](int fz, R (&fl)[S]) {
    const int cf = k0 + fz;
    R Lf[F], Rf[F];
    if (wall && cf == 0) {
#pragma unroll
      for (int f = 0; f < F; f++) Lf[f] = Rf[f] = EL[(f * (TZ + 2) + fz + 1) * TX + c];
      Lf[iW] = Rf[iW] = Lf[iT] = Rf[iT] = R(0);
    } else if (wall && cf == nz) {
#pragma unroll
      for (int f = 0; f < F; f++) Lf[f] = Rf[f] = ER[(f * (TZ + 2) + fz) * TX + c];
      Lf[iW] = Rf[iW] = Lf[iT] = Rf[iT] = R(0);
    } else {
#pragma unroll
      for (int f = 0; f < F; f++) {
        Lf[f] = ER[(f * (TZ + 2) + fz) * TX + c];
        Rf[f] = EL[(f * (TZ + 2) + fz + 1) * TX + c];
      }
    }
    riemann<R, NTR>(Lf, Rf, __ldg(G.rho_e + cf), __ldg(G.theta_e + cf), iW, fl);
  };
  R Fb[S], Ft[S], dF[S];
  face_flux(kz, Fb);
  face_flux(kz + 1, Ft);
  const size_t idx = size_t(k) * NP + row + gi;
  R qin[S], tx[S];
  const int cq = kz * TX + c;   // the cell in the [S][TZ][TX] buffers
#pragma unroll
  for (int s2 = 0; s2 < S; s2++) {
    qin[s2] = pref ? QIN[s2 * TZ * TX + cq] : sin[s2 * G.N + idx];
    tx[s2] = pref ? TXY[s2 * TZ * TX + cq] : txy[s2 * G.N + idx];
    dF[s2] = __fsub_rn(Ft[s2], Fb[s2]);   // not fused with the flux products: the march's bits
  }
  finish_cell<R, NTR, IMM>(
      G, qin, tx, [&](int s2) { return pref ? SN[s2 * TZ * TX + cq] : sn[s2 * G.N + idx]; }, dF, sn != nullptr,
      a_n, a_dt, n_enforce, idx, k, sout);
}

// a += b elementwise.
template <class T>
__global__ void k_add_inplace(T *__restrict__ a, const T *__restrict__ b, size_t n) {
  const size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e < n) a[e] += b[e];
}

// Enforcement pass on a state in place (the call at the top of
// time_step_rk_3_3, dynamics_rk.h:301).
// Cells [e0, e1) of the state (whole levels: e0, e1 multiples of NP).
template <class R, int NTR, bool IMM>
__global__ void k_enforce(const Grid<R> G, R *__restrict__ s, size_t e0, size_t e1) {
  const size_t idx = e0 + size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= e1) return;
  const int k = int(idx / G.NP);
  R q[5 + NTR];
#pragma unroll
  for (int v = 0; v < 5 + NTR; v++) q[v] = s[v * G.N + idx];
  enforce_cell<R, NTR, IMM>(G, q, idx, k);
#pragma unroll
  for (int v = 0; v < 5 + NTR; v++) s[v * G.N + idx] = q[v];
}

// ---------------------------------------------------------------------------
// Coupler <-> dycore conversions (FP64 arithmetic, dynamics_rk.h:1251-1352).
// ---------------------------------------------------------------------------
struct CouplerPtrs {
  const double *rho_d, *u, *v, *w, *T;
  const double *tr[8];
};
struct CouplerOut {
  double *rho_d, *u, *v, *w, *T;
  double *tr[8];
};
struct Thermo {
  double R_d, R_v, C0, gamma;
  int idWV;
  unsigned adds_mass;
};

// Cells [e0, e1) (whole levels) of the coupler arrays into the state.
template <class R, int NTR>
__global__ void k_load_coupler(CouplerPtrs cp, Thermo th, const double *__restrict__ rho_off,
                               const double *__restrict__ rt_off, size_t N, size_t NP, R *__restrict__ s, size_t e0,
                               size_t e1) {
  const size_t idx = e0 + size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= e1) return;
  const int k = int(idx / NP);
  const double rd = cp.rho_d[idx], u = cp.u[idx], v = cp.v[idx], w = cp.w[idx], temp = cp.T[idx];
  const double rho_v = cp.tr[th.idWV][idx];
  const double press = rd * th.R_d * temp + rho_v * th.R_v * temp;
  double rho = rd;
#pragma unroll
  for (int t = 0; t < NTR; t++)
    if ((th.adds_mass >> t) & 1u) rho += cp.tr[t][idx];
  const double theta = pow(press / th.C0, 1. / th.gamma) / rho;
  s[0 * N + idx] = R(rho - rho_off[k]);
  s[1 * N + idx] = R(rho * u);
  s[2 * N + idx] = R(rho * v);
  s[3 * N + idx] = R(rho * w);
  s[4 * N + idx] = R(rho * theta - rt_off[k]);
#pragma unroll
  for (int t = 0; t < NTR; t++) s[(5 + t) * N + idx] = R(cp.tr[t][idx]);
}

// Cells [e0, e1) (whole levels) of the state into the coupler arrays.
template <class R, int NTR>
__global__ void k_store_coupler(CouplerOut co, Thermo th, const double *__restrict__ rho_off,
                                const double *__restrict__ rt_off, size_t N, size_t NP, const R *__restrict__ s,
                                size_t e0, size_t e1) {
  const size_t idx = e0 + size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= e1) return;
  const int k = int(idx / NP);
  const double rho = rho_off[k] + double(s[idx]);
  const double u = double(s[1 * N + idx]) / rho, v = double(s[2 * N + idx]) / rho, w = double(s[3 * N + idx]) / rho;
  const double theta = (rt_off[k] + double(s[4 * N + idx])) / rho;
  const double press = th.C0 * pow(rho * theta, th.gamma);
  const double rho_v = double(s[(5 + th.idWV) * N + idx]);
  double rd = rho;
#pragma unroll
  for (int t = 0; t < NTR; t++)
    if ((th.adds_mass >> t) & 1u) rd -= double(s[(5 + t) * N + idx]);
  co.rho_d[idx] = rd;
  co.u[idx] = u;
  co.v[idx] = v;
  co.w[idx] = w;
  co.T[idx] = press / (rd * th.R_d + rho_v * th.R_v);
#pragma unroll
  for (int t = 0; t < NTR; t++) co.tr[t][idx] = double(s[(5 + t) * N + idx]);
}

// The perturbation fields of the dycore's output hook (dynamics_rk.h:1212-1232)
// from coupler arrays: rho, theta = rho*theta/rho and p = C0 (rho theta)^gamma
// as convert_coupler_to_dynamics forms them (dynamics_rk.h:1304-1352), minus
// the hydrostatic cell profiles (cells: [3][nz + 2*HS], density, theta,
// pressure).  out: [3][N] density_pert, theta_pert, pressure_pert (FP64).
template <int NTR>
__global__ void k_perturbations(CouplerPtrs cp, Thermo th, const double *__restrict__ cells, int nzh, size_t N,
                                size_t NP, double *__restrict__ out) {
  const size_t idx = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= N) return;
  const int kh = int(idx / NP) + HS;
  const double rd = cp.rho_d[idx], temp = cp.T[idx];
  const double rho_v = cp.tr[th.idWV][idx];
  const double press = rd * th.R_d * temp + rho_v * th.R_v * temp;
  double rho = rd;
#pragma unroll
  for (int t = 0; t < NTR; t++)
    if ((th.adds_mass >> t) & 1u) rho += cp.tr[t][idx];
  const double rt = rho * (pow(press / th.C0, 1. / th.gamma) / rho);
  out[idx] = rho - cells[kh];
  out[N + idx] = rt / rho - cells[nzh + kh];
  out[2 * N + idx] = th.C0 * pow(rt, th.gamma) - cells[2 * nzh + kh];
}

// Absolute conserved variables <-> perturbation storage.
template <class R, int NTR>
__global__ void k_get_conserved(const R *__restrict__ s, const double *__restrict__ rho_off,
                                const double *__restrict__ rt_off, size_t N, size_t NP, double *__restrict__ st,
                                double *__restrict__ tr) {
  const size_t idx = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= N) return;
  const int k = int(idx / NP);
  st[idx] = rho_off[k] + double(s[idx]);
  st[N + idx] = double(s[N + idx]);
  st[2 * N + idx] = double(s[2 * N + idx]);
  st[3 * N + idx] = double(s[3 * N + idx]);
  st[4 * N + idx] = rt_off[k] + double(s[4 * N + idx]);
#pragma unroll
  for (int t = 0; t < NTR; t++) tr[t * N + idx] = double(s[(5 + t) * N + idx]);
}

template <class R, int NTR>
__global__ void k_set_conserved(R *__restrict__ s, const double *__restrict__ rho_off, const double *__restrict__ rt_off,
                                size_t N, size_t NP, const double *__restrict__ st, const double *__restrict__ tr) {
  const size_t idx = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= N) return;
  const int k = int(idx / NP);
  s[idx] = R(st[idx] - rho_off[k]);
  s[N + idx] = R(st[N + idx]);
  s[2 * N + idx] = R(st[2 * N + idx]);
  s[3 * N + idx] = R(st[3 * N + idx]);
  s[4 * N + idx] = R(st[4 * N + idx] - rt_off[k]);
#pragma unroll
  for (int t = 0; t < NTR; t++) s[(5 + t) * N + idx] = R(tr[t * N + idx]);
}

// Re-express the perturbation state on new level offsets (after the
// hydrostatic profiles change).
template <class R>
__global__ void k_rebase(R *__restrict__ s, const double *__restrict__ old_r, const double *__restrict__ old_rt,
                         const double *__restrict__ new_r, const double *__restrict__ new_rt, size_t N, size_t NP) {
  const size_t idx = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= N) return;
  const int k = int(idx / NP);
  s[idx] = R(double(s[idx]) + old_r[k] - new_r[k]);
  s[4 * N + idx] = R(double(s[4 * N + idx]) + old_rt[k] - new_rt[k]);
}

// ---------------------------------------------------------------------------
// FP64 hydrostatic profiles (init, dynamics_rk.h:961-1008, 1145-1186).
// ---------------------------------------------------------------------------
// Neumaier-compensated running sum.
struct CSum {
  double s, c;
  __device__ void add(double x) {
    double t = s + x;
    c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
    s = t;
  }
  __device__ void merge(const CSum &o) {
    add(o.s);
    c += o.c;
  }
};

// Per level: compensated sums of rho, rho*theta/rho and C0*(rho*theta)^gamma
// over the level, from the coupler arrays (as the reference forms the state
// in convert_coupler_to_dynamics and then averages it, :967-975).
template <int NTR>
__global__ void k_column_sums(CouplerPtrs cp, Thermo th, int nx, int ny, double *__restrict__ sums) {
  const int k = blockIdx.x;
  const size_t base = size_t(k) * nx * ny;
  CSum a{0, 0}, b{0, 0}, c{0, 0};
  for (int e = threadIdx.x; e < nx * ny; e += blockDim.x) {
    const size_t idx = base + e;
    const double rd = cp.rho_d[idx], temp = cp.T[idx];
    const double rho_v = cp.tr[th.idWV][idx];
    const double press = rd * th.R_d * temp + rho_v * th.R_v * temp;
    double rho = rd;
#pragma unroll
    for (int t = 0; t < NTR; t++)
      if ((th.adds_mass >> t) & 1u) rho += cp.tr[t][idx];
    const double rt = rho * (pow(press / th.C0, 1. / th.gamma) / rho);
    a.add(rho);
    b.add(rt / rho);
    c.add(th.C0 * pow(rt, th.gamma));
  }
  __shared__ CSum sh[3][256];
  sh[0][threadIdx.x] = a;
  sh[1][threadIdx.x] = b;
  sh[2][threadIdx.x] = c;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int q = 0; q < 3; q++) sh[q][threadIdx.x].merge(sh[q][threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int q = 0; q < 3; q++) sums[q * gridDim.x + k] = sh[q][0].s + sh[q][0].c;
}

struct HydroOut {
  double *cells;   // [3][nz+2HS]  dens, theta, pressure
  double *edges;   // [3][nz+1]
  double *rho_off, *rt_off;  // [nz]
};

template <class R>
struct LevelTables {
  R *rho_h, *theta_h, *rt_inv, *p0_h, *dp_h;  // nz+2HS
  R *rho_e, *theta_e;                          // nz+1
  R *rt_target;                                // nz
};

// Means, isentropic halo extension and edge profiles in FP64.  With
// round32, every stored profile is rounded to float as the reference's
// float DataManager arrays are, and the derived tables use those values.
// If sums is null the cell profiles already in out.cells are used (restart).
// One block (HYDRO_THREADS threads): every phase is a loop over levels whose
// iterations are independent, with a barrier between phases that read what
// the previous one wrote; each value is computed as a serial loop would.
constexpr int HYDRO_THREADS = 256;

template <class R>
__global__ void __launch_bounds__(HYDRO_THREADS) k_hydro_finish(const double *__restrict__ sums, int nz, double r_nx_ny,
                                                                double gamma, double C0, double grav, double dz,
                                                                int round32, HydroOut out, LevelTables<R> tab) {
  if (blockIdx.x != 0) return;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int nzh = nz + 2 * HS;
  double *r = out.cells, *t = out.cells + nzh, *p = out.cells + 2 * nzh;
  auto rnd = [&](double x) { return round32 ? double(float(x)) : x; };
  if (!sums && round32)
    for (int k = tid; k < 3 * nzh; k += nt) out.cells[k] = rnd(out.cells[k]);
  if (sums) {
    // Level means (dynamics_rk.h:967-978).
    for (int k = tid; k < nz; k += nt) {
      r[HS + k] = rnd(sums[k] * r_nx_ny);
      t[HS + k] = rnd(sums[nz + k] * r_nx_ny);
      p[HS + k] = rnd(sums[2 * nz + k] * r_nx_ny);
    }
    __syncthreads();
    // Isentropic extension into the HS halo levels below and above
    // (dynamics_rk.h:980-1008): item q < HS below, q >= HS above.
    for (int q = tid; q < 2 * HS; q += nt) {
      const int kk = q % HS;
      const bool below = q < HS;
      const int k0 = below ? HS : HS + nz - 1, k = below ? k0 - 1 - kk : k0 + 1 + kk;
      const double rho0 = r[k0], theta0 = t[k0];
      const double rho0_gm1 = pow(rho0, gamma - 1), theta0_g = pow(theta0, gamma);
      const double dg = grav * (gamma - 1) * dz * (kk + 1) / (gamma * C0 * theta0_g);
      r[k] = rnd(pow(below ? rho0_gm1 + dg : rho0_gm1 - dg, 1. / (gamma - 1)));
      t[k] = rnd(theta0);
      p[k] = rnd(C0 * pow(r[k] * theta0, gamma));
    }
  }
  __syncthreads();
  // Edge profiles (dynamics_rk.h:1145-1186).
  double *re = out.edges, *te = out.edges + (nz + 1), *pe = out.edges + 2 * (nz + 1);
  for (int k = tid; k < nz + 1; k += nt) {
    re[k] = rnd(exp(-1. / 12. * log(r[HS + k - 2]) + 7. / 12. * log(r[HS + k - 1]) + 7. / 12. * log(r[HS + k]) +
                    -1. / 12. * log(r[HS + k + 1])));
    te[k] = rnd(-1. / 12. * t[HS + k - 2] + 7. / 12. * t[HS + k - 1] + 7. / 12. * t[HS + k] + -1. / 12. * t[HS + k + 1]);
    pe[k] = rnd(exp(-1. / 12. * log(p[HS + k - 2]) + 7. / 12. * log(p[HS + k - 1]) + 7. / 12. * log(p[HS + k]) +
                    -1. / 12. * log(p[HS + k + 1])));
    tab.rho_e[k] = R(re[k]);
    tab.theta_e[k] = R(te[k]);
  }
  for (int k = tid; k < nzh; k += nt) {
    const double rt = r[k] * t[k];
    const double P0 = C0 * pow(rt, gamma);
    tab.rho_h[k] = R(r[k]);
    tab.theta_h[k] = R(t[k]);
    tab.rt_inv[k] = R(1. / rt);
    tab.p0_h[k] = R(P0);
    tab.dp_h[k] = R(P0 - p[k]);
  }
  for (int k = tid; k < nz; k += nt) {
    const double rt = r[HS + k] * t[HS + k];
    out.rho_off[k] = r[HS + k];
    out.rt_off[k] = rt;
    // The reference's relaxation target for rho*theta is the float product
    // hy_dens_cells*hy_theta_cells (dynamics_rk.h:459).
    tab.rt_target[k] = R(round32 ? double(float(r[HS + k]) * float(t[HS + k])) - rt : 0.0);
  }
}

// ---------------------------------------------------------------------------
// Immersed-boundary preprocessing (init, :389-425 and :1010-1143).
// ---------------------------------------------------------------------------
// Chebyshev distance (capped at cap+1) to the nearest cell whose indicator is
// set, along one axis at a time; x and y wrap, z has nothing beyond the walls.
static __global__ void k_dist_init(const double *__restrict__ prop, int mode, size_t N, uint8_t *__restrict__ d, int cap) {
  const size_t idx = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= N) return;
  const bool set = mode == 0 ? prop[idx] > 0 : prop[idx] == 0;
  d[idx] = set ? 0 : uint8_t(cap + 1);
}

static __global__ void k_dist_pass(const uint8_t *__restrict__ in, uint8_t *__restrict__ out, int nx, int ny, int nz, int axis,
                            int cap) {
  const size_t N = size_t(nx) * ny * nz;
  const size_t idx = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= N) return;
  const int i = int(idx % nx), j = int((idx / nx) % ny), k = int(idx / (size_t(nx) * ny));
  int best = in[idx];
  for (int o = 1; o <= cap; o++) {
    for (int sgn = -1; sgn <= 1; sgn += 2) {
      int ii = i, jj = j, kk = k;
      if (axis == 0) ii = wrapi(i + sgn * o, nx);
      else if (axis == 1) jj = wrapi(j + sgn * o, ny);
      else {
        kk = k + sgn * o;
        if (kk < 0 || kk >= nz) continue;
      }
      const int v = in[(size_t(kk) * ny + jj) * nx + ii];
      const int cand = v > o ? v : o;
      if (cand < best) best = cand;
    }
  }
  out[idx] = uint8_t(best);
}

template <class R>
__global__ void k_imm_finish(const double *__restrict__ prop, const uint8_t *__restrict__ d_imm,
                             const uint8_t *__restrict__ d_zero, double power, size_t N, uint8_t *__restrict__ flags,
                             R *__restrict__ mult) {
  const size_t idx = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= N) return;
  const double pr = prop[idx];
  const int dz = d_zero[idx];
  const int tau = dz <= 1 ? 8 : dz == 2 ? 4 : dz == 3 ? 2 : 1;
  flags[idx] = uint8_t((pr > 0 ? FLAG_IMM : 0u) | (d_imm[idx] <= 10 ? FLAG_ANY10 : 0u));
  mult[idx] = R(pow(pr, power) / tau);
}

// ---------------------------------------------------------------------------
// FP64 compensated global integrals.
// ---------------------------------------------------------------------------
constexpr int NDIAG = 6 + 8;

template <class R, int NTR>
__global__ void k_diag_partial(const R *__restrict__ s, const double *__restrict__ rho_off,
                               const double *__restrict__ rt_off, size_t N, size_t NP, double dV, double dz,
                               double grav, double C0, double gamma, double *__restrict__ partial) {
  CSum acc[6 + NTR];
#pragma unroll
  for (int q = 0; q < 6 + NTR; q++) acc[q] = CSum{0, 0};
  for (size_t idx = size_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < N; idx += size_t(gridDim.x) * blockDim.x) {
    const int k = int(idx / NP);
    const double rho = rho_off[k] + double(s[idx]);
    const double mu = double(s[N + idx]), mv = double(s[2 * N + idx]), mw = double(s[3 * N + idx]);
    const double rt = rt_off[k] + double(s[4 * N + idx]);
    const double ke = 0.5 * (mu * mu + mv * mv + mw * mw) / rho;
    const double ie = C0 * pow(rt, gamma) / (gamma - 1);
    const double pe = rho * grav * (k + 0.5) * dz;
    acc[0].add(rho * dV);
    acc[1].add(rt * dV);
    acc[2].add(ke * dV);
    acc[3].add(ie * dV);
    acc[4].add(pe * dV);
    acc[5].add((ke + ie + pe) * dV);
#pragma unroll
    for (int t = 0; t < NTR; t++) acc[6 + t].add(double(s[(5 + t) * N + idx]) * dV);
  }
  __shared__ CSum sh[256];
  for (int q = 0; q < 6 + NTR; q++) {
    sh[threadIdx.x] = acc[q];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
      if (threadIdx.x < w) sh[threadIdx.x].merge(sh[threadIdx.x + w]);
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      partial[(size_t(blockIdx.x) * NDIAG + q) * 2 + 0] = sh[0].s;
      partial[(size_t(blockIdx.x) * NDIAG + q) * 2 + 1] = sh[0].c;
    }
    __syncthreads();
  }
}

static __global__ void k_diag_final(const double *__restrict__ partial, int nblocks, int nq, double *__restrict__ out) {
  const int q = threadIdx.x;
  if (q >= nq) return;
  CSum a{0, 0};
  for (int b = 0; b < nblocks; b++) {
    a.add(partial[(size_t(b) * NDIAG + q) * 2 + 0]);
    a.c += partial[(size_t(b) * NDIAG + q) * 2 + 1];
  }
  out[q] = a.s + a.c;
}

}  // namespace pu
