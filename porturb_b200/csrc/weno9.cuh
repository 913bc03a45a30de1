// Order-9 WENO reconstruction of the two cell-edge values of one stencil.
//
// Follows limiter::WenoLimiter<real,9>::compute_limited_edges
// (model/modules/helpers/WenoLimiter.h:349-437):
//   1. smoothness indicators TV_1..TV_5 of the five 5-cell sub-stencils
//      (TransformMatrices.h:429-433, 19841-19880), normalised to sum 1
//      (convexify, WenoLimiter.h:30-34);
//   2. imm_L: TV_5 = max(TV), imm_R: TV_1 = max(TV)  (WenoLimiter.h:430-437);
//   3. per edge: w_k = ideal_k / (TV_k^2 + 1e-20), normalise, optionally
//      apply map_rs (k=6, m=3, s=2000; WenoLimiter.h:75-82) and normalise
//      again, then the weighted sub-stencil edge values (WenoLimiter.h:382-426).
// The arithmetic is rearranged (see gen_weno9.py): stencil differences, an
// LDL^T form of TV, edge values as s_4 plus linear forms, one reciprocal
// shared by both edges for each 1/(TV_k^2+1e-20), and the normalisation
// after map_rs applied once to the weighted sum instead of to each weight.
// In FP32 the reciprocals use rcp.approx.ftz; every operand is a normal
// number there: TV_k^2+1e-20 >= 1e-20, the normalisation sums exceed 1e-20
// on the branch that divides (the weight sums always), and the map_rs
// denominator is at least ideal_k^6 > 2e-13.
#pragma once

#include "weno9_tables.cuh"

namespace pu {

template <class R>
__device__ __forceinline__ R fast_rcp(R x) { return R(1) / x; }

template <>
__device__ __forceinline__ float fast_rcp<float>(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

template <class R>
__device__ __forceinline__ void convexify5(R (&w)[5]) {
  R tot = w[0] + w[1] + w[2] + w[3] + w[4];
  if (tot > R(1.e-20)) {
    R r = fast_rcp(tot);
#pragma unroll
    for (int k = 0; k < 5; k++) w[k] *= r;
  }
}

// convexify of the ideal-weighted reciprocals, whose sum always passes the
// reference's test (> 1e-20): rk_k = 1/(TV_k^2 + 1e-20) is at least
// 1/(1 + 1e-20) when the TV were normalised (each is then at most 1 up to a
// rounding) and far above 1 when they were not (sum of TV <= 1e-20), so the
// sum is at least the sum of the ideal weights, 1.
template <class R>
__device__ __forceinline__ void normalize5(R (&w)[5]) {
  const R r = fast_rcp(w[0] + w[1] + w[2] + w[3] + w[4]);
#pragma unroll
  for (int k = 0; k < 5; k++) w[k] *= r;
}

// One edge: weights from the shared reciprocals rk = 1/(TV_k^2 + 1e-20).
// After map_rs the second convexify is folded into the edge value: the
// weighted sum of the sub-stencil edges is taken with the mapped weights
// m_k and scaled once by 1/sum(m) (the reference scales each weight).  The
// test of that convexify always passes: each m_k >= min(w_k, ideal_k) >= 0,
// and the k with w_k >= 1/5 gives m_k >= min_k ideal_k = 1/126.
template <class R, bool LEFT>
__device__ __forceinline__ R weno9_edge(const R (&d)[8], R s4, const R (&rk)[5], bool do_map) {
  using namespace pu_weno9;
  R w[5];
#pragma unroll
  for (int k = 0; k < 5; k++) w[k] = R(LEFT ? IDEAL_L[k] : IDEAL_R[k]) * rk[k];
  normalize5(w);
  R r = R(1);
  if (do_map) {
#pragma unroll
    for (int k = 0; k < 5; k++) {
      const R dk = R(LEFT ? IDEAL_L[k] : IDEAL_R[k]);
      R t = w[k] - dk;
      R t2 = t * t;
      R t6 = t2 * t2 * t2;
      R u = fma(-w[k], w[k], w[k]);   // w (1 - w)
      R u3 = u * u * u;
      R den = fma(R(2000.), u3, t6);
      w[k] = fma(t6 * t, fast_rcp(den), dk);
    }
    r = fast_rcp(w[0] + w[1] + w[2] + w[3] + w[4]);
  }
  R acc = R(0);
#pragma unroll
  for (int k = 0; k < 5; k++) {
    R lin = R(LEFT ? LIN_L[k][0] : LIN_R[k][0]) * d[k];
#pragma unroll
    for (int m = 1; m < 4; m++) lin = fma(R(LEFT ? LIN_L[k][m] : LIN_R[k][m]), d[k + m], lin);
    acc = fma(w[k], lin, acc);
  }
  return fma(acc, r, s4);
}

template <class R>
__device__ __forceinline__ void weno9_edges(const R (&s)[9], R &qL, R &qR, bool do_map, bool imm_L, bool imm_R) {
  using namespace pu_weno9;
  R d[8];
#pragma unroll
  for (int m = 0; m < 8; m++) d[m] = s[m + 1] - s[m];
  R tv[5];
#pragma unroll
  for (int k = 0; k < 5; k++) {
    R y3 = d[k + 3];
    R y2 = fma(R(TV_L[k][3][2]), d[k + 3], d[k + 2]);
    R y1 = fma(R(TV_L[k][3][1]), d[k + 3], fma(R(TV_L[k][2][1]), d[k + 2], d[k + 1]));
    R y0 = fma(R(TV_L[k][3][0]), d[k + 3], fma(R(TV_L[k][2][0]), d[k + 2], fma(R(TV_L[k][1][0]), d[k + 1], d[k])));
    R t = R(TV_D[k][3]) * y3 * y3;
    t = fma(R(TV_D[k][2]) * y2, y2, t);
    t = fma(R(TV_D[k][1]) * y1, y1, t);
    tv[k] = fma(R(TV_D[k][0]) * y0, y0, t);
  }
  convexify5(tv);
  if (imm_L || imm_R) {
    R mx = fmax(fmax(fmax(fmax(tv[0], tv[1]), tv[2]), tv[3]), tv[4]);
    if (imm_L) tv[4] = mx;
    if (imm_R) tv[0] = mx;
  }
  R rk[5];
#pragma unroll
  for (int k = 0; k < 5; k++) rk[k] = fast_rcp(fma(tv[k], tv[k], R(1.e-20)));
  qL = weno9_edge<R, true>(d, s[4], rk, do_map);
  qR = weno9_edge<R, false>(d, s[4], rk, do_map);
}

// ---------------------------------------------------------------------------
// Two stencils at once with packed FP32 arithmetic (FFMA2/FADD2/FMUL2 on
// sm_100): the same operations in the same order as weno9_edges<float>, per
// component, so each component's result is bit-identical to the scalar
// limiter's.  Halves the issue slots of the FP32 work; reciprocals stay
// scalar (rcp.approx.ftz per component).  Branches of the scalar form
// become per-component selects (a multiply by exactly 1 where the scalar
// form skips the normalisation).
// ---------------------------------------------------------------------------
struct bool2 {
  bool x, y;
};
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 rcp2(float2 a) { return make_float2(fast_rcp(a.x), fast_rcp(a.y)); }

__device__ __forceinline__ void convexify5x2(float2 (&w)[5]) {
  const float2 tot = add2(add2(add2(add2(w[0], w[1]), w[2]), w[3]), w[4]);
  const float2 r = make_float2(tot.x > 1.e-20f ? fast_rcp(tot.x) : 1.f, tot.y > 1.e-20f ? fast_rcp(tot.y) : 1.f);
#pragma unroll
  for (int k = 0; k < 5; k++) w[k] = mul2(w[k], r);
}

__device__ __forceinline__ void normalize5x2(float2 (&w)[5]) {
  const float2 tot = add2(add2(add2(add2(w[0], w[1]), w[2]), w[3]), w[4]);
  const float2 r = rcp2(tot);
#pragma unroll
  for (int k = 0; k < 5; k++) w[k] = mul2(w[k], r);
}

// Per-lane constants of one edge: SIDE 0 the left edge in both lanes, 1 the
// right edge in both, 2 the right edge in lane x and the left edge in lane y.
template <int SIDE>
__device__ __forceinline__ float2 ideal2(int k) {
  using namespace pu_weno9;
  return SIDE == 0 ? f2(float(IDEAL_L[k])) : SIDE == 1 ? f2(float(IDEAL_R[k]))
                                                       : make_float2(float(IDEAL_R[k]), float(IDEAL_L[k]));
}
template <int SIDE>
__device__ __forceinline__ float2 lin2(int k, int m) {
  using namespace pu_weno9;
  return SIDE == 0 ? f2(float(LIN_L[k][m])) : SIDE == 1 ? f2(float(LIN_R[k][m]))
                                                        : make_float2(float(LIN_R[k][m]), float(LIN_L[k][m]));
}

template <int SIDE>
__device__ __forceinline__ float2 weno9_edge2(const float2 (&d)[8], float2 s4, const float2 (&rk)[5], bool2 do_map) {
  float2 w[5];
#pragma unroll
  for (int k = 0; k < 5; k++) w[k] = mul2(ideal2<SIDE>(k), rk[k]);
  normalize5x2(w);
  float2 r = f2(1.f);
  if (do_map.x || do_map.y) {
    float2 m[5];
#pragma unroll
    for (int k = 0; k < 5; k++) {
      const float2 dk = ideal2<SIDE>(k);
      const float2 t = sub2(w[k], dk);
      const float2 t2 = mul2(t, t);
      const float2 t6 = mul2(mul2(t2, t2), t2);
      const float2 u = fma2(make_float2(-w[k].x, -w[k].y), w[k], w[k]);
      const float2 u3 = mul2(mul2(u, u), u);
      const float2 den = fma2(f2(2000.f), u3, t6);
      m[k] = fma2(mul2(t6, t), rcp2(den), dk);
    }
    const float2 tot = add2(add2(add2(add2(m[0], m[1]), m[2]), m[3]), m[4]);
    r = make_float2(do_map.x ? fast_rcp(tot.x) : 1.f, do_map.y ? fast_rcp(tot.y) : 1.f);
#pragma unroll
    for (int k = 0; k < 5; k++) w[k] = make_float2(do_map.x ? m[k].x : w[k].x, do_map.y ? m[k].y : w[k].y);
  }
  float2 acc = f2(0.f);
#pragma unroll
  for (int k = 0; k < 5; k++) {
    float2 lin = mul2(lin2<SIDE>(k, 0), d[k]);
#pragma unroll
    for (int m = 1; m < 4; m++) lin = fma2(lin2<SIDE>(k, m), d[k + m], lin);
    acc = fma2(w[k], lin, acc);
  }
  return fma2(acc, r, s4);
}

// Stencil differences and the shared reciprocals rk = 1/(TV_k^2 + 1e-20) of
// two stencils.
__device__ __forceinline__ void weno9_rk2(const float2 (&s)[9], float2 (&d)[8], float2 (&rk)[5], bool2 imm_L,
                                          bool2 imm_R) {
  using namespace pu_weno9;
#pragma unroll
  for (int m = 0; m < 8; m++) d[m] = sub2(s[m + 1], s[m]);
  float2 tv[5];
#pragma unroll
  for (int k = 0; k < 5; k++) {
    const float2 y3 = d[k + 3];
    const float2 y2 = fma2(f2(float(TV_L[k][3][2])), d[k + 3], d[k + 2]);
    const float2 y1 = fma2(f2(float(TV_L[k][3][1])), d[k + 3], fma2(f2(float(TV_L[k][2][1])), d[k + 2], d[k + 1]));
    const float2 y0 = fma2(f2(float(TV_L[k][3][0])), d[k + 3],
                           fma2(f2(float(TV_L[k][2][0])), d[k + 2], fma2(f2(float(TV_L[k][1][0])), d[k + 1], d[k])));
    float2 t = mul2(mul2(f2(float(TV_D[k][3])), y3), y3);
    t = fma2(mul2(f2(float(TV_D[k][2])), y2), y2, t);
    t = fma2(mul2(f2(float(TV_D[k][1])), y1), y1, t);
    tv[k] = fma2(mul2(f2(float(TV_D[k][0])), y0), y0, t);
  }
  convexify5x2(tv);
  if (imm_L.x || imm_L.y || imm_R.x || imm_R.y) {
    const float mx = fmaxf(fmaxf(fmaxf(fmaxf(tv[0].x, tv[1].x), tv[2].x), tv[3].x), tv[4].x);
    const float my = fmaxf(fmaxf(fmaxf(fmaxf(tv[0].y, tv[1].y), tv[2].y), tv[3].y), tv[4].y);
    if (imm_L.x) tv[4].x = mx;
    if (imm_L.y) tv[4].y = my;
    if (imm_R.x) tv[0].x = mx;
    if (imm_R.y) tv[0].y = my;
  }
#pragma unroll
  for (int k = 0; k < 5; k++) rk[k] = rcp2(fma2(tv[k], tv[k], f2(1.e-20f)));
}

__device__ __forceinline__ void weno9_edges2(const float2 (&s)[9], float2 &qL, float2 &qR, bool2 do_map, bool2 imm_L,
                                             bool2 imm_R) {
  float2 d[8], rk[5];
  weno9_rk2(s, d, rk, imm_L, imm_R);
  qL = weno9_edge2<0>(d, s[4], rk, do_map);
  qR = weno9_edge2<1>(d, s[4], rk, do_map);
}

// The right edge of stencil x and the left edge of stencil y, each
// bit-identical to that edge from weno9_edges2: the one edge a tile needs
// from each of the two halo cells that close a row of faces.
__device__ __forceinline__ float2 weno9_outer_edges2(const float2 (&s)[9], bool2 do_map, bool2 imm_L, bool2 imm_R) {
  float2 d[8], rk[5];
  weno9_rk2(s, d, rk, imm_L, imm_R);
  return weno9_edge2<2>(d, s[4], rk, do_map);
}

// Normalised nonlinear weights of the left edge (after map_rs when do_map),
// the quantity the learned network is trained to reproduce.
template <class R>
__device__ __forceinline__ void weno9_left_weights(const R (&s)[9], R (&w)[5]) {
  using namespace pu_weno9;
  R d[8];
#pragma unroll
  for (int m = 0; m < 8; m++) d[m] = s[m + 1] - s[m];
  R tv[5];
#pragma unroll
  for (int k = 0; k < 5; k++) {
    R y3 = d[k + 3];
    R y2 = fma(R(TV_L[k][3][2]), d[k + 3], d[k + 2]);
    R y1 = fma(R(TV_L[k][3][1]), d[k + 3], fma(R(TV_L[k][2][1]), d[k + 2], d[k + 1]));
    R y0 = fma(R(TV_L[k][3][0]), d[k + 3], fma(R(TV_L[k][2][0]), d[k + 2], fma(R(TV_L[k][1][0]), d[k + 1], d[k])));
    R t = R(TV_D[k][3]) * y3 * y3;
    t = fma(R(TV_D[k][2]) * y2, y2, t);
    t = fma(R(TV_D[k][1]) * y1, y1, t);
    tv[k] = fma(R(TV_D[k][0]) * y0, y0, t);
  }
  convexify5(tv);
#pragma unroll
  for (int k = 0; k < 5; k++) w[k] = R(IDEAL_L[k]) * fast_rcp(fma(tv[k], tv[k], R(1.e-20)));
  convexify5(w);
#pragma unroll
  for (int k = 0; k < 5; k++) {
    const R dk = R(IDEAL_L[k]);
    R t = w[k] - dk;
    R t2 = t * t;
    R t6 = t2 * t2 * t2;
    R u = fma(-w[k], w[k], w[k]);
    R u3 = u * u * u;
    w[k] = fma(t6 * t, fast_rcp(fma(R(2000.), u3, t6)), dk);
  }
  convexify5(w);
}

// Edge values from given left-edge and right-edge weights (the last step of
// gll_1 / gll_2, WenoLimiter.h:402-403, 425-426).
template <class R>
__device__ __forceinline__ void edges_from_weights(const R (&s)[9], const R (&wl)[5], const R (&wr)[5], R &qL, R &qR) {
  using namespace pu_weno9;
  R aL = R(0), aR = R(0);
#pragma unroll
  for (int k = 0; k < 5; k++) {
    R dk0 = s[k + 1] - s[k], dk1 = s[k + 2] - s[k + 1], dk2 = s[k + 3] - s[k + 2], dk3 = s[k + 4] - s[k + 3];
    R ll = fma(R(LIN_L[k][3]), dk3, fma(R(LIN_L[k][2]), dk2, fma(R(LIN_L[k][1]), dk1, R(LIN_L[k][0]) * dk0)));
    R lr = fma(R(LIN_R[k][3]), dk3, fma(R(LIN_R[k][2]), dk2, fma(R(LIN_R[k][1]), dk1, R(LIN_R[k][0]) * dk0)));
    aL = fma(wl[k], ll, aL);
    aR = fma(wr[k], lr, aR);
  }
  qL = s[4] + aL;
  qR = s[4] + aR;
}

// Nine-cell linear edges (weno_all == false away from immersed cells,
// dynamics_rk.h:539-545, 584-588).
template <class R>
__device__ __forceinline__ void linear9_edges(const R (&s)[9], R &qL, R &qR) {
  using namespace pu_weno9;
  R l = R(0), r = R(0);
#pragma unroll
  for (int m = 0; m < 8; m++) {
    R dm = s[m + 1] - s[m];
    l = fma(R(S2E_L[m]), dm, l);
    r = fma(R(S2E_R[m]), dm, r);
  }
  qL = s[4] + l;
  qR = s[4] + r;
}

// Zero-derivative extension past the first immersed cell, outward from the
// centre, for a stencil whose centre is not immersed (dynamics_rk.h:478-493).
// imm: bit m set when stencil entry m is immersed.
template <class R>
__device__ __forceinline__ void der0_modify(R (&s)[9], unsigned imm) {
  if (imm == 0u || (imm & 0x10u)) return;
  bool hit = false;
  R v = s[4];
#pragma unroll
  for (int i = 5; i < 9; i++) {
    if (!hit && ((imm >> i) & 1u)) { hit = true; v = s[i - 1]; }
    if (hit) s[i] = v;
  }
  hit = false;
#pragma unroll
  for (int i = 3; i >= 0; i--) {
    if (!hit && ((imm >> i) & 1u)) { hit = true; v = s[i + 1]; }
    if (hit) s[i] = v;
  }
}

}  // namespace pu
