// CPU oracle: a restatement of the reference dynamical core
// (model/modules/dynamics_rk.h, Dynamics_Euler_Stratified_WenoFV, order 9).
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product (porturb_b200/) links or
// calls this file; tests/, the smoke check and bench.py's CPU baseline use it
// as the checker.
//
// Two variants share one template:
//   REF  -- the reference's own mixed precision: FP64 state, FP32 primitive
//           fields, limiter, edge states, Riemann solver and hydrostatic
//           profiles (dynamics_rk.h:547,565,568-570,638-706,961-966).  With the
//           same compiler and -ffp-contract=off it is bit-identical to the
//           reference headers built in oracle/_ref (checked by the tests).
//   F64  -- every operation in FP64, including the smoothness indicator that
//           the reference returns as float (TransformMatrices.h:429).
//
// Halo semantics at one rank: x/y halos are periodic wraps (coupler.h:985-1165)
// taken modulo n, which equals the reference's exchange whenever the halo width
// is at most n and defines the case it leaves undefined (halo wider than n).
#include "oracle_api.h"
#include "weno9_tables.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int ORD = 9;
constexpr int HS = (ORD - 1) / 2;
constexpr int NUM_STATE = 5;
constexpr int idR = 0, idU = 1, idV = 2, idW = 3, idT = 4, idP = 5;

// ---------------------------------------------------------------------------
// Order-9 WENO limiter, WenoLimiter.h:349-437.  T is the arithmetic type; TVF
// truncates the smoothness indicator to float as TransformMatrices.h:429 does.
// ---------------------------------------------------------------------------
template <class T, bool TVF>
struct Limiter9 {
  static inline void convexify(T &w1, T &w2, T &w3, T &w4, T &w5) {  // WenoLimiter.h:30-34
    T tot = w1 + w2 + w3 + w4 + w5;
    if (tot > static_cast<T>(1.e-20)) { w1 /= tot; w2 /= tot; w3 /= tot; w4 /= tot; w5 /= tot; }
  }
  static inline void map_rs(T &w, T d) {  // WenoLimiter.h:75-82 with k=6, m=3, s=2000
    T term1 = w - d;
    for (int i = 1; i < 6; i++) term1 *= w - d;
    T term2 = w * (1 - w);
    for (int i = 1; i < 3; i++) term2 *= w * (1 - w);
    w = d + (term1 * (w - d)) / (term1 + static_cast<T>(2000.) * term2);
  }
  static inline T tv(const T *a) {  // TransformMatrices.h:429-433
    using namespace orc_tables;
    T r = T(TVW[0]) * (a[1] * a[1]) + T(TVW[1]) * (a[2] * a[2]) + T(TVW[2]) * a[1] * a[3] +
          T(TVW[3]) * (a[3] * a[3]) + T(TVW[4]) * a[2] * a[4] + T(TVW[5]) * (a[4] * a[4]);
    if (TVF) return static_cast<T>(static_cast<float>(r));
    return r;
  }
  static inline T weights_and_value(T TV_1, T TV_2, T TV_3, T TV_4, T TV_5, bool do_map, const T *s, bool left) {
    using namespace orc_tables;
    const double *id = left ? IDEAL_LEFT : IDEAL_RIGHT;
    T i_1 = static_cast<T>(id[0]), i_2 = static_cast<T>(id[1]), i_3 = static_cast<T>(id[2]),
      i_4 = static_cast<T>(id[3]), i_5 = static_cast<T>(id[4]);
    T w_1 = i_1 / (TV_1 * TV_1 + static_cast<T>(1.e-20));
    T w_2 = i_2 / (TV_2 * TV_2 + static_cast<T>(1.e-20));
    T w_3 = i_3 / (TV_3 * TV_3 + static_cast<T>(1.e-20));
    T w_4 = i_4 / (TV_4 * TV_4 + static_cast<T>(1.e-20));
    T w_5 = i_5 / (TV_5 * TV_5 + static_cast<T>(1.e-20));
    convexify(w_1, w_2, w_3, w_4, w_5);
    if (do_map) {
      map_rs(w_1, i_1); map_rs(w_2, i_2); map_rs(w_3, i_3); map_rs(w_4, i_4); map_rs(w_5, i_5);
      convexify(w_1, w_2, w_3, w_4, w_5);
    }
    if (left)
      return edge_left_win1(s) * w_1 + edge_left_win2(s) * w_2 + edge_left_win3(s) * w_3 +
             edge_left_win4(s) * w_4 + edge_left_win5(s) * w_5;
    return edge_right_win1(s) * w_1 + edge_right_win2(s) * w_2 + edge_right_win3(s) * w_3 +
           edge_right_win4(s) * w_4 + edge_right_win5(s) * w_5;
  }
  // compute_limited_edges, WenoLimiter.h:359-380.
  static inline void edges(const T *s, T &qL, T &qR, bool do_map, bool imm_L, bool imm_R) {
    using namespace orc_tables;
    T c1[5], c2[5], c3[5], c4[5], c5[5];
    coefs_win1(s[0], s[1], s[2], s[3], s[4], c1);
    coefs_win2(s[1], s[2], s[3], s[4], s[5], c2);
    coefs_win3(s[2], s[3], s[4], s[5], s[6], c3);
    coefs_win4(s[3], s[4], s[5], s[6], s[7], c4);
    coefs_win5(s[4], s[5], s[6], s[7], s[8], c5);
    T TV_1 = tv(c1), TV_2 = tv(c2), TV_3 = tv(c3), TV_4 = tv(c4), TV_5 = tv(c5);
    convexify(TV_1, TV_2, TV_3, TV_4, TV_5);
    if (imm_L) TV_5 = std::max(std::max(std::max(std::max(TV_1, TV_2), TV_3), TV_4), TV_5);  // :430-432
    if (imm_R) TV_1 = std::max(std::max(std::max(std::max(TV_1, TV_2), TV_3), TV_4), TV_5);  // :435-437
    qL = weights_and_value(TV_1, TV_2, TV_3, TV_4, TV_5, do_map, s, true);
    qR = weights_and_value(TV_1, TV_2, TV_3, TV_4, TV_5, do_map, s, false);
  }
  // Linear nine-cell edges for weno_all == false away from immersed cells
  // (dynamics_rk.h:539-545, 584-588): s2e = matmul_cr(c2e, s2c) formed in T
  // from sten_to_coefs and the edge powers of coefs_to_gll_lower, then
  // vals = matmul_cr(s2e, stencil), both as column-row products summed in
  // ascending index order.
  static inline void linear(const T *s, T &qL, T &qR) {
    using namespace orc_tables;
    T s2e[9][2];
    for (int st = 0; st < 9; st++)
      for (int pt = 0; pt < 2; pt++) {
        T tmp = 0;
        T x = pt == 0 ? T(-0.5) : T(0.5), xp = 1;
        for (int c = 0; c < 9; c++) {
          tmp += xp * T(STEN_TO_COEFS9[st][c]);
          xp *= x;
        }
        s2e[st][pt] = tmp;
      }
    T v[2];
    for (int pt = 0; pt < 2; pt++) {
      T tmp = 0;
      for (int st = 0; st < 9; st++) tmp += s2e[st][pt] * s[st];
      v[pt] = tmp;
    }
    qL = v[0];
    qR = v[1];
  }
};

// Zero-derivative extension past the first immersed cell, dynamics_rk.h:478-493.
template <class T>
inline void modify_stencil_immersed_der0(T *stencil, const bool *immersed) {
  constexpr int hs = (ORD - 1) / 2;
  if (!immersed[hs]) {
    for (int i2 = hs + 1; i2 < ORD; i2++) {
      if (immersed[i2]) { for (int i3 = i2; i3 < ORD; i3++) stencil[i3] = stencil[i2 - 1]; break; }
    }
    for (int i2 = hs - 1; i2 >= 0; i2--) {
      if (immersed[i2]) { for (int i3 = i2; i3 >= 0; i3--) stencil[i3] = stencil[i2 + 1]; break; }
    }
  }
}

inline int wrap(int i, int n) { i %= n; return i < 0 ? i + n : i; }

// ---------------------------------------------------------------------------
// The dynamical core.  SF = type of primitive fields, edge states, Riemann and
// hydrostatic profiles (float for REF, double for F64).
// ---------------------------------------------------------------------------
struct Base {
  virtual ~Base() {}
  orc_config c;
};

template <class SF, bool TVF>
struct Dycore : Base {
  using Lim = Limiter9<SF, TVF>;
  int nx, ny, nz, ntr, nxh, nyh, nzh;
  double dx, dy, dz;
  bool sim2d;
  std::vector<double> state, tracers;           // (5|ntr, nz+2hs, ny+2hs, nx+2hs)
  std::vector<SF> hy_dens_cells, hy_theta_cells, hy_pressure_cells;  // nz+2hs
  std::vector<SF> hy_dens_edges, hy_theta_edges, hy_pressure_edges;  // nz+1
  std::vector<double> imm_prop_halo;            // (nz+2hs, ny+2hs, nx+2hs)
  std::vector<uint8_t> any_immersed10;          // (nz, ny, nx)
  std::vector<int> immersed_tau;                // (nz, ny, nx)
  std::vector<bool> tracer_positive, tracer_adds_mass;

  size_t sidx(int l, int k, int j, int i) const { return ((size_t(l) * nzh + k) * nyh + j) * nxh + i; }
  size_t cidx(int k, int j, int i) const { return (size_t(k) * ny + j) * nx + i; }
  size_t hidx(int k, int j, int i) const { return (size_t(k) * nyh + j) * nxh + i; }

  explicit Dycore(const orc_config &cfg) {
    c = cfg;
    nx = c.nx; ny = c.ny; nz = c.nz; ntr = c.ntr;
    nxh = nx + 2 * HS; nyh = ny + 2 * HS; nzh = nz + 2 * HS;
    dx = c.xlen / nx; dy = c.ylen / ny; dz = c.zlen / nz;   // coupler.h:273-282 (one rank)
    sim2d = (ny == 1);
    state.assign(size_t(NUM_STATE) * nzh * nyh * nxh, 0.0);
    tracers.assign(size_t(std::max(ntr, 1)) * nzh * nyh * nxh, 0.0);
    for (int t = 0; t < ntr; t++) {
      tracer_positive.push_back(c.tracer_positive[t] != 0);
      tracer_adds_mass.push_back(c.tracer_adds_mass[t] != 0);
    }
  }

  double compute_time_step() const {  // dynamics_rk.h:57-64
    double constexpr maxwave = 350 + 100;
    return c.cfl * std::min(std::min(dx, dy), dz) / maxwave;
  }

  // convert_coupler_to_dynamics, dynamics_rk.h:1304-1352
  void load_coupler(const double *rho_d, const double *u, const double *v, const double *w, const double *T,
                    const double *trc) {
    const double R_d = c.R_d, R_v = c.R_v, gamma = c.gamma_d, C0 = c.C0;
    const int idWV = c.idWV;
#pragma omp parallel for collapse(2)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          size_t ci = cidx(k, j, i);
          double rd = rho_d[ci], uu = u[ci], vv = v[ci], ww = w[ci], temp = T[ci];
          double rho_v = trc[size_t(idWV) * nz * ny * nx + ci];
          double press = rd * R_d * temp + rho_v * R_v * temp;
          double rho = rd;
          for (int tr = 0; tr < ntr; tr++)
            if (tracer_adds_mass[tr]) rho += trc[size_t(tr) * nz * ny * nx + ci];
          double theta = std::pow(press / C0, 1. / gamma) / rho;
          state[sidx(idR, HS + k, HS + j, HS + i)] = rho;
          state[sidx(idU, HS + k, HS + j, HS + i)] = rho * uu;
          state[sidx(idV, HS + k, HS + j, HS + i)] = rho * vv;
          state[sidx(idW, HS + k, HS + j, HS + i)] = rho * ww;
          state[sidx(idT, HS + k, HS + j, HS + i)] = rho * theta;
          for (int tr = 0; tr < ntr; tr++)
            tracers[sidx(tr, HS + k, HS + j, HS + i)] = trc[size_t(tr) * nz * ny * nx + ci];
        }
  }

  // convert_dynamics_to_coupler, dynamics_rk.h:1251-1299
  void store_coupler(double *rho_d, double *u, double *v, double *w, double *T, double *trc) const {
    const double R_d = c.R_d, R_v = c.R_v, gamma = c.gamma_d, C0 = c.C0;
    const int idWV = c.idWV;
#pragma omp parallel for collapse(2)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          size_t ci = cidx(k, j, i);
          double rho = state[sidx(idR, HS + k, HS + j, HS + i)];
          double uu = state[sidx(idU, HS + k, HS + j, HS + i)] / rho;
          double vv = state[sidx(idV, HS + k, HS + j, HS + i)] / rho;
          double ww = state[sidx(idW, HS + k, HS + j, HS + i)] / rho;
          double theta = state[sidx(idT, HS + k, HS + j, HS + i)] / rho;
          double press = C0 * std::pow(rho * theta, gamma);
          double rho_v = tracers[sidx(idWV, HS + k, HS + j, HS + i)];
          double rd = rho;
          for (int tr = 0; tr < ntr; tr++)
            if (tracer_adds_mass[tr]) rd -= tracers[sidx(tr, HS + k, HS + j, HS + i)];
          double temp = press / (rd * R_d + rho_v * R_v);
          rho_d[ci] = rd; u[ci] = uu; v[ci] = vv; w[ci] = ww; T[ci] = temp;
          for (int tr = 0; tr < ntr; tr++) trc[size_t(tr) * nz * ny * nx + ci] = tracers[sidx(tr, HS + k, HS + j, HS + i)];
        }
  }

  // init, dynamics_rk.h:917-1246 (without the output/restart registrations).
  void init(const double *rho_d, const double *u, const double *v, const double *w, const double *T,
            const double *trc, const double *imm_prop) {
    std::fill(state.begin(), state.end(), 0.0);
    std::fill(tracers.begin(), tracers.end(), 0.0);
    load_coupler(rho_d, u, v, w, T, trc);
    const double gamma = c.gamma_d, C0 = c.C0, grav = c.grav;
    hy_dens_cells.assign(nzh, SF(0)); hy_theta_cells.assign(nzh, SF(0)); hy_pressure_cells.assign(nzh, SF(0));
    // Horizontal means accumulated in SF, one level per thread (:967-984).
#pragma omp parallel for
    for (int k = HS; k < HS + nz; k++) {
      SF r = 0, t = 0, p = 0;
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          r = SF(double(r) + state[sidx(idR, k, HS + j, HS + i)]);
          t = SF(double(t) + state[sidx(idT, k, HS + j, HS + i)] / state[sidx(idR, k, HS + j, HS + i)]);
          p = SF(double(p) + C0 * std::pow(state[sidx(idT, k, HS + j, HS + i)], gamma));
        }
      hy_dens_cells[k] = r; hy_theta_cells[k] = t; hy_pressure_cells[k] = p;
    }
    double r_nx_ny = 1. / (double(nx) * double(ny));
    for (int k = HS; k < HS + nz; k++) {
      hy_dens_cells[k] = SF(double(hy_dens_cells[k]) * r_nx_ny);
      hy_theta_cells[k] = SF(double(hy_theta_cells[k]) * r_nx_ny);
      hy_pressure_cells[k] = SF(double(hy_pressure_cells[k]) * r_nx_ny);
    }
    extrapolate_hydrostasis_halos();
    // Immersed proportion with halos (:1010-1143): periodic in x/y, z halos = 1.
    imm_prop_halo.assign(size_t(nzh) * nyh * nxh, 1.0);
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < nyh; j++)
        for (int i = 0; i < nxh; i++)
          imm_prop_halo[hidx(HS + k, j, i)] = imm_prop[cidx(k, wrap(j - HS, ny), wrap(i - HS, nx))];
    // any_immersed10: any prop > 0 within +-10 cells, x/y periodic, nothing beyond the z walls.
    any_immersed10.assign(size_t(nz) * ny * nx, 0);
    const int h10 = 10;
#pragma omp parallel for collapse(2)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          bool any = false;
          for (int kk = -h10; kk <= h10 && !any; kk++) {
            int kz = k + kk;
            if (kz < 0 || kz >= nz) continue;
            for (int jj = -h10; jj <= h10 && !any; jj++)
              for (int ii = -h10; ii <= h10; ii++)
                if (imm_prop[cidx(kz, wrap(j + jj, ny), wrap(i + ii, nx))] > 0) { any = true; break; }
          }
          any_immersed10[cidx(k, j, i)] = any;
        }
    // immersed_tau (:389-425).
    immersed_tau.assign(size_t(nz) * ny * nx, 1);
#pragma omp parallel for collapse(2)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          bool ni[4] = {false, false, false, false};
          for (int rad = 1; rad <= 3; rad++)
            for (int kk = -rad; kk <= rad; kk++)
              for (int jj = -rad; jj <= rad; jj++)
                for (int ii = -rad; ii <= rad; ii++)
                  if (imm_prop_halo[hidx(HS + k + kk, HS + j + jj, HS + i + ii)] == 0) ni[rad] = true;
          immersed_tau[cidx(k, j, i)] = ni[1] ? 8 : ni[2] ? 4 : ni[3] ? 2 : 1;
        }
    compute_hydrostasis_edges();
  }

  // Isentropic extension of the cell profiles into the z halos, :985-1008.
  void extrapolate_hydrostasis_halos() {
    const double gamma = c.gamma_d, C0 = c.C0, grav = c.grav;
    for (int kk = 0; kk < HS; kk++) {
      {
        int k0 = HS, k = k0 - 1 - kk;
        double rho0 = hy_dens_cells[k0], theta0 = hy_theta_cells[k0];
        double rho0_gm1 = std::pow(rho0, gamma - 1), theta0_g = std::pow(theta0, gamma);
        hy_dens_cells[k] = SF(std::pow(rho0_gm1 + grav * (gamma - 1) * dz * (kk + 1) / (gamma * C0 * theta0_g), 1. / (gamma - 1)));
        hy_theta_cells[k] = SF(theta0);
        hy_pressure_cells[k] = SF(C0 * std::pow(hy_dens_cells[k] * theta0, gamma));
      }
      {
        int k0 = HS + nz - 1, k = k0 + 1 + kk;
        double rho0 = hy_dens_cells[k0], theta0 = hy_theta_cells[k0];
        double rho0_gm1 = std::pow(rho0, gamma - 1), theta0_g = std::pow(theta0, gamma);
        hy_dens_cells[k] = SF(std::pow(rho0_gm1 - grav * (gamma - 1) * dz * (kk + 1) / (gamma * C0 * theta0_g), 1. / (gamma - 1)));
        hy_theta_cells[k] = SF(theta0);
        hy_pressure_cells[k] = SF(C0 * std::pow(hy_dens_cells[k] * theta0, gamma));
      }
    }
  }

  // compute_hydrostasis_edges for ord >= 5, :1170-1185.
  void compute_hydrostasis_edges() {
    hy_dens_edges.assign(nz + 1, SF(0)); hy_theta_edges.assign(nz + 1, SF(0)); hy_pressure_edges.assign(nz + 1, SF(0));
    for (int k = 0; k < nz + 1; k++) {
      const SF *r = hy_dens_cells.data(), *t = hy_theta_cells.data(), *p = hy_pressure_cells.data();
      hy_dens_edges[k] = SF(std::exp(-1. / 12. * std::log(r[HS + k - 2]) + 7. / 12. * std::log(r[HS + k - 1]) +
                                     7. / 12. * std::log(r[HS + k]) + -1. / 12. * std::log(r[HS + k + 1])));
      hy_theta_edges[k] = SF(-1. / 12. * t[HS + k - 2] + 7. / 12. * t[HS + k - 1] + 7. / 12. * t[HS + k] +
                             -1. / 12. * t[HS + k + 1]);
      hy_pressure_edges[k] = SF(std::exp(-1. / 12. * std::log(p[HS + k - 2]) + 7. / 12. * std::log(p[HS + k - 1]) +
                                         7. / 12. * std::log(p[HS + k]) + -1. / 12. * std::log(p[HS + k + 1])));
    }
  }

  // The restart hook re-reads the cell profiles and recomputes the edges (:1235-1242).
  void set_hydrostasis(const double *r, const double *t, const double *p) {
    for (int k = 0; k < nzh; k++) { hy_dens_cells[k] = SF(r[k]); hy_theta_cells[k] = SF(t[k]); hy_pressure_cells[k] = SF(p[k]); }
    compute_hydrostasis_edges();
  }

  // enforce_immersed_boundaries, :370-473.
  void enforce_immersed(std::vector<double> &st, std::vector<double> &tr) const {
    const double power = c.immersed_power;
#pragma omp parallel for collapse(2)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          double mult = std::pow(imm_prop_halo[hidx(HS + k, HS + j, HS + i)], power) / immersed_tau[cidx(k, j, i)];
          {
            double &var = st[sidx(idR, HS + k, HS + j, HS + i)];
            double target = hy_dens_cells[HS + k];
            var = var + (target - var) * mult;
          }
          for (int l = idU; l <= idW; l++) {
            double &var = st[sidx(l, HS + k, HS + j, HS + i)];
            double target = 0;
            var = var + (target - var) * mult;
          }
          {
            double &var = st[sidx(idT, HS + k, HS + j, HS + i)];
            double target = hy_dens_cells[HS + k] * hy_theta_cells[HS + k];
            var = var + (target - var) * mult;
          }
          for (int t = 0; t < ntr; t++) {
            double &var = tr[sidx(t, HS + k, HS + j, HS + i)];
            double target = 0;
            var = var + (target - var) * mult;
            if (tracer_positive[t]) var = std::max(0., var);
          }
        }
  }

  // compute_tendencies, :498-732.
  void compute_tendencies(const std::vector<double> &st, const std::vector<double> &tr, std::vector<double> &st_tend,
                          std::vector<double> &tr_tend) const {
    const int F = NUM_STATE + ntr + 1;
    const double C0 = c.C0, grav = c.grav, gamma = c.gamma_d;
    const bool enable_gravity = c.enable_gravity != 0, weno_all = c.weno_all != 0;
    const double r_dx = 1. / dx, r_dy = 1. / dy, r_dz = 1. / dz;
    const double fcor = 2 * 7.2921e-5 * std::sin(c.latitude / 180 * M_PI);
    const size_t NH = size_t(nzh) * nyh * nxh;
    std::vector<SF> fl(size_t(F) * NH, SF(0));
    auto FL = [&](int l, int k, int j, int i) -> SF & { return fl[size_t(l) * NH + hidx(k, j, i)]; };
    // Primitive perturbation fields (:550-558).
#pragma omp parallel for collapse(2)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          FL(idP, HS + k, HS + j, HS + i) = SF(C0 * std::pow(st[sidx(idT, HS + k, HS + j, HS + i)], gamma) - hy_pressure_cells[HS + k]);
          double r_r = 1. / st[sidx(idR, HS + k, HS + j, HS + i)];
          FL(idR, HS + k, HS + j, HS + i) = SF(st[sidx(idR, HS + k, HS + j, HS + i)]);
          for (int l = 1; l < NUM_STATE; l++) FL(l, HS + k, HS + j, HS + i) = SF(st[sidx(l, HS + k, HS + j, HS + i)] * r_r);
          for (int l = 0; l < ntr; l++) FL(NUM_STATE + 1 + l, HS + k, HS + j, HS + i) = SF(tr[sidx(l, HS + k, HS + j, HS + i)] * r_r);
          FL(idR, HS + k, HS + j, HS + i) -= hy_dens_cells[HS + k];
          FL(idT, HS + k, HS + j, HS + i) -= hy_theta_cells[HS + k];
        }
    // Periodic x then y halos (coupler.h:985-1021, 1128-1165), then precursor and z BCs (:736-804).
#pragma omp parallel for collapse(2)
    for (int l = 0; l < F; l++)
      for (int k = 0; k < nz; k++) {
        for (int j = 0; j < ny; j++)
          for (int ii = 0; ii < HS; ii++) {
            FL(l, HS + k, HS + j, ii) = FL(l, HS + k, HS + j, HS + wrap(ii - HS, nx));
            FL(l, HS + k, HS + j, HS + nx + ii) = FL(l, HS + k, HS + j, HS + wrap(ii, nx));
          }
        for (int jj = 0; jj < HS; jj++)
          for (int i = 0; i < nx; i++) {
            FL(l, HS + k, jj, HS + i) = FL(l, HS + k, HS + wrap(jj - HS, ny), HS + i);
            FL(l, HS + k, HS + ny + jj, HS + i) = FL(l, HS + k, HS + wrap(jj, ny), HS + i);
          }
        if (c.bc_x == ORC_BC_PRECURSOR)
          for (int j = 0; j < ny; j++)
            for (int ii = 0; ii < HS; ii++) {
              FL(l, HS + k, HS + j, ii) = FL(l, HS + k, HS + j, HS + 0);
              FL(l, HS + k, HS + j, HS + nx + ii) = FL(l, HS + k, HS + j, HS + nx - 1);
            }
        if (c.bc_y == ORC_BC_PRECURSOR)
          for (int jj = 0; jj < HS; jj++)
            for (int i = 0; i < nx; i++) {
              FL(l, HS + k, jj, HS + i) = FL(l, HS + k, HS + 0, HS + i);
              FL(l, HS + k, HS + ny + jj, HS + i) = FL(l, HS + k, HS + ny - 1, HS + i);
            }
      }
#pragma omp parallel for collapse(2)
    for (int l = 0; l < F; l++)
      for (int kk = 0; kk < HS; kk++)
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < nx; i++) {
            if (c.bc_z == ORC_BC_WALL) {
              if (l == idW || l == idT) {
                FL(l, kk, HS + j, HS + i) = 0;
                FL(l, HS + nz + kk, HS + j, HS + i) = 0;
              } else {
                FL(l, kk, HS + j, HS + i) = FL(l, HS + 0, HS + j, HS + i);
                FL(l, HS + nz + kk, HS + j, HS + i) = FL(l, HS + nz - 1, HS + j, HS + i);
              }
            } else {  // periodic
              FL(l, kk, HS + j, HS + i) = FL(l, nz + kk, HS + j, HS + i);
              FL(l, HS + nz + kk, HS + j, HS + i) = FL(l, HS + kk, HS + j, HS + i);
            }
          }
    // Edge states: lim_d[(side*F + l)*faces + face]
    const size_t NXF = size_t(nz) * ny * (nx + 1), NYF = size_t(nz) * (ny + 1) * nx, NZF = size_t(nz + 1) * ny * nx;
    std::vector<SF> lx(2 * F * NXF, SF(0)), ly(2 * F * NYF, SF(0)), lz(2 * F * NZF, SF(0));
    auto LX = [&](int s, int l, int k, int j, int i) -> SF & { return lx[(size_t(s) * F + l) * NXF + (size_t(k) * ny + j) * (nx + 1) + i]; };
    auto LY = [&](int s, int l, int k, int j, int i) -> SF & { return ly[(size_t(s) * F + l) * NYF + (size_t(k) * (ny + 1) + j) * nx + i]; };
    auto LZ = [&](int s, int l, int k, int j, int i) -> SF & { return lz[(size_t(s) * F + l) * NZF + (size_t(k) * ny + j) * nx + i]; };
    auto imm = [&](int k, int j, int i) { return imm_prop_halo[hidx(k, j, i)] > 0; };
    // WENO in x, y and z (:572-625).
#pragma omp parallel for collapse(2)
    for (int l = 0; l < F; l++)
      for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < nx; i++) {
            bool anyi = any_immersed10[cidx(k, j, i)] != 0;
            SF s[ORD];
            bool im[ORD];
            // x
            for (int ii = 0; ii < ORD; ii++) { im[ii] = imm(HS + k, HS + j, i + ii); s[ii] = FL(l, HS + k, HS + j, i + ii); }
            if (l == idV || l == idW || l == idP) modify_stencil_immersed_der0(s, im);
            if (anyi || weno_all) Lim::edges(s, LX(1, l, k, j, i), LX(0, l, k, j, i + 1), !anyi, im[HS - 1], im[HS + 1]);
            else Lim::linear(s, LX(1, l, k, j, i), LX(0, l, k, j, i + 1));
            // y
            for (int jj = 0; jj < ORD; jj++) { im[jj] = imm(HS + k, j + jj, HS + i); s[jj] = FL(l, HS + k, j + jj, HS + i); }
            if (l == idU || l == idW || l == idP) modify_stencil_immersed_der0(s, im);
            if (anyi || weno_all) Lim::edges(s, LY(1, l, k, j, i), LY(0, l, k, j + 1, i), !anyi, im[HS - 1], im[HS + 1]);
            else Lim::linear(s, LY(1, l, k, j, i), LY(0, l, k, j + 1, i));
            // z
            for (int kk = 0; kk < ORD; kk++) { im[kk] = imm(k + kk, HS + j, HS + i); s[kk] = FL(l, k + kk, HS + j, HS + i); }
            if (l == idU || l == idV || l == idP) modify_stencil_immersed_der0(s, im);
            if (anyi || weno_all) Lim::edges(s, LZ(1, l, k, j, i), LZ(0, l, k + 1, j, i), !anyi, im[HS - 1], im[HS + 1]);
            else Lim::linear(s, LZ(1, l, k, j, i), LZ(0, l, k + 1, j, i));
          }
    // Edge exchange (:808-912).
#pragma omp parallel for
    for (int l = 0; l < F; l++) {
      for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++) {
          LX(0, l, k, j, 0) = LX(0, l, k, j, nx);
          LX(1, l, k, j, nx) = LX(1, l, k, j, 0);
        }
      for (int k = 0; k < nz; k++)
        for (int i = 0; i < nx; i++) {
          LY(0, l, k, 0, i) = LY(0, l, k, ny, i);
          LY(1, l, k, ny, i) = LY(1, l, k, 0, i);
        }
      if (c.bc_x == ORC_BC_PRECURSOR)
        for (int k = 0; k < nz; k++)
          for (int j = 0; j < ny; j++) { LX(0, l, k, j, 0) = LX(1, l, k, j, 0); LX(1, l, k, j, nx) = LX(0, l, k, j, nx); }
      if (c.bc_y == ORC_BC_PRECURSOR)
        for (int k = 0; k < nz; k++)
          for (int i = 0; i < nx; i++) { LY(0, l, k, 0, i) = LY(1, l, k, 0, i); LY(1, l, k, ny, i) = LY(0, l, k, ny, i); }
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          if (c.bc_z == ORC_BC_WALL) {
            if (l == idW || l == idT) {
              LZ(0, l, 0, j, i) = 0; LZ(1, l, 0, j, i) = 0; LZ(0, l, nz, j, i) = 0; LZ(1, l, nz, j, i) = 0;
            } else {
              LZ(0, l, 0, j, i) = LZ(1, l, 0, j, i);
              LZ(1, l, nz, j, i) = LZ(0, l, nz, j, i);
            }
          } else {
            LZ(0, l, 0, j, i) = LZ(0, l, nz, j, i);
            LZ(1, l, nz, j, i) = LZ(1, l, 0, j, i);
          }
        }
    }
    // Upwind Riemann solver (:638-707).  Fluxes: fx[l*NXF + face].
    const int S = NUM_STATE + ntr;
    std::vector<SF> fx(size_t(S) * NXF), fy(size_t(S) * NYF), fz(size_t(S) * NZF);
    const SF cs = SF(350.);
    auto riemann = [&](auto &L, int k, int j, int i, SF hr, SF ht, int idN, SF *flux) {
      L(0, idR, k, j, i) += hr; L(1, idR, k, j, i) += hr;
      L(0, idT, k, j, i) += ht; L(1, idT, k, j, i) += ht;
      SF r_L = L(0, idR, k, j, i), r_R = L(1, idR, k, j, i);
      SF ru_L = L(0, idN, k, j, i) * r_L, ru_R = L(1, idN, k, j, i) * r_R;
      SF p_L = L(0, idP, k, j, i), p_R = L(1, idP, k, j, i);
      SF p_upw = SF(0.5 * (p_L + p_R - cs * (ru_R - ru_L)));
      SF ru_upw = SF(0.5 * (ru_L + ru_R - (p_R - p_L) / cs));
      int ind = ru_upw > 0 ? 0 : 1;
      flux[idR] = ru_upw;
      for (int l = idU; l <= idT; l++) flux[l] = ru_upw * L(ind, l, k, j, i);
      flux[idN] = ru_upw * L(ind, idN, k, j, i) + p_upw;
      for (int t = 0; t < ntr; t++) flux[NUM_STATE + t] = ru_upw * L(ind, NUM_STATE + 1 + t, k, j, i);
    };
#pragma omp parallel for collapse(2)
    for (int k = 0; k < nz + 1; k++)
      for (int j = 0; j < ny + 1; j++)
        for (int i = 0; i < nx + 1; i++) {
          SF flux[NUM_STATE + ORC_MAX_TRACERS];
          if (j < ny && k < nz) {
            riemann(LX, k, j, i, hy_dens_cells[HS + k], hy_theta_cells[HS + k], idU, flux);
            for (int l = 0; l < S; l++) fx[size_t(l) * NXF + (size_t(k) * ny + j) * (nx + 1) + i] = flux[l];
          }
          if (i < nx && k < nz && !sim2d) {
            riemann(LY, k, j, i, hy_dens_cells[HS + k], hy_theta_cells[HS + k], idV, flux);
            for (int l = 0; l < S; l++) fy[size_t(l) * NYF + (size_t(k) * (ny + 1) + j) * nx + i] = flux[l];
          }
          if (i < nx && j < ny) {
            riemann(LZ, k, j, i, hy_dens_edges[k], hy_theta_edges[k], idW, flux);
            for (int l = 0; l < S; l++) fz[size_t(l) * NZF + (size_t(k) * ny + j) * nx + i] = flux[l];
          }
        }
    // Flux divergence and sources (:710-728).
    auto FX = [&](int l, int k, int j, int i) { return fx[size_t(l) * NXF + (size_t(k) * ny + j) * (nx + 1) + i]; };
    auto FY = [&](int l, int k, int j, int i) { return fy[size_t(l) * NYF + (size_t(k) * (ny + 1) + j) * nx + i]; };
    auto FZ = [&](int l, int k, int j, int i) { return fz[size_t(l) * NZF + (size_t(k) * ny + j) * nx + i]; };
    const size_t NC = size_t(nz) * ny * nx;
#pragma omp parallel for collapse(2)
    for (int l = 0; l < S; l++)
      for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < nx; i++) {
            // In 2-D the reference's y term is an exact zero (both y faces hold the
            // same exchanged value), so leaving it out gives the same bits.
            double tend = -(FX(l, k, j, i + 1) - FX(l, k, j, i)) * r_dx;
            if (!sim2d) tend = tend - (FY(l, k, j + 1, i) - FY(l, k, j, i)) * r_dy;
            tend = tend - (FZ(l, k + 1, j, i) - FZ(l, k, j, i)) * r_dz;
            if (l < NUM_STATE) {
              if (l == idV && sim2d) tend = 0;
              if (l == idW && enable_gravity) tend += -grav * (st[sidx(idR, HS + k, HS + j, HS + i)] - hy_dens_cells[HS + k]);
              if (c.latitude != 0 && !sim2d && l == idU) tend += fcor * st[sidx(idV, HS + k, HS + j, HS + i)];
              if (c.latitude != 0 && !sim2d && l == idV) tend -= fcor * st[sidx(idU, HS + k, HS + j, HS + i)];
              st_tend[size_t(l) * NC + cidx(k, j, i)] = tend;
            } else {
              tr_tend[size_t(l - NUM_STATE) * NC + cidx(k, j, i)] = tend;
            }
          }
  }

  // time_step_rk_3_3, :279-367.
  void rk33(double dt_dyn) {
    const size_t NC = size_t(nz) * ny * nx;
    std::vector<double> state_tmp(state.size(), 0.0), tracers_tmp(tracers.size(), 0.0);
    std::vector<double> st_tend(NUM_STATE * NC), tr_tend(std::max(ntr, 1) * NC);
    enforce_immersed(state, tracers);
    for (int stage = 0; stage < 3; stage++) {
      const std::vector<double> &sin = stage == 0 ? state : state_tmp;
      const std::vector<double> &tin = stage == 0 ? tracers : tracers_tmp;
      compute_tendencies(sin, tin, st_tend, tr_tend);
      const int S = NUM_STATE + ntr;
#pragma omp parallel for collapse(2)
      for (int l = 0; l < S; l++)
        for (int k = 0; k < nz; k++)
          for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
              bool is_st = l < NUM_STATE;
              int ll = is_st ? l : l - NUM_STATE;
              double &s0 = is_st ? state[sidx(ll, HS + k, HS + j, HS + i)] : tracers[sidx(ll, HS + k, HS + j, HS + i)];
              double &s1 = is_st ? state_tmp[sidx(ll, HS + k, HS + j, HS + i)] : tracers_tmp[sidx(ll, HS + k, HS + j, HS + i)];
              double tend = is_st ? st_tend[size_t(ll) * NC + cidx(k, j, i)] : tr_tend[size_t(ll) * NC + cidx(k, j, i)];
              if (stage == 0) {
                s1 = s0 + dt_dyn * tend;
              } else if (stage == 1) {
                s1 = (3. / 4.) * s0 + (1. / 4.) * s1 + (1. / 4.) * dt_dyn * tend;
              } else {
                s0 = (1. / 3.) * s0 + (2. / 3.) * s1 + (2. / 3.) * dt_dyn * tend;
                if (!is_st && tracer_positive[ll]) s0 = std::max(0., s0);
              }
            }
      if (stage < 2) enforce_immersed(state_tmp, tracers_tmp);
      else enforce_immersed(state, tracers);
    }
  }

  // time_step, :103-137.
  int time_step(double *rho_d, double *u, double *v, double *w, double *T, double *trc, double dt_phys) {
    load_coupler(rho_d, u, v, w, T, trc);
    double dt_dyn = compute_time_step();
    int ncycles = (int)std::ceil(dt_phys / dt_dyn);
    dt_dyn = dt_phys / ncycles;
    for (int icycle = 0; icycle < ncycles; icycle++) rk33(dt_dyn);
    store_coupler(rho_d, u, v, w, T, trc);
    return ncycles;
  }

  void get_state(double *st, double *trc) const {
    const size_t NC = size_t(nz) * ny * nx;
    for (int l = 0; l < NUM_STATE; l++)
      for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < nx; i++) st[l * NC + cidx(k, j, i)] = state[sidx(l, HS + k, HS + j, HS + i)];
    for (int l = 0; l < ntr; l++)
      for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < nx; i++) trc[l * NC + cidx(k, j, i)] = tracers[sidx(l, HS + k, HS + j, HS + i)];
  }
  void set_state(const double *st, const double *trc) {
    const size_t NC = size_t(nz) * ny * nx;
    for (int l = 0; l < NUM_STATE; l++)
      for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < nx; i++) state[sidx(l, HS + k, HS + j, HS + i)] = st[l * NC + cidx(k, j, i)];
    for (int l = 0; l < ntr; l++)
      for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < nx; i++) tracers[sidx(l, HS + k, HS + j, HS + i)] = trc[l * NC + cidx(k, j, i)];
  }
};

struct Handle {
  int variant;
  Dycore<float, true> *ref = nullptr;
  Dycore<double, false> *f64 = nullptr;
};

template <class Fn>
auto dispatch(void *h, Fn fn) {
  Handle *H = static_cast<Handle *>(h);
  if (H->variant == ORC_VARIANT_REF) return fn(*H->ref);
  return fn(*H->f64);
}

}  // namespace

extern "C" {

void *orc_create(const orc_config *cfg, int variant) {
  if (cfg->ntr < 1 || cfg->ntr > ORC_MAX_TRACERS || cfg->idWV < 0 || cfg->idWV >= cfg->ntr) return nullptr;
  Handle *h = new Handle;
  h->variant = variant;
  if (variant == ORC_VARIANT_REF) h->ref = new Dycore<float, true>(*cfg);
  else h->f64 = new Dycore<double, false>(*cfg);
  return h;
}

void orc_destroy(void *h) {
  Handle *H = static_cast<Handle *>(h);
  delete H->ref;
  delete H->f64;
  delete H;
}

int orc_init(void *h, const double *rho_d, const double *u, const double *v, const double *w, const double *T,
             const double *trc, const double *imm_prop) {
  dispatch(h, [&](auto &d) { d.init(rho_d, u, v, w, T, trc, imm_prop); return 0; });
  return 0;
}

int orc_set_hydrostasis(void *h, const double *r, const double *t, const double *p) {
  dispatch(h, [&](auto &d) { d.set_hydrostasis(r, t, p); return 0; });
  return 0;
}

void orc_get_hydrostasis(void *h, double *rc, double *tc, double *pc, double *re, double *te, double *pe) {
  dispatch(h, [&](auto &d) {
    for (int k = 0; k < d.nzh; k++) { rc[k] = d.hy_dens_cells[k]; tc[k] = d.hy_theta_cells[k]; pc[k] = d.hy_pressure_cells[k]; }
    for (int k = 0; k < d.nz + 1; k++) { re[k] = d.hy_dens_edges[k]; te[k] = d.hy_theta_edges[k]; pe[k] = d.hy_pressure_edges[k]; }
    return 0;
  });
}

double orc_compute_time_step(void *h) {
  return dispatch(h, [&](auto &d) { return d.compute_time_step(); });
}

int orc_time_step(void *h, double *rho_d, double *u, double *v, double *w, double *T, double *trc, double dt_phys) {
  return dispatch(h, [&](auto &d) { return d.time_step(rho_d, u, v, w, T, trc, dt_phys); });
}

void orc_load_coupler(void *h, const double *rho_d, const double *u, const double *v, const double *w, const double *T,
                      const double *trc) {
  dispatch(h, [&](auto &d) { d.load_coupler(rho_d, u, v, w, T, trc); return 0; });
}

void orc_store_coupler(void *h, double *rho_d, double *u, double *v, double *w, double *T, double *trc) {
  dispatch(h, [&](auto &d) { d.store_coupler(rho_d, u, v, w, T, trc); return 0; });
}

void orc_advance(void *h, double dt_dyn, int nsteps) {
  dispatch(h, [&](auto &d) { for (int n = 0; n < nsteps; n++) d.rk33(dt_dyn); return 0; });
}

void orc_get_state(void *h, double *st, double *trc) {
  dispatch(h, [&](auto &d) { d.get_state(st, trc); return 0; });
}

void orc_set_state(void *h, const double *st, const double *trc) {
  dispatch(h, [&](auto &d) { d.set_state(st, trc); return 0; });
}

void orc_tendencies(void *h, double *st_tend, double *tr_tend) {
  dispatch(h, [&](auto &d) {
    std::vector<double> a(size_t(NUM_STATE) * d.nz * d.ny * d.nx), b(size_t(std::max(d.ntr, 1)) * d.nz * d.ny * d.nx);
    d.compute_tendencies(d.state, d.tracers, a, b);
    std::memcpy(st_tend, a.data(), a.size() * sizeof(double));
    std::memcpy(tr_tend, b.data(), size_t(d.ntr) * d.nz * d.ny * d.nx * sizeof(double));
    return 0;
  });
}

void orc_weno9_f32(const float *s, int do_map, int imm_L, int imm_R, float *qL, float *qR) {
  Limiter9<float, true>::edges(s, *qL, *qR, do_map != 0, imm_L != 0, imm_R != 0);
}

void orc_weno9_f64(const double *s, int do_map, int imm_L, int imm_R, double *qL, double *qR) {
  Limiter9<double, false>::edges(s, *qL, *qR, do_map != 0, imm_L != 0, imm_R != 0);
}

void orc_weno9_f64tvf(const double *s, int do_map, int imm_L, int imm_R, double *qL, double *qR) {
  Limiter9<double, true>::edges(s, *qL, *qR, do_map != 0, imm_L != 0, imm_R != 0);
}

void orc_weno9_batch_f32(const float *s, long n, int do_map, float *qL, float *qR) {
#pragma omp parallel for
  for (long m = 0; m < n; m++) Limiter9<float, true>::edges(s + 9 * m, qL[m], qR[m], do_map != 0, false, false);
}

int orc_num_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
