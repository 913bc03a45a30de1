// C entry points around the reference's own dycore (TEST INFRASTRUCTURE ONLY).
//
// Compiles model/modules/dynamics_rk.h of the reference unchanged (with
// PORTURB_ORD=9) against the single-rank shim in oracle/ref_shim, and exposes
// it through the ref_* functions of oracle/oracle_api.h.  The reference's own
// module API is what runs: Dynamics_Euler_Stratified_WenoFV::init,
// time_step, time_step_rk_3_3, compute_tendencies, convert_*; the coupler and
// the array library are the shim's.
#include "coupler.h"
#include "dynamics_rk.h"
#include "oracle_api.h"

#include <cstdio>

namespace {

struct RefHandle {
  core::Coupler coupler;
  modules::Dynamics_Euler_Stratified_WenoFV dycore;
  orc_config cfg;
  real4d state, tracers;
  std::string last_error;
  RefHandle(const orc_config &c) : coupler(c.nx, c.ny, c.nz, c.xlen, c.ylen, c.zlen), cfg(c) {}
};

std::string g_error;
constexpr int HS = modules::Dynamics_Euler_Stratified_WenoFV::hs;

const char *bc_name(int bc) { return bc == ORC_BC_PRECURSOR ? "precursor" : bc == ORC_BC_WALL ? "solid_wall" : "periodic"; }

void copy_in(RefHandle &h, const double *rho_d, const double *u, const double *v, const double *w, const double *T,
             const double *trc) {
  auto &dm = h.coupler.get_data_manager_readwrite();
  size_t n = size_t(h.cfg.nx) * h.cfg.ny * h.cfg.nz;
  std::memcpy(dm.get<real, 3>("density_dry").data(), rho_d, n * sizeof(double));
  std::memcpy(dm.get<real, 3>("uvel").data(), u, n * sizeof(double));
  std::memcpy(dm.get<real, 3>("vvel").data(), v, n * sizeof(double));
  std::memcpy(dm.get<real, 3>("wvel").data(), w, n * sizeof(double));
  std::memcpy(dm.get<real, 3>("temp").data(), T, n * sizeof(double));
  auto names = h.coupler.get_tracer_names();
  for (size_t t = 0; t < names.size(); t++) std::memcpy(dm.get<real, 3>(names[t]).data(), trc + t * n, n * sizeof(double));
}

void copy_out(RefHandle &h, double *rho_d, double *u, double *v, double *w, double *T, double *trc) {
  auto &dm = h.coupler.get_data_manager_readonly();
  size_t n = size_t(h.cfg.nx) * h.cfg.ny * h.cfg.nz;
  std::memcpy(rho_d, dm.get<real const, 3>("density_dry").data(), n * sizeof(double));
  std::memcpy(u, dm.get<real const, 3>("uvel").data(), n * sizeof(double));
  std::memcpy(v, dm.get<real const, 3>("vvel").data(), n * sizeof(double));
  std::memcpy(w, dm.get<real const, 3>("wvel").data(), n * sizeof(double));
  std::memcpy(T, dm.get<real const, 3>("temp").data(), n * sizeof(double));
  auto names = h.coupler.get_tracer_names();
  for (size_t t = 0; t < names.size(); t++) std::memcpy(trc + t * n, dm.get<real const, 3>(names[t]).data(), n * sizeof(double));
}

template <class F>
int guarded(F f) {
  try {
    return f();
  } catch (std::exception &e) {
    g_error = e.what();
    return -1;
  }
}

}  // namespace

extern "C" {

const char *ref_last_error() { return g_error.c_str(); }

void *ref_create(const orc_config *cfg) {
  RefHandle *h = nullptr;
  int rc = guarded([&]() {
    h = new RefHandle(*cfg);
    auto &c = h->coupler;
    c.set_option<real>("R_d", cfg->R_d);
    c.set_option<real>("R_v", cfg->R_v);
    c.set_option<real>("cp_d", cfg->cp_d);
    c.set_option<real>("gamma_d", cfg->gamma_d);
    c.set_option<real>("C0", cfg->C0);
    c.set_option<real>("grav", cfg->grav);
    c.set_option<int>("idWV", cfg->idWV);
    c.set_option<real>("cfl", cfg->cfl);
    c.set_option<real>("immersed_power", cfg->immersed_power);
    c.set_option<real>("latitude", cfg->latitude);
    c.set_option<std::string>("bc_x", bc_name(cfg->bc_x));
    c.set_option<std::string>("bc_y", bc_name(cfg->bc_y));
    c.set_option<std::string>("bc_z", bc_name(cfg->bc_z));
    c.set_option<bool>("enable_gravity", cfg->enable_gravity != 0);
    c.set_option<bool>("weno_all", cfg->weno_all != 0);
    auto &dm = c.get_data_manager_readwrite();
    for (auto nm : {"density_dry", "uvel", "vvel", "wvel", "temp", "immersed_proportion"})
      dm.register_and_allocate<real>(nm, "", {cfg->nz, cfg->ny, cfg->nx});
    for (int t = 0; t < cfg->ntr; t++) {
      char name[32];
      if (t == cfg->idWV) std::snprintf(name, sizeof(name), "water_vapor");
      else std::snprintf(name, sizeof(name), "tracer_%d", t);
      c.add_tracer(name, name, cfg->tracer_positive[t] != 0, cfg->tracer_adds_mass[t] != 0, true);
    }
    h->state = real4d("state", 5, cfg->nz + 2 * HS, cfg->ny + 2 * HS, cfg->nx + 2 * HS);
    h->tracers = real4d("tracers", cfg->ntr, cfg->nz + 2 * HS, cfg->ny + 2 * HS, cfg->nx + 2 * HS);
    return 0;
  });
  if (rc != 0) { delete h; return nullptr; }
  return h;
}

void ref_destroy(void *p) { delete static_cast<RefHandle *>(p); }

int ref_init(void *p, const double *rho_d, const double *u, const double *v, const double *w, const double *T,
             const double *trc, const double *imm_prop) {
  RefHandle &h = *static_cast<RefHandle *>(p);
  return guarded([&]() {
    copy_in(h, rho_d, u, v, w, T, trc);
    size_t n = size_t(h.cfg.nx) * h.cfg.ny * h.cfg.nz;
    std::memcpy(h.coupler.get_data_manager_readwrite().get<real, 3>("immersed_proportion").data(), imm_prop, n * sizeof(double));
    h.dycore.init(h.coupler);
    return 0;
  });
}

// Overwrite the cell profiles and rerun the dycore's restart hook
// (dynamics_rk.h:1235-1242), which recomputes the edge profiles.
int ref_set_hydrostasis(void *p, const double *r, const double *t, const double *pr) {
  RefHandle &h = *static_cast<RefHandle *>(p);
  return guarded([&]() {
    auto &dm = h.coupler.get_data_manager_readwrite();
    auto dr = dm.get<float, 1>("hy_dens_cells"), dt = dm.get<float, 1>("hy_theta_cells"), dp = dm.get<float, 1>("hy_pressure_cells");
    for (size_t k = 0; k < dr.size(); k++) { dr(k) = float(r[k]); dt(k) = float(t[k]); dp(k) = float(pr[k]); }
    yakl::SimplePNetCDF nc;
    h.coupler.run_restart_hooks(nc);
    return 0;
  });
}

void ref_get_hydrostasis(void *p, double *rc, double *tc, double *pc, double *re, double *te, double *pe) {
  RefHandle &h = *static_cast<RefHandle *>(p);
  auto &dm = h.coupler.get_data_manager_readonly();
  auto a = dm.get<float const, 1>("hy_dens_cells"), b = dm.get<float const, 1>("hy_theta_cells"), c = dm.get<float const, 1>("hy_pressure_cells");
  for (size_t k = 0; k < a.size(); k++) { rc[k] = a(k); tc[k] = b(k); pc[k] = c(k); }
  auto d = dm.get<float const, 1>("hy_dens_edges"), e = dm.get<float const, 1>("hy_theta_edges"), f = dm.get<float const, 1>("hy_pressure_edges");
  for (size_t k = 0; k < d.size(); k++) { re[k] = d(k); te[k] = e(k); pe[k] = f(k); }
}

double ref_compute_time_step(void *p) {
  RefHandle &h = *static_cast<RefHandle *>(p);
  return h.dycore.compute_time_step(h.coupler);
}

int ref_time_step(void *p, double *rho_d, double *u, double *v, double *w, double *T, double *trc, double dt_phys) {
  RefHandle &h = *static_cast<RefHandle *>(p);
  return guarded([&]() {
    copy_in(h, rho_d, u, v, w, T, trc);
    h.dycore.time_step(h.coupler, dt_phys);
    copy_out(h, rho_d, u, v, w, T, trc);
    return (int)std::ceil(dt_phys / h.dycore.compute_time_step(h.coupler));
  });
}

int ref_load_coupler(void *p, const double *rho_d, const double *u, const double *v, const double *w, const double *T,
                     const double *trc) {
  RefHandle &h = *static_cast<RefHandle *>(p);
  return guarded([&]() {
    copy_in(h, rho_d, u, v, w, T, trc);
    h.dycore.convert_coupler_to_dynamics(h.coupler, h.state, h.tracers);
    return 0;
  });
}

int ref_store_coupler(void *p, double *rho_d, double *u, double *v, double *w, double *T, double *trc) {
  RefHandle &h = *static_cast<RefHandle *>(p);
  return guarded([&]() {
    h.dycore.convert_dynamics_to_coupler(h.coupler, h.state, h.tracers);
    copy_out(h, rho_d, u, v, w, T, trc);
    return 0;
  });
}

int ref_advance(void *p, double dt_dyn, int nsteps) {
  RefHandle &h = *static_cast<RefHandle *>(p);
  return guarded([&]() {
    for (int n = 0; n < nsteps; n++) h.dycore.time_step_rk_3_3(h.coupler, h.state, h.tracers, dt_dyn);
    return 0;
  });
}

void ref_get_state(void *p, double *st, double *trc) {
  RefHandle &h = *static_cast<RefHandle *>(p);
  int nx = h.cfg.nx, ny = h.cfg.ny, nz = h.cfg.nz;
  size_t NC = size_t(nx) * ny * nz;
  for (int l = 0; l < 5; l++)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) st[l * NC + (size_t(k) * ny + j) * nx + i] = h.state(l, HS + k, HS + j, HS + i);
  for (int l = 0; l < h.cfg.ntr; l++)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) trc[l * NC + (size_t(k) * ny + j) * nx + i] = h.tracers(l, HS + k, HS + j, HS + i);
}

int ref_tendencies(void *p, double *st_tend, double *tr_tend) {
  RefHandle &h = *static_cast<RefHandle *>(p);
  return guarded([&]() {
    real4d a("state_tend", 5, h.cfg.nz, h.cfg.ny, h.cfg.nx), b("tracers_tend", h.cfg.ntr, h.cfg.nz, h.cfg.ny, h.cfg.nx);
    h.dycore.compute_tendencies(h.coupler, h.state, a, h.tracers, b);
    std::memcpy(st_tend, a.data(), a.size() * sizeof(double));
    std::memcpy(tr_tend, b.data(), b.size() * sizeof(double));
    return 0;
  });
}

void ref_weno9_f32(const float *s, int do_map, int imm_L, int imm_R, float *qL, float *qR) {
  SArray<float, 1, 9> st;
  for (int i = 0; i < 9; i++) st(i) = s[i];
  limiter::WenoLimiter<float, 9>::compute_limited_edges(st, *qL, *qR, {do_map != 0, imm_L != 0, imm_R != 0});
}

void ref_weno9_f64(const double *s, int do_map, int imm_L, int imm_R, double *qL, double *qR) {
  SArray<double, 1, 9> st;
  for (int i = 0; i < 9; i++) st(i) = s[i];
  limiter::WenoLimiter<double, 9>::compute_limited_edges(st, *qL, *qR, {do_map != 0, imm_L != 0, imm_R != 0});
}

}  // extern "C"
