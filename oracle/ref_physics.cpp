// C entry points around the reference's own physics modules (TEST
// INFRASTRUCTURE ONLY).
//
// Compiles model/modules/les_closure.h, sponge_layer.h,
// geostrophic_wind_forcing.h, surface_flux.h and uniform_pg_wind_forcing.h,
// and experiments/examples/custom_modules/time_averager.h and edge_sponge.h,
// of the reference unchanged
// against the single-rank shim in oracle/ref_shim and exposes them through
// the ref_phys_* functions of oracle/physics_api.h.  Each call copies the
// given coupler arrays into the shim coupler's DataManager, runs the module
// and copies the arrays back.
#include "coupler.h"
#include "geostrophic_wind_forcing.h"
#include "les_closure.h"
#include "physics_api.h"
#include "sponge_layer.h"
#include "surface_flux.h"
#include "uniform_pg_wind_forcing.h"
#include "time_averager.h"
#include "edge_sponge.h"

#include <cstdio>
#include <cstring>

namespace {

struct PhysHandle {
  core::Coupler coupler;
  orc_phys_config cfg;
  PhysHandle(const orc_phys_config &c) : coupler(c.nx, c.ny, c.nz, c.xlen, c.ylen, c.zlen), cfg(c) {}
};

const char *bc_name(int bc) { return bc == 1 ? "precursor" : bc == 2 ? "solid_wall" : "periodic"; }

size_t ncell(const orc_phys_config &c) { return size_t(c.nx) * c.ny * c.nz; }

void copy_in(PhysHandle &h, const double *rho_d, const double *u, const double *v, const double *w, const double *T,
             const double *trc) {
  auto &dm = h.coupler.get_data_manager_readwrite();
  const size_t n = ncell(h.cfg);
  std::memcpy(dm.get<real, 3>("density_dry").data(), rho_d, n * sizeof(double));
  std::memcpy(dm.get<real, 3>("uvel").data(), u, n * sizeof(double));
  std::memcpy(dm.get<real, 3>("vvel").data(), v, n * sizeof(double));
  std::memcpy(dm.get<real, 3>("wvel").data(), w, n * sizeof(double));
  std::memcpy(dm.get<real, 3>("temp").data(), T, n * sizeof(double));
  auto names = h.coupler.get_tracer_names();
  for (size_t t = 0; t < names.size(); t++) std::memcpy(dm.get<real, 3>(names[t]).data(), trc + t * n, n * sizeof(double));
}

void copy_out(PhysHandle &h, double *rho_d, double *u, double *v, double *w, double *T, double *trc) {
  auto &dm = h.coupler.get_data_manager_readonly();
  const size_t n = ncell(h.cfg);
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
    std::fprintf(stderr, "ref_phys: %s\n", e.what());
    return -1;
  }
}

}  // namespace

extern "C" {

void *ref_phys_create(const orc_phys_config *cfg, const double *imm_prop_h, const double *imm_rough_h,
                      const double *imm_temp_h) {
  PhysHandle *h = nullptr;
  int rc = guarded([&]() {
    h = new PhysHandle(*cfg);
    auto &c = h->coupler;
    c.set_option<real>("R_d", cfg->R_d);
    c.set_option<real>("R_v", cfg->R_v);
    c.set_option<real>("cp_d", cfg->cp_d);
    c.set_option<real>("gamma_d", cfg->gamma_d);
    c.set_option<real>("C0", cfg->C0);
    c.set_option<real>("grav", cfg->grav);
    c.set_option<real>("p0", cfg->p0);
    c.set_option<bool>("enable_gravity", cfg->enable_gravity != 0);
    c.set_option<real>("kinematic_viscosity", cfg->kinematic_viscosity);
    c.set_option<bool>("dns", cfg->dns != 0);
    c.set_option<real>("les_total_mult", cfg->les_total_mult);
    c.set_option<real>("les_dissipation_mult", cfg->les_dissipation_mult);
    c.set_option<real>("les_shear_prod_mult", cfg->les_shear_prod_mult);
    c.set_option<std::string>("bc_x", bc_name(cfg->bc_x));
    c.set_option<std::string>("bc_y", bc_name(cfg->bc_y));
    c.set_option<std::string>("bc_z", bc_name(cfg->bc_z));
    auto &dm = c.get_data_manager_readwrite();
    for (auto nm : {"density_dry", "uvel", "vvel", "wvel", "temp"})
      dm.register_and_allocate<real>(nm, "", {cfg->nz, cfg->ny, cfg->nx});
    for (int t = 0; t < cfg->ntr; t++) {
      char name[32];
      if (t == cfg->idWV) std::snprintf(name, sizeof(name), "water_vapor");
      else if (t == cfg->idTKE) std::snprintf(name, sizeof(name), "TKE");
      else std::snprintf(name, sizeof(name), "tracer_%d", t);
      c.add_tracer(name, name, cfg->tracer_positive[t] != 0, cfg->tracer_adds_mass[t] != 0, cfg->tracer_diffuse[t] != 0);
    }
    const size_t nh = size_t(cfg->nz + 2) * (cfg->ny + 2) * (cfg->nx + 2);
    const char *names[3] = {"immersed_proportion_halos", "immersed_roughness_halos", "immersed_temp_halos"};
    const double *src[3] = {imm_prop_h, imm_rough_h, imm_temp_h};
    for (int a = 0; a < 3; a++) {
      dm.register_and_allocate<real>(names[a], "", {cfg->nz + 2, cfg->ny + 2, cfg->nx + 2});
      std::memcpy(dm.get<real, 3>(names[a]).data(), src[a], nh * sizeof(double));
    }
    return 0;
  });
  if (rc != 0) {
    delete h;
    return nullptr;
  }
  return h;
}

void ref_phys_destroy(void *p) { delete static_cast<PhysHandle *>(p); }

int ref_phys_les(void *p, double *rho_d, double *u, double *v, double *w, double *T, double *trc, double dt) {
  PhysHandle &h = *static_cast<PhysHandle *>(p);
  return guarded([&]() {
    copy_in(h, rho_d, u, v, w, T, trc);
    modules::LES_Closure les;
    les.apply(h.coupler, dt);
    copy_out(h, rho_d, u, v, w, T, trc);
    return 0;
  });
}

int ref_phys_sponge(void *p, double *rho_d, double *u, double *v, double *w, double *T, double *trc, double dt,
                    double time_scale, double top_prop) {
  PhysHandle &h = *static_cast<PhysHandle *>(p);
  return guarded([&]() {
    copy_in(h, rho_d, u, v, w, T, trc);
    modules::sponge_layer(h.coupler, dt, time_scale, top_prop);
    copy_out(h, rho_d, u, v, w, T, trc);
    return 0;
  });
}

int ref_phys_geostrophic(void *p, double *rho_d, double *u, double *v, double *w, double *T, double *trc, double dt,
                         double lat_g, double u_g, double v_g) {
  PhysHandle &h = *static_cast<PhysHandle *>(p);
  return guarded([&]() {
    copy_in(h, rho_d, u, v, w, T, trc);
    modules::geostrophic_wind_forcing(h.coupler, dt, lat_g, u_g, v_g);
    copy_out(h, rho_d, u, v, w, T, trc);
    return 0;
  });
}

int ref_phys_surface_fluxes(void *p, double *rho_d, double *u, double *v, double *w, double *T, double *trc,
                            double dt) {
  PhysHandle &h = *static_cast<PhysHandle *>(p);
  return guarded([&]() {
    copy_in(h, rho_d, u, v, w, T, trc);
    modules::apply_surface_fluxes(h.coupler, dt);
    copy_out(h, rho_d, u, v, w, T, trc);
    return 0;
  });
}

int ref_phys_uniform_pg(void *p, double *rho_d, double *u, double *v, double *w, double *T, double *trc, double dt,
                        double tau, unsigned long long update_cycles, double *st) {
  PhysHandle &h = *static_cast<PhysHandle *>(p);
  return guarded([&]() {
    copy_in(h, rho_d, u, v, w, T, trc);
    auto &c = h.coupler;
    const std::string pre = "uniform_pg_wind_forcing_";
    c.set_option<size_t>(pre + "counter", size_t(st[0]));
    if (st[0] > 0) {
      c.set_option<real>(pre + "u0", st[1]);
      c.set_option<real>(pre + "v0", st[2]);
      c.set_option<real>(pre + "u", st[3]);
      c.set_option<real>(pre + "v", st[4]);
    }
    modules::uniform_pg_wind_forcing(c, dt, tau, size_t(update_cycles));
    copy_out(h, rho_d, u, v, w, T, trc);
    st[0] = double(c.get_option<size_t>(pre + "counter"));
    st[1] = c.get_option<real>(pre + "u0");
    st[2] = c.get_option<real>(pre + "v0");
    st[3] = c.get_option<real>(pre + "u");
    st[4] = c.get_option<real>(pre + "v");
    return 0;
  });
}

int ref_phys_uniform_pg_height(void *p, double *rho_d, double *u, double *v, double *w, double *T, double *trc,
                               double dt, double height, double u0, double v0, double tau) {
  PhysHandle &h = *static_cast<PhysHandle *>(p);
  return guarded([&]() {
    copy_in(h, rho_d, u, v, w, T, trc);
    modules::uniform_pg_wind_forcing_height(h.coupler, dt, height, u0, v0, tau);
    copy_out(h, rho_d, u, v, w, T, trc);
    return 0;
  });
}

int ref_phys_time_average(void *p, double *rho_d, double *u, double *v, double *w, double *T, double *trc,
                          double *avgs, double *etime, double elapsed_time, double dt) {
  PhysHandle &h = *static_cast<PhysHandle *>(p);
  return guarded([&]() {
    static const char *names[13] = {"avg_u",      "avg_v",      "avg_w",     "avg_tke",   "avg_up_up",
                                    "avg_up_vp",  "avg_up_wp",  "avg_vp_vp", "avg_vp_wp", "avg_wp_wp",
                                    "long_avg_u", "long_avg_v", "long_avg_w"};
    auto &c = h.coupler;
    custom_modules::Time_Averager ta;
    if (!c.get_data_manager_readonly().entry_exists("avg_u")) ta.init(c);
    copy_in(h, rho_d, u, v, w, T, trc);
    const size_t n = ncell(h.cfg);
    auto &dm = c.get_data_manager_readwrite();
    for (int q = 0; q < 13; q++) std::memcpy(dm.get<real, 3>(names[q]).data(), avgs + q * n, n * sizeof(double));
    c.set_option<real>("time_averager_etime", *etime);
    c.set_option<real>("elapsed_time", elapsed_time);
    ta.accumulate(c, dt);
    for (int q = 0; q < 13; q++)
      std::memcpy(avgs + q * n, dm.get<real const, 3>(names[q]).data(), n * sizeof(double));
    *etime = c.get_option<real>("time_averager_etime");
    copy_out(h, rho_d, u, v, w, T, trc);
    return 0;
  });
}

int ref_phys_edge_sponge_set_column(void *p, double *rho_d, double *u, double *v, double *w, double *T, double *trc,
                                    double *column) {
  PhysHandle &h = *static_cast<PhysHandle *>(p);
  return guarded([&]() {
    copy_in(h, rho_d, u, v, w, T, trc);
    custom_modules::EdgeSponge es;
    es.set_column(h.coupler);
    const int nz = h.cfg.nz;
    for (int l = 0; l < 5; l++)
      for (int k = 0; k < nz; k++) column[size_t(l) * nz + k] = es.column(l, k);
    return 0;
  });
}

int ref_phys_edge_sponge_apply(void *p, double *rho_d, double *u, double *v, double *w, double *T, double *trc,
                               const double *column, double px1, double px2, double py1, double py2) {
  PhysHandle &h = *static_cast<PhysHandle *>(p);
  return guarded([&]() {
    copy_in(h, rho_d, u, v, w, T, trc);
    custom_modules::EdgeSponge es;
    es.names = {"density_dry", "uvel", "vvel", "wvel", "temp"};
    const int nz = h.cfg.nz;
    es.column = real2d("column", 5, nz);
    for (int l = 0; l < 5; l++)
      for (int k = 0; k < nz; k++) es.column(l, k) = column[size_t(l) * nz + k];
    es.apply(h.coupler, px1, px2, py1, py2);
    copy_out(h, rho_d, u, v, w, T, trc);
    return 0;
  });
}

}  // extern "C"
