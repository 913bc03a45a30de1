// Shared part of the drop-in physics modules (les_closure.h, sponge_layer.h,
// geostrophic_wind_forcing.h, surface_flux.h, uniform_pg_wind_forcing.h in
// this directory) on top of
// libpu_dycore's physics entry points (include/pu_physics.h).
//
// The reference's modules read their options and the immersed halo arrays
// from the coupler on every call.  Here the first call builds one pu_physics
// handle from the same options and DataManager entries (immersed_proportion_
// halos, immersed_roughness_halos, immersed_temp_halos -- registered by the
// drivers' init, sc_init.h:727-768), records it in the coupler's options
// ("pu_physics_handle") and reuses it; call pu_physics_module_finalize
// before the coupler goes away.  Errors end the run through Kokkos::abort, as
// in the reference.
#pragma once

#include <string>
#include <vector>

#include "coupler.h"
#include "pu_physics.h"

namespace modules {
namespace pu_detail {

inline void check_physics(int status) {
  if (status != PU_OK) Kokkos::abort((std::string("pu_physics: ") + pu_last_error()).c_str());
}

inline int physics_bc(std::string const &bc) {
  if (bc == "periodic") return PU_BC_PERIODIC;
  if (bc == "precursor") return PU_BC_PRECURSOR;
  if (bc == "solid_wall") return PU_BC_WALL;
  Kokkos::abort("ERROR: Specified invalid boundary condition in coupler options");
  return -1;
}

inline bool have_immersed_halos(core::Coupler const &coupler) {
  auto const &dm = coupler.get_data_manager_readonly();
  return dm.entry_exists("immersed_proportion_halos") && dm.entry_exists("immersed_roughness_halos") &&
         dm.entry_exists("immersed_temp_halos");
}

// need_halos = false (modules that read no immersed arrays: the pressure-
// gradient forcings): without the immersed_*_halos entries the handle is made
// with no immersed cells and kept under its own option key, so a later module
// that needs the entries still finds them missing, as in the reference.
inline pu_physics *physics_handle(core::Coupler &coupler, bool need_halos = true) {
  const bool plain = !need_halos && !have_immersed_halos(coupler);
  const char *key = plain ? "pu_physics_handle_no_immersed" : "pu_physics_handle";
  if (coupler.option_exists(key) && coupler.get_option<size_t>(key) != 0)
    return reinterpret_cast<pu_physics *>(coupler.get_option<size_t>(key));
  pu_physics_config c{};
  c.nx = coupler.get_nx();
  c.ny = coupler.get_ny();
  c.nz = coupler.get_nz();
  c.dx = coupler.get_dx();
  c.dy = coupler.get_dy();
  c.dz = coupler.get_dz();
  auto names = coupler.get_tracer_names();
  if (int(names.size()) > PU_MAX_TRACERS) Kokkos::abort("pu_physics: too many tracers");
  c.ntracers = int(names.size());
  c.idTKE = -1;
  for (int t = 0; t < c.ntracers; t++) {
    std::string desc;
    bool found, positive, adds_mass, diffuse;
    coupler.get_tracer_info(names[t], desc, found, positive, adds_mass, diffuse);
    c.tracer_diffuse[t] = diffuse ? 1 : 0;
    if (names[t] == "TKE") c.idTKE = t;
  }
  c.R_d = coupler.get_option<real>("R_d");
  c.gamma_d = coupler.get_option<real>("gamma_d");
  c.C0 = coupler.get_option<real>("C0");
  c.grav = coupler.get_option<real>("grav");
  c.enable_gravity = coupler.get_option<bool>("enable_gravity", true) ? 1 : 0;
  c.kinematic_viscosity = coupler.get_option<real>("kinematic_viscosity", 0);
  c.dns = coupler.get_option<bool>("dns", false) ? 1 : 0;
  c.les_total_mult = coupler.get_option<real>("les_total_mult", 1.);
  c.les_dissipation_mult = coupler.get_option<real>("les_dissipation_mult", 1.);
  c.les_shear_prod_mult = coupler.get_option<real>("les_shear_prod_mult", 1.);
  c.bc_x = physics_bc(coupler.get_option<std::string>("bc_x", "periodic"));
  c.bc_y = physics_bc(coupler.get_option<std::string>("bc_y", "periodic"));
  c.bc_z = physics_bc(coupler.get_option<std::string>("bc_z", "solid_wall"));
  c.device = 0;
  c.stream = nullptr;
  pu_physics *h = nullptr;
  if (plain) {
    std::vector<double> zero(size_t(c.nz + 2) * (c.ny + 2) * (c.nx + 2), 0.0);
    check_physics(pu_physics_create(&c, zero.data(), zero.data(), zero.data(), PU_MEM_HOST, &h));
  } else {
    auto const &dm = coupler.get_data_manager_readonly();
    auto prop = dm.get<real const, 3>("immersed_proportion_halos");
    auto rough = dm.get<real const, 3>("immersed_roughness_halos");
    auto temp = dm.get<real const, 3>("immersed_temp_halos");
    check_physics(pu_physics_create(&c, prop.data(), rough.data(), temp.data(), PU_MEM_AUTO, &h));
  }
  coupler.set_option<size_t>(key, reinterpret_cast<size_t>(h));
  return h;
}

// The coupler's state arrays as a pu_state_view (host or device memory).
inline pu_state_view physics_view(core::Coupler &coupler) {
  auto &dm = coupler.get_data_manager_readwrite();
  pu_state_view v{};
  v.rho_d = dm.get<real, 3>("density_dry").data();
  v.uvel = dm.get<real, 3>("uvel").data();
  v.vvel = dm.get<real, 3>("vvel").data();
  v.wvel = dm.get<real, 3>("wvel").data();
  v.temp = dm.get<real, 3>("temp").data();
  auto names = coupler.get_tracer_names();
  for (size_t t = 0; t < names.size() && t < PU_MAX_TRACERS; t++) v.tracers[t] = dm.get<real, 3>(names[t]).data();
  v.mem = PU_MEM_AUTO;
  return v;
}

}  // namespace pu_detail

// Releases the handles the physics modules created on this coupler.
inline void pu_physics_module_finalize(core::Coupler &coupler) {
  for (const char *key : {"pu_physics_handle", "pu_physics_handle_no_immersed"}) {
    if (!coupler.option_exists(key) || coupler.get_option<size_t>(key) == 0) continue;
    pu_physics_destroy(reinterpret_cast<pu_physics *>(coupler.get_option<size_t>(key)));
    coupler.set_option<size_t>(key, size_t(0));
  }
}

}  // namespace modules
