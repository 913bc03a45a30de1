// Drop-in replacement of the reference's modules::geostrophic_wind_forcing
// (model/modules/geostrophic_wind_forcing.h:7-42) on libpu_dycore
// (pu_geostrophic_forcing).
#pragma once

#include "pu_physics_module.h"

namespace modules {

inline void geostrophic_wind_forcing(core::Coupler &coupler, real dt, real lat_g, real u_g, real v_g) {
  pu_physics *h = pu_detail::physics_handle(coupler);
  pu_state_view v = pu_detail::physics_view(coupler);
  pu_detail::check_physics(pu_geostrophic_forcing(h, &v, dt, lat_g, u_g, v_g));
  pu_detail::check_physics(pu_physics_synchronize(h));
}

}  // namespace modules
