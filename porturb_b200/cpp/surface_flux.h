// Drop-in replacement of the reference's modules::apply_surface_fluxes
// (model/modules/surface_flux.h:9-125) on libpu_dycore (pu_surface_fluxes).
#pragma once

#include "pu_physics_module.h"

namespace modules {

inline void apply_surface_fluxes(core::Coupler &coupler, real dt) {
  pu_physics *h = pu_detail::physics_handle(coupler);
  pu_state_view v = pu_detail::physics_view(coupler);
  pu_detail::check_physics(pu_surface_fluxes(h, &v, dt));
  pu_detail::check_physics(pu_physics_synchronize(h));
}

}  // namespace modules
