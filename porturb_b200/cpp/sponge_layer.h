// Drop-in replacement of the reference's modules::sponge_layer
// (model/modules/sponge_layer.h:7-62) on libpu_dycore (pu_sponge_layer).
#pragma once

#include "pu_physics_module.h"

namespace modules {

inline void sponge_layer(core::Coupler &coupler, real dt, real time_scale, real top_prop) {
  pu_physics *h = pu_detail::physics_handle(coupler);
  pu_state_view v = pu_detail::physics_view(coupler);
  pu_detail::check_physics(pu_sponge_layer(h, &v, dt, time_scale, top_prop));
  pu_detail::check_physics(pu_physics_synchronize(h));
}

}  // namespace modules
