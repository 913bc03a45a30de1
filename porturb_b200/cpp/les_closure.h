// Drop-in replacement of the reference's modules::LES_Closure
// (model/modules/les_closure.h:9-574) on libpu_dycore (pu_les_apply).
//     void init(core::Coupler &) const;           les_closure.h:19-26
//     void apply(core::Coupler &, real dt) const;  les_closure.h:30-320
#pragma once

#include "pu_physics_module.h"

namespace modules {

struct LES_Closure {
  int static constexpr hs = 1;
  int static constexpr num_state = 5;
  int static constexpr idR = 0;
  int static constexpr idU = 1;
  int static constexpr idV = 2;
  int static constexpr idW = 3;
  int static constexpr idT = 4;

  // Adds the mass-weighted TKE tracer and sets it to 0.1 everywhere.
  void init(core::Coupler &coupler) const {
    auto nx = coupler.get_nx(), ny = coupler.get_ny(), nz = coupler.get_nz();
    coupler.add_tracer("TKE", "mass-weighted TKE", true, false, false);
    auto tke = coupler.get_data_manager_readwrite().get<real, 3>("TKE");
    real *p = tke.data();
    for (size_t q = 0; q < size_t(nx) * ny * nz; q++) p[q] = 0.1;
  }

  void apply(core::Coupler &coupler, real dtphys) const {
    pu_physics *h = pu_detail::physics_handle(coupler);
    pu_state_view v = pu_detail::physics_view(coupler);
    pu_detail::check_physics(pu_les_apply(h, &v, dtphys));
    pu_detail::check_physics(pu_physics_synchronize(h));
  }
};

}  // namespace modules
