// Drop-in replacements of the reference's modules::uniform_pg_wind_forcing
// and modules::uniform_pg_wind_forcing_height
// (model/modules/uniform_pg_wind_forcing.h:6-82) on libpu_dycore
// (pu_uniform_pg_wind_forcing, pu_uniform_pg_wind_forcing_height).  The state
// carried between calls stays in the coupler options
// uniform_pg_wind_forcing_counter, _u0, _v0, _u and _v, as in the reference;
// neither module needs the immersed arrays on the coupler.
#pragma once

#include "pu_physics_module.h"

namespace modules {

inline void uniform_pg_wind_forcing(core::Coupler &coupler, real dt, real tau = 10, size_t update_cycles = 1) {
  pu_physics *h = pu_detail::physics_handle(coupler, false);
  pu_state_view v = pu_detail::physics_view(coupler);
  const std::string pre = "uniform_pg_wind_forcing_";
  pu_uniform_pg_state st{};
  st.counter = coupler.get_option<size_t>(pre + "counter", 0);
  if (st.counter != 0) {
    st.u0 = coupler.get_option<real>(pre + "u0");
    st.v0 = coupler.get_option<real>(pre + "v0");
    st.u = coupler.get_option<real>(pre + "u");
    st.v = coupler.get_option<real>(pre + "v");
  }
  pu_detail::check_physics(pu_uniform_pg_wind_forcing(h, &v, dt, tau, update_cycles, &st));
  pu_detail::check_physics(pu_physics_synchronize(h));
  coupler.set_option<real>(pre + "u0", st.u0);
  coupler.set_option<real>(pre + "v0", st.v0);
  coupler.set_option<real>(pre + "u", st.u);
  coupler.set_option<real>(pre + "v", st.v);
  coupler.set_option<size_t>(pre + "counter", size_t(st.counter));
}

inline void uniform_pg_wind_forcing_height(core::Coupler &coupler, real dt, real height, real u0, real v0,
                                           real tau = 10) {
  pu_physics *h = pu_detail::physics_handle(coupler, false);
  pu_state_view v = pu_detail::physics_view(coupler);
  pu_detail::check_physics(pu_uniform_pg_wind_forcing_height(h, &v, dt, height, u0, v0, tau));
  pu_detail::check_physics(pu_physics_synchronize(h));
}

}  // namespace modules
