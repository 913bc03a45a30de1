// Drop-in replacement of the reference's custom_modules::Time_Averager
// (experiments/examples/custom_modules/time_averager.h:7-111) on libpu_dycore
// (pu_time_averager_accumulate).  The averages stay in the coupler arrays
// avg_u .. long_avg_w and the option time_averager_etime, as in the
// reference; accumulate runs on the GPU (FP64, the reference's order of
// operations) over the coupler's arrays, host or device.
#pragma once

#include "pu_physics_module.h"

namespace custom_modules {

struct Time_Averager {
  static constexpr int NAVG = 13;
  static const char *name(int q) {
    static const char *names[NAVG] = {"avg_u",     "avg_v",     "avg_w",     "avg_tke",    "avg_up_up",
                                      "avg_up_vp", "avg_up_wp", "avg_vp_vp", "avg_vp_wp",  "avg_wp_wp",
                                      "long_avg_u", "long_avg_v", "long_avg_w"};
    return names[q];
  }

  void init(core::Coupler &coupler) {
    auto nx = coupler.get_nx();
    auto ny = coupler.get_ny();
    auto nz = coupler.get_nz();
    auto &dm = coupler.get_data_manager_readwrite();
    coupler.set_option<real>("time_averager_etime", 0);
    for (int q = 0; q < NAVG; q++) {
      dm.register_and_allocate<real>(name(q), "", {nz, ny, nx});
      dm.get<real, 3>(name(q)) = real(0);
      coupler.register_output_variable<real>(name(q), core::Coupler::DIMS_3D);
    }
  }

  void reset(core::Coupler &coupler) {
    coupler.set_option<real>("time_averager_etime", 0);
    auto &dm = coupler.get_data_manager_readwrite();
    for (int q = 0; q < 10; q++) dm.get<real, 3>(name(q)) = real(0);
  }

  void accumulate(core::Coupler &coupler, real dt) {
    pu_physics *h = modules::pu_detail::physics_handle(coupler, false);
    pu_state_view v = modules::pu_detail::physics_view(coupler);
    auto &dm = coupler.get_data_manager_readwrite();
    double *arr[NAVG];
    for (int q = 0; q < NAVG; q++) arr[q] = dm.get<real, 3>(name(q)).data();
    pu_time_averages a{arr[0], arr[1], arr[2],  arr[3],  arr[4],  arr[5],  arr[6],
                       arr[7], arr[8], arr[9],  arr[10], arr[11], arr[12], 0.0};
    a.etime = coupler.get_option<real>("time_averager_etime");
    modules::pu_detail::check_physics(
        pu_time_averager_accumulate(h, &v, &a, coupler.get_option<real>("elapsed_time"), dt));
    modules::pu_detail::check_physics(pu_physics_synchronize(h));
    coupler.set_option<real>("time_averager_etime", a.etime);
  }
};

}  // namespace custom_modules
