// Drop-in replacement of the reference's custom_modules::EdgeSponge
// (experiments/examples/custom_modules/edge_sponge.h:8-101; the urban and
// turbine drivers, city.cpp:97,137) on libpu_dycore
// (pu_edge_sponge_set_column, pu_edge_sponge_apply).  set_column records the
// horizontal-mean profile of the named coupler fields -- summed over the
// ranks through the coupler's communicator as the reference does -- and
// apply relaxes the fields toward it near the lateral edges of the global
// domain, on the GPU.
#pragma once

#include <string>
#include <vector>

#include "pu_physics_module.h"

namespace custom_modules {

class EdgeSponge {
 public:
  std::vector<std::string> names;
  std::vector<double> column;   // names.size() x nz, field-major

  void set_column(core::Coupler &coupler,
                  std::vector<std::string> names_in = {"density_dry", "uvel", "vvel", "wvel", "temp"}) {
    names = names_in;
    const int nz = coupler.get_nz();
    std::vector<int> f = fields(coupler);
    pu_physics *h = modules::pu_detail::physics_handle(coupler, false);
    pu_state_view v = modules::pu_detail::physics_view(coupler);
    column.assign(names.size() * nz, 0.0);
    modules::pu_detail::check_physics(pu_edge_sponge_set_column(h, &v, f.data(), int(f.size()), column.data()));
    // Tile means -> global means (edge_sponge.h:86-94).
    const double nloc = double(coupler.get_nx()) * coupler.get_ny();
    const double nglob = double(coupler.get_nx_glob()) * coupler.get_ny_glob();
    if (nglob != nloc) {
      yakl::Array<real, 2, yakl::memHost, yakl::styleC> sums("edge_sponge_sums", int(names.size()), nz);
      for (size_t q = 0; q < column.size(); q++) sums.data()[q] = column[q] * nloc;
      auto tot = coupler.get_parallel_comm().all_reduce(sums, MPI_SUM, "column_nudging_Allreduce");
      for (size_t q = 0; q < column.size(); q++) column[q] = tot.data()[q] / nglob;
    }
  }

  void apply(core::Coupler &coupler, real prop_x1 = 0.1, real prop_x2 = 0.1, real prop_y1 = 0.1,
             real prop_y2 = 0.1) {
    std::vector<int> f = fields(coupler);
    pu_physics *h = modules::pu_detail::physics_handle(coupler, false);
    pu_state_view v = modules::pu_detail::physics_view(coupler);
    modules::pu_detail::check_physics(pu_edge_sponge_apply(
        h, &v, f.data(), int(f.size()), column.data(), prop_x1, prop_x2, prop_y1, prop_y2,
        (long long)coupler.get_i_beg(), (long long)coupler.get_j_beg(), (long long)coupler.get_nx_glob(),
        (long long)coupler.get_ny_glob()));
    modules::pu_detail::check_physics(pu_physics_synchronize(h));
  }

 private:
  // Indices of the named fields in the state view (pu_physics.h).
  std::vector<int> fields(core::Coupler &coupler) const {
    static const char *state[5] = {"density_dry", "uvel", "vvel", "wvel", "temp"};
    auto trc = coupler.get_tracer_names();
    std::vector<int> f;
    for (auto const &n : names) {
      int idx = -1;
      for (int a = 0; a < 5; a++)
        if (n == state[a]) idx = a;
      for (size_t t = 0; t < trc.size() && idx < 0; t++)
        if (n == trc[t]) idx = 5 + int(t);
      if (idx < 0) Kokkos::abort(("EdgeSponge: no coupler field " + n).c_str());
      f.push_back(idx);
    }
    return f;
  }
};

}  // namespace custom_modules
