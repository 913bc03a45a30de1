// Drop-in replacement of the reference's modules::Dynamics_Euler_Stratified_WenoFV
// (model/modules/dynamics_rk.h:25-1355) on top of libpu_dycore (include/pu_dycore.h).
//
// A portUrb driver includes this header instead of the reference's
// dynamics_rk.h and links libpu_dycore.so; the module keeps the reference's
// members and signatures:
//     real compute_time_step(core::Coupler const &) const;   dynamics_rk.h:57-64
//     void time_step(core::Coupler &, real dt_phys) const;    dynamics_rk.h:103-137
//     void init(core::Coupler &) const;                        dynamics_rk.h:917-1246
// It reads the same coupler options and DataManager entries, and registers the
// entries other modules read after init (tracer_positive, tracer_adds_mass,
// hy_{dens,theta,pressure}_{cells,edges}).  The order is fixed at 9.
//
// The GPU state lives in a pu_dycore handle owned by the module; the handle is
// recorded in the coupler's options ("pu_dycore_handle") so the module itself
// stays stateless like the reference's.  DataManager arrays may be host or
// device memory (the library inspects the pointers, PU_MEM_AUTO).  Errors end
// the run through Kokkos::abort, as the reference does.
#pragma once

#include <algorithm>
#include <cstddef>
#include <string>
#include <vector>

#include "coupler.h"
#include "pu_dycore.h"

namespace modules {

struct Dynamics_Euler_Stratified_WenoFV {
  size_t static constexpr ord = 9;
  int static constexpr hs = (ord - 1) / 2;
  int static constexpr num_state = 5;
  int static constexpr idR = 0;
  int static constexpr idU = 1;
  int static constexpr idV = 2;
  int static constexpr idW = 3;
  int static constexpr idT = 4;

  static void check(int status) {
    if (status != PU_OK) Kokkos::abort((std::string("pu_dycore: ") + pu_last_error()).c_str());
  }

  static int bc_code(std::string const &bc) {
    if (bc == "periodic") return PU_BC_PERIODIC;
    if (bc == "precursor") return PU_BC_PRECURSOR;
    if (bc == "solid_wall") return PU_BC_WALL;
    Kokkos::abort("ERROR: Specified invalid boundary condition in coupler options");
    return -1;
  }

  static pu_dycore *handle(core::Coupler const &coupler) {
    if (!coupler.option_exists("pu_dycore_handle")) Kokkos::abort("pu_dycore: time_step before init");
    return reinterpret_cast<pu_dycore *>(coupler.get_option<size_t>("pu_dycore_handle"));
  }

  static pu_state_view coupler_view(core::Coupler &coupler) {
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

  real compute_time_step(core::Coupler const &coupler) const {
    real cfl = coupler.get_option<real>("cfl", 0.60);
    return cfl * std::min(std::min(coupler.get_dx(), coupler.get_dy()), coupler.get_dz()) / (350 + 100);
  }

  void init(core::Coupler &coupler) const {
    pu_config cfg{};
    cfg.nx = coupler.get_nx();
    cfg.ny = coupler.get_ny();
    cfg.nz = coupler.get_nz();
    cfg.dx = coupler.get_dx();
    cfg.dy = coupler.get_dy();
    cfg.dz = coupler.get_dz();
    auto names = coupler.get_tracer_names();
    cfg.ntracers = int(names.size());
    if (cfg.ntracers > PU_MAX_TRACERS) Kokkos::abort("pu_dycore: too many tracers for this build");
    for (int t = 0; t < cfg.ntracers; t++) {
      std::string desc;
      bool found, positive, adds_mass, diffuse;
      coupler.get_tracer_info(names[t], desc, found, positive, adds_mass, diffuse);
      cfg.tracer_positive[t] = positive;
      cfg.tracer_adds_mass[t] = adds_mass;
    }
    cfg.idWV = coupler.get_option<int>("idWV");
    cfg.R_d = coupler.get_option<real>("R_d");
    cfg.R_v = coupler.get_option<real>("R_v");
    cfg.cp_d = coupler.get_option<real>("cp_d");
    cfg.gamma_d = coupler.get_option<real>("gamma_d");
    cfg.C0 = coupler.get_option<real>("C0");
    cfg.grav = coupler.get_option<real>("grav");
    cfg.cfl = coupler.get_option<real>("cfl", 0.60);
    cfg.immersed_power = coupler.get_option<real>("immersed_power", 5);
    cfg.latitude = coupler.get_option<real>("latitude", 0);
    cfg.bc_x = bc_code(coupler.get_option<std::string>("bc_x", "periodic"));
    cfg.bc_y = bc_code(coupler.get_option<std::string>("bc_y", "periodic"));
    cfg.bc_z = bc_code(coupler.get_option<std::string>("bc_z", "solid_wall"));
    cfg.enable_gravity = coupler.get_option<bool>("enable_gravity", true);
    cfg.weno_all = coupler.get_option<bool>("weno_all", true);
    cfg.precision = coupler.get_option<std::string>("pu_precision", "f32") == "f64" ? PU_F64 : PU_F32;
    cfg.weno_mode = PU_WENO_PLAIN;
    cfg.device = coupler.get_option<int>("pu_device", 0);
    cfg.stream = nullptr;
    pu_dycore *h = nullptr;
    check(pu_dycore_create(&cfg, &h));
    coupler.set_option<size_t>("pu_dycore_handle", reinterpret_cast<size_t>(h));
    // A coupler distributed over several ranks (coupler.h:132-229): this
    // rank's handle becomes its tile of the domain, exchanging halos with the
    // other ranks' tiles over NCCL.  Rank 0 (px = py = 0) makes the NCCL id
    // and broadcasts it over the coupler's communicator.
    if (coupler.get_nproc_x() * coupler.get_nproc_y() > 1) {
      int id[PU_NCCL_ID_BYTES / sizeof(int)] = {};
      if (coupler.get_px() == 0 && coupler.get_py() == 0)
        check(pu_nccl_get_unique_id(reinterpret_cast<unsigned char *>(id)));
      auto comm = coupler.get_parallel_comm();
      for (auto &w : id) comm.broadcast(w, 0);
      pu_decomp d{coupler.get_nproc_x(), coupler.get_nproc_y(), coupler.get_px(), coupler.get_py(),
                  (long long)coupler.get_nx_glob(), (long long)coupler.get_ny_glob()};
      check(pu_dycore_set_decomposition(h, &d, reinterpret_cast<unsigned char *>(id)));
    }

    auto &dm = coupler.get_data_manager_readwrite();
    pu_state_view v = coupler_view(coupler);
    const double *prop = dm.entry_exists("immersed_proportion")
                             ? dm.get<real const, 3>("immersed_proportion").data() : nullptr;
    // The optional windmill projection joins the proportion (:1019-1025).
    const double *proj = dm.entry_exists("windmill_proj_weight")
                             ? dm.get<real const, 3>("windmill_proj_weight").data() : nullptr;
    check(pu_dycore_init_windmill(h, &v, prop, proj, PU_MEM_AUTO));

    // Entries the reference's init registers for other modules (:951-956, :961-966, :1152-1154).
    const int nz = cfg.nz, nzh = nz + 2 * hs;
    std::vector<double> c[3], e[3];
    for (int q = 0; q < 3; q++) { c[q].resize(nzh); e[q].resize(nz + 1); }
    check(pu_dycore_get_hydrostasis(h, c[0].data(), c[1].data(), c[2].data(), e[0].data(), e[1].data(), e[2].data()));
    const char *cn[3] = {"hy_dens_cells", "hy_theta_cells", "hy_pressure_cells"};
    const char *en[3] = {"hy_dens_edges", "hy_theta_edges", "hy_pressure_edges"};
    for (int q = 0; q < 3; q++) {
      if (!dm.entry_exists(cn[q])) dm.register_and_allocate<float>(cn[q], "", {nzh});
      if (!dm.entry_exists(en[q])) dm.register_and_allocate<float>(en[q], "", {nz + 1});
      yakl::Array<float, 1, yakl::memHost, yakl::styleC> hc("hc", nzh), he("he", nz + 1);
      for (int k = 0; k < nzh; k++) hc(k) = float(c[q][k]);
      for (int k = 0; k < nz + 1; k++) he(k) = float(e[q][k]);
      hc.deep_copy_to(dm.get<float, 1>(cn[q]));
      he.deep_copy_to(dm.get<float, 1>(en[q]));
    }
    const char *tn[2] = {"tracer_positive", "tracer_adds_mass"};
    for (int q = 0; q < 2; q++) {
      if (!dm.entry_exists(tn[q])) dm.register_and_allocate<bool>(tn[q], "", {cfg.ntracers});
      yakl::Array<bool, 1, yakl::memHost, yakl::styleC> hb("hb", cfg.ntracers);
      for (int t = 0; t < cfg.ntracers; t++) hb(t) = q == 0 ? cfg.tracer_positive[t] : cfg.tracer_adds_mass[t];
      hb.deep_copy_to(dm.get<bool, 1>(tn[q]));
    }
  }

  void time_step(core::Coupler &coupler, real dt_phys) const {
    pu_state_view v = coupler_view(coupler);
    int ncycles = 0;
    check(pu_dycore_time_step(handle(coupler), &v, dt_phys, &ncycles));
  }

  // Releases the GPU state (the reference frees its DataManager entries in
  // Coupler::finalize).
  void finalize(core::Coupler &coupler) const {
    if (coupler.option_exists("pu_dycore_handle")) {
      pu_dycore_destroy(handle(coupler));
      coupler.set_option<size_t>("pu_dycore_handle", size_t(0));
    }
  }
};

}  // namespace modules
