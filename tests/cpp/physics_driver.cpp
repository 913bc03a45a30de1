// Driver of the C++ drop-in modules in the order of the reference's
// boundary-layer driver (abl_neutral.cpp:49-108): les_closure.init adds the
// TKE tracer, dycore.init, time_averager.init, then per call geostrophic
// forcing, dycore time_step, sponge, surface fluxes, LES closure, time
// averager, and elapsed_time advanced by dt.  The coupler is the
// single-rank stand-in of oracle/ref_shim; the modules are the headers of
// porturb_b200/cpp on libpu_dycore.so.
//
// Usage: physics_driver <input.bin> <output.bin>
//   input : int32 nx, ny, nz, ncalls; float64 xlen, ylen, zlen, dt_phys, R_d,
//           R_v, cp_d, gamma_d, C0, grav, cfl, lat_g, u_g, v_g, sponge_time,
//           sponge_top; float64 base 6*N and pert 6*N (density_dry, uvel,
//           vvel, wvel, temp, water_vapor); immersed proportion, roughness and
//           temperature halo arrays, 3*(nz+2)(ny+2)(nx+2)
//   output: float64 7*N (the five fields, water_vapor, TKE) and 13*N (the time
//           averages avg_u .. long_avg_w) after ncalls
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "dynamics_rk.h"
#include "geostrophic_wind_forcing.h"
#include "les_closure.h"
#include "sponge_layer.h"
#include "surface_flux.h"
#include "time_averager.h"

template <class T>
static void rd(FILE *f, T *p, size_t n) {
  if (fread(p, sizeof(T), n, f) != n) { fprintf(stderr, "short read\n"); exit(2); }
}

int main(int argc, char **argv) {
  if (argc != 3) return 2;
  FILE *f = fopen(argv[1], "rb");
  int hdr[4];
  rd(f, hdr, 4);
  const int nx = hdr[0], ny = hdr[1], nz = hdr[2], ncalls = hdr[3];
  double g[16];
  rd(f, g, 16);
  const size_t N = size_t(nx) * ny * nz, NH = size_t(nx + 2) * (ny + 2) * (nz + 2);
  std::vector<double> base(6 * N), pert(6 * N), halos(3 * NH);
  rd(f, base.data(), base.size());
  rd(f, pert.data(), pert.size());
  rd(f, halos.data(), halos.size());
  fclose(f);

  core::Coupler coupler(nx, ny, nz, g[0], g[1], g[2]);
  const char *on[7] = {"R_d", "R_v", "cp_d", "gamma_d", "C0", "grav", "cfl"};
  for (int q = 0; q < 7; q++) coupler.set_option<real>(on[q], g[4 + q]);
  coupler.set_option<int>("idWV", 0);
  coupler.set_option<std::string>("bc_x", "periodic");
  coupler.set_option<std::string>("bc_y", "periodic");
  coupler.set_option<std::string>("bc_z", "solid_wall");
  auto &dm = coupler.get_data_manager_readwrite();
  const char *sn[6] = {"density_dry", "uvel", "vvel", "wvel", "temp", "water_vapor"};
  for (int a = 0; a < 5; a++) dm.register_and_allocate<real>(sn[a], "", {nz, ny, nx});
  coupler.add_tracer("water_vapor", "water_vapor", true, true, true);
  const char *hn[3] = {"immersed_proportion_halos", "immersed_roughness_halos", "immersed_temp_halos"};
  for (int a = 0; a < 3; a++) {
    dm.register_and_allocate<real>(hn[a], "", {nz + 2, ny + 2, nx + 2});
    std::copy(halos.begin() + a * NH, halos.begin() + (a + 1) * NH, dm.get<real, 3>(hn[a]).data());
  }
  auto load = [&](const std::vector<double> &src) {
    for (int a = 0; a < 6; a++) std::copy(src.begin() + a * N, src.begin() + (a + 1) * N, dm.get<real, 3>(sn[a]).data());
  };
  modules::LES_Closure les;
  modules::Dynamics_Euler_Stratified_WenoFV dycore;
  custom_modules::Time_Averager tavg;
  coupler.set_option<real>("elapsed_time", 0);
  load(base);
  les.init(coupler);
  dycore.init(coupler);
  tavg.init(coupler);
  load(pert);
  const double dt = g[3];
  double etime = 0;
  for (int c = 0; c < ncalls; c++) {
    modules::geostrophic_wind_forcing(coupler, dt, g[11], g[12], g[13]);
    dycore.time_step(coupler, dt);
    modules::sponge_layer(coupler, dt, g[14], g[15]);
    modules::apply_surface_fluxes(coupler, dt);
    les.apply(coupler, dt);
    tavg.accumulate(coupler, dt);
    etime += dt;
    coupler.set_option<real>("elapsed_time", etime);
  }
  FILE *o = fopen(argv[2], "wb");
  for (int a = 0; a < 6; a++) fwrite(dm.get<real, 3>(sn[a]).data(), sizeof(double), N, o);
  fwrite(dm.get<real, 3>("TKE").data(), sizeof(double), N, o);
  for (int q = 0; q < custom_modules::Time_Averager::NAVG; q++)
    fwrite(dm.get<real, 3>(custom_modules::Time_Averager::name(q)).data(), sizeof(double), N, o);
  fclose(o);
  modules::pu_physics_module_finalize(coupler);
  dycore.finalize(coupler);
  printf("physics driver ok\n");
  return 0;
}
