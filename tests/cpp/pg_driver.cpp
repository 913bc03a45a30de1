// Driver of the C++ drop-in pressure-gradient forcings
// (porturb_b200/cpp/uniform_pg_wind_forcing.h) and edge sponge
// (porturb_b200/cpp/edge_sponge.h) on the single-rank stand-in coupler of
// oracle/ref_shim, with no immersed arrays registered: the edge sponge
// records its column profile, then ncalls of uniform_pg_wind_forcing with
// +0.25 m/s added to uvel after each, then one
// uniform_pg_wind_forcing_height, then the edge sponge (city.cpp:137).
//
// Usage: pg_driver <input.bin> <output.bin>
//   input : int32 nx, ny, nz, ncalls, update_cycles; float64 xlen, ylen, zlen,
//           dt, tau, height, u0, v0, tau_height; float64 uvel N, vvel N
//   output: float64 uvel N, vvel N, then counter, u0, v0, u, v of the
//           coupler options after the uniform forcing calls, then the five
//           state fields after the edge sponge (5 N)
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "edge_sponge.h"
#include "uniform_pg_wind_forcing.h"

template <class T>
static void rd(FILE *f, T *p, size_t n) {
  if (fread(p, sizeof(T), n, f) != n) { fprintf(stderr, "short read\n"); exit(2); }
}

int main(int argc, char **argv) {
  if (argc != 3) return 2;
  FILE *f = fopen(argv[1], "rb");
  int hdr[5];
  rd(f, hdr, 5);
  const int nx = hdr[0], ny = hdr[1], nz = hdr[2], ncalls = hdr[3], cycles = hdr[4];
  double g[10];
  rd(f, g, 10);
  const size_t N = size_t(nx) * ny * nz;
  std::vector<double> u(N), v(N);
  rd(f, u.data(), N);
  rd(f, v.data(), N);
  fclose(f);

  core::Coupler coupler(nx, ny, nz, g[0], g[1], g[2]);
  const char *on[4] = {"R_d", "gamma_d", "C0", "grav"};
  const double ov[4] = {287., 1003. / 716., 27.56, 9.81};
  for (int q = 0; q < 4; q++) coupler.set_option<real>(on[q], ov[q]);
  auto &dm = coupler.get_data_manager_readwrite();
  for (auto nm : {"density_dry", "uvel", "vvel", "wvel", "temp"}) dm.register_and_allocate<real>(nm, "", {nz, ny, nx});
  std::copy(u.begin(), u.end(), dm.get<real, 3>("uvel").data());
  std::copy(v.begin(), v.end(), dm.get<real, 3>("vvel").data());
  custom_modules::EdgeSponge edge_sponge;
  edge_sponge.set_column(coupler);
  for (int c = 0; c < ncalls; c++) {
    modules::uniform_pg_wind_forcing(coupler, g[3], g[4], size_t(cycles));
    auto uu = dm.get<real, 3>("uvel");
    for (size_t q = 0; q < N; q++) uu.data()[q] += 0.25;
  }
  const std::string pre = "uniform_pg_wind_forcing_";
  const double st[5] = {double(coupler.get_option<size_t>(pre + "counter")), coupler.get_option<real>(pre + "u0"),
                        coupler.get_option<real>(pre + "v0"), coupler.get_option<real>(pre + "u"),
                        coupler.get_option<real>(pre + "v")};
  modules::uniform_pg_wind_forcing_height(coupler, g[3], g[5], g[6], g[7], g[8]);
  FILE *o = fopen(argv[2], "wb");
  fwrite(dm.get<real, 3>("uvel").data(), sizeof(double), N, o);
  fwrite(dm.get<real, 3>("vvel").data(), sizeof(double), N, o);
  fwrite(st, sizeof(double), 5, o);
  edge_sponge.apply(coupler, 0.2, 0.1, 0.15, 0.25);
  for (auto nm : {"density_dry", "uvel", "vvel", "wvel", "temp"}) fwrite(dm.get<real, 3>(nm).data(), sizeof(double), N, o);
  fclose(o);
  modules::pu_physics_module_finalize(coupler);
  printf("pg driver ok\n");
  return 0;
}
