// Driver of the C++ drop-in module, written like the reference's example
// drivers (abl_neutral.cpp:49-119): a coupler with options, grid, tracers and
// state; dycore.init(coupler); dycore.time_step(coupler, dt).  The coupler is
// the single-rank stand-in of oracle/ref_shim; the module is
// porturb_b200/cpp/dynamics_rk.h on libpu_dycore.so.
//
// Usage: dropin_driver <input.bin> <output.bin>
//   input : int32 nx, ny, nz, ntr, ncalls; float64 xlen, ylen, zlen, dt_phys,
//           R_d, R_v, cp_d, gamma_d, C0, grav, cfl; int32 idWV, positive[ntr],
//           adds_mass[ntr]; float64 base (5+ntr)*N, pert (5+ntr)*N
//   output: float64 (5+ntr)*N after ncalls time_step calls
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "dynamics_rk.h"

template <class T>
static void rd(FILE *f, T *p, size_t n) {
  if (fread(p, sizeof(T), n, f) != n) { fprintf(stderr, "short read\n"); exit(2); }
}

int main(int argc, char **argv) {
  if (argc != 3) return 2;
  FILE *f = fopen(argv[1], "rb");
  int hdr[5];
  rd(f, hdr, 5);
  const int nx = hdr[0], ny = hdr[1], nz = hdr[2], ntr = hdr[3], ncalls = hdr[4];
  double g[11];
  rd(f, g, 11);
  int idWV;
  rd(f, &idWV, 1);
  std::vector<int> pos(ntr), am(ntr);
  rd(f, pos.data(), ntr);
  rd(f, am.data(), ntr);
  const size_t N = size_t(nx) * ny * nz;
  std::vector<double> base((5 + ntr) * N), pert((5 + ntr) * N);
  rd(f, base.data(), base.size());
  rd(f, pert.data(), pert.size());
  fclose(f);

  core::Coupler coupler(nx, ny, nz, g[0], g[1], g[2]);
  const char *on[7] = {"R_d", "R_v", "cp_d", "gamma_d", "C0", "grav", "cfl"};
  for (int q = 0; q < 7; q++) coupler.set_option<real>(on[q], g[4 + q]);
  coupler.set_option<int>("idWV", idWV);
  coupler.set_option<std::string>("bc_x", "periodic");
  coupler.set_option<std::string>("bc_y", "periodic");
  coupler.set_option<std::string>("bc_z", "solid_wall");
  auto &dm = coupler.get_data_manager_readwrite();
  const char *sn[5] = {"density_dry", "uvel", "vvel", "wvel", "temp"};
  for (auto nm : sn) dm.register_and_allocate<real>(nm, "", {nz, ny, nx});
  for (int t = 0; t < ntr; t++) {
    char name[32];
    snprintf(name, sizeof(name), t == idWV ? "water_vapor" : "tracer_%d", t);
    coupler.add_tracer(name, name, pos[t] != 0, am[t] != 0, true);
  }
  auto names = coupler.get_tracer_names();
  auto load = [&](const std::vector<double> &src) {
    for (int a = 0; a < 5 + ntr; a++) {
      double *dst = a < 5 ? dm.get<real, 3>(sn[a]).data() : dm.get<real, 3>(names[a - 5]).data();
      std::copy(src.begin() + a * N, src.begin() + (a + 1) * N, dst);
    }
  };
  modules::Dynamics_Euler_Stratified_WenoFV dycore;
  load(base);
  dycore.init(coupler);
  load(pert);
  for (int c = 0; c < ncalls; c++) dycore.time_step(coupler, g[3]);
  FILE *o = fopen(argv[2], "wb");
  for (int a = 0; a < 5 + ntr; a++) {
    const double *src = a < 5 ? dm.get<real, 3>(sn[a]).data() : dm.get<real, 3>(names[a - 5]).data();
    fwrite(src, sizeof(double), N, o);
  }
  fclose(o);
  dycore.finalize(coupler);
  printf("dropin ok\n");
  return 0;
}
