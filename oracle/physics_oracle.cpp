// CPU restatement of the physics modules that run beside the dycore in the
// boundary-layer drivers (TEST INFRASTRUCTURE ONLY: the oracle that the GPU
// kernels of porturb_b200/csrc/physics.cu are checked against).
//
// Follows, file:line in the reference's model/modules/:
//   LES_Closure::apply                les_closure.h:30-320
//     conversions                     les_closure.h:326-407
//     halo_bcs                        les_closure.h:411-532
//   sponge_layer                      sponge_layer.h:7-62
//   geostrophic_wind_forcing          geostrophic_wind_forcing.h:7-42
//   apply_surface_fluxes              surface_flux.h:9-125
//   uniform_pg_wind_forcing           uniform_pg_wind_forcing.h:6-40
//   uniform_pg_wind_forcing_height    uniform_pg_wind_forcing.h:43-82
//   Time_Averager::accumulate         experiments/examples/custom_modules/time_averager.h:56-110
//   EdgeSponge::set_column / apply    experiments/examples/custom_modules/edge_sponge.h:14-72
// The arithmetic of each quantity is evaluated in the reference's order
// (the build uses -ffp-contract=off), so the restatement is compared with the
// reference's own modules bit for bit in the tests.  The code is organised
// differently: one face-flux routine serves the three directions.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "physics_api.h"

namespace {

struct Phys {
  orc_phys_config c;
  std::vector<double> prop, rough, temp;   // (nz+2, ny+2, nx+2)
  size_t hidx(int k, int j, int i) const { return (size_t(k) * (c.ny + 2) + j) * (c.nx + 2) + i; }
};

// Padded field with one halo cell on each side.
struct Pad {
  int nz, ny, nx;
  std::vector<double> a;
  Pad(int z, int y, int x) : nz(z), ny(y), nx(x), a(size_t(z + 2) * (y + 2) * (x + 2)) {}
  double &operator()(int k, int j, int i) { return a[(size_t(k) * (ny + 2) + j) * (nx + 2) + i]; }
};

// ---------------------------------------------------------------------------
// LES closure.
// ---------------------------------------------------------------------------
constexpr int R = 0, U = 1, V = 2, W = 3, T = 4;

struct LesFields {
  std::vector<Pad> s;   // R, U, V, W, T (theta), then K, then diffused tracers
  int nd;               // number of diffused tracers
  Pad &K() { return s[5]; }
  Pad &q(int t) { return s[6 + t]; }
};

// Periodic x then y wrap of interior levels (corners wrap in both), then the
// closure's own boundary conditions (les_closure.h:411-532).
void les_halos(const orc_phys_config &c, LesFields &f) {
  const int nx = c.nx, ny = c.ny, nz = c.nz;
  const double grav = c.enable_gravity ? c.grav : 0.0, gamma = c.gamma_d, C0 = c.C0, dz = c.zlen / nz;
  for (auto &p : f.s) {
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++) {
        p(k, j, 0) = p(k, j, nx);
        p(k, j, nx + 1) = p(k, j, 1);
      }
    for (int k = 1; k <= nz; k++)
      for (int i = 0; i < nx + 2; i++) {
        p(k, 0, i) = p(k, ny, i);
        p(k, ny + 1, i) = p(k, 1, i);
      }
  }
  // Precursor x / y: the edge value replicated into the halo (interior rows).
  // Rho is replicated as well; the z pass below then covers every column.
  for (auto &p : f.s) {
    if (c.bc_x == 1)
      for (int k = 1; k <= nz; k++)
        for (int j = 1; j <= ny; j++) {
          p(k, j, 0) = p(k, j, 1);
          p(k, j, nx + 1) = p(k, j, nx);
        }
    if (c.bc_y == 1)
      for (int k = 1; k <= nz; k++)
        for (int i = 1; i <= nx; i++) {
          p(k, 0, i) = p(k, 1, i);
          p(k, ny + 1, i) = p(k, ny, i);
        }
  }
  if (c.bc_z == 2) {
    for (int j = 0; j < ny + 2; j++)
      for (int i = 0; i < nx + 2; i++) {
        for (int v = 0; v < int(f.s.size()); v++) {
          if (v == R) continue;
          Pad &p = f.s[v];
          p(0, j, i) = v == W ? 0.0 : p(1, j, i);
          p(nz + 1, j, i) = v == W ? 0.0 : p(nz, j, i);
        }
        // Isentropic extrapolation of rho into the halo (kk = 0 of hs = 1).
        {
          const double rho0 = f.s[R](1, j, i), theta0 = f.s[T](1, j, i);
          const double rho0_gm1 = std::pow(rho0, gamma - 1), theta0_g = std::pow(theta0, gamma);
          f.s[R](0, j, i) = std::pow(rho0_gm1 + grav * (gamma - 1) * dz * (0 + 1) / (gamma * C0 * theta0_g), 1. / (gamma - 1));
        }
        {
          const double rho0 = f.s[R](nz, j, i), theta0 = f.s[T](nz, j, i);
          const double rho0_gm1 = std::pow(rho0, gamma - 1), theta0_g = std::pow(theta0, gamma);
          f.s[R](nz + 1, j, i) = std::pow(rho0_gm1 - grav * (gamma - 1) * dz * (0 + 1) / (gamma * C0 * theta0_g), 1. / (gamma - 1));
        }
      }
  } else {
    for (auto &p : f.s)
      for (int j = 0; j < ny + 2; j++)
        for (int i = 0; i < nx + 2; i++) {
          p(0, j, i) = p(nz, j, i);
          p(nz + 1, j, i) = p(1, j, i);
        }
  }
}

struct Coef {
  double delta, nu, total_mult, grav;
  bool gravity, dns;
};

// Mixing length, eddy viscosity, turbulent Prandtl number at a face or cell
// (les_closure.h:122-127).
inline void eddy(const Coef &q, double K, double t, double dt_dz, double mult, double &ell, double &km, double &Pr_t) {
  const double N = dt_dz >= 0 && q.gravity ? std::sqrt(q.grav / t * dt_dz) : 0;
  ell = std::min(0.76 * std::sqrt(K) / (N + 1.e-20), q.delta);
  km = mult * 0.1 * ell * std::sqrt(K);
  Pr_t = q.delta / (1 + 2 * ell);
}

// Diffusive fluxes through the face between cell A = (k,j,i) - e_dir and
// cell B = (k,j,i) (les_closure.h:87-232).  out: rho*u, rho*v, rho*w,
// rho*theta, TKE, then the diffused tracers.
void face_flux(const Phys &P, const Coef &q, LesFields &f, int dir, int k, int j, int i, double visc_max, double *out) {
  const double d[3] = {P.c.xlen / P.c.nx, P.c.ylen / P.c.ny, P.c.zlen / P.c.nz};
  const int off[3][3] = {{0, 0, 1}, {0, 1, 0}, {1, 0, 0}};   // (dk, dj, di) of a step along x, y, z
  const int ka = k - off[dir][0], ja = j - off[dir][1], ia = i - off[dir][2];
  const int nf = 5 + 1 + f.nd;
  if (P.prop[P.hidx(ka, ja, ia)] == 1 || P.prop[P.hidx(k, j, i)] == 1) {
    for (int v = 0; v < nf; v++) out[v] = 0;
    return;
  }
  // g[c][e]: derivative of velocity component c along direction e at the face.
  double g[3][3];
  auto normal = [&](Pad &p) { return (p(k, j, i) - p(ka, ja, ia)) / d[dir]; };
  auto tang = [&](Pad &p, int e) {
    const int dk = off[e][0], dj = off[e][1], di = off[e][2];
    return 0.5 * ((p(ka + dk, ja + dj, ia + di) - p(ka - dk, ja - dj, ia - di)) / (2 * d[e]) +
                  (p(k + dk, j + dj, i + di) - p(k - dk, j - dj, i - di)) / (2 * d[e]));
  };
  for (int c = 0; c < 3; c++) {
    g[c][dir] = normal(f.s[U + c]);
    for (int e = 0; e < 3; e++)
      if (e != dir && (c == e || c == dir)) g[c][e] = tang(f.s[U + c], e);
  }
  const double dt_dz = dir == 2 ? normal(f.s[T]) : tang(f.s[T], 2);
  const double rho = 0.5 * (f.s[R](ka, ja, ia) + f.s[R](k, j, i));
  const double K = 0.5 * (f.K()(ka, ja, ia) + f.K()(k, j, i));
  const double t = 0.5 * (f.s[T](ka, ja, ia) + f.s[T](k, j, i));
  double ell, km, Pr_t;
  eddy(q, K, t, dt_dz, q.total_mult, ell, km, Pr_t);
  constexpr double Pr = 0.7;
  const double visc_tot = q.dns ? q.nu : std::min(km + q.nu, 0.5 * visc_max);
  const double visc_tot_th = q.dns ? q.nu : std::min(km / Pr_t + q.nu / Pr, 0.5 * visc_max);
  const double div = g[0][0] + g[1][1] + g[2][2];
  for (int c = 0; c < 3; c++) {
    if (c == dir) out[c] = -rho * visc_tot * (g[c][c] + g[c][c] - 2. / 3. * div);
    else out[c] = -rho * visc_tot * (g[c][dir] + g[dir][c]);
  }
  out[3] = -rho * visc_tot_th * (normal(f.s[T]));
  out[4] = -rho * visc_tot * 2 * (normal(f.K()));
  for (int tr = 0; tr < f.nd; tr++) out[5 + tr] = -rho * visc_tot * normal(f.q(tr));
}

// Cell-centred TKE source: buoyancy, dissipation, shear production
// (les_closure.h:236-282).
double tke_source(const Phys &P, const Coef &q, LesFields &f, int k, int j, int i) {
  const double dx = P.c.xlen / P.c.nx, dy = P.c.ylen / P.c.ny, dz = P.c.zlen / P.c.nz;
  const double rho = f.s[R](k, j, i), K = f.K()(k, j, i), t = f.s[T](k, j, i);
  const double dt_dz = (f.s[T](k + 1, j, i) - f.s[T](k - 1, j, i)) / (2 * dz);
  double ell, km, Pr_t;
  eddy(q, K, t, dt_dz, 1.0, ell, km, Pr_t);
  double src = 0;
  auto imm = [&](int kk, int jj, int ii) { return P.prop[P.hidx(kk, jj, ii)]; };
  if (imm(k, j, i) < 1) {
    if (q.gravity) src += -(q.grav * rho * km) / (t * Pr_t) * dt_dz;
    src -= P.c.les_dissipation_mult * rho * (0.19 + 0.51 * ell / q.delta) / q.delta * std::pow(K, 1.5);
    // Neighbours inside immersed material are replaced by the cell itself,
    // except along a component's own direction.
    const int im1 = imm(k, j, i - 1) > 0 ? i : i - 1, ip1 = imm(k, j, i + 1) > 0 ? i : i + 1;
    const int jm1 = imm(k, j - 1, i) > 0 ? j : j - 1, jp1 = imm(k, j + 1, i) > 0 ? j : j + 1;
    const int km1 = imm(k - 1, j, i) > 0 ? k : k - 1, kp1 = imm(k + 1, j, i) > 0 ? k : k + 1;
    Pad &u = f.s[U], &v = f.s[V], &w = f.s[W];
    double g[3][3];   // g[e][c]: derivative of component c along direction e
    g[0][0] = (u(k, j, i + 1) - u(k, j, i - 1)) / (2 * dx);
    g[0][1] = (v(k, j, ip1) - v(k, j, im1)) / (2 * dx);
    g[0][2] = (w(k, j, ip1) - w(k, j, im1)) / (2 * dx);
    g[1][0] = (u(k, jp1, i) - u(k, jm1, i)) / (2 * dy);
    g[1][1] = (v(k, j + 1, i) - v(k, j - 1, i)) / (2 * dy);
    g[1][2] = (w(k, jp1, i) - w(k, jm1, i)) / (2 * dy);
    g[2][0] = (u(kp1, j, i) - u(km1, j, i)) / (2 * dz);
    g[2][1] = (v(kp1, j, i) - v(km1, j, i)) / (2 * dz);
    g[2][2] = (w(k + 1, j, i) - w(k - 1, j, i)) / (2 * dz);
    double sum = 0;
    bool first = true;
    for (int e = 0; e < 3; e++)
      for (int c = 0; c < 3; c++) {
        const double term = (g[e][c] + g[c][e]) * g[e][c];
        sum = first ? term : sum + term;
        first = false;
      }
    src += P.c.les_shear_prod_mult * rho * km * sum;
  }
  return src;
}

void les_apply(Phys &P, double *rho_d, double *uu, double *vv, double *ww, double *TT, double *trc, double dtphys) {
  const orc_phys_config &c = P.c;
  const int nx = c.nx, ny = c.ny, nz = c.nz;
  const size_t N = size_t(nx) * ny * nz;
  const double dx = c.xlen / nx, dy = c.ylen / ny, dz = c.zlen / nz;
  std::vector<int> diffused;
  for (int t = 0; t < c.ntr; t++)
    if (c.tracer_diffuse[t]) diffused.push_back(t);
  LesFields f;
  f.nd = int(diffused.size());
  for (int v = 0; v < 6 + f.nd; v++) f.s.emplace_back(nz, ny, nx);
  // Coupler -> closure state (les_closure.h:326-365).
#pragma omp parallel for collapse(2)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        const size_t q = (size_t(k) * ny + j) * nx + i;
        const double rd = rho_d[q];
        f.s[R](k + 1, j + 1, i + 1) = rd;
        f.s[U](k + 1, j + 1, i + 1) = uu[q];
        f.s[V](k + 1, j + 1, i + 1) = vv[q];
        f.s[W](k + 1, j + 1, i + 1) = ww[q];
        f.s[T](k + 1, j + 1, i + 1) = std::pow(rd * c.R_d * TT[q] / c.C0, 1. / c.gamma_d) / rd;
        f.K()(k + 1, j + 1, i + 1) = std::max(0., trc[size_t(c.idTKE) * N + q] / rd);
        for (int t = 0; t < f.nd; t++) f.q(t)(k + 1, j + 1, i + 1) = trc[size_t(diffused[t]) * N + q] / rd;
      }
  les_halos(c, f);
  Coef q;
  q.delta = std::pow(dx * dy * dz, 1. / 3.);
  q.nu = c.kinematic_viscosity;
  q.total_mult = c.les_total_mult;
  q.grav = c.grav;
  q.gravity = c.enable_gravity != 0;
  q.dns = c.dns != 0;
  const double vmax[3] = {0.25 * dx * dx / dtphys, 0.25 * dy * dy / dtphys, 0.25 * dz * dz / dtphys};
  const int nf = 6 + f.nd;
  // Face fluxes: fx(k,j,i) on the face at i-1/2, i = 0..nx, etc.
  std::vector<double> fx(size_t(nf) * nz * ny * (nx + 1)), fy(size_t(nf) * nz * (ny + 1) * nx),
      fz(size_t(nf) * (nz + 1) * ny * nx);
#pragma omp parallel for collapse(2)
  for (int k = 0; k <= nz; k++)
    for (int j = 0; j <= ny; j++)
      for (int i = 0; i <= nx; i++) {
        double out[32];
        if (j < ny && k < nz) {
          face_flux(P, q, f, 0, k + 1, j + 1, i + 1, vmax[0], out);
          for (int v = 0; v < nf; v++) fx[((size_t(v) * nz + k) * ny + j) * (nx + 1) + i] = out[v];
        }
        if (i < nx && k < nz) {
          face_flux(P, q, f, 1, k + 1, j + 1, i + 1, vmax[1], out);
          for (int v = 0; v < nf; v++) fy[((size_t(v) * nz + k) * (ny + 1) + j) * nx + i] = out[v];
        }
        if (i < nx && j < ny) {
          face_flux(P, q, f, 2, k + 1, j + 1, i + 1, vmax[2], out);
          for (int v = 0; v < nf; v++) fz[((size_t(v) * (nz + 1) + k) * ny + j) * nx + i] = out[v];
        }
      }
  // Divergence, sources and the update (les_closure.h:285-319), then back
  // to the coupler (les_closure.h:371-407).
#pragma omp parallel for collapse(2)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        auto FX = [&](int v, int ii) { return fx[((size_t(v) * nz + k) * ny + j) * (nx + 1) + ii]; };
        auto FY = [&](int v, int jj) { return fy[((size_t(v) * nz + k) * (ny + 1) + jj) * nx + i]; };
        auto FZ = [&](int v, int kk) { return fz[((size_t(v) * (nz + 1) + kk) * ny + j) * nx + i]; };
        auto tend = [&](int v) {
          return -(FX(v, i + 1) - FX(v, i)) / dx - (FY(v, j + 1) - FY(v, j)) / dy - (FZ(v, k + 1) - FZ(v, k)) / dz;
        };
        const size_t qc = (size_t(k) * ny + j) * nx + i;
        const double rho = f.s[R](k + 1, j + 1, i + 1);
        const double src = tke_source(P, q, f, k + 1, j + 1, i + 1);
        double ru = f.s[U](k + 1, j + 1, i + 1) * rho + dtphys * tend(0);
        double rv = f.s[V](k + 1, j + 1, i + 1) * rho + dtphys * tend(1);
        double rw = f.s[W](k + 1, j + 1, i + 1) * rho + dtphys * tend(2);
        double rt = f.s[T](k + 1, j + 1, i + 1) * rho + dtphys * tend(3);
        double rk = f.K()(k + 1, j + 1, i + 1) * rho + dtphys * (tend(4) + src);
        rk = std::max(0., rk);
        uu[qc] = ru / rho;
        vv[qc] = rv / rho;
        ww[qc] = rw / rho;
        TT[qc] = c.C0 * std::pow(rt, c.gamma_d) / (rho * c.R_d);
        trc[size_t(c.idTKE) * N + qc] = rk;
        for (int t = 0; t < f.nd; t++)
          trc[size_t(diffused[t]) * N + qc] = f.q(t)(k + 1, j + 1, i + 1) * rho + dtphys * tend(5 + t);
      }
}

// Horizontal means of the given fields per level, each term scaled by
// 1/(nx*ny) before it is added, summed j-major then i as the reference does
// (sponge_layer.h:36-47, geostrophic_wind_forcing.h:21-30).
double level_mean(const orc_phys_config &c, const double *a, int k) {
  const double r = 1. / (double(c.nx) * c.ny);
  double s = 0;
  for (int j = 0; j < c.ny; j++)
    for (int i = 0; i < c.nx; i++) s += a[(size_t(k) * c.ny + j) * c.nx + i] * r;
  return s;
}

}  // namespace

extern "C" {

void *orc_phys_create(const orc_phys_config *cfg, const double *imm_prop_h, const double *imm_rough_h,
                      const double *imm_temp_h) {
  Phys *p = new Phys;
  p->c = *cfg;
  const size_t nh = size_t(cfg->nz + 2) * (cfg->ny + 2) * (cfg->nx + 2);
  p->prop.assign(imm_prop_h, imm_prop_h + nh);
  p->rough.assign(imm_rough_h, imm_rough_h + nh);
  p->temp.assign(imm_temp_h, imm_temp_h + nh);
  return p;
}

void orc_phys_destroy(void *h) { delete static_cast<Phys *>(h); }

int orc_phys_les(void *h, double *rho_d, double *u, double *v, double *w, double *T, double *trc, double dt) {
  les_apply(*static_cast<Phys *>(h), rho_d, u, v, w, T, trc, dt);
  return 0;
}

// sponge_layer (sponge_layer.h:7-62): relax u, v, T toward their level means
// and w toward 0 with weight ((z-z1)/(z2-z1))^3 dt/time_scale above z1.
int orc_phys_sponge(void *h, double *, double *u, double *v, double *w, double *T, double *, double dt,
                    double time_scale, double top_prop) {
  const orc_phys_config &c = static_cast<Phys *>(h)->c;
  const double dz = c.zlen / c.nz, z1 = (1 - top_prop) * c.zlen, z2 = c.zlen;
  const int k1 = int(std::floor(z1 / dz - 0.5));
  for (int k = k1; k < c.nz; k++) {
    const double mu = level_mean(c, u, k), mv = level_mean(c, v, k), mT = level_mean(c, T, k);
    const double z = (k + 0.5) * dz;
    if (!(z > z1)) continue;
    const double factor = std::pow((z - z1) / (z2 - z1), 3.0) * dt / time_scale;
    for (size_t q = size_t(k) * c.ny * c.nx; q < size_t(k + 1) * c.ny * c.nx; q++) {
      u[q] = factor * mu + (1 - factor) * u[q];
      v[q] = factor * mv + (1 - factor) * v[q];
      w[q] = factor * 0 + (1 - factor) * w[q];
      T[q] = factor * mT + (1 - factor) * T[q];
    }
  }
  return 0;
}

// geostrophic_wind_forcing (geostrophic_wind_forcing.h:7-42): Coriolis
// acceleration of the level-mean wind's departure from (u_g, v_g).
int orc_phys_geostrophic(void *h, double *, double *u, double *v, double *, double *, double *, double dt,
                         double lat_g, double u_g, double v_g) {
  const orc_phys_config &c = static_cast<Phys *>(h)->c;
  const double fcor = 2 * 7.2921e-5 * std::sin(lat_g / 180 * M_PI);
  for (int k = 0; k < c.nz; k++) {
    const double mu = level_mean(c, u, k), mv = level_mean(c, v, k);
    for (size_t q = size_t(k) * c.ny * c.nx; q < size_t(k + 1) * c.ny * c.nx; q++) {
      u[q] += dt * (fcor * (mv - v_g));
      v[q] += dt * (-fcor * (mu - u_g));
    }
  }
  return 0;
}

// apply_surface_fluxes (surface_flux.h:9-125): log-law drag (and heat flux
// where the immersed temperature is set) from each immersed face neighbour.
int orc_phys_surface_fluxes(void *h, double *, double *u, double *v, double *w, double *T, double *, double dt) {
  const Phys &P = *static_cast<Phys *>(h);
  const orc_phys_config &c = P.c;
  const double d[3] = {c.xlen / c.nx, c.ylen / c.ny, c.zlen / c.nz};
  const double vk = 0.40;
  const size_t N = size_t(c.nx) * c.ny * c.nz;
  std::vector<double> tu(N), tv(N), tw(N), tT(N);
#pragma omp parallel for collapse(2)
  for (int k = 0; k < c.nz; k++)
    for (int j = 0; j < c.ny; j++)
      for (int i = 0; i < c.nx; i++) {
        const size_t q = (size_t(k) * c.ny + j) * c.nx + i;
        const double vel[3] = {u[q], v[q], w[q]}, Tc = T[q];
        double tend[3] = {0, 0, 0}, tendT = 0;
        // Neighbours in the order x-, x+, y-, y+, z-, z+.
        const int nb[6][3] = {{0, 0, -1}, {0, 0, 1}, {0, -1, 0}, {0, 1, 0}, {-1, 0, 0}, {1, 0, 0}};
        for (int n = 0; n < 6; n++) {
          const int dir = n / 2;   // 0: x, 1: y, 2: z
          const size_t hq = P.hidx(k + 1 + nb[n][0], j + 1 + nb[n][1], i + 1 + nb[n][2]);
          if (!(P.prop[hq] > 0)) continue;
          const double roughness = P.rough[hq];
          const double lg = std::log((d[dir] / 2 + roughness) / roughness);
          const double cd = vk * vk / (lg * lg);
          const double T0 = P.temp[hq];
          const int a = dir == 0 ? 1 : 0, b = dir == 2 ? 1 : 2;   // the two tangential components
          const double mag = std::sqrt(vel[a] * vel[a] + vel[b] * vel[b]);
          tend[a] += -cd * (vel[a] - 0) * mag / d[dir];
          tend[b] += -cd * (vel[b] - 0) * mag / d[dir];
          if (T0 != 0) tendT += -cd * (Tc - T0) * mag / d[dir];
        }
        tu[q] = tend[0];
        tv[q] = tend[1];
        tw[q] = tend[2];
        tT[q] = tendT;
      }
  for (size_t q = 0; q < N; q++) {
    u[q] += dt * tu[q];
    v[q] += dt * tv[q];
    w[q] += dt * tw[q];
    T[q] += dt * tT[q];
  }
  return 0;
}

// uniform_pg_wind_forcing (uniform_pg_wind_forcing.h:6-40): every
// update_cycles calls the domain means of u and v (sums in memory order over
// all cells, divided by the cell count); u += dt/tau*(u0-u), likewise v.
int orc_phys_uniform_pg(void *h, double *, double *u, double *v, double *, double *, double *, double dt, double tau,
                        unsigned long long update_cycles, double *st) {
  const orc_phys_config &c = static_cast<Phys *>(h)->c;
  if (update_cycles == 0) return 1;
  const size_t n = size_t(c.nz) * c.ny * c.nx;
  const unsigned long long counter = (unsigned long long)st[0];
  if (counter % update_cycles == 0) {
    double su = 0, sv = 0;
    for (size_t q = 0; q < n; q++) su += u[q];
    for (size_t q = 0; q < n; q++) sv += v[q];
    st[3] = su / double(n);
    st[4] = sv / double(n);
    if (counter == 0) {
      st[1] = st[3];
      st[2] = st[4];
    }
  }
  const double fu = dt / tau * (st[1] - st[3]), fv = dt / tau * (st[2] - st[4]);
  for (size_t q = 0; q < n; q++) {
    u[q] += fu;
    v[q] += fv;
  }
  st[0] = double(counter + 1);
  return 0;
}

// uniform_pg_wind_forcing_height (uniform_pg_wind_forcing.h:43-82): level
// means of the two levels whose centres bracket `height`, linear in z
// between them.  Returns 1 where the reference would read outside the levels.
int orc_phys_uniform_pg_height(void *h, double *, double *u, double *v, double *, double *, double *, double dt,
                               double height, double u0, double v0, double tau) {
  const orc_phys_config &c = static_cast<Phys *>(h)->c;
  const double dz = c.zlen / c.nz;
  int k1 = 0;
  for (int k = 0; k < c.nz; k++)
    if ((k + 0.5) * dz > height) {
      k1 = k - 1;
      break;
    }
  if (k1 < 0 || k1 + 1 >= c.nz) return 1;
  const size_t nl = size_t(c.ny) * c.nx;
  double m[2][2];
  for (int l = 0; l < 2; l++) {
    double su = 0, sv = 0;
    for (size_t q = (k1 + l) * nl; q < (k1 + l + 1) * nl; q++) su += u[q];
    for (size_t q = (k1 + l) * nl; q < (k1 + l + 1) * nl; q++) sv += v[q];
    m[l][0] = su / double(nl);
    m[l][1] = sv / double(nl);
  }
  const double z1 = (k1 + 0.5) * dz, z2 = (k1 + 1.5) * dz;
  const double w1 = (z2 - height) / dz, w2 = (height - z1) / dz;
  const double um = w1 * m[0][0] + w2 * m[1][0], vm = w1 * m[0][1] + w2 * m[1][1];
  const double fu = dt / tau * (u0 - um), fv = dt / tau * (v0 - vm);
  const size_t n = nl * c.nz;
  for (size_t q = 0; q < n; q++) {
    u[q] += fu;
    v[q] += fv;
  }
  return 0;
}

// Time_Averager::accumulate (time_averager.h:56-110): exponential running
// averages with inertia etime/(etime+dt) (long ones: elapsed/(elapsed+dt)),
// the covariances of the departures from the updated long averages.
int orc_phys_time_average(void *h, double *, double *u, double *v, double *w, double *, double *trc, double *avgs,
                          double *etime, double elapsed_time, double dt) {
  const orc_phys_config &c = static_cast<Phys *>(h)->c;
  if (c.idTKE < 0) return 1;
  const size_t n = size_t(c.nz) * c.ny * c.nx;
  const double *tke = trc + size_t(c.idTKE) * n;
  double *a[13];
  for (int q = 0; q < 13; q++) a[q] = avgs + size_t(q) * n;
  const double inertia = *etime / (*etime + dt), inertia_long = elapsed_time / (elapsed_time + dt);
  for (size_t e = 0; e < n; e++) {
    a[10][e] = inertia_long * a[10][e] + (1 - inertia_long) * u[e];
    a[11][e] = inertia_long * a[11][e] + (1 - inertia_long) * v[e];
    a[12][e] = inertia_long * a[12][e] + (1 - inertia_long) * w[e];
    const double up = u[e] - a[10][e], vp = v[e] - a[11][e], wp = w[e] - a[12][e];
    a[0][e] = inertia * a[0][e] + (1 - inertia) * u[e];
    a[1][e] = inertia * a[1][e] + (1 - inertia) * v[e];
    a[2][e] = inertia * a[2][e] + (1 - inertia) * w[e];
    a[3][e] = inertia * a[3][e] + (1 - inertia) * tke[e];
    a[4][e] = inertia * a[4][e] + (1 - inertia) * up * up;
    a[5][e] = inertia * a[5][e] + (1 - inertia) * up * vp;
    a[6][e] = inertia * a[6][e] + (1 - inertia) * up * wp;
    a[7][e] = inertia * a[7][e] + (1 - inertia) * vp * vp;
    a[8][e] = inertia * a[8][e] + (1 - inertia) * vp * wp;
    a[9][e] = inertia * a[9][e] + (1 - inertia) * wp * wp;
  }
  *etime = *etime + dt;
  return 0;
}

// EdgeSponge::set_column (edge_sponge.h:14-28, 75-96): per field and level
// the sum over the level in (j, i) order, divided by nx*ny.
int orc_phys_edge_sponge_set_column(void *h, double *rho_d, double *u, double *v, double *w, double *T, double *,
                                    double *column) {
  const orc_phys_config &c = static_cast<Phys *>(h)->c;
  const double *f[5] = {rho_d, u, v, w, T};
  const size_t nl = size_t(c.ny) * c.nx;
  for (int l = 0; l < 5; l++)
    for (int k = 0; k < c.nz; k++) {
      double s = 0;
      for (size_t q = 0; q < nl; q++) s += f[l][size_t(k) * nl + q];
      column[size_t(l) * c.nz + k] = s / (c.nx * c.ny);
    }
  return 0;
}

// EdgeSponge::apply (edge_sponge.h:31-72): the four edge zones in turn, each
// blending toward the column profile with weight ((p1-p)/p1)^5.
int orc_phys_edge_sponge_apply(void *h, double *rho_d, double *u, double *v, double *w, double *T, double *,
                               const double *column, double px1, double px2, double py1, double py2) {
  const orc_phys_config &c = static_cast<Phys *>(h)->c;
  double *f[5] = {rho_d, u, v, w, T};
  const float pwr = 5;
  for (int l = 0; l < 5; l++)
    for (int k = 0; k < c.nz; k++)
      for (int j = 0; j < c.ny; j++)
        for (int i = 0; i < c.nx; i++) {
          double &x = f[l][(size_t(k) * c.ny + j) * c.nx + i];
          const double col = column[size_t(l) * c.nz + k];
          const double prop_x = double(i) / c.nx, prop_y = double(j) / c.ny;
          if (px1 > 0 && prop_x <= px1) {
            const double wt = std::pow((px1 - prop_x) / px1, pwr);
            x = wt * col + (1 - wt) * x;
          }
          if (px2 > 0 && prop_x >= 1 - px2) {
            const double wt = std::pow((prop_x - (1 - px2)) / px2, pwr);
            x = wt * col + (1 - wt) * x;
          }
          if (py1 > 0 && prop_y <= py1) {
            const double wt = std::pow((py1 - prop_y) / py1, pwr);
            x = wt * col + (1 - wt) * x;
          }
          if (py2 > 0 && prop_y >= 1 - py2) {
            const double wt = std::pow((prop_y - (1 - py2)) / py2, pwr);
            x = wt * col + (1 - wt) * x;
          }
        }
  return 0;
}

}  // extern "C"
