// B200 kernels and C entry points of the physics modules of include/pu_physics.h:
// the LES closure, sponge layer, geostrophic forcing and surface fluxes that
// the boundary-layer drivers run beside the dycore (FP64, as the reference).
//
// k_les: one 32x8 column tile per block marches up a chunk of levels with a
// 3-plane ring of the closure's primitive fields (rho_d, u, v, w, theta, K,
// diffused tracer ratios) and immersed flags in shared memory; each level's
// x and y face fluxes are computed once per face into shared memory, the
// z face flux of a column is carried to the next level in registers; the
// TKE source and the update are fused; the result goes to a separate output
// (neighbouring blocks still read the input).
// k_level_partial / k_level_final: deterministic level means (Neumaier-
// compensated FP64 sums in a fixed order) for the sponge and the
// geostrophic forcing and the pressure-gradient wind forcings; k_sponge /
// k_geostrophic / k_surface_fluxes / k_add_uv / k_pg_height /
// k_time_average / k_edge_sponge are pointwise updates in place.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/pu_physics.h"

namespace pu {
void set_error(const std::string &msg);

namespace phys {

constexpr int TX = 32, TY = 8, NT = TX * TY;
constexpr int HX = TX + 2, HY = TY + 2, HP = HX * HY;   // tile plus one halo cell per side
constexpr int KC = 16;                                  // levels per block
constexpr int BC_PRECURSOR = 1, BC_WALL = 2;
constexpr uint8_t F_EQ1 = 1, F_GT0 = 2, F_LT1 = 4;      // immersed proportion == 1, > 0, < 1
constexpr int iR = 0, iU = 1, iV = 2, iW = 3, iT = 4, iK = 5;

struct Grid {
  int nx, ny, nz;
  double dz, rdx, rdy, rdz, r2dx, r2dy, r2dz;
  int bc_x, bc_y, bc_z;
  double R_d, gamma, C0, grav, rgamma, rgm1;
  int gravity, dns;
  double nu, nu_Pr, total_mult, diss_mult, shear_mult, delta;
  const double *prop;   // immersed_proportion_halos (nz+2, ny+2, nx+2)
};

// q[t]: the t-th diffused tracer (resolved on the host, so the kernels index
// it with compile-time constants only).
struct In {
  const double *rd, *u, *v, *w, *T, *tke, *q[3];
};
struct Out {
  double *u, *v, *w, *T, *tke, *q[3];
};

__device__ __forceinline__ int wrapi(int i, int n) {
  i %= n;
  return i < 0 ? i + n : i;
}
__device__ __forceinline__ int clampi(int i, int n) { return i < 0 ? 0 : (i >= n ? n - 1 : i); }

template <int ND>
struct Les {
  static constexpr int F = 6 + ND, NF = 6 + ND;   // fields in the ring; fluxes per face
  static constexpr size_t ring_bytes = sizeof(double) * 3 * F * HP;
  static constexpr size_t flux_bytes = sizeof(double) * NF * (TY * (TX + 1) + (TY + 1) * TX);
  static constexpr size_t bytes = ring_bytes + flux_bytes + 3 * HP;
};

// One plane p (-1..nz) of the tile with its halo: primitive fields of the
// closure (les_closure.h:356-365) with the boundary conditions of
// coupler.h:785-855 and les_closure.h:411-532 applied while loading: periodic
// x/y (corners wrap in both), precursor x/y copies the edge cell into the
// halo of interior rows, solid walls copy the edge level with w = 0 and an
// isentropic density, periodic z wraps.
template <int ND>
__device__ void load_plane(const Grid &G, const In &in, int p, int i0, int j0, double *ring, uint8_t *flag) {
  constexpr int F = Les<ND>::F;
  const int nx = G.nx, ny = G.ny, nz = G.nz;
  for (int c = threadIdx.x; c < HP; c += NT) {
    const int r = c / HX, cc = c % HX;
    const int gj = j0 - 1 + r, gi = i0 - 1 + cc;
    const bool inx = gi >= 0 && gi < nx, iny = gj >= 0 && gj < ny;
    int si = gi, sj = gj;
    if (!inx && iny) si = G.bc_x == BC_PRECURSOR ? clampi(gi, nx) : wrapi(gi, nx);
    else if (inx && !iny) sj = G.bc_y == BC_PRECURSOR ? clampi(gj, ny) : wrapi(gj, ny);
    else if (!inx && !iny) {
      si = wrapi(gi, nx);
      sj = wrapi(gj, ny);
    }
    int sp = p;
    bool zhalo = false;
    if (p < 0 || p >= nz) {
      if (G.bc_z == BC_WALL) {
        sp = p < 0 ? 0 : nz - 1;
        zhalo = true;
      } else {
        sp = wrapi(p, nz);
      }
    }
    const size_t q = (size_t(sp) * ny + sj) * nx + si;
    const double rd = in.rd[q];
    const double th = pow(rd * G.R_d * in.T[q] / G.C0, G.rgamma) / rd;
    double val[F];
    val[iR] = rd;
    val[iU] = in.u[q];
    val[iV] = in.v[q];
    val[iW] = zhalo ? 0.0 : in.w[q];
    val[iT] = th;
    val[iK] = fmax(0.0, in.tke[q] / rd);
#pragma unroll
    for (int t = 0; t < ND; t++) val[6 + t] = in.q[t][q] / rd;
    if (zhalo) {
      const double g = G.gravity ? G.grav : 0.0;
      const double rho0_gm1 = pow(rd, G.gamma - 1), theta0_g = pow(th, G.gamma);
      const double add = g * (G.gamma - 1) * G.dz / (G.gamma * G.C0 * theta0_g);
      val[iR] = pow(p < 0 ? rho0_gm1 + add : rho0_gm1 - add, G.rgm1);
    }
#pragma unroll
    for (int f = 0; f < F; f++) ring[f * HP + c] = val[f];
    // Flags from the halo array (tile columns past the domain clamp onto its halo).
    const int hj = min(gj, ny) + 1, hi = min(gi, nx) + 1;
    const double pr = G.prop[(size_t(p + 1) * (ny + 2) + hj) * (nx + 2) + hi];
    flag[c] = uint8_t((pr == 1 ? F_EQ1 : 0) | (pr > 0 ? F_GT0 : 0) | (pr < 1 ? F_LT1 : 0));
  }
}

// Face quantities (les_closure.h:87-232) for the face between cells A and B
// along DIR (0 x, 1 y, 2 z).  Cells are (slot, halo row, halo column);
// sm / sp are the slots of the levels below and above the face's level
// (x and y faces only).  out: fluxes of rho*u, rho*v, rho*w, rho*theta, TKE,
// diffused tracers.
template <int ND, int DIR>
__device__ __forceinline__ void face_flux(const Grid &G, const double *ring, const uint8_t *flag, int sA, int rA, int cA,
                                          int sB, int rB, int cB, int sm, int sp, double visc_half,
                                          double (&out)[Les<ND>::NF]) {
  constexpr int F = Les<ND>::F, NF = Les<ND>::NF;
  const int oA = rA * HX + cA, oB = rB * HX + cB;
  if ((flag[sA * HP + oA] & F_EQ1) || (flag[sB * HP + oB] & F_EQ1)) {
#pragma unroll
    for (int v = 0; v < NF; v++) out[v] = 0.0;
    return;
  }
  auto X = [&](int f, int s, int o) { return ring[(s * F + f) * HP + o]; };
  const double rn = DIR == 0 ? G.rdx : DIR == 1 ? G.rdy : G.rdz;
  auto normal = [&](int f) { return (X(f, sB, oB) - X(f, sA, oA)) * rn; };
  // Centred derivative of f along E at A and at B, averaged.
  auto tang = [&](int f, int E) {
    double a, b;
    if (E == 0) {
      a = (X(f, sA, oA + 1) - X(f, sA, oA - 1)) * G.r2dx;
      b = (X(f, sB, oB + 1) - X(f, sB, oB - 1)) * G.r2dx;
    } else if (E == 1) {
      a = (X(f, sA, oA + HX) - X(f, sA, oA - HX)) * G.r2dy;
      b = (X(f, sB, oB + HX) - X(f, sB, oB - HX)) * G.r2dy;
    } else {
      a = (X(f, sp, oA) - X(f, sm, oA)) * G.r2dz;
      b = (X(f, sp, oB) - X(f, sm, oB)) * G.r2dz;
    }
    return 0.5 * (a + b);
  };
  double g[3][3];   // g[c][e]: d(velocity c)/d(direction e)
#pragma unroll
  for (int c = 0; c < 3; c++) {
    g[c][DIR] = normal(iU + c);
#pragma unroll
    for (int e = 0; e < 3; e++)
      if (e != DIR && (c == e || c == DIR)) g[c][e] = tang(iU + c, e);
  }
  const double dt_dz = DIR == 2 ? normal(iT) : tang(iT, 2);
  const double rho = 0.5 * (X(iR, sA, oA) + X(iR, sB, oB));
  const double K = 0.5 * (X(iK, sA, oA) + X(iK, sB, oB));
  const double t = 0.5 * (X(iT, sA, oA) + X(iT, sB, oB));
  const double N = dt_dz >= 0 && G.gravity ? sqrt(G.grav / t * dt_dz) : 0.0;
  const double sK = sqrt(K);
  const double ell = fmin(0.76 * sK / (N + 1.e-20), G.delta);
  const double km = G.total_mult * 0.1 * ell * sK;
  const double Pr_t = G.delta / (1 + 2 * ell);
  const double visc = G.dns ? G.nu : fmin(km + G.nu, visc_half);
  const double visc_th = G.dns ? G.nu : fmin(km / Pr_t + G.nu_Pr, visc_half);
  const double div = g[0][0] + g[1][1] + g[2][2];
  const double mrv = -rho * visc;
#pragma unroll
  for (int c = 0; c < 3; c++) out[c] = c == DIR ? mrv * (g[c][c] + g[c][c] - 2. / 3. * div) : mrv * (g[c][DIR] + g[DIR][c]);
  out[3] = -rho * visc_th * normal(iT);
  out[4] = mrv * 2 * normal(iK);
#pragma unroll
  for (int t2 = 0; t2 < ND; t2++) out[5 + t2] = mrv * normal(6 + t2);
}

// Cell TKE source: buoyancy, dissipation, shear production (les_closure.h:236-282).
template <int ND>
__device__ __forceinline__ double tke_source(const Grid &G, const double *ring, const uint8_t *flag, int s, int sm, int sp,
                                             int o) {
  constexpr int F = Les<ND>::F;
  auto X = [&](int f, int sl, int oo) { return ring[(sl * F + f) * HP + oo]; };
  if (!(flag[s * HP + o] & F_LT1)) return 0.0;
  const double rho = X(iR, s, o), K = X(iK, s, o), t = X(iT, s, o);
  const double dt_dz = (X(iT, sp, o) - X(iT, sm, o)) * G.r2dz;
  const double N = dt_dz >= 0 && G.gravity ? sqrt(G.grav / t * dt_dz) : 0.0;
  const double sK = sqrt(K);
  const double ell = fmin(0.76 * sK / (N + 1.e-20), G.delta);
  const double km = 0.1 * ell * sK;
  const double Pr_t = G.delta / (1 + 2 * ell);
  double src = 0.0;
  if (G.gravity) src += -(G.grav * rho * km) / (t * Pr_t) * dt_dz;
  src -= G.diss_mult * rho * (0.19 + 0.51 * ell / G.delta) / G.delta * (K * sK);
  // Neighbours inside immersed material are replaced by the cell itself
  // except along a component's own direction.
  const int oxm = (flag[s * HP + o - 1] & F_GT0) ? o : o - 1, oxp = (flag[s * HP + o + 1] & F_GT0) ? o : o + 1;
  const int oym = (flag[s * HP + o - HX] & F_GT0) ? o : o - HX, oyp = (flag[s * HP + o + HX] & F_GT0) ? o : o + HX;
  const int szm = (flag[sm * HP + o] & F_GT0) ? s : sm, szp = (flag[sp * HP + o] & F_GT0) ? s : sp;
  double g[3][3];   // g[e][c]: d(component c)/d(direction e)
  g[0][0] = (X(iU, s, o + 1) - X(iU, s, o - 1)) * G.r2dx;
  g[0][1] = (X(iV, s, oxp) - X(iV, s, oxm)) * G.r2dx;
  g[0][2] = (X(iW, s, oxp) - X(iW, s, oxm)) * G.r2dx;
  g[1][0] = (X(iU, s, oyp) - X(iU, s, oym)) * G.r2dy;
  g[1][1] = (X(iV, s, o + HX) - X(iV, s, o - HX)) * G.r2dy;
  g[1][2] = (X(iW, s, oyp) - X(iW, s, oym)) * G.r2dy;
  g[2][0] = (X(iU, szp, o) - X(iU, szm, o)) * G.r2dz;
  g[2][1] = (X(iV, szp, o) - X(iV, szm, o)) * G.r2dz;
  g[2][2] = (X(iW, sp, o) - X(iW, sm, o)) * G.r2dz;
  double sum = (g[0][0] + g[0][0]) * g[0][0];
#pragma unroll
  for (int e = 0; e < 3; e++)
#pragma unroll
    for (int c = 0; c < 3; c++)
      if (e + c > 0) sum += (g[e][c] + g[c][e]) * g[e][c];
  src += G.shear_mult * rho * km * sum;
  return src;
}

__device__ __forceinline__ int slot_of(int p) { return ((p % 3) + 3) % 3; }

template <int ND>
__global__ void __launch_bounds__(NT) k_les(const Grid G, const In in, const Out out, double dt, double vhx,
                                            double vhy, double vhz) {
  constexpr int F = Les<ND>::F, NF = Les<ND>::NF;
  extern __shared__ __align__(16) unsigned char smem[];
  double *ring = reinterpret_cast<double *>(smem);                        // [3][F][HP]
  double *fx = ring + 3 * F * HP;                                          // [NF][TY][TX+1]
  double *fy = fx + NF * TY * (TX + 1);                                    // [NF][TY+1][TX]
  uint8_t *flag = reinterpret_cast<uint8_t *>(fy + NF * (TY + 1) * TX);   // [3][HP]
  const int tid = threadIdx.x, tj = tid / TX, ti = tid % TX;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int k0 = blockIdx.z * KC, k1 = min(G.nz, k0 + KC);
  const int i = i0 + ti, j = j0 + tj;
  const bool live = i < G.nx && j < G.ny;
  const int oc = (tj + 1) * HX + (ti + 1);   // this column's offset in the halo tile
  for (int p = k0 - 1; p <= k0 + 1; p++)
    load_plane<ND>(G, in, p, i0, j0, ring + slot_of(p) * F * HP, flag + slot_of(p) * HP);
  __syncthreads();
  double Fb[NF];   // flux through the bottom face of the current cell
  face_flux<ND, 2>(G, ring, flag, slot_of(k0 - 1), tj + 1, ti + 1, slot_of(k0), tj + 1, ti + 1, 0, 0, vhz, Fb);
  for (int k = k0; k < k1; k++) {
    const int sm = slot_of(k - 1), s = slot_of(k), sp = slot_of(k + 1);
    // x faces (i-1/2 for i = 0..TX) and y faces of this level into shared memory.
    for (int e = tid; e < TY * (TX + 1) + (TY + 1) * TX; e += NT) {
      double fl[NF];
      if (e < TY * (TX + 1)) {
        const int r = e / (TX + 1), fi = e % (TX + 1);
        face_flux<ND, 0>(G, ring, flag, s, r + 1, fi, s, r + 1, fi + 1, sm, sp, vhx, fl);
#pragma unroll
        for (int v = 0; v < NF; v++) fx[v * TY * (TX + 1) + e] = fl[v];
      } else {
        const int e2 = e - TY * (TX + 1), fj = e2 / TX, c = e2 % TX;
        face_flux<ND, 1>(G, ring, flag, s, fj, c + 1, s, fj + 1, c + 1, sm, sp, vhy, fl);
#pragma unroll
        for (int v = 0; v < NF; v++) fy[v * (TY + 1) * TX + e2] = fl[v];
      }
    }
    double Ft[NF];
    face_flux<ND, 2>(G, ring, flag, s, tj + 1, ti + 1, sp, tj + 1, ti + 1, 0, 0, vhz, Ft);
    const double src = tke_source<ND>(G, ring, flag, s, sm, sp, oc);
    double cell[F];
#pragma unroll
    for (int f = 0; f < F; f++) cell[f] = ring[(s * F + f) * HP + oc];
    __syncthreads();   // face fluxes visible; plane k-1 no longer read
    // The next level's upper plane (k+2 <= k1 <= nz) into the slot of level k-1.
    if (k + 1 < k1) load_plane<ND>(G, in, k + 2, i0, j0, ring + slot_of(k + 2) * F * HP, flag + slot_of(k + 2) * HP);
    if (live) {
      double tend[NF];
#pragma unroll
      for (int v = 0; v < NF; v++) {
        const double ax = fx[v * TY * (TX + 1) + tj * (TX + 1) + ti + 1] - fx[v * TY * (TX + 1) + tj * (TX + 1) + ti];
        const double ay = fy[v * (TY + 1) * TX + (tj + 1) * TX + ti] - fy[v * (TY + 1) * TX + tj * TX + ti];
        tend[v] = -ax * G.rdx - ay * G.rdy - (Ft[v] - Fb[v]) * G.rdz;
      }
      tend[4] += src;
      const double rho = cell[iR];
      const size_t q = (size_t(k) * G.ny + j) * G.nx + i;
      out.u[q] = (cell[iU] * rho + dt * tend[0]) / rho;
      out.v[q] = (cell[iV] * rho + dt * tend[1]) / rho;
      out.w[q] = (cell[iW] * rho + dt * tend[2]) / rho;
      out.T[q] = G.C0 * pow(cell[iT] * rho + dt * tend[3], G.gamma) / (rho * G.R_d);
      out.tke[q] = fmax(0.0, cell[iK] * rho + dt * tend[4]);
#pragma unroll
      for (int t = 0; t < ND; t++) out.q[t][q] = cell[6 + t] * rho + dt * tend[5 + t];
    }
#pragma unroll
    for (int v = 0; v < NF; v++) Fb[v] = Ft[v];
    __syncthreads();   // next plane loaded; face fluxes consumed
  }
}

// ---------------------------------------------------------------------------
// Level means: each term scaled by 1/(nx*ny) (as the reference adds
// u*r_nx_ny), Neumaier-compensated sums in a fixed order.
// ---------------------------------------------------------------------------
struct CSum {
  double s, c;
  __host__ __device__ void add(double x) {
    const double t = s + x;
    c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
    s = t;
  }
};

constexpr int PARTS = 8, RED_T = 256;

// partial[((lvl * PARTS) + part) * 3 + f] = (s, c) of a part of level klo+lvl.
__global__ void __launch_bounds__(RED_T) k_level_partial(const double *a0, const double *a1, const double *a2, int nf,
                                                         int klo, int nx, int ny, double r, double2 *partial) {
  const int lvl = blockIdx.x, part = blockIdx.y;
  const size_t n = size_t(nx) * ny, base = size_t(klo + lvl) * n;
  const size_t lo = n * part / PARTS, hi = n * (part + 1) / PARTS;
  __shared__ double ss[3][RED_T], cs[3][RED_T];
  const double *src[3] = {a0, a1, a2};
  for (int f = 0; f < nf; f++) {
    CSum acc{0.0, 0.0};
    for (size_t e = lo + threadIdx.x; e < hi; e += RED_T) acc.add(src[f][base + e] * r);
    ss[f][threadIdx.x] = acc.s;
    cs[f][threadIdx.x] = acc.c;
  }
  __syncthreads();
  if (threadIdx.x < nf) {
    const int f = threadIdx.x;
    CSum acc{0.0, 0.0};
    double c = 0.0;
    for (int t = 0; t < RED_T; t++) {
      acc.add(ss[f][t]);
      c += cs[f][t];
    }
    partial[(size_t(lvl) * PARTS + part) * 3 + f] = make_double2(acc.s, acc.c + c);
  }
}

__global__ void k_level_final(const double2 *partial, int nlev, int nf, double *mean) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nlev * nf) return;
  const int lvl = e / nf, f = e % nf;
  CSum acc{0.0, 0.0};
  double c = 0.0;
  for (int p = 0; p < PARTS; p++) {
    const double2 v = partial[(size_t(lvl) * PARTS + p) * 3 + f];
    acc.add(v.x);
    c += v.y;
  }
  mean[size_t(lvl) * 3 + f] = acc.s + (acc.c + c);
}

__global__ void k_sponge(double *u, double *v, double *w, double *T, const double *mean, int klo, int nz, int nx,
                         int ny, double dz, double z1, double z2, double dt, double time_scale) {
  const size_t n = size_t(nx) * ny;
  const size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= size_t(nz - klo) * n) return;
  const int k = klo + int(e / n);
  const size_t q = size_t(klo) * n + e;
  const double z = (k + 0.5) * dz;
  if (!(z > z1)) return;
  const double factor = pow((z - z1) / (z2 - z1), 3.0) * dt / time_scale;
  const double *m = mean + size_t(k - klo) * 3;
  u[q] = factor * m[0] + (1 - factor) * u[q];
  v[q] = factor * m[1] + (1 - factor) * v[q];
  w[q] = factor * 0 + (1 - factor) * w[q];
  T[q] = factor * m[2] + (1 - factor) * T[q];
}

__global__ void k_geostrophic(double *u, double *v, const double *mean, int nz, size_t n, double dt, double fcor,
                              double u_g, double v_g) {
  const size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= size_t(nz) * n) return;
  const double *m = mean + (e / n) * 3;
  u[e] += dt * (fcor * (m[1] - v_g));
  v[e] += dt * (-fcor * (m[0] - u_g));
}

// uvel += fu, vvel += fv everywhere (uniform_pg_wind_forcing.h:35-38).
__global__ void k_add_uv(double *u, double *v, size_t n, double fu, double fv) {
  const size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= n) return;
  u[e] += fu;
  v[e] += fv;
}

// The forcing of uniform_pg_wind_forcing_height (uniform_pg_wind_forcing.h:
// 69-80) from the level means of the two bracketing levels, mean[0..1] and
// mean[3..4]; each thread forms the same scalars, so no host round trip.
__global__ void k_pg_height(double *u, double *v, const double *mean, size_t n, double w1, double w2, double dt_tau,
                            double u0, double v0) {
  const size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const double um = w1 * mean[0] + w2 * mean[3];
  const double vm = w1 * mean[1] + w2 * mean[4];
  u[e] += dt_tau * (u0 - um);
  v[e] += dt_tau * (v0 - vm);
}

// Time_Averager::accumulate (time_averager.h:88-108), one cell per thread,
// each product and sum rounded separately in the reference's order.  a[0..12]:
// avg_u, avg_v, avg_w, avg_tke, avg_up_up, avg_up_vp, avg_up_wp, avg_vp_vp,
// avg_vp_wp, avg_wp_wp, long_avg_u, long_avg_v, long_avg_w.
struct TavgArrays {
  double *a[13];
};

__global__ void k_time_average(const double *__restrict__ u, const double *__restrict__ v,
                               const double *__restrict__ w, const double *__restrict__ tke, TavgArrays A, size_t n,
                               double in, double omi, double inl, double omil) {
  const size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const double U = u[e], V = v[e], W = w[e], K = tke[e];
  auto relax = [](double inertia, double avg, double om, double x) {
    return __dadd_rn(__dmul_rn(inertia, avg), __dmul_rn(om, x));
  };
  const double lu = relax(inl, A.a[10][e], omil, U);
  const double lv = relax(inl, A.a[11][e], omil, V);
  const double lw = relax(inl, A.a[12][e], omil, W);
  A.a[10][e] = lu;
  A.a[11][e] = lv;
  A.a[12][e] = lw;
  const double up = __dsub_rn(U, lu), vp = __dsub_rn(V, lv), wp = __dsub_rn(W, lw);
  A.a[0][e] = relax(in, A.a[0][e], omi, U);
  A.a[1][e] = relax(in, A.a[1][e], omi, V);
  A.a[2][e] = relax(in, A.a[2][e], omi, W);
  A.a[3][e] = relax(in, A.a[3][e], omi, K);
  // (1-inertia)*up*up groups as ((1-inertia)*up)*up.
  auto relax2 = [](double inertia, double avg, double om, double x, double y) {
    return __dadd_rn(__dmul_rn(inertia, avg), __dmul_rn(__dmul_rn(om, x), y));
  };
  A.a[4][e] = relax2(in, A.a[4][e], omi, up, up);
  A.a[5][e] = relax2(in, A.a[5][e], omi, up, vp);
  A.a[6][e] = relax2(in, A.a[6][e], omi, up, wp);
  A.a[7][e] = relax2(in, A.a[7][e], omi, vp, vp);
  A.a[8][e] = relax2(in, A.a[8][e], omi, vp, wp);
  A.a[9][e] = relax2(in, A.a[9][e], omi, wp, wp);
}

// EdgeSponge::apply (edge_sponge.h:47-71) on up to 8 fields: the four edge
// zones in the reference's order, each weight ((p1-p)/p1)^5.
struct SpongeFields {
  double *f[8];
};

__global__ void k_edge_sponge(SpongeFields S, int nfields, const double *__restrict__ column, int nx, int ny, int nz,
                              long long i_beg, long long j_beg, long long nx_glob, long long ny_glob, double px1,
                              double px2, double py1, double py2) {
  const size_t n = size_t(nx) * ny * nz;
  const size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const int i = int(e % nx), j = int((e / nx) % ny), k = int(e / (size_t(nx) * ny));
  const double prop_x = double(i_beg + i) / double(nx_glob), prop_y = double(j_beg + j) / double(ny_glob);
  double w[4];
  bool on[4];
  on[0] = px1 > 0 && prop_x <= px1;
  on[1] = px2 > 0 && prop_x >= 1 - px2;
  on[2] = py1 > 0 && prop_y <= py1;
  on[3] = py2 > 0 && prop_y >= 1 - py2;
  if (!(on[0] || on[1] || on[2] || on[3])) return;
  w[0] = on[0] ? pow((px1 - prop_x) / px1, 5.0) : 0.0;
  w[1] = on[1] ? pow((prop_x - (1 - px2)) / px2, 5.0) : 0.0;
  w[2] = on[2] ? pow((py1 - prop_y) / py1, 5.0) : 0.0;
  w[3] = on[3] ? pow((prop_y - (1 - py2)) / py2, 5.0) : 0.0;
  for (int l = 0; l < nfields; l++) {
    double x = S.f[l][e];
    const double c = column[size_t(l) * nz + k];
#pragma unroll
    for (int z = 0; z < 4; z++)
      if (on[z]) x = w[z] * c + (1 - w[z]) * x;
    S.f[l][e] = x;
  }
}

// Log-law drag and heat flux from each immersed face neighbour, in the
// order x-, x+, y-, y+, z-, z+ (surface_flux.h:40-117).
__global__ void k_surface_fluxes(double *u, double *v, double *w, double *T, const double *prop, const double *rough,
                                 const double *temp, int nx, int ny, int nz, double dx, double dy, double dz, double dt) {
  const size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= size_t(nx) * ny * nz) return;
  const int i = int(e % nx), j = int((e / nx) % ny), k = int(e / (size_t(nx) * ny));
  const double vel[3] = {u[e], v[e], w[e]}, Tc = T[e];
  const double d[3] = {dx, dy, dz};
  double tend[3] = {0.0, 0.0, 0.0}, tendT = 0.0;
  const double vk = 0.40;
#pragma unroll
  for (int n = 0; n < 6; n++) {
    const int dir = n / 2, sgn = (n & 1) ? 1 : -1;
    const int hk = k + 1 + (dir == 2 ? sgn : 0), hj = j + 1 + (dir == 1 ? sgn : 0), hi = i + 1 + (dir == 0 ? sgn : 0);
    const size_t hq = (size_t(hk) * (ny + 2) + hj) * (nx + 2) + hi;
    if (!(prop[hq] > 0)) continue;
    const double roughness = rough[hq];
    const double lg = log((d[dir] / 2 + roughness) / roughness);
    const double cd = vk * vk / (lg * lg);
    const double T0 = temp[hq];
    const int a = dir == 0 ? 1 : 0, b = dir == 2 ? 1 : 2;
    const double mag = sqrt(vel[a] * vel[a] + vel[b] * vel[b]);
    tend[a] += -cd * (vel[a] - 0) * mag / d[dir];
    tend[b] += -cd * (vel[b] - 0) * mag / d[dir];
    if (T0 != 0) tendT += -cd * (Tc - T0) * mag / d[dir];
  }
  u[e] = vel[0] + dt * tend[0];
  v[e] = vel[1] + dt * tend[1];
  w[e] = vel[2] + dt * tend[2];
  T[e] = Tc + dt * tendT;
}

}  // namespace phys
}  // namespace pu

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
using namespace pu::phys;

struct pu_physics {
  pu_physics_config cfg;
  cudaStream_t st = nullptr;
  size_t N = 0, NH = 0;
  double *prop = nullptr, *rough = nullptr, *temp = nullptr;   // halo arrays
  double *stage = nullptr;     // (5 + ntr) * N: host views, and the in-place LES output
  double2 *partial = nullptr;  // level-sum partials
  double *mean = nullptr;      // level means [nz][3]
  double *tavg_stage = nullptr;  // 13 * N: time averages given in host memory (allocated on first use)
  double *column = nullptr;      // edge-sponge column profiles, column_cap doubles
  size_t column_cap = 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int nd = 0, qidx[4] = {0, 0, 0, 0};
};

namespace {

int fail(int code, const std::string &msg) {
  pu::set_error(msg);
  return code;
}

#define PH_CK(x)                                                                                   \
  do {                                                                                             \
    cudaError_t e_ = (x);                                                                          \
    if (e_ != cudaSuccess) return fail(PU_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// Makes the handle's device current for one call and restores the caller's
// device afterwards; `status` is the switch's result.
struct Dev {
  int prev = -1;
  cudaError_t status = cudaSuccess;
  explicit Dev(int d) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != d) status = cudaSetDevice(d);
  }
  ~Dev() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

// A named range for profilers (NVTX; a no-op unless a tool is attached).
struct PhRange {
  explicit PhRange(const char *name) { nvtxRangePushA(name); }
  ~PhRange() { nvtxRangePop(); }
  PhRange(const PhRange &) = delete;
  PhRange &operator=(const PhRange &) = delete;
};

// The guard of a call; returns PU_ERR_CUDA from it when the device cannot be
// made current.
#define PH_DEVICE(dev)  \
  Dev g(dev);           \
  if (g.status != cudaSuccess) return fail(PU_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(g.status))

bool on_device(int mem, const void *p) {
  if (mem == PU_MEM_DEVICE) return true;
  if (mem == PU_MEM_HOST) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

Grid make_grid(const pu_physics &h) {
  const pu_physics_config &c = h.cfg;
  Grid G;
  G.nx = c.nx;
  G.ny = c.ny;
  G.nz = c.nz;
  G.dz = c.dz;
  G.rdx = 1.0 / c.dx;
  G.rdy = 1.0 / c.dy;
  G.rdz = 1.0 / c.dz;
  G.r2dx = 1.0 / (2 * c.dx);
  G.r2dy = 1.0 / (2 * c.dy);
  G.r2dz = 1.0 / (2 * c.dz);
  G.bc_x = c.bc_x;
  G.bc_y = c.bc_y;
  G.bc_z = c.bc_z;
  G.R_d = c.R_d;
  G.gamma = c.gamma_d;
  G.C0 = c.C0;
  G.grav = c.grav;
  G.rgamma = 1.0 / c.gamma_d;
  G.rgm1 = 1.0 / (c.gamma_d - 1);
  G.gravity = c.enable_gravity != 0;
  G.dns = c.dns != 0;
  G.nu = c.kinematic_viscosity;
  G.nu_Pr = c.kinematic_viscosity / 0.7;
  G.total_mult = c.les_total_mult;
  G.diss_mult = c.les_dissipation_mult;
  G.shear_mult = c.les_shear_prod_mult;
  G.delta = std::pow(c.dx * c.dy * c.dz, 1.0 / 3.0);
  G.prop = h.prop;
  return G;
}

// Device pointers of a view: host arrays are staged into h.stage.
int device_arrays(pu_physics &h, const pu_state_view *v, double *(&d)[5 + PU_MAX_TRACERS], bool &staged) {
  const int S = 5 + h.cfg.ntracers;
  double *src[5 + PU_MAX_TRACERS] = {v->rho_d, v->uvel, v->vvel, v->wvel, v->temp};
  for (int t = 0; t < h.cfg.ntracers; t++) src[5 + t] = v->tracers[t];
  for (int a = 0; a < S; a++)
    if (!src[a]) return fail(PU_ERR_INVALID, "state view has a null array");
  staged = !on_device(v->mem, v->rho_d);
  for (int a = 0; a < S; a++) {
    if (staged) {
      d[a] = h.stage + size_t(a) * h.N;
      PH_CK(cudaMemcpyAsync(d[a], src[a], h.N * sizeof(double), cudaMemcpyHostToDevice, h.st));
    } else {
      d[a] = src[a];
    }
  }
  return PU_OK;
}

int copy_back(pu_physics &h, const pu_state_view *v, double *const (&d)[5 + PU_MAX_TRACERS], const int *which, int n) {
  double *dst[5 + PU_MAX_TRACERS] = {v->rho_d, v->uvel, v->vvel, v->wvel, v->temp};
  for (int t = 0; t < h.cfg.ntracers; t++) dst[5 + t] = v->tracers[t];
  for (int e = 0; e < n; e++)
    PH_CK(cudaMemcpyAsync(dst[which[e]], d[which[e]], h.N * sizeof(double), cudaMemcpyDeviceToHost, h.st));
  PH_CK(cudaStreamSynchronize(h.st));
  return PU_OK;
}

template <int ND>
int launch_les(pu_physics &h, const In &in, const Out &out, double dt) {
  const Grid G = make_grid(h);
  const size_t bytes = Les<ND>::bytes;
  PH_CK(cudaFuncSetAttribute(k_les<ND>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
  dim3 grid((h.cfg.nx + TX - 1) / TX, (h.cfg.ny + TY - 1) / TY, (h.cfg.nz + KC - 1) / KC);
  const double vhx = 0.5 * (0.25 * h.cfg.dx * h.cfg.dx / dt), vhy = 0.5 * (0.25 * h.cfg.dy * h.cfg.dy / dt),
               vhz = 0.5 * (0.25 * h.cfg.dz * h.cfg.dz / dt);
  cudaEventRecord(h.e0, h.st);
  k_les<ND><<<grid, NT, bytes, h.st>>>(G, in, out, dt, vhx, vhy, vhz);
  cudaEventRecord(h.e1, h.st);
  PH_CK(cudaGetLastError());
  return PU_OK;
}

int run_les(pu_physics &h, const In &in, const Out &out, double dt) {
  switch (h.nd) {
    case 0: return launch_les<0>(h, in, out, dt);
    case 1: return launch_les<1>(h, in, out, dt);
    case 2: return launch_les<2>(h, in, out, dt);
    default: return launch_les<3>(h, in, out, dt);
  }
}

In make_in(const pu_physics &h, double *const (&d)[5 + PU_MAX_TRACERS]) {
  In in;
  in.rd = d[0];
  in.u = d[1];
  in.v = d[2];
  in.w = d[3];
  in.T = d[4];
  in.tke = d[5 + h.cfg.idTKE];
  for (int t = 0; t < 3; t++) in.q[t] = t < h.nd ? d[5 + h.qidx[t]] : nullptr;
  return in;
}

Out make_out(const pu_physics &h, double *const (&d)[5 + PU_MAX_TRACERS]) {
  Out o;
  o.u = d[1];
  o.v = d[2];
  o.w = d[3];
  o.T = d[4];
  o.tke = d[5 + h.cfg.idTKE];
  for (int t = 0; t < 3; t++) o.q[t] = t < h.nd ? d[5 + h.qidx[t]] : nullptr;
  return o;
}

// Indices (into the 5 + ntr coupler arrays) that the LES writes.
int les_written(const pu_physics &h, int *which) {
  int n = 0;
  for (int a = 1; a <= 4; a++) which[n++] = a;
  which[n++] = 5 + h.cfg.idTKE;
  for (int t = 0; t < h.nd; t++) which[n++] = 5 + h.qidx[t];
  return n;
}

// Means of levels klo .. klo+nlev-1 (all levels from klo up when nlev < 0)
// into h.mean[(k - klo) * 3 + f].
int level_means(pu_physics &h, const double *a0, const double *a1, const double *a2, int nf, int klo, int nlev = -1) {
  if (nlev < 0) nlev = h.cfg.nz - klo;
  if (nlev <= 0) return PU_OK;
  const double r = 1. / (double(h.cfg.nx) * h.cfg.ny);
  k_level_partial<<<dim3(nlev, PARTS), RED_T, 0, h.st>>>(a0, a1, a2, nf, klo, h.cfg.nx, h.cfg.ny, r, h.partial);
  PH_CK(cudaGetLastError());
  k_level_final<<<(nlev * nf + 127) / 128, 128, 0, h.st>>>(h.partial, nlev, nf, h.mean);
  PH_CK(cudaGetLastError());
  return PU_OK;
}

}  // namespace

extern "C" {

int pu_physics_create(const pu_physics_config *cfg, const double *imm_prop_h, const double *imm_rough_h,
                      const double *imm_temp_h, int mem, pu_physics **out) {
  if (!cfg || !out || !imm_prop_h || !imm_rough_h || !imm_temp_h) return fail(PU_ERR_INVALID, "null argument");
  *out = nullptr;
  if (cfg->nx < 1 || cfg->ny < 1 || cfg->nz < 1 || !(cfg->dx > 0 && cfg->dy > 0 && cfg->dz > 0))
    return fail(PU_ERR_INVALID, "bad grid");
  if (cfg->ntracers < 0 || cfg->ntracers > PU_MAX_TRACERS) return fail(PU_ERR_INVALID, "bad tracer count");
  if (cfg->idTKE >= cfg->ntracers) return fail(PU_ERR_INVALID, "idTKE out of range");
  if (cfg->bc_z != PU_BC_WALL && cfg->bc_z != PU_BC_PERIODIC)
    return fail(PU_ERR_INVALID, "ERROR: Specified invalid bc_z in coupler options");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(PU_ERR_CUDA, "no CUDA device");
  if (cfg->device < 0 || cfg->device >= ndev) return fail(PU_ERR_INVALID, "bad device ordinal");
  PH_DEVICE(cfg->device);
  pu_physics *h = new pu_physics;
  h->cfg = *cfg;
  h->st = static_cast<cudaStream_t>(cfg->stream);
  h->N = size_t(cfg->nx) * cfg->ny * cfg->nz;
  h->NH = size_t(cfg->nx + 2) * (cfg->ny + 2) * (cfg->nz + 2);
  int ndiff = 0;
  for (int t = 0; t < cfg->ntracers; t++)
    if (cfg->tracer_diffuse[t] && t != cfg->idTKE) {
      if (ndiff < 4) h->qidx[ndiff] = t;
      ndiff++;
    }
  h->nd = std::min(ndiff, 3);
  auto cleanup = [&](int rc) {
    pu_physics_destroy(h);
    return rc;
  };
  if (ndiff > 3) return cleanup(fail(PU_ERR_UNSUPPORTED, "at most 3 diffused tracers besides TKE"));
  void *p;
  const size_t S = 5 + size_t(cfg->ntracers);
  for (double **dst : {&h->prop, &h->rough, &h->temp}) {
    if (cudaMalloc(&p, h->NH * sizeof(double)) != cudaSuccess) return cleanup(fail(PU_ERR_NOMEM, "cudaMalloc failed"));
    *dst = static_cast<double *>(p);
  }
  if (cudaMalloc(&p, S * h->N * sizeof(double)) != cudaSuccess) return cleanup(fail(PU_ERR_NOMEM, "cudaMalloc failed"));
  h->stage = static_cast<double *>(p);
  if (cudaMalloc(&p, size_t(cfg->nz) * PARTS * 3 * sizeof(double2)) != cudaSuccess)
    return cleanup(fail(PU_ERR_NOMEM, "cudaMalloc failed"));
  h->partial = static_cast<double2 *>(p);
  if (cudaMalloc(&p, size_t(cfg->nz) * 3 * sizeof(double)) != cudaSuccess)
    return cleanup(fail(PU_ERR_NOMEM, "cudaMalloc failed"));
  h->mean = static_cast<double *>(p);
  cudaEventCreate(&h->e0);
  cudaEventCreate(&h->e1);
  const double *src[3] = {imm_prop_h, imm_rough_h, imm_temp_h};
  double *dst[3] = {h->prop, h->rough, h->temp};
  const bool dev = on_device(mem, imm_prop_h);
  for (int a = 0; a < 3; a++)
    if (cudaMemcpyAsync(dst[a], src[a], h->NH * sizeof(double), dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                        h->st) != cudaSuccess)
      return cleanup(fail(PU_ERR_CUDA, "copying the immersed halo arrays failed"));
  if (cudaStreamSynchronize(h->st) != cudaSuccess) return cleanup(fail(PU_ERR_CUDA, "stream synchronize failed"));
  *out = h;
  return PU_OK;
}

int pu_physics_destroy(pu_physics *h) {
  if (!h) return PU_OK;
  {
    Dev g(h->cfg.device);
    cudaStreamSynchronize(h->st);
    for (void *p : {(void *)h->prop, (void *)h->rough, (void *)h->temp, (void *)h->stage, (void *)h->partial,
                    (void *)h->mean, (void *)h->tavg_stage, (void *)h->column})
      if (p) cudaFree(p);
    if (h->e0) cudaEventDestroy(h->e0);
    if (h->e1) cudaEventDestroy(h->e1);
  }
  delete h;
  return PU_OK;
}

int pu_les_apply(pu_physics *h, pu_state_view *v, double dt) {
  if (!h || !v) return fail(PU_ERR_INVALID, "null argument");
  if (h->cfg.idTKE < 0) return fail(PU_ERR_INVALID, "the LES closure needs the TKE tracer (les_closure.h:24-25)");
  if (!(dt > 0)) return fail(PU_ERR_INVALID, "dt must be positive");
  PH_DEVICE(h->cfg.device);
  PhRange range(__func__);
  double *d[5 + PU_MAX_TRACERS];
  bool staged;
  int rc = device_arrays(*h, v, d, staged);
  if (rc) return rc;
  int which[5 + PU_MAX_TRACERS];
  const int nw = les_written(*h, which);
  if (staged) {
    // Input in the staging area; output into a second copy of the written
    // fields (the rest of the staging area is the input).
    double *o[5 + PU_MAX_TRACERS];
    void *p;
    if (cudaMalloc(&p, size_t(nw) * h->N * sizeof(double)) != cudaSuccess) return fail(PU_ERR_NOMEM, "cudaMalloc failed");
    for (int a = 0; a < 5 + h->cfg.ntracers; a++) o[a] = d[a];
    for (int e = 0; e < nw; e++) o[which[e]] = static_cast<double *>(p) + size_t(e) * h->N;
    rc = run_les(*h, make_in(*h, d), make_out(*h, o), dt);
    if (!rc) rc = copy_back(*h, v, o, which, nw);
    cudaFree(p);
    return rc;
  }
  // Device arrays: output into the staging area, then copied back in place.
  double *o[5 + PU_MAX_TRACERS];
  for (int a = 0; a < 5 + h->cfg.ntracers; a++) o[a] = h->stage + size_t(a) * h->N;
  rc = run_les(*h, make_in(*h, d), make_out(*h, o), dt);
  if (rc) return rc;
  for (int e = 0; e < nw; e++)
    PH_CK(cudaMemcpyAsync(d[which[e]], o[which[e]], h->N * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
  return PU_OK;
}

int pu_les_apply_to(pu_physics *h, const pu_state_view *in, pu_state_view *out, double dt) {
  if (!h || !in || !out) return fail(PU_ERR_INVALID, "null argument");
  if (h->cfg.idTKE < 0) return fail(PU_ERR_INVALID, "the LES closure needs the TKE tracer (les_closure.h:24-25)");
  if (!(dt > 0)) return fail(PU_ERR_INVALID, "dt must be positive");
  PH_DEVICE(h->cfg.device);
  PhRange range(__func__);
  if (!in->rho_d || !out->uvel) return fail(PU_ERR_INVALID, "state view has a null array");
  if (!on_device(in->mem, in->rho_d) || !on_device(out->mem, out->uvel))
    return fail(PU_ERR_INVALID, "pu_les_apply_to takes device arrays");
  double *di[5 + PU_MAX_TRACERS] = {in->rho_d, in->uvel, in->vvel, in->wvel, in->temp};
  double *dout[5 + PU_MAX_TRACERS] = {out->rho_d, out->uvel, out->vvel, out->wvel, out->temp};
  for (int t = 0; t < h->cfg.ntracers; t++) {
    di[5 + t] = in->tracers[t];
    dout[5 + t] = out->tracers[t];
  }
  int which[5 + PU_MAX_TRACERS];
  const int nw = les_written(*h, which);
  for (int e = 0; e < nw; e++) {
    if (!di[which[e]] || !dout[which[e]]) return fail(PU_ERR_INVALID, "state view has a null array");
    if (di[which[e]] == dout[which[e]]) return fail(PU_ERR_INVALID, "pu_les_apply_to needs distinct in and out arrays");
  }
  return run_les(*h, make_in(*h, di), make_out(*h, dout), dt);
}

int pu_sponge_layer(pu_physics *h, pu_state_view *v, double dt, double time_scale, double top_prop) {
  if (!h || !v) return fail(PU_ERR_INVALID, "null argument");
  if (!(time_scale > 0) || !(top_prop > 0 && top_prop <= 1)) return fail(PU_ERR_INVALID, "bad sponge parameters");
  PH_DEVICE(h->cfg.device);
  PhRange range(__func__);
  double *d[5 + PU_MAX_TRACERS];
  bool staged;
  int rc = device_arrays(*h, v, d, staged);
  if (rc) return rc;
  const double dz = h->cfg.dz, zlen = dz * h->cfg.nz;
  const double z1 = (1 - top_prop) * zlen, z2 = zlen;
  const int k1 = std::max(0, int(std::floor(z1 / dz - 0.5)));
  rc = level_means(*h, d[1], d[2], d[4], 3, k1);
  if (rc) return rc;
  const size_t n = size_t(h->cfg.nz - k1) * h->cfg.nx * h->cfg.ny;
  if (n) {
    k_sponge<<<unsigned((n + 255) / 256), 256, 0, h->st>>>(d[1], d[2], d[3], d[4], h->mean, k1, h->cfg.nz, h->cfg.nx,
                                                          h->cfg.ny, dz, z1, z2, dt, time_scale);
    PH_CK(cudaGetLastError());
  }
  if (staged) {
    const int which[4] = {1, 2, 3, 4};
    return copy_back(*h, v, d, which, 4);
  }
  return PU_OK;
}

int pu_geostrophic_forcing(pu_physics *h, pu_state_view *v, double dt, double lat_g, double u_g, double v_g) {
  if (!h || !v) return fail(PU_ERR_INVALID, "null argument");
  PH_DEVICE(h->cfg.device);
  PhRange range(__func__);
  double *d[5 + PU_MAX_TRACERS];
  bool staged;
  int rc = device_arrays(*h, v, d, staged);
  if (rc) return rc;
  rc = level_means(*h, d[1], d[2], nullptr, 2, 0);
  if (rc) return rc;
  const double fcor = 2 * 7.2921e-5 * std::sin(lat_g / 180 * M_PI);
  const size_t n = size_t(h->cfg.nx) * h->cfg.ny;
  k_geostrophic<<<unsigned((h->N + 255) / 256), 256, 0, h->st>>>(d[1], d[2], h->mean, h->cfg.nz, n, dt, fcor, u_g, v_g);
  PH_CK(cudaGetLastError());
  if (staged) {
    const int which[2] = {1, 2};
    return copy_back(*h, v, d, which, 2);
  }
  return PU_OK;
}

int pu_surface_fluxes(pu_physics *h, pu_state_view *v, double dt) {
  if (!h || !v) return fail(PU_ERR_INVALID, "null argument");
  PH_DEVICE(h->cfg.device);
  PhRange range(__func__);
  double *d[5 + PU_MAX_TRACERS];
  bool staged;
  int rc = device_arrays(*h, v, d, staged);
  if (rc) return rc;
  k_surface_fluxes<<<unsigned((h->N + 255) / 256), 256, 0, h->st>>>(d[1], d[2], d[3], d[4], h->prop, h->rough, h->temp,
                                                                    h->cfg.nx, h->cfg.ny, h->cfg.nz, h->cfg.dx,
                                                                    h->cfg.dy, h->cfg.dz, dt);
  PH_CK(cudaGetLastError());
  if (staged) {
    const int which[4] = {1, 2, 3, 4};
    return copy_back(*h, v, d, which, 4);
  }
  return PU_OK;
}

int pu_uniform_pg_wind_forcing(pu_physics *h, pu_state_view *v, double dt, double tau,
                               unsigned long long update_cycles, pu_uniform_pg_state *state) {
  if (!h || !v || !state) return fail(PU_ERR_INVALID, "null argument");
  if (update_cycles == 0 || !(tau > 0)) return fail(PU_ERR_INVALID, "bad uniform_pg_wind_forcing parameters");
  PH_DEVICE(h->cfg.device);
  PhRange range(__func__);
  double *d[5 + PU_MAX_TRACERS];
  bool staged;
  int rc = device_arrays(*h, v, d, staged);
  if (rc) return rc;
  if (state->counter % update_cycles == 0) {
    // Domain mean = mean of the level means (all levels hold nx*ny cells),
    // summed over the levels with compensation on the host.
    rc = level_means(*h, d[1], d[2], nullptr, 2, 0);
    if (rc) return rc;
    std::vector<double> m(size_t(h->cfg.nz) * 3);
    PH_CK(cudaMemcpyAsync(m.data(), h->mean, m.size() * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    PH_CK(cudaStreamSynchronize(h->st));
    double mean[2];
    for (int f = 0; f < 2; f++) {
      CSum acc{0.0, 0.0};
      for (int k = 0; k < h->cfg.nz; k++) acc.add(m[size_t(k) * 3 + f]);
      mean[f] = (acc.s + acc.c) / h->cfg.nz;
    }
    state->u = mean[0];
    state->v = mean[1];
    if (state->counter == 0) {
      state->u0 = mean[0];
      state->v0 = mean[1];
    }
  }
  k_add_uv<<<unsigned((h->N + 255) / 256), 256, 0, h->st>>>(d[1], d[2], h->N, dt / tau * (state->u0 - state->u),
                                                            dt / tau * (state->v0 - state->v));
  PH_CK(cudaGetLastError());
  state->counter++;
  if (staged) {
    const int which[2] = {1, 2};
    return copy_back(*h, v, d, which, 2);
  }
  return PU_OK;
}

int pu_uniform_pg_wind_forcing_height(pu_physics *h, pu_state_view *v, double dt, double height, double u0, double v0,
                                      double tau) {
  if (!h || !v) return fail(PU_ERR_INVALID, "null argument");
  if (!(tau > 0)) return fail(PU_ERR_INVALID, "bad uniform_pg_wind_forcing_height parameters");
  const int nz = h->cfg.nz;
  const double dz = h->cfg.dz;
  // The lower bracketing level, found as the reference does
  // (uniform_pg_wind_forcing.h:56-57): 0 when no level centre is above height.
  int k1 = 0;
  for (int k = 0; k < nz; k++)
    if ((k + 0.5) * dz > height) {
      k1 = k - 1;
      break;
    }
  if (k1 < 0) return fail(PU_ERR_INVALID, "uniform_pg_wind_forcing_height: height below the first level centre");
  if (k1 + 1 >= nz) return fail(PU_ERR_INVALID, "uniform_pg_wind_forcing_height needs nz >= 2");
  PH_DEVICE(h->cfg.device);
  PhRange range(__func__);
  double *d[5 + PU_MAX_TRACERS];
  bool staged;
  int rc = device_arrays(*h, v, d, staged);
  if (rc) return rc;
  rc = level_means(*h, d[1], d[2], nullptr, 2, k1, 2);
  if (rc) return rc;
  const double z1 = (k1 + 0.5) * dz, z2 = (k1 + 1.5) * dz;
  const double w1 = (z2 - height) / dz, w2 = (height - z1) / dz;
  k_pg_height<<<unsigned((h->N + 255) / 256), 256, 0, h->st>>>(d[1], d[2], h->mean, h->N, w1, w2, dt / tau, u0, v0);
  PH_CK(cudaGetLastError());
  if (staged) {
    const int which[2] = {1, 2};
    return copy_back(*h, v, d, which, 2);
  }
  return PU_OK;
}

int pu_time_averager_accumulate(pu_physics *h, const pu_state_view *v, pu_time_averages *a, double elapsed_time,
                                double dt) {
  if (!h || !v || !a) return fail(PU_ERR_INVALID, "null argument");
  if (h->cfg.idTKE < 0) return fail(PU_ERR_INVALID, "the time averager needs the TKE tracer");
  double *host[13] = {a->avg_u,     a->avg_v,     a->avg_w,     a->avg_tke,    a->avg_up_up,
                      a->avg_up_vp, a->avg_up_wp, a->avg_vp_vp, a->avg_vp_wp,  a->avg_wp_wp,
                      a->long_avg_u, a->long_avg_v, a->long_avg_w};
  for (double *p : host)
    if (!p) return fail(PU_ERR_INVALID, "null time-average array");
  PH_DEVICE(h->cfg.device);
  PhRange range(__func__);
  double *d[5 + PU_MAX_TRACERS];
  bool staged;
  int rc = device_arrays(*h, v, d, staged);
  if (rc) return rc;
  TavgArrays A;
  if (staged) {
    if (!h->tavg_stage) PH_CK(cudaMalloc(&h->tavg_stage, 13 * h->N * sizeof(double)));
    for (int q = 0; q < 13; q++) {
      A.a[q] = h->tavg_stage + size_t(q) * h->N;
      PH_CK(cudaMemcpyAsync(A.a[q], host[q], h->N * sizeof(double), cudaMemcpyHostToDevice, h->st));
    }
  } else {
    for (int q = 0; q < 13; q++) A.a[q] = host[q];
  }
  // time_averager.h:78-81: inertia from this averager's elapsed time, the
  // long inertia from the coupler's.
  const double inertia = a->etime / (a->etime + dt);
  const double inertia_long = elapsed_time / (elapsed_time + dt);
  k_time_average<<<unsigned((h->N + 255) / 256), 256, 0, h->st>>>(d[1], d[2], d[3], d[5 + h->cfg.idTKE], A, h->N,
                                                                   inertia, 1 - inertia, inertia_long,
                                                                   1 - inertia_long);
  PH_CK(cudaGetLastError());
  if (staged) {
    for (int q = 0; q < 13; q++)
      PH_CK(cudaMemcpyAsync(host[q], A.a[q], h->N * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    PH_CK(cudaStreamSynchronize(h->st));
  }
  a->etime = a->etime + dt;
  return PU_OK;
}

int pu_edge_sponge_set_column(pu_physics *h, const pu_state_view *v, const int *fields, int nfields, double *column) {
  if (!h || !v || !fields || !column) return fail(PU_ERR_INVALID, "null argument");
  const int S = 5 + h->cfg.ntracers;
  if (nfields < 1 || nfields > 8) return fail(PU_ERR_INVALID, "edge sponge: 1 to 8 fields");
  for (int l = 0; l < nfields; l++)
    if (fields[l] < 0 || fields[l] >= S) return fail(PU_ERR_INVALID, "edge sponge: bad field index");
  PH_DEVICE(h->cfg.device);
  double *d[5 + PU_MAX_TRACERS];
  bool staged;
  int rc = device_arrays(*h, v, d, staged);
  if (rc) return rc;
  const int nz = h->cfg.nz;
  std::vector<double> m(size_t(nz) * 3);
  for (int l0 = 0; l0 < nfields; l0 += 3) {
    const int nf = std::min(3, nfields - l0);
    rc = level_means(*h, d[fields[l0]], nf > 1 ? d[fields[l0 + 1]] : nullptr, nf > 2 ? d[fields[l0 + 2]] : nullptr,
                     nf, 0);
    if (rc) return rc;
    PH_CK(cudaMemcpyAsync(m.data(), h->mean, m.size() * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    PH_CK(cudaStreamSynchronize(h->st));
    for (int f = 0; f < nf; f++)
      for (int k = 0; k < nz; k++) column[size_t(l0 + f) * nz + k] = m[size_t(k) * 3 + f];
  }
  return PU_OK;
}

int pu_edge_sponge_apply(pu_physics *h, pu_state_view *v, const int *fields, int nfields, const double *column,
                         double prop_x1, double prop_x2, double prop_y1, double prop_y2, long long i_beg,
                         long long j_beg, long long nx_glob, long long ny_glob) {
  if (!h || !v || !fields || !column) return fail(PU_ERR_INVALID, "null argument");
  const int S = 5 + h->cfg.ntracers;
  if (nfields < 1 || nfields > 8) return fail(PU_ERR_INVALID, "edge sponge: 1 to 8 fields");
  for (int l = 0; l < nfields; l++)
    if (fields[l] < 0 || fields[l] >= S) return fail(PU_ERR_INVALID, "edge sponge: bad field index");
  if (nx_glob < h->cfg.nx || ny_glob < h->cfg.ny || i_beg < 0 || j_beg < 0)
    return fail(PU_ERR_INVALID, "edge sponge: bad tile placement");
  PH_DEVICE(h->cfg.device);
  PhRange range(__func__);
  double *d[5 + PU_MAX_TRACERS];
  bool staged;
  int rc = device_arrays(*h, v, d, staged);
  if (rc) return rc;
  const size_t nc = size_t(nfields) * h->cfg.nz;
  if (h->column_cap < nc) {
    if (h->column) cudaFree(h->column);
    h->column = nullptr;
    h->column_cap = 0;
    PH_CK(cudaMalloc(&h->column, nc * sizeof(double)));
    h->column_cap = nc;
  }
  PH_CK(cudaMemcpyAsync(h->column, column, nc * sizeof(double), cudaMemcpyHostToDevice, h->st));
  SpongeFields F{};
  for (int l = 0; l < nfields; l++) F.f[l] = d[fields[l]];
  k_edge_sponge<<<unsigned((h->N + 255) / 256), 256, 0, h->st>>>(F, nfields, h->column, h->cfg.nx, h->cfg.ny,
                                                                 h->cfg.nz, i_beg, j_beg, nx_glob, ny_glob, prop_x1,
                                                                 prop_x2, prop_y1, prop_y2);
  PH_CK(cudaGetLastError());
  // The column is a host array: it must stay valid until the copy is done.
  PH_CK(cudaStreamSynchronize(h->st));
  if (staged) {
    int which[8];
    for (int l = 0; l < nfields; l++) which[l] = fields[l];
    return copy_back(*h, v, d, which, nfields);
  }
  return PU_OK;
}

int pu_physics_synchronize(pu_physics *h) {
  if (!h) return fail(PU_ERR_INVALID, "null handle");
  PH_DEVICE(h->cfg.device);
  PH_CK(cudaStreamSynchronize(h->st));
  return PU_OK;
}

int pu_physics_last_les_ms(pu_physics *h, double *ms) {
  if (!h || !ms) return fail(PU_ERR_INVALID, "null argument");
  PH_DEVICE(h->cfg.device);
  PH_CK(cudaEventSynchronize(h->e1));
  float f = 0;
  PH_CK(cudaEventElapsedTime(&f, h->e0, h->e1));
  *ms = f;
  return PU_OK;
}

}  // extern "C"
