// C entry points of libpu_dycore (declared in include/pu_dycore.h).
#include <cuda_runtime.h>

#include <cmath>
#include <memory>
#include <string>

#include "impl.cuh"

namespace pu {

namespace {
thread_local std::string g_error;
}
void set_error(const std::string &msg) { g_error = msg; }

#define PU_DECL(tag) ImplBase *make_impl_##tag();
PU_DECL(f32_1) PU_DECL(f32_2) PU_DECL(f32_3) PU_DECL(f32_4)
PU_DECL(f64_1) PU_DECL(f64_2) PU_DECL(f64_3) PU_DECL(f64_4)
#undef PU_DECL

static ImplBase *make_impl(int precision, int ntr) {
  if (precision == PU_F32) {
    switch (ntr) {
      case 1: return make_impl_f32_1();
      case 2: return make_impl_f32_2();
      case 3: return make_impl_f32_3();
      case 4: return make_impl_f32_4();
    }
  } else {
    switch (ntr) {
      case 1: return make_impl_f64_1();
      case 2: return make_impl_f64_2();
      case 3: return make_impl_f64_3();
      case 4: return make_impl_f64_4();
    }
  }
  return nullptr;
}

}  // namespace pu

using pu::set_error;

struct pu_dycore {
  std::unique_ptr<pu::ImplBase> impl;
  int device = 0;
};

namespace {

int fail(int code, const std::string &msg) {
  set_error(msg);
  return code;
}

// Every entry point runs with the handle's device current and restores the
// caller's device afterwards.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

}  // namespace

namespace pu {
int check_config(const pu_config *c) {
  if (!c) return fail(PU_ERR_INVALID, "null config");
  if (c->nx < 1 || c->ny < 1 || c->nz < 1) return fail(PU_ERR_INVALID, "grid dimensions must be positive");
  if (c->nx < PU_HS + 1 && c->bc_x == PU_BC_PERIODIC)
    return fail(PU_ERR_UNSUPPORTED, "nx must exceed the halo width for periodic x");
  if (c->nz < PU_HS) return fail(PU_ERR_UNSUPPORTED, "nz must be at least the halo width");
  if (!(c->dx > 0 && c->dy > 0 && c->dz > 0)) return fail(PU_ERR_INVALID, "grid spacing must be positive");
  if (c->ntracers < 1 || c->ntracers > PU_MAX_TRACERS)
    return fail(PU_ERR_UNSUPPORTED, "the dycore needs 1..PU_MAX_TRACERS tracers (water_vapor is required)");
  if (c->idWV < 0 || c->idWV >= c->ntracers) return fail(PU_ERR_INVALID, "idWV must index the water_vapor tracer");
  if (c->bc_x != PU_BC_PERIODIC && c->bc_x != PU_BC_PRECURSOR) return fail(PU_ERR_INVALID, "bc_x must be periodic or precursor");
  if (c->bc_y != PU_BC_PERIODIC && c->bc_y != PU_BC_PRECURSOR) return fail(PU_ERR_INVALID, "bc_y must be periodic or precursor");
  if (c->bc_z != PU_BC_WALL && c->bc_z != PU_BC_PERIODIC)
    return fail(PU_ERR_INVALID, "ERROR: Specified invalid bc_z in coupler options");
  if (c->precision != PU_F32 && c->precision != PU_F64) return fail(PU_ERR_INVALID, "precision must be PU_F32 or PU_F64");
  if (c->weno_mode != PU_WENO_PLAIN && c->weno_mode != PU_WENO_LEARNED) return fail(PU_ERR_INVALID, "bad WENO mode");
  if (!(c->gamma_d > 1 && c->C0 > 0 && c->R_d > 0 && c->cfl > 0)) return fail(PU_ERR_INVALID, "bad thermodynamic options");
  if (c->z_chunk < 0) return fail(PU_ERR_INVALID, "z_chunk must be >= 0");
  return PU_OK;
}
}  // namespace pu

namespace {
using pu::check_config;
}  // namespace

extern "C" {

int pu_version(void) { return 100; }

const char *pu_last_error(void) { return pu::g_error.c_str(); }

int pu_dycore_create(const pu_config *cfg, pu_dycore **out) {
  if (!out) return fail(PU_ERR_INVALID, "null output pointer");
  *out = nullptr;
  int rc = check_config(cfg);
  if (rc) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(PU_ERR_CUDA, "no CUDA device");
  if (cfg->device < 0 || cfg->device >= ndev) return fail(PU_ERR_INVALID, "bad device ordinal");
  DeviceGuard g(cfg->device);
  std::unique_ptr<pu_dycore> h(new pu_dycore);
  h->device = cfg->device;
  h->impl.reset(pu::make_impl(cfg->precision, cfg->ntracers));
  if (!h->impl) return fail(PU_ERR_UNSUPPORTED, "no implementation for this precision/tracer count");
  auto &I = *h->impl;
  I.cfg = *cfg;
  I.st = static_cast<cudaStream_t>(cfg->stream);
  I.ntr = cfg->ntracers;
  I.N = size_t(cfg->nx) * cfg->ny * cfg->nz;
  I.NP = size_t(cfg->nx) * cfg->ny;
  I.nzh = cfg->nz + 2 * PU_HS;
  I.weno_mode = cfg->weno_mode;
  rc = I.alloc();
  if (rc) return rc;
  *out = h.release();
  return PU_OK;
}

int pu_dycore_destroy(pu_dycore *h) {
  if (!h) return PU_OK;
  {
    DeviceGuard g(h->device);
    if (h->impl) cudaStreamSynchronize(h->impl->st);
    h->impl.reset();
  }
  delete h;
  return PU_OK;
}

int pu_dycore_init(pu_dycore *h, const pu_state_view *coupler, const double *immersed_proportion, int mem) {
  if (!h || !coupler) return fail(PU_ERR_INVALID, "null argument");
  DeviceGuard g(h->device);
  return h->impl->init(coupler, immersed_proportion, mem);
}

int pu_dycore_init_windmill(pu_dycore *h, const pu_state_view *coupler, const double *immersed_proportion,
                            const double *windmill_proj_weight, int mem) {
  if (!h || !coupler) return fail(PU_ERR_INVALID, "null argument");
  if (windmill_proj_weight && !immersed_proportion)
    return fail(PU_ERR_INVALID, "windmill_proj_weight needs immersed_proportion");
  DeviceGuard g(h->device);
  return h->impl->init(coupler, immersed_proportion, mem, windmill_proj_weight);
}

int pu_dycore_compute_time_step(const pu_dycore *h, double *dt) {
  if (!h || !dt) return fail(PU_ERR_INVALID, "null argument");
  const pu_config &c = h->impl->cfg;
  const double maxwave = 350 + 100;
  *dt = c.cfl * std::fmin(std::fmin(c.dx, c.dy), c.dz) / maxwave;
  return PU_OK;
}

int pu_dycore_load_state(pu_dycore *h, const pu_state_view *coupler) {
  if (!h || !coupler) return fail(PU_ERR_INVALID, "null argument");
  if (!h->impl->inited) return fail(PU_ERR_STATE, "pu_dycore_init has not been called");
  DeviceGuard g(h->device);
  return h->impl->load_state(coupler);
}

int pu_dycore_store_state(pu_dycore *h, pu_state_view *coupler) {
  if (!h || !coupler) return fail(PU_ERR_INVALID, "null argument");
  if (!h->impl->inited) return fail(PU_ERR_STATE, "pu_dycore_init has not been called");
  DeviceGuard g(h->device);
  return h->impl->store_state(coupler);
}

int pu_dycore_advance(pu_dycore *h, double dt_dyn, int nsteps) {
  if (!h) return fail(PU_ERR_INVALID, "null handle");
  if (!h->impl->inited) return fail(PU_ERR_STATE, "pu_dycore_init has not been called");
  if (!(dt_dyn > 0) || nsteps < 0) return fail(PU_ERR_INVALID, "dt must be positive and nsteps non-negative");
  DeviceGuard g(h->device);
  return h->impl->advance(dt_dyn, nsteps);
}

int pu_dycore_time_step(pu_dycore *h, pu_state_view *coupler, double dt_phys, int *ncycles) {
  if (!h || !coupler) return fail(PU_ERR_INVALID, "null argument");
  if (!h->impl->inited) return fail(PU_ERR_STATE, "pu_dycore_init has not been called");
  if (!(dt_phys > 0)) return fail(PU_ERR_INVALID, "dt_phys must be positive");
  DeviceGuard g(h->device);
  double dt_dyn;
  pu_dycore_compute_time_step(h, &dt_dyn);
  const int n = (int)std::ceil(dt_phys / dt_dyn);
  dt_dyn = dt_phys / n;
  int rc = h->impl->load_state(coupler);
  if (!rc) rc = h->impl->advance(dt_dyn, n);
  if (!rc) rc = h->impl->store_state(coupler);
  if (ncycles) *ncycles = n;
  return rc;
}

int pu_dycore_get_conserved(pu_dycore *h, double *state, double *tracers, int mem) {
  if (!h || !state) return fail(PU_ERR_INVALID, "null argument");
  if (!h->impl->inited) return fail(PU_ERR_STATE, "pu_dycore_init has not been called");
  DeviceGuard g(h->device);
  return h->impl->get_conserved(state, tracers, mem);
}

int pu_dycore_set_conserved(pu_dycore *h, const double *state, const double *tracers, int mem) {
  if (!h || !state || !tracers) return fail(PU_ERR_INVALID, "null argument");
  if (!h->impl->inited) return fail(PU_ERR_STATE, "pu_dycore_init has not been called");
  DeviceGuard g(h->device);
  return h->impl->set_conserved(state, tracers, mem);
}

int pu_dycore_get_hydrostasis(pu_dycore *h, double *dc, double *tc, double *pc, double *de, double *te, double *pe) {
  if (!h) return fail(PU_ERR_INVALID, "null handle");
  if (!h->impl->inited) return fail(PU_ERR_STATE, "pu_dycore_init has not been called");
  DeviceGuard g(h->device);
  auto &I = *h->impl;
  const int nzh = I.nzh, ne = I.cfg.nz + 1;
  double *dst_c[3] = {dc, tc, pc}, *dst_e[3] = {de, te, pe};
  for (int q = 0; q < 3; q++) {
    if (dst_c[q] && cudaMemcpyAsync(dst_c[q], I.cells + q * nzh, nzh * sizeof(double), cudaMemcpyDeviceToHost, I.st))
      return fail(PU_ERR_CUDA, "copy of hydrostatic profiles failed");
    if (dst_e[q] && cudaMemcpyAsync(dst_e[q], I.edges + q * ne, ne * sizeof(double), cudaMemcpyDeviceToHost, I.st))
      return fail(PU_ERR_CUDA, "copy of hydrostatic profiles failed");
  }
  if (cudaStreamSynchronize(I.st) != cudaSuccess) return fail(PU_ERR_CUDA, "stream synchronize failed");
  return PU_OK;
}

int pu_dycore_set_hydrostasis(pu_dycore *h, const double *dens, const double *theta, const double *pressure) {
  if (!h || !dens || !theta || !pressure) return fail(PU_ERR_INVALID, "null argument");
  if (!h->impl->inited) return fail(PU_ERR_STATE, "pu_dycore_init has not been called");
  DeviceGuard g(h->device);
  return h->impl->set_hydrostasis(dens, theta, pressure);
}

int pu_dycore_diagnostics(pu_dycore *h, pu_diag *out) {
  if (!h || !out) return fail(PU_ERR_INVALID, "null argument");
  if (!h->impl->inited) return fail(PU_ERR_STATE, "pu_dycore_init has not been called");
  DeviceGuard g(h->device);
  return h->impl->diagnostics(out);
}

int pu_dycore_perturbations(pu_dycore *h, const pu_state_view *v, double *density_pert, double *theta_pert,
                            double *pressure_pert, int mem) {
  if (!h || !v || !density_pert || !theta_pert || !pressure_pert) return fail(PU_ERR_INVALID, "null argument");
  if (!h->impl->inited) return fail(PU_ERR_STATE, "pu_dycore_init has not been called");
  DeviceGuard g(h->device);
  return h->impl->perturbations(v, density_pert, theta_pert, pressure_pert, mem);
}

int pu_dycore_synchronize(pu_dycore *h) {
  if (!h) return fail(PU_ERR_INVALID, "null handle");
  DeviceGuard g(h->device);
  return h->impl->check_err();
}

long long pu_dycore_kernel_launches(const pu_dycore *h) { return h ? h->impl->launches : 0; }

int pu_dycore_learned_harvest(pu_dycore *h, long long n, unsigned long long seed) {
  if (!h || n <= 0) return fail(PU_ERR_INVALID, "bad argument");
  if (!h->impl->inited) return fail(PU_ERR_STATE, "pu_dycore_init has not been called");
  DeviceGuard g(h->device);
  return h->impl->ml_harvest(long(n), seed);
}

int pu_dycore_learned_train(pu_dycore *h, int steps, int batch, double lr, unsigned long long seed,
                            pu_learn_stats *out) {
  if (!h || steps < 0 || batch <= 0 || !(lr > 0)) return fail(PU_ERR_INVALID, "bad argument");
  DeviceGuard g(h->device);
  int rc = h->impl->ml_alloc();
  if (rc) return rc;
  return h->impl->ml_train(steps, batch, lr, seed, out);
}

int pu_dycore_learned_get_weights(pu_dycore *h, float *theta) {
  if (!h || !theta) return fail(PU_ERR_INVALID, "null argument");
  DeviceGuard g(h->device);
  int rc = h->impl->ml_alloc();
  if (rc) return rc;
  return h->impl->ml_get(theta);
}

int pu_dycore_learned_set_weights(pu_dycore *h, const float *theta) {
  if (!h || !theta) return fail(PU_ERR_INVALID, "null argument");
  DeviceGuard g(h->device);
  int rc = h->impl->ml_alloc();
  if (rc) return rc;
  return h->impl->ml_set(theta);
}

int pu_dycore_learned_eval(pu_dycore *h, const float *x, long long n, float *wl, float *wr, int use_mma) {
  if (!h || !x || !wl || n <= 0) return fail(PU_ERR_INVALID, "bad argument");
  DeviceGuard g(h->device);
  int rc = h->impl->ml_alloc();
  if (rc) return rc;
  return h->impl->ml_eval(x, long(n), wl, wr, use_mma);
}

int pu_dycore_learned_gradient(pu_dycore *h, const float *x, const float *t, long long n, float *grad,
                               double *loss) {
  if (!h || !x || !t || !grad || n <= 0 || n > (1 << 20)) return fail(PU_ERR_INVALID, "bad argument");
  DeviceGuard g(h->device);
  int rc = h->impl->ml_alloc();
  if (rc) return rc;
  return h->impl->ml_gradient(x, t, long(n), grad, loss);
}

int pu_dycore_set_weno_mode(pu_dycore *h, int mode) {
  if (!h) return fail(PU_ERR_INVALID, "null handle");
  if (mode != PU_WENO_PLAIN && mode != PU_WENO_LEARNED) return fail(PU_ERR_INVALID, "bad WENO mode");
  if (mode == PU_WENO_LEARNED) {
    if (h->impl->cfg.precision != PU_F32) return fail(PU_ERR_UNSUPPORTED, "learned weights run in the FP32 build only");
    if (!h->impl->cfg.weno_all)
      return fail(PU_ERR_UNSUPPORTED, "learned weights replace the limiter of weno_all; this dycore uses linear edges");
    if (!h->impl->ml_ready) return fail(PU_ERR_STATE, "learned weights are neither trained nor loaded");
  }
  h->impl->weno_mode = mode;
  return PU_OK;
}

int pu_dycore_learned_set_threshold(pu_dycore *h, double max_jump) {
  if (!h) return fail(PU_ERR_INVALID, "null handle");
  if (!(max_jump >= 0)) return fail(PU_ERR_INVALID, "the jump threshold must be >= 0");
  h->impl->ml_jump = float(max_jump);
  return PU_OK;
}

int pu_dycore_learned_counts(pu_dycore *h, long long *learned, long long *fallback) {
  if (!h) return fail(PU_ERR_INVALID, "null handle");
  DeviceGuard g(h->device);
  unsigned long long c[2] = {0, 0};
  auto &I = *h->impl;
  if (I.ml_counts) {
    if (cudaMemcpyAsync(c, I.ml_counts, sizeof(c), cudaMemcpyDeviceToHost, I.st) != cudaSuccess ||
        cudaMemsetAsync(I.ml_counts, 0, sizeof(c), I.st) != cudaSuccess || cudaStreamSynchronize(I.st) != cudaSuccess)
      return fail(PU_ERR_CUDA, "reading the learned-path counters failed");
  }
  if (learned) *learned = (long long)c[0];
  if (fallback) *fallback = (long long)c[1];
  return PU_OK;
}

int pu_dycore_profile(pu_dycore *h, int enable) {
  if (!h) return fail(PU_ERR_INVALID, "null handle");
  DeviceGuard g(h->device);
  if (cudaStreamSynchronize(h->impl->st) != cudaSuccess) return fail(PU_ERR_CUDA, "stream synchronize failed");
  h->impl->prof_reset();
  h->impl->profiling = enable != 0;
  return PU_OK;
}

int pu_dycore_profile_read(pu_dycore *h, pu_profile *out) {
  if (!h || !out) return fail(PU_ERR_INVALID, "null argument");
  DeviceGuard g(h->device);
  return h->impl->prof_read(out);
}

}  // extern "C"
