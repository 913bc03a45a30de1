// pu_dycore_time_step_noalloc: the dycore's time_step for callers that cannot
// allocate device memory (declared in include/pu_dycore.h).
//
// Working memory -- the error word, the FP64 profiles, the level tables, the
// resident state, both SSPRK3 stage buffers and the x/y tendency scratch of the
// flux kernels -- comes from one file-scope device array of
// PU_NOALLOC_SCRATCH_BYTES bytes.  Every GPU that loads this library holds that
// array until the process exits.  In host code `g_noalloc_scratch` is only a
// host-side stand-in for the symbol, not a device address: its device address
// is looked up with cudaGetSymbolAddress once per device, with that device
// current, on the first call that runs on it, and that address is what the
// kernels receive.  The address is cached per device; a device reset
// (cudaDeviceReset, or a reset of the primary context) while the library is
// loaded is not supported: the cached address would outlive the context it
// belongs to.
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <string>

#include "impl.cuh"

namespace pu {

int check_config(const pu_config *c);

#define PU_DECL(tag)                                                                                     \
  size_t noalloc_bytes_##tag(const pu_config &c);                                                        \
  int noalloc_time_step_##tag(const pu_config &c, unsigned char *scratch, const double *dc, const double *tc, \
                              const double *pc, pu_state_view *v, double dt_phys, int *ncycles);
PU_DECL(f32_1) PU_DECL(f32_2) PU_DECL(f32_3) PU_DECL(f32_4)
#undef PU_DECL

}  // namespace pu

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[PU_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
// Device address of g_noalloc_scratch per device ordinal.  Two host threads
// making their first call on one device may both look it up; they store the
// same value, and the atomic makes that race well defined.
std::atomic<unsigned char *> g_scratch_addr[kMaxDevices] = {};

int fail(int code, const std::string &msg) {
  pu::set_error(msg);
  return code;
}

// Makes `dev` current for the call and restores the previous device after it;
// `ok` is false when the switch failed (nothing may then run on `dev`).
struct DeviceGuard {
  int prev = -1;
  cudaError_t status = cudaSuccess;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) status = cudaSetDevice(dev);
  }
  bool ok() const { return status == cudaSuccess; }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

}  // namespace

extern "C" int pu_dycore_time_step_noalloc(const pu_config *cfg, const double *dens_cells, const double *theta_cells,
                                           const double *pressure_cells, pu_state_view *coupler, double dt_phys,
                                           int *ncycles) {
  int rc = pu::check_config(cfg);
  if (rc) return rc;
  if (!coupler || !dens_cells || !theta_cells || !pressure_cells) return fail(PU_ERR_INVALID, "null argument");
  if (!(dt_phys > 0)) return fail(PU_ERR_INVALID, "dt_phys must be positive");
  if (cfg->precision != PU_F32) return fail(PU_ERR_UNSUPPORTED, "the no-allocation time step is FP32 only");
  size_t need = 0;
  switch (cfg->ntracers) {
    case 1: need = pu::noalloc_bytes_f32_1(*cfg); break;
    case 2: need = pu::noalloc_bytes_f32_2(*cfg); break;
    case 3: need = pu::noalloc_bytes_f32_3(*cfg); break;
    default: need = pu::noalloc_bytes_f32_4(*cfg); break;
  }
  if (need > size_t(PU_NOALLOC_SCRATCH_BYTES))
    return fail(PU_ERR_UNSUPPORTED, "grid too large for the no-allocation time step: it needs " +
                                        std::to_string(need) + " bytes of scratch and has " +
                                        std::to_string(size_t(PU_NOALLOC_SCRATCH_BYTES)));
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(PU_ERR_CUDA, "no CUDA device");
  if (cfg->device < 0 || cfg->device >= ndev || cfg->device >= kMaxDevices)
    return fail(PU_ERR_INVALID, "bad device ordinal");
  DeviceGuard g(cfg->device);
  if (!g.ok()) return fail(PU_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(g.status));
  // Coupler arrays must already be on the device: there is no staging buffer.
  const double *arrs[5] = {coupler->rho_d, coupler->uvel, coupler->vvel, coupler->wvel, coupler->temp};
  for (int a = 0; a < 5 + cfg->ntracers; a++) {
    const double *p = a < 5 ? arrs[a] : coupler->tracers[a - 5];
    if (!p) return fail(PU_ERR_INVALID, "coupler view has a null array");
    const int m = coupler->mem == PU_MEM_AUTO ? pu::resolve_mem(PU_MEM_AUTO, p) : coupler->mem;
    if (m != PU_MEM_DEVICE) return fail(PU_ERR_INVALID, "the no-allocation time step needs device-resident coupler arrays");
  }
  pu_state_view v = *coupler;
  v.mem = PU_MEM_DEVICE;
  // Set-up, once per device: the device address of the scratch array.
  unsigned char *scratch = g_scratch_addr[cfg->device].load(std::memory_order_acquire);
  if (!scratch) {
    void *addr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
    if (e != cudaSuccess) return fail(PU_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    scratch = static_cast<unsigned char *>(addr);
    g_scratch_addr[cfg->device].store(scratch, std::memory_order_release);
  }
  switch (cfg->ntracers) {
    case 1: return pu::noalloc_time_step_f32_1(*cfg, scratch, dens_cells, theta_cells, pressure_cells, &v, dt_phys, ncycles);
    case 2: return pu::noalloc_time_step_f32_2(*cfg, scratch, dens_cells, theta_cells, pressure_cells, &v, dt_phys, ncycles);
    case 3: return pu::noalloc_time_step_f32_3(*cfg, scratch, dens_cells, theta_cells, pressure_cells, &v, dt_phys, ncycles);
    default: return pu::noalloc_time_step_f32_4(*cfg, scratch, dens_cells, theta_cells, pressure_cells, &v, dt_phys, ncycles);
  }
}
