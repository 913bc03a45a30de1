// One instantiation of the dycore implementation; compiled once per stencil
// type and tracer count with -DPU_REAL=<float|double> -DPU_NTR=<n> -DPU_TAG=<name>.
#include "impl.cuh"

#define PU_CAT2(a, b) a##b
#define PU_CAT(a, b) PU_CAT2(a, b)

namespace pu {
ImplBase *PU_CAT(make_impl_, PU_TAG)() { return new Impl<PU_REAL, PU_NTR>(); }

size_t PU_CAT(noalloc_bytes_, PU_TAG)(const pu_config &c) { return Impl<PU_REAL, PU_NTR>::scratch_bytes(c); }

int PU_CAT(noalloc_time_step_, PU_TAG)(const pu_config &c, unsigned char *scratch, const double *dc, const double *tc,
                                       const double *pc, pu_state_view *v, double dt_phys, int *ncycles) {
  return Impl<PU_REAL, PU_NTR>::noalloc_time_step(c, scratch, dc, tc, pc, v, dt_phys, ncycles);
}
}  // namespace pu
