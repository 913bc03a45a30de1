// One instantiation of the dycore implementation; compiled once per stencil
// type and tracer count with -DPU_REAL=<float|double> -DPU_NTR=<n> -DPU_TAG=<name>.
#include "impl.cuh"

#define PU_CAT2(a, b) a##b
#define PU_CAT(a, b) PU_CAT2(a, b)

namespace pu {
ImplBase *PU_CAT(make_impl_, PU_TAG)() { return new Impl<PU_REAL, PU_NTR>(); }
}  // namespace pu
