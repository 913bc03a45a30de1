/* C interface of the CPU oracles (test infrastructure only).
 *
 * Two libraries export this interface with different symbol prefixes:
 *   orc_*  oracle/_build/liboracle.so      -- this project's restatement of the
 *                                            reference dycore (variants REF and F64)
 *   ref_*  oracle/_ref/libporturb_ref.so   -- the reference's own dycore headers
 *                                            (model/modules/dynamics_rk.h,
 *                                            helpers/WenoLimiter.h, helpers/TransformMatrices.h)
 *                                            compiled against a small single-rank shim
 *
 * Both take the same configuration and the same coupler-side arrays, so tests
 * can compare them element by element.  All 3-D arrays are C-order (nz,ny,nx)
 * doubles, tracers are (ntr,nz,ny,nx).
 */
#pragma once

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_TRACERS 16

enum { ORC_BC_PERIODIC = 0, ORC_BC_PRECURSOR = 1, ORC_BC_WALL = 2 };
enum { ORC_VARIANT_REF = 0, ORC_VARIANT_F64 = 1 };

typedef struct orc_config {
  int nx, ny, nz, ntr;
  double xlen, ylen, zlen;
  int tracer_positive[ORC_MAX_TRACERS];
  int tracer_adds_mass[ORC_MAX_TRACERS];
  int idWV;
  /* Options as the reference's coupler holds them (sc_init.h:31-51 derives
   * gamma_d and C0 from R_d, cp_d and p0). */
  double R_d, R_v, cp_d, gamma_d, C0, grav;
  double cfl, immersed_power, latitude;
  int bc_x, bc_y, bc_z;
  int enable_gravity, weno_all;
} orc_config;

#ifdef __cplusplus
}
#endif
