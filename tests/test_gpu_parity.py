"""GPU parity: libpu_dycore against the CPU oracle on identical inputs.

* FP64 build vs the FP64 oracle: the same algorithm in double; the only
  differences are rearranged arithmetic (difference/LDL^T form of the
  smoothness indicator, perturbation storage, reciprocal-multiply), at the
  1e-16 level.  WENO's nonlinear weights amplify them where the stencils are
  nearly uniform, so the bound is 1e-7 of the change the steps produce (L2)
  and 1e-6 (Linf) -- ten times below FP32 round-off.
* FP32 build vs the REF oracle, which is bit-identical to the reference's own
  path (FP64 state, FP32 stencil arithmetic).  The FP32 build also stores the
  state in FP32 (as departures from the hydrostatic background), so each
  stage rounds every prognostic at 2^-24 of its departure.  Tolerance after
  4 steps: L2 error <= 1e-5 and Linf error <= 1e-4 of the field's departure
  from the hydrostatic background.
* Over a longer run (60 steps of a warm bubble), the FP32 build must be as
  close to the FP64 oracle as the reference's own path is: L2 error against
  FP64, relative to the change the run produced, at most 3x the reference's
  plus 1e-6.
"""
import numpy as np
import pytest

from porturb_b200 import cases
from helpers import background, gpu_run, oracle_run, rel_change_err, rel_pert_err

pytestmark = pytest.mark.gpu

CASES = {
    "mixed_immersed": lambda: cases.small_mixed(),
    "plain_one_tracer": lambda: cases.small_mixed(immersed=False, ntr=1),
    "three_tracers": lambda: cases.small_mixed(ntr=3),
    "precursor_xy": lambda: cases.small_mixed(bc_x="precursor", bc_y="precursor"),
    "periodic_z": lambda: cases.small_mixed(bc_z="periodic", immersed=False),
    "coriolis": lambda: cases.small_mixed(latitude=43.29),
    "linear_edges": lambda: cases.small_mixed(weno_all=False, immersed=False),
    "sim2d": lambda: cases.small_mixed(ny=1, nx=24, nz=16),
    "bubble_small": lambda: cases.warm_bubble(nx=64, ny=4, nz=32, xlen=5000.0, ylen=312.5, zlen=2500.0,
                                              radius=500.0, x0=2500.0, z0=600.0),
}
NSTEPS = 4


@pytest.mark.parametrize("name", sorted(CASES))
def test_f64_build_matches_f64_oracle(name, oracle_lib, gpu_lib):
    case = CASES[name]()
    dt = 0.9 * oracle_lib.Dycore(case, "f64").compute_time_step()
    st_o, tr_o, cells, (st0, tr0) = oracle_run(case, "f64", NSTEPS, dt)
    st_g, tr_g, _ = gpu_run(case, "f64", NSTEPS, dt, hydro=cells)
    errs = rel_change_err(np.concatenate([st_g, tr_g]), np.concatenate([st_o, tr_o]), np.concatenate([st0, tr0]))
    print(name, "f64 rel-to-change errors (L2, Linf):", ["%.2e/%.2e" % e for e in errs])
    for e2, ei in errs:
        assert e2 < 1e-7 and ei < 1e-6


@pytest.mark.parametrize("name", sorted(CASES))
def test_f32_build_matches_reference_path(name, oracle_lib, gpu_lib):
    case = CASES[name]()
    dt = 0.9 * oracle_lib.Dycore(case, "ref").compute_time_step()
    st_r, tr_r, cells, (st0, tr0) = oracle_run(case, "ref", NSTEPS, dt)
    st_64, tr_64, _, _ = oracle_run(case, "f64", NSTEPS, dt, hydro=cells)
    st_g, tr_g, _ = gpu_run(case, "f32", NSTEPS, dt, hydro=cells)
    base = np.concatenate([st0, tr0])
    g, r, f = np.concatenate([st_g, tr_g]), np.concatenate([st_r, tr_r]), np.concatenate([st_64, tr_64])
    bg = background(case, cells, tr_g.shape[0])
    e_pert = rel_pert_err(g, r, bg)
    print(name, "gpu32-vs-ref (of departure, L2/Linf):", ["%.1e/%.1e" % e for e in e_pert])
    print(name, "gpu32-vs-f64 (of change):", ["%.1e" % e[0] for e in rel_change_err(g, f, base)],
          " ref-vs-f64 (of change):", ["%.1e" % e[0] for e in rel_change_err(r, f, base)])
    for e2, ei in e_pert:
        assert e2 < 1e-5 and ei < 1e-4


def test_f32_long_run_as_accurate_as_reference(oracle_lib, gpu_lib):
    case = cases.warm_bubble(nx=64, ny=4, nz=32, xlen=5000.0, ylen=312.5, zlen=2500.0, radius=500.0,
                             x0=2500.0, z0=600.0, cfl=0.8)
    n = 60
    dt = oracle_lib.Dycore(case, "ref").compute_time_step()
    st_r, tr_r, cells, (st0, tr0) = oracle_run(case, "ref", n, dt)
    st_64, tr_64, _, _ = oracle_run(case, "f64", n, dt, hydro=cells)
    st_g, tr_g, _ = gpu_run(case, "f32", n, dt, hydro=cells)
    e_g = rel_change_err(st_g, st_64, st0)
    e_r = rel_change_err(st_r, st_64, st0)
    bg = background(case, cells, 0)
    p_g = rel_pert_err(st_g, st_64, bg)
    p_r = rel_pert_err(st_r, st_64, bg)
    print("long run gpu32-vs-f64 (of change):", ["%.2e" % e[0] for e in e_g],
          " ref-vs-f64:", ["%.2e" % e[0] for e in e_r])
    print("long run gpu32-vs-f64 (of departure):", ["%.2e" % e[0] for e in p_g],
          " ref-vs-f64:", ["%.2e" % e[0] for e in p_r])
    # Momentum and rho*theta: as close to FP64 as the reference's own path.
    for f in (1, 3, 4):
        assert e_g[f][0] <= 3 * e_r[f][0] + 1e-6
    # Density: bounded by FP32 storage of its departure from hydrostatic balance.
    for f in range(5):
        assert p_g[f][0] < 1e-5
