"""The optional windmill projection weight of the dycore's init
(dynamics_rk.h:1019-1025): added to a copy of immersed_proportion before the
immersed halos, flags and relaxation time scales are built.  A turbine-like
projection makes a disk of small fractional proportions, so a wide region
takes the immersed stencil paths (zero-derivative extrapolation, no mapping
of the weights) and weak relaxation.

* pu_dycore_init_windmill against the CPU oracle given the summed
  proportion: FP64 build within 1e-7 (L2) / 1e-6 (Linf) of the change the
  steps make, FP32 build within 1e-5 / 1e-4 of the departure from the
  hydrostatic background against the reference path -- the bounds of the
  other parity cases.
* The Coupler front end picks the entry up, leaves the coupler's
  immersed_proportion untouched, and equals a handle initialised with the
  sum, bit for bit.
* A projection without immersed_proportion is an error, as the reference's
  missing entry is."""
import ctypes as C

import numpy as np
import pytest

from porturb_b200 import Dycore, Dynamics_Euler_Stratified_WenoFV, assign_coupler_state, capi, case_coupler, cases
from porturb_b200.dycore import make_view
from helpers import background, oracle_run, rel_change_err, rel_pert_err

pytestmark = pytest.mark.gpu
NSTEPS = 4


def _projection(case, i0=8, hub=(8.0, 7.5), radius=6.0, peak=0.3):
    """A rotor disk two cells thick in x: peak*exp(-(r/radius)^2) inside the
    radius, zero outside (the shape of an actuator-disk projection)."""
    w = np.zeros((case.nz, case.ny, case.nx))
    k, j = np.meshgrid(np.arange(case.nz) + 0.5, np.arange(case.ny) + 0.5, indexing="ij")
    r = np.hypot(k - hub[0], j - hub[1])
    disk = np.where(r < radius, peak * np.exp(-(r / radius) ** 2), 0.0)
    w[:, :, i0] = disk
    w[:, :, i0 + 1] = 0.5 * disk
    return w


def _cases():
    case = cases.small_mixed(nx=24, ny=16, nz=16)
    proj = _projection(case)
    prop = case.immersed_proportion.copy()
    summed = cases.small_mixed(nx=24, ny=16, nz=16)
    summed.immersed_proportion[...] = prop + proj
    return case, prop, proj, summed


def _gpu(case, prop, proj, precision, dt, cells):
    g = Dycore.from_case(case, precision=precision)
    rd, u, v, w, T, trc = [np.ascontiguousarray(a) for a in case.coupler_arrays(perturbed=False)]
    g.init(rd, u, v, w, T, list(trc), np.ascontiguousarray(prop), np.ascontiguousarray(proj))
    g.set_hydrostasis(*cells)
    rd, u, v, w, T, trc = [np.ascontiguousarray(a) for a in case.coupler_arrays(perturbed=True)]
    g.load_state(rd, u, v, w, T, list(trc))
    g.advance(dt, NSTEPS)
    g.synchronize()
    st, tr = g.get_conserved()
    g.close()
    return st, tr


def test_f64_build_matches_f64_oracle(oracle_lib, gpu_lib):
    case, prop, proj, summed = _cases()
    dt = 0.9 * oracle_lib.Dycore(summed, "f64").compute_time_step()
    st_o, tr_o, cells, (st0, tr0) = oracle_run(summed, "f64", NSTEPS, dt)
    st_g, tr_g = _gpu(case, prop, proj, "f64", dt, cells)
    errs = rel_change_err(np.concatenate([st_g, tr_g]), np.concatenate([st_o, tr_o]), np.concatenate([st0, tr0]))
    print("windmill f64 rel-to-change errors (L2, Linf):", ["%.2e/%.2e" % e for e in errs])
    for e2, ei in errs:
        assert e2 < 1e-7 and ei < 1e-6


def test_f32_build_matches_reference_path(oracle_lib, gpu_lib):
    case, prop, proj, summed = _cases()
    dt = 0.9 * oracle_lib.Dycore(summed, "ref").compute_time_step()
    st_r, tr_r, cells, _ = oracle_run(summed, "ref", NSTEPS, dt)
    st_g, tr_g = _gpu(case, prop, proj, "f32", dt, cells)
    g, r = np.concatenate([st_g, tr_g]), np.concatenate([st_r, tr_r])
    e_pert = rel_pert_err(g, r, background(summed, cells, tr_g.shape[0]))
    print("windmill gpu32-vs-ref (of departure, L2/Linf):", ["%.1e/%.1e" % e for e in e_pert])
    for e2, ei in e_pert:
        assert e2 < 1e-5 and ei < 1e-4


def test_coupler_front_end_adds_the_projection(gpu_lib):
    case, prop, proj, summed = _cases()
    c = case_coupler(case)
    c.register_and_allocate("windmill_proj_weight", "", proj.shape)
    c.get("windmill_proj_weight")[...] = proj
    dyn = Dynamics_Euler_Stratified_WenoFV()
    dyn.init(c)
    assert np.array_equal(c.get("immersed_proportion"), prop)
    assign_coupler_state(c, case, perturbed=True)
    dt = dyn.compute_time_step(c)
    for _ in range(2):
        dyn.time_step(c, 2 * dt)
    got = np.stack([c.get(n) for n in ("density_dry", "uvel", "vvel", "wvel", "temp")])

    g = Dycore.from_case(summed, precision="f32")
    rd, u, v, w, T, trc = [np.ascontiguousarray(a) for a in summed.coupler_arrays(perturbed=False)]
    g.init(rd, u, v, w, T, list(trc), np.ascontiguousarray(prop + proj))
    rd, u, v, w, T, trc = [np.ascontiguousarray(a) for a in summed.coupler_arrays(perturbed=True)]
    for _ in range(2):
        g.time_step(rd, u, v, w, T, list(trc), 2 * dt)
    g.close()
    assert np.array_equal(got, np.stack([rd, u, v, w, T]))


def test_projection_without_proportion_is_an_error(gpu_lib):
    case, prop, proj, _ = _cases()
    g = Dycore.from_case(case, precision="f32")
    rd, u, v, w, T, trc = [np.ascontiguousarray(a) for a in case.coupler_arrays(perturbed=False)]
    view = make_view(rd, u, v, w, T, list(trc))
    rc = g.lib.pu_dycore_init_windmill(g.h, C.byref(view), None, np.ascontiguousarray(proj).ctypes.data,
                                       capi.PU_MEM_HOST)
    assert rc == capi.PU_ERR_INVALID
    with pytest.raises(ValueError):
        g.init(rd, u, v, w, T, list(trc), None, np.ascontiguousarray(proj))
    g.close()
