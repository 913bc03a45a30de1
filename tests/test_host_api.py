"""Host-side mirror of the reference's Coupler / module API (no GPU calls)."""
import numpy as np
import pytest

import pyoracle
from porturb_b200 import Coupler, Dynamics_Euler_Stratified_WenoFV, PortUrbError, capi, case_coupler, cases


def test_options_are_typed_and_required():
    c = Coupler()
    with pytest.raises(KeyError):
        c.get_option("R_d")
    assert c.get_option("cfl", 0.6) == 0.6
    c.set_option("cfl", 0.8)
    assert c.get_option("cfl") == 0.8
    with pytest.raises(TypeError):
        c.get_option("cfl", typ=str)


def test_tracer_registry_conflicts():
    c = Coupler()
    c.distribute_mpi_and_allocate_coupled_state(4, 3, 5)
    assert c.add_tracer("water_vapor", "", True, True) == 0
    assert c.add_tracer("water_vapor", "", True, True) == 0
    with pytest.raises(ValueError):
        c.add_tracer("water_vapor", "", False, True)
    assert c.get("water_vapor").shape == (4, 3, 5)


def test_time_step_before_init_is_an_error():
    case = cases.small_mixed()
    c = case_coupler(case)
    with pytest.raises(PortUrbError) as e:
        Dynamics_Euler_Stratified_WenoFV().time_step(c, 1.0)
    assert e.value.status == capi.PU_ERR_STATE


def test_invalid_bc_z_rejected_like_the_reference():
    case = cases.small_mixed()
    c = case_coupler(case)
    c.set_option("bc_z", "open_top")
    with pytest.raises(PortUrbError) as e:
        Dynamics_Euler_Stratified_WenoFV().init(c)
    assert "bc_z" in str(e.value)


def test_missing_thermodynamic_option_is_an_error():
    case = cases.small_mixed()
    c = case_coupler(case)
    del c.options["C0"]
    with pytest.raises(KeyError):
        Dynamics_Euler_Stratified_WenoFV().init(c)


def test_compute_time_step_matches_reference_formula(oracle_lib):
    case = cases.warm_bubble(nx=32, ny=4, nz=16)
    c = case_coupler(case)
    dt = Dynamics_Euler_Stratified_WenoFV().compute_time_step(c)
    assert dt == pytest.approx(0.8 * min(case.xlen / 32, case.ylen / 4, case.zlen / 16) / 450.0, rel=1e-15)
    assert dt == pyoracle.Dycore(case, "ref").compute_time_step()
    assert abs(dt - 0.13888888888888) < 1e-9 or case.nx != 256


def test_case_generators():
    b = cases.warm_bubble()
    assert (b.nx, b.ny, b.nz) == (256, 4, 128)
    dth = (b.perturbed["rho_d"] - b.rho_d)
    assert dth.max() <= 0 and dth.min() < 0                       # warm air is lighter
    opts = b.options
    # the base column is isentropic and hydrostatic: p decreases with height
    p = b.rho_d * opts["R_d"] * b.temp
    assert np.all(np.diff(p[:, 0, 0]) < 0)
    a = cases.abl_neutral(nx=16, ny=16, nz=64)
    theta = (p_ := a.perturbed["rho_d"] * opts["R_d"] * a.perturbed["temp"]) ** 0  # noqa: F841
    assert a.tracer_data[1].min() == 0.1 and a.tracer_data[0].max() == 0.0
    u = cases.urban_canopy(nx=128, ny=128, nz=40)
    m = u.immersed_proportion
    assert set(np.unique(m)) <= {0.0, 1.0}
    assert m[0].mean() > 0.2 and m[-1].max() == 0.0
    u2 = cases.urban_canopy(nx=128, ny=128, nz=40)
    assert np.array_equal(u2.immersed_proportion, m)               # seeded, deterministic


def test_urban_window_is_the_block_of_the_full_domain():
    """The bounded CPU sample of the urban workloads is a window of the full
    grid: the same buildings and noise as that block of the whole domain."""
    full = cases.urban_canopy(nx=160, ny=120, nz=40, dx=2.0)
    for w in [(0, 0, 64, 48), (37, 53, 80, 60), (0, 0, 160, 120)]:
        b = cases.urban_canopy(nx=160, ny=120, nz=40, dx=2.0, window=w)
        c = full.block(*w)
        for nm in ("rho_d", "uvel", "vvel", "wvel", "temp", "tracer_data", "immersed_proportion"):
            assert np.array_equal(getattr(b, nm), getattr(c, nm)), nm
        for k in ("rho_d", "temp"):
            assert np.array_equal(b.perturbed[k], c.perturbed[k])
        assert (b.nx, b.ny, b.xlen, b.ylen) == (c.nx, c.ny, c.xlen, c.ylen)
    with pytest.raises(ValueError):
        cases.urban_canopy(nx=160, ny=120, nz=40, window=(100, 0, 64, 48))
