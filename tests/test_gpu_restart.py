"""Restart through the output file with the dycore's hooks on the GPU:
continuing from a float64 restart file (option output_f64) reproduces the
uninterrupted run bit for bit, and the perturbation fields the dycore writes
(dynamics_rk.h:1212-1232, computed by pu_dycore_perturbations) agree with a
numpy evaluation of the same formulas on the written state."""
import numpy as np
import pytest
from scipy.io import netcdf_file

from porturb_b200 import Dynamics_Euler_Stratified_WenoFV, case_coupler, cases

pytestmark = pytest.mark.gpu


def _setup(case, precision):
    c = case_coupler(case)
    dyn = Dynamics_Euler_Stratified_WenoFV(precision=precision)
    dyn.init(c)
    pert = case.perturbed
    c.get("density_dry")[...] = pert["rho_d"]
    c.get("temp")[...] = pert["temp"]
    return c, dyn


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_restart_continues_bit_for_bit(gpu_lib, tmp_path, precision):
    case = cases.warm_bubble(nx=64, ny=4, nz=32, xlen=5000.0, zlen=2500.0, radius=500.0, x0=2500.0, z0=600.0)
    a, dyn_a = _setup(case, precision)
    a.set_option("output_f64", True)
    dt = 5 * dyn_a.compute_time_step(a)
    for _ in range(2):
        dyn_a.time_step(a, dt)
    fname = a.write_output_file(str(tmp_path / "rst"))
    b, dyn_b = _setup(case, precision)
    b.set_option("restart_file", fname)
    b.overwrite_with_restart()
    dyn_a.time_step(a, dt)
    dyn_b.time_step(b, dt)
    for name in ["density_dry", "uvel", "vvel", "wvel", "temp"] + a.get_tracer_names():
        assert np.array_equal(a.get(name), b.get(name)), name

    # The dycore's perturbation fields in the file.
    nc = netcdf_file(fname, "r", mmap=False)
    o = case.options
    rd = nc.variables["density_dry"].data.astype(np.float64)
    T = nc.variables["temperature"].data.astype(np.float64)
    qv = nc.variables["water_vapor"].data.astype(np.float64)
    hs = 4
    cells = [nc.variables[n].data.astype(np.float64)[hs:hs + case.nz, None, None]
             for n in ("hy_dens_cells", "hy_theta_cells", "hy_pressure_cells")]
    rho = rd + qv     # water_vapor adds mass
    press = rd * o["R_d"] * T + qv * o["R_v"] * T
    rt = rho * ((press / o["C0"]) ** (1.0 / o["gamma_d"]) / rho)
    want = [rho - cells[0], rt / rho - cells[1], o["C0"] * rt ** o["gamma_d"] - cells[2]]
    for name, w in zip(("density_pert", "theta_pert", "pressure_pert"), want):
        got = nc.variables[name].data
        assert got.dtype.kind == "f" and got.dtype.itemsize == 8
        scale = np.abs(w).max() + 1e-300
        assert np.abs(got - w).max() <= 1e-9 * scale + 1e-12 * np.abs(cells[0]).max(), name
    nc.close()
