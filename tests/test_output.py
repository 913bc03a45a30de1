"""Output and restart files (porturb_b200/output.py) without a GPU: the
variables, dimensions and types of the reference's output file
(coupler.h:533-649), the counter-numbered file names, and the restart read
(coupler.h:653-723): float32 fields come back rounded, float64 fields
(option output_f64) exactly."""
import numpy as np
import pytest
from scipy.io import netcdf_file

from porturb_b200 import case_coupler, cases
from porturb_b200.output import DIMS_3D


def _coupler():
    case = cases.small_mixed(immersed=True)
    c = case_coupler(case)
    rng = np.random.default_rng(0)
    for name in ("uvel", "vvel", "wvel"):
        c.get(name)[...] = rng.standard_normal(c.get(name).shape)
    c.register_output_variable("immersed_proportion", DIMS_3D)
    c.set_option("elapsed_time", 12.5)
    return case, c


def test_file_layout_matches_the_reference(tmp_path):
    case, c = _coupler()
    f1 = c.write_output_file(str(tmp_path / "out"))
    f2 = c.write_output_file(str(tmp_path / "out"))
    assert f1.endswith("out_00000000.nc") and f2.endswith("out_00000001.nc")
    nc = netcdf_file(f1, "r", mmap=False)
    assert nc.dimensions == {"x": case.nx, "y": case.ny, "z": case.nz, "t": 1}
    for name in ("density_dry", "uvel", "vvel", "wvel", "temperature", "immersed_proportion") + \
            tuple(t.name for t in case.tracers):
        v = nc.variables[name]
        assert v.dimensions == ("z", "y", "x") and v.data.dtype.kind == "f" and v.data.dtype.itemsize == 4, name
    assert nc.variables["x"].data[0] == np.float32(0.5 * case.xlen / case.nx)
    assert nc.variables["etime"].data[0] == np.float32(12.5)
    assert nc.variables["file_counter"].data[0] == 0
    assert np.array_equal(nc.variables["temperature"].data, c.get("temp").astype(np.float32))
    nc.close()


@pytest.mark.parametrize("f64", [False, True])
def test_restart_round_trip(tmp_path, f64):
    case, c = _coupler()
    if f64:
        c.set_option("output_f64", True)
    fname = c.write_output_file(str(tmp_path / "rst"))
    _, d = _coupler()
    for name in ("uvel", "temp"):
        d.get(name)[...] = 0.0
    d.set_option("restart_file", fname)
    d.overwrite_with_restart()
    assert d.get_option("elapsed_time") == 12.5
    assert d.file_counter == 1
    for name in ("density_dry", "uvel", "vvel", "wvel", "temp"):
        want = c.get(name) if f64 else c.get(name).astype(np.float32).astype(np.float64)
        assert np.array_equal(d.get(name), want), name
