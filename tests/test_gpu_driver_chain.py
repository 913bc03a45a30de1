"""The reference drivers' module chains on device coupler arrays
(porturb_b200.run_case._driver_run), with the FP32 dycore against the FP64
build from the same state and dt_phys:

* abl      -- abl_neutral.cpp:93-108 on the boundary layer, 64x64x48;
* city     -- city.cpp:137-142 on the urban canopy, 64x64x32;
* periodic -- cubes_periodic.cpp:144-156 on the urban canopy, 64x64x64
  with an 8 m/s initial wind (mean wind at 100 m relaxed toward 10 m/s on a
  time scale of 100 dt_phys).

Two calls of dt_phys = 10 dycore steps each.  Every coupler array stays
finite; the FP32 run is within L2 < 1e-4 and Linf < 1e-3 of the FP64 run's
departure from its level means (the physics modules are FP64 in both, so the
difference is the dycore's FP32 state over 20 steps); the LES closure moved
the TKE off its initial 0.1; in the periodic chain the mean wind at 100 m
rose by the forcing's 0.01 (10 - u) per call, 0.02 + 0.0198 m/s, to 10 %.
"""
import types

import numpy as np
import pytest

from porturb_b200 import cases
from porturb_b200.run_case import _driver_run, _release, coupler_errors

pytestmark = pytest.mark.gpu

CHAIN_CASES = {
    "abl": lambda: cases.abl_neutral(nx=64, ny=64, nz=48),
    "city": lambda: cases.urban_canopy(nx=64, ny=64, nz=32),
    "periodic": lambda: cases.urban_canopy(nx=64, ny=64, nz=64, u0=8.0),
}


def _args(case, chain):
    return types.SimpleNamespace(case=case.name, nx=case.nx, ny=case.ny, nz=case.nz, chain=chain)


@pytest.mark.parametrize("chain", sorted(CHAIN_CASES))
def test_driver_chain_f32_against_f64(chain, gpu_lib):
    import torch
    case = CHAIN_CASES[chain]()
    a = _args(case, chain)
    c, dt, ms, sub = _driver_run(case, a, "f32", 2, warm=0)
    assert sub == 10
    names = ["density_dry", "uvel", "vvel", "wvel", "temp"] + list(c.get_tracer_names())
    f32 = {n: c.get(n).clone() for n in names}
    _release(c)
    c, _, _, _ = _driver_run(case, a, "f64", 2, dt=dt, warm=0)
    f64 = {n: c.get(n) for n in names}
    for n, x in f32.items():
        assert torch.isfinite(x).all(), (chain, n)
        assert torch.isfinite(f64[n]).all(), (chain, n)
    errs = coupler_errors({n: f32[n] for n in names[:5]}, f64)
    for n, e in errs.items():
        print(chain, n, "FP32 run vs FP64 run (of departure): %.2e / %.2e" % (e["l2"], e["linf"]))
        assert e["l2"] is not None and e["l2"] < 1e-4 and e["linf"] < 1e-3, (chain, n, e)
    assert float((f64["TKE"] - 0.1).abs().max()) > 1e-6, chain
    if chain == "periodic":
        # Levels 49 and 50 (centres 99 m and 101 m) hold the 100 m mean.
        u0 = float(np.asarray(case.uvel)[49:51].mean())
        u1 = float(f64["uvel"][49:51].mean())
        print("mean u at 100 m: %.5f -> %.5f" % (u0, u1))
        assert abs((u1 - u0) - 0.0398) < 0.004, (u0, u1)
    _release(c)
