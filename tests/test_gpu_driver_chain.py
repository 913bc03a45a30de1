"""The reference drivers' module chains on device coupler arrays
(porturb_b200.run_case._driver_run), with the FP32 dycore against the FP64
build from the same state and dt_phys:

* abl      -- abl_neutral.cpp:93-108 on the boundary layer, 64x64x48;
* city     -- city.cpp:137-142 on the urban canopy, 64x64x32;
* periodic -- cubes_periodic.cpp:144-156 on the urban canopy, 64x64x64
  with an 8 m/s initial wind (mean wind at 100 m relaxed toward 10 m/s on a
  time scale of 100 dt_phys).

Two calls of dt_phys = 10 dycore steps each, and the same two calls of the
dycore alone (chain "dycore": the same init, no other module).  Every coupler
array stays finite.  The physics modules are FP64 in both runs, so the
difference between the FP32 and FP64 runs starts in the dycore's FP32 state;
the modules must not amplify it: per coupler array, the chain's L2 (Linf) of
FP32 - FP64 over the FP64 run's departure from its level means is within 2x
(5x) of the dycore-alone difference.  Measured on a B200: 1.0-1.35x (L2) and
up to 2.1x (Linf); the dycore-alone differences are 1e-5 - 4e-2 of the
departure (largest for the winds of the boundary layer, whose departures
from the level means are still small).  The LES closure moved the TKE off
its initial 0.1; in the periodic chain the mean wind at 100 m rose by the
forcing's 0.01 (10 - u) per call, 0.02 + 0.0198 m/s (0.0398 measured).
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


def _f32_vs_f64(case, chain, names):
    a = _args(case, chain)
    c, dt, _, sub = _driver_run(case, a, "f32", 2, warm=0)
    assert sub == 10
    f32 = {n: c.get(n).clone() for n in names}
    _release(c)
    c, _, _, _ = _driver_run(case, a, "f64", 2, dt=dt, warm=0)
    return f32, c


@pytest.mark.parametrize("chain", sorted(CHAIN_CASES))
def test_driver_chain_f32_against_f64(chain, gpu_lib):
    import torch
    case = CHAIN_CASES[chain]()
    names = ["density_dry", "uvel", "vvel", "wvel", "temp"]
    f32, c = _f32_vs_f64(case, chain, names + ["water_vapor", "TKE"])
    f64 = {n: c.get(n) for n in f32}
    for n, x in f32.items():
        assert torch.isfinite(x).all(), (chain, n)
        assert torch.isfinite(f64[n]).all(), (chain, n)
    errs = coupler_errors({n: f32[n] for n in names}, f64)
    assert float((f64["TKE"] - 0.1).abs().max()) > 1e-6, chain
    if chain == "periodic":
        # Levels 49 and 50 (centres 99 m and 101 m) hold the 100 m mean.
        u0 = float(np.asarray(case.uvel)[49:51].mean())
        u1 = float(f64["uvel"][49:51].mean())
        print("mean u at 100 m: %.5f -> %.5f" % (u0, u1))
        assert abs((u1 - u0) - 0.0398) < 0.002, (u0, u1)
    _release(c)
    del f32, f64
    d32, c = _f32_vs_f64(case, "dycore", names)
    base = coupler_errors(d32, {n: c.get(n) for n in names})
    _release(c)
    for n in names:
        e, b = errs[n], base[n]
        print(chain, n, "FP32 - FP64 (of departure): chain %.2e / %.2e, dycore alone %.2e / %.2e"
              % (e["l2"], e["linf"], b["l2"], b["linf"]))
        assert e["l2"] is not None and b["l2"] is not None, (chain, n)
        assert e["l2"] <= 2 * b["l2"] + 1e-7 and e["linf"] <= 5 * b["linf"] + 1e-6, (chain, n, e, b)
