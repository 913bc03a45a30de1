"""FP64 compensated global diagnostics (pu_dycore_diagnostics): the integrals
match an exactly rounded numpy evaluation of the same integrands on the
resident state, and the flux-form dycore conserves mass, rho*theta and
tracer mass over 20 steps of a closed domain (periodic x/y, walls in z, no
immersed cells): to round-off in the FP64 build (measured on a B200: no
change at all), and within FP32 storage rounding in the FP32 build
(measured: mass 3e-13, rho*theta 5e-13, tracer 7e-10 relative)."""
import math

import numpy as np
import pytest

from porturb_b200 import Dycore, cases

pytestmark = pytest.mark.gpu


def _case():
    c = cases.warm_bubble(nx=64, ny=4, nz=32, xlen=5000.0, zlen=2500.0, radius=500.0, x0=2500.0, z0=600.0)
    c.tracer_data[0] = 1e-3 * (1.0 + 0.5 * np.sin(np.arange(c.nx) / 5.0))[None, None, :]
    return c


def _handle(case, precision):
    g = Dycore.from_case(case, precision=precision)
    rd, u, v, w, T, trc = [np.ascontiguousarray(a) for a in case.coupler_arrays(perturbed=True)]
    g.init(rd, u, v, w, T, list(trc), None)
    return g


def _fsum(a):
    return math.fsum(np.asarray(a, dtype=np.float64).ravel())


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_diagnostics_match_exact_sums(gpu_lib, precision):
    case = _case()
    g = _handle(case, precision)
    g.advance(g.compute_time_step(), 3)
    d = g.diagnostics()
    st, tr = g.get_conserved()
    o = case.options
    dV = (case.xlen / case.nx) * (case.ylen / case.ny) * (case.zlen / case.nz)
    dz = case.zlen / case.nz
    rho, mu, mv, mw, rt = st
    z = ((np.arange(case.nz) + 0.5) * dz)[:, None, None]
    ke = 0.5 * (mu * mu + mv * mv + mw * mw) / rho
    ie = o["C0"] * rt ** o["gamma_d"] / (o["gamma_d"] - 1)
    pe = rho * o["grav"] * z
    want = {"mass": _fsum(rho * dV), "rho_theta": _fsum(rt * dV), "kinetic": _fsum(ke * dV),
            "internal": _fsum(ie * dV), "potential": _fsum(pe * dV), "total_energy": _fsum((ke + ie + pe) * dV)}
    for k, w in want.items():
        assert abs(d[k] - w) <= 1e-12 * abs(w), (k, d[k], w)
    assert abs(d["tracer_mass"][0] - _fsum(tr[0] * dV)) <= 1e-12 * abs(_fsum(tr[0] * dV))


@pytest.mark.parametrize("precision,bound", [("f64", 1e-13), ("f32", 1e-8)])
def test_closed_domain_conserves(gpu_lib, precision, bound):
    case = _case()
    g = _handle(case, precision)
    d0 = g.diagnostics()
    g.advance(g.compute_time_step(), 20)
    d1 = g.diagnostics()
    drift = {k: abs(d1[k] - d0[k]) / abs(d0[k]) for k in ("mass", "rho_theta")}
    drift["tracer"] = abs(d1["tracer_mass"][0] - d0["tracer_mass"][0]) / abs(d0["tracer_mass"][0])
    print(precision, "relative drift over 20 steps:", drift)
    for k, v in drift.items():
        assert v <= bound, (k, v)
    assert d1["kinetic"] > 0
