"""Known-answer tests of the oracle's numerics (FP64 variant unless stated)."""
import numpy as np
import pytest

import pyoracle
from porturb_b200 import cases


def cell_averages(coefs, offsets):
    """Unit-cell averages of sum_d c_d x^d over cells centred at the offsets."""
    out = []
    for o in offsets:
        a, b = o - 0.5, o + 0.5
        out.append(sum(c * (b ** (d + 1) - a ** (d + 1)) / (d + 1) for d, c in enumerate(coefs)))
    return np.array(out)


@pytest.mark.parametrize("do_map", [False, True])
def test_limiter_exact_for_quartics(oracle_lib, do_map):
    rng = np.random.default_rng(0)
    for _ in range(200):
        c = rng.normal(size=5)
        s = cell_averages(c, range(-4, 5))
        qL, qR = pyoracle.weno9(s, do_map, False, False, kind="f64")
        exact_L = sum(cd * (-0.5) ** d for d, cd in enumerate(c))
        exact_R = sum(cd * 0.5 ** d for d, cd in enumerate(c))
        assert abs(qL - exact_L) < 1e-11 * (1 + abs(exact_L))
        assert abs(qR - exact_R) < 1e-11 * (1 + abs(exact_R))


def test_limiter_reflection_identity(oracle_lib):
    """The right edge of a stencil is the left edge of the mirrored stencil
    (the right-edge ideal weights are the left ones reversed)."""
    rng = np.random.default_rng(1)
    for _ in range(500):
        s = rng.normal(size=9) * 10 ** rng.uniform(-3, 3)
        qL, qR = pyoracle.weno9(s, True, False, False, kind="f64")
        mL, mR = pyoracle.weno9(s[::-1].copy(), True, False, False, kind="f64")
        scale = np.abs(s).max()
        assert abs(qR - mL) < 1e-12 * scale and abs(qL - mR) < 1e-12 * scale


def test_limiter_constant_and_bounded(oracle_lib):
    for v in (0.0, 1.0, -3.5e-4, 2.0e5):
        q = pyoracle.weno9(np.full(9, v), True, False, False, kind="f64")
        assert q == pytest.approx((v, v), rel=1e-14, abs=0)
    # A step: edge values stay within the stencil's range (essentially non-oscillatory).
    s = np.array([0, 0, 0, 0, 1, 1, 1, 1, 1.0])
    qL, qR = pyoracle.weno9(s, True, False, False, kind="f64")
    assert -1e-6 <= qL <= 1 + 1e-6 and -1e-6 <= qR <= 1 + 1e-6


def _rest_case():
    c = cases.small_mixed(immersed=False, ntr=1)
    c.uvel[...] = 0.0
    c.vvel[...] = 0.0
    c.wvel[...] = 0.0
    c.tracer_data[...] = 0.0
    c.perturbed = None
    return c


def test_hydrostatic_rest_state_stays_at_rest(oracle_lib):
    case = _rest_case()
    d = pyoracle.Dycore(case, "f64")
    d.init_case()
    st0, _ = d.get_state()
    d.advance(d.compute_time_step(), 5)
    st, _ = d.get_state()
    assert np.abs(st[1:4]).max() < 1e-9
    assert np.abs(st[0] - st0[0]).max() < 1e-12
    assert np.abs(st[4] - st0[4]).max() < 1e-9


@pytest.mark.parametrize("kind", ["f64", "ref"])
def test_mass_and_rho_theta_conserved(oracle_lib, kind):
    case = cases.small_mixed(immersed=False)
    d = pyoracle.Dycore(case, kind)
    d.init_case()
    d.load_coupler(list(case.coupler_arrays(perturbed=True)))
    st0, tr0 = d.get_state()
    d.advance(d.compute_time_step(), 5)
    st, tr = d.get_state()
    tol = 1e-13 if kind == "f64" else 1e-9
    assert abs(st[0].sum() - st0[0].sum()) < tol * st0[0].sum()
    assert abs(st[4].sum() - st0[4].sum()) < tol * st0[4].sum()
    assert abs(tr[1].sum() - tr0[1].sum()) < tol * tr0[1].sum() * 10


def test_bubble_mirror_symmetry(oracle_lib):
    case = cases.warm_bubble(nx=32, ny=4, nz=24, xlen=3200.0, ylen=400.0, zlen=2400.0, radius=600.0,
                             x0=1600.0, z0=700.0)
    d = pyoracle.Dycore(case, "f64")
    d.init_case()
    d.load_coupler(list(case.coupler_arrays(perturbed=True)))
    d.advance(d.compute_time_step(), 8)
    st, _ = d.get_state()
    mir = st[:, :, :, ::-1]
    assert np.abs(st[0] - mir[0]).max() < 1e-12
    assert np.abs(st[4] - mir[4]).max() < 1e-9
    assert np.abs(st[3] - mir[3]).max() < 1e-9          # w symmetric
    assert np.abs(st[1] + mir[1]).max() < 1e-9          # u antisymmetric
    assert np.abs(st[3]).max() > 1e-3                   # the bubble did move
