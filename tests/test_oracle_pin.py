"""Pins the CPU oracle to the reference's own dycore code.

The reference's dynamics_rk.h / WenoLimiter.h / TransformMatrices.h compile
unchanged against a single-rank shim (oracle/_ref); the golden fixtures in
tests/golden/ were produced by that build (tests/golden/make_golden.py).  The
oracle's REF variant must reproduce them bit for bit; where the reference
tree is mounted the comparison also runs live on fresh random inputs.
"""
import os

import numpy as np
import pytest

import pyoracle
from porturb_b200 import cases

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = {
    "small_mixed": lambda: cases.small_mixed(),
    "small_precursor": lambda: cases.small_mixed(bc_x="precursor", bc_y="precursor", ntr=1, immersed=False),
    "bubble_64x4x32": lambda: cases.warm_bubble(nx=64, ny=4, nz=32, xlen=5000.0, ylen=312.5, zlen=2500.0,
                                                radius=500.0, x0=2500.0, z0=600.0, cfl=0.8),
}


def test_limiter_matches_golden(oracle_lib):
    g = np.load(os.path.join(GOLDEN, "limiter.npz"))
    s, flags = g["stencils"], g["flags"]
    for m in range(len(s)):
        q32 = pyoracle.weno9(s[m], *flags[m], kind="ref_f32")
        assert np.array_equal(np.array(q32, np.float32).view(np.uint32), g["edges_f32"][m].view(np.uint32)), m
        q64 = pyoracle.weno9(s[m], *flags[m], kind="f64tvf")
        assert q64[0] == g["edges_f64"][m][0] and q64[1] == g["edges_f64"][m][1], m


@pytest.mark.parametrize("name", sorted(CASES))
def test_steps_match_golden(name, oracle_lib):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    case = CASES[name]()
    # The fixture's inputs are the arrays the case builder produces.
    assert np.array_equal(g["base"][0], case.rho_d) and np.array_equal(g["pert"][4], case.perturbed["temp"])
    d = pyoracle.Dycore(case, "ref")
    b, bt, im = g["base"], g["base_tracers"], g["immersed"]
    d.init(b[0], b[1], b[2], b[3], b[4], bt, im)
    cells, edges = d.get_hydrostasis()
    assert np.array_equal(np.stack(cells), g["hy_cells"])
    assert np.array_equal(np.stack(edges), g["hy_edges"])
    p, pt = g["pert"], g["pert_tracers"]
    d.load_coupler([p[0], p[1], p[2], p[3], p[4], pt])
    d.advance(float(g["dt"]), int(g["nsteps"]))
    st, tr = d.get_state()
    assert np.array_equal(st, g["state"])
    assert np.array_equal(tr, g["tracers"])


needs_ref = pytest.mark.skipif(not os.path.isdir(os.path.join(pyoracle.REFERENCE_DIR, "model")),
                               reason="the reference tree is not mounted here")


@needs_ref
def test_limiter_matches_reference_live(oracle_lib):
    rng = np.random.default_rng(11)
    for n in range(3000):
        s = rng.normal(size=9) * 10 ** rng.uniform(-8, 4)
        if n % 5 == 0:
            s[rng.integers(0, 9)] += 1e3 * abs(s[0])
        fl = (bool(n % 2), bool(n % 3 == 0), bool(n % 7 == 0))
        a = pyoracle.weno9(s, *fl, kind="ref_f32")
        b = pyoracle.weno9(s, *fl, kind="reference_f32")
        assert np.array_equal(np.array(a, np.float32).view(np.uint32), np.array(b, np.float32).view(np.uint32))
        assert pyoracle.weno9(s, *fl, kind="f64tvf") == pyoracle.weno9(s, *fl, kind="reference_f64")


@needs_ref
@pytest.mark.parametrize("variant", ["immersed_2tr", "periodic_z", "coriolis_2d", "linear"])
def test_time_step_matches_reference_live(variant, oracle_lib):
    """The full time_step entry point (coupler conversion, sub-cycling,
    conversion back) of the REF oracle equals the reference's, bit for bit."""
    case = {"immersed_2tr": lambda: cases.small_mixed(seed=5),
            "periodic_z": lambda: cases.small_mixed(bc_z="periodic", seed=6),
            "coriolis_2d": lambda: cases.small_mixed(ny=1, nx=20, nz=14, latitude=30.0, seed=7),
            "linear": lambda: cases.small_mixed(weno_all=False, immersed=False, seed=8)}[variant]()
    out = {}
    for kind in ("ref", "reference"):
        d = pyoracle.Dycore(case, kind)
        d.init_case()
        arrs = [np.ascontiguousarray(a.copy()) for a in case.coupler_arrays(perturbed=True)]
        nc = d.time_step(arrs, 2.5 * d.compute_time_step())
        out[kind] = (nc, arrs)
    assert out["ref"][0] == out["reference"][0] == 3
    for a, b in zip(out["ref"][1], out["reference"][1]):
        assert np.array_equal(a, b)
