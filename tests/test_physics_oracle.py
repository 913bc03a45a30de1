"""The physics-module oracle (oracle/physics_oracle.cpp) against the
reference's own modules compiled from their headers (oracle/ref_physics.cpp):
LES closure, sponge layer, geostrophic forcing and surface fluxes, bit for
bit on small grids that exercise every branch (immersed faces and cells,
ground and lid, precursor and periodic boundaries, DNS viscosity, gravity
off, closure multipliers, surface heat flux)."""
import numpy as np
import pytest

import pyoracle
import pyphysics
from porturb_b200 import cases

pytestmark = pytest.mark.skipif(not pyoracle.have_ref(), reason="reference library not built")


def _case(kind):
    c = cases.abl_neutral(nx=16, ny=12, nz=10, dx=10.0)
    halos_kw = {}
    opts = {}
    if kind in ("immersed", "immersed_heat"):
        m = np.zeros((c.nz, c.ny, c.nx))
        m[:4, 3:7, 5:9] = 1.0
        m[6, 8, 2] = 0.5
        m[0, 10, 12] = 1.0
        c.immersed_proportion[...] = m
        if kind == "immersed_heat":
            halos_kw = dict(surface_temp=300.5, immersed_temp=301.0, roughness=0.05)
    elif kind == "precursor":
        c.options["bc_x"] = "precursor"
        c.options["bc_y"] = "precursor"
    elif kind == "periodic_z":
        c.options["bc_z"] = "periodic"
    elif kind == "dns":
        opts = dict(nu=1.5e-2, dns=True)
    elif kind == "no_gravity":
        c.options["enable_gravity"] = False
        opts = dict(nu=1e-3, total_mult=0.7, dissipation_mult=1.3, shear_prod_mult=0.8)
    return c, cases.immersed_halos(c, **halos_kw), opts


KINDS = ["plain", "immersed", "immersed_heat", "precursor", "periodic_z", "dns", "no_gravity"]


@pytest.mark.parametrize("kind", KINDS)
def test_restatement_matches_reference_modules(oracle_lib, kind):
    case, halos, opts = _case(kind)
    st = pyphysics.state_of(case, seed=KINDS.index(kind))
    orc = pyphysics.Physics(case, "orc", halos, **opts)
    ref = pyphysics.Physics(case, "ref", halos, **opts)
    dt = 0.1
    calls = [("les", (dt,)), ("sponge", (dt, 100 * dt, 0.3)), ("geostrophic", (dt, 43.0, 10.0, -2.0)),
             ("surface_fluxes", (dt,))]
    for name, args in calls:
        a = getattr(orc, name)(st, *args)
        b = getattr(ref, name)(st, *args)
        for key in a:
            same = np.array_equal(a[key], b[key])
            if not same:
                d = np.abs(a[key] - b[key]).max()
                pytest.fail("%s/%s: %s differs from the reference (max |diff| %.3e)" % (kind, name, key, d))
        # the call changed something (the branch was exercised)
        changed = any(not np.array_equal(a[k], st[k]) for k in a)
        assert changed, (kind, name)


def test_les_conserves_and_keeps_tke_positive(oracle_lib):
    """Known-answer properties of the closure: with periodic x/y and walls
    in z, a diffused tracer's mass rho*q is conserved (the ground face is
    closed by the immersed ground halo and the lid halo copies the top
    level, so no flux leaves), and TKE stays non-negative."""
    case, halos, opts = _case("plain")
    st = pyphysics.state_of(case, seed=3)
    out = pyphysics.Physics(case, "orc", halos).les(st, 0.1)
    wv = [t.name for t in case.tracers].index("water_vapor")
    before, after = st["tracers"][wv].sum(), out["tracers"][wv].sum()
    assert abs(after - before) <= 1e-12 * abs(before)
    tke = [t.name for t in case.tracers].index("TKE")
    assert out["tracers"][tke].min() >= 0.0


def _pg_state(case, seed):
    st = pyphysics.state_of(case, seed=seed)
    rng = np.random.default_rng(seed)
    st["uvel"] = st["uvel"] + 3.0 + rng.standard_normal(st["uvel"].shape)
    st["vvel"] = st["vvel"] - 1.0 + rng.standard_normal(st["vvel"].shape)
    return st


@pytest.mark.parametrize("update_cycles", [1, 3])
def test_uniform_pg_matches_reference_across_calls(oracle_lib, update_cycles):
    """uniform_pg_wind_forcing keeps (counter, u0, v0, u, v) between calls;
    the wind is disturbed between calls so every update shows."""
    case, halos, _ = _case("plain")
    orc = pyphysics.Physics(case, "orc", halos)
    ref = pyphysics.Physics(case, "ref", halos)
    st = _pg_state(case, 1)
    so, sr = np.zeros(5), np.zeros(5)
    rng = np.random.default_rng(7)
    for call in range(7):
        a = orc.uniform_pg(st, 0.05, 2.0, update_cycles, so)
        b = ref.uniform_pg(st, 0.05, 2.0, update_cycles, sr)
        assert np.array_equal(so, sr), (call, so, sr)
        for key in a:
            assert np.array_equal(a[key], b[key]), (call, key)
        st = a
        st["uvel"] = st["uvel"] + 0.3 * rng.standard_normal(st["uvel"].shape)
        st["vvel"] = st["vvel"] + 0.3 * rng.standard_normal(st["vvel"].shape)
    assert so[0] == 7


def test_uniform_pg_relaxes_the_domain_mean(oracle_lib):
    """Known answer: the first call records the mean and forces nothing; after
    a uniform +1 m/s gust the next call removes dt/tau of it."""
    case, halos, _ = _case("plain")
    orc = pyphysics.Physics(case, "orc", halos)
    st = _pg_state(case, 2)
    so = np.zeros(5)
    a = orc.uniform_pg(st, 0.1, 4.0, 1, so)
    assert np.array_equal(a["uvel"], st["uvel"]) and np.array_equal(a["vvel"], st["vvel"])
    assert so[1] == so[3] and abs(so[1] - st["uvel"].mean()) < 1e-12
    a["uvel"] = a["uvel"] + 1.0
    b = orc.uniform_pg(a, 0.1, 4.0, 1, so)
    assert abs(b["uvel"].mean() - (st["uvel"].mean() + 1.0 - 0.1 / 4.0)) < 1e-12
    assert abs(b["vvel"].mean() - st["vvel"].mean()) < 1e-12


@pytest.mark.parametrize("where", ["between", "on_centre", "above_top", "first_centre"])
def test_uniform_pg_height_matches_reference(oracle_lib, where):
    case, halos, _ = _case("plain")
    dz = case.zlen / case.nz
    height = {"between": 3.3 * dz, "on_centre": 4.5 * dz, "above_top": (case.nz + 0.2) * dz,
              "first_centre": 0.5 * dz}[where]
    st = _pg_state(case, 3)
    a = pyphysics.Physics(case, "orc", halos).uniform_pg_height(st, 0.05, height, 8.0, 0.5, 3.0)
    b = pyphysics.Physics(case, "ref", halos).uniform_pg_height(st, 0.05, height, 8.0, 0.5, 3.0)
    for key in a:
        assert np.array_equal(a[key], b[key]), key
    assert not np.array_equal(a["uvel"], st["uvel"])


def test_uniform_pg_height_known_answer_and_bad_height(oracle_lib):
    """Linear interpolation between the bracketing level means; a height
    below the first level centre is refused (the reference would read level
    -1, so it is not called there)."""
    case, halos, _ = _case("plain")
    dz = case.zlen / case.nz
    st = _pg_state(case, 4)
    orc = pyphysics.Physics(case, "orc", halos)
    height = 2.75 * dz   # between the centres of levels 2 (2.5 dz) and 3 (3.5 dz)
    a = orc.uniform_pg_height(st, 0.2, height, 6.0, 1.0, 5.0)
    um = 0.75 * st["uvel"][2].mean() + 0.25 * st["uvel"][3].mean()
    vm = 0.75 * st["vvel"][2].mean() + 0.25 * st["vvel"][3].mean()
    assert np.allclose(a["uvel"] - st["uvel"], 0.2 / 5.0 * (6.0 - um), rtol=0, atol=1e-13)
    assert np.allclose(a["vvel"] - st["vvel"], 0.2 / 5.0 * (1.0 - vm), rtol=0, atol=1e-13)
    with pytest.raises(RuntimeError):
        orc.uniform_pg_height(st, 0.2, 0.4 * dz, 6.0, 1.0, 5.0)


def test_time_averager_matches_reference_across_calls(oracle_lib):
    """custom_modules::Time_Averager::accumulate over 6 calls with a changing
    state and elapsed time, a reset (etime 0, short averages zeroed) midway:
    the restatement equals the reference's header bit for bit."""
    case, halos, _ = _case("plain")
    orc = pyphysics.Physics(case, "orc", halos)
    ref = pyphysics.Physics(case, "ref", halos)
    st = pyphysics.state_of(case, seed=9)
    shape = (13,) + st["uvel"].shape
    ao, ar = np.zeros(shape), np.zeros(shape)
    eo = er = 0.0
    elapsed = 0.0
    rng = np.random.default_rng(4)
    for call in range(6):
        if call == 3:
            eo = er = 0.0
            ao[:10] = 0
            ar[:10] = 0
        dt = 0.1 + 0.05 * call
        eo = orc.time_average(st, ao, eo, elapsed, dt)
        er = ref.time_average(st, ar, er, elapsed, dt)
        assert eo == er
        assert np.array_equal(ao, ar), call
        elapsed += dt
        st = dict(st)
        st["uvel"] = st["uvel"] + 0.2 * rng.standard_normal(st["uvel"].shape)
        st["wvel"] = st["wvel"] + 0.1 * rng.standard_normal(st["wvel"].shape)
    assert np.abs(ao[4]).max() > 0 and np.abs(ao[10] - st["uvel"]).max() > 0


@pytest.mark.parametrize("props", [(0.1, 0.1, 0.1, 0.1), (0.01, 0.01, 0.01, 0.01), (0.3, 0.0, 0.0, 0.25),
                                   (0.0, 0.5, 0.2, 0.0)])
def test_edge_sponge_matches_reference(oracle_lib, props):
    """custom_modules::EdgeSponge: the column profile recorded from one state
    and the edge relaxation of a later one, bit for bit (corner cells take
    both zones in the reference's order)."""
    case, halos, _ = _case("plain")
    orc = pyphysics.Physics(case, "orc", halos)
    ref = pyphysics.Physics(case, "ref", halos)
    st0 = pyphysics.state_of(case, seed=21)
    co, cr = orc.edge_sponge_set_column(st0), ref.edge_sponge_set_column(st0)
    assert np.array_equal(co, cr)
    st = pyphysics.state_of(case, seed=22)
    a = orc.edge_sponge_apply(st, co, *props)
    b = ref.edge_sponge_apply(st, cr, *props)
    for key in a:
        assert np.array_equal(a[key], b[key]), key
    assert not np.array_equal(a["uvel"], st["uvel"])
