"""GPU physics modules (include/pu_physics.h) against the CPU oracle that is
pinned bit for bit to the reference's own modules (tests/test_physics_oracle.py).

The GPU kernels multiply by reciprocals of the grid spacings where the
reference divides, evaluate K^1.5 as K*sqrt(K), and sum the level means with
Neumaier compensation in parallel, so results agree to round-off: per field,
max |GPU - oracle| <= 1e-10 of the change the call made plus 1e-13 of the
field's magnitude.  Grids are not multiples of the 32x8x16 LES tile so that
partial tiles and level chunks are covered; host arrays and device arrays,
the in-place and the out-of-place forms, and the Coupler-level module API
are all checked."""
import numpy as np
import pytest

import pyphysics
from porturb_b200 import cases
from porturb_b200.physics import Physics

pytestmark = pytest.mark.gpu

KINDS = ["plain", "immersed", "immersed_heat", "precursor", "periodic_z", "dns", "no_gravity"]


def _case(kind, nx=40, ny=20, nz=20):
    c = cases.abl_neutral(nx=nx, ny=ny, nz=nz, dx=10.0)
    halos_kw, opts = {}, {}
    if kind in ("immersed", "immersed_heat"):
        m = np.zeros((nz, ny, nx))
        m[:6, 4:9, 6:15] = 1.0
        m[10, 12, 3] = 0.5
        m[0, 15, 33] = 1.0
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


def _gpu_opts(o):
    m = {"nu": "kinematic_viscosity", "dns": "dns", "total_mult": "les_total_mult",
         "dissipation_mult": "les_dissipation_mult", "shear_prod_mult": "les_shear_prod_mult"}
    return {m[k]: v for k, v in o.items()}


def _check(name, got, want, before):
    for key in want:
        g, w, b = np.asarray(got[key]), want[key], before[key]
        err = np.abs(g - w).max()
        tol = 1e-10 * np.abs(w - b).max() + 1e-13 * np.abs(w).max()
        assert err <= tol, "%s: %s max |gpu - oracle| %.3e > %.3e" % (name, key, err, tol)


def _run_gpu(ph, name, st, args, device):
    s = {k: np.array(v, copy=True) for k, v in st.items()}
    if device:
        import torch
        t = {k: torch.from_numpy(s[k]).cuda() for k in ("rho_d", "uvel", "vvel", "wvel", "temp")}
        trc = [torch.from_numpy(np.ascontiguousarray(s["tracers"][i])).cuda() for i in range(s["tracers"].shape[0])]
        getattr(ph, name)(t["rho_d"], t["uvel"], t["vvel"], t["wvel"], t["temp"], trc, *args)
        ph.synchronize()
        out = {k: t[k].cpu().numpy() for k in t}
        out["tracers"] = np.stack([x.cpu().numpy() for x in trc])
        return out
    trc = [np.ascontiguousarray(s["tracers"][i]) for i in range(s["tracers"].shape[0])]
    getattr(ph, name)(s["rho_d"], s["uvel"], s["vvel"], s["wvel"], s["temp"], trc, *args)
    s["tracers"] = np.stack(trc)
    return s


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("device", [False, True])
def test_physics_modules_match_oracle(oracle_lib, gpu_lib, kind, device):
    case, halos, opts = _case(kind)
    st = pyphysics.state_of(case, seed=KINDS.index(kind))
    orc = pyphysics.Physics(case, "orc", halos, **opts)
    ph = Physics.from_case(case, halos=halos, **_gpu_opts(opts))
    dt = 0.1
    calls = [("les", (dt,)), ("sponge", (dt, 100 * dt, 0.3)), ("geostrophic", (dt, 43.0, 10.0, -2.0)),
             ("surface_fluxes", (dt,))]
    for name, args in calls:
        want = getattr(orc, name)(st, *args)
        got = _run_gpu(ph, name, st, args, device)
        _check("%s/%s/%s" % (kind, name, "device" if device else "host"), got, want, st)
    ph.close()


def test_les_out_of_place_equals_in_place(gpu_lib):
    import torch
    case, halos, _ = _case("immersed")
    st = pyphysics.state_of(case, seed=7)
    ph = Physics.from_case(case, halos=halos)
    names = ("rho_d", "uvel", "vvel", "wvel", "temp")
    a = {k: torch.from_numpy(st[k].copy()).cuda() for k in names}
    ta = [torch.from_numpy(st["tracers"][t].copy()).cuda() for t in range(st["tracers"].shape[0])]
    b = {k: torch.empty_like(a[k]) for k in names}
    tb = [torch.empty_like(x) for x in ta]
    ph.les_to(tuple(a[k] for k in names) + (ta,), tuple(b[k] for k in names) + (tb,), 0.1)
    ph.les(*[a[k] for k in names], ta, 0.1)
    ph.synchronize()
    for k in names[1:]:
        assert torch.equal(a[k], b[k]), k
    tke = [t.name for t in case.tracers].index("TKE")
    assert torch.equal(ta[tke], tb[tke])
    ph.close()


def test_module_api_on_a_coupler(oracle_lib, gpu_lib):
    """LES_Closure.init/apply, sponge_layer, geostrophic_wind_forcing and
    apply_surface_fluxes on a Coupler, in the ABL driver's order, against
    the oracle."""
    from porturb_b200 import (LES_Closure, apply_surface_fluxes, case_coupler, geostrophic_wind_forcing,
                              sponge_layer)
    from porturb_b200.physics import register_immersed_halos
    case, halos, _ = _case("plain", nx=36, ny=16, nz=18)
    c = case_coupler(case)
    register_immersed_halos(c, case)
    st = pyphysics.state_of(case, seed=11)
    for k, name in (("rho_d", "density_dry"), ("uvel", "uvel"), ("vvel", "vvel"), ("wvel", "wvel"),
                    ("temp", "temp")):
        c.get(name)[...] = st[k]
    for t, n in enumerate(c.get_tracer_names()):
        c.get(n)[...] = st["tracers"][t]
    LES_Closure().init(c)   # the TKE tracer exists already: same attributes, value reset to 0.1
    st["tracers"][[t.name for t in case.tracers].index("TKE")] = 0.1
    dt = 0.1
    geostrophic_wind_forcing(c, dt, 43.0, 10.0, 0.0)
    sponge_layer(c, dt, dt * 100, 0.1)
    apply_surface_fluxes(c, dt)
    LES_Closure().apply(c, dt)
    orc = pyphysics.Physics(case, "orc", halos)
    want = orc.geostrophic(st, dt, 43.0, 10.0, 0.0)
    want = orc.sponge(want, dt, dt * 100, 0.1)
    want = orc.surface_fluxes(want, dt)
    want = orc.les(want, dt)
    got = dict(rho_d=c.get("density_dry"), uvel=c.get("uvel"), vvel=c.get("vvel"), wvel=c.get("wvel"),
               temp=c.get("temp"), tracers=np.stack([c.get(n) for n in c.get_tracer_names()]))
    _check("coupler", got, want, st)


def _pg_state(case, seed):
    st = pyphysics.state_of(case, seed=seed)
    rng = np.random.default_rng(seed)
    st["uvel"] = st["uvel"] + 3.0 + rng.standard_normal(st["uvel"].shape)
    st["vvel"] = st["vvel"] - 1.0 + rng.standard_normal(st["vvel"].shape)
    return st


@pytest.mark.parametrize("update_cycles", [1, 3])
@pytest.mark.parametrize("device", [False, True])
def test_uniform_pg_matches_oracle_across_calls(oracle_lib, gpu_lib, update_cycles, device):
    """uniform_pg_wind_forcing over 7 calls with the wind disturbed between
    them: the carried state (counter, u0, v0, u, v) and the fields match."""
    from porturb_b200 import capi
    case, halos, _ = _case("plain")
    orc = pyphysics.Physics(case, "orc", halos)
    ph = Physics.from_case(case, halos=halos)
    st = _pg_state(case, 5)
    so, sg = np.zeros(5), capi.pu_uniform_pg_state()
    rng = np.random.default_rng(9)
    for call in range(7):
        want = orc.uniform_pg(st, 0.05, 2.0, update_cycles, so)
        got = _run_gpu(ph, "uniform_pg", st, (0.05, 2.0, update_cycles, sg), device)
        _check("uniform_pg/%d" % call, got, want, st)
        assert sg.counter == so[0]
        for i, k in enumerate(("u0", "v0", "u", "v")):
            assert abs(getattr(sg, k) - so[1 + i]) <= 1e-14 * abs(so[1 + i]), (call, k)
        st = want
        st["uvel"] = st["uvel"] + 0.3 * rng.standard_normal(st["uvel"].shape)
        st["vvel"] = st["vvel"] + 0.3 * rng.standard_normal(st["vvel"].shape)
    ph.close()


@pytest.mark.parametrize("device", [False, True])
def test_uniform_pg_height_matches_oracle(oracle_lib, gpu_lib, device):
    from porturb_b200.capi import PortUrbError
    case, halos, _ = _case("plain")
    dz = case.zlen / case.nz
    orc = pyphysics.Physics(case, "orc", halos)
    ph = Physics.from_case(case, halos=halos)
    st = _pg_state(case, 6)
    for height in (3.3 * dz, 7.5 * dz, 0.5 * dz, (case.nz + 0.4) * dz):
        args = (0.05, height, 8.0, 0.5, 3.0)
        want = orc.uniform_pg_height(st, *args)
        got = _run_gpu(ph, "uniform_pg_height", st, args, device)
        _check("uniform_pg_height/%.3f" % height, got, want, st)
    with pytest.raises(PortUrbError):
        _run_gpu(ph, "uniform_pg_height", st, (0.05, 0.4 * dz, 8.0, 0.5, 3.0), device)
    ph.close()


def test_uniform_pg_module_api_on_a_coupler(oracle_lib, gpu_lib):
    """uniform_pg_wind_forcing keeps its state in the coupler options, as the
    reference does, and needs no immersed arrays on the coupler."""
    from porturb_b200 import case_coupler, uniform_pg_wind_forcing, uniform_pg_wind_forcing_height
    case, halos, _ = _case("plain", nx=36, ny=16, nz=18)
    c = case_coupler(case)
    st = _pg_state(case, 12)
    for k, name in (("uvel", "uvel"), ("vvel", "vvel")):
        c.get(name)[...] = st[k]
    orc = pyphysics.Physics(case, "orc", halos)
    so = np.zeros(5)
    want = dict(st)
    for _ in range(3):
        uniform_pg_wind_forcing(c, 0.1, 5.0, 2)
        want = orc.uniform_pg(want, 0.1, 5.0, 2, so)
        c.get("uvel")[...] += 0.25
        want["uvel"] = want["uvel"] + 0.25
    assert c.get_option("uniform_pg_wind_forcing_counter") == 3
    assert abs(c.get_option("uniform_pg_wind_forcing_u") - so[3]) <= 1e-14 * abs(so[3])
    dz = case.zlen / case.nz
    uniform_pg_wind_forcing_height(c, 0.1, 2.2 * dz, 7.0, 0.0, 4.0)
    want = orc.uniform_pg_height(want, 0.1, 2.2 * dz, 7.0, 0.0, 4.0)
    got = dict(want, uvel=c.get("uvel"), vvel=c.get("vvel"))
    _check("coupler_pg", got, want, st)


@pytest.mark.parametrize("device", [False, True])
def test_time_averager_matches_oracle_bit_for_bit(oracle_lib, gpu_lib, device):
    """pu_time_averager_accumulate over 5 calls with a changing state and a
    reset: the GPU kernel rounds every product and sum as the reference does,
    so it equals the oracle (itself equal to the reference's header) exactly."""
    import torch
    case, halos, _ = _case("plain")
    orc = pyphysics.Physics(case, "orc", halos)
    ph = Physics.from_case(case, halos=halos)
    st = pyphysics.state_of(case, seed=13)
    shape = (13,) + st["uvel"].shape
    ao = np.zeros(shape)
    ag = torch.zeros(shape, dtype=torch.float64, device="cuda") if device else np.zeros(shape)
    eo = eg = 0.0
    elapsed = 0.0
    rng = np.random.default_rng(5)
    for call in range(5):
        if call == 3:
            eo = eg = 0.0
            ao[:10] = 0
            ag[:10] = 0
        dt = 0.2
        eo = orc.time_average(st, ao, eo, elapsed, dt)
        if device:
            t = {k: torch.from_numpy(np.ascontiguousarray(st[k])).cuda() for k in ("rho_d", "uvel", "vvel", "wvel", "temp")}
            trc = [torch.from_numpy(np.ascontiguousarray(st["tracers"][i])).cuda() for i in range(st["tracers"].shape[0])]
            eg = ph.time_average(t["rho_d"], t["uvel"], t["vvel"], t["wvel"], t["temp"], trc, list(ag), eg, elapsed, dt)
            ph.synchronize()
            got = ag.cpu().numpy()
        else:
            trc = [np.ascontiguousarray(st["tracers"][i]) for i in range(st["tracers"].shape[0])]
            eg = ph.time_average(st["rho_d"], st["uvel"], st["vvel"], st["wvel"], st["temp"], trc, list(ag), eg,
                                 elapsed, dt)
            got = ag
        assert eg == eo
        assert np.array_equal(got, ao), (call, np.abs(got - ao).max())
        elapsed += dt
        st = dict(st)
        st["uvel"] = st["uvel"] + 0.3 * rng.standard_normal(st["uvel"].shape)
    ph.close()


def test_time_averager_module_api_on_a_coupler(oracle_lib, gpu_lib):
    """Time_Averager.init / accumulate / reset on a Coupler keep the arrays and
    the option time_averager_etime as the reference does."""
    from porturb_b200 import LES_Closure, Time_Averager, case_coupler
    case, halos, _ = _case("plain", nx=36, ny=16, nz=18)
    c = case_coupler(case)
    st = pyphysics.state_of(case, seed=14)
    for k, name in (("uvel", "uvel"), ("vvel", "vvel"), ("wvel", "wvel")):
        c.get(name)[...] = st[k]
    for t, n in enumerate(c.get_tracer_names()):
        c.get(n)[...] = st["tracers"][t]
    ta = Time_Averager()
    ta.init(c)
    orc = pyphysics.Physics(case, "orc", halos)
    avgs = np.zeros((13,) + st["uvel"].shape)
    etime = 0.0
    for call in range(3):
        ta.accumulate(c, 0.5)
        etime = orc.time_average(st, avgs, etime, c.get_option("elapsed_time"), 0.5)
        c.set_option("elapsed_time", c.get_option("elapsed_time") + 0.5)
    from porturb_b200 import capi
    for q, n in enumerate(capi.TAVG_NAMES):
        assert np.array_equal(c.get(n), avgs[q]), n
    assert c.get_option("time_averager_etime") == etime == 1.5
    ta.reset(c)
    assert c.get_option("time_averager_etime") == 0.0
    assert not c.get("avg_u").any() and c.get("long_avg_u").any()


@pytest.mark.parametrize("device", [False, True])
def test_edge_sponge_matches_oracle(oracle_lib, gpu_lib, device):
    """pu_edge_sponge_set_column / _apply against the oracle (itself equal to
    the reference's header): column means within 1e-14 of each field's
    magnitude (each value scaled by 1/(nx ny) before a compensated parallel
    sum, against the reference's sequential sum divided once), relaxed
    fields within the _check bound."""
    case, halos, _ = _case("plain")
    orc = pyphysics.Physics(case, "orc", halos)
    ph = Physics.from_case(case, halos=halos)
    st0 = pyphysics.state_of(case, seed=23)
    want_col = orc.edge_sponge_set_column(st0)
    trc0 = [np.ascontiguousarray(st0["tracers"][i]) for i in range(st0["tracers"].shape[0])]
    col = ph.edge_sponge_set_column(st0["rho_d"], st0["uvel"], st0["vvel"], st0["wvel"], st0["temp"], trc0)
    mags = np.array([np.abs(st0[k]).max() for k in ("rho_d", "uvel", "vvel", "wvel", "temp")])
    assert np.all(np.abs(col - want_col) <= 1e-14 * mags[:, None])
    st = pyphysics.state_of(case, seed=24)
    for props in ((0.1, 0.1, 0.1, 0.1), (0.3, 0.0, 0.0, 0.25)):
        want = orc.edge_sponge_apply(st, want_col, *props)
        got = _run_gpu(ph, "edge_sponge", st, (want_col,) + props, device)
        _check("edge_sponge/%s" % (props,), got, want, st)
    ph.close()


def test_edge_sponge_module_api_on_a_coupler(oracle_lib, gpu_lib):
    """EdgeSponge.set_column / apply on a Coupler, as the urban driver calls
    them (city.cpp:97, 137)."""
    from porturb_b200 import EdgeSponge, case_coupler
    case, halos, _ = _case("plain", nx=36, ny=16, nz=18)
    c = case_coupler(case)
    st = pyphysics.state_of(case, seed=25)
    for k, name in (("rho_d", "density_dry"), ("uvel", "uvel"), ("vvel", "vvel"), ("wvel", "wvel"), ("temp", "temp")):
        c.get(name)[...] = st[k]
    es = EdgeSponge()
    es.set_column(c)
    orc = pyphysics.Physics(case, "orc", halos)
    col = orc.edge_sponge_set_column(st)
    mags = np.array([np.abs(st[k]).max() for k in ("rho_d", "uvel", "vvel", "wvel", "temp")])
    assert np.all(np.abs(es.column - col) <= 1e-14 * mags[:, None])
    st2 = pyphysics.state_of(case, seed=26)
    for k, name in (("rho_d", "density_dry"), ("uvel", "uvel"), ("vvel", "vvel"), ("wvel", "wvel"), ("temp", "temp")):
        c.get(name)[...] = st2[k]
    es.apply(c, 0.01, 0.01, 0.01, 0.01)
    want = orc.edge_sponge_apply(st2, es.column, 0.01, 0.01, 0.01, 0.01)
    got = dict(want, rho_d=c.get("density_dry"), uvel=c.get("uvel"), vvel=c.get("vvel"), wvel=c.get("wvel"),
               temp=c.get("temp"))
    _check("coupler_edge_sponge", got, want, st2)
