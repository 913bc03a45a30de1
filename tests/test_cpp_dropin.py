"""The C++ drop-in module (porturb_b200/cpp/dynamics_rk.h) used the way the
reference's drivers use Dynamics_Euler_Stratified_WenoFV.  The build runs on
CPU; the run needs a GPU and must reproduce the Python front end's results."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "tests", "cpp", "_build", "dropin_driver")


def build_driver():
    from porturb_b200 import build
    import importlib.util
    spec = importlib.util.spec_from_file_location("build_driver", os.path.join(ROOT, "tests", "cpp", "build_driver.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    exe = mod.build(os.path.dirname(build.build()))
    if exe is None:
        pytest.skip("no reference tree to build the stand-in coupler and no prebuilt driver")
    return exe


def test_dropin_builds_and_links():
    assert os.path.exists(build_driver())


def _write_input(path, case, ncalls, dt_phys):
    o = case.options
    rd, u, v, w, T, trc = case.coupler_arrays(perturbed=False)
    prd, pu_, pv, pw, pT, ptr = case.coupler_arrays(perturbed=True)
    ntr = len(case.tracers)
    with open(path, "wb") as f:
        np.array([case.nx, case.ny, case.nz, ntr, ncalls], np.int32).tofile(f)
        np.array([case.xlen, case.ylen, case.zlen, dt_phys, o["R_d"], o["R_v"], o["cp_d"], o["gamma_d"], o["C0"],
                  o["grav"], o["cfl"]], np.float64).tofile(f)
        np.array([[t.name for t in case.tracers].index("water_vapor")], np.int32).tofile(f)
        np.array([t.positive for t in case.tracers], np.int32).tofile(f)
        np.array([t.adds_mass for t in case.tracers], np.int32).tofile(f)
        np.concatenate([np.stack([rd, u, v, w, T]).ravel(), trc.ravel()]).tofile(f)
        np.concatenate([np.stack([prd, pu_, pv, pw, pT]).ravel(), ptr.ravel()]).tofile(f)


@pytest.mark.gpu
@pytest.mark.parametrize("grid", ["small", "abl_32x32x64"])
def test_dropin_matches_python_front_end(tmp_path, grid):
    """abl_32x32x64: two 32-level chunks, so time_step on the drop-in's host
    arrays takes the overlapped form (and the Python front end's too)."""
    from porturb_b200 import Dycore, cases
    exe = build_driver()
    case = cases.small_mixed(immersed=False) if grid == "small" else cases.abl_neutral(nx=32, ny=32, nz=64)
    g = Dycore.from_case(case, precision="f32")
    dt_phys = 2.5 * g.compute_time_step()
    _write_input(tmp_path / "in.bin", case, 2, dt_phys)
    r = subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = np.fromfile(tmp_path / "out.bin", np.float64).reshape(5 + len(case.tracers), case.nz, case.ny, case.nx)
    rd, u, v, w, T, trc = [np.ascontiguousarray(a) for a in case.coupler_arrays(perturbed=False)]
    g.init(rd, u, v, w, T, list(trc), None)
    arrs = [np.ascontiguousarray(a.copy()) for a in case.coupler_arrays(perturbed=True)]
    trs = [np.ascontiguousarray(a) for a in arrs[5]]
    for _ in range(2):
        g.time_step(*arrs[:5], trs, dt_phys)
    ref = np.concatenate([np.stack(arrs[:5]), np.stack(trs)])
    assert np.array_equal(out, ref)


@pytest.mark.gpu
def test_physics_dropin_chain_matches_python_front_end(tmp_path):
    """The drop-in LES closure, sponge, geostrophic forcing, surface-flux and
    time-averager headers with the dycore, in the boundary-layer driver's
    order (abl_neutral.cpp:93-108), give the same arrays as the same chain
    through the Python API."""
    from porturb_b200 import Dycore, cases
    from porturb_b200.physics import Physics
    build_driver()
    exe = os.path.join(ROOT, "tests", "cpp", "_build", "physics_driver")
    case = cases.abl_neutral(nx=32, ny=16, nz=24)
    halos = cases.immersed_halos(case)
    g = Dycore.from_case(case, precision="f32")
    dt = 2 * g.compute_time_step()
    o = case.options
    lat_g, u_g, v_g, t_sp, top = 43.29, 10.0, 0.0, 100 * dt, 0.1
    ncalls = 2
    base = [np.asarray(a) for a in case.coupler_arrays(perturbed=False)]
    pert = [np.asarray(a) for a in case.coupler_arrays(perturbed=True)]
    with open(tmp_path / "in.bin", "wb") as f:
        np.array([case.nx, case.ny, case.nz, ncalls], np.int32).tofile(f)
        np.array([case.xlen, case.ylen, case.zlen, dt, o["R_d"], o["R_v"], o["cp_d"], o["gamma_d"], o["C0"],
                  o["grav"], o["cfl"], lat_g, u_g, v_g, t_sp, top], np.float64).tofile(f)
        for st in (base, pert):
            np.concatenate([np.stack(st[:5]).ravel(), st[5][0].ravel()]).astype(np.float64).tofile(f)
        np.concatenate([h.ravel() for h in halos]).tofile(f)
    r = subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = np.fromfile(tmp_path / "out.bin", np.float64).reshape(20, case.nz, case.ny, case.nx)

    rd, u, v, w, T, trc = [np.ascontiguousarray(a) for a in base]
    g.init(rd, u, v, w, T, [np.ascontiguousarray(t) for t in trc], None)
    a = [np.ascontiguousarray(x.copy()) for x in pert[:5]]
    trs = [np.ascontiguousarray(t.copy()) for t in pert[5]]
    ph = Physics.from_case(case, halos=halos)
    avgs = np.zeros((13, case.nz, case.ny, case.nx))
    etime = elapsed = 0.0
    for _ in range(ncalls):
        ph.geostrophic(*a, trs, dt, lat_g, u_g, v_g)
        g.time_step(*a, trs, dt)
        ph.sponge(*a, trs, dt, t_sp, top)
        ph.surface_fluxes(*a, trs, dt)
        ph.les(*a, trs, dt)
        etime = ph.time_average(*a, trs, avgs, etime, elapsed, dt)
        elapsed += dt
    ref = np.concatenate([np.stack(a), np.stack(trs), avgs])
    assert np.array_equal(out, ref)
    assert not np.array_equal(ref[6], np.asarray(pert[5][1]))   # the closure changed TKE
    assert np.abs(avgs[4]).max() > 0                             # the averager saw the fluctuations


@pytest.mark.gpu
def test_pg_forcing_dropin_matches_python_front_end(tmp_path):
    """The drop-in uniform_pg_wind_forcing / _height and edge-sponge headers on
    a coupler with no immersed arrays give the same arrays and carried options
    as the Python module API."""
    from porturb_b200 import EdgeSponge, case_coupler, cases, uniform_pg_wind_forcing, uniform_pg_wind_forcing_height
    build_driver()
    exe = os.path.join(ROOT, "tests", "cpp", "_build", "pg_driver")
    case = cases.abl_neutral(nx=24, ny=20, nz=16)
    rng = np.random.default_rng(3)
    u = 4.0 + rng.standard_normal((case.nz, case.ny, case.nx))
    v = -1.0 + rng.standard_normal((case.nz, case.ny, case.nx))
    dz = case.zlen / case.nz
    ncalls, cycles, dt, tau = 4, 2, 0.1, 3.0
    height, u0, v0, tau_h = 5.3 * dz, 7.0, 0.5, 2.0
    with open(tmp_path / "in.bin", "wb") as f:
        np.array([case.nx, case.ny, case.nz, ncalls, cycles], np.int32).tofile(f)
        np.array([case.xlen, case.ylen, case.zlen, dt, tau, height, u0, v0, tau_h, 0.0], np.float64).tofile(f)
        u.tofile(f)
        v.tofile(f)
    r = subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = np.fromfile(tmp_path / "out.bin", np.float64)
    n = u.size
    c = case_coupler(case)
    c.get("uvel")[...] = u
    c.get("vvel")[...] = v
    c.get("density_dry")[...] = 0.0   # as the driver's freshly allocated arrays
    c.get("wvel")[...] = 0.0
    c.get("temp")[...] = 0.0
    es = EdgeSponge()
    es.set_column(c)
    for _ in range(ncalls):
        uniform_pg_wind_forcing(c, dt, tau, cycles)
        c.get("uvel")[...] += 0.25
    st = [c.get_option("uniform_pg_wind_forcing_" + k) for k in ("counter", "u0", "v0", "u", "v")]
    uniform_pg_wind_forcing_height(c, dt, height, u0, v0, tau_h)
    assert np.array_equal(out[:n].reshape(u.shape), c.get("uvel"))
    assert np.array_equal(out[n:2 * n].reshape(v.shape), c.get("vvel"))
    assert np.array_equal(out[2 * n:2 * n + 5], np.array(st, np.float64))
    assert not np.array_equal(c.get("vvel"), v)
    es.apply(c, 0.2, 0.1, 0.15, 0.25)
    for q, nm in enumerate(("density_dry", "uvel", "vvel", "wvel", "temp")):
        assert np.array_equal(out[2 * n + 5 + q * n:2 * n + 5 + (q + 1) * n].reshape(u.shape), c.get(nm)), nm
