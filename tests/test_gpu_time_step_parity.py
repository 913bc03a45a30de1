"""The reference-facing entry points against the CPU oracle.

* pu_dycore_time_step (time_step, dynamics_rk.h:103-137): conversion of the
  coupler arrays in (convert_coupler_to_dynamics, :1304-1352),
  ncycles = ceil(dt_phys/dt_dyn) SSPRK3 steps of dt_phys/ncycles, conversion
  back (convert_dynamics_to_coupler, :1251-1299), compared with the oracle's
  own time_step on the returned coupler arrays (density_dry, uvel, vvel,
  wvel, temp, tracers).  dt_phys = 2.5 dt_dyn, so ncycles = 3.
    - FP64 build vs the F64 oracle on the same cell profiles: L2 < 1e-7 and
      Linf < 1e-6 of the change the call made to each array (the bound of the
      resident-state parity tests).
    - FP32 build vs the REF oracle (bit-identical to the reference's own
      path) on the same cell profiles: L2 < 1e-5 and Linf < 1e-4 of each
      array's departure from its level mean.
* The GPU's own init (no profile override): cell and edge profiles
  (dynamics_rk.h:961-1008, 1145-1186) against the F64 oracle's -- FP64 build
  within the oracle's own summation error (nx*ny*2^-53 relative), FP32 build
  to 3 float ulps of the F64 oracle's values rounded to float -- and a
  time_step from the GPU's own profiles against the oracle's time_step from
  its own: FP64 build vs F64 within the bound above; FP32 build within 3x the
  reference path's own error against F64 (plus 1e-5) of the departure.
"""
import numpy as np
import pytest

import pyoracle
from porturb_b200 import Dycore, cases

pytestmark = pytest.mark.gpu

CASES = {
    "mixed_immersed": lambda: cases.small_mixed(),
    "plain_one_tracer": lambda: cases.small_mixed(immersed=False, ntr=1),
    "three_tracers": lambda: cases.small_mixed(ntr=3),
    "precursor_xy": lambda: cases.small_mixed(bc_x="precursor", bc_y="precursor"),
    "periodic_z": lambda: cases.small_mixed(bc_z="periodic", immersed=False),
    "coriolis": lambda: cases.small_mixed(latitude=43.29),
    "linear_edges": lambda: cases.small_mixed(weno_all=False, immersed=False),
    "sim2d": lambda: cases.small_mixed(ny=1, nx=24, nz=16),
    "bubble_small": lambda: cases.warm_bubble(nx=64, ny=4, nz=32, xlen=5000.0, ylen=312.5, zlen=2500.0,
                                              radius=500.0, x0=2500.0, z0=600.0),
}


def _windmill_case():
    """small_mixed with a rotor-disk projection weight summed into its
    immersed proportion (what init does with windmill_proj_weight,
    dynamics_rk.h:1019-1025); the sum is passed as the proportion."""
    case = cases.small_mixed(nx=24, ny=16, nz=16)
    k, j = np.meshgrid(np.arange(case.nz) + 0.5, np.arange(case.ny) + 0.5, indexing="ij")
    r = np.hypot(k - 8.0, j - 7.5)
    disk = np.where(r < 6.0, 0.3 * np.exp(-(r / 6.0) ** 2), 0.0)
    case.immersed_proportion[:, :, 8] += disk
    case.immersed_proportion[:, :, 9] += 0.5 * disk
    return case


CASES["windmill"] = _windmill_case
DT_FACTOR = 2.5          # dt_phys / dt_dyn: ncycles = 3


def _arrays(case, perturbed):
    rd, u, v, w, T, trc = case.coupler_arrays(perturbed=perturbed)
    return [np.ascontiguousarray(np.array(a, dtype=np.float64)) for a in (rd, u, v, w, T)] + \
           [np.ascontiguousarray(np.array(trc, dtype=np.float64))]


def _flat(arrs):
    return [a for a in arrs[:5]] + [t for t in arrs[5]]


def oracle_time_step(case, kind, dt_phys, own_profiles=True, cells=None):
    d = pyoracle.Dycore(case, kind)
    d.init_case()
    if cells is not None:
        d.set_hydrostasis(*cells)
    out = _arrays(case, True)
    d.time_step(out, dt_phys)
    c, e = d.get_hydrostasis()
    return _flat(out), c, e


def gpu_time_step(case, precision, dt_phys, cells=None):
    g = Dycore.from_case(case, precision=precision, device=0)
    base = _arrays(case, False)
    imm = np.ascontiguousarray(case.immersed_proportion)
    g.init(*base[:5], list(base[5]), imm if imm.any() else None)
    if cells is not None:
        g.set_hydrostasis(*cells)
    out = _arrays(case, True)
    trs = [np.ascontiguousarray(t) for t in out[5]]
    n = g.time_step(*out[:5], trs, dt_phys)
    c, e = g.get_hydrostasis()
    g.close()
    return out[:5] + trs, n, c, e


def change_err(a, b, base):
    """(L2, Linf) of a-b relative to the change b-base."""
    d = a - b
    ch = b - base
    if not d.any():
        return 0.0, 0.0
    return (np.sqrt(np.mean(d ** 2)) / (np.sqrt(np.mean(ch ** 2)) + 1e-300),
            np.abs(d).max() / (np.abs(ch).max() + 1e-300))


def departure_err(a, b):
    """(L2, Linf) of a-b relative to b's departure from its level means."""
    d = a - b
    if not d.any():
        return 0.0, 0.0
    dep = b - b.mean(axis=(1, 2), keepdims=True)
    return (np.sqrt(np.mean(d ** 2)) / (np.sqrt(np.mean(dep ** 2)) + 1e-300),
            np.abs(d).max() / (np.abs(dep).max() + 1e-300))


NAMES = ["density_dry", "uvel", "vvel", "wvel", "temp"]


@pytest.mark.parametrize("name", sorted(CASES))
def test_time_step_f64_matches_f64_oracle(name, oracle_lib, gpu_lib):
    case = CASES[name]()
    dt_phys = DT_FACTOR * oracle_lib.Dycore(case, "f64").compute_time_step()
    o, cells, _ = oracle_time_step(case, "f64", dt_phys)
    g, n, _, _ = gpu_time_step(case, "f64", dt_phys, cells=cells)
    assert n == 3
    base = _flat(_arrays(case, True))
    for q, (x, y, b) in enumerate(zip(g, o, base)):
        e2, ei = change_err(x, y, b)
        print(name, NAMES[q] if q < 5 else "tracer%d" % (q - 5), "f64 vs F64 (of change): %.2e / %.2e" % (e2, ei))
        assert e2 < 1e-7 and ei < 1e-6, (name, q, e2, ei)


@pytest.mark.parametrize("name", sorted(CASES))
def test_time_step_f32_matches_reference_path(name, oracle_lib, gpu_lib):
    case = CASES[name]()
    dt_phys = DT_FACTOR * oracle_lib.Dycore(case, "ref").compute_time_step()
    o, cells, _ = oracle_time_step(case, "ref", dt_phys)
    g, n, _, _ = gpu_time_step(case, "f32", dt_phys, cells=cells)
    assert n == 3
    for q, (x, y) in enumerate(zip(g, o)):
        e2, ei = departure_err(x, y)
        print(name, NAMES[q] if q < 5 else "tracer%d" % (q - 5), "f32 vs REF (of departure): %.2e / %.2e" % (e2, ei))
        assert e2 < 1e-5 and ei < 1e-4, (name, q, e2, ei)


PROFILE_CASES = {
    "mixed_immersed": lambda: cases.small_mixed(),
    "bubble_small": CASES["bubble_small"],
    "abl_block_64x64x48": lambda: cases.abl_neutral(nx=64, ny=64, nz=48),
    "urban_block_64x64x32": lambda: cases.urban_canopy(nx=64, ny=64, nz=32),
    "windmill": _windmill_case,
}


@pytest.mark.parametrize("name", sorted(PROFILE_CASES))
def test_gpu_init_profiles_match_oracle(name, oracle_lib, gpu_lib):
    case = PROFILE_CASES[name]()
    f64 = pyoracle.Dycore(case, "f64")
    f64.init_case()
    c64, e64 = f64.get_hydrostasis()
    ref = pyoracle.Dycore(case, "ref")
    ref.init_case()
    cref, eref = ref.get_hydrostasis()
    for prec in ("f64", "f32"):
        g = Dycore.from_case(case, precision=prec, device=0)
        base = _arrays(case, False)
        imm = np.ascontiguousarray(case.immersed_proportion)
        g.init(*base[:5], list(base[5]), imm if imm.any() else None)
        cg, eg = g.get_hydrostasis()
        g.close()
        for kind, got, want, wref in (("cells", cg, c64, cref), ("edges", eg, e64, eref)):
            for q in range(3):
                a, b = np.asarray(got[q]), np.asarray(want[q])
                if prec == "f64":
                    # The oracle sums each level's nx*ny cells in order in
                    # double (error up to nx*ny*2^-53 relative); the GPU's
                    # sums are compensated.
                    rel = np.abs(a - b).max() / np.abs(b).max()
                    assert rel < case.nx * case.ny * 2.0 ** -53 + 1e-14, (name, prec, kind, q, rel)
                else:
                    b32 = b.astype(np.float32).astype(np.float64)
                    ulps = np.abs(a - b32) / np.spacing(np.abs(b32).astype(np.float32)).astype(np.float64)
                    rel_ref = np.abs(a - np.asarray(wref[q])).max() / np.abs(np.asarray(wref[q])).max()
                    print(name, kind, q, "f32 build vs float(F64): %.1f ulp; vs REF's float sums: %.2e relative"
                          % (ulps.max(), rel_ref))
                    assert ulps.max() <= 3, (name, kind, q, ulps.max())


OWN_CASES = ["mixed_immersed", "plain_one_tracer", "bubble_small", "windmill", "sim2d"]


@pytest.mark.parametrize("name", OWN_CASES)
def test_time_step_on_own_profiles(name, oracle_lib, gpu_lib):
    """The whole reference-facing path, init included, on each side's own
    profiles."""
    case = CASES[name]()
    dt_phys = DT_FACTOR * oracle_lib.Dycore(case, "f64").compute_time_step()
    o64, _, _ = oracle_time_step(case, "f64", dt_phys)
    oref, _, _ = oracle_time_step(case, "ref", dt_phys)
    g64, n, _, _ = gpu_time_step(case, "f64", dt_phys)
    assert n == 3
    g32, n, _, _ = gpu_time_step(case, "f32", dt_phys)
    base = _flat(_arrays(case, True))
    for q in range(len(o64)):
        e2, ei = change_err(g64[q], o64[q], base[q])
        assert e2 < 1e-7 and ei < 1e-6, (name, q, e2, ei)
        g2, gi = departure_err(g32[q], o64[q])
        r2, ri = departure_err(oref[q], o64[q])
        print(name, NAMES[q] if q < 5 else "tracer%d" % (q - 5),
              "own profiles, of departure: f64 build %.1e; f32 build %.1e / %.1e; reference path %.1e / %.1e"
              % (e2, g2, gi, r2, ri))
        assert g2 <= 3 * r2 + 1e-5 and gi <= 3 * ri + 1e-4, (name, q, g2, r2, gi, ri)
