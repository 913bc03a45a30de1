"""Run one of the synthetic cases on the GPU dycore and report its speed.

    python -m porturb_b200.run_case abl_neutral --nx 256 --ny 256 --nz 64 --steps 3
    python -m porturb_b200.run_case abl_neutral --nz 64 --learned --train-steps 300
    python -m porturb_b200.run_case urban_canopy --nx 1024 --ny 1024 --nz 256 --dx 1 --steps 300 --diag-every 50
    python -m porturb_b200.run_case abl_neutral --nx 512 --ny 512 --nz 256 --steps 500 --compare
    python -m porturb_b200.run_case abl_neutral --driver --compare --steps 50
    python -m porturb_b200.run_case urban_canopy --driver --chain periodic --compare --steps 100

Plain mode advances the FP32 (or --precision f64) dycore; --learned first
harvests stencils from the initial state, trains the network on the GPU and
then advances with learned weights; --modules times the physics modules
(LES closure, sponge, geostrophic forcing, surface fluxes) instead; --driver
runs the reference driver's whole chain of modules per dt_phys (--chain abl,
city or periodic; with --compare, the FP32 and FP64 dycore in the same chain
from the same state, with the errors per coupler array).  Prints
one JSON line with the per-kernel CUDA-event times and, in learned mode, the
fallback fraction.  --compare runs the plain FP32 form, the learned form
(trained on stencils harvested from the initial state) and the FP64 build
from the same initial state for `steps` steps each and reports their rates
and, per prognostic, the L2 and Linf error of the FP32 forms against the
FP64 build relative to its departure from the hydrostatic background.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import cases
from .dycore import Dycore

def _dx(a):
    return {} if a.dx is None else {"dx": a.dx}


CASES = {
    "abl_neutral": lambda a: cases.abl_neutral(nx=a.nx, ny=a.ny, nz=a.nz, **_dx(a)),
    "warm_bubble": lambda a: cases.warm_bubble(nx=a.nx, ny=a.ny, nz=a.nz),
    "urban_canopy": lambda a: cases.urban_canopy(nx=a.nx, ny=a.ny, nz=a.nz, **_dx(a)),
}


def run_modules(case, a):
    """Each physics module `steps` times on device copies of the coupler
    arrays (FP64); the LES closure out of place (kernel time by CUDA events)."""
    import torch
    from .physics import Physics
    ph = Physics.from_case(case)
    rd, u, v, w, T, trc = [np.ascontiguousarray(x) for x in case.coupler_arrays(perturbed=True)]
    dev = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()
    A = [dev(x) for x in (rd, u, v, w, T)]
    At = [dev(trc[t]) for t in range(trc.shape[0])]
    B = [torch.empty_like(x) for x in A]
    Bt = [torch.empty_like(x) for x in At]
    dt = 0.1
    les_ms = []
    for _ in range(a.steps):
        ph.les_to(tuple(A) + (At,), tuple(B) + (Bt,), dt)
        les_ms.append(ph.last_les_ms())
    out = {"case": a.case, "grid": [a.nx, a.ny, a.nz], "steps": a.steps, "les_kernel_ms": les_ms}
    for name, args in (("sponge", (dt, 100 * dt, 0.25)), ("geostrophic", (dt, 43.29, 10.0, 0.0)),
                       ("surface_fluxes", (dt,))):
        t0 = time.perf_counter()
        for _ in range(a.steps):
            getattr(ph, name)(*A, At, *args)
        ph.synchronize()
        out[name + "_ms"] = (time.perf_counter() - t0) * 1e3 / max(a.steps, 1)
    ph.close()
    return out


CHAINS = {
    "abl": "boundary layer (abl_neutral.cpp:93-108)",
    "city": "urban with edge sponge (city.cpp:137-142)",
    "periodic": "periodic urban driven by a pressure gradient (cubes_periodic.cpp:144-156)",
    "dycore": "the dycore's time_step alone (no other module)",
}


def _chain_of(a):
    chain = getattr(a, "chain", None)
    if chain:
        return chain
    return "city" if a.case == "urban_canopy" else "abl"


def _driver_run(case, a, precision, calls, dt=None, warm=1):
    """One driver run: a coupler of the case on this GPU, the chain's modules
    initialised as the reference's drivers do (LES closure, dycore, time
    averager), the perturbed state, then `warm` untimed and `calls` timed
    calls of dt_phys = 10 dycore steps (or `dt`).  Per call:
      abl      -- geostrophic forcing, dycore, sponge, surface fluxes, LES
                  closure, time averager (abl_neutral.cpp:93-108), the sponge
                  over the top 300 m of the domain (the boundary layer's
                  damping layer; the reference driver's top_prop is 0.1);
      city     -- edge sponge, dycore, sponge, surface fluxes, LES closure,
                  time averager (city.cpp:137-142);
      periodic -- the mean wind at 100 m relaxed to (10, 0) m/s on a time
                  scale of 100 dt_phys, dycore, LES closure, surface fluxes,
                  time averager (cubes_periodic.cpp:144-156);
      dycore   -- the dycore alone (the same init, no other module applied).
    Returns the coupler, dt_phys, the ms per timed call (CUDA events) and
    the dycore steps per call."""
    import torch
    from . import (Dynamics_Euler_Stratified_WenoFV, EdgeSponge, LES_Closure, Time_Averager, apply_surface_fluxes,
                   assign_coupler_state, case_coupler, geostrophic_wind_forcing, sponge_layer)
    from .physics import register_immersed_halos, uniform_pg_wind_forcing_height
    chain = _chain_of(a)
    c = case_coupler(case, device="cuda:%d" % torch.cuda.current_device())
    register_immersed_halos(c, case)
    les, dyn, tavg, edge = LES_Closure(), Dynamics_Euler_Stratified_WenoFV(precision=precision), Time_Averager(), \
        EdgeSponge()
    les.init(c)
    dyn.init(c)
    tavg.init(c)
    if chain == "city":
        edge.set_column(c)
    assign_coupler_state(c, case, perturbed=True)
    if dt is None:
        dt = 10 * dyn.compute_time_step(c)
    sub = []

    def call():
        if chain == "dycore":
            sub.append(dyn.time_step(c, dt))
            c.set_option("elapsed_time", c.get_option("elapsed_time") + dt)
            return
        if chain == "city":
            edge.apply(c, 0.01, 0.01, 0.01, 0.01)
        elif chain == "abl":
            geostrophic_wind_forcing(c, dt, 43.289340204, 10.0, 0.0)
        else:
            uniform_pg_wind_forcing_height(c, dt, 100.0, 10.0, 0.0, dt * 100)
        sub.append(dyn.time_step(c, dt))
        if chain == "periodic":
            les.apply(c, dt)
            apply_surface_fluxes(c, dt)
        else:
            sponge_layer(c, dt, dt if chain == "city" else dt * 100,
                         0.02 if chain == "city" else min(1.0, 300.0 / case.zlen))
            apply_surface_fluxes(c, dt)
            les.apply(c, dt)
        tavg.accumulate(c, dt)
        c.set_option("elapsed_time", c.get_option("elapsed_time") + dt)

    for _ in range(warm):
        call()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(calls):
        call()
    e1.record()
    torch.cuda.synchronize()
    return c, dt, e0.elapsed_time(e1) / max(calls, 1), sub[-1]


def _release(c):
    for h in list(c.module_state.values()):
        if hasattr(h, "close"):
            h.close()
    c.module_state.clear()


def run_driver(case, a):
    """The reference driver's loop with this package's modules on device
    coupler arrays (the chains of `_driver_run`); CUDA-event time of `steps`
    calls after one."""
    c, dt, ms, sub = _driver_run(case, a, a.precision, a.steps)
    _release(c)
    return {"case": a.case, "grid": [a.nx, a.ny, a.nz], "driver": CHAINS[_chain_of(a)], "calls": a.steps,
            "dycore_steps_per_call": sub, "ms_per_call": ms, "cell_steps_per_s": case.ncells * sub / (ms / 1e3),
            "note": "cell-steps/s of the whole driver step: the dycore's 10 steps and the modules beside it"}


def coupler_errors(X, D):
    """Per coupler array (density_dry, uvel, vvel, wvel, temp, tracers): L2
    and Linf of X - D over D's departure from its level means (FP64 on the
    GPU)."""
    import torch
    out = {}
    for name, x in X.items():
        d = D[name].to(torch.float64)
        diff = x.to(torch.float64) - d
        dep = d - d.mean(dim=(1, 2), keepdim=True)
        dl2, dli = float(torch.sqrt(torch.mean(diff * diff))), float(diff.abs().max())
        pl2, pli = float(torch.sqrt(torch.mean(dep * dep))), float(dep.abs().max())
        out[name] = {"l2": dl2 / pl2 if pl2 > 0 else (0.0 if dl2 == 0 else None),
                     "linf": dli / pli if pli > 0 else (0.0 if dli == 0 else None)}
        del d, diff, dep
    return out


def run_driver_compare(case, a):
    """The driver chain with the FP32 dycore and with the FP64 build from the
    same initial state and the same dt_phys, `steps` timed calls each (after
    none: every dycore step of the run is in the timed calls): rates and, per
    coupler array, the FP32 run's error against the FP64 run."""
    import torch
    names = ["density_dry", "uvel", "vvel", "wvel", "temp"]
    c, dt, ms32, sub = _driver_run(case, a, "f32", a.steps, warm=0)
    keep = {n: c.get(n).clone() for n in names + list(c.get_tracer_names())}
    _release(c)
    del c
    torch.cuda.empty_cache()
    c, _, ms64, _ = _driver_run(case, a, "f64", a.steps, dt=dt, warm=0)
    ref = {n: c.get(n) for n in keep}
    errs = coupler_errors(keep, ref)
    _release(c)
    n = case.ncells * sub
    return {"case": a.case, "grid": [a.nx, a.ny, a.nz], "driver": CHAINS[_chain_of(a)], "calls": a.steps,
            "dycore_steps": a.steps * sub, "dt_phys": dt,
            "f32": {"ms_per_call": ms32, "cell_steps_per_s": n / (ms32 / 1e3)},
            "f64": {"ms_per_call": ms64, "cell_steps_per_s": n / (ms64 / 1e3)},
            "f32_vs_f64": errs,
            "error_norm": "L2 and Linf of (FP32 run - FP64 run) over the FP64 run's departure from its level means",
            "note": "the physics modules are FP64 in both runs; only the dycore's precision differs"}


def _snapshot(g, S, shape):
    """Conserved variables of a handle as one FP64 device tensor (S, nz, ny, nx)."""
    import torch
    from . import capi
    t = torch.empty((S,) + tuple(shape), dtype=torch.float64, device="cuda:%d" % g.cfg.device)
    capi.check(g.lib.pu_dycore_get_conserved(g.h, t.data_ptr(), t[5].data_ptr() if S > 5 else None,
                                             capi.PU_MEM_DEVICE))
    return t


def field_errors(X, D, cells, nz):
    """Per prognostic: L2 and Linf of X - D over D's departure from the
    hydrostatic background (rho_h, 0, 0, 0, rho_h*theta_h, 0 for tracers),
    computed on the GPU in FP64.  A field that is zero in D and in X reports 0;
    one that is zero only in D reports None."""
    import torch
    hs = 4
    r = torch.tensor(np.asarray(cells[0][hs:hs + nz]), dtype=torch.float64, device=D.device)
    t = torch.tensor(np.asarray(cells[1][hs:hs + nz]), dtype=torch.float64, device=D.device)
    names = ["rho", "rho_u", "rho_v", "rho_w", "rho_theta"] + ["tracer%d" % q for q in range(D.shape[0] - 5)]
    out = {}
    for f in range(D.shape[0]):
        d = D[f]
        dep = d - r[:, None, None] if f == 0 else (d - (r * t)[:, None, None] if f == 4 else d)
        diff = X[f] - d
        dl2, dli = float(torch.sqrt(torch.mean(diff * diff))), float(diff.abs().max())
        pl2, pli = float(torch.sqrt(torch.mean(dep * dep))), float(dep.abs().max())
        out[names[f]] = {"l2": dl2 / pl2 if pl2 > 0 else (0.0 if dl2 == 0 else None),
                         "linf": dli / pli if pli > 0 else (0.0 if dli == 0 else None)}
        del dep, diff
    return out


def run_compare(case, a):
    """Plain FP32, learned and FP64 from the same initial state: rates and
    errors against FP64 after `steps` steps."""
    import torch
    N, S, shape = case.ncells, 5 + len(case.tracers), (case.nz, case.ny, case.nx)
    base = [np.ascontiguousarray(x) for x in case.coupler_arrays(perturbed=False)]
    pert = [np.ascontiguousarray(x) for x in case.coupler_arrays(perturbed=True)]
    prop = np.ascontiguousarray(case.immersed_proportion)
    prop = prop if prop.any() else None
    out = {"case": a.case, "grid": [case.nx, case.ny, case.nz], "steps": a.steps, "mode": "compare"}

    def timed(g, dt, n):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        g.advance(dt, n)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    g = Dycore.from_case(case, precision="f32")
    g.init(*base[:5], list(base[5]), prop)
    g.load_state(*pert[:5], list(pert[5]))
    dt = g.compute_time_step()
    g.learned_harvest(a.harvest, seed=1)
    tr = g.learned_train(a.train_steps, batch=a.batch, lr=2e-3, seed=3)
    ms = timed(g, dt, a.steps)
    P = _snapshot(g, S, shape)
    out["plain"] = {"cell_steps_per_s": N * a.steps / (ms / 1e3), "ms_per_step": ms / a.steps}
    g.load_state(*pert[:5], list(pert[5]))
    g.set_weno_mode("learned")
    g.learned_set_threshold(a.threshold)
    g.learned_counts()
    ms = timed(g, dt, a.steps)
    nl, nf = g.learned_counts()
    L = _snapshot(g, S, shape)
    out["learned"] = {"cell_steps_per_s": N * a.steps / (ms / 1e3), "ms_per_step": ms / a.steps,
                      "threshold": a.threshold, "fallback_frac": nf / max(1, nl + nf),
                      "training": dict(tr, batch=a.batch)}
    g.close()
    h = Dycore.from_case(case, precision="f64")
    h.init(*base[:5], list(base[5]), prop)
    h.load_state(*pert[:5], list(pert[5]))
    ms = timed(h, dt, a.steps)
    D = _snapshot(h, S, shape)
    cells, _ = h.get_hydrostasis()
    h.close()
    out["f64"] = {"cell_steps_per_s": N * a.steps / (ms / 1e3), "ms_per_step": ms / a.steps}
    out["plain_vs_f64"] = field_errors(P, D, cells, case.nz)
    out["learned_vs_f64"] = field_errors(L, D, cells, case.nz)
    out["error_norm"] = "L2 and Linf of (X - FP64) over the FP64 field's departure from the hydrostatic background"
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=sorted(CASES))
    ap.add_argument("--nx", type=int, default=256)
    ap.add_argument("--ny", type=int, default=256)
    ap.add_argument("--nz", type=int, default=128)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--dx", type=float, default=None, help="grid spacing in m (the case's default if absent)")
    ap.add_argument("--diag-every", type=int, default=0,
                    help="FP64 compensated mass / rho*theta / energy sums every N steps (timed with the steps)")
    ap.add_argument("--precision", default="f32", choices=["f32", "f64"])
    ap.add_argument("--learned", action="store_true")
    ap.add_argument("--harvest", type=int, default=1 << 18)
    ap.add_argument("--train-steps", type=int, default=300)
    ap.add_argument("--threshold", type=float, default=0.5)
    ap.add_argument("--batch", type=int, default=16384, help="training batch (--learned, --compare)")
    ap.add_argument("--compare", action="store_true",
                    help="plain FP32, learned and FP64 from the same initial state: rates and errors against FP64")
    ap.add_argument("--driver", action="store_true",
                    help="run the reference driver's module chain per dt_phys (boundary layer or urban) on device "
                         "coupler arrays")
    ap.add_argument("--chain", choices=sorted(CHAINS), default=None,
                    help="--driver: the module chain (default: city for urban_canopy, abl otherwise)")
    ap.add_argument("--modules", action="store_true",
                    help="time the physics modules (LES closure, sponge, geostrophic forcing, surface fluxes) "
                         "on the case's coupler arrays instead of dycore steps")
    a = ap.parse_args(argv)

    case = CASES[a.case](a)
    if a.driver and a.compare:
        print(json.dumps(run_driver_compare(case, a)), flush=True)
        return
    if a.compare:
        print(json.dumps(run_compare(case, a)), flush=True)
        return
    if a.modules:
        print(json.dumps(run_modules(case, a)), flush=True)
        return
    if a.driver:
        print(json.dumps(run_driver(case, a)), flush=True)
        return
    g = Dycore.from_case(case, precision=a.precision)
    rd, u, v, w, T, trc = [np.ascontiguousarray(x) for x in case.coupler_arrays(perturbed=True)]
    prop = np.ascontiguousarray(case.immersed_proportion)
    g.init(rd, u, v, w, T, list(trc), prop if prop.any() else None)
    dt = g.compute_time_step()
    out = {"case": a.case, "grid": [a.nx, a.ny, a.nz], "precision": a.precision, "steps": a.steps,
           "weno": "learned" if a.learned else "plain"}
    if a.learned:
        g.learned_harvest(a.harvest, seed=1)
        out["training"] = g.learned_train(a.train_steps, batch=a.batch, lr=2e-3, seed=3)
        g.set_weno_mode("learned")
        g.learned_set_threshold(a.threshold)
        g.learned_counts()
    g.synchronize()
    diags = []
    if a.diag_every > 0:
        diags.append(dict(step=0, **{k: v for k, v in g.diagnostics().items() if k != "tracer_mass"}))
    g.profile(True)
    t0 = time.perf_counter()
    if a.diag_every > 0:
        done = 0
        while done < a.steps:
            n = min(a.diag_every, a.steps - done)
            g.advance(dt, n)
            done += n
            diags.append(dict(step=done, **{k: v for k, v in g.diagnostics().items() if k != "tracer_mass"}))
    else:
        g.advance(dt, a.steps)
    g.synchronize()
    wall = time.perf_counter() - t0
    if diags:
        out["diagnostics"] = diags
        out["relative_drift"] = {k: abs(diags[-1][k] - diags[0][k]) / abs(diags[0][k])
                                 for k in ("mass", "rho_theta", "total_energy")}
    prof = g.profile_read()
    g.profile(False)
    out["ms_per_step"] = wall * 1e3 / max(a.steps, 1)
    out["kernel_ms"] = {k: v[0] / max(v[1], 1) for k, v in prof.items()}
    out["cell_steps_per_s"] = case.ncells * a.steps / wall
    if a.learned:
        nl, nf = g.learned_counts()
        out["fallback_frac"] = nf / max(1, nl + nf)
    g.close()
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
