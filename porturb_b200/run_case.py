"""Run one of the synthetic cases on the GPU dycore and report its speed.

    python -m porturb_b200.run_case abl_neutral --nx 256 --ny 256 --nz 64 --steps 3
    python -m porturb_b200.run_case abl_neutral --nz 64 --learned --train-steps 300
    python -m porturb_b200.run_case urban_canopy --nx 1024 --ny 1024 --nz 256 --dx 1 --steps 300 --diag-every 50

Plain mode advances the FP32 (or --precision f64) dycore; --learned first
harvests stencils from the initial state, trains the network on the GPU and
then advances with learned weights; --modules times the physics modules
(LES closure, sponge, geostrophic forcing, surface fluxes) instead; --driver
runs the reference driver's whole chain of modules per dt_phys.  Prints
one JSON line with the per-kernel CUDA-event times and, in learned mode, the
fallback fraction.
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


def run_driver(case, a):
    """The reference driver's loop with this package's modules on device
    coupler arrays: per call of dt_phys = 10 dycore steps, the boundary-layer
    chain (abl_neutral.cpp:93-108: geostrophic forcing, dycore, sponge,
    surface fluxes, LES closure, time averager) or the urban one
    (city.cpp:137-142: edge sponge, dycore, sponge, surface fluxes, LES
    closure, time averager).  CUDA-event time of `steps` calls after one."""
    import torch
    from . import (Dynamics_Euler_Stratified_WenoFV, EdgeSponge, LES_Closure, Time_Averager, apply_surface_fluxes,
                   assign_coupler_state, case_coupler, geostrophic_wind_forcing, sponge_layer)
    from .physics import register_immersed_halos
    c = case_coupler(case, device="cuda:%d" % torch.cuda.current_device())
    register_immersed_halos(c, case)
    les, dyn, tavg, edge = LES_Closure(), Dynamics_Euler_Stratified_WenoFV(precision=a.precision), Time_Averager(), \
        EdgeSponge()
    les.init(c)
    dyn.init(c)
    tavg.init(c)
    urban = a.case == "urban_canopy"
    if urban:
        edge.set_column(c)
    assign_coupler_state(c, case, perturbed=True)
    dt = 10 * dyn.compute_time_step(c)
    sub = []

    def call():
        if urban:
            edge.apply(c, 0.01, 0.01, 0.01, 0.01)
        else:
            geostrophic_wind_forcing(c, dt, 43.289340204, 10.0, 0.0)
        sub.append(dyn.time_step(c, dt))
        sponge_layer(c, dt, dt if urban else dt * 100, 0.02 if urban else 0.1)
        apply_surface_fluxes(c, dt)
        les.apply(c, dt)
        tavg.accumulate(c, dt)
        c.set_option("elapsed_time", c.get_option("elapsed_time") + dt)

    call()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.steps):
        call()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.steps
    return {"case": a.case, "grid": [a.nx, a.ny, a.nz], "driver": "urban (city.cpp)" if urban else
            "boundary layer (abl_neutral.cpp)", "calls": a.steps, "dycore_steps_per_call": sub[-1], "ms_per_call": ms,
            "cell_steps_per_s": case.ncells * sub[-1] / (ms / 1e3),
            "note": "cell-steps/s of the whole driver step: the dycore's 10 steps and the modules beside it"}


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
    ap.add_argument("--driver", action="store_true",
                    help="run the reference driver's module chain per dt_phys (boundary layer or urban) on device "
                         "coupler arrays")
    ap.add_argument("--modules", action="store_true",
                    help="time the physics modules (LES closure, sponge, geostrophic forcing, surface fluxes) "
                         "on the case's coupler arrays instead of dycore steps")
    a = ap.parse_args(argv)

    case = CASES[a.case](a)
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
        out["training"] = g.learned_train(a.train_steps, batch=16384, lr=2e-3, seed=3)
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
