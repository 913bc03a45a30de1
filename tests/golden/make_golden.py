#!/usr/bin/env python3
"""Generate the golden fixtures of the parity tests from the reference's own
dycore code.

Runs oracle/_ref/libporturb_ref.so -- the reference's dynamics_rk.h,
WenoLimiter.h and TransformMatrices.h compiled unchanged against the
single-rank shim in oracle/ref_shim (build it with `make -C oracle ref`,
which needs the reference tree) -- and stores, per case:
  * the coupler-side inputs (base state, perturbed state, immersed proportion),
  * the hydrostatic profiles the reference's init computed,
  * the conserved state (rho, rho*u, rho*v, rho*w, rho*theta, tracers) after
    the stated number of SSPRK3 steps of the stated dt,
  * the limiter edges of a set of stencils (float and double instantiations).

Usage: python tests/golden/make_golden.py   (writes tests/golden/*.npz)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import pyoracle  # noqa: E402
from porturb_b200 import cases  # noqa: E402

CASES = {
    "small_mixed": (lambda: cases.small_mixed(), 3),
    "small_precursor": (lambda: cases.small_mixed(bc_x="precursor", bc_y="precursor", ntr=1, immersed=False), 3),
    "bubble_64x4x32": (lambda: cases.warm_bubble(nx=64, ny=4, nz=32, xlen=5000.0, ylen=312.5, zlen=2500.0,
                                                 radius=500.0, x0=2500.0, z0=600.0, cfl=0.8), 10),
}


def limiter_stencils(n=2000, seed=7):
    rng = np.random.default_rng(seed)
    s = rng.normal(size=(n, 9)) * 10.0 ** rng.uniform(-6, 3, size=(n, 1))
    s[::7] = s[::7, :1]                                   # constant stencils
    s[1::11] = np.cumsum(np.abs(s[1::11]), axis=1)        # monotone
    s[2::13, 4:] += 100.0 * np.abs(s[2::13, :1])          # jumps
    flags = np.stack([np.arange(n) % 2, (np.arange(n) % 3) == 0, (np.arange(n) % 5) == 0], axis=1).astype(np.int32)
    return s, flags


def main():
    pyoracle.build(ref=True)
    if not pyoracle.have_ref():
        raise SystemExit("the reference library was not built (is the reference tree mounted?)")
    for name, (fn, nsteps) in CASES.items():
        case = fn()
        d = pyoracle.Dycore(case, "reference")
        d.init_case()
        cells, edges = d.get_hydrostasis()
        d.load_coupler(list(case.coupler_arrays(perturbed=True)))
        dt = 0.9 * d.compute_time_step()
        d.advance(dt, nsteps)
        st, tr = d.get_state()
        rd, u, v, w, T, trc = case.coupler_arrays(perturbed=False)
        prd, pu_, pv, pw, pT, ptr = case.coupler_arrays(perturbed=True)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), nsteps=nsteps, dt=dt,
                            base=np.stack([rd, u, v, w, T]), base_tracers=trc,
                            pert=np.stack([prd, pu_, pv, pw, pT]), pert_tracers=ptr,
                            immersed=case.immersed_proportion,
                            hy_cells=np.stack(cells), hy_edges=np.stack(edges), state=st, tracers=tr)
        print(name, case.nx, case.ny, case.nz, nsteps, "steps")
    s, flags = limiter_stencils()
    q32 = np.zeros((len(s), 2), np.float32)
    q64 = np.zeros((len(s), 2))
    for m in range(len(s)):
        q32[m] = pyoracle.weno9(s[m], *flags[m], kind="reference_f32")
        q64[m] = pyoracle.weno9(s[m], *flags[m], kind="reference_f64")
    np.savez_compressed(os.path.join(HERE, "limiter.npz"), stencils=s, flags=flags, edges_f32=q32, edges_f64=q64)
    print("limiter", len(s), "stencils")


if __name__ == "__main__":
    main()
