"""Shared helpers of the parity tests: run the same case through the CPU
oracle and through libpu_dycore on identical inputs and compare."""
import numpy as np

import pyoracle
from porturb_b200 import Dycore


def oracle_run(case, kind, nsteps, dt, hydro=None):
    """Init from the base state, optionally overwrite the cell profiles, load
    the perturbed state, advance, return (state, tracers, hydro)."""
    d = pyoracle.Dycore(case, kind)
    d.init_case()
    if hydro is not None:
        d.set_hydrostasis(*hydro)
    cells, _ = d.get_hydrostasis()
    d.load_coupler(list(case.coupler_arrays(perturbed=True)))
    st0, tr0 = d.get_state()
    if nsteps:
        d.advance(dt, nsteps)
    st, tr = d.get_state()
    return st, tr, cells, (st0, tr0)


def gpu_run(case, precision, nsteps, dt, hydro=None, **kw):
    g = Dycore.from_case(case, precision=precision, **kw)
    rd, u, v, w, T, trc = [np.ascontiguousarray(a) for a in case.coupler_arrays(perturbed=False)]
    imm = np.ascontiguousarray(case.immersed_proportion)
    g.init(rd, u, v, w, T, list(trc), imm if imm.any() else None)
    if hydro is not None:
        g.set_hydrostasis(*hydro)
    rd, u, v, w, T, trc = [np.ascontiguousarray(a) for a in case.coupler_arrays(perturbed=True)]
    g.load_state(rd, u, v, w, T, list(trc))
    if nsteps:
        g.advance(dt, nsteps)
    g.synchronize()
    st, tr = g.get_conserved()
    return st, tr, g


def rel_change_err(a, b, base):
    """||a-b|| / ||b-base|| per field (L2 and Linf), the error measured
    against the change the run produced."""
    out = []
    for f in range(a.shape[0]):
        d = a[f] - b[f]
        ch = b[f] - base[f]
        den2 = np.sqrt(np.mean(ch ** 2)) + 1e-300
        deni = np.abs(ch).max() + 1e-300
        out.append((np.sqrt(np.mean(d ** 2)) / den2, np.abs(d).max() / deni))
    return out


def background(case, cells, ntr):
    """Hydrostatic background of the conserved variables: (rho_h, 0, 0, 0,
    rho_h*theta_h) per level and zero tracers, on the (nz,ny,nx) grid."""
    hs = 4
    nz, ny, nx = case.nz, case.ny, case.nx
    r = np.asarray(cells[0][hs:hs + nz])
    t = np.asarray(cells[1][hs:hs + nz])
    bg = np.zeros((5 + ntr, nz, ny, nx))
    bg[0] = r[:, None, None]
    bg[4] = (r * t)[:, None, None]
    return bg


def rel_pert_err(a, b, bg):
    """||a-b|| / ||b-bg|| per field (L2 and Linf): the error measured against
    the departure from the hydrostatic background."""
    out = []
    for f in range(a.shape[0]):
        d = a[f] - b[f]
        p = b[f] - bg[f]
        out.append((np.sqrt(np.mean(d ** 2)) / (np.sqrt(np.mean(p ** 2)) + 1e-300),
                    np.abs(d).max() / (np.abs(p).max() + 1e-300)))
    return out
