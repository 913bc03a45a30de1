"""Decomposed tiles (include/pu_dycore.h, coupler.h:132-229 and the halo and
edge exchanges of coupler.h:985-1165, dynamics_rk.h:808-912).

A decomposed run computes every cell from the same inputs as the
undecomposed run -- the halo slabs carry exactly the neighbours' values,
precursor conditions apply at the global edges only, and the immersed flags
come from a 12-cell halo of the proportion -- so once both runs share the
same hydrostatic profiles the states agree bit for bit.  (The profiles
themselves are summed over the tiles in a different order; they agree to a
few ulp.)  Covered here on one GPU: in-process groups of 3x2 tiles of unequal
sizes with an immersed cuboid across tile edges and a partially immersed
cell, 2x2 tiles with precursor x/y boundaries, a 2-D grid in 4x1 tiles, a
single tile exchanging with itself, FP32 and FP64 builds; and the NCCL path
with one rank (communicator, all-gather of the tile table, all-reduce of the
profile sums, send/receive to itself), in a child process with a time limit.
Several GPUs are not available here: more ranks over NCCL are covered by the
CPU test of the exchange schedule (tests/test_decomp_host.py)."""
import os
import subprocess
import sys

import numpy as np
import pytest

from porturb_b200 import Dycore, cases, decomp
from porturb_b200.capi import PortUrbError, PU_ERR_INVALID, PU_ERR_STATE

pytestmark = pytest.mark.gpu
NSTEPS = 3
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _case(kind):
    if kind == "sim2d":
        return cases.small_mixed(nx=60, ny=1, nz=16, immersed=False)
    nx, ny = (50, 36) if kind == "immersed_3x2" else (40, 32)
    c = cases.small_mixed(nx=nx, ny=ny, nz=16, immersed=False,
                          bc_x="precursor" if kind == "precursor_2x2" else "periodic",
                          bc_y="precursor" if kind == "precursor_2x2" else "periodic")
    if kind == "immersed_3x2":
        m = np.zeros((c.nz, c.ny, c.nx))
        m[:6, 14:22, 12:21] = 1.0       # crosses the tile edges at x = 17 and y = 18
        m[8, 17, 33] = 0.5              # a partially immersed cell next to the edge at x = 33
        m[:3, 30:36, 45:50] = 1.0       # touches the global x and y edges (periodic wrap)
        c.immersed_proportion[...] = m
    return c


GRIDS = {"immersed_3x2": (3, 2), "precursor_2x2": (2, 2), "single_1x1": (1, 1), "sim2d": (4, 1)}


def _whole(case, precision, dt):
    g = Dycore.from_case(case, precision=precision)
    rd, u, v, w, T, trc = [np.ascontiguousarray(a) for a in case.coupler_arrays(perturbed=False)]
    prop = np.ascontiguousarray(case.immersed_proportion)
    g.init(rd, u, v, w, T, list(trc), prop if prop.any() else None)
    cells, _ = g.get_hydrostasis()
    rd, u, v, w, T, trc = [np.ascontiguousarray(a) for a in case.coupler_arrays(perturbed=True)]
    g.load_state(rd, u, v, w, T, list(trc))
    st0, _ = g.get_conserved()
    g.advance(dt, NSTEPS)
    st, tr = g.get_conserved()
    g.close()
    return st, tr, cells, st0


def _load_tiles(grp, cells=None):
    if cells is not None:
        for h in grp.handles:
            h.set_hydrostasis(*cells)
    for h, c in zip(grp.handles, grp.cases):
        rd, u, v, w, T, trc = [np.ascontiguousarray(a) for a in c.coupler_arrays(perturbed=True)]
        h.load_state(rd, u, v, w, T, [np.ascontiguousarray(x) for x in trc])


@pytest.mark.parametrize("precision", ["f32", "f64"])
@pytest.mark.parametrize("kind", sorted(GRIDS))
def test_group_equals_undecomposed(gpu_lib, kind, precision):
    case = _case(kind)
    g = Dycore.from_case(case, precision=precision)
    dt = g.compute_time_step()
    g.close()
    st, tr, cells, st0 = _whole(case, precision, dt)
    grp = decomp.TileGroup(case, *GRIDS[kind], precision=precision)
    grp.init_case(perturbed=False)
    # The group's own profiles: sums over the tiles in another order.
    for h in grp.handles:
        c, _ = h.get_hydrostasis()
        for q in range(3):
            assert np.allclose(c[q], cells[q], rtol=4e-16 if precision == "f64" else 1.2e-7, atol=0), q
    _load_tiles(grp, cells)
    grp.advance(dt, NSTEPS)
    st_g, tr_g = grp.get_conserved()
    grp.close()
    assert np.array_equal(st_g, st), np.abs(st_g - st).max()
    assert np.array_equal(tr_g, tr)
    assert not np.array_equal(st, st0)


def test_group_time_step_on_coupler_arrays(gpu_lib):
    """pu_dycore_group_time_step: convert, sub-cycle and convert back per tile
    equals the undecomposed time_step."""
    case = _case("immersed_3x2")
    g = Dycore.from_case(case, precision="f32")
    rd, u, v, w, T, trc = [np.ascontiguousarray(a) for a in case.coupler_arrays(perturbed=False)]
    g.init(rd, u, v, w, T, list(trc), np.ascontiguousarray(case.immersed_proportion))
    cells, _ = g.get_hydrostasis()
    dt = 2.5 * g.compute_time_step()
    whole = [np.ascontiguousarray(a).copy() for a in case.coupler_arrays(perturbed=True)[:5]]
    wtr = [np.ascontiguousarray(t).copy() for t in case.tracer_data]
    n = g.time_step(*whole, wtr, dt)
    g.close()
    grp = decomp.TileGroup(case, 3, 2)
    grp.init_case(perturbed=False)
    for h in grp.handles:
        h.set_hydrostasis(*cells)
    arrays = []
    for c in grp.cases:
        rd, u, v, w, T, trc = [np.ascontiguousarray(a).copy() for a in c.coupler_arrays(perturbed=True)]
        arrays.append((rd, u, v, w, T, [np.ascontiguousarray(x).copy() for x in trc]))
    assert grp.time_step(arrays, dt) == n == 3
    for f in range(5):
        got = decomp.assemble([a[f] for a in arrays], grp.tiles, case.nx, case.ny)
        assert np.array_equal(got, whole[f]), f
    got = decomp.assemble([np.stack(a[5]) for a in arrays], grp.tiles, case.nx, case.ny)
    assert np.array_equal(got, np.stack(wtr))
    grp.close()


_NCCL_CHILD = r"""
import sys
sys.path[:0] = [%r]
import numpy as np
from porturb_b200 import Dycore, cases, decomp
launches = {}
for nx, ny, serial in ((40, 32, False), (64, 64, False), (64, 64, True)):
    case = cases.small_mixed(nx=nx, ny=ny, nz=16, immersed=True)
    g = Dycore.from_case(case)
    dt = g.compute_time_step()
    rd, u, v, w, T, trc = [np.ascontiguousarray(a) for a in case.coupler_arrays(perturbed=False)]
    prop = np.ascontiguousarray(case.immersed_proportion)
    g.init(rd, u, v, w, T, list(trc), prop)
    cells, _ = g.get_hydrostasis()
    h = Dycore.from_case(case, serial_io=serial)
    t = decomp.tiles(case.nx, case.ny, 1, 1)[0]
    decomp.set_decomposition(h, t, case.nx, case.ny, nccl_id=decomp.nccl_unique_id())
    h.init(rd, u, v, w, T, list(trc), prop)
    c2, _ = h.get_hydrostasis()
    assert all(np.allclose(c2[q], cells[q], rtol=1.2e-7, atol=0) for q in range(3))
    h.set_hydrostasis(*cells)
    for d in (g, h):
        rd, u, v, w, T, trc = [np.ascontiguousarray(a) for a in case.coupler_arrays(perturbed=True)]
        d.load_state(rd, u, v, w, T, list(trc))
        l0 = d.kernel_launches()
        d.advance(dt, 3)
        launches[(nx, serial, d is h)] = d.kernel_launches() - l0
    a, b = g.get_conserved(), h.get_conserved()
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), (nx, ny, serial)
    g.close()
    h.close()
# 64x64: the interior tiles ran while the halos crossed (more launches than
# the whole-tile form); 40x32 has no interior tile.
assert launches[(64, False, True)] > launches[(64, True, True)], launches
print("nccl one-rank decomposition ok", launches)
"""


def test_nccl_single_rank_equals_undecomposed(gpu_lib):
    env = dict(os.environ, NCCL_NVLS_ENABLE="0")
    r = subprocess.run([sys.executable, "-c", _NCCL_CHILD % ROOT], capture_output=True, text=True, timeout=180,
                       env=env)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "nccl one-rank decomposition ok" in r.stdout


def test_decomposition_errors(gpu_lib):
    case = _case("precursor_2x2")
    small = cases.small_mixed(nx=10, ny=16, nz=8, immersed=False)
    h = Dycore.from_case(small)
    with pytest.raises(PortUrbError) as e:
        decomp.set_decomposition(h, decomp.Tile(2, 1, 0, 0, 0, 0, 10, 16), 20, 16)
    assert e.value.status == PU_ERR_INVALID
    h.close()
    grp = decomp.TileGroup(case, 2, 2)
    # A group without every tile of the grid.
    import ctypes as C
    hs = (C.c_void_p * 3)(*[x.h for x in grp.handles[:3]])
    assert grp.lib.pu_dycore_group_advance(hs, 3, 0.1, 1) == PU_ERR_STATE   # not initialised yet
    grp.init_case()
    assert grp.lib.pu_dycore_group_advance(hs, 3, 0.1, 1) == PU_ERR_INVALID
    # A group tile cannot advance alone, nor take learned weights.
    with pytest.raises(PortUrbError) as e:
        grp.handles[0].advance(0.1, 1)
    assert e.value.status == PU_ERR_STATE
    assert grp.lib.pu_dycore_set_weno_mode(grp.handles[0].h, 1) != 0
    grp.close()
