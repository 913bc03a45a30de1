"""TMA staging of the stage kernels' tiles gives the same bits as the
threads' own loads (pu_config.thread_loads = 1).

On domains without immersed cells the x/y kernel stages the cross of every
16x16 tile that lies whole in the domain in five boxes (interior, 5 rows
above and below, 5 columns left and right in 8-wide boxes), each wrapping
periodically on its own; tiles at a precursor edge, partial tiles and halo
boxes that would straddle the domain's edge keep the thread loads, as does
the immersed x/y kernel.

The tiled z kernel copies its raw tile (levels k0-5 .. k0+36) and, where
the buffers fit beside four blocks per SM (up to three tracers), the cell
inputs of its finalisation with bulk tensor copies; wall halo levels come
from the replicated boundary row of the box, the wrapped levels of a
periodic z from the threads, columns beyond the domain read zero (their
results are discarded).  Cases: walls and periodic z, immersed cells, one to
four tracers (with and without the prefetched cell inputs), partial tiles in
x (nx = 20, 52), y (ny = 37) and z (nz = 40), precursor x and y (only the
inner tiles staged), and a grid whose nx breaks the TMA stride rule
(nx % 4 != 0: thread loads everywhere).
"""
import numpy as np
import pytest

from porturb_b200 import cases
from helpers import gpu_run

pytestmark = pytest.mark.gpu

CASES = {
    "abl_64x48x40": lambda: cases.abl_neutral(nx=64, ny=48, nz=40),
    "abl_80x37x40_partial_y": lambda: cases.abl_neutral(nx=80, ny=37, nz=40),
    "urban_64x48x48": lambda: cases.urban_canopy(nx=64, ny=48, nz=48, dx=2.0),
    "urban_52x40x48_partial_x": lambda: cases.urban_canopy(nx=52, ny=40, nz=48, dx=2.0),
    "mixed_periodic_z": lambda: cases.small_mixed(nx=20, ny=12, nz=40, bc_z="periodic"),
    "mixed_immersed_3tr": lambda: cases.small_mixed(nx=48, ny=32, nz=36, ntr=3),
    "mixed_4tr_precursor_xy": lambda: cases.small_mixed(nx=48, ny=48, nz=24, ntr=4, bc_x="precursor",
                                                        bc_y="precursor", immersed=False),
    "odd_nx_no_tma": lambda: cases.small_mixed(nx=18, ny=10, nz=20),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_tma_staging_equals_thread_loads(name, gpu_lib):
    case = CASES[name]()
    runs = []
    for thread_loads in (False, True):
        st, tr, g = gpu_run(case, "f32", 0, 1.0, thread_loads=thread_loads)
        dt = g.compute_time_step()
        g.advance(dt, 3)
        g.synchronize()
        st, tr = g.get_conserved()
        rd, u, v, w, T, trc = [np.ascontiguousarray(np.array(a)) for a in case.coupler_arrays(perturbed=True)]
        trs = [np.ascontiguousarray(x) for x in trc]
        n = g.time_step(rd, u, v, w, T, trs, 2.5 * dt)
        g.close()
        assert n == 3
        runs.append((st, tr, [rd, u, v, w, T] + trs))
    (a_st, a_tr, a_cpl), (b_st, b_tr, b_cpl) = runs
    assert np.array_equal(a_st, b_st), np.abs(a_st - b_st).max()
    assert np.array_equal(a_tr, b_tr)
    for x, y in zip(a_cpl, b_cpl):
        assert np.array_equal(x, y)


SPLIT_CASES = {
    # buildings up to 30 levels, flags reach ~40 of 96 levels: both kernels split
    "urban_64x48x96": lambda: cases.urban_canopy(nx=64, ny=48, nz=96, dx=2.0),
    # cuboid to level 16, flags to ~26 of 48; precursor x keeps the edge tiles on thread loads
    "mixed_48x32x48_precursor": lambda: cases.small_mixed(nx=48, ny=32, nz=48, bc_x="precursor"),
    # periodic z: the x/y kernel splits, the z kernel stays immersed in every chunk
    "mixed_32x32x48_periodic_z": lambda: cases.small_mixed(nx=32, ny=32, nz=48, bc_z="periodic"),
    # flags reach the top: no split
    "mixed_32x32x20": lambda: cases.small_mixed(nx=32, ny=32, nz=20),
}


@pytest.mark.parametrize("thread_loads", [False, True])
@pytest.mark.parametrize("name", sorted(SPLIT_CASES))
def test_immersed_kernels_only_where_flags_reach(name, thread_loads, gpu_lib):
    """On an immersed domain the stage kernels take the immersed code on the
    levels (z chunks) an immersed flag reaches and the plain code above; the
    same bits as the immersed code on every level (imm_all_levels = 1)."""
    case = SPLIT_CASES[name]()
    runs = []
    for all_levels in (False, True):
        st, tr, g = gpu_run(case, "f32", 0, 1.0, thread_loads=thread_loads, imm_all_levels=all_levels)
        dt = g.compute_time_step()
        n0 = g.kernel_launches()
        g.advance(dt, 3)
        g.synchronize()
        launches = g.kernel_launches() - n0
        st, tr = g.get_conserved()
        rd, u, v, w, T, trc = [np.ascontiguousarray(np.array(a)) for a in case.coupler_arrays(perturbed=True)]
        trs = [np.ascontiguousarray(x) for x in trc]
        assert g.time_step(rd, u, v, w, T, trs, 2.5 * dt) == 3
        g.close()
        runs.append((st, tr, [rd, u, v, w, T] + trs, launches))
    (a_st, a_tr, a_cpl, a_n), (b_st, b_tr, b_cpl, b_n) = runs
    print(name, "launches in 3 steps: split", a_n, "all levels", b_n)
    if name != "mixed_32x32x20":
        assert a_n > b_n          # the split ran extra launches
    assert np.array_equal(a_st, b_st), np.abs(a_st - b_st).max()
    assert np.array_equal(a_tr, b_tr)
    for x, y in zip(a_cpl, b_cpl):
        assert np.array_equal(x, y)
