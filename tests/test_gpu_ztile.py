"""The tiled z kernel (k_zt: 8 columns x 32 levels per block, the default
for FP32 with weno_all) gives the bits of the z march (k_z, selected by an
explicit z chunk): the same primitive fields, wall and periodic halos,
immersed and wall-adjacent stencil modifications, face states, limiter bits
per stencil, Riemann fluxes, stage combination, immersed relaxation and
positivity clip.  Cases: walls with and without an immersed cuboid,
periodic z, three tracers (an odd number of fields), precursor x/y,
Coriolis, a 2-D domain, the warm bubble, and grids whose x and z extents
are not multiples of the tile (partial tiles, several z tiles)."""
import numpy as np
import pytest

from porturb_b200 import cases
from helpers import gpu_run

pytestmark = pytest.mark.gpu

CASES = {
    "walls": lambda: cases.small_mixed(immersed=False),
    "walls_immersed": lambda: cases.small_mixed(),
    "periodic_z_immersed": lambda: cases.small_mixed(bc_z="periodic", nz=40),
    "partial_tiles_immersed": lambda: cases.small_mixed(nx=37, ny=6, nz=75),
    "periodic_z": lambda: cases.small_mixed(bc_z="periodic", immersed=False),
    "periodic_z_tall": lambda: cases.small_mixed(bc_z="periodic", nz=70, immersed=False),
    "three_tracers": lambda: cases.small_mixed(ntr=3, immersed=False),
    "precursor_xy": lambda: cases.small_mixed(bc_x="precursor", bc_y="precursor", immersed=False),
    "coriolis": lambda: cases.small_mixed(latitude=43.29, immersed=False),
    "sim2d": lambda: cases.small_mixed(ny=1, nx=24, nz=16, immersed=False),
    "partial_tiles": lambda: cases.small_mixed(nx=37, ny=6, nz=75, immersed=False),
    "bubble_small": lambda: cases.warm_bubble(nx=64, ny=4, nz=32, xlen=5000.0, ylen=312.5, zlen=2500.0,
                                              radius=500.0, x0=2500.0, z0=600.0),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_tiled_z_kernel_gives_the_march_bits(name, gpu_lib):
    case = CASES[name]()
    _, _, g = gpu_run(case, "f32", 0, 0.0)
    dt = 0.9 * g.compute_time_step()
    st_t, tr_t, _ = gpu_run(case, "f32", 4, dt)
    st_m, tr_m, _ = gpu_run(case, "f32", 4, dt, z_chunk=16)
    st0, _, _ = gpu_run(case, "f32", 0, dt)
    assert not np.array_equal(st_t, st0)
    assert np.array_equal(st_t, st_m), np.abs(st_t - st_m).max()
    assert np.array_equal(tr_t, tr_m), np.abs(tr_t - tr_m).max()
