"""pu_dycore_time_step on host coupler arrays with the copies overlapped
(pu_config.serial_io = 0) gives the same bits as copies in, steps, copies
out (serial_io = 1).

The overlapped call runs as a wavefront over chunks of 32 levels: the input
crosses chunk by chunk on a copy stream, and stage g runs on chunk c once
stage g-1 has run on chunks c-1, c and c+1 (launches in diagonals g + c),
each chunk's final state converted back and copied out while the others
finish.  Cases: a plain boundary layer (3 chunks), the urban canopy whose
immersed levels end inside the second chunk (the immersed/plain split falls
inside a chunk's range), a last chunk of 16 levels (nz = 80), three tracers
with immersed cells; each with 1, 2 and 3 SSPRK3 cycles per call, from
pageable numpy arrays and from pinned torch tensors; and the urban canopy at
its configuration's size (512x512x128).  The overlapped call
must launch more kernels than the serial one (the chunked stages: the path
was taken), and a periodic z or nz < 64 must launch the same number (the
path is not taken).  The launch order itself is checked on the CPU against
the serial order in tests/test_io_wavefront_order.py.
"""
import numpy as np
import pytest

from porturb_b200 import Dycore, cases

pytestmark = pytest.mark.gpu

CASES = {
    "abl_64x48x96": lambda: cases.abl_neutral(nx=64, ny=48, nz=96),
    "urban_64x48x96_split_in_chunk": lambda: cases.urban_canopy(nx=64, ny=48, nz=96, dx=2.0),
    "abl_48x32x80_partial_chunk": lambda: cases.abl_neutral(nx=48, ny=32, nz=80),
    "mixed_48x32x64_3tr": lambda: cases.small_mixed(nx=48, ny=32, nz=64, ntr=3),
}


def _arrays(case, perturbed, pinned):
    rd, u, v, w, T, trc = case.coupler_arrays(perturbed=perturbed)
    arrs = [np.ascontiguousarray(np.array(a, dtype=np.float64)) for a in (rd, u, v, w, T)]
    trs = [np.ascontiguousarray(np.array(t, dtype=np.float64)) for t in trc]
    if not pinned:
        return arrs, trs
    import torch
    pin = lambda a: torch.from_numpy(a).pin_memory()
    return [pin(a) for a in arrs], [pin(t) for t in trs]


def _call(case, serial_io, factor, pinned):
    g = Dycore.from_case(case, precision="f32", device=0, serial_io=serial_io)
    base, btr = _arrays(case, False, False)
    imm = np.ascontiguousarray(case.immersed_proportion)
    g.init(*base, btr, imm if imm.any() else None)
    dt = g.compute_time_step()
    arrs, trs = _arrays(case, True, pinned)
    l0 = g.kernel_launches()
    n = g.time_step(*arrs, trs, factor * dt)
    launches = g.kernel_launches() - l0
    st, tr = g.get_conserved()
    g.close()
    out = [np.asarray(a) for a in arrs] + [np.asarray(t) for t in trs]
    return n, launches, out, st, tr


@pytest.mark.parametrize("pinned", [False, True], ids=["pageable", "pinned"])
@pytest.mark.parametrize("factor", [1.0, 2.0, 2.5])
@pytest.mark.parametrize("name", sorted(CASES))
def test_overlapped_time_step_same_bits(name, factor, pinned, gpu_lib):
    case = CASES[name]()
    n1, l1, out1, st1, tr1 = _call(case, True, factor, pinned)
    n0, l0, out0, st0, tr0 = _call(case, False, factor, pinned)
    assert n0 == n1 == int(np.ceil(factor))
    assert l0 > l1, (l0, l1)
    for q, (a, b) in enumerate(zip(out0, out1)):
        assert np.array_equal(a, b), (name, q, np.abs(a - b).max())
    assert np.array_equal(st0, st1) and np.array_equal(tr0, tr1)


def test_overlapped_time_step_same_bits_at_config_size(gpu_lib):
    """The urban canopy at the size of its configuration (512x512x128, 2 m:
    33.5 M cells, 4 chunks, the immersed levels ending inside chunk 1), 3
    cycles per call from pinned arrays: the same bits both ways."""
    case = cases.urban_canopy(nx=512, ny=512, nz=128, dx=2.0)
    n1, l1, out1, st1, tr1 = _call(case, True, 2.5, True)
    n0, l0, out0, st0, tr0 = _call(case, False, 2.5, True)
    assert n0 == n1 == 3 and l0 > l1
    for q, (a, b) in enumerate(zip(out0, out1)):
        assert np.array_equal(a, b), (q, np.abs(a - b).max())
    assert np.array_equal(st0, st1) and np.array_equal(tr0, tr1)


@pytest.mark.parametrize("name,make", [
    ("periodic_z", lambda: cases.small_mixed(nx=32, ny=32, nz=64, bc_z="periodic")),
    ("nz_48", lambda: cases.abl_neutral(nx=32, ny=32, nz=48)),
])
def test_serial_where_overlap_does_not_apply(name, make, gpu_lib):
    case = make()
    n1, l1, out1, _, _ = _call(case, True, 2.5, False)
    n0, l0, out0, _, _ = _call(case, False, 2.5, False)
    assert l0 == l1, (name, l0, l1)
    for a, b in zip(out0, out1):
        assert np.array_equal(a, b)
