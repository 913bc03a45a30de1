"""The decomposed dycore on two ranks that talk through the host transport.

Two processes on the one GPU each own a tile of a global case and drive the
library's own decomposed path: pu_dycore_set_decomposition_host (the tile
table checked through allgather), the decomposed init (column sums summed
over the ranks through allreduce_sum_f64 into the tiles' profiles, the
immersed proportion's 12-cell halo gathered through two exchanges, flags and
relaxation factors on the extended block), 3 SSPRK3 steps with a halo
exchange per stage, and a time_step call (conversion in, 3 cycles, conversion
out).  The halo slabs go device -> pinned host -> gloo -> pinned host ->
device, as the reference's coupler moves them through MPI
(coupler.h:985-1165, dynamics_rk.h:976-978).  No kernel waits on another
rank: every wait is on the host.

Checks: the tiles' own profiles agree with the undecomposed run's (FP64
build to 1e-14 relative, FP32 build within one float ulp); with the same
profiles set on both, the assembled state after 3 steps and the coupler
arrays after time_step equal the undecomposed run bit for bit, FP32 and
FP64, for a grid split in x and one split in y, with an immersed cuboid
that reaches the tile edge (x split) or crosses it (y split).
"""
import os
import socket

import numpy as np
import pytest

from porturb_b200 import Dycore, cases, decomp

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(600)]

CASES = {
    "x_split": lambda: cases.small_mixed(nx=40, ny=24, nz=16),
    "y_split": lambda: cases.small_mixed(nx=24, ny=40, nz=16),
    # tiles of 64x64 and 64x56: interior 16x16 tiles run while the halos cross
    "x_split_interior": lambda: cases.small_mixed(nx=128, ny=64, nz=16),
    "y_split_interior": lambda: cases.small_mixed(nx=64, ny=112, nz=16),
}
NSTEPS = 3


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _arrays(case, perturbed):
    rd, u, v, w, T, trc = case.coupler_arrays(perturbed=perturbed)
    return [np.ascontiguousarray(np.array(a, dtype=np.float64)) for a in (rd, u, v, w, T)], \
           [np.ascontiguousarray(np.array(t, dtype=np.float64)) for t in trc]


def _rank(rank, world, port, name, precision, tmp):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        case = CASES[name]()
        h, t, tc, tr = decomp.host_transport_tile(case, precision=precision, device=0)
        st, trc = _arrays(tc, False)
        prop = np.ascontiguousarray(tc.immersed_proportion)
        h.init(*st, trc, prop if case.immersed_proportion.any() else None)
        own = h.get_hydrostasis()[0]
        ref = np.load(os.path.join(tmp, "cells.npy"))
        h.set_hydrostasis(*ref)
        st, trc = _arrays(tc, True)
        h.load_state(*st, trc)
        dt = h.compute_time_step()
        h.advance(dt, NSTEPS)
        cons, ctr = h.get_conserved()
        st, trc = _arrays(tc, True)
        n = h.time_step(*st, trc, 2.5 * dt)
        np.savez(os.path.join(tmp, "rank%d.npz" % rank), cons=cons, ctr=ctr, arrays=np.stack(st + trc),
                 own=np.stack(own), n=n, calls=np.array([tr.calls["exchange"], tr.calls["allreduce_sum_f64"],
                                                         tr.calls["allgather"]]))
        h.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("precision", ["f32", "f64"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_two_ranks_over_host_transport_equal_undecomposed(name, precision, tmp_path, gpu_lib):
    import torch.multiprocessing as mp
    case = CASES[name]()
    assert case.immersed_proportion.any()
    g = Dycore.from_case(case, precision=precision, device=0)
    st, trc = _arrays(case, False)
    g.init(*st, trc, np.ascontiguousarray(case.immersed_proportion))
    cells = g.get_hydrostasis()[0]
    np.save(tmp_path / "cells.npy", np.stack(cells))
    st, trc = _arrays(case, True)
    g.load_state(*st, trc)
    dt = g.compute_time_step()
    g.advance(dt, NSTEPS)
    cons_ref, ctr_ref = g.get_conserved()
    st, trc = _arrays(case, True)
    n_ref = g.time_step(*st, trc, 2.5 * dt)
    arr_ref = np.stack(st + trc)
    g.close()

    world = 2
    mp.start_processes(_rank, args=(world, _free_port(), name, precision, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    npx, npy = decomp.process_grid(world, case.nx, case.ny)
    assert (npx, npy) == ((2, 1) if name.startswith("x_split") else (1, 2))
    ts = decomp.tiles(case.nx, case.ny, npx, npy)
    res = [np.load(tmp_path / ("rank%d.npz" % r)) for r in range(world)]
    # The tiles' own profiles: sums over the two ranks against the whole grid's.
    for r in res:
        own, want = r["own"], np.stack(cells)
        if precision == "f64":
            assert np.abs(own - want).max() <= 1e-14 * np.abs(want).max()
        else:
            ulp = np.spacing(np.abs(want).astype(np.float32)).astype(np.float64)
            assert (np.abs(own - want) <= ulp).all()
        assert int(r["n"]) == n_ref == 3
        # exchanges: init x and y, then one per stage over 3 steps and 3 cycles
        assert r["calls"].tolist() == [2 + 3 * (NSTEPS + 3), 1, 1]
    cons = decomp.assemble([r["cons"] for r in res], ts, case.nx, case.ny)
    ctr = decomp.assemble([r["ctr"] for r in res], ts, case.nx, case.ny)
    arr = decomp.assemble([r["arrays"] for r in res], ts, case.nx, case.ny)
    assert np.array_equal(cons, cons_ref), np.abs(cons - cons_ref).max()
    assert np.array_equal(ctr, ctr_ref)
    assert np.array_equal(arr, arr_ref), np.abs(arr - arr_ref).max()


class _OneRank:
    """pu_host_transport callbacks for a grid of one tile (the rank is every
    neighbour of itself); `fail` names a callback that reports failure from
    its n-th call on."""

    def __init__(self, fail=None, after=0):
        import ctypes as C
        from porturb_b200 import capi
        self.C, self.fail, self.after = C, fail, after
        self.calls = {"exchange": 0, "allreduce_sum_f64": 0, "allgather": 0}
        self._fns = (capi.EXCHANGE_FN(self._ex), capi.ALLREDUCE_FN(self._ar), capi.ALLGATHER_FN(self._ag))
        self.struct = capi.pu_host_transport(self._fns[0], self._fns[1], self._fns[2], None)

    def _bad(self, name):
        self.calls[name] += 1
        return self.fail == name and self.calls[name] > self.after

    def _ex(self, user, snd, rcv, nbytes, nbr):
        if self._bad("exchange"):
            return 5
        for d in range(4):
            if nbytes[d]:
                assert nbr[d] == 0 and nbytes[d ^ 1] == nbytes[d]
                self.C.memmove(rcv[d], snd[d ^ 1], nbytes[d])
        return 0

    def _ar(self, user, buf, n):
        return 5 if self._bad("allreduce_sum_f64") else 0

    def _ag(self, user, src, out, nbytes):
        if self._bad("allgather"):
            return 5
        self.C.memmove(out, src, nbytes)
        return 0


def _one_tile(case, tr, precision="f32"):
    t = decomp.tiles(case.nx, case.ny, 1, 1)[0]
    h = Dycore.from_case(case, precision=precision, device=0)
    decomp.set_decomposition_host(h, t, case.nx, case.ny, tr)
    return h


def test_one_tile_over_host_transport_equals_undecomposed(gpu_lib):
    """One tile whose halos come back through the host transport from its own
    edges (periodic): the library's host exchange, summed profiles and
    immersed halo gather, bit for bit against the undecomposed run."""
    case = cases.small_mixed(nx=24, ny=16, nz=12)
    tr = _OneRank()
    h = _one_tile(case, tr)
    g = Dycore.from_case(case, precision="f32", device=0)
    prop = np.ascontiguousarray(case.immersed_proportion)
    outs = []
    for d in (h, g):
        st, trc = _arrays(case, False)
        d.init(*st, trc, prop)
        st, trc = _arrays(case, True)
        d.load_state(*st, trc)
        d.advance(d.compute_time_step(), 3)
        outs.append(d.get_conserved())
        d.close()
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
    assert tr.calls == {"exchange": 2 + 3 * 3, "allreduce_sum_f64": 1, "allgather": 1}


@pytest.mark.parametrize("where", ["allgather", "allreduce_sum_f64", "init_exchange", "step_exchange"])
def test_transport_failure_is_reported(where, gpu_lib):
    """A callback that returns non-zero makes the call that used it return
    PU_ERR_TRANSPORT: set-up (allgather; the handle stays undecomposed and can
    be decomposed again), init (the column sums, the immersed halo exchange)
    or a step (the halo exchange of a stage)."""
    from porturb_b200 import PortUrbError, capi
    case = cases.small_mixed(nx=24, ny=16, nz=12)
    name = {"init_exchange": "exchange", "step_exchange": "exchange"}.get(where, where)
    tr = _OneRank(fail=name, after=2 if where == "step_exchange" else 0)
    t = decomp.tiles(case.nx, case.ny, 1, 1)[0]
    h = Dycore.from_case(case, precision="f32", device=0)
    if where == "allgather":
        with pytest.raises(PortUrbError) as e:
            decomp.set_decomposition_host(h, t, case.nx, case.ny, tr)
        assert e.value.status == capi.PU_ERR_TRANSPORT
        decomp.set_decomposition_host(h, t, case.nx, case.ny, _OneRank())   # not left half decomposed
        h.close()
        return
    decomp.set_decomposition_host(h, t, case.nx, case.ny, tr)
    st, trc = _arrays(case, False)
    prop = np.ascontiguousarray(case.immersed_proportion)
    if where in ("allreduce_sum_f64", "init_exchange"):
        with pytest.raises(PortUrbError) as e:
            h.init(*st, trc, prop)
        assert e.value.status == capi.PU_ERR_TRANSPORT
        h.close()
        return
    h.init(*st, trc, prop)
    st, trc = _arrays(case, True)
    h.load_state(*st, trc)
    with pytest.raises(PortUrbError) as e:
        h.advance(h.compute_time_step(), 1)
    assert e.value.status == capi.PU_ERR_TRANSPORT
    assert b"exchange returned 5" in capi.load().pu_last_error()
    h.close()
