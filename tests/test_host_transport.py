"""The host transport of decomposed tiles (pu_host_transport, driven by
porturb_b200.decomp.TorchHostTransport) on gloo ranks, on CPU.

Each rank calls the transport's C function pointers the way the library
does (through the ctypes struct it hands to pu_dycore_set_decomposition_host):
exchange with the four 5-cell slabs next to its tile's edges, then
allreduce_sum_f64 and allgather.  Every rank's received slabs must be the
periodic neighbours of its tile in the global array (coupler.h:985-1165),
for grids where both neighbours along a direction are one rank (2 tiles), the
rank itself (1 tile), or two different ranks (3 tiles); the sum and the
gather must be the same on every rank.
"""
import ctypes as C
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from porturb_b200 import capi, decomp

W = 5


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, nxg, nyg, nz, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        tr = decomp.TorchHostTransport()
        npx, npy = decomp.process_grid(world, nxg, nyg)
        t = decomp.tiles(nxg, nyg, npx, npy)[rank]
        nbr = decomp.neighbors(npx, npy, t.px, t.py)
        G = np.arange(nz * nyg * nxg, dtype=np.float32).reshape(nz, nyg, nxg)
        tile = np.ascontiguousarray(G[:, t.j_beg:t.j_beg + t.ny, t.i_beg:t.i_beg + t.nx])
        snd = [np.ascontiguousarray(tile[:, :, :W]), np.ascontiguousarray(tile[:, :, -W:]),
               np.ascontiguousarray(tile[:, :W, :]), np.ascontiguousarray(tile[:, -W:, :])]
        rcv = [np.zeros_like(a) for a in snd]
        S = (C.c_void_p * 4)(*[a.ctypes.data for a in snd])
        R = (C.c_void_p * 4)(*[a.ctypes.data for a in rcv])
        B = (C.c_size_t * 4)(*[a.nbytes for a in snd])
        N = (C.c_int * 4)(*nbr)
        st = tr.struct
        assert st.exchange(None, S, R, B, N) == 0, tr.error
        ii = np.arange(t.i_beg, t.i_beg + t.nx)
        jj = np.arange(t.j_beg, t.j_beg + t.ny)
        want = [G[:, jj][:, :, (t.i_beg - W + np.arange(W)) % nxg],
                G[:, jj][:, :, (t.i_beg + t.nx + np.arange(W)) % nxg],
                G[:, (t.j_beg - W + np.arange(W)) % nyg][:, :, ii],
                G[:, (t.j_beg + t.ny + np.arange(W)) % nyg][:, :, ii]]
        ok = [bool(np.array_equal(r, w)) for r, w in zip(rcv, want)]
        # x only (the init's x exchange): the y slabs are not touched.
        rcv2 = [np.full_like(a, -1) for a in snd]
        R2 = (C.c_void_p * 4)(*[a.ctypes.data for a in rcv2])
        B2 = (C.c_size_t * 4)(snd[0].nbytes, snd[1].nbytes, 0, 0)
        assert st.exchange(None, S, R2, B2, N) == 0, tr.error
        ok.append(bool(np.array_equal(rcv2[0], want[0]) and np.array_equal(rcv2[1], want[1])
                       and (rcv2[2] == -1).all() and (rcv2[3] == -1).all()))
        buf = np.arange(7, dtype=np.float64) * (rank + 1) + 0.25
        assert st.allreduce_sum_f64(None, buf.ctypes.data_as(C.POINTER(C.c_double)), buf.size) == 0, tr.error
        mine = np.array([rank, t.nx, t.ny, 17], np.int32)
        allg = np.zeros(4 * world, np.int32)
        assert st.allgather(None, mine.ctypes.data, allg.ctypes.data, mine.nbytes) == 0, tr.error
        out[rank] = (ok, buf.tolist(), allg.tolist(), tr.calls)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,nxg,nyg", [(2, 40, 24), (2, 24, 40), (3, 48, 20), (4, 40, 36)])
def test_host_transport_exchange_reduce_gather(world, nxg, nyg):
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(world, _free_port(), nxg, nyg, 3, out), nprocs=world, join=True,
                           start_method="spawn")
        res = dict(out)
    assert sorted(res) == list(range(world))
    npx, npy = decomp.process_grid(world, nxg, nyg)
    want_sum = sum(np.arange(7, dtype=np.float64) * (r + 1) + 0.25 for r in range(world)).tolist()
    for r in range(world):
        ok, s, g, calls = res[r]
        assert all(ok), (world, npx, npy, r, ok)
        assert s == want_sum
        t = decomp.tiles(nxg, nyg, npx, npy)
        assert g == sum(([q, t[q].nx, t[q].ny, 17] for q in range(world)), [])
        assert calls == {"exchange": 2, "allreduce_sum_f64": 1, "allgather": 1}


def test_transport_callback_errors_are_reported_not_raised():
    """A callback that raises returns 1 (the library's PU_ERR_TRANSPORT) and
    keeps the exception."""
    class Broken(decomp.TorchHostTransport):
        def __init__(self):
            self.error = None
            self.calls = {"exchange": 0, "allreduce_sum_f64": 0, "allgather": 0}
            self.dist = None          # every use raises
            self.group = None
            self.rank, self.world = 0, 1
            self._fns = (capi.EXCHANGE_FN(self._exchange), capi.ALLREDUCE_FN(self._allreduce),
                         capi.ALLGATHER_FN(self._allgather))
            self.struct = capi.pu_host_transport(self._fns[0], self._fns[1], self._fns[2], None)
    b = Broken()
    buf = np.zeros(4)
    assert b.struct.allreduce_sum_f64(None, buf.ctypes.data_as(C.POINTER(C.c_double)), 4) == 1
    assert isinstance(b.error, AttributeError)
