"""Host logic of the decomposed dycore, on CPU.

* The process grid, tile ranges and neighbour ranks of libpu_dycore
  (pu_decomp_process_grid / pu_decomp_tile / pu_decomp_neighbors) against a
  transcription of the reference's coupler (coupler.h:148-214).
* The halo exchange schedule with several ranks: gloo ranks post their sends
  and receives in the order the library posts them to NCCL
  (ImplBase::nccl_exchange: per direction pair, send snd[lo] to the low
  neighbour, receive rcv[hi] from the high one, send snd[hi] to the high
  neighbour, receive rcv[lo] from the low one; x pair, then y pair) and every
  rank's received slabs must be the periodic neighbours of its tile in the
  global array -- for grids where both neighbours along a direction are one
  rank (2 tiles) or the rank itself (1 tile), and where they differ (3 tiles).
  gloo has no channel from a rank to itself, so those messages are matched
  in posting order by the test, as NCCL matches them (NCCL's own handling of
  them is run on the GPU with one rank, tests/test_gpu_decomp.py).
"""
import math
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from porturb_b200 import decomp


def _ref_process_grid(nranks, nx_glob, ny_glob):
    """coupler.h:148-171 as written (each candidate over nranks/best-so-far)."""
    if ny_glob == 1:
        return nranks, 1
    choices = [float(q) for q in range(1, nranks + 1) if nranks % q == 0]
    aspect_real = ny_glob / nx_glob
    npy = int(choices[0])
    aspect = npy / (nranks // npy)
    min_dist = abs(aspect - aspect_real)
    for c in choices[1:]:
        aspect = c / (nranks // npy)
        dist_ = abs(aspect - aspect_real)
        if dist_ < min_dist:
            npy = int(c)
            min_dist = dist_
    return nranks // npy, npy


def _round_half_away(x):
    return math.floor(x + 0.5) if x >= 0 else -math.floor(-x + 0.5)


def test_process_grid_tiles_and_neighbors_match_the_coupler():
    for nranks in (1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 64):
        for nxg, nyg in ((256, 256), (512, 256), (256, 512), (1000, 300), (100, 1), (64, 2048), (4096, 1024)):
            assert decomp.process_grid(nranks, nxg, nyg) == _ref_process_grid(nranks, nxg, nyg)
    for n_glob in (12, 50, 97, 256, 1000, 4097):
        for nproc in (1, 2, 3, 4, 7, 8):
            if n_glob // nproc < 1:
                continue
            ranges = [decomp.tile(n_glob, nproc, p) for p in range(nproc)]
            nper = n_glob / nproc
            for p, (beg, n) in enumerate(ranges):
                assert beg == _round_half_away(nper * p)
                assert beg + n - 1 == _round_half_away(nper * (p + 1)) - 1
            assert ranges[0][0] == 0 and sum(n for _, n in ranges) == n_glob
            assert all(ranges[p][0] + ranges[p][1] == ranges[p + 1][0] for p in range(nproc - 1))
    for npx, npy in ((1, 1), (2, 1), (3, 2), (4, 4)):
        for py in range(npy):
            for px in range(npx):
                want = [py * npx + (px - 1) % npx, py * npx + (px + 1) % npx,
                        ((py - 1) % npy) * npx + px, ((py + 1) % npy) * npx + px]
                assert decomp.neighbors(npx, npy, px, py) == want


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


W = 5


def _worker(rank, world, port, nxg, nyg, out):
    import datetime
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        npx, npy = decomp.process_grid(world, nxg, nyg)
        t = decomp.tiles(nxg, nyg, npx, npy)[rank]
        nz = 3
        g = np.arange(nz * nyg * nxg, dtype=np.float32).reshape(nz, nyg, nxg)
        loc = g[:, t.j_beg:t.j_beg + t.ny, t.i_beg:t.i_beg + t.nx]
        snd = [loc[:, :, :W], loc[:, :, -W:], loc[:, :W, :], loc[:, -W:, :]]
        snd = [torch.from_numpy(np.ascontiguousarray(a)) for a in snd]
        rcv = [torch.empty_like(a) for a in snd]
        nbr = decomp.neighbors(npx, npy, t.px, t.py)
        posts = []
        for lo in ((0, 2) if nyg > 1 else (0,)):
            hi = lo + 1
            posts += [("send", snd[lo], nbr[lo]), ("recv", rcv[hi], nbr[hi]),
                      ("send", snd[hi], nbr[hi]), ("recv", rcv[lo], nbr[lo])]
        # gloo has no channel to the rank itself; messages to itself are matched
        # here in posting order, as NCCL matches them.
        own_sends = [buf for kind, buf, peer in posts if kind == "send" and peer == rank]
        own_recvs = [buf for kind, buf, peer in posts if kind == "recv" and peer == rank]
        for a, b in zip(own_sends, own_recvs):
            b.copy_(a)
        ops = [dist.P2POp(dist.isend if kind == "send" else dist.irecv, buf, peer)
               for kind, buf, peer in posts if peer != rank]
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        jj = np.arange(t.j_beg, t.j_beg + t.ny)
        ii = np.arange(t.i_beg, t.i_beg + t.nx)
        want = [g[:, jj][:, :, (t.i_beg - W + np.arange(W)) % nxg], g[:, jj][:, :, (t.i_beg + t.nx + np.arange(W)) % nxg],
                g[:, (t.j_beg - W + np.arange(W)) % nyg][:, :, ii], g[:, (t.j_beg + t.ny + np.arange(W)) % nyg][:, :, ii]]
        ok = all(np.array_equal(rcv[d].numpy(), want[d]) for d in ((0, 1, 2, 3) if nyg > 1 else (0, 1)))
        out[rank] = ok
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,nxg,nyg", [(2, 64, 64), (3, 96, 24), (4, 64, 64), (4, 80, 1)])
def test_exchange_schedule_with_gloo_ranks(world, nxg, nyg):
    port = _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_worker, args=(r, world, port, nxg, nyg, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert all(out[r] for r in range(world)), dict(out)
