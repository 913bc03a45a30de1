"""Domain decomposition of the dycore across GPUs (coupler.h:132-229), on the
decomposition entry points of include/pu_dycore.h.

* :func:`process_grid`, :func:`tile`, :func:`neighbors` -- the reference
  coupler's process grid, tile ranges and neighbour ranks (host-only library
  calls).
* :func:`tile_case` -- one tile of a global case (the arrays a rank's coupler
  holds after distribute_mpi_and_allocate_coupled_state).
* One process (rank) per GPU: rank 0 makes :func:`nccl_unique_id`, the host
  broadcasts it, and every rank calls ``Dycore.set_decomposition(...,
  nccl_id=...)`` before ``init``; init and time steps are then collective.
  :func:`distributed_tile` does this over ``torch.distributed``.
* :class:`TileGroup` -- the tiles of a grid as handles of one process on one
  stream, stepped together with device copies for the exchange.
* :class:`TorchHostTransport` -- a pu_host_transport over a torch.distributed
  process group with CPU tensors (gloo): the halo slabs and the init
  reductions go through host memory, as the reference's coupler sends them
  through MPI; :func:`host_transport_tile` makes this rank's tile with it.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import capi
from .capi import check
from .dycore import Dycore, _ptr, make_view


def process_grid(nranks: int, nx_glob: int, ny_glob: int) -> Tuple[int, int]:
    """(nproc_x, nproc_y) the reference's coupler picks (coupler.h:148-171)."""
    lib = capi.load()
    px, py = C.c_int(), C.c_int()
    check(lib.pu_decomp_process_grid(int(nranks), int(nx_glob), int(ny_glob), C.byref(px), C.byref(py)))
    return px.value, py.value


def tile(n_glob: int, nproc: int, p: int) -> Tuple[int, int]:
    """(first index, size) of tile p along an axis (coupler.h:176-183)."""
    lib = capi.load()
    beg, n = C.c_longlong(), C.c_longlong()
    check(lib.pu_decomp_tile(int(n_glob), int(nproc), int(p), C.byref(beg), C.byref(n)))
    return beg.value, n.value


def make_decomp(nproc_x, nproc_y, px, py, nx_glob, ny_glob) -> capi.pu_decomp:
    d = capi.pu_decomp()
    d.nproc_x, d.nproc_y, d.px, d.py, d.nx_glob, d.ny_glob = nproc_x, nproc_y, px, py, nx_glob, ny_glob
    return d


def neighbors(nproc_x, nproc_y, px, py) -> List[int]:
    """Ranks beyond the x-, x+, y-, y+ edges of tile (px, py) (coupler.h:203-214)."""
    lib = capi.load()
    d = make_decomp(nproc_x, nproc_y, px, py, 1, 1)
    nbr = (C.c_int * 4)()
    check(lib.pu_decomp_neighbors(C.byref(d), nbr))
    return list(nbr)


def nccl_unique_id() -> bytes:
    """A new NCCL unique id for Dycore.set_decomposition (one rank makes it)."""
    lib = capi.load()
    buf = C.create_string_buffer(capi.PU_NCCL_ID_BYTES)
    check(lib.pu_nccl_get_unique_id(buf))
    return buf.raw


@dataclasses.dataclass
class Tile:
    nproc_x: int
    nproc_y: int
    px: int
    py: int
    i_beg: int
    j_beg: int
    nx: int
    ny: int


def tiles(nx_glob, ny_glob, nproc_x, nproc_y) -> List[Tile]:
    """Every tile of the grid, in rank order (rank = py*nproc_x + px)."""
    out = []
    for py in range(nproc_y):
        for px in range(nproc_x):
            i0, nx = tile(nx_glob, nproc_x, px)
            j0, ny = tile(ny_glob, nproc_y, py)
            out.append(Tile(nproc_x, nproc_y, px, py, i0, j0, nx, ny))
    return out


def tile_case(case, t: Tile):
    """The tile of a global case: the same grid spacing, options and tracers,
    the arrays cut to the tile."""
    sl = (slice(None), slice(t.j_beg, t.j_beg + t.ny), slice(t.i_beg, t.i_beg + t.nx))
    cut = lambda a: np.ascontiguousarray(a[sl])
    pert = None
    if case.perturbed is not None:
        pert = {k: cut(v) for k, v in case.perturbed.items()}
    return dataclasses.replace(
        case, nx=t.nx, ny=t.ny, xlen=case.xlen / case.nx * t.nx, ylen=case.ylen / case.ny * t.ny,
        rho_d=cut(case.rho_d), uvel=cut(case.uvel), vvel=cut(case.vvel), wvel=cut(case.wvel), temp=cut(case.temp),
        tracer_data=np.ascontiguousarray(case.tracer_data[(slice(None),) + sl]),
        immersed_proportion=cut(case.immersed_proportion), perturbed=pert)


def assemble(parts: Sequence[np.ndarray], ts: Sequence[Tile], nx_glob: int, ny_glob: int) -> np.ndarray:
    """Global (..., nz, ny_glob, nx_glob) array from per-tile (..., nz, ny, nx) arrays."""
    lead = parts[0].shape[:-2]
    out = np.empty(lead + (ny_glob, nx_glob), dtype=parts[0].dtype)
    for a, t in zip(parts, ts):
        out[..., t.j_beg:t.j_beg + t.ny, t.i_beg:t.i_beg + t.nx] = a
    return out


def set_decomposition(dyc: Dycore, t: Tile, nx_glob: int, ny_glob: int, nccl_id: Optional[bytes] = None):
    d = make_decomp(t.nproc_x, t.nproc_y, t.px, t.py, nx_glob, ny_glob)
    check(dyc.lib.pu_dycore_set_decomposition(dyc.h, C.byref(d), nccl_id))


class TileGroup:
    """The tiles of an nproc_x x nproc_y grid over a global case as handles of
    one process on one device and stream (pu_dycore_group_*)."""

    def __init__(self, case, nproc_x, nproc_y, precision="f32", device=0, stream=None, **kw):
        self.case = case
        self.tiles = tiles(case.nx, case.ny, nproc_x, nproc_y)
        self.cases = [tile_case(case, t) for t in self.tiles]
        self.handles = [Dycore.from_case(c, precision=precision, device=device, stream=stream, **kw)
                        for c in self.cases]
        for h, t in zip(self.handles, self.tiles):
            set_decomposition(h, t, case.nx, case.ny)
        self.lib = self.handles[0].lib
        self._hs = (C.c_void_p * len(self.handles))(*[h.h for h in self.handles])

    def _views(self, arrays):
        views = (capi.pu_state_view * len(arrays))()
        for i, (rd, u, v, w, T, trc) in enumerate(arrays):
            views[i] = make_view(rd, u, v, w, T, list(trc))
        return views

    def init(self, arrays, props=None, projs=None):
        """arrays[i] = (rho_d, u, v, w, T, tracers) of tile i; props/projs: the
        tiles' immersed_proportion / windmill_proj_weight, or None."""
        n = len(self.handles)
        views = self._views(arrays)
        mem = views[0].mem
        pp = pj = None
        if props is not None:
            pp = (C.c_void_p * n)(*[None if a is None else _ptr(a)[0] for a in props])
        if projs is not None:
            pj = (C.c_void_p * n)(*[None if a is None else _ptr(a)[0] for a in projs])
        check(self.lib.pu_dycore_group_init(self._hs, n, views, pp, pj, mem))

    def init_case(self, perturbed=False):
        """init from the tiles' coupler arrays of the case."""
        arrays = [[np.ascontiguousarray(a) for a in c.coupler_arrays(perturbed=perturbed)] for c in self.cases]
        arrays = [(rd, u, v, w, T, [np.ascontiguousarray(x) for x in trc]) for rd, u, v, w, T, trc in arrays]
        props = [np.ascontiguousarray(c.immersed_proportion) for c in self.cases]
        self.init(arrays, props if any(p.any() for p in props) else None)

    def advance(self, dt, nsteps=1):
        check(self.lib.pu_dycore_group_advance(self._hs, len(self.handles), float(dt), int(nsteps)))

    def time_step(self, arrays, dt_phys) -> int:
        views = self._views(arrays)
        n = C.c_int()
        check(self.lib.pu_dycore_group_time_step(self._hs, len(self.handles), views, float(dt_phys), C.byref(n)))
        return n.value

    def get_conserved(self):
        """Global (5, nz, ny, nx) state and (ntr, nz, ny, nx) tracers."""
        parts = [h.get_conserved() for h in self.handles]
        return (assemble([p[0] for p in parts], self.tiles, self.case.nx, self.case.ny),
                assemble([p[1] for p in parts], self.tiles, self.case.nx, self.case.ny))

    def close(self):
        for h in self.handles:
            h.close()


def distributed_tile(case, precision="f32", device=None, stream=None, group=None, **kw):
    """This rank's tile of a global case over torch.distributed (one process
    per GPU): the process grid of coupler.h:148-171 for the world size, the
    NCCL id broadcast from rank 0, the handle decomposed (collective).
    Returns (Dycore, Tile, tile case)."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    npx, npy = process_grid(world, case.nx, case.ny)
    t = tiles(case.nx, case.ny, npx, npy)[rank]
    tc = tile_case(case, t)
    if device is None:
        device = torch.cuda.current_device() if torch.cuda.is_available() else 0
    box = [nccl_unique_id() if rank == 0 else None]
    dist.broadcast_object_list(box, src=0, group=group)
    h = Dycore.from_case(tc, precision=precision, device=device, stream=stream, **kw)
    set_decomposition(h, t, case.nx, case.ny, nccl_id=box[0])
    return h, t, tc


class TorchHostTransport:
    """The callbacks of a pu_host_transport on a torch.distributed process
    group that carries CPU tensors (gloo).

    exchange: for each active direction d, the slab snd[d] goes to rank
    nbr[d] with tag d ^ 1 (the receiver's slot for it) and rcv[d] is received
    from nbr[d] with tag d; a rank that is its own neighbour takes its own
    snd[d ^ 1].  allreduce_sum_f64 and allgather map to the group's
    all_reduce and all_gather.  A callback that raises returns 1 (the dycore
    call then returns PU_ERR_TRANSPORT) and keeps the exception in `error`.
    Keep the object alive while the handle that uses it lives."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.error: Optional[BaseException] = None
        self.calls = {"exchange": 0, "allreduce_sum_f64": 0, "allgather": 0}
        self._fns = (capi.EXCHANGE_FN(self._exchange), capi.ALLREDUCE_FN(self._allreduce),
                     capi.ALLGATHER_FN(self._allgather))
        self.struct = capi.pu_host_transport(self._fns[0], self._fns[1], self._fns[2], None)

    def _global(self, r):
        return r if self.group is None else self.dist.get_global_rank(self.group, r)

    @staticmethod
    def _bytes(ptr, n):
        import torch
        return torch.from_numpy(np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_uint8)), shape=(int(n),)))

    def _exchange(self, user, snd, rcv, nbytes, nbr):
        try:
            self.calls["exchange"] += 1
            reqs, local = [], []
            for d in range(4):
                b = int(nbytes[d])
                if not b:
                    continue
                if nbr[d] == self.rank:
                    local.append(d)
                    continue
                peer = self._global(int(nbr[d]))
                reqs.append(self.dist.isend(self._bytes(snd[d], b), dst=peer, tag=d ^ 1, group=self.group))
                reqs.append(self.dist.irecv(self._bytes(rcv[d], b), src=peer, tag=d, group=self.group))
            for d in local:
                if int(nbytes[d ^ 1]) != int(nbytes[d]):
                    raise ValueError("own-neighbour slabs differ in size")
                C.memmove(rcv[d], snd[d ^ 1], int(nbytes[d]))
            for q in reqs:
                q.wait()
            return 0
        except BaseException as e:  # a ctypes callback must not raise
            self.error = e
            return 1

    def _allreduce(self, user, buf, n):
        try:
            import torch
            self.calls["allreduce_sum_f64"] += 1
            t = torch.from_numpy(np.ctypeslib.as_array(buf, shape=(int(n),)))
            self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
            return 0
        except BaseException as e:
            self.error = e
            return 1

    def _allgather(self, user, src, out, nbytes):
        try:
            import torch
            self.calls["allgather"] += 1
            b = int(nbytes)
            mine = self._bytes(src, b).clone()
            parts = [torch.empty(b, dtype=torch.uint8) for _ in range(self.world)]
            self.dist.all_gather(parts, mine, group=self.group)
            dst = self._bytes(out, b * self.world)
            for r, part in enumerate(parts):
                dst[r * b:(r + 1) * b] = part
            return 0
        except BaseException as e:
            self.error = e
            return 1


def set_decomposition_host(dyc: Dycore, t: Tile, nx_glob: int, ny_glob: int, transport: TorchHostTransport):
    d = make_decomp(t.nproc_x, t.nproc_y, t.px, t.py, nx_glob, ny_glob)
    dyc._transport = transport          # the callbacks must outlive the handle's use of them
    check(dyc.lib.pu_dycore_set_decomposition_host(dyc.h, C.byref(d), C.byref(transport.struct)))


def host_transport_tile(case, precision="f32", device=0, stream=None, group=None, **kw):
    """This rank's tile of a global case, its halos moved through host memory
    by a :class:`TorchHostTransport` on ``group`` (gloo): the process grid of
    coupler.h:148-171 for the group's size, the handle decomposed
    (collective).  Returns (Dycore, Tile, tile case, transport)."""
    tr = TorchHostTransport(group)
    npx, npy = process_grid(tr.world, case.nx, case.ny)
    t = tiles(case.nx, case.ny, npx, npy)[tr.rank]
    tc = tile_case(case, t)
    h = Dycore.from_case(tc, precision=precision, device=device, stream=stream, **kw)
    set_decomposition_host(h, t, case.nx, case.ny, tr)
    return h, t, tc, tr
