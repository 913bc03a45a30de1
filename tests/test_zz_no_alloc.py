"""The time step that allocates no device memory.

pu_dycore_time_step_noalloc serves callers that cannot call cudaMalloc -- a
host model whose own allocator has already reserved the GPU's memory, or a
plug-in running inside a time loop where device allocation is not allowed.
Its working memory is one static device array inside the library.  This test
drives it through the C-ABI twice in a row and checks each result against the
handle-based pu_dycore_time_step on identical device-resident coupler arrays.
Both run the same kernels on the same cell profiles, so they must agree bit
for bit.  Each call reuses the array the previous call left behind.  The
device's free memory (cudaMemGetInfo) must not change across the two calls,
after one warm-up call has loaded the kernels.
"""
import ctypes as C

import numpy as np
import pytest

from porturb_b200 import Dycore, capi, cases
from porturb_b200.dycore import make_view

pytestmark = pytest.mark.gpu

CASES = {
    "small_two_tracers": lambda: cases.small_mixed(immersed=False),
    "abl_block_48x40x32": lambda: cases.abl_neutral(nx=48, ny=40, nz=32),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_noalloc_matches_time_step_on_two_calls(name):
    import torch
    case = CASES[name]()
    g = Dycore.from_case(case, precision="f32", device=0)
    base = [np.ascontiguousarray(a) for a in case.coupler_arrays(perturbed=False)]
    g.init(*base[:5], list(base[5]), None)
    cells = [np.ascontiguousarray(c) for c in g.get_hydrostasis()[0]]
    dt_phys = 2.5 * g.compute_time_step()
    pert = case.coupler_arrays(perturbed=True)
    dev = torch.device("cuda", 0)

    def device_copy():
        st = [torch.tensor(np.ascontiguousarray(a), device=dev) for a in pert[:5]]
        tr = [torch.tensor(np.ascontiguousarray(t), device=dev) for t in pert[5]]
        return st, tr

    lib = capi.load()

    def noalloc(view):
        n = C.c_int()
        capi.check(lib.pu_dycore_time_step_noalloc(C.byref(g.cfg), cells[0].ctypes.data, cells[1].ctypes.data,
                                                   cells[2].ctypes.data, C.byref(view), dt_phys, C.byref(n)))
        return n.value

    # Warm-up call on a throw-away copy: it loads the kernels (lazy module
    # loading takes device memory once) and sets up the scratch address.
    w_st, w_tr = device_copy()
    noalloc(make_view(*w_st, w_tr))
    torch.cuda.synchronize()

    a_st, a_tr = device_copy()        # existing entry point
    b_st, b_tr = device_copy()        # no-allocation entry point
    view_b = make_view(*b_st, b_tr)
    for call in range(2):
        n_ref = g.time_step(*a_st, a_tr, dt_phys)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info(0)[0]
        n = noalloc(view_b)
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info(0)[0]
        assert free1 == free0, (name, call, free0, free1)
        assert n == n_ref == 3
        for x, y in zip(b_st + b_tr, a_st + a_tr):
            assert torch.equal(x, y), (name, call, (x - y).abs().max().item())
    g.close()


def test_noalloc_rejects_grids_beyond_its_scratch():
    case = cases.abl_neutral(nx=128, ny=128, nz=64)     # ~1M cells, above the 64 MiB limit
    g = Dycore.from_case(case, precision="f32", device=0)
    cells = [np.ones(case.nz + 8) for _ in range(3)]
    dummy = np.zeros(1)
    view = capi.pu_state_view()
    for name in ("rho_d", "uvel", "vvel", "wvel", "temp"):
        setattr(view, name, dummy.ctypes.data)
    for t in range(len(case.tracers)):
        view.tracers[t] = dummy.ctypes.data
    view.mem = capi.PU_MEM_DEVICE
    rc = capi.load().pu_dycore_time_step_noalloc(C.byref(g.cfg), cells[0].ctypes.data, cells[1].ctypes.data,
                                                 cells[2].ctypes.data, C.byref(view), 1.0, None)
    assert rc == capi.PU_ERR_UNSUPPORTED
    assert b"too large" in capi.load().pu_last_error()
    g.close()
