"""Failure detection through the C-ABI, without a GPU fault.

The reference checks the coupler state for NaN/Inf when built with
PORTURB_NAN_CHECKS (coupler.h:349-376, around every module call) and aborts.
Here every output cell of the z kernels is tested with isfinite and a device
flag makes the next synchronising call return PU_ERR_NONFINITE, after which
the flag is clear.  The failure is made on the host: a NaN or an Inf written
into one cell of the coupler arrays the caller passes in (host or device
memory).  Bad arguments and calls out of order return PU_ERR_INVALID /
PU_ERR_STATE before any GPU work, where the reference aborts
(Options.h:122-148, dynamics_rk.h:799).  The stage kernels' bounded wait is
made to run out on a barrier that nothing completes, and reports it; a
device allocation that cannot succeed returns PU_ERR_NOMEM and leaves
nothing allocated.
"""
import ctypes as C

import numpy as np
import pytest

from porturb_b200 import Dycore, PortUrbError, capi, cases
from porturb_b200.dycore import make_view

pytestmark = pytest.mark.gpu


def _arrays(case, perturbed=True):
    rd, u, v, w, T, trc = case.coupler_arrays(perturbed=perturbed)
    return [np.ascontiguousarray(np.array(a, dtype=np.float64)) for a in (rd, u, v, w, T)], \
           [np.ascontiguousarray(np.array(t, dtype=np.float64)) for t in trc]


def _handle(case, precision="f32"):
    g = Dycore.from_case(case, precision=precision, device=0)
    st, tr = _arrays(case, perturbed=False)
    imm = np.ascontiguousarray(case.immersed_proportion)
    g.init(*st, tr, imm if imm.any() else None)
    return g


@pytest.mark.parametrize("field,value,where", [(1, np.nan, "host"), (4, np.inf, "host"), (3, np.nan, "device"),
                                               (0, -np.inf, "host")])
@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_nonfinite_input_is_reported_then_cleared(field, value, where, precision):
    import torch
    case = cases.small_mixed()
    g = _handle(case, precision)
    dt_phys = 2.5 * g.compute_time_step()
    st, tr = _arrays(case)
    k, j, i = case.nz // 2, case.ny // 3, case.nx // 4
    st[field][k, j, i] = value
    if where == "device":
        st = [torch.tensor(a, device="cuda:0") for a in st]
        tr = [torch.tensor(a, device="cuda:0") for a in tr]
    with pytest.raises(PortUrbError) as e:
        g.time_step(*st, tr, dt_phys)
    assert e.value.status == capi.PU_ERR_NONFINITE
    assert b"non-finite" in capi.load().pu_last_error()
    # The flag was cleared by the failing call: a clean call succeeds and
    # gives what a fresh handle gives on the same arrays, bit for bit.
    st, tr = _arrays(case)
    assert g.time_step(*st, tr, dt_phys) == 3
    assert g.synchronize() is None
    g2 = _handle(case, precision)
    st2, tr2 = _arrays(case)
    g2.time_step(*st2, tr2, dt_phys)
    for a, b in zip(st + tr, st2 + tr2):
        assert np.array_equal(a, b)
    g.close()
    g2.close()


@pytest.mark.parametrize("k", [5, 70])
def test_nonfinite_input_overlapped_time_step(k):
    """The same on a grid whose time_step on host arrays overlaps the copies
    with the steps (nz = 96: three 32-level chunks; the NaN in the first or
    the last chunk): the call returns PU_ERR_NONFINITE after its copies
    finished, and the next clean call gives a fresh handle's bits."""
    case = cases.abl_neutral(nx=32, ny=32, nz=96)
    g = _handle(case)
    dt_phys = 2.5 * g.compute_time_step()
    st, tr = _arrays(case)
    l0 = g.kernel_launches()
    st[2][k, 7, 9] = np.nan
    with pytest.raises(PortUrbError) as e:
        g.time_step(*st, tr, dt_phys)
    assert e.value.status == capi.PU_ERR_NONFINITE
    # The chunked launches (63 here against 21 for the serial form): the
    # overlapped path ran.
    assert g.kernel_launches() - l0 > 40
    st, tr = _arrays(case)
    assert g.time_step(*st, tr, dt_phys) == 3
    g2 = _handle(case)
    st2, tr2 = _arrays(case)
    g2.time_step(*st2, tr2, dt_phys)
    for a, b in zip(st + tr, st2 + tr2):
        assert np.array_equal(a, b)
    g.close()
    g2.close()


def test_nonfinite_state_through_advance_is_reported_by_synchronize():
    case = cases.small_mixed(immersed=False)
    g = _handle(case)
    st, tr = _arrays(case)
    st[2][1, 2, 3] = np.nan
    g.load_state(*st, tr)
    g.advance(g.compute_time_step(), 2)
    with pytest.raises(PortUrbError) as e:
        g.synchronize()
    assert e.value.status == capi.PU_ERR_NONFINITE
    g.synchronize()          # cleared
    g.close()


def test_bad_arguments_and_calls_out_of_order():
    lib = capi.load()
    case = cases.small_mixed(immersed=False)
    g = Dycore.from_case(case, precision="f32", device=0)
    st, tr = _arrays(case)
    view = make_view(*st, tr)
    n = C.c_int()
    # Before init: every call that needs the state is out of order.
    assert lib.pu_dycore_time_step(g.h, C.byref(view), 1.0, C.byref(n)) == capi.PU_ERR_STATE
    assert lib.pu_dycore_advance(g.h, 1.0, 1) == capi.PU_ERR_STATE
    assert lib.pu_dycore_load_state(g.h, C.byref(view)) == capi.PU_ERR_STATE
    assert lib.pu_dycore_store_state(g.h, C.byref(view)) == capi.PU_ERR_STATE
    assert lib.pu_dycore_diagnostics(g.h, C.byref(capi.pu_diag())) == capi.PU_ERR_STATE
    assert lib.pu_dycore_learned_harvest(g.h, 16, 0) == capi.PU_ERR_STATE
    assert lib.pu_dycore_set_weno_mode(g.h, capi.PU_WENO_LEARNED) == capi.PU_ERR_STATE   # untrained
    assert b"neither trained nor loaded" in lib.pu_last_error()
    base, btr = _arrays(case, perturbed=False)
    capi.check(lib.pu_dycore_init(g.h, C.byref(make_view(*base, btr)), None, capi.PU_MEM_HOST))
    # Bad arguments after init.
    assert lib.pu_dycore_time_step(g.h, C.byref(view), 0.0, C.byref(n)) == capi.PU_ERR_INVALID
    assert lib.pu_dycore_time_step(g.h, C.byref(view), -1.0, None) == capi.PU_ERR_INVALID
    assert lib.pu_dycore_time_step(g.h, None, 1.0, None) == capi.PU_ERR_INVALID
    assert lib.pu_dycore_advance(g.h, 0.0, 1) == capi.PU_ERR_INVALID
    assert lib.pu_dycore_advance(g.h, 1.0, -1) == capi.PU_ERR_INVALID
    assert lib.pu_dycore_set_weno_mode(g.h, 7) == capi.PU_ERR_INVALID
    assert lib.pu_dycore_learned_set_threshold(g.h, -0.5) == capi.PU_ERR_INVALID
    assert lib.pu_dycore_learned_train(g.h, 10, 64, 1e-3, 0, None) == capi.PU_ERR_STATE   # nothing harvested
    bad = make_view(*st, tr)
    bad.uvel = None
    assert lib.pu_dycore_load_state(g.h, C.byref(bad)) == capi.PU_ERR_INVALID
    assert b"null array" in lib.pu_last_error()
    # A handle on a device that does not exist.
    cfg = capi.pu_config.from_buffer_copy(g.cfg)
    cfg.device = 4096
    h = C.c_void_p()
    assert lib.pu_dycore_create(C.byref(cfg), C.byref(h)) == capi.PU_ERR_INVALID
    # The handle still works after all of the above.
    assert g.time_step(*st, tr, 2.5 * g.compute_time_step()) == 3
    g.close()


def test_bounded_wait_runs_out_and_the_context_stays_usable(gpu_lib):
    """The wait of the stage kernels' TMA staging (pu::tma::mbar_wait) made to
    run out on an mbarrier whose announced copies are never issued
    (pu_check_bounded_wait): it gives up after its time limit (2 ms here, then
    the stage kernels' own 20 ms) and reports that it did, the kernel returns
    within a few ms of the limit, and the context keeps working (a dycore
    step afterwards matches a fresh handle's)."""
    lib = capi.load()
    done = C.c_int(-1)
    assert lib.pu_check_bounded_wait(100, C.byref(done), None, None) == capi.PU_OK   # loads the kernel
    assert done.value == 0
    for limit_us, limit_ms in ((2000, 2.0), (0, 20.0)):
        done, ms, cyc = C.c_int(-1), C.c_double(), C.c_longlong()
        assert lib.pu_check_bounded_wait(limit_us, C.byref(done), C.byref(ms), C.byref(cyc)) == capi.PU_OK
        print("bounded wait with a %.0f ms limit: gave up after %.3f ms (%d cycles)" % (limit_ms, ms.value, cyc.value))
        assert done.value == 0
        assert limit_ms <= ms.value < limit_ms + 10.0
    done = C.c_int(-1)
    assert lib.pu_check_bounded_wait(-1, C.byref(done), None, None) == capi.PU_ERR_INVALID
    case = cases.small_mixed()
    dt_phys = None
    outs = []
    for _ in range(2):
        g = _handle(case)
        dt_phys = dt_phys or 2.5 * g.compute_time_step()
        st, tr = _arrays(case)
        assert g.time_step(*st, tr, dt_phys) == 3
        outs.append(st + tr)
        g.close()
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


def test_allocation_failure_is_reported_and_released(gpu_lib):
    """A grid larger than the device (2048^3 cells: ~600 GB of state
    buffers) makes pu_dycore_create return PU_ERR_NOMEM; nothing of it stays
    allocated (the free device memory is what it was), and handles created
    afterwards work."""
    import torch
    case = cases.small_mixed()
    g = _handle(case)          # the library's kernels loaded, the context warm
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    with pytest.raises(PortUrbError) as e:
        Dycore(2048, 2048, 2048, 1.0, 1.0, 1.0, case.tracers, case.options, precision="f32", device=0)
    assert e.value.status == capi.PU_ERR_NOMEM
    assert b"cudaMalloc" in capi.load().pu_last_error()
    free1 = torch.cuda.mem_get_info(0)[0]
    assert abs(free1 - free0) <= 8 << 20, (free0, free1)
    dt_phys = 2.5 * g.compute_time_step()
    st, tr = _arrays(case)
    assert g.time_step(*st, tr, dt_phys) == 3
    g.close()
    g2 = _handle(case)
    st2, tr2 = _arrays(case)
    assert g2.time_step(*st2, tr2, dt_phys) == 3
    for a, b in zip(st + tr, st2 + tr2):
        assert np.array_equal(a, b)
    g2.close()


def test_normalize9_matches_oracle(gpu_lib):
    """The learned path's input convention (WenoLimiter.h:85-96, threshold
    1e-20) on random, constant, near-constant, wide-range and negative
    stencils, against oracle/mlp_oracle.normalize: within 2 float ulps of 1
    (the kernel multiplies by the reciprocal of the range where the oracle
    divides), and exactly zero where the range is at most 1e-20."""
    import mlp_oracle
    rng = np.random.default_rng(11)
    s = [rng.standard_normal((4096, 9)),
         np.full((8, 9), 3.25),
         1.0 + np.linspace(0, 1, 9)[None, :] * np.array([1e-21, 5e-21, 1e-20, 2e-20, 1e-19, 1e-12, 1e-7, 1.0])[:, None],
         np.linspace(0, 1, 9)[None, :] * np.array([5e-21, 1e-20, 2e-20, 1e-19])[:, None],
         1e30 * rng.standard_normal((64, 9)),
         -1e-3 * rng.random((64, 9)) - 5.0,
         np.where(rng.random((256, 9)) < 0.5, 0.0, 1.0) * rng.standard_normal((256, 9))]
    s = np.concatenate(s).astype(np.float32)
    n = s.shape[0]
    x = np.zeros((n, 9), np.float32)
    jump = np.zeros(n, np.float32)
    capi.check(gpu_lib.pu_learned_normalize_f32(s.ctypes.data, n, x.ctypes.data, jump.ctypes.data))
    want = mlp_oracle.normalize(s)
    assert np.abs(x - want).max() <= 2 * 2.0 ** -24 * 2
    rng_ = s.max(axis=1) - s.min(axis=1)
    assert np.all(x[rng_ <= np.float32(1e-20)] == 0.0)
    assert np.all(x[rng_ > np.float32(1e-20)].max(axis=1) > 0.999999)
    jw = np.abs(np.diff(want, axis=1)).max(axis=1)
    assert np.abs(jump - jw).max() <= 4 * 2.0 ** -24 * 2
