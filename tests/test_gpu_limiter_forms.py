"""The FP32 order-9 limiter's forms agree bit for bit
(pu_weno9_edges_f32): the scalar form (z march, fallbacks), the packed
two-stencil form of the x/y kernel (FFMA2/FADD2/FMUL2) and its one-edge
form for the halo cells.  Stencils: random
normal, polynomials of degree <= 4, constants, smooth data plus noise of
amplitude 1e-9 .. 1e-1 (weights from ideal to far from it), steps, with
random map and immersed flags.  The scalar form is also held to the
reference's float limiter (the oracle's weno9_batch_f32, bit-identical to
WenoLimiter<float,9>): within 2e-5 of each stencil's range plus 5 % of its
magnitude, the effect of the rearranged arithmetic (on a constant stencil
this form returns the value exactly, the reference's polynomial
coefficients only to float rounding)."""
import ctypes as C

import numpy as np
import pytest

import pyoracle
from porturb_b200 import capi

pytestmark = pytest.mark.gpu

def _stencils(n, seed=0):
    rng = np.random.default_rng(seed)
    x = np.arange(-4, 5, dtype=np.float64)
    parts = [rng.standard_normal((n, 9))]
    c = rng.standard_normal((n, 5))
    poly = sum(c[:, j:j + 1] * (x[None, :] / 4) ** j for j in range(5))
    parts.append(poly)
    parts.append(np.repeat(rng.standard_normal((n // 8, 1)), 9, axis=1))
    amp = 10.0 ** rng.uniform(-9, -1, size=(n, 1))
    parts.append(poly + amp * rng.standard_normal((n, 9)))
    step = np.where(x[None, :] >= rng.integers(-4, 5, size=(n, 1)), 1.0, 0.0) + 1e-3 * rng.standard_normal((n, 9))
    parts.append(step)
    s = np.concatenate(parts).astype(np.float32)
    flags = rng.integers(0, 8, size=s.shape[0]).astype(np.uint8)
    flags[: s.shape[0] // 2] = 1      # half the stencils: do_map, no immersed neighbours
    return np.ascontiguousarray(s), flags


def _run(lib, s, flags, variant):
    n = s.shape[0]
    qL = np.empty(n, np.float32)
    qR = np.empty(n, np.float32)
    rc = lib.pu_weno9_edges_f32(s.ctypes.data, flags.ctypes.data, n, variant, qL.ctypes.data, qR.ctypes.data,
                                capi.PU_MEM_HOST)
    assert rc == 0, lib.pu_last_error()
    return qL, qR


def test_limiter_forms_agree_bit_for_bit(gpu_lib):
    s, flags = _stencils(40000)
    out = [_run(gpu_lib, s, flags, v) for v in range(2)]
    assert np.array_equal(out[1][0].view(np.uint32), out[0][0].view(np.uint32))
    assert np.array_equal(out[1][1].view(np.uint32), out[0][1].view(np.uint32))
    assert np.all(np.isfinite(out[0][0])) and np.all(np.isfinite(out[0][1]))


def test_one_edge_form_gives_the_same_bits(gpu_lib):
    """Variant 4, the halo cells of the x/y kernel: the right edge of each
    even stencil and the left edge of each odd one, bit for bit those of the
    two-edge forms (random map and immersed flags per lane)."""
    s, flags = _stencils(40000, seed=3)
    qL0, qR0 = _run(gpu_lib, s, flags, 0)
    qL4, qR4 = _run(gpu_lib, s, flags, 4)
    assert np.array_equal(qR4[0::2].view(np.uint32), qR0[0::2].view(np.uint32))
    assert np.array_equal(qL4[1::2].view(np.uint32), qL0[1::2].view(np.uint32))
    assert np.all(np.isnan(qL4[0::2])) and np.all(np.isnan(qR4[1::2]))


def test_scalar_form_against_the_reference_limiter(oracle_lib, gpu_lib):
    s, _ = _stencils(4000, seed=1)
    flags = np.ones(s.shape[0], np.uint8)
    qL, qR = _run(gpu_lib, s, flags, 0)
    rL, rR = pyoracle.weno9_batch_f32(s, do_map=True)
    # Scale: the stencil's range, plus its magnitude for nearly constant
    # stencils (the reference forms edge values through polynomial
    # coefficients that sum to 1 only to float rounding).
    scale = (s.max(1) - s.min(1)) + 0.05 * np.abs(s).max(1) + 1e-30
    eL, eR = np.abs(qL - rL) / scale, np.abs(qR - rR) / scale
    print("max |gpu - reference| / scale: %.2e %.2e" % (eL.max(), eR.max()))
    assert eL.max() <= 2e-5 and eR.max() <= 2e-5


def test_tensor_core_form_matches_the_fp32_forms(oracle_lib, gpu_lib):
    """The tensor-core form (linear forms by tcgen05.mma in 3xTF32): within
    the rounding of its reordered sums of the FP32 form, and as close to the
    reference's float limiter as the FP32 form is (on the same stencils:
    at most 3x the FP32 form's largest deviation)."""
    s, flags = _stencils(40000, seed=2)
    q0 = _run(gpu_lib, s, flags, 0)
    q2 = _run(gpu_lib, s, flags, 2)
    q3 = _run(gpu_lib, s, flags, 3)
    assert np.array_equal(q2[0].view(np.uint32), q3[0].view(np.uint32))   # A in shared or tensor memory
    assert np.array_equal(q2[1].view(np.uint32), q3[1].view(np.uint32))
    scale = (s.max(1) - s.min(1)) + 0.05 * np.abs(s).max(1) + 1e-30
    eL = np.abs(q2[0] - q0[0]) / scale
    eR = np.abs(q2[1] - q0[1]) / scale
    print("max |tensor-core - fp32| / scale: %.2e %.2e" % (eL.max(), eR.max()))
    assert eL.max() <= 1e-5 and eR.max() <= 1e-5
    f1 = np.ones(s.shape[0], np.uint8)
    rL, rR = pyoracle.weno9_batch_f32(s, do_map=True)
    e = {}
    for v in (0, 2):
        qL, qR = _run(gpu_lib, s, f1, v)
        e[v] = max((np.abs(qL - rL) / scale).max(), (np.abs(qR - rR) / scale).max())
    print("max deviation from the reference / scale: fp32 %.2e, tensor-core %.2e" % (e[0], e[2]))
    assert e[2] <= 3 * e[0] + 1e-6
