"""ctypes front end of the CPU oracles (TEST INFRASTRUCTURE ONLY).

Loads ``oracle/_build/liboracle.so`` (this project's restatement, variants
REF and F64) or ``oracle/_ref/libporturb_ref.so`` (the reference's own dycore
headers built against the single-rank shim) and drives either with the same
calls.  Only tests/, ``__graft_entry__.smoke`` and bench.py's CPU baseline use
this module, as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libporturb_ref.so")
# The reference tree: $PORTURB_REFERENCE, by default where this image mounts it.
REFERENCE_DIR = os.environ.get("PORTURB_REFERENCE", "/root/reference")

MAX_TRACERS = 16
BC = {"periodic": 0, "precursor": 1, "solid_wall": 2}
HS = 4


class OrcConfig(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("ntr", C.c_int),
                ("xlen", C.c_double), ("ylen", C.c_double), ("zlen", C.c_double),
                ("tracer_positive", C.c_int * MAX_TRACERS), ("tracer_adds_mass", C.c_int * MAX_TRACERS),
                ("idWV", C.c_int),
                ("R_d", C.c_double), ("R_v", C.c_double), ("cp_d", C.c_double), ("gamma_d", C.c_double),
                ("C0", C.c_double), ("grav", C.c_double),
                ("cfl", C.c_double), ("immersed_power", C.c_double), ("latitude", C.c_double),
                ("bc_x", C.c_int), ("bc_y", C.c_int), ("bc_z", C.c_int),
                ("enable_gravity", C.c_int), ("weno_all", C.c_int)]


def build(ref: bool | None = None) -> None:
    """Build liboracle.so and, when the reference tree is present, the
    reference library."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if ref is None:
        ref = os.path.isdir(os.path.join(REFERENCE_DIR, "model"))
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref", "REFERENCE=" + REFERENCE_DIR], check=True)


def have_ref() -> bool:
    return os.path.exists(REF_SO)


def make_config(case) -> OrcConfig:
    o = case.options
    cfg = OrcConfig()
    cfg.nx, cfg.ny, cfg.nz, cfg.ntr = case.nx, case.ny, case.nz, len(case.tracers)
    cfg.xlen, cfg.ylen, cfg.zlen = case.xlen, case.ylen, case.zlen
    for t, tr in enumerate(case.tracers):
        cfg.tracer_positive[t] = int(tr.positive)
        cfg.tracer_adds_mass[t] = int(tr.adds_mass)
    cfg.idWV = [t.name for t in case.tracers].index("water_vapor")
    cfg.R_d, cfg.R_v, cfg.cp_d = o["R_d"], o["R_v"], o["cp_d"]
    cfg.gamma_d, cfg.C0, cfg.grav = o["gamma_d"], o["C0"], o["grav"]
    cfg.cfl, cfg.immersed_power, cfg.latitude = o["cfl"], o["immersed_power"], o["latitude"]
    cfg.bc_x, cfg.bc_y, cfg.bc_z = BC[o["bc_x"]], BC[o["bc_y"]], BC[o["bc_z"]]
    cfg.enable_gravity, cfg.weno_all = int(o["enable_gravity"]), int(o["weno_all"])
    return cfg


_libs = {}


def _lib(path, prefix):
    if path in _libs:
        return _libs[path]
    lib = C.CDLL(path)
    P = C.c_void_p
    D = C.POINTER(C.c_double)
    F = C.POINTER(C.c_float)
    I = C.c_int
    def sig(name, res, args):
        fn = getattr(lib, prefix + name)
        fn.restype = res
        fn.argtypes = args
    if prefix == "orc_":
        sig("create", P, [C.POINTER(OrcConfig), I])
    else:
        sig("create", P, [C.POINTER(OrcConfig)])
        sig("last_error", C.c_char_p, [])
    sig("destroy", None, [P])
    sig("init", I, [P, D, D, D, D, D, D, D])
    sig("set_hydrostasis", I, [P, D, D, D])
    sig("get_hydrostasis", None, [P, D, D, D, D, D, D])
    sig("compute_time_step", C.c_double, [P])
    sig("time_step", I, [P, D, D, D, D, D, D, C.c_double])
    sig("load_coupler", None if prefix == "orc_" else I, [P, D, D, D, D, D, D])
    sig("store_coupler", None if prefix == "orc_" else I, [P, D, D, D, D, D, D])
    sig("advance", None if prefix == "orc_" else I, [P, C.c_double, I])
    sig("get_state", None, [P, D, D])
    sig("tendencies", None if prefix == "orc_" else I, [P, D, D])
    sig("weno9_f32", None, [F, I, I, I, F, F])
    sig("weno9_f64", None, [D, I, I, I, D, D])
    if prefix == "orc_":
        sig("weno9_f64tvf", None, [D, I, I, I, D, D])
        sig("weno9_batch_f32", None, [F, C.c_long, I, F, F])
        sig("set_state", None, [P, D, D])
        sig("num_threads", I, [])
    _libs[path] = lib
    return lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Dycore:
    """One oracle instance.  kind: 'ref' (this project's REF restatement),
    'f64' (pure FP64 restatement) or 'reference' (the reference's own code)."""

    def __init__(self, case, kind="ref"):
        self.case = case
        self.kind = kind
        self.ntr = len(case.tracers)
        if kind == "reference":
            self.lib = _lib(REF_SO, "ref_")
            self.p = "ref_"
            self.h = self.lib.ref_create(C.byref(make_config(case)))
        else:
            self.lib = _lib(ORACLE_SO, "orc_")
            self.p = "orc_"
            self.h = self.lib.orc_create(C.byref(make_config(case)), 0 if kind == "ref" else 1)
        if not self.h:
            raise RuntimeError("oracle create failed")

    def _f(self, name):
        return getattr(self.lib, self.p + name)

    def _check(self, rc):
        if rc is not None and rc < 0:
            msg = self.lib.ref_last_error().decode() if self.p == "ref_" else "oracle error"
            raise RuntimeError(msg)
        return rc

    def __del__(self):
        try:
            if self.h:
                self._f("destroy")(self.h)
                self.h = None
        except Exception:
            pass

    def init(self, rho_d, u, v, w, T, trc, imm):
        arrs = [_c(x) for x in (rho_d, u, v, w, T, trc, imm)]
        self._check(self._f("init")(self.h, *[_dp(a) for a in arrs]))

    def init_case(self):
        c = self.case
        self.init(c.rho_d, c.uvel, c.vvel, c.wvel, c.temp, c.tracer_data, c.immersed_proportion)

    def set_hydrostasis(self, r, t, p):
        arrs = [_c(x) for x in (r, t, p)]
        self._check(self._f("set_hydrostasis")(self.h, *[_dp(a) for a in arrs]))

    def get_hydrostasis(self):
        nz = self.case.nz
        cells = [np.zeros(nz + 2 * HS) for _ in range(3)]
        edges = [np.zeros(nz + 1) for _ in range(3)]
        self._f("get_hydrostasis")(self.h, *[_dp(a) for a in cells + edges])
        return cells, edges

    def compute_time_step(self):
        return self._f("compute_time_step")(self.h)

    def time_step(self, arrays, dt_phys):
        """arrays: [rho_d, u, v, w, T, tracers] numpy float64, updated in place."""
        for a in arrays:
            assert a.dtype == np.float64 and a.flags.c_contiguous
        return self._check(self._f("time_step")(self.h, *[_dp(a) for a in arrays], dt_phys))

    def load_coupler(self, arrays):
        arrs = [_c(a) for a in arrays]
        self._check(self._f("load_coupler")(self.h, *[_dp(a) for a in arrs]))

    def store_coupler(self):
        c = self.case
        shp = (c.nz, c.ny, c.nx)
        out = [np.zeros(shp) for _ in range(5)] + [np.zeros((self.ntr,) + shp)]
        self._check(self._f("store_coupler")(self.h, *[_dp(a) for a in out]))
        return out

    def advance(self, dt_dyn, nsteps):
        self._check(self._f("advance")(self.h, dt_dyn, nsteps))

    def get_state(self):
        c = self.case
        st = np.zeros((5, c.nz, c.ny, c.nx))
        tr = np.zeros((self.ntr, c.nz, c.ny, c.nx))
        self._f("get_state")(self.h, _dp(st), _dp(tr))
        return st, tr

    def set_state(self, st, tr):
        st, tr = _c(st), _c(tr)
        self._f("set_state")(self.h, _dp(st), _dp(tr))

    def tendencies(self):
        c = self.case
        st = np.zeros((5, c.nz, c.ny, c.nx))
        tr = np.zeros((self.ntr, c.nz, c.ny, c.nx))
        self._check(self._f("tendencies")(self.h, _dp(st), _dp(tr)))
        return st, tr


def weno9(s, do_map=True, imm_L=False, imm_R=False, kind="ref_f32"):
    """Order-9 limiter on one stencil.  kind: ref_f32 / f64 / f64tvf (this
    project's restatement) or reference_f32 / reference_f64."""
    if kind.startswith("reference"):
        lib, p = _lib(REF_SO, "ref_"), "ref_"
        kind = kind[len("reference_"):]
    else:
        lib, p = _lib(ORACLE_SO, "orc_"), "orc_"
        kind = {"ref_f32": "f32"}.get(kind, kind)
    if kind == "f32":
        s = np.ascontiguousarray(s, dtype=np.float32)
        qL, qR = C.c_float(), C.c_float()
        getattr(lib, p + "weno9_f32")(s.ctypes.data_as(C.POINTER(C.c_float)), int(do_map), int(imm_L), int(imm_R),
                                      C.byref(qL), C.byref(qR))
        return np.float32(qL.value), np.float32(qR.value)
    s = np.ascontiguousarray(s, dtype=np.float64)
    qL, qR = C.c_double(), C.c_double()
    getattr(lib, p + "weno9_" + kind)(_dp(s), int(do_map), int(imm_L), int(imm_R), C.byref(qL), C.byref(qR))
    return qL.value, qR.value


def weno9_batch_f32(stencils, do_map=True):
    lib = _lib(ORACLE_SO, "orc_")
    s = np.ascontiguousarray(stencils, dtype=np.float32)
    n = s.shape[0]
    qL = np.zeros(n, np.float32)
    qR = np.zeros(n, np.float32)
    fp = C.POINTER(C.c_float)
    lib.orc_weno9_batch_f32(s.ctypes.data_as(fp), n, int(do_map), qL.ctypes.data_as(fp), qR.ctypes.data_as(fp))
    return qL, qR
