"""Host-side mirror of the reference's dycore module API on top of libpu_dycore.

Two layers:

* :class:`Dycore` -- a thin owner of one pu_dycore handle (create, init,
  load/store of the coupler state, advance, conserved variables, hydrostatic
  profiles, diagnostics).
* :class:`Coupler` and :class:`Dynamics_Euler_Stratified_WenoFV` -- the
  reference's module convention (model/core/coupler.h, dynamics_rk.h):
  ``dycore.init(coupler)``, ``dycore.time_step(coupler, dt_phys)`` and
  ``dycore.compute_time_step(coupler)``, with the state held by name in the
  coupler's data manager.  Arrays may be numpy float64 (host) or torch float64
  CUDA tensors (device); the library is told which.

Errors: the reference aborts on a missing option or a bad value
(Options.h:122-148, dynamics_rk.h:799); here they raise KeyError / TypeError
(options) or :class:`~porturb_b200.capi.PortUrbError` (library status codes).
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import capi
from .capi import check

PRECISIONS = {"f32": capi.PU_F32, "f64": capi.PU_F64}


def _ptr(a):
    """(pointer, mem) of a C-contiguous float64 numpy array or torch CUDA tensor."""
    if isinstance(a, np.ndarray):
        if a.dtype != np.float64 or not a.flags.c_contiguous:
            raise TypeError("arrays must be C-contiguous float64")
        return a.ctypes.data, capi.PU_MEM_HOST
    try:
        import torch
    except ImportError:  # pragma: no cover - torch is part of the image
        torch = None
    if torch is not None and isinstance(a, torch.Tensor):
        if a.dtype != torch.float64 or not a.is_contiguous():
            raise TypeError("tensors must be contiguous float64")
        return a.data_ptr(), (capi.PU_MEM_DEVICE if a.is_cuda else capi.PU_MEM_HOST)
    raise TypeError("unsupported array type %r" % type(a))


def make_view(rho_d, u, v, w, T, tracers: Sequence) -> capi.pu_state_view:
    view = capi.pu_state_view()
    mems = set()
    for name, a in (("rho_d", rho_d), ("uvel", u), ("vvel", v), ("wvel", w), ("temp", T)):
        p, m = _ptr(a)
        setattr(view, name, p)
        mems.add(m)
    for t, a in enumerate(tracers):
        p, m = _ptr(a)
        view.tracers[t] = p
        mems.add(m)
    if len(mems) != 1:
        raise TypeError("all coupler arrays must live in the same memory space")
    view.mem = mems.pop()
    return view


class Dycore:
    """One pu_dycore handle."""

    def __init__(self, nx, ny, nz, dx, dy, dz, tracers, options, precision="f32", device=0, stream=None,
                 z_chunk=0, weno_mode="plain", thread_loads=False, imm_all_levels=False, serial_io=False):
        self.lib = capi.load()
        cfg = capi.pu_config()
        cfg.nx, cfg.ny, cfg.nz = nx, ny, nz
        cfg.dx, cfg.dy, cfg.dz = dx, dy, dz
        cfg.ntracers = len(tracers)
        if len(tracers) > capi.PU_MAX_TRACERS:
            raise capi.PortUrbError(capi.PU_ERR_UNSUPPORTED, "at most %d tracers" % capi.PU_MAX_TRACERS)
        for t, tr in enumerate(tracers):
            cfg.tracer_positive[t] = int(bool(tr.positive))
            cfg.tracer_adds_mass[t] = int(bool(tr.adds_mass))
        names = [tr.name for tr in tracers]
        cfg.idWV = int(options["idWV"]) if "idWV" in options else names.index("water_vapor")
        for key in ("R_d", "R_v", "cp_d", "gamma_d", "C0", "grav"):
            setattr(cfg, key, float(options[key]))
        cfg.cfl = float(options.get("cfl", 0.60))
        cfg.immersed_power = float(options.get("immersed_power", 5.0))
        cfg.latitude = float(options.get("latitude", 0.0))
        cfg.bc_x = capi.BC_NAMES[options.get("bc_x", "periodic")]
        cfg.bc_y = capi.BC_NAMES[options.get("bc_y", "periodic")]
        cfg.bc_z = capi.BC_NAMES.get(options.get("bc_z", "solid_wall"), -1)
        cfg.enable_gravity = int(bool(options.get("enable_gravity", True)))
        cfg.weno_all = int(bool(options.get("weno_all", True)))
        cfg.precision = PRECISIONS[precision]
        cfg.weno_mode = {"plain": capi.PU_WENO_PLAIN, "learned": capi.PU_WENO_LEARNED}[weno_mode]
        cfg.device = device
        cfg.stream = stream
        cfg.z_chunk = z_chunk
        cfg.thread_loads = int(bool(thread_loads))
        cfg.imm_all_levels = int(bool(imm_all_levels))
        cfg.serial_io = int(bool(serial_io))
        self.cfg = cfg
        self.ntr = len(tracers)
        self.shape = (nz, ny, nx)
        h = C.c_void_p()
        check(self.lib.pu_dycore_create(C.byref(cfg), C.byref(h)))
        self.h = h

    @classmethod
    def from_case(cls, case, precision="f32", **kw):
        return cls(case.nx, case.ny, case.nz, case.xlen / case.nx, case.ylen / case.ny, case.zlen / case.nz,
                   case.tracers, case.options, precision=precision, **kw)

    def close(self):
        if getattr(self, "h", None):
            self.lib.pu_dycore_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- reference entry points -------------------------------------------
    def init(self, rho_d, u, v, w, T, tracers, immersed_proportion=None, windmill_proj_weight=None):
        """windmill_proj_weight (optional) is added to immersed_proportion
        before the immersed arrays are built (dynamics_rk.h:1019-1025)."""
        view = make_view(rho_d, u, v, w, T, tracers)
        if windmill_proj_weight is not None:
            if immersed_proportion is None:
                raise ValueError("windmill_proj_weight needs immersed_proportion")
            p, m = _ptr(immersed_proportion)
            q, mq = _ptr(windmill_proj_weight)
            if mq != m:
                raise ValueError("immersed_proportion and windmill_proj_weight must be in the same memory")
            check(self.lib.pu_dycore_init_windmill(self.h, C.byref(view), p, q, m))
        elif immersed_proportion is None:
            check(self.lib.pu_dycore_init(self.h, C.byref(view), None, view.mem))
        else:
            p, m = _ptr(immersed_proportion)
            check(self.lib.pu_dycore_init(self.h, C.byref(view), p, m))

    def compute_time_step(self) -> float:
        dt = C.c_double()
        check(self.lib.pu_dycore_compute_time_step(self.h, C.byref(dt)))
        return dt.value

    def time_step(self, rho_d, u, v, w, T, tracers, dt_phys) -> int:
        view = make_view(rho_d, u, v, w, T, tracers)
        n = C.c_int()
        check(self.lib.pu_dycore_time_step(self.h, C.byref(view), dt_phys, C.byref(n)))
        return n.value

    def load_state(self, rho_d, u, v, w, T, tracers):
        view = make_view(rho_d, u, v, w, T, tracers)
        check(self.lib.pu_dycore_load_state(self.h, C.byref(view)))

    def store_state(self, rho_d, u, v, w, T, tracers):
        view = make_view(rho_d, u, v, w, T, tracers)
        check(self.lib.pu_dycore_store_state(self.h, C.byref(view)))

    def advance(self, dt_dyn, nsteps=1):
        check(self.lib.pu_dycore_advance(self.h, dt_dyn, nsteps))

    def synchronize(self):
        check(self.lib.pu_dycore_synchronize(self.h))

    def get_conserved(self):
        nz, ny, nx = self.shape
        st = np.zeros((5, nz, ny, nx))
        tr = np.zeros((self.ntr, nz, ny, nx))
        check(self.lib.pu_dycore_get_conserved(self.h, st.ctypes.data, tr.ctypes.data, capi.PU_MEM_HOST))
        return st, tr

    def set_conserved(self, st, tr):
        st = np.ascontiguousarray(st, dtype=np.float64)
        tr = np.ascontiguousarray(tr, dtype=np.float64)
        check(self.lib.pu_dycore_set_conserved(self.h, st.ctypes.data, tr.ctypes.data, capi.PU_MEM_HOST))

    def get_hydrostasis(self):
        nz = self.shape[0]
        cells = [np.zeros(nz + 2 * capi.PU_HS) for _ in range(3)]
        edges = [np.zeros(nz + 1) for _ in range(3)]
        check(self.lib.pu_dycore_get_hydrostasis(self.h, *[a.ctypes.data for a in cells + edges]))
        return cells, edges

    def set_hydrostasis(self, dens, theta, pressure):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (dens, theta, pressure)]
        check(self.lib.pu_dycore_set_hydrostasis(self.h, *[a.ctypes.data for a in arrs]))

    def diagnostics(self) -> Dict[str, float]:
        d = capi.pu_diag()
        check(self.lib.pu_dycore_diagnostics(self.h, C.byref(d)))
        out = {k: getattr(d, k) for k in ("mass", "rho_theta", "kinetic", "internal", "potential", "total_energy")}
        out["tracer_mass"] = [d.tracer_mass[t] for t in range(self.ntr)]
        return out

    def perturbations(self, rho_d, u, v, w, T, tracers):
        """(density_pert, theta_pert, pressure_pert) of coupler arrays against
        the handle's cell profiles: the dycore's output fields
        (dynamics_rk.h:1212-1232), float64 numpy arrays."""
        view = make_view(rho_d, u, v, w, T, tracers)
        out = [np.empty(self.shape) for _ in range(3)]
        check(self.lib.pu_dycore_perturbations(self.h, C.byref(view), out[0].ctypes.data, out[1].ctypes.data,
                                               out[2].ctypes.data, capi.PU_MEM_HOST))
        return tuple(out)

    def kernel_launches(self) -> int:
        return int(self.lib.pu_dycore_kernel_launches(self.h))

    # -- learned WENO weights -----------------------------------------------
    def learned_harvest(self, n, seed=0):
        check(self.lib.pu_dycore_learned_harvest(self.h, int(n), int(seed)))

    def learned_train(self, steps, batch=65536, lr=1e-3, seed=0):
        s = capi.pu_learn_stats()
        check(self.lib.pu_dycore_learned_train(self.h, int(steps), int(batch), float(lr), int(seed), C.byref(s)))
        return dict(loss_first=s.loss_first, loss_last=s.loss_last, steps=s.steps, samples=s.samples, ms=s.ms)

    def learned_get_weights(self):
        th = np.zeros(capi.PU_MLP_PARAMS, np.float32)
        check(self.lib.pu_dycore_learned_get_weights(self.h, th.ctypes.data))
        return th

    def learned_set_weights(self, theta):
        th = np.ascontiguousarray(theta, dtype=np.float32)
        assert th.size == capi.PU_MLP_PARAMS
        check(self.lib.pu_dycore_learned_set_weights(self.h, th.ctypes.data))

    def learned_eval(self, x, use_mma=True):
        x = np.ascontiguousarray(x, dtype=np.float32)
        n = x.shape[0]
        wl = np.zeros((n, 5), np.float32)
        wr = np.zeros((n, 5), np.float32)
        check(self.lib.pu_dycore_learned_eval(self.h, x.ctypes.data, n, wl.ctypes.data, wr.ctypes.data, int(use_mma)))
        return wl, wr

    def learned_gradient(self, x, t):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.zeros(capi.PU_MLP_PARAMS, np.float32)
        loss = C.c_double()
        check(self.lib.pu_dycore_learned_gradient(self.h, x.ctypes.data, t.ctypes.data, x.shape[0], g.ctypes.data,
                                                  C.byref(loss)))
        return g, loss.value

    def set_weno_mode(self, mode):
        check(self.lib.pu_dycore_set_weno_mode(self.h, {"plain": capi.PU_WENO_PLAIN,
                                                        "learned": capi.PU_WENO_LEARNED}[mode]))

    def learned_set_threshold(self, max_jump):
        check(self.lib.pu_dycore_learned_set_threshold(self.h, float(max_jump)))

    def learned_counts(self):
        """(stencils given learned weights, limiter fallbacks) since the last call."""
        a, b = C.c_longlong(), C.c_longlong()
        check(self.lib.pu_dycore_learned_counts(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def profile(self, enable=True):
        check(self.lib.pu_dycore_profile(self.h, int(enable)))

    def profile_read(self):
        """{kind: (total ms, launches)} for kinds 'xy', 'z', 'other'."""
        p = capi.pu_profile()
        check(self.lib.pu_dycore_profile_read(self.h, C.byref(p)))
        return {nm: (p.ms[q], int(p.launches[q])) for q, nm in enumerate(("xy", "z", "other"))}


# ---------------------------------------------------------------------------
# The reference's module convention.
# ---------------------------------------------------------------------------
class Coupler:
    """A single-rank coupler: grid, typed options, tracer registry and a data
    manager of named arrays (model/core/coupler.h, Options.h, DataManager.h)."""

    DIMS_3D = 3

    def __init__(self, device: Optional[str] = None):
        self.options: Dict[str, object] = {}
        self.tracers: List[tuple] = []
        self.dm: Dict[str, object] = {}
        self.device = device  # None: numpy host arrays; "cuda:N": torch device arrays
        self.nx = self.ny = self.nz = -1
        self.xlen = self.ylen = self.zlen = -1.0
        self.module_state: Dict[str, object] = {}
        # output / restart registry (coupler.h:474-531)
        self.file_counter = 0
        self.output_vars: List[tuple] = []
        self.write_output_modules: List = []
        self.restart_modules: List = []

    # grid (coupler.h:132-341, one rank)
    def distribute_mpi_and_allocate_coupled_state(self, nz, ny_glob, nx_glob):
        self.nx, self.ny, self.nz = int(nx_glob), int(ny_glob), int(nz)
        self.set_option("elapsed_time", 0.0)   # coupler.h:216

    def set_grid(self, xlen, ylen, zlen):
        self.xlen, self.ylen, self.zlen = float(xlen), float(ylen), float(zlen)

    def get_nx(self): return self.nx
    def get_ny(self): return self.ny
    def get_nz(self): return self.nz
    def get_dx(self): return self.xlen / self.nx
    def get_dy(self): return self.ylen / self.ny
    def get_dz(self): return self.zlen / self.nz
    def is_sim2d(self): return self.ny == 1

    # options (Options.h: a missing key or a wrong type is an error)
    def set_option(self, key, value):
        self.options[key] = value

    def add_option(self, key, value):
        self.options[key] = value

    def option_exists(self, key):
        return key in self.options

    _MISSING = object()

    def get_option(self, key, default=_MISSING, typ=None):
        if key not in self.options:
            if default is Coupler._MISSING:
                raise KeyError("ERROR: option [%s] does not exist" % key)
            return default
        v = self.options[key]
        if typ is not None and not isinstance(v, typ):
            raise TypeError("ERROR: option [%s] has type %s, not %s" % (key, type(v).__name__, typ.__name__))
        return v

    # tracers (coupler.h:417-471)
    def add_tracer(self, name, desc="", positive=True, adds_mass=False, diffuse=True):
        for t, tr in enumerate(self.tracers):
            if tr[0] == name:
                if (tr[2], tr[3], tr[4]) != (positive, adds_mass, diffuse):
                    raise ValueError("ERROR: adding tracer [%s] that already exists with different attributes" % name)
                return t
        self.tracers.append((name, desc, positive, adds_mass, diffuse))
        self.register_and_allocate(name, desc, (self.nz, self.ny, self.nx))
        return len(self.tracers) - 1

    def get_num_tracers(self): return len(self.tracers)
    def get_tracer_names(self): return [t[0] for t in self.tracers]

    def get_tracer_info(self, name):
        for t in self.tracers:
            if t[0] == name:
                return dict(desc=t[1], found=True, positive=t[2], adds_mass=t[3], diffuse=t[4])
        return dict(found=False)

    # output and restart (coupler.h:474-723; porturb_b200/output.py)
    def register_output_variable(self, name, dims, dtype=np.float64):
        self.output_vars.append((name, dims, dtype))

    def register_write_output_module(self, f):
        self.write_output_modules.append(f)

    def register_overwrite_with_restart_module(self, f):
        self.restart_modules.append(f)

    def write_output_file(self, prefix, verbose=False):
        from .output import write_output_file
        return write_output_file(self, prefix, verbose)

    def overwrite_with_restart(self):
        from .output import overwrite_with_restart
        overwrite_with_restart(self)

    # data manager (DataManager.h:127-299)
    def register_and_allocate(self, name, desc, dims, dtype=np.float64):
        if name in self.dm:
            raise ValueError("ERROR: entry [%s] already exists" % name)
        if self.device is None:
            self.dm[name] = np.zeros(dims, dtype=dtype)
        else:
            import torch
            tdt = {np.float64: torch.float64, np.float32: torch.float32, np.bool_: torch.bool}[dtype]
            self.dm[name] = torch.zeros(tuple(dims), dtype=tdt, device=self.device)

    def entry_exists(self, name): return name in self.dm

    def get(self, name):
        if name not in self.dm:
            raise KeyError("ERROR: entry [%s] does not exist" % name)
        return self.dm[name]


class _TracerSpec:
    def __init__(self, name, positive, adds_mass):
        self.name, self.positive, self.adds_mass = name, positive, adds_mass


class Dynamics_Euler_Stratified_WenoFV:
    """Drop-in for modules::Dynamics_Euler_Stratified_WenoFV at order 9
    (dynamics_rk.h:25-1355), running on one GPU through libpu_dycore."""

    ord = 9
    hs = (ord - 1) // 2
    num_state = 5
    idR, idU, idV, idW, idT = 0, 1, 2, 3, 4

    def __init__(self, precision="f32", device=0, stream=None, z_chunk=0):
        self.precision = precision
        self.device = device
        self.stream = stream
        self.z_chunk = z_chunk

    def _handle(self, coupler) -> Dycore:
        h = coupler.module_state.get("pu_dycore")
        if h is None:
            raise capi.PortUrbError(capi.PU_ERR_STATE, "init(coupler) has not been called")
        return h

    @staticmethod
    def _options(coupler):
        o = {}
        for key in ("R_d", "R_v", "cp_d", "gamma_d", "C0", "grav"):
            o[key] = coupler.get_option(key)  # missing thermodynamic options are an error
        o["idWV"] = coupler.get_option("idWV")
        o["cfl"] = coupler.get_option("cfl", 0.60)
        o["immersed_power"] = coupler.get_option("immersed_power", 5.0)
        o["latitude"] = coupler.get_option("latitude", 0.0)
        o["bc_x"] = coupler.get_option("bc_x", "periodic")
        o["bc_y"] = coupler.get_option("bc_y", "periodic")
        o["bc_z"] = coupler.get_option("bc_z", "solid_wall")
        o["enable_gravity"] = coupler.get_option("enable_gravity", True)
        o["weno_all"] = coupler.get_option("weno_all", True)
        if o["bc_z"] not in ("solid_wall", "periodic"):
            raise capi.PortUrbError(capi.PU_ERR_INVALID, "ERROR: Specified invalid bc_z in coupler options")
        return o

    def _state_arrays(self, coupler):
        return ([coupler.get(n) for n in ("density_dry", "uvel", "vvel", "wvel", "temp")],
                [coupler.get(n) for n in coupler.get_tracer_names()])

    def compute_time_step(self, coupler) -> float:
        """dynamics_rk.h:57-64."""
        cfl = coupler.get_option("cfl", 0.60)
        return cfl * min(min(coupler.get_dx(), coupler.get_dy()), coupler.get_dz()) / (350 + 100)

    def init(self, coupler):
        """dynamics_rk.h:917-1246."""
        opts = self._options(coupler)
        specs = []
        for name in coupler.get_tracer_names():
            info = coupler.get_tracer_info(name)
            specs.append(_TracerSpec(name, info["positive"], info["adds_mass"]))
        stream = self.stream
        if coupler.device is not None and stream is None:
            import torch
            stream = torch.cuda.current_stream(torch.device(coupler.device)).cuda_stream
        h = Dycore(coupler.nx, coupler.ny, coupler.nz, coupler.get_dx(), coupler.get_dy(), coupler.get_dz(),
                   specs, opts, precision=self.precision, device=self.device, stream=stream, z_chunk=self.z_chunk)
        (rd, u, v, w, T), trs = self._state_arrays(coupler)
        prop = coupler.get("immersed_proportion") if coupler.entry_exists("immersed_proportion") else None
        proj = coupler.get("windmill_proj_weight") if coupler.entry_exists("windmill_proj_weight") else None
        h.init(rd, u, v, w, T, trs, prop, proj)
        coupler.module_state["pu_dycore"] = h
        # The entries other modules read from the data manager (:951-956, :961-966, :1152-1154).
        dm = coupler.dm
        dm["tracer_positive"] = np.array([s.positive for s in specs], dtype=bool)
        dm["tracer_adds_mass"] = np.array([s.adds_mass for s in specs], dtype=bool)
        cells, edges = h.get_hydrostasis()
        for nm, a in zip(("hy_dens_cells", "hy_theta_cells", "hy_pressure_cells"), cells):
            dm[nm] = a.astype(np.float32)
        for nm, a in zip(("hy_dens_edges", "hy_theta_edges", "hy_pressure_edges"), edges):
            dm[nm] = a.astype(np.float32)
        # Output and restart hooks (dynamics_rk.h:1191-1242).
        from . import output
        if coupler.entry_exists("immersed_proportion"):
            coupler.register_output_variable("immersed_proportion", output.DIMS_3D)
        coupler.register_write_output_module(output.dycore_write_hook(self._handle))
        coupler.register_overwrite_with_restart_module(output.dycore_restart_hook(self._handle))

    def time_step(self, coupler, dt_phys) -> int:
        """dynamics_rk.h:103-137; returns the number of SSPRK3 cycles taken."""
        (rd, u, v, w, T), trs = self._state_arrays(coupler)
        return self._handle(coupler).time_step(rd, u, v, w, T, trs, dt_phys)

    def overwrite_with_restart(self, coupler, hy_dens_cells, hy_theta_cells, hy_pressure_cells):
        """The dycore's restart hook (dynamics_rk.h:1235-1242)."""
        self._handle(coupler).set_hydrostasis(hy_dens_cells, hy_theta_cells, hy_pressure_cells)


def case_coupler(case, device: Optional[str] = None) -> Coupler:
    """A coupler holding a case's base (unperturbed) state, as the reference's
    drivers build it before dycore.init (abl_neutral.cpp:49-65)."""
    c = Coupler(device=device)
    for k, v in case.options.items():
        c.set_option(k, v)
    c.distribute_mpi_and_allocate_coupled_state(case.nz, case.ny, case.nx)
    c.set_grid(case.xlen, case.ylen, case.zlen)
    for t in case.tracers:
        c.add_tracer(t.name, t.desc, t.positive, t.adds_mass, t.diffuse)
    c.set_option("idWV", c.get_tracer_names().index("water_vapor"))
    for nm in ("density_dry", "uvel", "vvel", "wvel", "temp", "immersed_proportion"):
        c.register_and_allocate(nm, "", (case.nz, case.ny, case.nx))
    assign_coupler_state(c, case, perturbed=False)
    _copy(c.get("immersed_proportion"), case.immersed_proportion)
    return c


def _copy(dst, src):
    if isinstance(dst, np.ndarray):
        dst[...] = src
    else:
        import torch
        dst.copy_(torch.as_tensor(np.ascontiguousarray(src)))


def assign_coupler_state(c: Coupler, case, perturbed=True):
    rd, u, v, w, T, trc = case.coupler_arrays(perturbed=perturbed)
    for nm, a in zip(("density_dry", "uvel", "vvel", "wvel", "temp"), (rd, u, v, w, T)):
        _copy(c.get(nm), a)
    # By name: tracers that modules registered beside the case's own (the LES
    # closure's TKE) keep what those modules set.
    for t, tr in enumerate(case.tracers):
        _copy(c.get(tr.name), trc[t])
