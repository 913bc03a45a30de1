"""ctypes front end of the physics-module oracles (TEST INFRASTRUCTURE ONLY).

``orc`` is this project's restatement (oracle/physics_oracle.cpp in
liboracle.so), ``ref`` the reference's own module headers compiled against
the single-rank shim (oracle/ref_physics.cpp in libporturb_ref.so); both
take the same configuration and update the coupler arrays in place.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

import pyoracle

MAX_TRACERS = 16


class PhysConfig(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("xlen", C.c_double), ("ylen", C.c_double), ("zlen", C.c_double),
                ("ntr", C.c_int),
                ("tracer_positive", C.c_int * MAX_TRACERS), ("tracer_adds_mass", C.c_int * MAX_TRACERS),
                ("tracer_diffuse", C.c_int * MAX_TRACERS),
                ("idWV", C.c_int), ("idTKE", C.c_int),
                ("R_d", C.c_double), ("R_v", C.c_double), ("cp_d", C.c_double), ("gamma_d", C.c_double),
                ("C0", C.c_double), ("grav", C.c_double), ("p0", C.c_double),
                ("enable_gravity", C.c_int), ("kinematic_viscosity", C.c_double), ("dns", C.c_int),
                ("les_total_mult", C.c_double), ("les_dissipation_mult", C.c_double),
                ("les_shear_prod_mult", C.c_double),
                ("bc_x", C.c_int), ("bc_y", C.c_int), ("bc_z", C.c_int)]


def make_config(case, nu=0.0, dns=False, total_mult=1.0, dissipation_mult=1.0, shear_prod_mult=1.0) -> PhysConfig:
    o = case.options
    c = PhysConfig()
    c.nx, c.ny, c.nz = case.nx, case.ny, case.nz
    c.xlen, c.ylen, c.zlen = case.xlen, case.ylen, case.zlen
    c.ntr = len(case.tracers)
    for t, tr in enumerate(case.tracers):
        c.tracer_positive[t] = int(tr.positive)
        c.tracer_adds_mass[t] = int(tr.adds_mass)
        c.tracer_diffuse[t] = int(tr.diffuse)
    names = [t.name for t in case.tracers]
    c.idWV = names.index("water_vapor")
    c.idTKE = names.index("TKE") if "TKE" in names else -1
    c.R_d, c.R_v, c.cp_d, c.gamma_d = o["R_d"], o["R_v"], o["cp_d"], o["gamma_d"]
    c.C0, c.grav, c.p0 = o["C0"], o["grav"], o["p0"]
    c.enable_gravity = int(o["enable_gravity"])
    c.kinematic_viscosity, c.dns = nu, int(dns)
    c.les_total_mult, c.les_dissipation_mult, c.les_shear_prod_mult = total_mult, dissipation_mult, shear_prod_mult
    c.bc_x, c.bc_y, c.bc_z = pyoracle.BC[o["bc_x"]], pyoracle.BC[o["bc_y"]], pyoracle.BC[o["bc_z"]]
    return c


_sigs = False


def _lib(kind):
    global _sigs
    path = pyoracle.ORACLE_SO if kind == "orc" else pyoracle.REF_SO
    lib = C.CDLL(path)
    P, D = C.c_void_p, C.c_double
    pre = kind + "_phys_"
    getattr(lib, pre + "create").restype = P
    getattr(lib, pre + "create").argtypes = [C.POINTER(PhysConfig), P, P, P]
    getattr(lib, pre + "destroy").argtypes = [P]
    arr = [P] * 7
    getattr(lib, pre + "les").argtypes = arr + [D]
    getattr(lib, pre + "sponge").argtypes = arr + [D, D, D]
    getattr(lib, pre + "geostrophic").argtypes = arr + [D, D, D, D]
    getattr(lib, pre + "surface_fluxes").argtypes = arr + [D]
    getattr(lib, pre + "uniform_pg").argtypes = arr + [D, D, C.c_ulonglong, P]
    getattr(lib, pre + "uniform_pg_height").argtypes = arr + [D, D, D, D, D]
    getattr(lib, pre + "time_average").argtypes = arr + [P, P, D, D]
    getattr(lib, pre + "edge_sponge_set_column").argtypes = arr + [P]
    getattr(lib, pre + "edge_sponge_apply").argtypes = arr + [P, D, D, D, D]
    for nm in ("les", "sponge", "geostrophic", "surface_fluxes", "uniform_pg", "uniform_pg_height", "time_average",
               "edge_sponge_set_column", "edge_sponge_apply"):
        getattr(lib, pre + nm).restype = C.c_int
    return lib


class Physics:
    """One configuration of the physics modules on the CPU (kind "orc" or
    "ref").  Each call takes a state dict of float64 arrays (rho_d, uvel,
    vvel, wvel, temp, tracers) and returns an updated copy."""

    def __init__(self, case, kind="orc", halos=None, **opts):
        self.kind = kind
        self.lib = _lib(kind)
        self.cfg = make_config(case, **opts)
        from porturb_b200 import cases
        self.halos = [np.ascontiguousarray(h) for h in (halos or cases.immersed_halos(case))]
        self.h = getattr(self.lib, kind + "_phys_create")(C.byref(self.cfg), *[h.ctypes.data for h in self.halos])
        if not self.h:
            raise RuntimeError("physics oracle creation failed")

    def close(self):
        if self.h:
            getattr(self.lib, self.kind + "_phys_destroy")(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _call(self, name, state, *extra):
        s = {k: np.array(v, dtype=np.float64, order="C", copy=True) for k, v in state.items()}
        ptrs = [s[k].ctypes.data for k in ("rho_d", "uvel", "vvel", "wvel", "temp", "tracers")]
        rc = getattr(self.lib, self.kind + "_phys_" + name)(self.h, *ptrs, *[float(e) for e in extra])
        if rc != 0:
            raise RuntimeError("%s_phys_%s failed" % (self.kind, name))
        return s

    def les(self, state, dt):
        return self._call("les", state, dt)

    def sponge(self, state, dt, time_scale, top_prop):
        return self._call("sponge", state, dt, time_scale, top_prop)

    def geostrophic(self, state, dt, lat_g, u_g, v_g):
        return self._call("geostrophic", state, dt, lat_g, u_g, v_g)

    def surface_fluxes(self, state, dt):
        return self._call("surface_fluxes", state, dt)

    def uniform_pg(self, state, dt, tau, update_cycles, st):
        """st: float64 array [counter, u0, v0, u, v], updated in place."""
        s = {k: np.array(v, dtype=np.float64, order="C", copy=True) for k, v in state.items()}
        ptrs = [s[k].ctypes.data for k in ("rho_d", "uvel", "vvel", "wvel", "temp", "tracers")]
        rc = getattr(self.lib, self.kind + "_phys_uniform_pg")(self.h, *ptrs, float(dt), float(tau), int(update_cycles),
                                                               st.ctypes.data)
        if rc != 0:
            raise RuntimeError("%s_phys_uniform_pg failed" % self.kind)
        return s

    def time_average(self, state, avgs, etime, elapsed_time, dt):
        """avgs: float64 (13, nz, ny, nx) in the order of capi.TAVG_NAMES,
        updated in place; returns the new etime."""
        s = {k: np.array(v, dtype=np.float64, order="C", copy=True) for k, v in state.items()}
        ptrs = [s[k].ctypes.data for k in ("rho_d", "uvel", "vvel", "wvel", "temp", "tracers")]
        et = np.array([float(etime)])
        rc = getattr(self.lib, self.kind + "_phys_time_average")(self.h, *ptrs, avgs.ctypes.data, et.ctypes.data,
                                                                 float(elapsed_time), float(dt))
        if rc != 0:
            raise RuntimeError("%s_phys_time_average failed" % self.kind)
        return float(et[0])

    def edge_sponge_set_column(self, state):
        """(5, nz) column profiles of density_dry, uvel, vvel, wvel, temp."""
        s = {k: np.array(v, dtype=np.float64, order="C", copy=True) for k, v in state.items()}
        ptrs = [s[k].ctypes.data for k in ("rho_d", "uvel", "vvel", "wvel", "temp", "tracers")]
        col = np.zeros((5, s["uvel"].shape[0]))
        if getattr(self.lib, self.kind + "_phys_edge_sponge_set_column")(self.h, *ptrs, col.ctypes.data) != 0:
            raise RuntimeError("%s_phys_edge_sponge_set_column failed" % self.kind)
        return col

    def edge_sponge_apply(self, state, column, px1, px2, py1, py2):
        s = {k: np.array(v, dtype=np.float64, order="C", copy=True) for k, v in state.items()}
        ptrs = [s[k].ctypes.data for k in ("rho_d", "uvel", "vvel", "wvel", "temp", "tracers")]
        col = np.ascontiguousarray(column, dtype=np.float64)
        rc = getattr(self.lib, self.kind + "_phys_edge_sponge_apply")(self.h, *ptrs, col.ctypes.data, float(px1),
                                                                      float(px2), float(py1), float(py2))
        if rc != 0:
            raise RuntimeError("%s_phys_edge_sponge_apply failed" % self.kind)
        return s

    def uniform_pg_height(self, state, dt, height, u0, v0, tau):
        return self._call("uniform_pg_height", state, dt, height, u0, v0, tau)


def state_of(case, seed=0, wind_noise=0.5, tke_noise=0.05):
    """Coupler state of a case with seeded velocity, temperature and TKE
    perturbations (so every derivative in the closure is exercised)."""
    rng = np.random.default_rng(seed)
    rd, u, v, w, T, trc = [np.array(a, dtype=np.float64) for a in case.coupler_arrays(perturbed=True)]
    shape = rd.shape
    u = u + wind_noise * rng.standard_normal(shape)
    v = v + wind_noise * rng.standard_normal(shape)
    w = w + 0.5 * wind_noise * rng.standard_normal(shape)
    T = T + 0.2 * rng.standard_normal(shape)
    trc = trc.copy()
    names = [t.name for t in case.tracers]
    if "TKE" in names:
        k = names.index("TKE")
        trc[k] = np.abs(trc[k] + tke_noise * rng.standard_normal(shape))
    wv = names.index("water_vapor")
    trc[wv] = np.abs(1e-3 * rng.standard_normal(shape))
    prop = np.asarray(case.immersed_proportion)
    u, v, w = (np.where(prop >= 1, 0.0, a) for a in (u, v, w))
    return dict(rho_d=rd, uvel=u, vvel=v, wvel=w, temp=T, tracers=trc)
