"""Host-side mirror of the physics modules that the boundary-layer drivers
run beside the dycore every dt_phys (abl_neutral.cpp:93-104 of the
reference), on top of include/pu_physics.h:

* :class:`Physics` -- one pu_physics handle (options and immersed halo arrays
  held on the GPU) with ``les``, ``les_to``, ``sponge``, ``geostrophic``,
  ``surface_fluxes``, ``uniform_pg`` and ``uniform_pg_height`` on coupler
  arrays (numpy float64 or torch CUDA float64).
* The reference's module API on a :class:`~porturb_b200.dycore.Coupler`:
  :class:`LES_Closure` (``init`` adds the TKE tracer, ``apply``),
  :func:`sponge_layer`, :func:`geostrophic_wind_forcing`,
  :func:`apply_surface_fluxes`, :func:`uniform_pg_wind_forcing`,
  :func:`uniform_pg_wind_forcing_height`, :class:`Time_Averager` and
  :class:`EdgeSponge`, reading the options and the
  ``immersed_*_halos`` entries the drivers' init registers
  (sc_init.h:727-768).
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import capi
from .capi import check
from .dycore import _ptr, make_view

BC = {"periodic": capi.PU_BC_PERIODIC, "precursor": capi.PU_BC_PRECURSOR, "solid_wall": capi.PU_BC_WALL}


class Physics:
    """One pu_physics handle.

    tracers: sequence of (name, diffuse) in coupler order; the tracer named
    "TKE" is the closure's mass-weighted TKE.  halos: the three
    (nz+2, ny+2, nx+2) immersed halo arrays (proportion, roughness,
    temperature)."""

    def __init__(self, nx, ny, nz, dx, dy, dz, tracers: Sequence, options: dict, halos, device=0, stream=None):
        self.lib = capi.load()
        self.shape = (nz, ny, nx)
        cfg = capi.pu_physics_config()
        cfg.nx, cfg.ny, cfg.nz = nx, ny, nz
        cfg.dx, cfg.dy, cfg.dz = dx, dy, dz
        names = [t[0] for t in tracers]
        cfg.ntracers = len(tracers)
        for t, (_, diffuse) in enumerate(tracers):
            cfg.tracer_diffuse[t] = int(bool(diffuse))
        cfg.idTKE = names.index("TKE") if "TKE" in names else -1
        cfg.R_d, cfg.gamma_d, cfg.C0 = options["R_d"], options["gamma_d"], options["C0"]
        cfg.grav = options["grav"]
        cfg.enable_gravity = int(bool(options.get("enable_gravity", True)))
        cfg.kinematic_viscosity = float(options.get("kinematic_viscosity", 0.0))
        cfg.dns = int(bool(options.get("dns", False)))
        cfg.les_total_mult = float(options.get("les_total_mult", 1.0))
        cfg.les_dissipation_mult = float(options.get("les_dissipation_mult", 1.0))
        cfg.les_shear_prod_mult = float(options.get("les_shear_prod_mult", 1.0))
        cfg.bc_x = BC[options.get("bc_x", "periodic")]
        cfg.bc_y = BC[options.get("bc_y", "periodic")]
        cfg.bc_z = BC[options.get("bc_z", "solid_wall")]
        cfg.device = device
        cfg.stream = stream
        self.cfg = cfg
        self.ntr = len(tracers)
        hp = [_ptr(h) for h in halos]
        self._halos = halos
        h = C.c_void_p()
        check(self.lib.pu_physics_create(C.byref(cfg), hp[0][0], hp[1][0], hp[2][0], hp[0][1], C.byref(h)))
        self.h = h

    @classmethod
    def from_case(cls, case, halos=None, device=0, stream=None, **options):
        from . import cases as _cases
        opts = dict(case.options)
        opts.update(options)
        halos = halos if halos is not None else _cases.immersed_halos(case)
        return cls(case.nx, case.ny, case.nz, case.xlen / case.nx, case.ylen / case.ny, case.zlen / case.nz,
                   [(t.name, t.diffuse) for t in case.tracers], opts, halos, device=device, stream=stream)

    def close(self):
        if getattr(self, "h", None):
            self.lib.pu_physics_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def les(self, rho_d, u, v, w, T, tracers, dt):
        """LES_Closure::apply on the coupler arrays, in place."""
        view = make_view(rho_d, u, v, w, T, tracers)
        check(self.lib.pu_les_apply(self.h, C.byref(view), float(dt)))

    def les_to(self, state_in, state_out, dt):
        """The closure from one set of device arrays into another:
        state_* = (rho_d, u, v, w, T, tracers)."""
        vin = make_view(*state_in[:5], state_in[5])
        vout = make_view(*state_out[:5], state_out[5])
        check(self.lib.pu_les_apply_to(self.h, C.byref(vin), C.byref(vout), float(dt)))

    def sponge(self, rho_d, u, v, w, T, tracers, dt, time_scale, top_prop):
        view = make_view(rho_d, u, v, w, T, tracers)
        check(self.lib.pu_sponge_layer(self.h, C.byref(view), float(dt), float(time_scale), float(top_prop)))

    def geostrophic(self, rho_d, u, v, w, T, tracers, dt, lat_g, u_g, v_g):
        view = make_view(rho_d, u, v, w, T, tracers)
        check(self.lib.pu_geostrophic_forcing(self.h, C.byref(view), float(dt), float(lat_g), float(u_g), float(v_g)))

    def surface_fluxes(self, rho_d, u, v, w, T, tracers, dt):
        view = make_view(rho_d, u, v, w, T, tracers)
        check(self.lib.pu_surface_fluxes(self.h, C.byref(view), float(dt)))

    def uniform_pg(self, rho_d, u, v, w, T, tracers, dt, tau, update_cycles, state: capi.pu_uniform_pg_state):
        """uniform_pg_wind_forcing on coupler arrays; `state` (counter, u0, v0,
        u, v) is updated in place."""
        view = make_view(rho_d, u, v, w, T, tracers)
        check(self.lib.pu_uniform_pg_wind_forcing(self.h, C.byref(view), float(dt), float(tau), int(update_cycles),
                                                  C.byref(state)))

    def uniform_pg_height(self, rho_d, u, v, w, T, tracers, dt, height, u0, v0, tau):
        view = make_view(rho_d, u, v, w, T, tracers)
        check(self.lib.pu_uniform_pg_wind_forcing_height(self.h, C.byref(view), float(dt), float(height), float(u0),
                                                         float(v0), float(tau)))

    def time_average(self, rho_d, u, v, w, T, tracers, averages, etime, elapsed_time, dt) -> float:
        """Time_Averager.accumulate on coupler arrays: `averages` holds the 13
        arrays named in capi.TAVG_NAMES (dict or sequence), updated in place;
        returns the averager's new elapsed time (etime + dt)."""
        view = make_view(rho_d, u, v, w, T, tracers)
        a = capi.pu_time_averages()
        seq = [averages[n] for n in capi.TAVG_NAMES] if isinstance(averages, dict) else list(averages)
        for n, arr in zip(capi.TAVG_NAMES, seq):
            setattr(a, n, _ptr(arr)[0])
        a.etime = float(etime)
        check(self.lib.pu_time_averager_accumulate(self.h, C.byref(view), C.byref(a), float(elapsed_time),
                                                   float(dt)))
        return a.etime

    def edge_sponge_set_column(self, rho_d, u, v, w, T, tracers, fields=(0, 1, 2, 3, 4)) -> np.ndarray:
        """EdgeSponge.set_column: (len(fields), nz) horizontal means of the
        state-view fields (0..4 = density_dry, uvel, vvel, wvel, temp; 5+t
        tracer t)."""
        view = make_view(rho_d, u, v, w, T, tracers)
        idx = np.ascontiguousarray(fields, dtype=np.int32)
        col = np.zeros((len(idx), self.shape[0]))
        check(self.lib.pu_edge_sponge_set_column(self.h, C.byref(view), idx.ctypes.data, len(idx), col.ctypes.data))
        return col

    def edge_sponge(self, rho_d, u, v, w, T, tracers, column, prop_x1=0.1, prop_x2=0.1, prop_y1=0.1, prop_y2=0.1,
                    fields=(0, 1, 2, 3, 4)):
        """EdgeSponge.apply on one rank (the tile is the whole domain)."""
        view = make_view(rho_d, u, v, w, T, tracers)
        idx = np.ascontiguousarray(fields, dtype=np.int32)
        col = np.ascontiguousarray(column, dtype=np.float64)
        nz, ny, nx = self.shape
        check(self.lib.pu_edge_sponge_apply(self.h, C.byref(view), idx.ctypes.data, len(idx), col.ctypes.data,
                                            float(prop_x1), float(prop_x2), float(prop_y1), float(prop_y2), 0, 0,
                                            nx, ny))

    def synchronize(self):
        check(self.lib.pu_physics_synchronize(self.h))

    def last_les_ms(self) -> float:
        ms = C.c_double()
        check(self.lib.pu_physics_last_les_ms(self.h, C.byref(ms)))
        return ms.value


# ---------------------------------------------------------------------------
# The reference's module API on a Coupler.
# ---------------------------------------------------------------------------
_HALO_NAMES = ("immersed_proportion_halos", "immersed_roughness_halos", "immersed_temp_halos")


def _handle(coupler, need_halos=True) -> Physics:
    """The coupler's physics handle.  Modules that read no immersed arrays
    (the pressure-gradient forcings) get one with no immersed cells when the
    coupler has none registered; the others need the entries, as in the
    reference."""
    key = "pu_physics"
    if not need_halos and not all(coupler.entry_exists(n) for n in _HALO_NAMES):
        key = "pu_physics_no_immersed"
    h = coupler.module_state.get(key)
    if h is None:
        opts = {k: coupler.get_option(k) for k in ("R_d", "gamma_d", "C0", "grav")}
        for k, default in (("enable_gravity", True), ("kinematic_viscosity", 0.0), ("dns", False),
                           ("les_total_mult", 1.0), ("les_dissipation_mult", 1.0), ("les_shear_prod_mult", 1.0),
                           ("bc_x", "periodic"), ("bc_y", "periodic"), ("bc_z", "solid_wall")):
            opts[k] = coupler.get_option(k, default)
        if key == "pu_physics":
            halos = [coupler.get(n) for n in _HALO_NAMES]
        else:
            shape = (coupler.get_nz() + 2, coupler.get_ny() + 2, coupler.get_nx() + 2)
            halos = [np.zeros(shape) for _ in _HALO_NAMES]
        tracers = [(t[0], t[4]) for t in coupler.tracers]
        dev = 0
        if coupler.device is not None and ":" in str(coupler.device):
            dev = int(str(coupler.device).split(":")[1])
        h = Physics(coupler.get_nx(), coupler.get_ny(), coupler.get_nz(), coupler.get_dx(), coupler.get_dy(),
                    coupler.get_dz(), tracers, opts, halos, device=dev)
        coupler.module_state[key] = h
    return h


def _arrays(coupler):
    dm = coupler.get
    return (dm("density_dry"), dm("uvel"), dm("vvel"), dm("wvel"), dm("temp"),
            [dm(n) for n in coupler.get_tracer_names()])


class LES_Closure:
    """modules::LES_Closure (les_closure.h:9-320)."""

    def init(self, coupler):
        """Adds the mass-weighted TKE tracer and sets it to 0.1 (les_closure.h:19-26)."""
        coupler.add_tracer("TKE", "mass-weighted TKE", True, False, False)
        tke = coupler.get("TKE")
        tke[...] = 0.1

    def apply(self, coupler, dtphys):
        rd, u, v, w, T, trc = _arrays(coupler)
        _handle(coupler).les(rd, u, v, w, T, trc, dtphys)


def sponge_layer(coupler, dt, time_scale, top_prop):
    """modules::sponge_layer (sponge_layer.h:7-62)."""
    rd, u, v, w, T, trc = _arrays(coupler)
    _handle(coupler).sponge(rd, u, v, w, T, trc, dt, time_scale, top_prop)


def geostrophic_wind_forcing(coupler, dt, lat_g, u_g, v_g):
    """modules::geostrophic_wind_forcing (geostrophic_wind_forcing.h:7-42)."""
    rd, u, v, w, T, trc = _arrays(coupler)
    _handle(coupler).geostrophic(rd, u, v, w, T, trc, dt, lat_g, u_g, v_g)


def apply_surface_fluxes(coupler, dt):
    """modules::apply_surface_fluxes (surface_flux.h:9-125)."""
    rd, u, v, w, T, trc = _arrays(coupler)
    _handle(coupler).surface_fluxes(rd, u, v, w, T, trc, dt)


_PG = "uniform_pg_wind_forcing_"


def uniform_pg_wind_forcing(coupler, dt, tau=10.0, update_cycles=1):
    """modules::uniform_pg_wind_forcing (uniform_pg_wind_forcing.h:6-40):
    relaxes the domain-mean wind toward its value at the first call.  The
    state lives in the coupler options uniform_pg_wind_forcing_counter, _u0,
    _v0, _u, _v, as in the reference."""
    st = capi.pu_uniform_pg_state()
    st.counter = int(coupler.get_option(_PG + "counter", 0))
    if st.counter:
        st.u0, st.v0 = coupler.get_option(_PG + "u0"), coupler.get_option(_PG + "v0")
        st.u, st.v = coupler.get_option(_PG + "u"), coupler.get_option(_PG + "v")
    rd, u, v, w, T, trc = _arrays(coupler)
    _handle(coupler, need_halos=False).uniform_pg(rd, u, v, w, T, trc, dt, tau, update_cycles, st)
    for k in ("u0", "v0", "u", "v"):
        coupler.set_option(_PG + k, float(getattr(st, k)))
    coupler.set_option(_PG + "counter", int(st.counter))


def uniform_pg_wind_forcing_height(coupler, dt, height, u0, v0, tau=10.0):
    """modules::uniform_pg_wind_forcing_height (uniform_pg_wind_forcing.h:43-82):
    relaxes the mean wind at `height` toward (u0, v0)."""
    rd, u, v, w, T, trc = _arrays(coupler)
    _handle(coupler, need_halos=False).uniform_pg_height(rd, u, v, w, T, trc, dt, height, u0, v0, tau)


class Time_Averager:
    """custom_modules::Time_Averager (experiments/examples/custom_modules/
    time_averager.h:7-111): running averages of u, v, w, TKE and of the
    velocity covariances, kept in coupler arrays avg_* / long_avg_* and the
    option time_averager_etime."""

    def init(self, coupler):
        """time_averager.h:9-39."""
        from . import output
        coupler.set_option("time_averager_etime", 0.0)
        shape = (coupler.get_nz(), coupler.get_ny(), coupler.get_nx())
        for n in capi.TAVG_NAMES:
            coupler.register_and_allocate(n, "", shape)
            coupler.get(n)[...] = 0
            coupler.register_output_variable(n, output.DIMS_3D)

    def reset(self, coupler):
        """time_averager.h:42-54: the short averages restart; the long ones do not."""
        coupler.set_option("time_averager_etime", 0.0)
        for n in capi.TAVG_NAMES[:10]:
            coupler.get(n)[...] = 0

    def accumulate(self, coupler, dt):
        """time_averager.h:56-110."""
        rd, u, v, w, T, trc = _arrays(coupler)
        avgs = {n: coupler.get(n) for n in capi.TAVG_NAMES}
        etime = _handle(coupler, need_halos=False).time_average(
            rd, u, v, w, T, trc, avgs, coupler.get_option("time_averager_etime"),
            coupler.get_option("elapsed_time"), dt)
        coupler.set_option("time_averager_etime", etime)


_STATE_FIELDS = ("density_dry", "uvel", "vvel", "wvel", "temp")


class EdgeSponge:
    """custom_modules::EdgeSponge (experiments/examples/custom_modules/
    edge_sponge.h:8-101): set_column records the horizontal-mean profile of
    the named coupler fields; apply relaxes them toward it near the lateral
    edges of the domain."""

    def __init__(self):
        self.names = []
        self.column = None

    def _fields(self, coupler):
        trc = list(coupler.get_tracer_names())
        return [(_STATE_FIELDS.index(n) if n in _STATE_FIELDS else 5 + trc.index(n)) for n in self.names]

    def set_column(self, coupler, names_in=_STATE_FIELDS):
        """edge_sponge.h:14-28."""
        self.names = list(names_in)
        rd, u, v, w, T, trc = _arrays(coupler)
        self.column = _handle(coupler, need_halos=False).edge_sponge_set_column(rd, u, v, w, T, trc,
                                                                                self._fields(coupler))

    def apply(self, coupler, prop_x1=0.1, prop_x2=0.1, prop_y1=0.1, prop_y2=0.1):
        """edge_sponge.h:31-72."""
        rd, u, v, w, T, trc = _arrays(coupler)
        _handle(coupler, need_halos=False).edge_sponge(rd, u, v, w, T, trc, self.column, prop_x1, prop_x2, prop_y1,
                                                       prop_y2, self._fields(coupler))


def register_immersed_halos(coupler, case, **kw):
    """Registers the immersed_*_halos entries the way the drivers' init does
    (see porturb_b200.cases.immersed_halos)."""
    from . import cases as _cases
    names = ("immersed_proportion_halos", "immersed_roughness_halos", "immersed_temp_halos")
    for name, arr in zip(names, _cases.immersed_halos(case, **kw)):
        coupler.register_and_allocate(name, "", arr.shape)
        dst = coupler.get(name)
        if isinstance(dst, np.ndarray):
            dst[...] = arr
        else:
            import torch
            dst.copy_(torch.from_numpy(arr))
