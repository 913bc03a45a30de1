"""Initial states for the dycore workloads, built on the host with numpy.

Each builder returns a :class:`Case`: the coupler-side arrays the reference's
drivers hand to ``Dynamics_Euler_Stratified_WenoFV::init`` and ``time_step``
(``density_dry``, ``uvel``, ``vvel``, ``wvel``, ``temp``, tracers and
``immersed_proportion``; C-order ``(nz, ny, nx)`` doubles), together with the
grid, tracer registry and options.

Thermodynamic constants and derived options follow the reference's
``sc_init`` (experiments/examples/custom_modules/sc_init.h:31-51).  The
hydrostatic state is evaluated at cell centres as the reference's closed-form
isentropic column does (sc_init.h:580-607).  Perturbations are applied to
potential temperature at fixed pressure *after* the dycore's ``init`` has
taken the horizontal-mean profiles, the order the reference's drivers use
(abl_neutral.cpp:61-65: ``sc_init``, ``dycore.init``, then ``sc_perturb``).

Random fields use a counter-based generator (splitmix64 of the seed and the
global cell index ``k*ny*nx + j*nx + i``), keyed like the reference's
``yakl::Random(k*ny_glob*nx_glob + j*nx_glob + i)`` (sc_perturb.h:74-79).
YAKL's generator itself is not available, so the noise is not bit-identical to
the reference's; parity is defined on identical input arrays.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Dict, List, Optional

import numpy as np

R_D = 287.0
CP_D = 1003.0
R_V = 461.0
CP_V = 1859.0
P0 = 1.0e5
GRAV = 9.81


def thermo_options(R_d=R_D, cp_d=CP_D, R_v=R_V, p0=P0, grav=GRAV) -> Dict[str, float]:
    """Options set by sc_init.h:31-51."""
    cv_d = cp_d - R_d
    gamma = cp_d / cv_d
    kappa = R_d / cp_d
    C0 = math.pow(R_d * math.pow(p0, -kappa), gamma)
    return dict(R_d=R_d, cp_d=cp_d, R_v=R_v, cv_d=cv_d, gamma_d=gamma, kappa_d=kappa, C0=C0, p0=p0, grav=grav)


@dataclasses.dataclass
class Tracer:
    name: str
    desc: str = ""
    positive: bool = True
    adds_mass: bool = False
    diffuse: bool = True


@dataclasses.dataclass
class Case:
    name: str
    nx: int
    ny: int
    nz: int
    xlen: float
    ylen: float
    zlen: float
    options: Dict[str, object]
    tracers: List[Tracer]
    rho_d: np.ndarray
    uvel: np.ndarray
    vvel: np.ndarray
    wvel: np.ndarray
    temp: np.ndarray
    tracer_data: np.ndarray          # (ntr, nz, ny, nx)
    immersed_proportion: np.ndarray
    # Perturbation applied after init: (rho_d, temp) replacements, or None.
    perturbed: Optional[Dict[str, np.ndarray]] = None
    steps: int = 1

    @property
    def ncells(self) -> int:
        return self.nx * self.ny * self.nz

    def coupler_arrays(self, perturbed: bool = True):
        """(rho_d, u, v, w, T, tracers) as the coupler holds them."""
        rd, T = self.rho_d, self.temp
        if perturbed and self.perturbed is not None:
            rd, T = self.perturbed["rho_d"], self.perturbed["temp"]
        return rd, self.uvel, self.vvel, self.wvel, T, self.tracer_data

    def block(self, i0: int, j0: int, nx: int, ny: int) -> "Case":
        """The columns [i0, i0+nx) x [j0, j0+ny) of this case as a case of its
        own (copies; same spacing, levels and options; its lateral boundaries
        are whatever the options say, periodic for the generators here)."""
        xs, ys = slice(i0, i0 + nx), slice(j0, j0 + ny)
        cut = lambda a: np.ascontiguousarray(a[..., ys, xs])
        pert = None if self.perturbed is None else {k: cut(v) for k, v in self.perturbed.items()}
        return Case(name="%s_block" % self.name, nx=nx, ny=ny, nz=self.nz, xlen=self.xlen * nx / self.nx,
                    ylen=self.ylen * ny / self.ny, zlen=self.zlen, options=dict(self.options),
                    tracers=list(self.tracers), rho_d=cut(self.rho_d), uvel=cut(self.uvel), vvel=cut(self.vvel),
                    wvel=cut(self.wvel), temp=cut(self.temp), tracer_data=cut(self.tracer_data),
                    immersed_proportion=cut(self.immersed_proportion), perturbed=pert, steps=self.steps)


def splitmix64_uniform(seed: int, index: np.ndarray) -> np.ndarray:
    """Uniform [0,1) doubles from splitmix64(seed * 2^32 + index)."""
    with np.errstate(over="ignore"):
        z = (np.uint64(seed) << np.uint64(32)) + index.astype(np.uint64) + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def _exner_column(zc: np.ndarray, theta_of_z, opts) -> np.ndarray:
    """Hydrostatic Exner function pi=(p/p0)^(R_d/cp_d) at heights zc for a
    theta profile, from d(pi)/dz = -g/(cp_d*theta), integrated with a fine
    composite Simpson rule from the surface (p = p0)."""
    cp, g = opts["cp_d"], opts["grav"]
    pis = np.empty_like(zc)
    for idx, z in enumerate(zc):
        n = max(64, int(z / 0.5) * 2)
        zz = np.linspace(0.0, z, n + 1)
        f = 1.0 / theta_of_z(zz)
        h = z / n
        integral = h / 3.0 * (f[0] + f[-1] + 4.0 * f[1:-1:2].sum() + 2.0 * f[2:-1:2].sum()) if z > 0 else 0.0
        pis[idx] = 1.0 - g / cp * integral
    return pis


def _state_from_theta_p(theta, p, opts):
    """(rho, T) for dry air from potential temperature and pressure,
    using p = C0*(rho*theta)^gamma (dynamics_rk.h:1338-1341)."""
    rt = np.power(p / opts["C0"], 1.0 / opts["gamma_d"])
    rho = rt / theta
    T = p / (opts["R_d"] * rho)
    return rho, T


def _base(name, nx, ny, nz, xlen, ylen, zlen, tracers, opts):
    shape = (nz, ny, nx)
    ntr = len(tracers)
    return dict(name=name, nx=nx, ny=ny, nz=nz, xlen=xlen, ylen=ylen, zlen=zlen, options=opts, tracers=tracers,
                uvel=np.zeros(shape), vvel=np.zeros(shape), wvel=np.zeros(shape),
                tracer_data=np.zeros((ntr,) + shape), immersed_proportion=np.zeros(shape))


def default_options(**kw):
    opts = thermo_options()
    opts.update(dict(cfl=0.6, immersed_power=5.0, latitude=0.0, enable_gravity=True, weno_all=True,
                     bc_x="periodic", bc_y="periodic", bc_z="solid_wall"))
    opts.update(kw)
    return opts


def warm_bubble(nx=256, ny=4, nz=128, xlen=20000.0, ylen=312.5, zlen=10000.0, theta0=300.0, amp=3.0,
                radius=2000.0, x0=10000.0, z0=2000.0, cfl=0.8, steps=200, with_vapor_noise=False) -> Case:
    """Dry warm bubble: constant-theta isentropic column with p_s = 1e5 Pa
    (closed form of sc_init.h:586-591), no wind, a water_vapor tracer that is
    zero, and a +3 K cos^2 theta bubble of radius 2 km centred at
    (x, z) = (10 km, 2 km), evaluated at cell centres and applied at fixed
    pressure after init."""
    opts = default_options(cfl=cfl)
    tr = [Tracer("water_vapor", "water_vapor", True, True, True)]
    b = _base("warm_bubble", nx, ny, nz, xlen, ylen, zlen, tr, opts)
    dz = zlen / nz
    R_d, cp_d, p0, g = opts["R_d"], opts["cp_d"], opts["p0"], opts["grav"]
    slope = -g * p0 ** (R_d / cp_d) / (cp_d * theta0)
    press = np.empty(nz)
    press[0] = p0 ** (R_d / cp_d) + slope * dz / 2
    for k in range(1, nz):
        press[k] = press[k - 1] + slope * dz
    press = press ** (cp_d / R_d)
    p3 = np.broadcast_to(press[:, None, None], (nz, ny, nx)).copy()
    theta = np.full((nz, ny, nx), theta0)
    rho, T = _state_from_theta_p(theta, p3, opts)
    xc = (np.arange(nx) + 0.5) * (xlen / nx)
    zc = (np.arange(nz) + 0.5) * dz
    rad = np.sqrt(((xc[None, :] - x0) / radius) ** 2 + ((zc[:, None] - z0) / radius) ** 2)
    dth = np.where(rad <= 1.0, amp * np.cos(np.pi * rad / 2.0) ** 2, 0.0)
    theta_p = theta + dth[:, None, :]
    rho_p, T_p = _state_from_theta_p(theta_p, p3, opts)
    return Case(rho_d=rho, temp=T, perturbed=dict(rho_d=rho_p, temp=T_p), steps=steps, **b)


def abl_neutral(nx=256, ny=256, nz=128, dx=10.0, theta0=300.0, z_inv=500.0, lapse=0.01, u_g=10.0,
                noise_amp=0.25, noise_top=400.0, seed=0, cfl=0.6, steps=500, tke0=0.1) -> Case:
    """Neutral boundary layer: theta = 300 K below 500 m with a 0.01 K/m
    inversion above, uniform (u_g, 0) wind, seeded +-0.25 K theta noise in the
    lowest 400 m applied after init, tracers water_vapor (zero) and TKE
    (mass-weighted, 0.1, les_closure.h:24-25)."""
    opts = default_options(cfl=cfl)
    tr = [Tracer("water_vapor", "water_vapor", True, True, True), Tracer("TKE", "mass-weighted TKE", True, False, False)]
    b = _base("abl_neutral", nx, ny, nz, nx * dx, ny * dx, nz * dx, tr, opts)
    zc = (np.arange(nz) + 0.5) * dx

    def theta_of_z(z):
        return np.where(z < z_inv, theta0, theta0 + lapse * (z - z_inv))

    pi = _exner_column(zc, theta_of_z, opts)
    press = opts["p0"] * pi ** (opts["cp_d"] / opts["R_d"])
    shape = (nz, ny, nx)
    p3 = np.broadcast_to(press[:, None, None], shape).copy()
    th = np.broadcast_to(theta_of_z(zc)[:, None, None], shape).copy()
    rho, T = _state_from_theta_p(th, p3, opts)
    b["uvel"][...] = u_g
    b["tracer_data"][1] = tke0
    idx = np.arange(nz * ny * nx, dtype=np.uint64).reshape(shape)
    noise = (splitmix64_uniform(seed, idx) * 2.0 - 1.0) * noise_amp
    noise = np.where((zc <= noise_top)[:, None, None], noise, 0.0)
    rho_p, T_p = _state_from_theta_p(th + noise, p3, opts)
    return Case(rho_d=rho, temp=T, perturbed=dict(rho_d=rho_p, temp=T_p), steps=steps, **b)


def urban_canopy(nx=512, ny=512, nz=128, dx=2.0, theta0=300.0, lot=40.0, foot=(20.0, 32.0), height=(10.0, 60.0),
                 occupancy=0.7, noise_amp=0.1, seed=0, cfl=0.6, steps=1000, u0=10.0, window=None,
                 layout_seed=None) -> Case:
    """Immersed-boundary urban canopy: seeded cuboid buildings, one per
    occupied 40 m lot, footprints U[20,32] m, heights U[10,60] m, 70 % lot
    occupancy, a binary immersed mask, theta = 300 K with seeded +-0.1 K noise
    applied after init, and a uniform 10 m/s initial flow outside buildings.

    window = (i0, j0, bx, by) gives only the columns [i0, i0+bx) x [j0, j0+by)
    of the nx x ny domain, as a case of its own (the same buildings and noise,
    which are keyed by lot and by global cell index), without forming the rest.
    The noise is keyed by `seed`, the buildings by `layout_seed` (seed + 1 by
    default): ensemble members share a city with layout_seed fixed."""
    i0, j0, bx, by = window if window is not None else (0, 0, nx, ny)
    if not (0 <= i0 and i0 + bx <= nx and 0 <= j0 and j0 + by <= ny and bx > 0 and by > 0):
        raise ValueError("window outside the domain")
    opts = default_options(cfl=cfl)
    tr = [Tracer("water_vapor", "water_vapor", True, True, True)]
    b = _base("urban_canopy", bx, by, nz, bx * dx, by * dx, nz * dx, tr, opts)
    xlen, ylen = nx * dx, ny * dx
    nlx, nly = int(xlen // lot), int(ylen // lot)
    rng_idx = np.arange(nlx * nly * 5, dtype=np.uint64)
    r = splitmix64_uniform(seed + 1 if layout_seed is None else layout_seed, rng_idx).reshape(nly, nlx, 5)
    xc = (np.arange(i0, i0 + bx) + 0.5) * dx
    yc = (np.arange(j0, j0 + by) + 0.5) * dx
    zc = (np.arange(nz) + 0.5) * dx
    mask = np.zeros((nz, by, bx))
    for jl in range(nly):
        for il in range(nlx):
            occ, fx, fy, h, _ = r[jl, il]
            if occ >= occupancy:
                continue
            wx = foot[0] + fx * (foot[1] - foot[0])
            wy = foot[0] + fy * (foot[1] - foot[0])
            hh = height[0] + h * (height[1] - height[0])
            cx, cy = (il + 0.5) * lot, (jl + 0.5) * lot
            inx = np.abs(xc - cx) <= wx / 2
            iny = np.abs(yc - cy) <= wy / 2
            if not (inx.any() and iny.any()):
                continue
            inz = zc <= hh
            mask[np.ix_(inz, iny, inx)] = 1.0
    b["immersed_proportion"][...] = mask
    shape = (nz, by, bx)
    pi = _exner_column(zc, lambda z: np.full_like(z, theta0), opts)
    press = opts["p0"] * pi ** (opts["cp_d"] / opts["R_d"])
    p3 = np.broadcast_to(press[:, None, None], shape).copy()
    th = np.full(shape, theta0)
    rho, T = _state_from_theta_p(th, p3, opts)
    b["uvel"][...] = np.where(mask > 0, 0.0, u0)
    k = np.arange(nz, dtype=np.uint64)[:, None, None]
    j = np.arange(j0, j0 + by, dtype=np.uint64)[None, :, None]
    i = np.arange(i0, i0 + bx, dtype=np.uint64)[None, None, :]
    idx = (k * np.uint64(ny) + j) * np.uint64(nx) + i
    noise = (splitmix64_uniform(seed, idx) * 2.0 - 1.0) * noise_amp
    rho_p, T_p = _state_from_theta_p(th + noise, p3, opts)
    return Case(rho_d=rho, temp=T, perturbed=dict(rho_d=rho_p, temp=T_p), steps=steps, **b)


def small_mixed(nx=16, ny=8, nz=12, dx=100.0, seed=3, immersed=True, ntr=2, bc_x="periodic", bc_y="periodic",
                bc_z="solid_wall", latitude=0.0, weno_all=True) -> Case:
    """A small grid that exercises every branch of the operator: a stratified
    column, random wind and theta perturbations, two tracers (one adds mass),
    an immersed cuboid touching the floor and a partially immersed cell."""
    opts = default_options(cfl=0.5, bc_x=bc_x, bc_y=bc_y, bc_z=bc_z, latitude=latitude, weno_all=weno_all)
    tr = [Tracer("water_vapor", "water_vapor", True, True, True)]
    for t in range(1, ntr):
        tr.append(Tracer("tracer_%d" % t, "", t % 2 == 1, False, True))
    b = _base("small_mixed", nx, ny, nz, nx * dx, ny * dx, nz * dx, tr, opts)
    shape = (nz, ny, nx)
    zc = (np.arange(nz) + 0.5) * dx

    def theta_of_z(z):
        return 300.0 + 0.003 * z

    pi = _exner_column(zc, theta_of_z, opts)
    press = opts["p0"] * pi ** (opts["cp_d"] / opts["R_d"])
    p3 = np.broadcast_to(press[:, None, None], shape).copy()
    th = np.broadcast_to(theta_of_z(zc)[:, None, None], shape).copy()
    idx = np.arange(nz * ny * nx, dtype=np.uint64).reshape(shape)
    u = lambda s: splitmix64_uniform(seed + s, idx) * 2.0 - 1.0
    rho, T = _state_from_theta_p(th, p3, opts)
    b["uvel"][...] = 5.0 + 2.0 * u(1)
    b["vvel"][...] = -3.0 + 2.0 * u(2) if ny > 1 else 0.0
    b["wvel"][...] = 0.5 * u(3)
    b["tracer_data"][0] = 1e-3 * (1.0 + u(4)) * rho
    for t in range(1, ntr):
        b["tracer_data"][t] = 0.1 + 0.05 * u(4 + t)
    if immersed:
        m = np.zeros(shape)
        m[: nz // 3, ny // 4: ny // 4 + max(1, ny // 3), nx // 4: nx // 4 + max(1, nx // 4)] = 1.0
        m[nz // 2, ny // 2, (3 * nx) // 4] = 0.5
        b["immersed_proportion"][...] = m
    rho_p, T_p = _state_from_theta_p(th + 0.5 * u(9), p3, opts)
    return Case(rho_d=rho, temp=T, perturbed=dict(rho_d=rho_p, temp=T_p), steps=3, **b)


CONFIGS = {
    "warm_bubble": warm_bubble,
    "abl_neutral": abl_neutral,
    "urban_canopy": urban_canopy,
}


def immersed_halos(case: Case, roughness: float = 0.1, surface_temp: float = 0.0, immersed_temp: float = 0.0):
    """The one-cell-halo immersed arrays that the physics modules read
    (immersed_proportion_halos, immersed_roughness_halos,
    immersed_temp_halos), built as the drivers' init does (sc_init.h:52-89,
    727-768): interior proportion from the case, roughness everywhere
    `roughness`, immersed temperature `immersed_temp`; periodic x/y halos
    (corners wrap in both); the bottom z halo is the ground (proportion 1,
    surface roughness, surface temperature), the top z halo is empty.
    Returns three (nz+2, ny+2, nx+2) arrays."""
    nz, ny, nx = case.nz, case.ny, case.nx
    interior = [np.asarray(case.immersed_proportion, dtype=np.float64), np.full((nz, ny, nx), roughness),
                np.full((nz, ny, nx), immersed_temp)]
    bottom = [1.0, roughness, surface_temp]
    out = []
    for a, b in zip(interior, bottom):
        h = np.zeros((nz + 2, ny + 2, nx + 2))
        h[1:-1] = np.pad(a, ((0, 0), (1, 1), (1, 1)), mode="wrap")
        h[0] = b
        h[-1] = 0.0
        out.append(np.ascontiguousarray(h))
    return tuple(out)
