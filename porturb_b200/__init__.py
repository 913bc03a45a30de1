"""B200-native dynamical core with the module API of portUrb's
Dynamics_Euler_Stratified_WenoFV (order-9 WENO finite volume, SSPRK3), and
the physics modules that run beside it in the boundary-layer drivers (LES
closure, sponge layer, geostrophic forcing, surface fluxes).

The compute path is libpu_dycore.so (porturb_b200/csrc, built by
porturb_b200/build.py); this package holds its ctypes bindings, the host-side
mirror of the reference's Coupler/module API and the workload generators.
"""
from . import capi, cases  # noqa: F401
from .capi import PortUrbError  # noqa: F401
from .dycore import (Coupler, Dycore, Dynamics_Euler_Stratified_WenoFV, assign_coupler_state,  # noqa: F401
                     case_coupler)
from .physics import (EdgeSponge, LES_Closure, Physics, Time_Averager, apply_surface_fluxes,  # noqa: F401
                      geostrophic_wind_forcing, sponge_layer, uniform_pg_wind_forcing,
                      uniform_pg_wind_forcing_height)

__version__ = "0.1.0"
