"""B200-native dynamical core with the module API of portUrb's
Dynamics_Euler_Stratified_WenoFV (order-9 WENO finite volume, SSPRK3).

The compute path is libpu_dycore.so (porturb_b200/csrc, built by
porturb_b200/build.py); this package holds its ctypes bindings, the host-side
mirror of the reference's Coupler/module API and the workload generators.
"""
from . import capi, cases  # noqa: F401
from .capi import PortUrbError  # noqa: F401
from .dycore import (Coupler, Dycore, Dynamics_Euler_Stratified_WenoFV, assign_coupler_state,  # noqa: F401
                     case_coupler)

__version__ = "0.1.0"
