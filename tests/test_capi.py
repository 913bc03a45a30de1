"""The C-ABI library loads without a GPU, exports every function that
include/*.h declares, and rejects bad configurations on the host."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for hdr in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not hdr.endswith(".h"):
            continue
        txt = open(os.path.join(ROOT, "include", hdr)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names.update(re.findall(r"\b(pu_\w+)\s*\(", txt))
    return sorted(names)


def test_header_declares_the_entry_points():
    names = declared_functions()
    for required in ("pu_dycore_create", "pu_dycore_init", "pu_dycore_time_step", "pu_dycore_compute_time_step",
                     "pu_dycore_advance", "pu_dycore_destroy", "pu_last_error", "pu_physics_create",
                     "pu_les_apply", "pu_sponge_layer", "pu_geostrophic_forcing", "pu_surface_fluxes"):
        assert required in names


def test_library_exports_every_declared_symbol(gpu_lib):
    from porturb_b200 import capi
    lib = C.CDLL(capi.LIB_PATH)
    for name in declared_functions():
        assert hasattr(lib, name), name
        assert name in capi.SIGNATURES, name


def test_config_validation_on_host(gpu_lib):
    from porturb_b200 import capi
    lib = capi.load()
    h = C.c_void_p()
    assert lib.pu_dycore_create(None, C.byref(h)) == capi.PU_ERR_INVALID
    cfg = capi.pu_config(nx=16, ny=8, nz=12, dx=10.0, dy=10.0, dz=10.0, ntracers=1, idWV=0, R_d=287.0, R_v=461.0,
                         cp_d=1003.0, gamma_d=1.4, C0=27.0, grav=9.81, cfl=0.6, bc_x=0, bc_y=0, bc_z=7)
    assert lib.pu_dycore_create(C.byref(cfg), C.byref(h)) == capi.PU_ERR_INVALID
    assert b"bc_z" in lib.pu_last_error()
    cfg.bc_z = capi.PU_BC_WALL
    cfg.ntracers = 0
    assert lib.pu_dycore_create(C.byref(cfg), C.byref(h)) == capi.PU_ERR_UNSUPPORTED
    cfg.ntracers = 1
    cfg.idWV = 3
    assert lib.pu_dycore_create(C.byref(cfg), C.byref(h)) == capi.PU_ERR_INVALID
    assert lib.pu_version() >= 100
