"""ctypes bindings of libpu_dycore (include/pu_dycore.h).

The library is built in-tree by porturb_b200/build.py.  There is no fallback:
if the library is missing or no GPU is present the calls fail loudly.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libpu_dycore.so")

PU_MAX_TRACERS = 4
PU_HS = 4
(PU_OK, PU_ERR_INVALID, PU_ERR_CUDA, PU_ERR_NONFINITE, PU_ERR_STATE, PU_ERR_NOMEM, PU_ERR_UNSUPPORTED,
 PU_ERR_TRANSPORT) = range(8)
PU_BC_PERIODIC, PU_BC_PRECURSOR, PU_BC_WALL = 0, 1, 2
PU_F32, PU_F64 = 0, 1
PU_WENO_PLAIN, PU_WENO_LEARNED = 0, 1
PU_MEM_HOST, PU_MEM_DEVICE = 0, 1
BC_NAMES = {"periodic": PU_BC_PERIODIC, "precursor": PU_BC_PRECURSOR, "solid_wall": PU_BC_WALL}

STATUS_NAMES = {0: "PU_OK", 1: "PU_ERR_INVALID", 2: "PU_ERR_CUDA", 3: "PU_ERR_NONFINITE", 4: "PU_ERR_STATE",
                5: "PU_ERR_NOMEM", 6: "PU_ERR_UNSUPPORTED", 7: "PU_ERR_TRANSPORT"}


class PortUrbError(RuntimeError):
    """A pu_dycore call returned an error status."""

    def __init__(self, status: int, message: str):
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, status), message))
        self.status = status


class pu_config(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("ntracers", C.c_int),
                ("tracer_positive", C.c_int * PU_MAX_TRACERS), ("tracer_adds_mass", C.c_int * PU_MAX_TRACERS),
                ("idWV", C.c_int),
                ("R_d", C.c_double), ("R_v", C.c_double), ("cp_d", C.c_double), ("gamma_d", C.c_double),
                ("C0", C.c_double), ("grav", C.c_double),
                ("cfl", C.c_double), ("immersed_power", C.c_double), ("latitude", C.c_double),
                ("bc_x", C.c_int), ("bc_y", C.c_int), ("bc_z", C.c_int),
                ("enable_gravity", C.c_int), ("weno_all", C.c_int),
                ("precision", C.c_int), ("weno_mode", C.c_int), ("device", C.c_int),
                ("stream", C.c_void_p), ("z_chunk", C.c_int), ("thread_loads", C.c_int),
                ("imm_all_levels", C.c_int),
                ("serial_io", C.c_int)]


class pu_state_view(C.Structure):
    _fields_ = [("rho_d", C.c_void_p), ("uvel", C.c_void_p), ("vvel", C.c_void_p), ("wvel", C.c_void_p),
                ("temp", C.c_void_p), ("tracers", C.c_void_p * PU_MAX_TRACERS), ("mem", C.c_int)]


class pu_diag(C.Structure):
    _fields_ = [("mass", C.c_double), ("rho_theta", C.c_double), ("kinetic", C.c_double),
                ("internal", C.c_double), ("potential", C.c_double), ("total_energy", C.c_double),
                ("tracer_mass", C.c_double * PU_MAX_TRACERS)]


# pu_host_transport callbacks (include/pu_dycore.h)
EXCHANGE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_size_t),
                          C.POINTER(C.c_int))
ALLREDUCE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_double), C.c_size_t)
ALLGATHER_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t)


class pu_host_transport(C.Structure):
    _fields_ = [("exchange", EXCHANGE_FN), ("allreduce_sum_f64", ALLREDUCE_FN), ("allgather", ALLGATHER_FN),
                ("user", C.c_void_p)]


PU_MLP_PARAMS = 1541


class pu_learn_stats(C.Structure):
    _fields_ = [("loss_first", C.c_double), ("loss_last", C.c_double), ("steps", C.c_longlong),
                ("samples", C.c_longlong), ("ms", C.c_double)]


PU_PROFILE_KINDS = 3


class pu_physics_config(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("ntracers", C.c_int), ("tracer_diffuse", C.c_int * PU_MAX_TRACERS), ("idTKE", C.c_int),
                ("R_d", C.c_double), ("gamma_d", C.c_double), ("C0", C.c_double), ("grav", C.c_double),
                ("enable_gravity", C.c_int), ("kinematic_viscosity", C.c_double), ("dns", C.c_int),
                ("les_total_mult", C.c_double), ("les_dissipation_mult", C.c_double),
                ("les_shear_prod_mult", C.c_double),
                ("bc_x", C.c_int), ("bc_y", C.c_int), ("bc_z", C.c_int),
                ("device", C.c_int), ("stream", C.c_void_p)]


class pu_decomp(C.Structure):
    _fields_ = [("nproc_x", C.c_int), ("nproc_y", C.c_int), ("px", C.c_int), ("py", C.c_int),
                ("nx_glob", C.c_longlong), ("ny_glob", C.c_longlong)]


PU_NCCL_ID_BYTES = 128


class pu_uniform_pg_state(C.Structure):
    _fields_ = [("counter", C.c_ulonglong), ("u0", C.c_double), ("v0", C.c_double),
                ("u", C.c_double), ("v", C.c_double)]


TAVG_NAMES = ("avg_u", "avg_v", "avg_w", "avg_tke", "avg_up_up", "avg_up_vp", "avg_up_wp", "avg_vp_vp", "avg_vp_wp",
              "avg_wp_wp", "long_avg_u", "long_avg_v", "long_avg_w")


class pu_time_averages(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in TAVG_NAMES] + [("etime", C.c_double)]


class pu_profile(C.Structure):
    _fields_ = [("ms", C.c_double * PU_PROFILE_KINDS), ("launches", C.c_longlong * PU_PROFILE_KINDS)]


# Every function declared in include/pu_dycore.h with its ctypes signature.
_P = C.c_void_p
_D = C.c_double
_I = C.c_int
SIGNATURES = {
    "pu_version": (_I, []),
    "pu_last_error": (C.c_char_p, []),
    "pu_dycore_create": (_I, [C.POINTER(pu_config), C.POINTER(C.c_void_p)]),
    "pu_dycore_destroy": (_I, [_P]),
    "pu_dycore_init": (_I, [_P, C.POINTER(pu_state_view), _P, _I]),
    "pu_dycore_init_windmill": (_I, [_P, C.POINTER(pu_state_view), _P, _P, _I]),
    "pu_dycore_compute_time_step": (_I, [_P, C.POINTER(_D)]),
    "pu_dycore_time_step": (_I, [_P, C.POINTER(pu_state_view), _D, C.POINTER(_I)]),
    "pu_dycore_load_state": (_I, [_P, C.POINTER(pu_state_view)]),
    "pu_dycore_store_state": (_I, [_P, C.POINTER(pu_state_view)]),
    "pu_dycore_advance": (_I, [_P, _D, _I]),
    "pu_dycore_get_conserved": (_I, [_P, _P, _P, _I]),
    "pu_dycore_set_conserved": (_I, [_P, _P, _P, _I]),
    "pu_dycore_get_hydrostasis": (_I, [_P, _P, _P, _P, _P, _P, _P]),
    "pu_dycore_set_hydrostasis": (_I, [_P, _P, _P, _P]),
    "pu_dycore_diagnostics": (_I, [_P, C.POINTER(pu_diag)]),
    "pu_dycore_synchronize": (_I, [_P]),
    "pu_dycore_perturbations": (_I, [_P, C.POINTER(pu_state_view), _P, _P, _P, _I]),
    "pu_dycore_kernel_launches": (C.c_longlong, [_P]),
    "pu_dycore_learned_harvest": (_I, [_P, C.c_longlong, C.c_ulonglong]),
    "pu_dycore_learned_train": (_I, [_P, _I, _I, _D, C.c_ulonglong, C.POINTER(pu_learn_stats)]),
    "pu_dycore_learned_get_weights": (_I, [_P, _P]),
    "pu_dycore_learned_set_weights": (_I, [_P, _P]),
    "pu_dycore_learned_eval": (_I, [_P, _P, C.c_longlong, _P, _P, _I]),
    "pu_dycore_learned_gradient": (_I, [_P, _P, _P, C.c_longlong, _P, C.POINTER(_D)]),
    "pu_dycore_set_weno_mode": (_I, [_P, _I]),
    "pu_dycore_learned_set_threshold": (_I, [_P, _D]),
    "pu_dycore_learned_counts": (_I, [_P, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "pu_dycore_profile": (_I, [_P, _I]),
    "pu_dycore_profile_read": (_I, [_P, C.POINTER(pu_profile)]),
    "pu_dycore_time_step_noalloc": (_I, [C.POINTER(pu_config), _P, _P, _P, C.POINTER(pu_state_view), _D,
                                         C.POINTER(_I)]),
    "pu_weno9_edges_f32": (_I, [_P, _P, C.c_longlong, _I, _P, _P, _I]),
    "pu_learned_normalize_f32": (_I, [_P, C.c_longlong, _P, _P]),
    "pu_check_bounded_wait": (_I, [_I, _P, _P, _P]),
    "pu_decomp_process_grid": (_I, [_I, C.c_longlong, C.c_longlong, C.POINTER(_I), C.POINTER(_I)]),
    "pu_decomp_tile": (_I, [C.c_longlong, _I, _I, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "pu_decomp_neighbors": (_I, [C.POINTER(pu_decomp), C.POINTER(_I)]),
    "pu_nccl_get_unique_id": (_I, [C.c_char_p]),
    "pu_dycore_set_decomposition": (_I, [_P, C.POINTER(pu_decomp), C.c_char_p]),
    "pu_dycore_set_decomposition_host": (_I, [_P, C.POINTER(pu_decomp), C.POINTER(pu_host_transport)]),
    "pu_dycore_group_init": (_I, [C.POINTER(_P), _I, C.POINTER(pu_state_view), C.POINTER(_P), C.POINTER(_P), _I]),
    "pu_dycore_group_advance": (_I, [C.POINTER(_P), _I, _D, _I]),
    "pu_dycore_group_time_step": (_I, [C.POINTER(_P), _I, C.POINTER(pu_state_view), _D, C.POINTER(_I)]),
    # include/pu_physics.h
    "pu_physics_create": (_I, [C.POINTER(pu_physics_config), _P, _P, _P, _I, C.POINTER(C.c_void_p)]),
    "pu_physics_destroy": (_I, [_P]),
    "pu_les_apply": (_I, [_P, C.POINTER(pu_state_view), _D]),
    "pu_les_apply_to": (_I, [_P, C.POINTER(pu_state_view), C.POINTER(pu_state_view), _D]),
    "pu_sponge_layer": (_I, [_P, C.POINTER(pu_state_view), _D, _D, _D]),
    "pu_geostrophic_forcing": (_I, [_P, C.POINTER(pu_state_view), _D, _D, _D, _D]),
    "pu_surface_fluxes": (_I, [_P, C.POINTER(pu_state_view), _D]),
    "pu_uniform_pg_wind_forcing": (_I, [_P, C.POINTER(pu_state_view), _D, _D, C.c_ulonglong,
                                        C.POINTER(pu_uniform_pg_state)]),
    "pu_uniform_pg_wind_forcing_height": (_I, [_P, C.POINTER(pu_state_view), _D, _D, _D, _D, _D]),
    "pu_time_averager_accumulate": (_I, [_P, C.POINTER(pu_state_view), C.POINTER(pu_time_averages), _D, _D]),
    "pu_edge_sponge_set_column": (_I, [_P, C.POINTER(pu_state_view), _P, _I, _P]),
    "pu_edge_sponge_apply": (_I, [_P, C.POINTER(pu_state_view), _P, _I, _P, _D, _D, _D, _D, C.c_longlong,
                                  C.c_longlong, C.c_longlong, C.c_longlong]),
    "pu_physics_synchronize": (_I, [_P]),
    "pu_physics_last_les_ms": (_I, [_P, C.POINTER(_D)]),
}
PU_NOALLOC_SCRATCH_BYTES = 64 << 20

_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load libpu_dycore.so (build it first with porturb_b200.build.build())."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError("libpu_dycore.so is not built (%s); run porturb_b200/build.py" % path)
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int) -> int:
    if status != PU_OK:
        raise PortUrbError(status, load().pu_last_error().decode())
    return status
