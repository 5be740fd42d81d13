"""ctypes binding of the C ABI in include/gaukuk_cuda.h (lib/libgk_cuda.so).

There is no fallback: if the library is missing or no CUDA device is present,
loading or creating a handle raises.
"""
from __future__ import annotations

import ctypes
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libgk_cuda.so")
# GK_CHECKED=1: the bounds-checked build of the same library (gk_checked_report)
CHECKED_LIB_PATH = os.path.join(_PKG, "lib", "checked", "libgk_cuda.so")

GK_OK = 0
GK_MODE_PARITY = 0
GK_MODE_FAST = 1


class GridDesc(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("nghost", ctypes.c_int),
                ("xmin", ctypes.c_double), ("xmax", ctypes.c_double),
                ("ymin", ctypes.c_double), ("ymax", ctypes.c_double),
                ("zmin", ctypes.c_double), ("zmax", ctypes.c_double)]


class PhysDesc(ctypes.Structure):
    _fields_ = [("gamma", ctypes.c_double), ("cfl", ctypes.c_double),
                ("integrator", ctypes.c_int), ("rc_order", ctypes.c_int),
                ("bc", ctypes.c_int * 6), ("grav", ctypes.c_double * 3),
                ("dfloor", ctypes.c_double), ("pfloor", ctypes.c_double),
                ("stepmax", ctypes.c_int), ("mode", ctypes.c_int), ("device", ctypes.c_int)]


# Every exported symbol with its signature: (restype, argtypes).
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p
SIGNATURES = {
    "gk_create": (ctypes.c_int, [ctypes.POINTER(GridDesc), ctypes.POINTER(PhysDesc),
                                 ctypes.POINTER(ctypes.c_void_p)]),
    "gk_destroy": (None, [_vp]),
    "gk_state_size": (ctypes.c_longlong, [_vp]),
    "gk_upload_cons": (ctypes.c_int, [_vp, _vp]),
    "gk_download_cons": (ctypes.c_int, [_vp, _vp]),
    "gk_download_planes": (ctypes.c_int, [_vp, _vp]),
    "gk_floor_hits": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_ulonglong),
                                     ctypes.POINTER(ctypes.c_ulonglong)]),
    "gk_io_bytes": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_longlong),
                                   ctypes.POINTER(ctypes.c_longlong)]),
    "gk_advance": (ctypes.c_int, [_vp, ctypes.c_double, _dp, _ip, _ip]),
    "gk_run_steps": (ctypes.c_int, [_vp, ctypes.c_int, _ip]),
    "gk_enqueue_steps": (ctypes.c_int, [_vp, ctypes.c_int]),
    "gk_get_time": (ctypes.c_int, [_vp, _dp, _dp, _ip, _ip]),
    "gk_set_time": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_int]),
    "gk_dt_log": (ctypes.c_int, [_vp, _dp, ctypes.c_int, _ip]),
    "gk_cmax": (ctypes.c_int, [_vp, _dp]),
    "gk_stream": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_void_p)]),
    "gk_path": (ctypes.c_int, [_vp, _ip]),
    "gk_graph_info": (ctypes.c_int, [_vp, _ip, _ip]),
    "gk_profile_steps": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_char_p, ctypes.c_int, _dp,
                                        _ip, ctypes.c_int, _ip]),
    "gk_fastmath_check": (ctypes.c_int, [ctypes.c_int, ctypes.c_ulonglong, _dp]),
    "gk_checked_report": (ctypes.c_int, [ctypes.POINTER(ctypes.c_ulonglong),
                                         ctypes.POINTER(ctypes.c_ulonglong)]),
    "gk_rk2_step_noalloc": (ctypes.c_int, [ctypes.POINTER(GridDesc), ctypes.POINTER(PhysDesc),
                                           _vp, ctypes.c_double, _dp, _vp]),
    "gk_set_tiling": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    "gk_ens_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_void_p)]),
    "gk_ens_destroy": (None, [_vp]),
    "gk_ens_set_tiling": (ctypes.c_int, [_vp, ctypes.c_int, _ip]),
    "gk_ens_advance": (ctypes.c_int, [_vp, ctypes.c_double]),
    "gk_ens_run_steps": (ctypes.c_int, [_vp, ctypes.c_int]),
    "gk_ens_enqueue_steps": (ctypes.c_int, [_vp, ctypes.c_int]),
    "gk_ens_info": (ctypes.c_int, [_vp, _ip, _ip, ctypes.POINTER(ctypes.c_void_p)]),
    "gk_ens_last_error": (ctypes.c_char_p, [_vp]),
    "gk_mlp_nparams": (ctypes.c_int, []),
    "gk_mlp_nmodel": (ctypes.c_int, []),
    "gk_mlp_create": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_void_p)]),
    "gk_mlp_destroy": (None, [_vp]),
    "gk_mlp_get": (ctypes.c_int, [_vp, _vp]),
    "gk_mlp_set_pair_loss": (ctypes.c_int, [_vp, ctypes.c_float]),
    "gk_mlp_grad": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_longlong, ctypes.c_int, _vp, _vp]),
    "gk_mlp_train": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_longlong, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_float, ctypes.c_ulonglong, _vp]),
    "gk_mlp_forward": (ctypes.c_int, [_vp, _vp, ctypes.c_longlong, _vp]),
    "gk_set_fixed_boundary": (ctypes.c_int, [_vp, _vp, ctypes.c_int]),
    "gk_set_immersed": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp, _vp]),
    "gk_set_point_gravity": (ctypes.c_int, [_vp, ctypes.c_int, _vp]),
    "gk_set_host_fill": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp]),
    "gk_set_flux_model": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                         ctypes.c_float, ctypes.c_float]),
    "gk_flux_model_fired": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_uint)]),
    "gk_set_flux_model_fused": (ctypes.c_int, [_vp, ctypes.c_int]),
    "gk_face_fluxes": (ctypes.c_int, [_vp, _vp, _vp]),
    "gk_tap_substeps": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, _vp, _vp]),
    "gk_slab_layout": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      _ip, _ip, _ip, _ip]),
    "gk_slab_exchange_plan": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _ip, _ip]),
    "gk_slabs_create": (ctypes.c_int, [ctypes.POINTER(GridDesc), ctypes.POINTER(PhysDesc),
                                       ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "gk_slabs_nccl_id": (ctypes.c_int, [_vp]),
    "gk_slabs_create_nccl": (ctypes.c_int, [ctypes.POINTER(GridDesc), ctypes.POINTER(PhysDesc),
                                            ctypes.c_int, ctypes.c_int, _vp,
                                            ctypes.POINTER(ctypes.c_void_p)]),
    "gk_slabs_destroy": (None, [_vp]),
    "gk_slabs_upload_cons": (ctypes.c_int, [_vp, _vp]),
    "gk_slabs_download_cons": (ctypes.c_int, [_vp, _vp]),
    "gk_slabs_advance": (ctypes.c_int, [_vp, ctypes.c_double, _dp, _ip, _ip]),
    "gk_slabs_run_steps": (ctypes.c_int, [_vp, ctypes.c_int, _ip]),
    "gk_slabs_dt_log": (ctypes.c_int, [_vp, _dp, ctypes.c_int, _ip]),
    "gk_slabs_info": (ctypes.c_int, [_vp, _ip, _ip, _ip, _ip]),
    "gk_slabs_last_error": (ctypes.c_char_p, [_vp]),
    "gk_strerror": (ctypes.c_char_p, [ctypes.c_int]),
    "gk_last_error": (ctypes.c_char_p, [_vp]),
}

_lib = None


def load(path: str = None):
    """Load libgk_cuda.so (the bounds-checked build when GK_CHECKED=1) and
    declare every entry point; raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if path is None:
        path = CHECKED_LIB_PATH if os.environ.get("GK_CHECKED") == "1" else LIB_PATH
    if not os.path.exists(path):
        raise RuntimeError(
            f"CUDA extension not built: {path} is missing (run __graft_entry__.build())")
    L = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


class GkError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{msg} (status {code})")
        self.code = code


def check(code: int, handle=None) -> None:
    if code == GK_OK:
        return
    L = load()
    msg = L.gk_strerror(code).decode()
    if handle:
        detail = L.gk_last_error(handle).decode()
        if detail:
            msg = f"{msg}: {detail}"
    raise GkError(code, msg)
