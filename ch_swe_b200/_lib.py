"""ctypes binding of ``libchswe.so`` (declarations in include/chswe.h).

The library is the only compute path: if it cannot be loaded, or no CUDA
device is present, every call raises.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libchswe.so")

SWE_OK = 0
SWE_FP64 = 0
SWE_FP32 = 1
SWE_OP_LINEAR = 0
SWE_OP_ADVECTIVE = 1
SWE_STAG_CH = 0
SWE_STAG_AH = 1
SWE_STAG_C = 2

ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "out of device memory", -4: "no CUDA device",
          -5: "cube size above SWE_NOALLOC_MAX_N"}
SWE_ETOOBIG = -5
SWE_NOALLOC_MAX_N = 64

EXPORTED = [
    "swe_cfg_default", "swe_ctx_create", "swe_ctx_destroy", "swe_last_error", "swe_set_stream",
    "swe_synchronize", "swe_set_member_h_mean", "swe_stvec_create", "swe_stvec_destroy",
    "swe_stvec_upload", "swe_stvec_download", "swe_stvec_upload_all", "swe_stvec_download_all",
    "swe_stvec_assign", "swe_stvec_update", "swe_stvec_device_view", "swe_operator_apply",
    "swe_rk4_step", "swe_rk4_steps", "swe_integrals", "swe_launch_count", "swe_edge_links",
    "swe_kernel_times", "swe_operator_contravariant", "swe_operator_apply_noalloc",
    "swe_set_tile", "swe_get_tile", "swe_autotune", "swe_rk4_steps_members",
    "swe_set_kernel_config", "swe_get_kernel_config", "swe_diag", "swe_energies", "swe_curl", "swe_regrid_latlon", "swe_regrid_latlon_wind",
    "swe_set_orography", "swe_c_grad", "swe_c_div",
    "swe_group_create", "swe_group_destroy", "swe_group_rk4_steps_members", "swe_group_synchronize",
    "swe_group_last_error", "swe_group_launch_count", "swe_diffusion_apply", "swe_diffusion_step",
    "swe_set_diffusion",
]


class SweCfg(ctypes.Structure):
    _fields_ = [
        ("N", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("n_members", ctypes.c_int),
        ("operator_kind", ctypes.c_int),
        ("radius", ctypes.c_double),
        ("grav", ctypes.c_double),
        ("omega", ctypes.c_double),
        ("rotation_axis", ctypes.c_double * 3),
        ("coriolis_constant", ctypes.c_int),
        ("h_mean", ctypes.c_double),
        ("sbp_order", ctypes.c_int),
        ("staggering", ctypes.c_int),
    ]


class SweError(RuntimeError):
    pass


_lib = None
_dp = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p


def load(path: str = LIB_PATH):
    """Load libchswe.so; raises if it is missing (build it with ch_swe_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise SweError(f"{path} is missing: run `python -m ch_swe_b200.build` (nvcc, sm_100a)")
    L = ctypes.CDLL(path)
    L.swe_cfg_default.argtypes = [ctypes.POINTER(SweCfg)]
    L.swe_ctx_create.argtypes = [ctypes.POINTER(SweCfg), ctypes.POINTER(_vp)]
    L.swe_ctx_destroy.argtypes = [_vp]
    L.swe_last_error.argtypes = [_vp]
    L.swe_last_error.restype = ctypes.c_char_p
    L.swe_set_stream.argtypes = [_vp, _vp]
    L.swe_synchronize.argtypes = [_vp]
    L.swe_set_member_h_mean.argtypes = [_vp, ctypes.c_int, ctypes.c_double]
    L.swe_set_orography.argtypes = [_vp, _vp]
    L.swe_c_grad.argtypes = [_vp, _vp, _vp]
    L.swe_c_div.argtypes = [_vp, _vp, _vp]
    L.swe_stvec_create.argtypes = [_vp, ctypes.POINTER(_vp)]
    L.swe_stvec_destroy.argtypes = [_vp]
    L.swe_stvec_upload.argtypes = [_vp, ctypes.c_int, _dp, _dp, _dp]
    L.swe_stvec_download.argtypes = [_vp, ctypes.c_int, _dp, _dp, _dp]
    L.swe_stvec_upload_all.argtypes = [_vp, _dp, _dp, _dp]
    L.swe_stvec_download_all.argtypes = [_vp, _dp, _dp, _dp]
    L.swe_stvec_assign.argtypes = [_vp, ctypes.c_double, _vp, ctypes.c_double, _vp]
    L.swe_stvec_update.argtypes = [_vp, ctypes.c_double, _vp, ctypes.c_double, _vp]
    L.swe_stvec_device_view.argtypes = [_vp, ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_size_t),
                                        ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    L.swe_operator_apply.argtypes = [_vp, _vp, _vp]
    L.swe_operator_contravariant.argtypes = [_vp, _vp, _vp]
    L.swe_operator_apply_noalloc.argtypes = [ctypes.POINTER(SweCfg), _vp, _vp, _vp]
    L.swe_rk4_step.argtypes = [_vp, _vp, ctypes.c_double]
    L.swe_rk4_steps.argtypes = [_vp, _vp, ctypes.c_double, ctypes.c_int]
    L.swe_rk4_steps_members.argtypes = [_vp, _vp, _dp, ctypes.c_int]
    L.swe_integrals.argtypes = [_vp, _vp, ctypes.c_int, _dp, _dp]
    L.swe_diffusion_apply.argtypes = [_vp, _vp, _vp, ctypes.c_int, ctypes.c_double, ctypes.c_double]
    L.swe_diffusion_step.argtypes = [_vp, _vp, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double]
    L.swe_set_diffusion.argtypes = [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_double]
    L.swe_launch_count.argtypes = [_vp]
    L.swe_launch_count.restype = ctypes.c_longlong
    L.swe_edge_links.argtypes = [ctypes.POINTER(ctypes.c_int)]
    L.swe_kernel_times.argtypes = [_vp, _vp, ctypes.c_double, ctypes.c_int, _dp, _dp, _dp]
    L.swe_set_tile.argtypes = [_vp, ctypes.c_int]
    L.swe_get_tile.argtypes = [_vp, ctypes.POINTER(ctypes.c_int)]
    L.swe_autotune.argtypes = [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), _dp]
    L.swe_diag.argtypes = [_vp, _vp, ctypes.c_int, ctypes.c_double, _dp]
    L.swe_energies.argtypes = [_vp, _vp, ctypes.c_int, _dp]
    L.swe_curl.argtypes = [_vp, _vp, ctypes.c_int, _dp]
    L.swe_regrid_latlon.argtypes = [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp]
    L.swe_regrid_latlon_wind.argtypes = [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp]
    L.swe_set_kernel_config.argtypes = [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.swe_get_kernel_config.argtypes = [_vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_int)]
    L.swe_group_create.argtypes = [ctypes.POINTER(_vp), ctypes.c_int, ctypes.POINTER(_vp)]
    L.swe_group_destroy.argtypes = [_vp]
    L.swe_group_rk4_steps_members.argtypes = [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_dp), ctypes.c_int]
    L.swe_group_synchronize.argtypes = [_vp]
    L.swe_group_last_error.argtypes = [_vp]
    L.swe_group_last_error.restype = ctypes.c_char_p
    L.swe_group_launch_count.argtypes = [_vp]
    L.swe_group_launch_count.restype = ctypes.c_longlong
    for name in EXPORTED:
        if not hasattr(L, name):
            raise SweError(f"libchswe.so does not export {name}")
    _lib = L
    return L


def check(rc: int, ctx=None, what: str = "") -> None:
    if rc != SWE_OK:
        msg = ERRORS.get(rc, f"error {rc}")
        if ctx:
            detail = load().swe_last_error(ctx)
            if detail:
                msg += ": " + detail.decode(errors="replace")
        raise SweError(f"{what}: {msg}" if what else msg)


def dptr(a):
    return a.ctypes.data_as(_dp)
