"""ctypes binding of ``libreconnet_b200.so`` (the C ABI in include/reconnet_b200.h).

The library is loaded from ``reconnet_b200/_lib``; if it is missing this
module raises at import time -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libreconnet_b200.so")
PRIOR_LIB_PATH = os.path.join(_HERE, "_lib", "libreconnet_b200_prior.so")

RN_OK = 0
RN_ERR_ARG = 1
RN_ERR_CUDA = 2
RN_ERR_ALLOC = 3
RN_ERR_TIMEOUT = 4
RN_TYPE_ITERATIVE = 0
RN_TYPE_FBP = 1
RN_TYPE_MATCHED = 2
RN_TYPE_SIDDON = 3
RN_TYPE_PIXEL = 4
RN_WEIGHT_PARKER = 0
RN_WEIGHT_RIESS = 1

_f = ctypes.c_float
_i = ctypes.c_int
_fp = ctypes.POINTER(ctypes.c_float)
_vp = ctypes.c_void_p
_d = ctypes.c_double


class RnFanGeom(ctypes.Structure):
    """Mirror of ``RnFanGeom`` (fields of Projector, ReconNet4D/Projector.h:10-37)."""
    _fields_ = [("nBatches", _i), ("nChannels", _i), ("nx", _i), ("ny", _i), ("nz", _i),
                ("dx", _f), ("dy", _f), ("dz", _f), ("cx", _f), ("cy", _f), ("cz", _f),
                ("nu", _i), ("nview", _i), ("nv", _i),
                ("du", _f), ("dv", _f), ("off_u", _f), ("off_v", _f), ("dsd", _f), ("dso", _f)]


class RnConeGeom(ctypes.Structure):
    """Mirror of ``RnConeGeom`` (the SiddonCone setup, ReconNet4D/SiddonCone.cu:126-201)."""
    _fields_ = [("nBatches", _i), ("nChannels", _i), ("nx", _i), ("ny", _i), ("nz", _i),
                ("dx", _f), ("dy", _f), ("dz", _f), ("cx", _f), ("cy", _f), ("cz", _f),
                ("nu", _i), ("nview", _i), ("nv", _i),
                ("du", _f), ("dv", _f), ("off_u", _f), ("off_v", _f)]


class RnCylGeom(ctypes.Structure):
    """Mirror of ``RnCylGeom`` (cylindrical-detector cone-beam DD, circular orbit)."""
    _fields_ = [("nBatches", _i), ("nx", _i), ("ny", _i), ("nz", _i),
                ("dx", _f), ("dy", _f), ("dz", _f), ("cx", _f), ("cy", _f), ("cz", _f),
                ("nu", _i), ("nview", _i), ("nv", _i),
                ("da", _f), ("dv", _f), ("off_a", _f), ("off_v", _f), ("dsd", _f), ("dso", _f)]


class ReconNetError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"reconnet_b200 error {code}: {msg}")
        self.code = code


_FAN = [_i, _i, _i, _i, _i, _f, _f, _f, _i, _i, _i, _f, _f, _f, _f, _f, _f, _i]
_TOMO = [_i, _i, _i, _i, _i, _f, _f, _f, _f, _f, _f, _i, _i, _i, _f, _f, _f, _f]
_FILT = [_i, _i, _i, _i, _i, _f, _f, _f, _f, _f, _f, _i, _i]

# name -> (restype, argtypes); every entry point of include/reconnet_b200.h
SIGNATURES = {
    "rn_last_error": (ctypes.c_char_p, []),
    "rn_last_status": (_i, []),
    "rn_version": (_i, []),
    "SetDevice": (_i, [_i]),
    "cDistanceDrivenFanProjection": (None, [_fp, _fp, _fp] + _FAN),
    "cDistanceDrivenFanBackprojection": (None, [_fp, _fp, _fp] + _FAN),
    "cSiddonFanProjection": (None, [_fp, _fp, _fp] + _FAN),
    "cSiddonFanBackprojection": (None, [_fp, _fp, _fp] + _FAN),
    "cPixelDrivenFanBackprojection": (None, [_fp, _fp, _fp] + _FAN),
    "cDistanceDrivenTomoProjection": (None, [_fp, _fp, _fp, _fp] + _TOMO),
    "cDistanceDrivenTomoBackprojection": (None, [_fp, _fp, _fp, _fp] + _TOMO),
    "cFilterFanFilter": (None, [_fp, _fp] + _FILT),
    "cFilterParallelFilter": (None, [_fp, _fp] + _FILT),
    "cOSSQS": (None, [_fp, _fp, _fp, _fp, _fp, _fp, _f, _f, _i, _i] + _FAN[:-1] + [_i, _f]),
    "cDDFanOSSQS": (None, [_fp, _fp, _fp, _fp, _fp, _fp, _f, _f, _i, _i] + _FAN[:-1] + [_i, _f]),
    "cTVSQS2D": (_f, [_fp, _fp, _fp, _i, _i]),
    "rn_fan_plan_create": (_i, [ctypes.POINTER(_vp), ctypes.POINTER(RnFanGeom), _fp, _vp]),
    "rn_fan_plan_create_ragged": (_i, [ctypes.POINTER(_vp), ctypes.POINTER(RnFanGeom),
                                       ctypes.POINTER(_i), _fp, _vp]),
    "rn_fan_plan_destroy": (_i, [_vp]),
    "rn_cone_plan_create": (_i, [ctypes.POINTER(_vp), ctypes.POINTER(RnConeGeom), _fp, _fp, _fp, _fp, _vp]),
    "rn_cone_plan_destroy": (_i, [_vp]),
    "rn_cone_project": (_i, [_vp, _vp, _vp, _vp]),
    "rn_cone_backproject": (_i, [_vp, _vp, _vp, _i, _vp]),
    "rn_cone_plan_launches": (ctypes.c_longlong, [_vp]),
    "cSiddonConeProjectionAbitrary": (None, [_fp] * 6 + _TOMO),
    "cSiddonConeBackprojectionAbitrary": (None, [_fp] * 6 + _TOMO),
    "cOSSQSConeAbitrary": (None, [_fp] * 9 + [_f, _f, _i, _i] + _TOMO + [_i, _f]),
    "rn_fan_plan_total_views": (ctypes.c_int64, [_vp]),
    "rn_fan_project": (_i, [_vp, _vp, _vp, _vp]),
    "rn_fan_project_siddon": (_i, [_vp, _vp, _vp, _vp]),
    "rn_fan_backproject": (_i, [_vp, _vp, _vp, _i, _i, _vp]),
    "rn_fan_plan_check": (_i, [_vp, _vp]),
    "rn_fan_plan_set_timing": (_i, [_vp, _i]),
    "rn_fan_plan_autotune": (_i, [_vp, _vp, _vp, _i, _vp]),
    "rn_fan_plan_set_tuning": (_i, [_vp, _i, _i, _i, _vp]),
    "rn_fan_plan_get_tuning": (_i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "rn_fan_plan_read_timing": (_i, [_vp, _fp, ctypes.POINTER(_i), _i, ctypes.POINTER(ctypes.c_longlong)]),
    "rn_filter": (_i, [_vp, _vp, _i, _i, _i, _i, _i, _f, _f, _f, _f, _i, _i, _vp]),
    "rn_filter_set_form": (_i, [_i]),
    "rn_filter_weighted": (_i, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _f, _f, _f, _f, _i, _i, _vp]),
    "rn_fan_shortscan_weights": (_i, [_vp, _vp, _i, _i, _d, _d, _i, _d, _d, _i, _vp]),
    "rn_fan_shortscan_weights_host": (_i, [_fp, _fp, _i, _i, _d, _d, _i, _d, _d, _i]),
    "rn_tv_sqs": (_i, [_vp, _vp, _vp, _vp, _i, _i, _i, _vp]),
    "rn_tv_iso_sqs": (_i, [_vp, _vp, _vp, _vp, _i, _i, _i, _i, _i, _f, _i, _vp]),
    "rn_tv_iso_sqs_host": (_i, [_fp, _fp, _fp, _fp, _i, _i, _i, _i, _i, _f, _i]),
    "rn_fan_sqs_update": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _f, _f, _i, _f, _f, _i, _vp]),
    "rn_fan_project_noalloc": (_i, [_vp, _vp, _fp, _i, _i, _f, _f, _i, _i, _f, _f, _f, _f, _vp]),
    "rn_tomo_sat_bytes": (_i, [_i, _i, _i, _i, _i, _i, ctypes.POINTER(ctypes.c_size_t),
                               ctypes.POINTER(ctypes.c_size_t)]),
    "rn_tomo_project": (_i, [_vp, _vp, _vp, _vp, _vp] + _TOMO + [_vp]),
    "rn_tomo_backproject": (_i, [_vp, _vp, _vp, _vp, _vp] + _TOMO + [_i, _vp]),
    "rn_fan_plan_set_spin_limit": (_i, [_vp, ctypes.c_longlong]),
    "rn_cyl_plan_create": (_i, [ctypes.POINTER(_vp), ctypes.POINTER(RnCylGeom), _fp, _vp]),
    "rn_cyl_plan_destroy": (_i, [_vp]),
    "rn_cyl_project": (_i, [_vp, _vp, _vp, _vp]),
    "rn_cyl_backproject": (_i, [_vp, _vp, _vp, _vp]),
    "rn_cyl_plan_launches": (ctypes.c_longlong, [_vp]),
    "rn_conv3x3": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _i, _i, _i, _i, _i, _vp, _vp]),
    "rn_conv3x3_wgrad_cols": (_i, [_i]),
    "rn_conv3x3_wgrad": (_i, [_vp, _vp, ctypes.c_size_t, _vp, _vp, _i, _i, _i, _i, _i, _vp, _vp]),
    "rn_conv_pack_image": (_i, [_vp, _vp, _vp, _f, _i, _i, _i, _vp]),
}


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"reconnet_b200 native library not built ({LIB_PATH}); run `python -m reconnet_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()

# the prior-solver shim (include/reconnet_b200_prior.h), loaded on first use
PRIOR_SIGNATURES = {
    "cTVSQS2D": (None, [_fp, _fp, _fp, _fp, _i, _i, _i, _i, _f]),
    "cTVSQS3D": (None, [_fp, _fp, _fp, _fp, _i, _i, _i, _i, _i, _f]),
}
_prior = None


def prior_lib():
    global _prior
    if _prior is None:
        if not os.path.exists(PRIOR_LIB_PATH):
            raise ImportError(f"prior-solver shim not built ({PRIOR_LIB_PATH}); run `python -m reconnet_b200.build`")
        p = ctypes.CDLL(PRIOR_LIB_PATH)
        for name, (res, args) in PRIOR_SIGNATURES.items():
            fn = getattr(p, name)
            fn.restype = res
            fn.argtypes = args
        _prior = p
    return _prior


def last_error() -> str:
    s = lib.rn_last_error()
    return s.decode() if s else ""


def check(status: int) -> None:
    """Raise ReconNetError if a native call returned a non-zero status."""
    if status != RN_OK:
        raise ReconNetError(status, last_error())


def check_last() -> None:
    """Raise if the most recent reference-named (void) call failed."""
    st = lib.rn_last_status()
    if st != RN_OK:
        raise ReconNetError(st, last_error())
