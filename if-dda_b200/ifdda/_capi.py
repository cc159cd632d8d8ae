"""ctypes binding of libifdda_gpu.so (declarations: include/ifdda_gpu.h).

The library is the product; this module only marshals numpy arrays (or raw
device pointers) to it.  There is no CPU fallback: if the shared library is
missing or no CUDA device is present the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

_PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG_DIR, "libifdda_gpu.so")
HEADER_PATH = os.path.join(os.path.dirname(_PKG_DIR), "include", "ifdda_gpu.h")

IFDDA_FP64 = 0
IFDDA_MIXED = 1
IFDDA_FP32 = 2


class DComplex(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


class SolveOptions(C.Structure):
    _fields_ = [("precision", C.c_int), ("check_every", C.c_int), ("max_outer", C.c_int),
                ("inner_floor", C.c_double), ("maxit", C.c_int)]


class MicroscopeOptions(C.Structure):
    _fields_ = [("ntypemic", C.c_int), ("nfft2d", C.c_int), ("numaper", C.c_double), ("numaperinc", C.c_double),
                ("gross", C.c_double), ("zlens", C.c_double), ("P0", C.c_double), ("w0", C.c_double),
                ("batch", C.c_int), ("nside", C.c_int), ("nquicklens", C.c_int)]


_lib = None

_vp = C.c_void_p
_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)

# name -> (restype, argtypes)
SIGNATURES = {
    "ifdda_abi_version": (C.c_int, []),
    "ifdda_ctx_create": (C.c_int, [C.c_int, C.POINTER(_vp)]),
    "ifdda_ctx_destroy": (C.c_int, [_vp]),
    "ifdda_ctx_last_error": (C.c_char_p, [_vp]),
    "ifdda_ctx_synchronize": (C.c_int, [_vp]),
    "ifdda_ctx_stream": (_vp, [_vp]),
    "ifdda_green_create": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.POINTER(_vp)]),
    "ifdda_green_create_nquad": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
                                           C.POINTER(_vp)]),
    "ifdda_green_recompute": (C.c_int, [_vp, C.c_double, C.c_double]),
    "ifdda_green_tiles": (C.c_int, [_vp, C.c_int, _ip, _ip, C.POINTER(C.c_float)]),
    "ifdda_green_set_tiles": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int]),
    "ifdda_green_create_box": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                         C.c_double, C.POINTER(_vp)]),
    "ifdda_inverserig_ragged": (C.c_int, [C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, C.c_char_p, C.c_double, _vp,
                                          _vp, _vp, _vp, _vp, _ip, C.c_char_p, C.POINTER(SolveOptions)]),
    "ifdda_inverserig_ragged_device": (C.c_int, [C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, C.c_char_p, C.c_double,
                                                 _vp, _vp, _vp, _vp, _vp, _ip, C.c_char_p, C.POINTER(SolveOptions)]),
    "ifdda_green_destroy": (C.c_int, [_vp]),
    "ifdda_green_release_workspace": (C.c_int, [_vp]),
    "ifdda_green_export": (C.c_int, [_vp] + [_vp] * 6),
    "ifdda_matvec": (C.c_int, [_vp, C.c_int, C.c_int, _vp, _vp, _vp]),
    "ifdda_matvec_device": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp]),
    "ifdda_matvec_noalloc": (C.c_int, [_vp, C.c_int, C.c_int, _vp, _vp, _vp]),
    "ifdda_inverserig": (C.c_int, [_vp, C.c_int, C.c_int, _vp, _vp, _vp, C.c_char_p, C.c_double, _vp, _vp, _dp,
                                   _ip, _ip, _ip, C.c_char_p, C.POINTER(SolveOptions)]),
    "ifdda_inverserig_batch": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, C.c_char_p, C.c_double,
                                         _vp, _vp, _vp, _vp, _vp, _ip, C.c_char_p, C.POINTER(SolveOptions)]),
    "ifdda_inverserig_batch_device": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, C.c_char_p,
                                                C.c_double, _vp, _vp, _vp, _vp, _vp, _ip, C.c_char_p,
                                                C.POINTER(SolveOptions)]),
    "ifdda_local_macro": (C.c_int, [_vp, C.c_int, C.c_int, _vp, _vp, C.c_double, C.c_double, _vp]),
    "ifdda_cross_sections": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp, C.c_double, C.c_double, _dp, _dp]),
    "ifdda_incident_planewaves": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp, C.c_double, DComplex, C.c_int, _vp, _vp,
                                            _vp, _vp, _vp]),
    "ifdda_incident_planewaves_device": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp, C.c_double, DComplex, C.c_int, _vp,
                                                   _vp, _vp, _vp, _vp]),
    "ifdda_farfield_csca": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp, _vp, C.c_double, C.c_double, C.c_double,
                                      C.c_double, C.c_int, C.c_int, _dp, _dp, _vp, _vp, _vp]),
    "ifdda_farfield_fft": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_double, _vp, _vp, _vp, _vp, C.c_double,
                                     C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, _dp, _dp, _vp,
                                     _vp, _vp, _ip, _vp, _vp]),
    "ifdda_nearfield_wide": (C.c_int, [_vp] + [C.c_int] * 6 + [C.c_double, C.c_double] + [C.c_int] * 3 +
                             [_vp] * 6 + [DComplex, C.c_double, C.c_double, C.c_double] + [_vp] * 6),
    "ifdda_holography": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, _vp, _vp, _vp,
                                   _vp, DComplex, C.c_double, C.c_double, C.c_double, C.c_int, C.c_double,
                                   C.c_double, C.c_double, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _ip, C.c_char_p]),
    "ifdda_microscope": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp, _vp, _vp, C.c_char_p, C.c_double,
                                   C.POINTER(MicroscopeOptions),
                                   _vp, _vp, _vp, _ip, _vp, _vp, _dp, _ip, _ip, _ip, C.c_char_p,
                                   C.POINTER(SolveOptions)]),
    "ifdda_launch_count": (C.c_ulonglong, []),
    "ifdda_timing_enable": (C.c_int, [C.c_int, C.c_int]),
    "ifdda_timing_read": (C.c_int, [_ip, _dp]),
}

PASS_FWD_X, PASS_FWD_Y, PASS_ZCONV, PASS_INV_Y, PASS_INV_X = 1, 2, 3, 4, 5


def load():
    """Load the library (no CUDA call is made by loading it)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libifdda_gpu.so not built (expected at {LIB_PATH}); run __graft_entry__.build()")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib
