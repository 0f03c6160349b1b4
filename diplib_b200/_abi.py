"""ctypes binding of libdipcu.so (include/dipcu.h).

The library must exist in-tree (``diplib_b200/lib/libdipcu.so``, built by
``diplib_b200.build``); there is no other implementation to fall back to, so a missing library
raises at import of the first operator that needs it.
"""
from __future__ import annotations

import ctypes
import os
import threading

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libdipcu.so")
MAX_DIMS = 8

# dipcu_dtype codes.
BIN, UINT8, UINT16, UINT32, UINT64, SINT8, SINT16, SINT32, SINT64, SFLOAT, DFLOAT = range(11)

# dipcu_status codes.
OK = 0
ERR_INVALID_ARG = 1
ERR_UNSUPPORTED_DTYPE = 2
ERR_UNSUPPORTED_BC = 3
ERR_ORDER_GT_3 = 4
ERR_CUDA = 5
ERR_TIMEOUT = 6
ERR_SIZES_DONT_MATCH = 7
ERR_KERNEL_TOO_LARGE = 8

# dipcu_gauss_iir design methods
IIR_DISCRETE_TIME_FIT = 0
IIR_FORWARD_BACKWARD = 1


class ImageDesc(ctypes.Structure):
    _fields_ = [
        ("data", ctypes.c_void_p),
        ("dtype", ctypes.c_int32),
        ("ndims", ctypes.c_int32),
        ("sizes", ctypes.c_int64 * MAX_DIMS),
        ("strides", ctypes.c_int64 * MAX_DIMS),
    ]


class Filter1D(ctypes.Structure):
    """dipcu_filter_1d: a real 1D filter (dip::OneDimensionalFilter)."""
    _fields_ = [
        ("weights", ctypes.POINTER(ctypes.c_double)),
        ("size", ctypes.c_int64),
        ("origin", ctypes.c_int64),
        ("symmetry", ctypes.c_int32),
    ]


# dipcu_symmetry codes, by dip::OneDimensionalFilter::symmetry string (real filters: "conj" is "even").
SYMMETRY = {"": 0, "general": 0, "even": 1, "odd": 2, "conj": 1, "d-even": 3, "d-odd": 4, "d-conj": 3}

_lib = None
_lock = threading.Lock()

# Every exported symbol of include/dipcu.h with (restype, argtypes).
_P = ctypes.POINTER
SIGNATURES = {
    "dipcu_gauss_fir": (ctypes.c_int, [_P(ImageDesc), _P(ImageDesc), _P(ctypes.c_double), _P(ctypes.c_uint32),
                                       _P(ctypes.c_int32), ctypes.c_double, ctypes.c_void_p]),
    "dipcu_gauss_fir_noalloc": (ctypes.c_int, [_P(ImageDesc), _P(ImageDesc), _P(ctypes.c_double),
                                               _P(ctypes.c_uint32), _P(ctypes.c_int32), ctypes.c_double,
                                               ctypes.c_void_p]),
    "dipcu_separable_convolution": (ctypes.c_int, [_P(ImageDesc), _P(ImageDesc), _P(Filter1D), ctypes.c_int,
                                                   _P(ctypes.c_int32), _P(ctypes.c_uint8), ctypes.c_void_p]),
    "dipcu_uniform": (ctypes.c_int, [_P(ImageDesc), _P(ImageDesc), _P(ctypes.c_double), _P(ctypes.c_int32),
                                     ctypes.c_void_p]),
    "dipcu_gauss_fir_multi": (ctypes.c_int, [_P(ImageDesc), _P(ImageDesc), ctypes.c_int, _P(ctypes.c_uint32), ctypes.c_int,
                                             ctypes.c_int32, _P(ctypes.c_double), _P(ctypes.c_int32), ctypes.c_double,
                                             ctypes.c_void_p]),
    "dipcu_gauss_fir_multi_supported": (ctypes.c_int, [_P(ImageDesc), _P(ctypes.c_uint32), ctypes.c_int, _P(ctypes.c_double),
                                                       _P(ctypes.c_int32), ctypes.c_double]),
    "dipcu_gauss_iir": (ctypes.c_int, [_P(ImageDesc), _P(ImageDesc), _P(ctypes.c_double), _P(ctypes.c_uint32),
                                       _P(ctypes.c_int32), _P(ctypes.c_uint32), ctypes.c_int32, ctypes.c_double,
                                       ctypes.c_void_p]),
    "dipcu_gauss_ft": (ctypes.c_int, [_P(ImageDesc), _P(ImageDesc), _P(ctypes.c_double), _P(ctypes.c_uint32),
                                      ctypes.c_double, _P(ctypes.c_int32), ctypes.c_int, ctypes.c_void_p]),
    "dipcu_gauss_fir_backward": (ctypes.c_int, [_P(ImageDesc), _P(ImageDesc), _P(ImageDesc), ctypes.c_void_p,
                                                _P(ctypes.c_double), _P(ctypes.c_uint32), _P(ctypes.c_int32),
                                                ctypes.c_double, ctypes.c_void_p]),
    "dipcu_structure_tensor": (ctypes.c_int, [_P(ImageDesc), _P(ImageDesc), _P(ctypes.c_double), _P(ctypes.c_double),
                                              _P(ctypes.c_int32), ctypes.c_double, ctypes.c_void_p]),
    "dipcu_structure_tensor_backward": (ctypes.c_int, [_P(ImageDesc), _P(ImageDesc), _P(ImageDesc),
                                                       _P(ctypes.c_double), _P(ctypes.c_double), _P(ctypes.c_int32),
                                                       ctypes.c_double, ctypes.c_void_p]),
    "dipcu_batch_plan_create": (ctypes.c_int, [_P(ImageDesc), _P(ImageDesc), ctypes.c_int, _P(ctypes.c_double),
                                               _P(ctypes.c_uint32), _P(ctypes.c_int32), ctypes.c_double, ctypes.c_int,
                                               _P(ctypes.c_void_p)]),
    "dipcu_batch_plan_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "dipcu_batch_plan_info": (ctypes.c_int, [ctypes.c_void_p, _P(ctypes.c_int), _P(ctypes.c_int), _P(ctypes.c_int),
                                             _P(ctypes.c_int)]),
    "dipcu_batch_plan_launches": (ctypes.c_int, [ctypes.c_void_p, _P(ctypes.c_int), _P(ctypes.c_int)]),
    "dipcu_batch_plan_sigmas": (ctypes.c_void_p, [ctypes.c_void_p]),
    "dipcu_batch_plan_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "dipcu_device_status": (ctypes.c_int, [_P(ctypes.c_int), ctypes.c_int]),
    "dipcu_half_gaussian_length": (ctypes.c_int, [ctypes.c_double, ctypes.c_uint32, ctypes.c_double, ctypes.c_int]),
    "dipcu_make_gauss_weights": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_double,
                                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                                ctypes.c_void_p]),
    "dipcu_bc_from_string": (ctypes.c_int, [ctypes.c_char_p]),
    "dipcu_last_error_message": (ctypes.c_char_p, []),
    "dipcu_version": (ctypes.c_char_p, []),
    "dipcu_launch_count": (ctypes.c_uint64, []),
}


def lib():
    """The loaded libdipcu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m diplib_b200.build`")
                l = ctypes.CDLL(LIB_PATH)
                for name, (res, args) in SIGNATURES.items():
                    fn = getattr(l, name)
                    fn.restype = res
                    fn.argtypes = args
                _lib = l
    return _lib


def last_error() -> str:
    return lib().dipcu_last_error_message().decode()
