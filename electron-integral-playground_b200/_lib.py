"""ctypes binding of the in-tree libmolecular_integral.so (the CUDA library).

The library is the product path: there is no CPU fallback.  Importing any
integral entry point raises if the shared object was not built
(``python -c "import __graft_entry__ as g; g.build()"`` builds it).
"""

import ctypes
import os
import pathlib

import numpy as np

LIB_PATH = pathlib.Path(os.environ.get("EIP_LIBRARY", pathlib.Path(__file__).resolve().parent / "lib" /
                                       "libmolecular_integral.so"))

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_lib = None


class IntegralError(RuntimeError):
    pass


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise IntegralError(f"CUDA integral library not built: {LIB_PATH} is missing")
        L = ctypes.CDLL(str(LIB_PATH))
        c_int, c_double, c_bool = ctypes.c_int, ctypes.c_double, ctypes.c_bool
        L.three_center.argtypes = [c_int, c_int, c_int, _dp, _dp, _dp, _dp, _ip, _ip, c_int, _dp, _dp, _ip, c_int,
                                   _dp, c_int, c_int, c_bool, c_double]
        L.two_center.argtypes = [c_int, c_int, _dp, _dp, _ip, c_int, _dp, _dp, _ip, c_int, _dp, c_int, c_bool,
                                 c_double]
        L.nuclear_attraction.argtypes = [c_int, c_int, _dp, _dp, _dp, _dp, _ip, _ip, c_int, _dp, c_int, _dp, c_int,
                                         c_bool, c_double]
        L.overlap.argtypes = [c_int, c_int, _dp, _dp, _dp, _ip, _ip, c_int, _dp, c_int, c_bool]
        for f in (L.three_center, L.two_center, L.nuclear_attraction, L.overlap):
            f.restype = c_int
        L.eip_init.argtypes = [c_int]
        L.eip_init.restype = c_int
        L.eip_last_error.restype = ctypes.c_char_p
        L.eip_kernel_launch_count.restype = ctypes.c_ulonglong
        L.eip_last_kernel_ms.restype = ctypes.c_float
        L.eip_tune_set.argtypes = [c_int, c_int, c_int, c_int]
        L.eip_tune_set.restype = c_int
        L.eip_tune_get.argtypes = [c_int, c_int, c_int]
        L.eip_tune_get.restype = c_int
        L.eip_tune_set_fp32.argtypes = [c_int, c_int, c_int, c_int]
        L.eip_tune_set_fp32.restype = c_int
        L.eip_tune_get_fp32.argtypes = [c_int, c_int, c_int]
        L.eip_tune_get_fp32.restype = c_int
        L.eip_boys.argtypes = [c_int, _dp, c_int, _dp]
        L.eip_boys.restype = c_int
        _lib = L
    return _lib


def dp(a):
    return a.ctypes.data_as(_dp)


def ip(a):
    return a.ctypes.data_as(_ip)


def check(rc, what):
    if rc == 1:
        raise IntegralError(f"{what}: unsupported angular momentum class")
    if rc != 0:
        msg = lib().eip_last_error().decode(errors="replace")
        raise IntegralError(f"{what} failed with status {rc}: {msg}")


def as_f64(a, shape_tail=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape_tail is not None and a.shape[1:] != shape_tail:
        raise ValueError(f"expected (n, {shape_tail}) array, got {a.shape}")
    return a


def as_i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def launch_count():
    return int(lib().eip_kernel_launch_count())


def device_boys(L, T):
    T = as_f64(np.atleast_1d(T))
    out = np.empty((T.shape[0], L + 1))
    check(lib().eip_boys(int(L), dp(T), int(T.shape[0]), dp(out)), "eip_boys")
    return out
