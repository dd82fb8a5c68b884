"""ctypes binding of the C ABI in include/coolbubble_b200.h.

The library is the in-tree build ``coolbubble_b200/lib/libcoolbubble_b200.so``
(``python -c "import __graft_entry__; __graft_entry__.build()"`` or
``make -C coolbubble_b200/csrc``). There is no fallback: if the library is
missing, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libcoolbubble_b200.so")

CB_OK, CB_EINVAL, CB_ENOMEM, CB_EDEVICE, CB_ETIMEOUT, CB_EUNSUPPORTED, CB_EBUSY, CB_ENOTFOUND = 0, -1, -2, -3, -4, -5, -6, -7
CB_EIO = -8
CB_FP64, CB_FP32C = 0, 1
CB_STEP_SUMS, CB_STEP_LOCAL = 1, 2


class cb_params(C.Structure):
    _fields_ = [("d", C.c_int), ("n_grids", C.c_int), ("L", C.c_double), ("c", C.c_double), ("dt", C.c_double),
                ("alpha", C.c_int), ("expansion", C.c_int), ("mpl", C.c_double), ("delta_v", C.c_double),
                ("precision", C.c_int), ("memorysave", C.c_int)]


class cb_ic_params(C.Structure):
    _fields_ = [("mode", C.c_int), ("n_bubbles", C.c_int), ("trad", C.c_double), ("deltar", C.c_double),
                ("test", C.c_int), ("position_seed", C.c_uint), ("thermal_seed", C.c_uint64)]


class cb_scalars(C.Structure):
    _fields_ = [("t", C.c_double), ("a", C.c_double), ("ap", C.c_double), ("H", C.c_double),
                ("ekin_half_prev", C.c_double), ("etot0", C.c_double)]


SUM_FIELDS = ("t", "a", "H", "C", "etot", "ekin", "egrad", "epot", "etot_var", "ekin_var", "egrad_var", "epot_var",
              "avphi", "avphi_var", "avphip", "avphip_var", "ap", "ekin_half_prev", "w", "etot_drift", "c_rel")


class cb_sums(C.Structure):
    _fields_ = [(f, C.c_double) for f in SUM_FIELDS]

    def asdict(self):
        return {f: getattr(self, f) for f in SUM_FIELDS}


class CBError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{message} (status {status})")
        self.status = status


if not os.path.exists(LIB_PATH):
    raise ImportError(f"CUDA library not built: {LIB_PATH} is missing "
                      "(run make -C coolbubble_b200/csrc or __graft_entry__.build())")

lib = C.CDLL(LIB_PATH)

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_h = C.c_void_p

_SIGS = {
    "cb_create": (C.c_int, [C.POINTER(cb_params), _dp, _dp, C.POINTER(cb_scalars), C.POINTER(_h)]),
    "cb_create_from_ic": (C.c_int, [C.POINTER(cb_params), _dp, _dp, C.POINTER(cb_sums), C.POINTER(_h)]),
    "cb_step": (C.c_int, [_h, C.c_int, C.c_int, C.POINTER(cb_sums)]),
    "cb_step_timed": (C.c_int, [_h, C.c_int, C.c_int, _dp]),
    "cb_sync": (C.c_int, [_h]),
    "cb_timer_start": (C.c_int, [_h]),
    "cb_timer_stop": (C.c_int, [_h, _dp]),
    "cb_set_device": (C.c_int, [C.c_int]),
    "cb_get_counters": (C.c_int, [_h, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "cb_pinned_alloc": (C.c_void_p, [C.c_size_t]),
    "cb_pinned_free": (C.c_int, [C.c_void_p]),
    "cb_get_sums": (C.c_int, [_h, C.POINTER(cb_sums)]),
    "cb_device_error": (C.c_int, [_h, C.POINTER(C.c_int)]),
    "cb_get_fields": (C.c_int, [_h, _dp, _dp, _dp, _dp, _dp]),
    "cb_get_fields_f32": (C.c_int, [_h, _fp, _fp, _fp, _fp, _fp]),
    "cb_get_line": (C.c_int, [_h, C.c_int, C.c_int, C.c_int, C.c_int, _dp]),
    "cb_nbins": (C.c_int, [C.c_int, C.c_int]),
    "cb_power_spectrum": (C.c_int, [_h, _dp, _dp, _dp, C.c_int]),
    "cb_dft_r2c": (C.c_int, [C.c_int, C.c_int, _dp, _dp]),
    "cb_dft_c2r": (C.c_int, [C.c_int, C.c_int, _dp, _dp]),
    "cb_initial_condition": (C.c_int, [C.POINTER(cb_params), C.POINTER(cb_ic_params), C.c_char_p, _dp, _dp,
                                       C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "cb_h5_write_floats": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.c_int,
                                     C.POINTER(C.c_char_p), C.POINTER(_fp), C.c_int, C.POINTER(C.c_char_p), _dp,
                                     C.c_int, C.c_int]),
    "cb_out_field": (C.c_int, [_h, C.c_char_p, C.c_int]),
    "cb_out_field_async": (C.c_int, [_h, C.c_char_p, C.c_int]),
    "cb_out_field_wait": (C.c_int, [_h]),
    "cb_destroy": (C.c_int, [_h]),
    "cb_step_static_noalloc": (C.c_int, [C.POINTER(cb_params), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_double, C.POINTER(cb_sums)]),
    "cb_last_error": (C.c_char_p, [_h]),
    "cb_status_string": (C.c_char_p, [C.c_int]),
    "cb_footprint_bytes": (C.c_int64, [C.POINTER(cb_params)]),
}

for _name, (_res, _args) in _SIGS.items():
    if hasattr(lib, _name):
        _f = getattr(lib, _name)
        _f.restype = _res
        _f.argtypes = _args


def check(status, handle=None):
    if status != CB_OK:
        msg = lib.cb_last_error(handle)
        raise CBError(status, (msg or b"").decode() or lib.cb_status_string(status).decode())
    return status


def dptr(a):
    return None if a is None else a.ctypes.data_as(_dp)


def fptr(a):
    return None if a is None else a.ctypes.data_as(_fp)


def pinned_array(n, dtype):
    """A numpy array over page-locked host memory (freed with the array's owner)."""
    import numpy as np
    dtype = np.dtype(dtype)
    nbytes = int(n) * dtype.itemsize
    p = lib.cb_pinned_alloc(nbytes)
    if not p:
        raise MemoryError("cb_pinned_alloc failed")
    buf = (C.c_char * nbytes).from_address(p)
    arr = np.frombuffer(buf, dtype=dtype, count=int(n))
    return arr, p
