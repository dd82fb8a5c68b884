"""The request loop (cb_pool_*): runs kept resident on the GPU, admitted
against a device-memory budget, advanced concurrently."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from ._lib import check

QUEUED, RUNNING, DONE, FAILED, CANCELLED = 0, 1, 2, 3, 4
INJECT_ADMISSION_FAILURE, INJECT_WORKER_EXCEPTION = 1, 2


class cb_request(C.Structure):
    _fields_ = [("params", L.cb_params), ("ic", L.cb_ic_params), ("nt", C.c_int), ("sums_every", C.c_int),
                ("want_fields", C.c_int)]


class cb_pool_stats(C.Structure):
    _fields_ = [(f, C.c_int64) for f in ("queued", "active", "completed", "failed", "cancelled", "admitted",
                                         "used_bytes", "budget_bytes")] + \
               [("site_updates", C.c_double), ("busy_s", C.c_double), ("wall_s", C.c_double)]


_p = C.c_void_p
_S = {
    "cb_pool_create": (C.c_int, [C.c_int64, C.c_int, C.POINTER(_p)]),
    "cb_pool_submit": (C.c_int, [_p, C.POINTER(cb_request), C.c_char_p, C.POINTER(C.c_int64)]),
    "cb_pool_status": (C.c_int, [_p, C.c_int64, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "cb_pool_wait": (C.c_int, [_p, C.c_int64, C.c_int]),
    "cb_pool_result": (C.c_int, [_p, C.c_int64, C.POINTER(L.cb_sums), C.c_int, C.POINTER(C.c_int),
                                 C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_double), C.c_char_p,
                                 C.c_size_t]),
    "cb_pool_cancel": (C.c_int, [_p, C.c_int64]),
    "cb_pool_get_stats": (C.c_int, [_p, C.POINTER(cb_pool_stats)]),
    "cb_pool_inject_failure": (C.c_int, [_p, C.c_int]),
    "cb_pool_destroy": (C.c_int, [_p]),
    "cb_create_from_seed": (C.c_int, [C.POINTER(L.cb_params), C.POINTER(L.cb_ic_params), C.c_char_p,
                                      C.POINTER(L.cb_sums), C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t),
                                      C.POINTER(_p)]),
}
for _n, (_r, _a) in _S.items():
    getattr(L.lib, _n).restype = _r
    getattr(L.lib, _n).argtypes = _a


def ic_params(mode=1, n_bubbles=5, trad=0.2, deltar=0.0, test=0, position_seed=42, thermal_seed=12345):
    return L.cb_ic_params(int(mode), int(n_bubbles), float(trad), float(deltar), int(test), int(position_seed),
                          int(thermal_seed))


class Pool:
    def __init__(self, budget_bytes, max_active):
        h = C.c_void_p()
        check(L.lib.cb_pool_create(int(budget_bytes), int(max_active), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            L.lib.cb_pool_destroy(self._h)
        self._h = None

    def __del__(self):
        self.close()

    def submit(self, params, ic, nt, sums_every=40, want_fields=False, xns=None):
        req = cb_request(params, ic, int(nt), int(sums_every), 1 if want_fields else 0)
        rid = C.c_int64()
        check(L.lib.cb_pool_submit(self._h, C.byref(req), None if xns is None else xns.encode(), C.byref(rid)))
        return rid.value

    def status(self, rid):
        st, done = C.c_int(), C.c_int()
        check(L.lib.cb_pool_status(self._h, int(rid), C.byref(st), C.byref(done)))
        return st.value, done.value

    def wait(self, rid, timeout_ms=600000):
        return L.lib.cb_pool_wait(self._h, int(rid), int(timeout_ms))

    def result(self, rid, n_sites=0, max_lines=4096):
        lines = (L.cb_sums * max_lines)()
        nl = C.c_int()
        lat = C.c_double()
        err = C.create_string_buffer(512)
        phi = np.zeros(n_sites, dtype=np.float32) if n_sites else None
        pi = np.zeros(n_sites, dtype=np.float32) if n_sites else None
        rc = L.lib.cb_pool_result(self._h, int(rid), lines, max_lines, C.byref(nl), L.fptr(phi), L.fptr(pi),
                                  C.byref(lat), err, 512)
        st, _ = self.status(rid)
        return dict(rc=rc, state=st, lines=[lines[i].asdict() for i in range(min(nl.value, max_lines))], phi=phi,
                    pi=pi, latency=lat.value, err=err.value.decode())

    def cancel(self, rid):
        check(L.lib.cb_pool_cancel(self._h, int(rid)))

    def stats(self):
        s = cb_pool_stats()
        check(L.lib.cb_pool_get_stats(self._h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in cb_pool_stats._fields_}

    def inject(self, kind):
        check(L.lib.cb_pool_inject_failure(self._h, int(kind)))


def create_from_seed(params, ic):
    """A Bubble whose start is built on the device (cb_create_from_seed)."""
    from .bubble import Bubble
    h = C.c_void_p()
    s = L.cb_sums()
    check(L.lib.cb_create_from_seed(C.byref(params), C.byref(ic), None, C.byref(s), None, 0, None, C.byref(h)))
    b = Bubble.__new__(Bubble)
    b.params = params
    b.d, b.n = params.d, params.n_grids
    b.N = b.n ** b.d
    b._h = h
    b._set(s.asdict())
    return b
