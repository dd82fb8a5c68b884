"""Many runs stepped together (cb_ensemble_*)."""
from __future__ import annotations

import ctypes as C

from . import _lib as L
from ._lib import check

_h = C.c_void_p
L.lib.cb_ensemble_create.argtypes = [C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]
L.lib.cb_ensemble_create.restype = C.c_int
L.lib.cb_ensemble_step.argtypes = [_h, C.c_int, C.c_int, C.POINTER(L.cb_sums)]
L.lib.cb_ensemble_step.restype = C.c_int
L.lib.cb_ensemble_member_plan.argtypes = [_h, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
L.lib.cb_ensemble_member_plan.restype = C.c_int
L.lib.cb_ensemble_destroy.argtypes = [_h]
L.lib.cb_ensemble_destroy.restype = C.c_int


class Ensemble:
    """A set of Bubble runs advanced together; the runs stay usable on their own."""

    def __init__(self, members):
        self.members = list(members)
        arr = (C.c_void_p * len(self.members))(*[m._h.value for m in self.members])
        h = C.c_void_p()
        check(L.lib.cb_ensemble_create(len(self.members), arr, C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            L.lib.cb_ensemble_destroy(h)
        self._h = None

    def plan(self, m):
        cs, nt = C.c_int(), C.c_int()
        check(L.lib.cb_ensemble_member_plan(self._h, m, C.byref(cs), C.byref(nt)))
        return cs.value, nt.value

    def step(self, nsteps, sums_every=0):
        """Advance all members; returns [member][event] lines (dicts) when sums_every > 0."""
        nev = nsteps // sums_every if sums_every > 0 else 0
        out = (L.cb_sums * max(1, len(self.members) * nev))()
        check(L.lib.cb_ensemble_step(self._h, int(nsteps), int(sums_every), out if nev else None))
        return [[out[m * nev + j].asdict() for j in range(nev)] for m in range(len(self.members))]
