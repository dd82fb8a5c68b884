"""Initial conditions of the reference constructor (cb_initial_condition)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from ._lib import check

MODES = {"random": 1, "given": 0, "diagonal": -1, "centre": -2, "thermal": -3}


def initial_condition(params, mode=1, n_bubbles=5, trad=0.2, deltar=0.0, test=0, position_seed=42,
                      thermal_seed=12345, xns=None):
    """(phi0, pi0, xns_text) at t = 0 for the given run parameters.

    Defaults are the reference's def.h values and hard-coded seeds; mode 1
    returns the __xns.dat text it generated, mode 0 takes it as ``xns``."""
    mode = MODES.get(mode, mode)
    N = params.n_grids ** params.d
    phi0, pi0 = np.empty(N), np.empty(N)
    ic = L.cb_ic_params(int(mode), int(n_bubbles), float(trad), float(deltar), int(test), int(position_seed),
                        int(thermal_seed))
    cap = 64 * 8 * max(int(n_bubbles), 1) + 64
    buf = C.create_string_buffer(cap)
    n = C.c_size_t()
    xin = None if xns is None else xns.encode()
    check(L.lib.cb_initial_condition(C.byref(params), C.byref(ic), xin, L.dptr(phi0), L.dptr(pi0), buf, cap,
                                     C.byref(n)))
    text = buf.value.decode() if n.value else None
    return phi0, pi0, text
