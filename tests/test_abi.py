"""The C ABI library loads, exports every declared entry point, and rejects
bad arguments on the host (no GPU needed)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names += re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\**\s*(cb_[a-z_0-9]+)\s*\(", src, flags=re.M)
    return names


def test_library_exports_every_declared_symbol():
    from coolbubble_b200 import _lib as L
    names = declared_functions()
    assert len(names) >= 14
    missing = [n for n in names if not hasattr(L.lib, n)]
    assert not missing, missing


def test_nbins_matches_reference_formula():
    from coolbubble_b200 import _lib as L
    for d, n, exp in ((2, 512, 363), (3, 256, 222), (3, 512, 444), (1, 100, 51)):
        assert L.lib.cb_nbins(d, n) == exp
    assert L.lib.cb_nbins(4, 10) == L.CB_EINVAL


@pytest.mark.parametrize("kw,msg", [
    (dict(d=4), "d must be"),
    (dict(n_grids=1), "n_grids"),
    (dict(L_box=-1.0), "L must be"),
    (dict(dt=0.2), "stability condition"),
    (dict(precision=7), "precision"),
    (dict(alpha=2), "alpha"),
])
def test_create_rejects_bad_parameters(kw, msg):
    import coolbubble_b200 as cb
    base = dict(d=2, n_grids=32, L_box=8.0, c=4.0, dt=0.025)
    base.update(kw)
    p = cb.make_params(**base)
    with pytest.raises(cb.CBError) as e:
        cb.Bubble(p, np.zeros(max(p.n_grids, 1) ** p.d))
    assert msg in str(e.value)
    assert e.value.status == -1


def test_footprint_counts_fields_and_local_arrays():
    import coolbubble_b200 as cb
    from coolbubble_b200 import _lib as L
    p = cb.make_params(3, 64, 8.0, 4.0, 0.01, precision="fp32c", memorysave=1)
    q = cb.make_params(3, 64, 8.0, 4.0, 0.01, precision="fp64", memorysave=0)
    fp = L.lib.cb_footprint_bytes(C.byref(p))
    fq = L.lib.cb_footprint_bytes(C.byref(q))
    assert fp >= 4 * 4 * 64 ** 3
    assert fq >= 7 * 8 * 64 ** 3
