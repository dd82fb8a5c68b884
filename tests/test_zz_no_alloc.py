"""The allocation-free step (cb_step_static_noalloc) against the handle path.

Callers that own all device memory themselves pass their own buffers; the
step's scratch is the library's fixed array. This file is collected last so
that a run stopping at the first failure has run every other test already.
Device buffers come from torch (plumbing only); the step itself runs through
the C ABI. Tolerances are those of the other step tests: fields 1e-12 of
their largest value, box averages 1e-10 relative."""
import ctypes as C

import numpy as np
import pytest

from ic_helpers import bubbles, smooth_noise

pytestmark = pytest.mark.gpu


def _dev(a, torch, dtype):
    return torch.tensor(a, dtype=dtype, device="cuda")


@pytest.mark.parametrize("case", [
    dict(d=3, n=64, L=16.0, c=4.0, precision="fp64"),     # tiled d = 3 kernel
    dict(d=2, n=96, L=30.0, c=5.0, precision="fp64"),     # generic kernel, exact-division path
    dict(d=3, n=128, L=32.0, c=2.0, precision="fp32c"),
    dict(d=2, n=1024, L=128.0, c=4.0, precision="fp32c"),   # d = 2 column-strip kernel (from 1024^2 sites)
    dict(d=1, n=1 << 20, L=131072.0, c=4.0, precision="fp64"),   # the strip kernel on one row (d = 1, 2^20 sites)
])
def test_noalloc_two_steps_match_handle_path(case):
    torch = pytest.importorskip("torch")
    import coolbubble_b200 as cb
    from coolbubble_b200 import _lib as L
    d, n, Lb, c = case["d"], case["n"], case["L"], case["c"]
    dt = 0.1 * Lb / n
    p = cb.make_params(d, n, Lb, c, dt, precision=case["precision"], memorysave=1)
    phi0 = bubbles(d, n, Lb, c, 4, seed=3)
    pi0 = smooth_noise(d, n, 0.02, seed=8)
    s = cb.Bubble(p, phi0, pi0)
    start = s.fields(local=False)
    ref = []
    for _ in range(2):
        sums = s.step(1, sums=True)
        ref.append((sums, s.fields(local=False)))
    tdt = torch.float64 if case["precision"] == "fp64" else torch.float32
    bufs = [_dev(start["phi"], torch, tdt), _dev(start["pi"], torch, tdt),
            torch.empty(n ** d, dtype=tdt, device="cuda"), torch.empty(n ** d, dtype=tdt, device="cuda")]
    torch.cuda.synchronize()
    t = 0.0
    for it in range(2):
        out = L.cb_sums()
        rc = L.lib.cb_step_static_noalloc(C.byref(p), bufs[0].data_ptr(), bufs[1].data_ptr(), bufs[2].data_ptr(),
                                          bufs[3].data_ptr(), t, C.byref(out))
        L.check(rc)
        got = out.asdict()
        rs, rf = ref[it]
        for k in ("etot", "ekin", "egrad", "epot", "avphi", "avphip", "etot_var", "ekin_var", "a", "t"):
            assert got[k] == pytest.approx(rs[k], rel=1e-10, abs=1e-300), (it, k)
        phi = bufs[2].double().cpu().numpy()
        pi = bufs[3].double().cpu().numpy()
        for name, a in (("phi", phi), ("pi", pi)):
            r = rf[name]
            assert np.abs(a - r).max() <= 1e-12 * np.abs(r).max(), (it, name)
        bufs = [bufs[2], bufs[3], bufs[0], bufs[1]]
        t = got["t"]


def test_noalloc_rejects_lattice_beyond_scratch():
    import coolbubble_b200 as cb
    from coolbubble_b200 import _lib as L
    p = cb.make_params(2, 8192, 512.0, 4.0, 0.005, precision="fp32c", memorysave=1)
    out = L.cb_sums()
    rc = L.lib.cb_step_static_noalloc(C.byref(p), 16, 32, 48, 64, 0.0, C.byref(out))
    assert rc == L.CB_EINVAL
    assert b"too large for the fixed scratch" in L.lib.cb_last_error(None)
