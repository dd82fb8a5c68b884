"""GPU power spectrum (hand-written FFT + shell binning) against numpy, the
reference's ComputePowerSpectrum output (golden) and the CPU oracle.

Bars: DFT 1e-12 of the largest mode; bin weights (mode counts) exact, which
pins the integer shell index of every mode; <k> per bin 1e-13; power per
bin 1e-10 relative for bins above 1e-8 of the peak (1e-10 of the peak
absolute below); FP32C fields: 1e-4 relative above 1e-7 of the peak. (At
1e-8 of the peak single shells of broad-band fields reach ~1.5e-4 after 50
steps: float rounding of the evolved field itself; the DFT runs in double.)
"""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, load_golden
from ic_helpers import bubbles, smooth_noise

pytestmark = pytest.mark.gpu


def dft(d, n, x):
    from coolbubble_b200 import _lib as L
    out = np.zeros(n ** (d - 1) * (n // 2 + 1) * 2)
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
    L.check(L.lib.cb_dft_r2c(d, n, L.dptr(x), L.dptr(out)))
    return out.view(np.complex128).reshape((n,) * (d - 1) + (n // 2 + 1,))


@pytest.mark.parametrize("d,n", [(1, 64), (1, 30), (1, 1000), (2, 48), (2, 96), (2, 384), (2, 100), (3, 12),
                                 (3, 16), (3, 64), (3, 192), (2, 28), (2, 39),
                                 # the register-resident kernels (powers of two, 64 .. 512)
                                 (2, 64), (2, 128), (2, 256), (2, 512), (3, 128), (3, 256)])
def test_dft_matches_numpy(d, n):
    rng = np.random.default_rng(d * 1000 + n)
    x = rng.standard_normal((n,) * d)
    got = dft(d, n, x)
    ref = np.fft.rfftn(x)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def check_rows(rows, ref_rows, tol=1e-10, floor=1e-8):
    assert rows.shape == ref_rows.shape
    np.testing.assert_allclose(rows[:, 0], ref_rows[:, 0], rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(rows[:, 1], ref_rows[:, 1], rtol=1e-13, atol=1e-13)
    peak = np.abs(ref_rows[:, 2]).max()
    big = np.abs(ref_rows[:, 2]) > floor * peak
    np.testing.assert_allclose(rows[big, 2], ref_rows[big, 2], rtol=tol)
    assert np.abs(rows[~big, 2] - ref_rows[~big, 2]).max(initial=0.0) <= tol * peak


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_spectrum_matches_reference_golden(name):
    import coolbubble_b200 as cb
    g = load_golden(name)
    m = g["meta"]
    p = cb.make_params(m["d"], m["n"], m["L"], m["c"], m["dt"], expansion=m.get("expansion", 0),
                       mpl=m.get("mpl", 200.0), alpha=m.get("alpha", 0))
    s = cb.Bubble(p, g["phi0"], g["pi0"])
    check_rows(s.ComputePowerSpectrum(), g["spec_start"])
    s.step(m["steps"], sums=True)
    check_rows(s.ComputePowerSpectrum(), g["spec_end"])


@pytest.mark.parametrize("case", [
    dict(d=2, n=512, L=32.0, c=4.0, ic="bubbles"),
    dict(d=2, n=384, L=48.0, c=3.0, ic="bubbles"),
    dict(d=3, n=128, L=32.0, c=2.0, ic="noise"),
    dict(d=3, n=64, L=16.0, c=2.0, ic="noise"),
    dict(d=2, n=64, L=16.0, c=4.0, ic="bubbles"),
    dict(d=3, n=96, L=24.0, c=4.0, ic="bubbles", expansion=1, mpl=10.0),
    dict(d=1, n=2048, L=64.0, c=4.0, ic="noise"),
])
def test_spectrum_matches_oracle(case):
    import coolbubble_b200 as cb
    from oracle import bridge as B
    d, n, L, c = case["d"], case["n"], case["L"], case["c"]
    dt = 0.1 * L / n
    phi0 = bubbles(d, n, L, c, 5, seed=9) if case["ic"] == "bubbles" else smooth_noise(d, n, 0.2, seed=8, kmax=12)
    kw = dict(expansion=case.get("expansion", 0), mpl=case.get("mpl", 200.0))
    s = cb.Bubble(cb.make_params(d, n, L, c, dt, **kw), phi0)
    o = B.Oracle(d, n, L, c, dt, phi0, None, **kw)
    s.step(30, sums=True)
    o.step(30)
    pw, ws, ks = s.spectrum_sums()
    opw, ows, oks = o.spectrum()
    np.testing.assert_array_equal(ws, ows)   # integer shells: every mode in the same bin
    m = ows > 0
    np.testing.assert_allclose(ks[m] / ws[m], oks[m] / ows[m], rtol=1e-13, atol=1e-13)
    ref = opw[m] / ows[m]
    got = pw[m] / ws[m]
    peak = ref.max()
    big = ref > 1e-8 * peak
    np.testing.assert_allclose(got[big], ref[big], rtol=1e-10)


@pytest.mark.parametrize("d,n", [(3, 128), (2, 256)])
def test_fp32c_spectrum_within_1e4(d, n):
    import coolbubble_b200 as cb
    from oracle import bridge as B
    L, c = (32.0, 2.0)
    dt = 0.1 * L / n
    phi0 = smooth_noise(d, n, 0.2, seed=21, kmax=10)
    s = cb.Bubble(cb.make_params(d, n, L, c, dt, precision="fp32c"), phi0)
    o = B.Oracle(d, n, L, c, dt, phi0, None)
    s.step(50, sums=True)
    o.step(50)
    pw, ws, _ = s.spectrum_sums()
    opw, ows, _ = o.spectrum()
    m = ows > 0
    ref, got = opw[m] / ows[m], pw[m] / ws[m]
    big = ref > 1e-7 * ref.max()
    np.testing.assert_allclose(got[big], ref[big], rtol=1e-4)
