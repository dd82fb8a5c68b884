"""Pins the CPU restatement (oracle/cb_oracle.cpp) to the reference.

1. Against tests/golden/ (made by tests/golden/make_golden.py from the
   reference's own bubble.cpp): set-up, every step's scalars, final fields and
   spectra. Runs anywhere.
2. Directly against the reference built in place (oracle/_ref), when its
   sources are present, on an extra randomised case.
"""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, load_golden
from oracle import bridge as B

SCAL = B.SCALAR_NAMES


def _oracle_for(g):
    m = g["meta"]
    return B.Oracle(m["d"], m["n"], m["L"], m["c"], m["dt"], g["phi0"], g["pi0"], alpha=m.get("alpha", 0),
                    expansion=m.get("expansion", 0), mpl=m.get("mpl", 200.0))


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_oracle_matches_golden(name):
    g = load_golden(name)
    o = _oracle_for(g)
    f = o.fields()
    # set-up (bubble.cpp:236-291) is elementwise-identical arithmetic
    np.testing.assert_array_equal(f["phi"], g["phi_start"])
    np.testing.assert_allclose(f["pi"], g["pi_start"], rtol=0, atol=1e-15 * max(1.0, np.abs(g["pi_start"]).max()))
    for k in ("ekin", "egrad", "epot"):
        np.testing.assert_allclose(f[k], g[k + "_start"], rtol=1e-14, atol=1e-300)
    s0 = o.scalars()
    ref0 = dict(zip(SCAL, g["scalars"][0]))
    for k in ("t", "a", "ap", "H", "Etot", "Ekintot", "Egradtot", "Epottot", "avphi", "avphiP", "EkinHalfPrev"):
        assert s0[k] == pytest.approx(ref0[k], rel=1e-13, abs=1e-300), k
    steps = g["meta"]["steps"]
    for it in range(1, steps + 1):
        o.step(1)
        s = o.scalars()
        ref = dict(zip(SCAL, g["scalars"][it]))
        for k in SCAL:
            if k == "C":   # H^2 - rho/(3 Mpl^2) cancels: compared on the scale of H^2
                assert abs(s[k] - ref[k]) <= 1e-12 * max(ref["H"] ** 2, 1e-300), it
            elif k in ("avphi", "avphiP"):   # signed sums: compared on sum |x| <= sqrt(N * sum x^2)
                scale = np.sqrt(o.N * ref[k + "Var"])
                assert abs(s[k] - ref[k]) <= 1e-12 * max(scale, 1e-300), (it, k)
            else:
                assert s[k] == pytest.approx(ref[k], rel=1e-12, abs=1e-300), (it, k)
    f = o.fields()
    for k in ("phi", "pi", "ekin", "egrad", "epot"):
        r = g[k + "_end"]
        err = np.abs(f[k] - r).max() / max(np.abs(r).max(), 1e-300)
        assert err <= 1e-13, (k, err)
    pw, ws, ks = o.spectrum()
    m = ws > 0
    rows = g["spec_end"]
    assert rows.shape[0] == m.sum()
    np.testing.assert_allclose(ks[m] / ws[m], rows[:, 0], rtol=1e-14, atol=1e-14)
    np.testing.assert_allclose(pw[m] / ws[m], rows[:, 2], rtol=1e-12, atol=1e-12 * np.abs(rows[:, 2]).max())


def test_spectrum_bins_are_integer_shells():
    for d, n in ((1, 64), (2, 48), (3, 12), (3, 16)):
        b = B.bins(d, n)
        h = n // 2 + 1
        idx = np.indices((n,) * (d - 1) + (h,)).reshape(d, -1)
        sig = [np.where(i <= n // 2, i, i - n) for i in idx[:-1]] + [idx[-1]]
        n2 = sum(s.astype(np.int64) ** 2 for s in sig)
        exp = np.floor(np.sqrt(n2.astype(np.float64))).astype(np.int64)
        exp[exp >= B.nbins(d, n)] = -1
        np.testing.assert_array_equal(b, exp)


@pytest.mark.parametrize("d,n", [(1, 30), (2, 24), (3, 12), (2, 16), (3, 10)])
def test_cpu_dft_matches_numpy(d, n):
    rng = np.random.default_rng(d * 100 + n)
    x = rng.standard_normal((n,) * d)
    got = B.r2c(d, n, x).reshape((n,) * (d - 1) + (n // 2 + 1,))
    np.testing.assert_allclose(got, np.fft.rfftn(x), rtol=0, atol=1e-12 * np.abs(got).max())
    back = B.c2r(d, n, got.copy())
    np.testing.assert_allclose(back.reshape(x.shape), x * n ** d, rtol=0, atol=1e-11 * n ** d)


needs_ref = pytest.mark.skipif(not B.reference_available(), reason="reference sources not present")


@needs_ref
def test_oracle_matches_reference_live():
    """Fresh case straight against the reference (not from fixtures)."""
    import subprocess, sys, json, os
    code = r"""
import sys, json, numpy as np
sys.path.insert(0, %r)
from oracle import bridge as B
d, n, L, c = 2, 40, 20.0, 5.0
dt = 0.1 * L / n
r0 = B.Reference(d, n, L, c, -3, 0.0, trad=0.08); f = r0.fields(); phi0, pi0 = f['phi'], f['pi']; del r0
r = B.Reference(d, n, L, c, -3, dt, trad=0.08)
o = B.Oracle(d, n, L, c, dt, phi0, pi0)
r.step(50); o.step(50)
a, b = r.fields(), o.fields()
print(json.dumps({k: float(np.abs(a[k]-b[k]).max()) for k in ('phi','pi','ekin','egrad','epot')}))
""" % os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True).stdout
    errs = json.loads(out.strip().splitlines()[-1])
    assert max(errs.values()) == 0.0, errs
