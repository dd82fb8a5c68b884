"""Parity at the benchmark configurations' own sizes, against the reference
itself (its src/bubble.cpp built in place: oracle/_ref), each run from the
reference's own seeded start.

  512^2, d = 2, L = 32, c = 4, mode 1 with 5 bubbles (srand(42)), static:
      the generic tile kernel at its launch-bound size, 200 steps
  256^3, d = 3, L = 32, c = 4, mode 1 with 8 bubbles (radius 1.3x), expanding,
      Mpl = 10: the staged kernel with drift-first ordering, 100 steps
  512^3, d = 3, L = 64, c = 2, mode -3 thermal, Trad = 0.05, static: the staged
      kernel's largest geometry (two-row double tiles, 24 plane parts), 40
      steps -- the reference's host step at this size takes about a second,
      so the comparison stops there

Per case the library's host IC (cb_initial_condition) and device set-up
(cb_create_from_ic) must reproduce the reference constructor's state, then
both evolve with dt = 0.1 dx:
  FP64 fields: max|gpu - ref| <= 1e-12 max|ref| at the end;
  FP64 box averages, a, a', H (C on the H^2 scale) and the line checks
      (w, energy drift, C/H^2) within 1e-10 at every compared line;
  bubble placement (__xns.dat bytes) exact; the spectrum's shells exact
      (<k> per shell to 1e-13 pins each shell's mode count), power 1e-10
      relative above 1e-8 of the peak;
  FP32C on the same start: energies within 1e-5 of the reference (Etot
      scale for the kinetic energy); its spectrum's error is reported in
      tests/fp32c_report.py.
"""
import numpy as np
import pytest

from test_step_gpu import FIELD_TOL, check_line_checks, check_sums, field_err

pytestmark = pytest.mark.gpu

CASES = {
    "bubbles-d2-n512": dict(d=2, n=512, L=32.0, c=4.0, mode=1, nb=5, trad=0.2, expansion=0, mpl=200.0,
                            steps=200, every=40, memorysave=0),
    "bubbles-d3-n256-expanding": dict(d=3, n=256, L=32.0, c=4.0, mode=1, nb=8, trad=0.2, expansion=1, mpl=10.0,
                                      steps=100, every=20, memorysave=0),
    "thermal-d3-n512": dict(d=3, n=512, L=64.0, c=2.0, mode=-3, nb=5, trad=0.05, expansion=0, mpl=200.0,
                            steps=40, every=20, memorysave=1),
}


def spectrum_check(rows, ref_rows, tol, floor=1e-8):
    assert rows.shape == ref_rows.shape
    np.testing.assert_allclose(rows[:, 0], ref_rows[:, 0], rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(rows[:, 1], ref_rows[:, 1], rtol=1e-13, atol=1e-13)
    big = ref_rows[:, 2] > floor * ref_rows[:, 2].max()
    err = np.abs(rows[big, 2] / ref_rows[big, 2] - 1.0).max()
    assert err <= tol, err
    return err


@pytest.mark.parametrize("name", list(CASES))
def test_config_matches_reference(name):
    import coolbubble_b200 as cb
    from coolbubble_b200.ic import initial_condition
    from oracle import bridge as B
    if not B.reference_available():
        pytest.skip("the reference build (oracle/_ref) is not present")
    cs = CASES[name]
    d, n, L, c = cs["d"], cs["n"], cs["L"], cs["c"]
    dt = 0.1 * L / n
    N = n ** d
    ms = cs["memorysave"]
    ref = B.Reference(d, n, L, c, cs["mode"], dt, nbubbles=cs["nb"], trad=cs["trad"], expansion=cs["expansion"],
                      mpl=cs["mpl"], memorysave=ms, nt=cs["steps"])
    sc0 = ref.scalars()
    f0 = ref.fields()

    # the start: host IC + device set-up against the reference constructor
    kw = dict(expansion=cs["expansion"], mpl=cs["mpl"], memorysave=ms)
    p64 = cb.make_params(d, n, L, c, dt, precision="fp64", **kw)
    phi0, pi0, xns = initial_condition(p64, mode=cs["mode"], n_bubbles=cs["nb"], trad=cs["trad"])
    if cs["mode"] == 1:
        assert xns == ref.xns_text()                      # positions and images, byte for byte
        np.testing.assert_array_equal(phi0, f0["phi"])    # profiles built from them: bit-exact
    s = cb.Bubble(p64, phi0, pi0)
    g = s.fields(local=ms == 0)
    assert field_err(g["phi"], f0["phi"]) <= FIELD_TOL
    assert field_err(g["pi"], f0["pi"]) <= FIELD_TOL
    for k, rk in (("etot", "Etot"), ("egrad", "Egradtot"), ("epot", "Epottot"), ("a", "a"), ("ap", "ap"),
                  ("H", "H"), ("ekin_half_prev", "EkinHalfPrev")):
        assert abs(s.last[k] - sc0[rk]) <= 1e-10 * max(abs(sc0[rk]), 1e-300), (k, s.last[k], sc0[rk])
    s32 = cb.Bubble(cb.make_params(d, n, L, c, dt, precision="fp32c", **kw), phi0, pi0)
    del phi0, pi0, g, f0

    # the evolution, compared at every `every`-th step
    done = 0
    while done < cs["steps"]:
        k = cs["every"]
        ref.step(k)
        done += k
        last = done >= cs["steps"]
        got = s.step(k, sums=True, local=last and ms == 0)
        r = ref.scalars()
        check_sums(got, r, N, where=(name, done))
        check_line_checks(got, r, d, sc0["Etot"], where=(name, done))
        assert got["t"] == r["t"]
        g32 = s32.step(k, sums=True)
        for key, rk in (("etot", "Etot"), ("egrad", "Egradtot"), ("epot", "Epottot")):
            assert abs(g32[key] - r[rk]) <= 1e-5 * abs(r[rk]), (name, done, key, g32[key], r[rk])
        assert abs(g32["ekin"] - r["Ekintot"]) <= 1e-5 * abs(r["Etot"])
        assert abs(g32["a"] - r["a"]) <= 1e-10 * r["a"]
    f, fr = s.fields(local=ms == 0), ref.fields()
    for key in ("phi", "pi") + (("ekin", "egrad", "epot") if ms == 0 else ()):
        assert field_err(f[key], fr[key]) <= FIELD_TOL, (key, field_err(f[key], fr[key]))
    del f, fr

    # the snapshot spectrum (FourierTransform + ComputePowerSpectrum, bubble.cpp:642-709)
    spectrum_check(s.ComputePowerSpectrum(), ref.spectrum_lines(), tol=1e-10)
