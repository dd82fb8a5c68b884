"""Ensembles: every member advanced together must give what it gives alone.

Bars: FP64 members' fields bit-identical to stepping the run alone (the
resident kernel does the same per-site arithmetic) and box averages within
1e-12 relative (only the summation order differs); FP32C members within 1e-5
(relative, fields normalised by their largest value) of the run alone."""
import numpy as np
import pytest

from ic_helpers import bubbles, smooth_noise

pytestmark = pytest.mark.gpu


def _member(d, n, L, c, prec, seed, thermal=False):
    import coolbubble_b200 as cb
    p = cb.make_params(d, n, L, c, 0.1 * L / n, precision=prec, memorysave=1)
    if thermal:
        phi0, pi0 = smooth_noise(d, n, 0.05, seed=seed, kmax=12), smooth_noise(d, n, 0.05, seed=seed + 1, kmax=12)
    else:
        phi0, pi0 = bubbles(d, n, L, c, 3 + seed % 5, seed=seed), None
    return p, phi0, pi0


SPECS = [
    (2, 128, 16.0, 3.0, "fp32c", 1, False),    # one CTA
    (2, 256, 32.0, 5.0, "fp32c", 2, True),     # 4-CTA cluster
    (2, 512, 32.0, 4.0, "fp32c", 3, False),    # 16-CTA cluster (or its own stream if a GPC cannot hold it)
    (2, 64, 8.0, 2.0, "fp64", 4, True),        # one CTA, double
    (2, 256, 32.0, 6.0, "fp64", 5, False),     # 8-CTA cluster, double
    (3, 32, 16.0, 4.0, "fp64", 6, False),      # own stream (d = 3)
    (2, 128, 16.0, 7.5, "fp32c", 7, True),
]


def test_members_match_their_solo_runs():
    import coolbubble_b200 as cb
    from coolbubble_b200.ensemble import Ensemble
    made = [_member(*s[:6], thermal=s[6]) for s in SPECS]
    mix = [cb.Bubble(p, a, b) for p, a, b in made]
    solo = [cb.Bubble(p, a, b) for p, a, b in made]
    ens = Ensemble(mix)
    plans = [ens.plan(i) for i in range(len(mix))]
    assert plans[0][0] == 1 and plans[1][0] == 4 and plans[3][0] == 1 and plans[4][0] == 8
    assert plans[5] == (0, 0)
    nsteps, every = 120, 40
    lines = ens.step(nsteps, every)
    for i, (s, spec) in enumerate(zip(solo, SPECS)):
        ref_lines = []
        for j in range(nsteps // every):
            ref_lines.append(s.step(every, sums=True))
        fa, fb = mix[i].fields(local=False), s.fields(local=False)
        prec = spec[4]
        for j, (got, ref) in enumerate(zip(lines[i], ref_lines)):
            assert got["t"] == ref["t"], (i, j)
            tol = 1e-12 if prec == "fp64" else 1e-5
            for k in ("etot", "ekin", "egrad", "epot", "etot_var", "ekin_var", "egrad_var", "epot_var",
                      "avphi_var", "avphip_var"):
                assert got[k] == pytest.approx(ref[k], rel=tol, abs=1e-300), (i, j, k)
            for k in ("avphi", "avphip"):
                scale = np.sqrt(spec[1] ** spec[0] * max(ref[k + "_var"], 1e-300))
                assert abs(got[k] - ref[k]) <= tol * max(scale, abs(ref[k]), 1e-300), (i, j, k)
        for k in ("phi", "pi"):
            if prec == "fp64":
                np.testing.assert_array_equal(fa[k], fb[k])
            else:
                assert np.abs(fa[k] - fb[k]).max() <= 1e-5 * np.abs(fb[k]).max(), (i, k)
        assert mix[i].sums()["t"] == s.sums()["t"], i   # the member's clock advanced as its solo run's


def test_ensemble_steps_continue_where_they_left_off():
    """Two ensemble calls equal one longer call (the fields stay in the runs)."""
    import coolbubble_b200 as cb
    from coolbubble_b200.ensemble import Ensemble
    p, a, b = _member(2, 128, 16.0, 4.0, "fp64", 11)
    x, y = cb.Bubble(p, a, b), cb.Bubble(p, a, b)
    ex, ey = Ensemble([x]), Ensemble([y])
    ex.step(30)
    ex.step(50)
    ey.step(80)
    np.testing.assert_array_equal(x.fields(local=False)["phi"], y.fields(local=False)["phi"])


def test_resident_fp64_members_match_the_oracle():
    """Resident double members (one CTA at 64^2, an 8-CTA cluster at 256^2)
    against the CPU restatement of the reference's step: fields within 1e-12 of
    their largest value and box averages within 1e-10 at every recorded line."""
    import coolbubble_b200 as cb
    from coolbubble_b200.ensemble import Ensemble
    from oracle import bridge as B
    specs = [(2, 64, 8.0, 2.0, "fp64", 4, True), (2, 256, 32.0, 6.0, "fp64", 5, False)]
    made = [_member(*s[:6], thermal=s[6]) for s in specs]
    runs = [cb.Bubble(p, a, b) for p, a, b in made]
    ens = Ensemble(runs)
    assert [ens.plan(i)[0] for i in range(2)] == [1, 8]
    nsteps, every = 80, 40
    lines = ens.step(nsteps, every)
    for i, ((p, phi0, pi0), spec) in enumerate(zip(made, specs)):
        d, n, L, c = spec[:4]
        o = B.Oracle(d, n, L, c, 0.1 * L / n, phi0, pi0)
        for j in range(nsteps // every):
            o.step(every)
            r = o.scalars()
            got = lines[i][j]
            for k, rk in (("etot", "Etot"), ("ekin", "Ekintot"), ("egrad", "Egradtot"), ("epot", "Epottot"),
                          ("etot_var", "EtotVar"), ("ekin_var", "EkintotVar")):
                assert abs(got[k] - r[rk]) <= 1e-10 * abs(r[rk]), (i, j, k, got[k], r[rk])
            assert got["t"] == r["t"]
        f, fo = runs[i].fields(local=False), o.fields()
        for k in ("phi", "pi"):
            assert np.abs(f[k] - fo[k]).max() <= 1e-12 * np.abs(fo[k]).max(), (i, k)
