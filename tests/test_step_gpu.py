"""GPU parity of the fused step kernels against the reference (golden
fixtures) and the CPU restatement (oracle), through the C ABI.

Bars (stated here, applied below):
  FP64 fields: max|gpu - ref| / max(max|ref|, 1e-300) <= 1e-12 over the run
  FP64 box averages and a, a', H: relative 1e-10 (C on the scale of H^2;
      signed sums <phi>, <phi'> on the scale sqrt(N * sum x^2) >= sum |x|)
  FP32C box averages: relative 1e-5 of the FP64 oracle (Etot scale for the
      kinetic energy, which starts near 0 for bubbles)
"""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, load_golden
from ic_helpers import bubbles, smooth_noise

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-12
SUM_TOL = 1e-10
SUM_KEYS = {"etot": "Etot", "ekin": "Ekintot", "egrad": "Egradtot", "epot": "Epottot", "a": "a", "ap": "ap",
            "H": "H", "ekin_half_prev": "EkinHalfPrev", "etot_var": "EtotVar", "ekin_var": "EkintotVar",
            "egrad_var": "EgradtotVar", "epot_var": "EpottotVar", "avphi_var": "avphiVar",
            "avphip_var": "avphiPVar"}


def field_err(a, ref):
    return float(np.abs(a - ref).max() / max(np.abs(ref).max(), 1e-300))


def check_sums(got, ref, N, tol=SUM_TOL, where=""):
    """got: cb_sums dict; ref: oracle/reference scalars dict (18 names)."""
    for k, rk in SUM_KEYS.items():
        r = ref[rk]
        assert abs(got[k] - r) <= tol * max(abs(r), 1e-300), (where, k, got[k], r)
    for k, rk in (("avphi", "avphi"), ("avphip", "avphiP")):
        scale = np.sqrt(N * ref[rk + "Var"]) if ref[rk + "Var"] > 0 else abs(ref[rk])
        assert abs(got[k] - ref[rk]) <= tol * max(scale, 1e-300), (where, k, got[k], ref[rk])
    assert abs(got["C"] - ref["C"]) <= tol * max(ref["H"] ** 2, 1e-300), (where, "C", got["C"], ref["C"])


def check_scale(key, s):
    """Scale on which a line's checks compare: the drift Etot/Etot0 - 1 on that
    of Etot/Etot0 (its error is Etot's relative error), C/H^2 on 1 + |C/H^2|,
    w on the sum of its terms' magnitudes over |Etot|."""
    if key == "etot_drift":
        return 1.0 + abs(s["etot_drift"])
    if key == "c_rel":
        return 1.0 + abs(s["c_rel"])
    if key == "w":
        return (abs(s["ekin"]) + abs(s["egrad"]) + abs(s["epot"])) / max(abs(s["etot"]), 1e-300)
    return 0.0


def w_of(ref, d):
    """Equation of state of a reference line (python/plot_SummaryPlots.py:91-95)."""
    return (ref["Ekintot"] - (d - 2) / d * ref["Egradtot"] - ref["Epottot"]) / ref["Etot"]


def check_line_checks(got, ref, d, etot0, tol=SUM_TOL, where=""):
    """w, the energy drift and C/H^2 of a line against those formed from the
    reference's own scalars (etot0: the reference's t = 0 total energy)."""
    w = w_of(ref, d)
    assert abs(got["w"] - w) <= tol * check_scale("w", got), (where, "w", got["w"], w)
    drift = ref["Etot"] / etot0 - 1.0
    assert abs(got["etot_drift"] - drift) <= tol * (1.0 + abs(drift)), (where, "drift", got["etot_drift"], drift)
    c_rel = ref["C"] / ref["H"] ** 2 if ref["H"] != 0 else 0.0
    assert abs(got["c_rel"] - c_rel) <= tol * (1.0 + abs(c_rel)), (where, "c_rel", got["c_rel"], c_rel)


def params_from(meta, precision="fp64", memorysave=0):
    import coolbubble_b200 as cb
    return cb.make_params(meta["d"], meta["n"], meta["L"], meta["c"], meta["dt"], alpha=meta.get("alpha", 0),
                          expansion=meta.get("expansion", 0), mpl=meta.get("mpl", 200.0), precision=precision,
                          memorysave=memorysave)


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_fp64_matches_reference_golden(name):
    import coolbubble_b200 as cb
    from oracle.bridge import SCALAR_NAMES
    g = load_golden(name)
    m = g["meta"]
    s = cb.Bubble(params_from(m), g["phi0"], g["pi0"])
    f = s.fields()
    # set-up on the device (bubble.cpp:236-291)
    assert field_err(f["phi"], g["phi_start"]) == 0.0
    assert field_err(f["pi"], g["pi_start"]) <= FIELD_TOL
    for k in ("ekin", "egrad", "epot"):
        assert field_err(f[k], g[k + "_start"]) <= FIELD_TOL, k
    ref0 = dict(zip(SCALAR_NAMES, g["scalars"][0]))
    for k, rk in (("etot", "Etot"), ("ekin", "Ekintot"), ("egrad", "Egradtot"), ("epot", "Epottot"), ("a", "a"),
                  ("ap", "ap"), ("H", "H"), ("ekin_half_prev", "EkinHalfPrev")):
        assert s.last[k] == pytest.approx(ref0[rk], rel=SUM_TOL, abs=1e-300), k
    N = m["n"] ** m["d"]
    assert s.last["etot_drift"] == 0.0 and s.last["c_rel"] == 0.0
    assert abs(s.last["w"] - w_of(ref0, m["d"])) <= SUM_TOL * check_scale("w", s.last)
    for it in range(1, m["steps"] + 1):
        got = s.step(1, sums=True, local=(it == m["steps"]))
        ref = dict(zip(SCALAR_NAMES, g["scalars"][it]))
        check_sums(got, ref, N, where=(name, it))
        check_line_checks(got, ref, m["d"], ref0["Etot"], where=(name, it))
        assert got["t"] == ref["t"]
    f = s.fields()
    for k in ("phi", "pi", "ekin", "egrad", "epot"):
        assert field_err(f[k], g[k + "_end"]) <= FIELD_TOL, (k, field_err(f[k], g[k + "_end"]))


@pytest.mark.parametrize("name", ["d2_bubbles", "d3_expanding", "d3_thermal"])
def test_dropin_create_from_reference_state(name):
    """cb_create takes the state the reference constructor leaves behind."""
    import coolbubble_b200 as cb
    from oracle.bridge import SCALAR_NAMES
    g = load_golden(name)
    m = g["meta"]
    sc0 = dict(zip(SCALAR_NAMES, g["scalars"][0]))
    state = (g["phi_start"], g["pi_start"], dict(t=0.0, a=sc0["a"], ap=sc0["ap"], H=sc0["H"],
                                                  ekin_half_prev=sc0["EkinHalfPrev"], etot0=sc0["Etot"]))
    s = cb.Bubble(params_from(m), state=state)
    got = s.step(m["steps"], sums=True, local=True)
    ref = dict(zip(SCALAR_NAMES, g["scalars"][-1]))
    check_sums(got, ref, m["n"] ** m["d"], where=name)
    check_line_checks(got, ref, m["d"], sc0["Etot"], where=name)
    f = s.fields()
    for k in ("phi", "pi", "ekin", "egrad", "epot"):
        assert field_err(f[k], g[k + "_end"]) <= FIELD_TOL, k


def test_chunked_steps_equal_single_steps_bitwise():
    import coolbubble_b200 as cb
    g = load_golden("d2_bubbles")
    p = params_from(g["meta"])
    a = cb.Bubble(p, g["phi0"], g["pi0"])
    b = cb.Bubble(p, g["phi0"], g["pi0"])
    sa = a.step(40, sums=True, local=True)
    for _ in range(39):
        b.step(1, sums=False)
    sb = b.step(1, sums=True, local=True)
    assert sa == sb
    fa, fb = a.fields(), b.fields()
    for k in fa:
        np.testing.assert_array_equal(fa[k], fb[k])


def _oracle_run(d, n, L, c, dt, phi0, pi0, steps, every, **kw):
    from oracle import bridge as B
    o = B.Oracle(d, n, L, c, dt, phi0, pi0, **kw)
    out = []
    done = 0
    while done < steps:
        o.step(every)
        done += every
        out.append(o.scalars())
    return o, out


@pytest.mark.parametrize("case", [
    # C1 shape: d = 2, N = 512, L = 32, c = 4, 5 bubbles, static, dt = 0.1 dx
    dict(d=2, n=512, L=32.0, c=4.0, steps=100, every=20, ic="bubbles", nb=5),
    # C2 shape at reduced N: d = 3 expanding, Mpl = 10, 8 bubbles with the 1.3 radius
    dict(d=3, n=64, L=16.0, c=4.0, steps=100, every=20, ic="bubbles", nb=8, expansion=1, mpl=10.0),
    # partial tiles (96 is not a multiple of 32 along the march chunk), static smooth field
    dict(d=3, n=40, L=20.0, c=2.0, steps=60, every=20, ic="noise"),
    # d = 1, long line
    dict(d=1, n=4096, L=64.0, c=4.0, steps=100, every=25, ic="noise"),
    # dx^2 not a power of two: the exact-division path
    dict(d=2, n=96, L=30.0, c=5.0, steps=80, every=20, ic="bubbles", nb=4),
    # conformal time (ALPHAVAL = 1) on the staged d = 3 kernel: gradient energy in every Friedmann update
    dict(d=3, n=64, L=16.0, c=4.0, steps=60, every=20, ic="bubbles", nb=6, expansion=1, mpl=10.0, alpha=1),
])
def test_fp64_matches_oracle(case):
    import coolbubble_b200 as cb
    d, n, L, c = case["d"], case["n"], case["L"], case["c"]
    dt = 0.1 * L / n
    if case["ic"] == "bubbles":
        phi0, pi0 = bubbles(d, n, L, c, case["nb"], seed=7), None
    else:
        phi0 = smooth_noise(d, n, 0.3, seed=3)
        pi0 = smooth_noise(d, n, 0.05, seed=4)
    kw = dict(expansion=case.get("expansion", 0), mpl=case.get("mpl", 200.0), alpha=case.get("alpha", 0))
    o, ref = _oracle_run(d, n, L, c, dt, phi0, pi0, case["steps"], case["every"], **kw)
    s = cb.Bubble(cb.make_params(d, n, L, c, dt, **kw), phi0, pi0)
    for r in ref:
        got = s.step(case["every"], sums=True, local=True)
        check_sums(got, r, n ** d, where=case)
    f, fo = s.fields(), o.fields()
    for k in ("phi", "pi", "ekin", "egrad", "epot"):
        assert field_err(f[k], fo[k]) <= FIELD_TOL, (k, field_err(f[k], fo[k]))


@pytest.mark.parametrize("case", [
    dict(d=3, n=64, L=16.0, c=4.0, steps=100, ic="bubbles", nb=8, expansion=1, mpl=10.0),
    dict(d=3, n=128, L=32.0, c=2.0, steps=100, ic="noise"),
    dict(d=2, n=256, L=32.0, c=4.0, steps=200, ic="bubbles", nb=5),
    dict(d=3, n=64, L=16.0, c=4.0, steps=100, ic="bubbles", nb=8, expansion=1, mpl=10.0, alpha=1),
])
def test_fp32c_energies_within_1e5_of_fp64_oracle(case):
    import coolbubble_b200 as cb
    d, n, L, c = case["d"], case["n"], case["L"], case["c"]
    dt = 0.1 * L / n
    if case["ic"] == "bubbles":
        phi0, pi0 = bubbles(d, n, L, c, case["nb"], seed=11), None
    else:
        phi0, pi0 = smooth_noise(d, n, 0.3, seed=5), smooth_noise(d, n, 0.05, seed=6)
    kw = dict(expansion=case.get("expansion", 0), mpl=case.get("mpl", 200.0), alpha=case.get("alpha", 0))
    o, ref = _oracle_run(d, n, L, c, dt, phi0, pi0, case["steps"], case["steps"], **kw)
    s = cb.Bubble(cb.make_params(d, n, L, c, dt, precision="fp32c", **kw), phi0, pi0)
    got = s.step(case["steps"], sums=True)
    r = ref[-1]
    etot = abs(r["Etot"])
    for k, rk in (("etot", "Etot"), ("egrad", "Egradtot"), ("epot", "Epottot")):
        assert abs(got[k] - r[rk]) <= 1e-5 * abs(r[rk]), (k, got[k], r[rk])
    assert abs(got["ekin"] - r["Ekintot"]) <= 1e-5 * etot
    assert abs(got["a"] - r["a"]) <= 1e-10 * abs(r["a"])


def test_runs_are_deterministic():
    import coolbubble_b200 as cb
    d, n, L, c = 3, 48, 12.0, 4.0
    phi0 = bubbles(d, n, L, c, 6, seed=2)
    p = cb.make_params(d, n, L, c, 0.1 * L / n, expansion=1, mpl=10.0)
    runs = []
    for _ in range(2):
        s = cb.Bubble(p, phi0)
        runs.append((s.step(30, sums=True), s.fields()["phi"]))
    assert runs[0][0] == runs[1][0]
    np.testing.assert_array_equal(runs[0][1], runs[1][1])


def test_f32_download_is_rounded_fp64_state():
    import coolbubble_b200 as cb
    g = load_golden("d3_thermal")
    s = cb.Bubble(params_from(g["meta"]), g["phi0"], g["pi0"])
    s.step(10, sums=True, local=True)
    f64, f32 = s.fields(), s.fields_f32()
    for k in f64:
        np.testing.assert_array_equal(f32[k], f64[k].astype(np.float32))


@pytest.mark.parametrize("case", [
    dict(d=3, n=64, L=16.0, c=4.0, expansion=1, mpl=10.0, prec="fp64"),
    dict(d=3, n=128, L=32.0, c=2.0, expansion=0, mpl=200.0, prec="fp64"),
    dict(d=3, n=96, L=24.0, c=3.0, expansion=0, mpl=200.0, prec="fp64"),
])
def test_tiled_kernel_equals_generic_kernel_fp64(case, monkeypatch):
    """The TMA-tiled d = 3 kernel does the generic kernel's per-site arithmetic op
    for op (bit-identical fields); only the order of the box sums differs."""
    import coolbubble_b200 as cb
    d, n, L, c = case["d"], case["n"], case["L"], case["c"]
    p = cb.make_params(d, n, L, c, 0.1 * L / n, expansion=case["expansion"], mpl=case["mpl"], precision=case["prec"])
    phi0 = bubbles(d, n, L, c, 6, seed=4)
    pi0 = smooth_noise(d, n, 0.02, seed=5)
    tiled = cb.Bubble(p, phi0, pi0)
    monkeypatch.setenv("CB_STEP_PATH", "generic")
    generic = cb.Bubble(p, phi0, pi0)
    monkeypatch.delenv("CB_STEP_PATH")
    a = tiled.step(25, sums=True, local=True)
    b = generic.step(25, sums=True, local=True)
    for key in a:
        # C = H^2 - a^(2 alpha) Etot / (3 Mpl^2) cancels: compared on the H^2 scale;
        # signed sums (<phi>, <phidot>) on the scale of sqrt(N sum x^2), a bound on sum |x|
        scale = abs(b["H"]) ** 2 if key == "C" else abs(b[key])
        if key in ("avphi", "avphip"):
            scale = max(scale, (n ** d * b[key + "_var"]) ** 0.5)
        scale = max(scale, check_scale(key, b))
        assert abs(a[key] - b[key]) <= 1e-14 * scale + 1e-300, key
    fa, fb = tiled.fields(), generic.fields()
    for key in fa:
        np.testing.assert_array_equal(fa[key], fb[key])


@pytest.mark.parametrize("d,n,prec,L", [(2, 1024, "fp64", None), (2, 1028, "fp32c", None), (2, 2048, "fp32c", None),
                                        (2, 1032, "fp64", None), (2, 1026, "fp64", None), (2, 4100, "fp32c", None),
                                        (1, 1 << 20, "fp64", None), (1, (1 << 20) + 4, "fp32c", None),
                                        (1, (1 << 20) + 2, "fp64", None), (2, 1032, "fp64", 100.0),
                                        (1, 1 << 20, "fp64", 100000.0)])
def test_strip_kernel_equals_generic_kernel_2d(d, n, prec, L, monkeypatch):
    """The strip kernel (column strips marched down the rows; d = 2 lattices of
    1024^2 sites and more, d = 1 rows of 2^20 and more) does the generic
    kernel's per-site arithmetic op for op: bit-identical fields and local
    energy arrays over measured and unmeasured steps; the box sums differ only
    in their order. Sizes cover rows ending inside a warp (one vector in the
    last strip) and inside a block, odd vector counts, several strips and
    bands, and (L = 100, 1e5) spacings whose square is not a power of two, where
    FP64 divides as the reference does."""
    import coolbubble_b200 as cb
    L = n / 8.0 if L is None else L
    c = 4.0
    p = cb.make_params(d, n, L, c, 0.1 * L / n, precision=prec)
    phi0 = bubbles(d, n, L, c, 6, seed=7)
    pi0 = smooth_noise(d, n, 0.02, seed=8)
    strip = cb.Bubble(p, phi0, pi0)
    monkeypatch.setenv("CB_STEP_PATH", "generic")
    generic = cb.Bubble(p, phi0, pi0)
    monkeypatch.delenv("CB_STEP_PATH")
    for steps in (1, 7, 40):
        a = strip.step(steps, sums=True, local=True)
        b = generic.step(steps, sums=True, local=True)
        tol = 1e-13 if prec == "fp64" else 1e-5
        for key in a:
            # C = H^2 - Etot / (3 Mpl^2) with H = 0 here: compared on the scale of its terms
            scale = abs(b["H"]) ** 2 + abs(b["etot"]) / (3 * 200.0 ** 2) if key == "C" else abs(b[key])
            if key in ("avphi", "avphip"):
                scale = max(scale, (n ** d * b[key + "_var"]) ** 0.5)
            scale = max(scale, check_scale(key, b))
            assert abs(a[key] - b[key]) <= tol * scale + 1e-300, key
        fa, fb = strip.fields(), generic.fields()
        for key in fa:
            np.testing.assert_array_equal(fa[key], fb[key])


@pytest.mark.parametrize("d,n,prec,expansion", [(2, 512, "fp64", 0), (2, 256, "fp32c", 0), (3, 64, "fp32c", 1),
                                                (3, 64, "fp64", 1), (3, 96, "fp32c", 0), (1, 4096, "fp64", 0)])
def test_step_graphs_equal_plain_launches(d, n, prec, expansion, monkeypatch):
    """Chains of plain steps replayed from a CUDA graph (small lattices) queue
    the same kernels with the same arguments as plain launches: fields, sums,
    time and launch counts identical, across chains that start from either
    buffer state and runs whose length is not a multiple of the chain."""
    import coolbubble_b200 as cb
    L = n / 8.0
    p = cb.make_params(d, n, L, 4.0, 0.1 * L / n, expansion=expansion, mpl=10.0, precision=prec, memorysave=0)
    phi0 = bubbles(d, n, L, 4.0, 4, seed=11) if d > 1 else smooth_noise(d, n, 0.5, seed=11)
    pi0 = smooth_noise(d, n, 0.02, seed=12)
    graphed = cb.Bubble(p, phi0, pi0)
    monkeypatch.setenv("CB_STEP_GRAPHS", "0")
    plain = cb.Bubble(p, phi0, pi0)
    for steps in (40, 17, 33, 1, 64):
        monkeypatch.delenv("CB_STEP_GRAPHS")
        a = graphed.step(steps, sums=True, local=steps == 64)
        monkeypatch.setenv("CB_STEP_GRAPHS", "0")
        b = plain.step(steps, sums=True, local=steps == 64)
        assert a == b
    assert graphed.counters() == plain.counters()
    fa, fb = graphed.fields(), plain.fields()
    for key in fa:
        np.testing.assert_array_equal(fa[key], fb[key])


@pytest.mark.parametrize("n,alpha,prec", [(64, 0, "fp32c"), (128, 0, "fp32c"), (256, 0, "fp32c"), (128, 1, "fp32c"),
                                          (128, 0, "fp64"), (128, 1, "fp64")])
def test_multi_step_launch_equals_single_launches(n, alpha, prec, monkeypatch):
    """Runs of plain expanding steps in one cooperative launch (every
    block forming the Friedmann update itself after a bounded grid barrier)
    give the fields, sums, time and background of one launch per step, bit
    for bit, in fewer launches."""
    import coolbubble_b200 as cb
    L = n / 8.0
    p = cb.make_params(3, n, L, 4.0, 0.1 * L / n, expansion=1, mpl=10.0, alpha=alpha, precision=prec,
                       memorysave=1)
    phi0 = bubbles(3, n, L, 4.0, 4, seed=11)
    pi0 = smooth_noise(3, n, 0.02, seed=12)
    multi = cb.Bubble(p, phi0, pi0)
    monkeypatch.setenv("CB_MULTI_STEP", "0")
    single = cb.Bubble(p, phi0, pi0)
    for steps in (40, 17, 2, 1, 33):
        monkeypatch.delenv("CB_MULTI_STEP")
        a = multi.step(steps, sums=True)
        monkeypatch.setenv("CB_MULTI_STEP", "0")
        b = single.step(steps, sums=True)
        assert a == b, steps
    (lm, nm), (ls_, ns) = multi.counters(), single.counters()
    assert nm == ns == 93 and lm < ls_
    fa, fb = multi.fields(), single.fields()
    for key in fa:
        np.testing.assert_array_equal(fa[key], fb[key])


def test_fp64_tiled_static_matches_oracle():
    import coolbubble_b200 as cb
    from oracle import bridge as B
    d, n, L, c = 3, 128, 32.0, 2.0
    dt = 0.1 * L / n
    phi0, pi0 = smooth_noise(d, n, 0.3, seed=13), smooth_noise(d, n, 0.05, seed=14)
    s = cb.Bubble(cb.make_params(d, n, L, c, dt), phi0, pi0)
    o = B.Oracle(d, n, L, c, dt, phi0, pi0)
    for _ in range(3):
        got = s.step(20, sums=True, local=True)
        o.step(20)
        check_sums(got, o.scalars(), n ** d)
    f, fo = s.fields(), o.fields()
    for k in ("phi", "pi", "ekin", "egrad", "epot"):
        assert field_err(f[k], fo[k]) <= FIELD_TOL, k


def test_fp64_strip_kernel_2d_matches_oracle():
    """The d = 2 column-strip kernel (1024^2 and up) against the oracle in FP64:
    fields and box averages after 3 x 20 steps, local arrays included."""
    import coolbubble_b200 as cb
    from oracle import bridge as B
    d, n, L, c = 2, 1024, 64.0, 4.0
    dt = 0.1 * L / n
    phi0, pi0 = bubbles(d, n, L, c, 5, seed=21), smooth_noise(d, n, 0.05, seed=22)
    s = cb.Bubble(cb.make_params(d, n, L, c, dt), phi0, pi0)
    o = B.Oracle(d, n, L, c, dt, phi0, pi0)
    for _ in range(3):
        got = s.step(20, sums=True, local=True)
        o.step(20)
        check_sums(got, o.scalars(), n ** d)
    f, fo = s.fields(), o.fields()
    for k in ("phi", "pi", "ekin", "egrad", "epot"):
        assert field_err(f[k], fo[k]) <= FIELD_TOL, k


def test_device_error_word_stays_clear():
    """The bounded waits of the tiled kernel never fired during a normal run."""
    import coolbubble_b200 as cb
    d, n, L, c = 3, 256, 32.0, 2.0
    s = cb.Bubble(cb.make_params(d, n, L, c, 0.1 * L / n, precision="fp32c"), smooth_noise(d, n, 0.1, seed=1))
    s.step(50, sums=True)
    assert s.device_error() == 0


@pytest.mark.parametrize("n,L,steps", [(128, 32.0, 41), (256, 32.0, 80), (384, 48.0, 21), (512, 64.0, 9)])
@pytest.mark.parametrize("tl", [2])
def test_temporal_blocking_matches_single_step_passes(n, L, steps, tl, monkeypatch):
    """Static float 3-D runs: two steps per HBM pass give the fields of one
    step per pass bit for bit (same per-site arithmetic) and energies within
    the FP32C bar. Sizes: 32-, 16- and 8-row tiles (128^3, 256^3, 512^3), a
    row of 96 vectors (384^3), odd step counts (a last single step)."""
    import coolbubble_b200 as cb
    from oracle import bridge as B
    d, c = 3, 2.0
    dt = 0.1 * L / n
    if n > 256:                         # white noise: the band-limited field's FFT is slow on the host at this size
        rng = np.random.default_rng(31)
        phi0, pi0 = 0.3 * rng.random(n ** d), 0.05 * rng.standard_normal(n ** d)
    else:
        phi0, pi0 = smooth_noise(d, n, 0.3, seed=31), smooth_noise(d, n, 0.05, seed=32)
    p = cb.make_params(d, n, L, c, dt, precision="fp32c", memorysave=1)
    monkeypatch.setenv("CB_TEMPORAL_BLOCK", str(tl))
    blocked = cb.Bubble(p, phi0, pi0)
    monkeypatch.setenv("CB_TEMPORAL_BLOCK", "1")
    single = cb.Bubble(p, phi0, pi0)
    monkeypatch.delenv("CB_TEMPORAL_BLOCK")
    a = blocked.step(steps, sums=True)
    b = single.step(steps, sums=True)
    launches, nsteps = blocked.counters()
    assert nsteps == steps and launches < steps   # passes of tl steps were used (opt-in path)
    assert single.counters() == (steps, steps)
    fa, fb = blocked.fields(local=False), single.fields(local=False)
    for k in ("phi", "pi"):
        np.testing.assert_array_equal(fa[k], fb[k])
    assert a == b
    if n > 256:
        return                          # the oracle's CPU run is the slow part; 512^3 checks the kernel only
    o = B.Oracle(d, n, L, c, dt, phi0, pi0)
    o.step(steps)
    r = o.scalars()
    for k, rk in (("etot", "Etot"), ("egrad", "Egradtot"), ("epot", "Epottot")):
        assert abs(a[k] - r[rk]) <= 1e-5 * abs(r[rk]), k
    assert a["t"] == b["t"] == r["t"]


@pytest.mark.parametrize("case", [
    dict(d=1, n=256, L=32.0, c=4.0, expansion=0, prec="fp64", start=(5, 0, 0)),
    dict(d=2, n=96, L=24.0, c=3.0, expansion=0, prec="fp64", start=(70, 13, 0)),
    dict(d=3, n=64, L=16.0, c=4.0, expansion=1, prec="fp64", start=(40, 7, 19)),    # a drift pending
    dict(d=3, n=64, L=16.0, c=4.0, expansion=1, prec="fp32c", start=(3, 60, 1)),
])
def test_line_equals_the_field(case):
    """cb_get_line (the wall finder's line) equals the same sites of the full
    field bit for bit, including a run whose last drift is still pending."""
    import coolbubble_b200 as cb
    d, n, L, c = case["d"], case["n"], case["L"], case["c"]
    p = cb.make_params(d, n, L, c, 0.1 * L / n, expansion=case["expansion"], mpl=10.0, precision=case["prec"])
    s = cb.Bubble(p, bubbles(d, n, L, c, 4, seed=9), smooth_noise(d, n, 0.02, seed=2))
    s.step(13, sums=False)
    i0, i1, i2 = case["start"]
    line = s.line(i0, i1, i2)
    phi = s.fields(local=False)["phi"].reshape((n,) * d)
    idx = [(i0 + m) % n for m in range(n)]
    want = phi[idx] if d == 1 else (phi[idx, i1] if d == 2 else phi[idx, i1, i2])
    np.testing.assert_array_equal(line, want)
    np.testing.assert_array_equal(s.line(i0, i1, i2, count=7), want[:7])


def test_temporal_block_autotuner_keeps_the_fields(monkeypatch):
    """With CB_TEMPORAL_BLOCK unset the steps per pass of a static float 3-D
    run are chosen by timing both passes once (on spare buffers: the run's
    state does not change); the fields equal those of one-step passes bit for
    bit whatever the choice."""
    import coolbubble_b200 as cb
    d, n, L, c, steps = 3, 256, 32.0, 2.0, 41
    phi0, pi0 = smooth_noise(d, n, 0.3, seed=41), smooth_noise(d, n, 0.05, seed=42)
    p = cb.make_params(d, n, L, c, 0.1 * L / n, precision="fp32c", memorysave=1)
    monkeypatch.delenv("CB_TEMPORAL_BLOCK", raising=False)
    auto = cb.Bubble(p, phi0, pi0)
    monkeypatch.setenv("CB_TEMPORAL_BLOCK", "1")
    single = cb.Bubble(p, phi0, pi0)
    monkeypatch.delenv("CB_TEMPORAL_BLOCK")
    a, b = auto.step(steps, sums=True), single.step(steps, sums=True)
    launches, nsteps = auto.counters()
    assert nsteps == steps and launches in (steps, steps // 2 + 1)   # one-step or two-step passes
    assert a == b
    fa, fb = auto.fields(local=False), single.fields(local=False)
    for k in ("phi", "pi"):
        np.testing.assert_array_equal(fa[k], fb[k])


def test_temporal_blocking_falls_back_where_it_does_not_apply(monkeypatch):
    """Rows that are not a multiple of 32 vectors (n % 128 != 0) take one-step
    passes even when two-step passes are asked for."""
    import coolbubble_b200 as cb
    d, n, L, c = 3, 96, 24.0, 2.0
    p = cb.make_params(d, n, L, c, 0.1 * L / n, precision="fp32c", memorysave=1)
    monkeypatch.setenv("CB_TEMPORAL_BLOCK", "2")
    s = cb.Bubble(p, smooth_noise(d, n, 0.3, seed=31), smooth_noise(d, n, 0.05, seed=32))
    s.step(10, sums=True)
    assert s.counters() == (10, 10)
