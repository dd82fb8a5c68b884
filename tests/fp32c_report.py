"""Error report of the FP32-compensated path against the FP64 path at the
benchmark configurations' full run lengths (test infrastructure; the FP64
path is itself pinned to the reference by tests/test_parity_configs_gpu.py).

Both precisions start from the same host IC (cb_initial_condition: the
reference's placement and thermal streams) and step side by side; at each of
the 20 snapshot steps of main.cpp's schedule (main.cpp:201-223, evenly spaced)
the report gives, FP32C against FP64:

  field_l2_phi / field_l2_pi  ||x32 - x64||_2 / ||x64||_2 over the lattice
  etot, egrad, epot           relative error; ekin on the Etot scale
  w                           absolute error of (Ekin - (d-2)/d Egrad - Epot) / Etot
  drift                       absolute error of Etot / Etot(0) - 1
  a                           relative error of the scale factor
  spec_1e8 .. spec_1e4        largest relative error of Delta_phi(k) over the
                              shells above 1e-8 .. 1e-4 of the peak
  spec_over_1e4               shells above 1e-8 of the peak whose error exceeds 1e-4

and, for a run with one centred bubble (mode -2, static), the tracked wall:
WallFinder's Rmin / Rmax (bubble.cpp:575-617, lattice radii) in both precisions
and the radius where phi crosses (phiZero + phiMax)/2, interpolated along the
line, at every 50th step while t < L/2.

  python tests/fp32c_report.py [--which NAME ...] [--nt N] > report.json
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

RUNS = {
    # the 256^3 expanding run with 8 bubbles (Mpl = 10), 2000 steps
    "bubbles-d3-n256-expanding": dict(d=3, n=256, L=32.0, c=4.0, mode=1, nb=8, trad=0.2, expansion=1, mpl=10.0,
                                      nt=2000),
    # the 512^3 static run with the thermal start (Trad = 0.05), 4000 steps
    "thermal-d3-n512": dict(d=3, n=512, L=64.0, c=2.0, mode=-3, nb=5, trad=0.05, expansion=0, mpl=200.0, nt=4000),
    # the 512^2 static run with 5 bubbles, 1000 steps
    "bubbles-d2-n512": dict(d=2, n=512, L=32.0, c=4.0, mode=1, nb=5, trad=0.2, expansion=0, mpl=200.0, nt=1000),
}
WALL = dict(d=3, n=256, L=32.0, c=4.0, mode=-2, nb=1, trad=0.2, expansion=0, mpl=200.0, nt=1280)


def snapshot_steps(nt, n=20):
    """main.cpp:201-223 with SnapshotSpacing = 0: steps lround(T k / n / dt), k = 1..n."""
    return sorted({min(nt, max(1, int(round(nt * k / n)))) for k in range(1, n + 1)})


def _pair(cfg):
    import coolbubble_b200 as cb
    from coolbubble_b200.ic import initial_condition
    d, n, L, c = cfg["d"], cfg["n"], cfg["L"], cfg["c"]
    dt = 0.1 * L / n
    kw = dict(expansion=cfg["expansion"], mpl=cfg["mpl"], memorysave=1)
    p64 = cb.make_params(d, n, L, c, dt, precision="fp64", **kw)
    phi0, pi0, _ = initial_condition(p64, mode=cfg["mode"], n_bubbles=cfg["nb"], trad=cfg["trad"])
    s64 = cb.Bubble(p64, phi0, pi0)
    s32 = cb.Bubble(cb.make_params(d, n, L, c, dt, precision="fp32c", **kw), phi0, pi0)
    return s64, s32


def _w(s, d):
    return (s["ekin"] - (d - 2) / d * s["egrad"] - s["epot"]) / s["etot"]


def _l2(a32, a64):
    num = 0.0
    den = 0.0
    step = 1 << 24
    for i in range(0, a64.size, step):
        x = a64[i:i + step]
        dlt = a32[i:i + step].astype(np.float64) - x
        num += float(np.dot(dlt, dlt))
        den += float(np.dot(x, x))
    return math.sqrt(num / den) if den > 0 else 0.0


def _spec_errors(s64, s32):
    pw, ws, _ = s64.spectrum_sums()
    pw32, ws32, _ = s32.spectrum_sums()
    assert np.array_equal(ws, ws32)
    m = ws > 0
    ref, got = pw[m] / ws[m], pw32[m] / ws[m]
    rel = np.abs(got / np.where(ref != 0, ref, 1.0) - 1.0)
    out = {}
    for name, floor in (("spec_1e8", 1e-8), ("spec_1e7", 1e-7), ("spec_1e6", 1e-6), ("spec_1e5", 1e-5),
                        ("spec_1e4", 1e-4)):
        big = ref > floor * ref.max()
        out[name] = float(rel[big].max(initial=0.0))
    big = ref > 1e-8 * ref.max()
    out["spec_over_1e4"] = int((rel[big] > 1e-4).sum())
    out["spec_shells_1e8"] = int(big.sum())
    return out


def run_config(name, nt=None, fields=True, spectra=True):
    """Rows of the report for one configuration (one per snapshot step)."""
    cfg = RUNS[name]
    nt = nt or cfg["nt"]
    d, N = cfg["d"], cfg["n"] ** cfg["d"]
    s64, s32 = _pair(cfg)
    e0_64, e0_32 = s64.last["etot"], s32.last["etot"]
    rows, done = [], 0
    for at in snapshot_steps(nt):
        k = at - done
        # energy lines every 40 steps, as main.cpp; the snapshot step measures too
        while k > 0:
            kk = min(k, 40 - (done % 40))
            a, b = s64.step(kk, sums=True), s32.step(kk, sums=True)
            done += kk
            k -= kk
        r = {"step": done, "t": a["t"]}
        et = abs(a["etot"])
        for key in ("etot", "egrad", "epot"):
            r[key] = abs(b[key] - a[key]) / abs(a[key])
        r["ekin"] = abs(b["ekin"] - a["ekin"]) / et
        r["w"] = abs(_w(b, d) - _w(a, d))
        r["w_device"] = abs(b["w"] - a["w"])
        r["drift"] = abs((b["etot"] / e0_32 - 1.0) - (a["etot"] / e0_64 - 1.0))
        r["drift_fp64"] = a["etot_drift"]
        r["a"] = abs(b["a"] - a["a"]) / a["a"]
        if cfg["expansion"]:
            r["c_rel_fp64"], r["c_rel_fp32c"] = a["c_rel"], b["c_rel"]
        if fields:
            f64, f32 = s64.fields(local=False), s32.fields_f32(local=False)
            r["field_l2_phi"] = _l2(f32["phi"], f64["phi"])
            r["field_l2_pi"] = _l2(f32["pi"], f64["pi"])
            del f64, f32
        if spectra:
            r.update(_spec_errors(s64, s32))
        rows.append(r)
    s64.close()
    s32.close()
    return {"config": name, "nt": nt, "sites": N, **{k: cfg[k] for k in ("d", "n", "L", "c", "mode", "expansion")},
            "rows": rows}


def _wall(line, cfg, dx, state):
    """WallFinder (bubble.cpp:575-617) on one line from the centre, plus the
    interpolated radius where phi crosses the mid value of phiZero and phiMax."""
    c, d, L = cfg["c"], cfg["d"], cfg["L"]
    phi_max = c / (6 + 2 * c)
    phi_zero = (2 + c - math.sqrt(4 + c)) / (3 + c)
    rn = 0.823 * c ** 0.203 * (1.3 if d == 3 else 1.0)
    lw = 0.496 * c ** -0.531
    maximal = L / 2.0

    def radius(i):
        return dx * math.sqrt((i + 0.5) ** 2 + 0.25 * (d - 1))

    istart = max(int((state["rmin"] - lw) / dx), int(rn / (2 * dx)))
    rmin = rmax = 0.0
    i = istart
    while (rmax == 0 or rmin == 0) and radius(i) < maximal:
        v = line[i % line.size]
        if v > phi_zero:
            rmin = radius(i)
        if v <= phi_max and rmax == 0:
            rmax = radius(i)
        i += 1
    state["rmin"], state["rmax"] = rmin, rmax
    mid = 0.5 * (phi_zero + phi_max)
    cross = None
    for j in range(line.size // 2 - 1):
        if line[j] > mid >= line[j + 1]:
            f = (line[j] - mid) / (line[j] - line[j + 1])
            cross = radius(j) + f * (radius(j + 1) - radius(j))
            break
    return rmin, rmax, cross


def run_wall(nt=None):
    cfg = WALL
    nt = nt or cfg["nt"]
    s64, s32 = _pair(cfg)
    n, L = cfg["n"], cfg["L"]
    dx = L / n
    centre = (n // 2, n // 2, n // 2 if cfg["d"] == 3 else 0)
    st64, st32 = {"rmin": 0.0}, {"rmin": 0.0}
    rows, done = [], 0
    while done < nt:
        s64.step(50, sums=False)
        s32.step(50, sums=False)
        done += 50
        t = done * 0.1 * dx
        if t >= L / 2:
            break
        a = _wall(s64.line(*centre), cfg, dx, st64)
        b = _wall(s32.line(*centre), cfg, dx, st32)
        rows.append({"step": done, "t": t, "rmin_fp64": a[0], "rmax_fp64": a[1], "rmin_fp32c": b[0],
                     "rmax_fp32c": b[1], "cross_fp64": a[2], "cross_fp32c": b[2],
                     "cross_err": None if a[2] is None or b[2] is None else abs(a[2] - b[2])})
    s64.close()
    s32.close()
    return {"config": "one centred bubble, d = 3, n = 256, L = 32, c = 4, static (mode -2)", "rows": rows}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--which", nargs="*", default=list(RUNS) + ["wall"])
    ap.add_argument("--nt", type=int, default=0, help="steps per run (default: each configuration's own)")
    args = ap.parse_args()
    out = {}
    for name in args.which:
        out[name] = run_wall(args.nt or None) if name == "wall" else run_config(name, args.nt or None)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
