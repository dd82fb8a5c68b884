"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's own src/bubble.cpp and src/main.cpp, compiled in place by
``make -C oracle ref`` (see oracle/Makefile), and stores small cases:

* ``<case>.npz`` -- initial condition (raw phi_0, pi_0 from a dt = 0 instance,
  so the set-up back-kick leaves pi unchanged), the state handed to the time
  loop, the 18 scalars after set-up and after every step, the fields after
  the last step, and the spectrum lines (ComputePowerSpectrum at 17 digits)
  at step 0 and at the end.
* ``<case>.xns.txt`` -- the __xns.dat text of bubble modes (bit-exact item).
* ``run_d2/`` -- the output files of one run of the reference executable
  (EnergyDensities.dat, parameters.dat without its timing line, __xns.dat,
  spectra, snapshot manifests and float32 payloads).

Each case runs in a fresh process: the reference keeps its spread sums in
file-static variables (bubble.cpp:44) that would leak between instances.

Usage: python tests/golden/make_golden.py            (all cases)
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

# name: (d, n, L, c, mode, steps, extra)
CASES = {
    "d1_static": dict(d=1, n=128, L=32.0, c=4.0, mode=1, steps=100),
    "d2_bubbles": dict(d=2, n=48, L=24.0, c=4.0, mode=1, steps=100),
    "d2_thermal": dict(d=2, n=32, L=32.0, c=2.0, mode=-3, steps=100, trad=0.05),
    "d2_diagonal": dict(d=2, n=32, L=16.0, c=4.0, mode=-1, steps=40),
    "d2_centre": dict(d=2, n=30, L=16.0, c=6.0, mode=-2, steps=40),
    "d2_wave": dict(d=2, n=32, L=16.0, c=4.0, mode=1, steps=40, test=1),
    "d2_given": dict(d=2, n=32, L=16.0, c=3.0, mode=0, steps=40,
                     xns="4.0 5.5 0.0\n12.25 9.0 0.0\n15.9 0.3 0.0\n"),
    "d3_expanding": dict(d=3, n=16, L=16.0, c=4.0, mode=1, steps=100, expansion=1, mpl=10.0, nbubbles=8),
    "d3_thermal": dict(d=3, n=16, L=32.0, c=2.0, mode=-3, steps=100, trad=0.05),
    "d3_odd_dx": dict(d=3, n=12, L=16.0, c=4.0, mode=1, steps=100, expansion=1, mpl=10.0, nbubbles=3),
    "d3_thermal_expanding": dict(d=3, n=12, L=24.0, c=3.0, mode=-3, steps=60, trad=0.1, expansion=1, mpl=10.0),
    # conformal time (ALPHAVAL = 1): the gradient energy enters the Friedmann update
    "d3_conformal": dict(d=3, n=16, L=16.0, c=4.0, mode=1, steps=100, expansion=1, mpl=10.0, nbubbles=4, alpha=1),
}


def _ref(cfg, dt, folder):
    from oracle import bridge as B
    return B.Reference(cfg["d"], cfg["n"], cfg["L"], cfg["c"], cfg["mode"], dt,
                       nbubbles=cfg.get("nbubbles", 5), trad=cfg.get("trad", 0.2), test=cfg.get("test", 0),
                       expansion=cfg.get("expansion", 0), alpha=cfg.get("alpha", 0), mpl=cfg.get("mpl", 200.0),
                       memorysave=0, folder=folder)


def one_case(name):
    cfg = CASES[name]
    dt = 0.1 * cfg["L"] / cfg["n"]
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        f0 = os.path.join(tmp, "ic")
        os.makedirs(f0)
        if "xns" in cfg:
            with open(os.path.join(f0, "__xns.dat"), "w") as f:
                f.write(cfg["xns"])
        r0 = _ref(cfg, 0.0, f0)
        fl = r0.fields()
        out["phi0"], out["pi0"] = fl["phi"], fl["pi"]
        xns = r0.xns_text() if cfg["mode"] in (0, 1) and cfg["d"] > 1 and not cfg.get("test") else None
        del r0
        f1 = os.path.join(tmp, "run")
        os.makedirs(f1)
        if "xns" in cfg:
            with open(os.path.join(f1, "__xns.dat"), "w") as f:
                f.write(cfg["xns"])
        r = _ref(cfg, dt, f1)
        fl = r.fields()
        out["phi_start"], out["pi_start"] = fl["phi"], fl["pi"]
        out["ekin_start"], out["egrad_start"], out["epot_start"] = fl["ekin"], fl["egrad"], fl["epot"]
        sc = [list(r.scalars().values())]
        out["spec_start"] = r.spectrum_lines()
        for _ in range(cfg["steps"]):
            r.step(1)
            sc.append(list(r.scalars().values()))
        fl = r.fields()
        for k in ("phi", "pi", "ekin", "egrad", "epot"):
            out[k + "_end"] = fl[k]
        out["scalars"] = np.array(sc)
        out["spec_end"] = r.spectrum_lines()
        del r
    meta = dict(cfg, dt=dt)
    meta.pop("xns", None)
    out["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    if xns is not None:
        with open(os.path.join(HERE, name + ".xns.txt"), "w") as f:
            f.write(xns)


def run_dir():
    """The reference executable's own output files for one small 2-D run."""
    from oracle import bridge as B
    B.build_reference()
    dst = os.path.join(HERE, "run_d2")
    shutil.rmtree(dst, ignore_errors=True)
    os.makedirs(dst)
    with tempfile.TemporaryDirectory() as tmp:
        env = dict(os.environ, CBREF_DT=repr(0.1 * 16.0 / 32), OMP_NUM_THREADS="2")
        args = [B.REF_EXE, "--D", "2", "--nGrids", "32", "--L", "16", "--nt", "120", "--c", "4",
                "--mode", "1", "--snapshots", "3", "--no-plots", "--out", tmp]
        subprocess.run(args, check=True, env=env, stdout=subprocess.DEVNULL)
        (folder,) = os.listdir(tmp)
        src = os.path.join(tmp, folder)
        with open(os.path.join(dst, "folder_name.txt"), "w") as f:
            f.write(folder + "\n")
        with open(os.path.join(dst, "args.json"), "w") as f:
            json.dump(dict(args=args[1:-2], dt=0.1 * 16.0 / 32), f)
        for fn in sorted(os.listdir(src)):
            p = os.path.join(src, fn)
            if fn == "parameters.dat":
                lines = [ln for ln in open(p) if not ln.startswith("Elapsed time")]
                open(os.path.join(dst, fn), "w").writelines(lines)
            else:
                shutil.copy(p, os.path.join(dst, fn))


WALL_RUNS = {
    # 1-D: the bubble at the box edge, wall tracked from step 112, FullField.dat every 100 steps
    "run_d1_wall": dict(args=["--D", "1", "--nGrids", "512", "--L", "32", "--nt", "1300", "--c", "4",
                              "--mode", "1", "--snapshots", "2"], dt=0.1 * 32.0 / 512),
    # 2-D: one bubble in the centre (mode -2)
    "run_d2_wall": dict(args=["--D", "2", "--nGrids", "128", "--L", "32", "--nt", "700", "--c", "4",
                              "--mode", "-2", "--snapshots", "2"], dt=0.1 * 32.0 / 128),
}


def run_wall_dirs():
    """Runs of the reference executable with wall tracking on (WallTracking = 1):
    only the files that tracking and the 1-D line writer produce are kept."""
    from oracle import bridge as B
    B.build_reference()
    for name, cfg in WALL_RUNS.items():
        dst = os.path.join(HERE, name)
        shutil.rmtree(dst, ignore_errors=True)
        os.makedirs(dst)
        with tempfile.TemporaryDirectory() as tmp:
            env = dict(os.environ, CBREF_DT=repr(cfg["dt"]), CBREF_WALLTRACKING="1", OMP_NUM_THREADS="2")
            args = [B.REF_EXE] + cfg["args"] + ["--no-plots", "--out", tmp]
            out = subprocess.run(args, check=True, env=env, capture_output=True, text=True).stdout
            (folder,) = os.listdir(tmp)
            src = os.path.join(tmp, folder)
            with open(os.path.join(dst, "folder_name.txt"), "w") as f:
                f.write(folder + "\n")
            with open(os.path.join(dst, "args.json"), "w") as f:
                json.dump(dict(args=cfg["args"] + ["--no-plots"], dt=cfg["dt"]), f)
            with open(os.path.join(dst, "stdout_wall.txt"), "w") as f:
                f.writelines(ln + "\n" for ln in out.splitlines()
                             if ln.startswith(("initial wall width", "WallWidth is", "gamma factor", "bubble has")))
            for fn in ("gamma.dat", "FullField.dat"):
                if os.path.exists(os.path.join(src, fn)):
                    shutil.copy(os.path.join(src, fn), os.path.join(dst, fn))


def main():
    from oracle import bridge as B
    B.build_reference()
    if len(sys.argv) > 2 and sys.argv[1] == "--case":
        one_case(sys.argv[2])
        return
    if len(sys.argv) > 1 and sys.argv[1] == "--wall":
        run_wall_dirs()
        print("wrote", ", ".join(WALL_RUNS))
        return
    for name in CASES:
        subprocess.run([sys.executable, __file__, "--case", name], check=True,
                       env=dict(os.environ, OMP_NUM_THREADS="2"), stdout=subprocess.DEVNULL)
        print("wrote", name)
    run_dir()
    print("wrote run_d2/")
    run_wall_dirs()
    print("wrote", ", ".join(WALL_RUNS))


if __name__ == "__main__":
    main()
