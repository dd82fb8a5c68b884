"""coolbubble_gpu: the reference program's command line and run folder on the
GPU library. CPU part: option errors and the stability check exit like
main.cpp (exit code 1). GPU part: a whole run compared file by file with the
reference executable's own run folder (tests/golden/run_d2, made by
tests/golden/make_golden.py)."""
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

import h5read

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "coolbubble_b200", "lib", "coolbubble_gpu")
GOLD = os.path.join(ROOT, "tests", "golden", "run_d2")


def run(args, cwd=None):
    return subprocess.run([EXE] + args, capture_output=True, text=True, cwd=cwd, timeout=600)


@pytest.mark.parametrize("args,msg", [
    (["--D", "4"], "--D must be 1, 2 or 3"),
    (["--nGrids", "1"], "must be positive"),
    (["--mode", "3"], "--mode must be between -3 and 1"),
    (["--snapshots", "0"], "--snapshots must be at least 1"),
    (["--bogus", "1"], "unknown option"),
    (["--L", "abc"], "cannot read the value"),
    (["--nt"], "needs a value"),
])
def test_bad_options_exit_1(args, msg):
    r = run(args)
    assert r.returncode == 1
    assert msg in r.stderr


def test_unstable_time_step_exits_1():
    r = run(["--D", "2", "--nGrids", "32", "--L", "16", "--dt", "0.4"])
    assert r.returncode == 1
    assert "is not satisfied" in r.stdout


def _numbers(path, skip_comments=True):
    rows = []
    for line in open(path):
        if skip_comments and line.startswith("#"):
            continue
        rows.append([float(x) for x in line.split()])
    return rows


def _check_snapshot_file(mine, manifest):
    """This build's HDF5 snapshot against the manifest the reference's OutField
    left (datasets with their shapes, attributes with their values), plus the
    storage settings OutField asks for (bubble.cpp:936-943)."""
    f = h5read.File(mine)
    lines = [ln.split() for ln in open(manifest).read().splitlines() if ln.strip()]
    sets = {ln[1]: tuple(int(x) for x in ln[3:]) for ln in lines if ln[0] == "dataset"}
    attrs = {ln[1]: float(ln[2]) for ln in lines if ln[0] == "attr"}
    assert sorted(f.keys()) == sorted(sets)
    for name, shape in sets.items():
        d = f[name]
        assert d.shape == shape and d.dtype == np.float32
        D, m = len(shape), shape[0]
        chunk = {1: (m,), 2: (min(m, max(1, 65536 // m)), m), 3: (1, m, m)}[D]
        assert d.kind == "chunked" and d.chunks == chunk
        assert [(x["name"], x["cd"]) for x in d.filters] == [("shuffle", [4]), ("deflate", [9])]
    assert sorted(f.attrs) == sorted(attrs)
    for k, v in attrs.items():
        assert float(f.attrs[k]) == pytest.approx(v, rel=1e-14, abs=1e-300)


@pytest.mark.gpu
def test_run_folder_matches_reference_executable():
    meta = json.load(open(os.path.join(GOLD, "args.json")))
    with tempfile.TemporaryDirectory() as tmp:
        r = run(meta["args"] + ["--dt", repr(meta["dt"]), "--out", tmp])
        assert r.returncode == 0, r.stderr
        (folder,) = os.listdir(tmp)
        assert folder == open(os.path.join(GOLD, "folder_name.txt")).read().strip()
        mine = os.path.join(tmp, folder)
        names = sorted(os.listdir(GOLD))
        for fn in names:
            if fn in ("args.json", "folder_name.txt"):
                continue
            a, b = os.path.join(mine, fn), os.path.join(GOLD, fn)
            assert fn.endswith(".f32") or os.path.exists(a), fn   # payloads live inside this build's .h5
            if fn == "__xns.dat":
                assert open(a).read() == open(b).read()            # bit-exact placement and images
            elif fn == "parameters.dat":
                la = [x for x in open(a) if not x.startswith("Elapsed time")]
                assert la == open(b).readlines()
            elif fn == "EnergyDensities.dat":
                A, B = _numbers(a), _numbers(b)
                assert len(A) == len(B)
                assert open(a).readlines()[:3] == open(b).readlines()[:3]
                for ra, rb in zip(A, B):
                    np.testing.assert_allclose(ra, rb, rtol=2e-9, atol=1e-14)
            elif fn.startswith("_phi_k_t="):
                A, B = _numbers(a), _numbers(b)
                assert len(A) == len(B)
                for ra, rb in zip(A, B):                            # printed with 6 significant digits
                    np.testing.assert_allclose(ra, rb, rtol=2e-6, atol=1e-300)
            elif fn.endswith(".f32"):
                # the reference's dataset payload (HDF5 stand-in of the oracle build) against
                # the same dataset of this build's HDF5 file
                h5name, ds = fn[:-len(".f32")].rsplit(".", 1)
                A = h5read.File(os.path.join(mine, h5name))[ds][:].ravel()
                B = np.fromfile(b, dtype=np.float32)
                assert A.shape == B.shape
                np.testing.assert_allclose(A, B, rtol=2e-7, atol=1e-12 * max(np.abs(B).max(), 1e-30))
            elif fn.endswith(".h5"):
                _check_snapshot_file(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["run_d1_wall", "run_d2_wall"])
def test_wall_tracking_matches_reference_executable(name):
    """Wall tracking (--wall-tracking 1, the reference's WallTracking = 1):
    gamma.dat, the wall messages on stdout and, in 1-D, FullField.dat against
    the reference executable's own run (tests/golden/<name>)."""
    gold = os.path.join(ROOT, "tests", "golden", name)
    meta = json.load(open(os.path.join(gold, "args.json")))
    with tempfile.TemporaryDirectory() as tmp:
        r = run(meta["args"] + ["--dt", repr(meta["dt"]), "--wall-tracking", "1", "--out", tmp])
        assert r.returncode == 0, r.stderr
        (folder,) = os.listdir(tmp)
        assert folder == open(os.path.join(gold, "folder_name.txt")).read().strip()
        mine = os.path.join(tmp, folder)
        ga, gb = open(os.path.join(mine, "gamma.dat")).read(), open(os.path.join(gold, "gamma.dat")).read()
        assert ga.split("\n")[0] == gb.split("\n")[0]
        A = [[float(x) for x in ln.split()] for ln in ga.split("\n")[1:] if ln.strip()]
        B = [[float(x) for x in ln.split()] for ln in gb.split("\n")[1:] if ln.strip()]
        assert len(A) == len(B) and len(B) >= 2
        np.testing.assert_allclose(A, B, rtol=0, atol=1.5e-3)     # printed with 3-4 decimals
        msgs = [ln for ln in r.stdout.splitlines()
                if ln.startswith(("initial wall width", "WallWidth is", "gamma factor", "bubble has"))]
        ref = open(os.path.join(gold, "stdout_wall.txt")).read().splitlines()
        assert [m.split(":")[0] for m in msgs] == [m.split(":")[0] for m in ref]
        for m, q in zip(msgs, ref):
            if ":" in m:
                assert float(m.split(":")[1]) == pytest.approx(float(q.split(":")[1]), rel=1e-5, abs=1e-5)
        if os.path.exists(os.path.join(gold, "FullField.dat")):
            A, B = _numbers(os.path.join(mine, "FullField.dat")), _numbers(os.path.join(gold, "FullField.dat"))
            assert len(A) == len(B)
            np.testing.assert_allclose(np.array(A), np.array(B), rtol=0, atol=1.5e-5)

