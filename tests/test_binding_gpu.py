"""The reference's own main.cpp with its time loop on the GPU
(coolbubble_b200/binding/cb_main_loop.hpp, built by `make -C oracle ref-gpu`
into oracle/_ref/coolbubble_ref_gpu) against the unmodified reference
executable (oracle/_ref/coolbubble_ref), run with the same arguments; the run
folders are compared file by file:

  folder name, __xns.dat and parameters.dat (but its "Elapsed time" line):
      byte for byte
  EnergyDensities.dat (bubble.cpp:981 formats): the same lines and t; a and
      the energies (11-13 digits) within 1e-10 relative; H and C (9 digits)
      within 2e-8 (C also 1e-9 of H^2); <phi>, <phi'> and the spreads
      (7 digits) within 2e-6 relative
  _phi_k_t=NNNN.dat (printed with 6 digits): the same lines; t, a, <k> and
      Delta(k) within 2e-5 relative, Delta for shells above 1e-8 of the peak
  snapshot payloads (float32 of FP64 fields): within 1e-6 relative of the
      field's largest value; attributes equal
  gamma.dat (wall tracking, 3-4 decimals) and FullField.dat (1-D, 5 decimals):
      within one unit of the last printed digit
"""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_EXE = os.path.join(ROOT, "oracle", "_ref", "coolbubble_ref")
GPU_EXE = os.path.join(ROOT, "oracle", "_ref", "coolbubble_ref_gpu")

CASES = {
    # 2-D, 5 random bubbles (srand(42)), static
    "d2_bubbles": (["--D", "2", "--nGrids", "128", "--L", "16", "--nt", "400", "--mode", "1", "--snapshots", "4"],
                   dict(CBREF_DT="0.0125")),
    # 3-D expanding, 8 bubbles, Mpl = 10, snapshots with the local energy arrays
    "d3_expanding": (["--D", "3", "--nGrids", "64", "--L", "16", "--nt", "200", "--mode", "1", "--snapshots", "4"],
                     dict(CBREF_DT="0.025", CBREF_EXPANSION="1", CBREF_MPL="10", CBREF_NBUBBLES="8")),
    # 3-D thermal start, static, memorysave = 1
    "d3_thermal": (["--D", "3", "--nGrids", "48", "--L", "12", "--nt", "120", "--mode", "-3", "--snapshots", "3",
                    "--c", "2"], dict(CBREF_DT="0.025", CBREF_TRAD="0.05", CBREF_MEMORYSAVE="1")),
    # 2-D one centred bubble with wall tracking (gamma.dat)
    "d2_wall": (["--D", "2", "--nGrids", "256", "--L", "32", "--nt", "1000", "--mode", "-2", "--snapshots", "5"],
                dict(CBREF_DT="0.0125", CBREF_WALLTRACKING="1")),
    # 1-D collision with wall tracking and FullField.dat
    "d1_wall": (["--D", "1", "--nGrids", "2048", "--L", "64", "--nt", "1200", "--snapshots", "4"],
                dict(CBREF_DT="0.003125", CBREF_WALLTRACKING="1")),
}


def _run(exe, args, env, out):
    e = dict(os.environ, **env)
    r = subprocess.run([exe] + args + ["--no-plots", "--out", out], capture_output=True, text=True, env=e,
                       timeout=900)
    assert r.returncode == 0, (exe, r.stdout[-2000:], r.stderr[-2000:])
    (folder,) = os.listdir(out)
    return folder, os.path.join(out, folder)


def _rows(path):
    return [[float(x) for x in ln.split()] for ln in open(path) if ln.strip() and not ln.startswith("#")]


def _close(a, b, rel, what):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    assert a.shape == b.shape, what
    assert np.all(np.abs(a - b) <= rel * np.abs(b) + 1e-300), (what, a, b)


def _energy_lines(mine, ref):
    la, lb = open(mine).readlines(), open(ref).readlines()
    assert len(la) == len(lb)
    assert [x for x in la if x.startswith("#")] == [x for x in lb if x.startswith("#")]
    A, B = np.array(_rows(mine)), np.array(_rows(ref))
    assert (A[:, 0] == B[:, 0]).all()                        # t
    for col in (1, 2, 3, 4, 5):                              # a, Etot, Ekin, Egrad, Epot
        _close(A[:, col], B[:, col], 1e-10, "column %d" % (col + 1))
    for col in (6, 7, 8, 9, 11, 13):                         # spreads
        _close(A[:, col], B[:, col], 2e-6, "spread %d" % (col + 1))
    for col in (10, 12):                                     # <phi>, <phi'>: signed sums, on their spread's scale too
        assert np.all(np.abs(A[:, col] - B[:, col]) <= 2e-6 * np.abs(B[:, col]) + 1e-12 * B[:, col + 1] + 1e-300)
    _close(A[:, 14], B[:, 14], 2e-8, "H")
    # C = H^2 - rho/(3 Mpl^2) cancels: its print precision, or 1e-9 of H^2
    assert np.all(np.abs(A[:, 15] - B[:, 15]) <= 2e-8 * np.abs(B[:, 15]) + 1e-9 * B[:, 14] ** 2 + 1e-300)


def _spectrum(mine, ref):
    la, lb = open(mine).readlines(), open(ref).readlines()
    assert len(la) == len(lb) and la[0] == lb[0]
    _close([float(x) for x in la[1].split()], [float(x) for x in lb[1].split()], 2e-5, "t a")
    A, B = np.array(_rows(mine)[1:]), np.array(_rows(ref)[1:])
    _close(A[:, 0], B[:, 0], 2e-5, "k")
    _close(A[:, 1], B[:, 1], 2e-5, "k/a")
    big = B[:, 2] > 1e-8 * B[:, 2].max()
    _close(A[big, 2], B[big, 2], 2e-5, "Delta")


def _snapshot(mine, ref):
    ma, mb = open(mine).read().split("\n"), open(ref).read().split("\n")
    sets_a = [ln for ln in ma if ln.startswith("dataset")]
    assert sets_a == [ln for ln in mb if ln.startswith("dataset")]
    attrs_a = {ln.split()[1]: float(ln.split()[2]) for ln in ma if ln.startswith("attr")}
    attrs_b = {ln.split()[1]: float(ln.split()[2]) for ln in mb if ln.startswith("attr")}
    assert sorted(attrs_a) == sorted(attrs_b)
    for k in attrs_a:
        assert abs(attrs_a[k] - attrs_b[k]) <= 1e-12 * abs(attrs_b[k]) + 1e-300, k
    for ln in sets_a:
        name = ln.split()[1]
        x = np.fromfile(mine + "." + name + ".f32", dtype=np.float32)
        y = np.fromfile(ref + "." + name + ".f32", dtype=np.float32)
        assert x.shape == y.shape
        assert np.abs(x.astype(float) - y).max() <= 1e-6 * max(np.abs(y).max(), 1e-30), name


def _fixed(mine, ref, unit):
    A, B = _rows(mine), _rows(ref)
    assert len(A) == len(B)
    for ra, rb in zip(A, B):
        assert len(ra) == len(rb)
        assert np.all(np.abs(np.array(ra) - np.array(rb)) <= unit * 1.01), (ra, rb)


@pytest.mark.parametrize("name", list(CASES))
def test_bound_main_matches_reference_run(name, tmp_path):
    if not (os.path.exists(REF_EXE) and os.path.exists(GPU_EXE)):
        pytest.skip("the reference build (oracle/_ref) is not present")
    args, env = CASES[name]
    fa, a = _run(GPU_EXE, args, env, str(tmp_path / "gpu"))
    fb, b = _run(REF_EXE, args, env, str(tmp_path / "ref"))
    assert fa == fb
    names = sorted(os.listdir(b))
    assert sorted(os.listdir(a)) == names
    for fn in names:
        pa, pb = os.path.join(a, fn), os.path.join(b, fn)
        if fn == "__xns.dat":
            assert open(pa).read() == open(pb).read()
        elif fn == "parameters.dat":
            assert [x for x in open(pa) if not x.startswith("Elapsed time")] == \
                   [x for x in open(pb) if not x.startswith("Elapsed time")]
        elif fn == "EnergyDensities.dat":
            _energy_lines(pa, pb)
        elif fn.startswith("_phi_k_t="):
            _spectrum(pa, pb)
        elif fn.endswith(".h5"):
            _snapshot(pa, pb)
        elif fn == "gamma.dat":
            assert open(pa).readline() == open(pb).readline()
            _fixed(pa, pb, 1e-3)
        elif fn == "FullField.dat":
            _fixed(pa, pb, 1e-5)
    if "CBREF_WALLTRACKING" in env:
        assert os.path.exists(os.path.join(a, "gamma.dat"))
