"""The FP32-compensated path over long runs, against the FP64 path on the
same start (the FP64 path is pinned to the reference at these sizes by
test_parity_configs_gpu.py): energies within 1e-5 relative (the kinetic
energy on the Etot scale) at every one of the 20 snapshot lines, at the
benchmark configurations' sizes and for at least 1000 steps:

  256^3 expanding, 8 bubbles, Mpl = 10: all 2000 steps of the run; the scale
      factor within 1e-7 relative (the Friedmann update is double, its
      energies are the float path's: measured 2.2e-8 at the end)
  512^3 static thermal start: the first 1000 of its 4000 steps
  512^2 static, 5 bubbles: all 1000 steps

w (absolute) and the energy drift Etot/Etot0 - 1 (absolute) within 1e-5.
The report with fields and spectra at full length is tests/fp32c_report.py.
"""
import pytest

from fp32c_report import run_config

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,nt", [("bubbles-d3-n256-expanding", 2000), ("thermal-d3-n512", 1000),
                                     ("bubbles-d2-n512", 1000)])
def test_fp32c_energies_stay_within_1e5_over_long_runs(name, nt):
    rep = run_config(name, nt=nt, fields=False, spectra=False)
    assert len(rep["rows"]) == 20 and rep["rows"][-1]["step"] == nt
    for r in rep["rows"]:
        for key in ("etot", "ekin", "egrad", "epot", "w", "drift"):
            assert r[key] <= 1e-5, (name, r["step"], key, r[key])
        assert r["a"] <= 1e-7, (name, r["step"], r["a"])
