"""Lattices of more than 2^32 sites.

The reference addresses sites with `int` (gridfuncs.cpp:25-51), which
overflows above about 1290^3 sites; this library uses 64-bit offsets in every
kernel (32-bit neighbour arithmetic only below 2^32 sites). Checked here at
1640^3 = 4.41e9 sites (FP32C, 71 GB on the device) through a size-independent
property: the reference's TEST = 1 start (bubble.cpp:337-352, 40 sine
wavelengths per box along each axis) is periodic with period n / 40 = 41
sites on every axis, and so is its evolution. The big lattice must therefore
evolve as the 41^3 lattice with the same spacing started from its first
41^3 block: lines through the whole address range (the last planes lie
beyond 2^32 floats) equal the small run's lines repeated, and the box
averages agree. The big lattice runs once on the staged d = 3 kernel and once
on the generic tile kernel (CB_STEP_PATH=generic); the 41^3 cell always runs
on the generic one. The kernels do the same per-site arithmetic up to
contraction, and the start is periodic only up to the rounding of sin:
tolerance 8 float ulps of 1.
"""
import numpy as np
import pytest

import coolbubble_b200 as cb
from coolbubble_b200.serving import create_from_seed, ic_params

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("path", ["staged", "generic"])
def test_periodic_wave_above_2_to_32_sites(path, monkeypatch):
    n, per, dx, steps = 1640, 41, 0.125, 5
    assert n ** 3 > 2 ** 32 and n == 40 * per
    p = cb.make_params(3, n, n * dx, 4.0, 0.1 * dx, precision="fp32c", memorysave=1)
    if path == "generic":
        monkeypatch.setenv("CB_STEP_PATH", "generic")
    big = create_from_seed(p, ic_params(mode=1, test=1))
    monkeypatch.delenv("CB_STEP_PATH", raising=False)
    try:
        block = np.empty((per, per, per))
        for i1 in range(per):
            for i2 in range(per):
                block[:, i1, i2] = big.line(0, i1, i2, per)
        ps = cb.make_params(3, per, per * dx, 4.0, 0.1 * dx, precision="fp32c", memorysave=1)
        small = cb.Bubble(ps, block.ravel(), np.zeros(per ** 3))
        try:
            s0b, s0s = big.sums(), small.sums()
            big.step(steps, sums=True)
            small.step(steps, sums=True)
            sb, ss = big.sums(), small.sums()
            for (i1, i2) in [(0, 0), (n - 1, n - 1), (n // 2, 7), (1000, n - 1), (n - 1, 3), (123, 1599)]:
                got = big.line(0, i1, i2)
                want = np.tile(small.line(0, i1 % per, i2 % per, per), n // per)
                assert np.abs(got - want).max() <= 8 * 2.0 ** -23, (i1, i2)
        finally:
            small.close()
    finally:
        big.close()
    for a, b in ((s0b, s0s), (sb, ss)):
        assert a["t"] == b["t"] and a["a"] == b["a"]
        assert a["avphi"] == pytest.approx(b["avphi"], rel=1e-6)
        for key in ("etot", "ekin", "egrad", "epot"):
            assert a[key] == pytest.approx(b[key], rel=1e-4, abs=1e-12), key
