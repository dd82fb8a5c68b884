"""Seeded synthetic initial conditions for tests (numpy; test infrastructure).

Bubble profiles follow the reference's fits (bubble.cpp:81-108); positions
come from numpy's generator rather than glibc rand(), so these are NOT the
reference's placements -- tests of bit-exact placement use the product's
host IC generator and the golden fixtures instead.
"""
import numpy as np


def fits(c, d):
    phic = 0.997 * (1 - np.exp(-c * 0.688))
    rn = 0.823 * c ** 0.203 * (1.3 if d == 3 else 1.0)
    lw = 0.496 * c ** -0.531
    return phic, rn, lw


def bubbles(d, n, L, c, nb, seed):
    rng = np.random.default_rng(seed)
    phic, rn, lw = fits(c, d)
    x = (np.arange(n) + 0.5) * L / n
    grids = np.meshgrid(*([x] * d), indexing="ij")
    phi = np.zeros((n,) * d)
    for _ in range(nb):
        c0 = rng.uniform(0, L, d)
        r2 = 0.0
        for g, cc in zip(grids, c0):
            dd = np.abs(g - cc)
            dd = np.minimum(dd, L - dd)
            r2 = r2 + dd * dd
        phi = np.minimum(phi + phic / 2 * (np.tanh((rn - np.sqrt(r2)) / lw) + 1), phic)
    return phi.reshape(-1)


def smooth_noise(d, n, amp, seed, kmax=6):
    """Band-limited random field (a few Fourier modes), amplitude ~amp."""
    rng = np.random.default_rng(seed)
    shape = (n,) * d
    spec = np.zeros(shape, dtype=complex)
    idx = tuple(slice(0, kmax) for _ in range(d))
    spec[idx] = rng.standard_normal(spec[idx].shape) + 1j * rng.standard_normal(spec[idx].shape)
    f = np.fft.ifftn(spec).real
    return (amp * f / np.abs(f).max()).reshape(-1)
