"""Host-side mirror of the reference's Bubble interface (src/bubble.hpp:34-135)
over the CUDA library. The field arrays, scalars and method names follow the
reference so that code and tests written against it read the same:

    s = Bubble(params, phi0, pi0)        # constructor set-up (bubble.cpp:236-291) on the device
    s.oneStep()                          # bubble.cpp:849-876
    s.Etot, s.Ekintot, s.a, s.H, s.C     # box averages of the last measured step
    s.phi, s.pi                          # downloaded on access
    rows = s.ComputePowerSpectrum()      # (kMean, kMean/a, Delta) per shell (bubble.cpp:668-709)

Everything site-level runs on the GPU; this class only moves arguments.
"""
from __future__ import annotations

import os

import numpy as np

from . import _lib as L
from ._lib import check


def make_params(d, n_grids, L_box, c, dt, alpha=0, expansion=0, mpl=200.0, delta_v=1.0, precision="fp64",
                memorysave=0):
    prec = {"fp64": L.CB_FP64, "fp32c": L.CB_FP32C}[precision] if isinstance(precision, str) else int(precision)
    return L.cb_params(int(d), int(n_grids), float(L_box), float(c), float(dt), int(alpha), int(expansion),
                       float(mpl), float(delta_v), prec, int(memorysave))


class Bubble:
    """One lattice run resident on the GPU."""

    def __init__(self, params, phi0=None, pi0=None, *, state=None):
        self.params = params
        self.d, self.n = params.d, params.n_grids
        self.N = self.n ** self.d
        h = L.C.c_void_p()
        if state is None:
            phi0 = np.ascontiguousarray(phi0, dtype=np.float64).reshape(-1)
            if phi0.size != self.N:
                raise ValueError("phi0 has the wrong size")
            if pi0 is not None:
                pi0 = np.ascontiguousarray(pi0, dtype=np.float64).reshape(-1)
                if pi0.size != self.N:
                    raise ValueError("pi0 has the wrong size")
            s = L.cb_sums()
            check(L.lib.cb_create_from_ic(L.C.byref(params), L.dptr(phi0), L.dptr(pi0), L.C.byref(s), L.C.byref(h)))
        else:
            phi, pi, sc = state
            phi = np.ascontiguousarray(phi, dtype=np.float64).reshape(-1)
            pi = np.ascontiguousarray(pi, dtype=np.float64).reshape(-1)
            s0 = L.cb_scalars(sc["t"], sc["a"], sc["ap"], sc["H"], sc["ekin_half_prev"], sc.get("etot0", 0.0))
            check(L.lib.cb_create(L.C.byref(params), L.dptr(phi), L.dptr(pi), L.C.byref(s0), L.C.byref(h)))
            s = L.cb_sums()
            s.t, s.a, s.ap, s.H, s.ekin_half_prev = sc["t"], sc["a"], sc["ap"], sc["H"], sc["ekin_half_prev"]
        self._h = h
        self._set(s.asdict())

    def __del__(self):
        self.close()

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            L.lib.cb_destroy(h)
        self._h = None

    # ---- scalars named as in bubble.hpp:75-84 ----------------------------
    def _set(self, s):
        self.last = s
        self.t, self.a, self.ap, self.H, self.C = s["t"], s["a"], s["ap"], s["H"], s["C"]
        self.Etot, self.Ekintot, self.Egradtot, self.Epottot = s["etot"], s["ekin"], s["egrad"], s["epot"]
        self.avphi, self.avphiP, self.EkinHalfPrev = s["avphi"], s["avphip"], s["ekin_half_prev"]
        self.EtotVar, self.EkintotVar, self.EgradtotVar = s["etot_var"], s["ekin_var"], s["egrad_var"]
        self.EpottotVar, self.avphiVar, self.avphiPVar = s["epot_var"], s["avphi_var"], s["avphip_var"]

    # ---- evolution --------------------------------------------------------
    def step(self, nsteps=1, sums=True, local=False):
        flags = (L.CB_STEP_SUMS if sums else 0) | (L.CB_STEP_LOCAL if local else 0)
        s = L.cb_sums()
        check(L.lib.cb_step(self._h, int(nsteps), flags, L.C.byref(s) if (sums or local) else None), self._h)
        if sums or local:
            self._set(s.asdict())
        return self.last

    def oneStep(self):
        return self.step(1, sums=True, local=self.params.memorysave == 0)

    def step_timed(self, nsteps):
        ms = L.C.c_double()
        check(L.lib.cb_step_timed(self._h, int(nsteps), 0, L.C.byref(ms)), self._h)
        return ms.value

    def sync(self):
        check(L.lib.cb_sync(self._h), self._h)

    def counters(self):
        """(kernel launches, leapfrog steps) queued by this run so far."""
        a, b = L.C.c_int64(), L.C.c_int64()
        check(L.lib.cb_get_counters(self._h, L.C.byref(a), L.C.byref(b)), self._h)
        return a.value, b.value

    def device_error(self):
        code = L.C.c_int()
        check(L.lib.cb_device_error(self._h, L.C.byref(code)), self._h)
        return code.value

    def sums(self):
        s = L.cb_sums()
        check(L.lib.cb_get_sums(self._h, L.C.byref(s)), self._h)
        return s.asdict()

    # ---- fields -----------------------------------------------------------
    def fields(self, local=True):
        out = [np.empty(self.N) for _ in range(5)]
        if not local or self.params.memorysave:
            out[2] = out[3] = out[4] = None
        check(L.lib.cb_get_fields(self._h, *[L.dptr(x) for x in out]), self._h)
        return dict(zip(("phi", "pi", "ekin", "egrad", "epot"), out))

    def fields_f32(self, local=True):
        out = [np.empty(self.N, dtype=np.float32) for _ in range(5)]
        if not local or self.params.memorysave:
            out[2] = out[3] = out[4] = None
        check(L.lib.cb_get_fields_f32(self._h, *[L.fptr(x) for x in out]), self._h)
        return dict(zip(("phi", "pi", "ekin", "egrad", "epot"), out))

    def line(self, i0, i1=0, i2=0, count=None):
        """phi[(i0 + m) mod n, i1, i2] for m < count (default n): one line along
        axis 0, as the wall finder reads it (bubble.cpp:588-592)."""
        count = self.n if count is None else int(count)
        out = np.empty(count)
        check(L.lib.cb_get_line(self._h, int(i0), int(i1), int(i2), count, L.dptr(out)), self._h)
        return out

    def OutField(self, path, threads=0, background=False):
        """Write the snapshot file <path> as Bubble::OutField does (bubble.cpp:887-953):
        an HDF5 file with phi, pi (and Ekin, gradphi, potEnergy when memorysave == 0),
        written by the library without libhdf5 (cb_out_field). With background=True
        the call returns once the fields are on the host and the file is written on a
        library thread; OutFieldWait() collects it."""
        fn = L.lib.cb_out_field_async if background else L.lib.cb_out_field
        check(fn(self._h, os.fsencode(path), int(threads)), self._h)

    def OutFieldWait(self):
        """Wait for a background OutField; raises CBError if its file could not be written."""
        check(L.lib.cb_out_field_wait(self._h), self._h)

    @property
    def phi(self):
        return self.fields(local=False)["phi"]

    @property
    def pi(self):
        return self.fields(local=False)["pi"]

    # ---- power spectrum ---------------------------------------------------
    def spectrum_sums(self):
        nb = L.lib.cb_nbins(self.d, self.n)
        pw, ws, ks = np.zeros(nb), np.zeros(nb), np.zeros(nb)
        check(L.lib.cb_power_spectrum(self._h, L.dptr(pw), L.dptr(ws), L.dptr(ks), nb), self._h)
        return pw, ws, ks

    def ComputePowerSpectrum(self):
        """Rows (kMean, kMean/a, power/weight) of the shells with weight > 0 (bubble.cpp:703-708)."""
        pw, ws, ks = self.spectrum_sums()
        m = ws > 0
        kmean = ks[m] / ws[m]
        return np.stack([kmean, kmean / self.a, pw[m] / ws[m]], axis=1)
