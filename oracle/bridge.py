"""oracle/bridge.py -- TEST INFRASTRUCTURE ONLY.

ctypes access to the two CPU checkers built by oracle/Makefile:

* ``Oracle`` -- the project's CPU restatement (oracle/cb_oracle.cpp ->
  oracle/_bin/libcboracle.so). Always buildable (g++ only).
* ``Reference`` -- the reference's own src/bubble.cpp compiled in place with
  the stand-ins of oracle/shim (oracle/_ref/libcbref.so). Only buildable where
  the reference sources are present.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module; the product (coolbubble_b200/) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_bin", "libcboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libcbref.so")
REF_EXE = os.path.join(HERE, "_ref", "coolbubble_ref")
# where the reference sources lie: CB_REFERENCE_SRC, else the checkout beside this repository
REF_SRC = os.environ.get("CB_REFERENCE_SRC") or os.path.normpath(os.path.join(HERE, "..", "..", "reference"))

SCALAR_NAMES = (
    "t", "a", "ap", "H", "C", "Etot", "Ekintot", "Egradtot", "Epottot", "avphi", "avphiP",
    "EkinHalfPrev", "EtotVar", "EkintotVar", "EgradtotVar", "EpottotVar", "avphiVar", "avphiPVar",
)

_dp = C.POINTER(C.c_double)


def _ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def build_oracle():
    """Build oracle/_bin/libcboracle.so if it is missing (g++ only)."""
    if not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    return ORACLE_SO


def reference_available():
    return os.path.exists(REF_SO) or os.path.isdir(os.path.join(REF_SRC, "src"))


def build_reference():
    if not (os.path.exists(REF_SO) and os.path.exists(REF_EXE)):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={REF_SRC}"], check=True)
    return REF_SO


class _OracleParams(C.Structure):
    _fields_ = [("d", C.c_int), ("n", C.c_int), ("L", C.c_double), ("c", C.c_double), ("dt", C.c_double),
                ("alpha", C.c_int), ("expansion", C.c_int), ("mpl", C.c_double), ("delta_v", C.c_double),
                ("memorysave", C.c_int)]


_olib = None


def _oracle_lib():
    global _olib
    if _olib is None:
        lib = C.CDLL(build_oracle())
        lib.cbo_create.restype = C.c_void_p
        lib.cbo_create.argtypes = [C.POINTER(_OracleParams), _dp, _dp]
        lib.cbo_destroy.argtypes = [C.c_void_p]
        lib.cbo_step.argtypes = [C.c_void_p, C.c_int]
        lib.cbo_fields.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp]
        lib.cbo_scalars.argtypes = [C.c_void_p, _dp]
        lib.cbo_nbins.argtypes = [C.c_int, C.c_int]
        lib.cbo_nbins.restype = C.c_int
        lib.cbo_bins.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int)]
        lib.cbo_spectrum.argtypes = [C.c_void_p, _dp, _dp, _dp]
        lib.cbo_spectrum_of.argtypes = [C.c_int, C.c_int, C.c_double, _dp, _dp, _dp, _dp]
        lib.cbo_r2c.argtypes = [C.c_int, C.c_int, _dp, _dp]
        lib.cbo_c2r.argtypes = [C.c_int, C.c_int, _dp, _dp]
        lib.cbo_set_threads.argtypes = [C.c_int]
        lib.cbo_get_threads.restype = C.c_int
        _olib = lib
    return _olib


def set_threads(n):
    _oracle_lib().cbo_set_threads(int(n))


def nbins(d, n):
    return _oracle_lib().cbo_nbins(d, n)


def bins(d, n):
    h = n // 2 + 1
    out = np.empty(n ** (d - 1) * h, dtype=np.int32)
    _oracle_lib().cbo_bins(d, n, out.ctypes.data_as(C.POINTER(C.c_int)))
    return out


def spectrum_of(d, n, L, field):
    field = np.ascontiguousarray(field, dtype=np.float64)
    nb = nbins(d, n)
    pw, ws, ks = np.zeros(nb), np.zeros(nb), np.zeros(nb)
    _oracle_lib().cbo_spectrum_of(d, n, float(L), _ptr(field), _ptr(pw), _ptr(ws), _ptr(ks))
    return pw, ws, ks


def r2c(d, n, field):
    field = np.ascontiguousarray(field, dtype=np.float64).reshape(-1)
    out = np.zeros(n ** (d - 1) * (n // 2 + 1), dtype=np.complex128)
    _oracle_lib().cbo_r2c(d, n, _ptr(field), out.view(np.float64).ctypes.data_as(_dp))
    return out


def c2r(d, n, half):
    half = np.array(half, dtype=np.complex128).reshape(-1)
    out = np.zeros(n ** d)
    _oracle_lib().cbo_c2r(d, n, half.view(np.float64).ctypes.data_as(_dp), _ptr(out))
    return out


class Oracle:
    """The CPU restatement of one lattice run (double precision)."""

    def __init__(self, d, n, L, c, dt, phi0, pi0=None, alpha=0, expansion=0, mpl=200.0, delta_v=1.0,
                 memorysave=0):
        self.d, self.n, self.L, self.memorysave = d, n, L, memorysave
        self.N = n ** d
        p = _OracleParams(d, n, L, c, dt, alpha, expansion, mpl, delta_v, memorysave)
        phi0 = np.ascontiguousarray(phi0, dtype=np.float64).reshape(-1)
        pi0 = None if pi0 is None else np.ascontiguousarray(pi0, dtype=np.float64).reshape(-1)
        assert phi0.size == self.N
        self._lib = _oracle_lib()
        self._h = self._lib.cbo_create(C.byref(p), _ptr(phi0), _ptr(pi0))

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.cbo_destroy(self._h)
            self._h = None

    def step(self, k=1):
        self._lib.cbo_step(self._h, int(k))

    def fields(self):
        out = [np.zeros(self.N) for _ in range(5)]
        self._lib.cbo_fields(self._h, *[_ptr(x) for x in out])
        return dict(zip(("phi", "pi", "ekin", "egrad", "epot"), out))

    def scalars(self):
        out = np.zeros(18)
        self._lib.cbo_scalars(self._h, _ptr(out))
        return dict(zip(SCALAR_NAMES, out.tolist()))

    def spectrum(self):
        nb = nbins(self.d, self.n)
        pw, ws, ks = np.zeros(nb), np.zeros(nb), np.zeros(nb)
        self._lib.cbo_spectrum(self._h, _ptr(pw), _ptr(ws), _ptr(ks))
        return pw, ws, ks


_rlib = None


def _ref_lib():
    global _rlib
    if _rlib is None:
        lib = C.CDLL(build_reference())
        lib.cbref_configure.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, C.c_double,
                                        C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_double,
                                        C.c_int]
        lib.cbref_create.restype = C.c_void_p
        lib.cbref_create.argtypes = [C.c_char_p]
        lib.cbref_destroy.argtypes = [C.c_void_p]
        lib.cbref_step.argtypes = [C.c_void_p, C.c_int]
        lib.cbref_fields.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp, _dp]
        lib.cbref_scalars.argtypes = [C.c_void_p, _dp]
        lib.cbref_spectrum.argtypes = [C.c_void_p, C.c_char_p]
        lib.cbref_spectrum.restype = C.c_int
        for f in ("cbref_out_ep", "cbref_out_parameters"):
            getattr(lib, f).argtypes = [C.c_void_p]
        for f in ("cbref_out_field", "cbref_fourier"):
            getattr(lib, f).argtypes = [C.c_void_p, C.c_int]
        _rlib = lib
    return _rlib


class Reference:
    """The reference's own Bubble (src/bubble.cpp), built in place.

    Its run parameters are process-wide globals (main.cpp:45-50), so only one
    instance should be alive at a time. The constructor writes its output
    files (EnergyDensities.dat header, __xns.dat) into ``folder``.
    """

    def __init__(self, d, n, L, c, mode, dt, nbubbles=5, trad=0.2, deltar=0.0, test=0, expansion=0, alpha=0,
                 mpl=200.0, memorysave=0, nt=1000, folder=None):
        self.d, self.n, self.L, self.memorysave = d, n, L, memorysave
        self.N = n ** d
        self._tmp = None
        if folder is None:
            self._tmp = tempfile.TemporaryDirectory(prefix="cbref_")
            folder = self._tmp.name
        os.makedirs(folder, exist_ok=True)
        self.folder = folder
        self._lib = _ref_lib()
        self._lib.cbref_configure(d, n, L, c, mode, nt, dt, nbubbles, trad, deltar, test, expansion, alpha, mpl,
                                  memorysave)
        self._h = self._lib.cbref_create(folder.encode())

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.cbref_destroy(self._h)
            self._h = None

    def step(self, k=1):
        self._lib.cbref_step(self._h, int(k))

    def fields(self):
        out = [np.zeros(self.N) for _ in range(6)]
        if self.memorysave:
            out[3] = out[4] = out[5] = None
        self._lib.cbref_fields(self._h, *[_ptr(x) for x in out])
        return dict(zip(("phi", "pi", "dpi", "ekin", "egrad", "epot"), out))

    def scalars(self):
        out = np.zeros(18)
        self._lib.cbref_scalars(self._h, _ptr(out))
        return dict(zip(SCALAR_NAMES, out.tolist()))

    def spectrum_lines(self):
        """(kMean, kMean/a, power/weight) rows of ComputePowerSpectrum, 17 digits."""
        with tempfile.NamedTemporaryFile(suffix=".dat", delete=False) as f:
            path = f.name
        try:
            assert self._lib.cbref_spectrum(self._h, path.encode()) == 0
            rows = np.loadtxt(path, ndmin=2)
        finally:
            os.unlink(path)
        return rows

    def xns_text(self):
        with open(os.path.join(self.folder, "__xns.dat")) as f:
            return f.read()
