"""HDF5 snapshot files without libhdf5 (coolbubble_b200/csrc/cb_h5.cpp).

The reference writes snapshots through the HDF5 C++ library
(src/bubble.cpp:919-953): chunked float datasets, shuffle + deflate 9, scalar
double attributes on the root group. Neither libhdf5 nor h5py is installed
here, so:

  1. the strict test reader tests/h5read.py is pinned first on a file written
     by libhdf5 itself (scipy's MATLAB 7.3 test file), whose values are
     checked against scipy's own read of the same variable from the MATLAB 5
     copy of that file;
  2. files written by the library are read back with it: values bit-exact,
     chunk grid, filters and attributes as requested, every structure inside
     the file and none overlapping;
  3. every stored chunk equals zlib's compress2 (level 9) of the shuffled
     chunk, the bytes libhdf5's deflate filter stores, when Python's zlib is
     the same zlib the library links.

CPU only: the writer is host code. The GPU part (cb_out_field against the
reference's own snapshots) is in tests/test_driver.py and tests/test_h5_gpu.py.
"""
import ctypes
import os
import zlib

import numpy as np
import pytest

import h5read
from coolbubble_b200 import CBError
from coolbubble_b200 import _lib as L
from coolbubble_b200.h5 import write_floats

SCIPY_DATA = None
try:
    import scipy.io.matlab as _m
    SCIPY_DATA = os.path.join(os.path.dirname(_m.__file__), "tests", "data")
except Exception:   # pragma: no cover
    pass


def _scipy_file(name):
    p = os.path.join(SCIPY_DATA or "", name)
    if not SCIPY_DATA or not os.path.exists(p):
        pytest.skip("scipy's MATLAB test files are not installed")
    return p


def test_reader_on_a_file_written_by_libhdf5():
    import scipy.io as sio
    f = h5read.File(_scipy_file("testhdf5_7.4_GLNX86.mat"))
    assert f.base == 512                                  # MATLAB's user block
    assert f.keys() == ["testdouble"]
    d = f["testdouble"]
    assert d.kind == "contiguous" and d.dtype == np.float64 and d.shape == (9, 1)
    assert d.attrs["MATLAB_class"] == b"double"
    v5 = sio.loadmat(_scipy_file("testdouble_7.4_GLNX86.mat"))["testdouble"]
    np.testing.assert_array_equal(d[:], v5.T)            # MATLAB stores the transpose
    np.testing.assert_allclose(d[:].ravel(), np.arange(9) * np.pi / 4, rtol=1e-15)


def _shuffle(a):
    return np.frombuffer(np.ascontiguousarray(a, np.float32).tobytes(), np.uint8).reshape(-1, 4).T.copy().tobytes()


def _chunk_payloads(path, name):
    """(offset, mask, stored bytes) of every chunk of a dataset, in key order."""
    f = h5read.File(path)
    d = f[name]
    leaves = []
    f._chunk_tree(d.btree, len(d.shape) + 1, None, leaves)
    return d, [(k[2][:-1], k[1], f.buf[f.base + a:f.base + a + k[0]]) for k, a in leaves]


CASES = [
    # shape, chunks: whole field (1-D), row blocks with an edge chunk (2-D), planes (3-D),
    # and enough chunks for two and three B-tree levels
    ((1000,), (1000,)),
    ((37, 50), (16, 50)),
    ((12, 20, 20), (1, 20, 20)),
    ((200, 32), (2, 32)),
    ((70000,), (10,)),
    ((5, 7, 9), (2, 3, 4)),
]


@pytest.mark.parametrize("shape,chunks", CASES)
def test_round_trip(tmp_path, shape, chunks):
    rng = np.random.default_rng(len(shape) * 1000 + shape[0])
    data = {
        "phi": rng.standard_normal(shape).astype(np.float32),              # hardly compressible
        "pi": np.full(shape, 0.25, np.float32),                            # very compressible
        "gradphi": (np.arange(np.prod(shape)).reshape(shape) % 7).astype(np.float32),
    }
    attrs = {"D": float(len(shape)), "L": 32.0, "nGrids": float(shape[0]), "t": 1.0 / 3.0, "a": 1.25}
    p = tmp_path / "x.h5"
    write_floats(p, data, chunks, attrs)
    f = h5read.File(str(p))
    assert sorted(f.keys()) == sorted(data)
    for k, v in data.items():
        d = f[k]
        assert d.kind == "chunked" and d.chunks == chunks and d.dtype == np.float32 and d.shape == shape
        assert [(x["id"], x["name"], x["cd"]) for x in d.filters] == [(2, "shuffle", [4]), (1, "deflate", [9])]
        got = d.read()
        assert got.tobytes() == v.tobytes()
        n_chunks = int(np.prod([-(-s // c) for s, c in zip(shape, chunks)]))
        assert d.chunk_count == n_chunks
    assert {k: float(v) for k, v in f.attrs.items()} == attrs
    assert f.regions[-1][0] + f.regions[-1][1] <= f.eof
    assert sum(s for _, s, _ in f.regions) == f.eof      # every byte of the file belongs to one structure


def test_compressible_chunks_are_smaller(tmp_path):
    p = tmp_path / "c.h5"
    write_floats(p, {"phi": np.zeros((64, 64), np.float32)}, (16, 64))
    d = h5read.File(str(p))["phi"]
    d.read()
    assert d.chunk_bytes < 64 * 64 * 4 // 20 and set(d.chunk_masks) == {0}


def test_incompressible_chunk_is_stored_shuffled_only(tmp_path):
    """A chunk that deflate would grow keeps the deflate bit in its filter mask."""
    rng = np.random.default_rng(7)
    v = rng.integers(0, 2**32, size=(4, 64), dtype=np.uint32).view(np.float32)
    v = np.where(np.isfinite(v), v, 1.0).astype(np.float32)
    p = tmp_path / "r.h5"
    write_floats(p, {"phi": v}, (4, 64))
    d, chunks = _chunk_payloads(str(p), "phi")
    assert d.read().tobytes() == v.tobytes()
    (off, mask, raw), = chunks
    assert mask == 2 and raw == _shuffle(v)


def test_bytes_do_not_depend_on_threads(tmp_path):
    rng = np.random.default_rng(3)
    data = {"phi": rng.standard_normal((40, 30, 30)).astype(np.float32), "pi": np.ones((40, 30, 30), np.float32)}
    outs = []
    for t in (1, 3, 8):
        p = tmp_path / ("t%d.h5" % t)
        write_floats(p, data, (1, 30, 30), {"t": 2.0}, threads=t)
        outs.append(p.read_bytes())
    assert outs[0] == outs[1] == outs[2]


def _system_zlib_version():
    try:
        z = ctypes.CDLL("libz.so.1")
    except OSError:
        return None
    z.zlibVersion.restype = ctypes.c_char_p
    return z.zlibVersion().decode()


def test_chunks_are_what_the_deflate_filter_stores(tmp_path):
    """libhdf5's deflate filter stores compress2(shuffled chunk, level); with the
    same zlib the stored chunks must be those bytes exactly."""
    if _system_zlib_version() != zlib.ZLIB_RUNTIME_VERSION:
        pytest.skip("Python's zlib is not the zlib the library links")
    rng = np.random.default_rng(11)
    phi = np.tanh(np.linspace(-4, 4, 48 * 48)).reshape(48, 48).astype(np.float32)
    phi += (1e-3 * rng.standard_normal(phi.shape)).astype(np.float32)
    p = tmp_path / "z.h5"
    write_floats(p, {"phi": phi}, (16, 48))
    _, chunks = _chunk_payloads(str(p), "phi")
    assert len(chunks) == 3
    for (off, mask, raw) in chunks:
        block = phi[off[0]:off[0] + 16]
        assert mask == 0
        assert raw == zlib.compress(_shuffle(block), 9)


def test_links_are_sorted_by_name(tmp_path):
    names = ["phi", "pi", "Ekin", "gradphi", "potEnergy"]       # the reference's order (bubble.cpp:896-903)
    p = tmp_path / "s.h5"
    write_floats(p, {k: np.full((8, 8), i, np.float32) for i, k in enumerate(names)}, (8, 8))
    f = h5read.File(str(p))
    assert f.keys() == sorted(names, key=lambda s: s.encode())
    for i, k in enumerate(names):
        assert (f[k][:] == i).all()


@pytest.mark.parametrize("kw,status", [
    (dict(chunks=(9, 8)), L.CB_EINVAL),                  # chunk larger than the dataset
    (dict(deflate_level=10), L.CB_EINVAL),
    (dict(path="/nonexistent-dir/x.h5"), L.CB_EIO),
])
def test_errors(tmp_path, kw, status):
    args = dict(path=tmp_path / "e.h5", datasets={"phi": np.zeros((8, 8), np.float32)}, chunks=(4, 8))
    args.update(kw)
    with pytest.raises(CBError) as e:
        write_floats(args.pop("path"), **args)
    assert e.value.status == status


def test_duplicate_and_too_many_datasets(tmp_path):
    a = np.zeros(4, np.float32)
    names = (L.C.c_char_p * 2)(b"phi", b"phi")
    data = (L._fp * 2)(L.fptr(a), L.fptr(a))
    dims = (L.C.c_int64 * 1)(4)
    st = L.lib.cb_h5_write_floats(str(tmp_path / "d.h5").encode(), 1, dims, dims, 2, names, data, 0, None, None, 9, 1)
    assert st == L.CB_EINVAL and b"twice" in L.lib.cb_last_error(None)
    with pytest.raises(CBError):
        write_floats(tmp_path / "m.h5", {"x%d" % i: a for i in range(9)}, (4,))


def _h5py_stand_in():
    """The part of h5py that the reference's reader uses (File as a context
    manager, `name in f`, f[name][:], f.attrs), over the strict test reader."""
    import types

    class _File:
        def __init__(self, path, mode="r"):
            assert mode == "r"
            self._f = h5read.File(str(path))
            self.attrs = self._f.attrs

        def __enter__(self):
            return self

        def __exit__(self, *exc):
            return False

        def __contains__(self, name):
            return name in self._f

        def __getitem__(self, name):
            return self._f[name]

    mod = types.ModuleType("h5py")
    mod.File = _File
    return mod


def test_reference_reader_opens_the_snapshots(tmp_path, monkeypatch):
    """The reference's own snapshot reader (python/runfiles.py, read_snapshot)
    on files with OutField's layout written by this library: fields, axes from
    the stored thinning stride, t and a."""
    import importlib.util
    import sys
    from oracle.bridge import REF_SRC as ref   # where the reference sources lie
    src = os.path.join(ref, "python", "runfiles.py")
    if not os.path.exists(src):
        pytest.skip("the reference sources are not present")
    monkeypatch.setitem(sys.modules, "h5py", _h5py_stand_in())
    spec = importlib.util.spec_from_file_location("reference_runfiles", src)
    runfiles = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(runfiles)
    rng = np.random.default_rng(21)
    for D, n_grids, reduc in [(2, 64, 1), (2, 4100, 2), (3, 16, 1), (1, 40, 1)]:
        m = -(-n_grids // reduc)
        shape = (m,) * D
        chunk = {1: (m,), 2: (min(m, max(1, 65536 // m)), m), 3: (1, m, m)}[D]
        data = {k: rng.standard_normal(shape).astype(np.float32) for k in ("phi", "pi", "gradphi")}
        attrs = {"D": D, "L": 16.0, "nGrids": n_grids, "reduc": reduc, "c": 4.0, "t": 2.5, "a": 1.5}
        p = tmp_path / ("_phi_t=%04d.h5" % n_grids)
        write_floats(p, data, chunk, attrs)
        fields, axes, info = runfiles.read_snapshot(p, {"D": D, "L": 16.0, "nGrids": n_grids})
        for k, v in data.items():
            assert fields[k].shape == shape and fields[k].tobytes() == v.tobytes()
        assert info == {"t": 2.5, "a": 1.5, "reduc": float(reduc)}
        assert len(axes) == D
        np.testing.assert_allclose(axes[0], (np.arange(m) * reduc + 0.5) * 16.0 / n_grids, rtol=0, atol=0)


def test_host_allocation_failure_is_a_status(tmp_path):
    """Nothing throws across the C ABI: an index of 2^40 chunks cannot be
    allocated, and the call returns CB_ENOMEM with a message instead of
    ending the process (no data is read before the allocation)."""
    a = np.zeros(4, np.float32)
    names = (L.C.c_char_p * 1)(b"phi")
    data = (L._fp * 1)(L.fptr(a))
    dims, chunk = (L.C.c_int64 * 1)(1 << 40), (L.C.c_int64 * 1)(1)
    st = L.lib.cb_h5_write_floats(str(tmp_path / "huge.h5").encode(), 1, dims, chunk, 1, names, data, 0, None, None,
                                  9, 1)
    assert st == L.CB_ENOMEM
    assert b"allocation" in L.lib.cb_last_error(None)
