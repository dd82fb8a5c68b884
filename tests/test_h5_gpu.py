"""cb_out_field / Bubble.OutField on the GPU: the snapshot file the reference's
Bubble::OutField writes (bubble.cpp:887-953), read back with the strict test
reader tests/h5read.py. Payloads are bit-exact against the fields downloaded
as float (the same conversion on the device); thinning (every reduc-th point
above 2048^2 and 512^3), chunking, filters and attributes follow OutField."""
import numpy as np
import pytest

import h5read
import coolbubble_b200 as cb

pytestmark = pytest.mark.gpu


def _bubble(d, n, precision, memorysave, seed=0):
    L = n / 8.0
    p = cb.make_params(d, n, L, 2.0, 0.1 * L / n, precision=precision, memorysave=memorysave)
    rng = np.random.default_rng(seed)
    N = n ** d
    return cb.Bubble(p, 0.3 * rng.random(N), 0.01 * rng.standard_normal(N))


def _reference_chunks(D, m):
    return {1: (m,), 2: (min(m, max(1, 65536 // m)), m), 3: (1, m, m)}[D]


@pytest.mark.parametrize("d,n,precision,memorysave", [
    (1, 1000, "fp64", 0),
    (2, 96, "fp32c", 1),
    (3, 64, "fp64", 0),
    (3, 48, "fp32c", 0),
])
def test_out_field(tmp_path, d, n, precision, memorysave):
    s = _bubble(d, n, precision, memorysave)
    s.step(3, sums=True, local=memorysave == 0)
    path = tmp_path / "_phi_t=0001.h5"
    s.OutField(path)
    ref = s.fields_f32(local=memorysave == 0)
    sums = s.sums()
    s.close()
    f = h5read.File(str(path))
    names = {"phi": "phi", "pi": "pi"}
    if memorysave == 0:
        names.update({"Ekin": "ekin", "gradphi": "egrad", "potEnergy": "epot"})
    assert sorted(f.keys()) == sorted(names)
    for name, key in names.items():
        ds = f[name]
        assert ds.shape == (n,) * d and ds.chunks == _reference_chunks(d, n)
        assert [(x["name"], x["cd"]) for x in ds.filters] == [("shuffle", [4]), ("deflate", [9])]
        assert ds[:].ravel().tobytes() == ref[key].tobytes()
    a = {k: float(v) for k, v in f.attrs.items()}
    assert a == {"D": d, "L": n / 8.0, "nGrids": n, "reduc": 1, "c": 2.0, "t": sums["t"], "a": sums["a"]}


def test_out_field_thins_large_2d_lattices(tmp_path):
    """2-D above 2048^2: every reduc-th point per axis, reduc = n / 2048 (bubble.cpp:891-895)."""
    n = 4100
    s = _bubble(2, n, "fp32c", 1, seed=5)
    path = tmp_path / "big.h5"
    s.OutField(path)
    phi = s.fields_f32(local=False)["phi"].reshape(n, n)
    s.close()
    f = h5read.File(str(path))
    m = (n + 1) // 2
    assert f.attrs["reduc"] == 2 and f.attrs["nGrids"] == n
    assert f["phi"].shape == (m, m) and f["phi"].chunks == _reference_chunks(2, m) == (31, m)
    assert f["phi"][:].tobytes() == phi[::2, ::2].tobytes()


def test_background_write_overlaps_steps(tmp_path):
    """cb_out_field_async: the file holds the fields of the call's time even though
    the run steps on while it is written; one write in flight per handle."""
    from coolbubble_b200 import CBError
    from coolbubble_b200 import _lib as L
    s = _bubble(3, 64, "fp32c", 0, seed=2)
    s.step(2, sums=True, local=True)
    ref = s.fields_f32()
    t0 = s.sums()["t"]
    s.OutField(tmp_path / "a.h5", background=True)
    with pytest.raises(CBError) as e:
        s.OutField(tmp_path / "b.h5")
    assert e.value.status == L.CB_EBUSY
    s.step(5, sums=True)
    s.OutFieldWait()
    s.OutFieldWait()                                  # nothing in flight: OK
    s.OutField(tmp_path / "c.h5", background=True)   # collected by close()
    later = s.fields_f32(local=False)
    s.close()
    f = h5read.File(str(tmp_path / "a.h5"))
    assert f["phi"][:].ravel().tobytes() == ref["phi"].tobytes()
    assert f["potEnergy"][:].ravel().tobytes() == ref["epot"].tobytes()
    assert float(f.attrs["t"]) == t0
    g = h5read.File(str(tmp_path / "c.h5"))
    assert g["phi"][:].ravel().tobytes() == later["phi"].tobytes()
    assert not (tmp_path / "b.h5").exists()


def test_background_write_error_is_reported_by_wait(tmp_path):
    from coolbubble_b200 import CBError
    from coolbubble_b200 import _lib as L
    s = _bubble(2, 64, "fp32c", 1)
    s.OutField(tmp_path / "missing-dir" / "x.h5", background=True)
    with pytest.raises(CBError) as e:
        s.OutFieldWait()
    assert e.value.status == L.CB_EIO
    s.OutField(tmp_path / "ok.h5")                   # the handle is usable afterwards
    s.close()
    assert sorted(h5read.File(str(tmp_path / "ok.h5")).keys()) == ["phi", "pi"]
