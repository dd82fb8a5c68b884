"""The request loop: device-built starts, continuous batching, admission
against a budget, timeouts, cancellation and host-side injected failures.
Results must be the same alone and in a mix (bit for bit: a run's kernels do
not depend on the other runs)."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _params(d, n, L, c, prec="fp32c", expansion=0, mpl=200.0):
    import coolbubble_b200 as cb
    return cb.make_params(d, n, L, c, 0.1 * L / n, precision=prec, memorysave=1, expansion=expansion, mpl=mpl)


@pytest.mark.parametrize("d,n,L,c,mode", [(2, 64, 16.0, 4.0, 1), (3, 32, 16.0, 4.0, 1), (2, 48, 24.0, 2.0, -3),
                                          (3, 24, 24.0, 3.0, -3), (2, 40, 16.0, 5.0, -1), (3, 24, 16.0, 6.0, -2),
                                          (1, 256, 32.0, 4.0, 1)])
def test_device_start_matches_host_start(d, n, L, c, mode):
    import coolbubble_b200 as cb
    from coolbubble_b200.ic import initial_condition
    from coolbubble_b200.serving import create_from_seed, ic_params
    p = _params(d, n, L, c, prec="fp64")
    phi0, pi0, _ = initial_condition(p, mode=mode, n_bubbles=6, trad=0.1, position_seed=77, thermal_seed=99)
    host = cb.Bubble(p, phi0, pi0)
    dev = create_from_seed(p, ic_params(mode=mode, n_bubbles=6, trad=0.1, position_seed=77, thermal_seed=99))
    a, b = host.fields(local=False), dev.fields(local=False)
    for k in ("phi", "pi"):
        scale = max(np.abs(a[k]).max(), 1e-300)
        assert np.abs(a[k] - b[k]).max() <= 1e-13 * scale, k
    if mode == -3:
        np.testing.assert_array_equal(a["phi"], b["phi"])   # same modes, same inverse DFT, same scaling
    assert dev.Etot == pytest.approx(host.Etot, rel=1e-12)


def _runs():
    from coolbubble_b200.serving import ic_params
    return [
        (_params(2, 128, 16.0, 4.0), ic_params(mode=1, n_bubbles=5, position_seed=3), 300),
        (_params(3, 64, 16.0, 3.0, expansion=1, mpl=10.0), ic_params(mode=1, n_bubbles=4, position_seed=4), 200),
        (_params(3, 48, 24.0, 2.0), ic_params(mode=-3, trad=0.05, thermal_seed=5), 240),
        (_params(2, 192, 32.0, 6.0), ic_params(mode=-3, trad=0.08, thermal_seed=6), 120),
        (_params(3, 64, 16.0, 5.0, prec="fp64"), ic_params(mode=1, n_bubbles=3, position_seed=7), 160),
    ]


def test_results_are_the_same_alone_and_in_the_mix():
    from coolbubble_b200.serving import Pool, DONE
    runs = _runs()
    alone = []
    pool = Pool(8 << 30, 1)
    for p, ic, nt in runs:
        rid = pool.submit(p, ic, nt, sums_every=40, want_fields=True)
        assert pool.wait(rid) == 0
        alone.append(pool.result(rid, n_sites=p.n_grids ** p.d))
    pool.close()
    pool = Pool(8 << 30, 8)
    ids = [pool.submit(p, ic, nt, sums_every=40, want_fields=True) for p, ic, nt in runs]
    mixed = []
    for rid, (p, ic, nt) in zip(ids, runs):
        assert pool.wait(rid) == 0
        mixed.append(pool.result(rid, n_sites=p.n_grids ** p.d))
    st = pool.stats()
    pool.close()
    assert st["completed"] == len(runs) and st["failed"] == 0
    for a, b, (p, ic, nt) in zip(alone, mixed, runs):
        assert a["state"] == b["state"] == DONE
        assert len(a["lines"]) == len(b["lines"]) == nt // 40
        assert a["lines"] == b["lines"]
        np.testing.assert_array_equal(a["phi"], b["phi"])
        np.testing.assert_array_equal(a["pi"], b["pi"])


def test_admission_keeps_within_budget_and_all_finish():
    import coolbubble_b200 as cb
    from coolbubble_b200 import _lib as L
    from coolbubble_b200.serving import Pool, ic_params
    import ctypes as C
    p = _params(3, 64, 16.0, 4.0)
    one = L.lib.cb_footprint_bytes(C.byref(p)) + 2 * 8 * 64 ** 3
    budget = int(2.5 * one)             # room for two runs at a time
    pool = Pool(budget, 16)
    ids = [pool.submit(p, ic_params(mode=1, n_bubbles=3, position_seed=10 + i), 400, sums_every=40) for i in range(6)]
    peak_active, peak_used = 0, 0
    t0 = time.time()
    while time.time() - t0 < 120:
        s = pool.stats()
        peak_active = max(peak_active, s["active"])
        peak_used = max(peak_used, s["used_bytes"])
        assert s["used_bytes"] <= budget
        if s["completed"] + s["failed"] == len(ids):
            break
        time.sleep(0.002)
    s = pool.stats()
    pool.close()
    assert s["completed"] == len(ids)
    assert 1 <= peak_active <= 2
    assert s["site_updates"] == pytest.approx(6 * 400 * 64 ** 3)


def test_oversized_run_fails_and_others_continue():
    from coolbubble_b200.serving import Pool, ic_params, FAILED, DONE
    pool = Pool(64 << 20, 4)
    big = pool.submit(_params(3, 256, 32.0, 4.0), ic_params(), 10)
    small = pool.submit(_params(2, 64, 16.0, 4.0), ic_params(), 80)
    assert pool.wait(big) == 0 and pool.wait(small) == 0
    rb, rs = pool.result(big), pool.result(small)
    pool.close()
    assert rb["state"] == FAILED and "budget" in rb["err"]
    assert rs["state"] == DONE


def test_timeout_and_cancel():
    from coolbubble_b200 import _lib as L
    from coolbubble_b200.serving import Pool, ic_params, CANCELLED
    pool = Pool(8 << 30, 2)
    rid = pool.submit(_params(3, 128, 32.0, 4.0), ic_params(mode=1, n_bubbles=3), 200000, sums_every=1000)
    assert pool.wait(rid, 50) == L.CB_ETIMEOUT
    pool.cancel(rid)
    assert pool.wait(rid, 60000) == 0
    r = pool.result(rid)
    pool.close()
    assert r["state"] == CANCELLED


def test_injected_admission_failure_is_contained():
    from coolbubble_b200.serving import Pool, ic_params, FAILED, DONE, INJECT_ADMISSION_FAILURE
    pool = Pool(8 << 30, 4)
    pool.inject(INJECT_ADMISSION_FAILURE)
    a = pool.submit(_params(2, 64, 16.0, 4.0), ic_params(), 80)
    b = pool.submit(_params(2, 64, 16.0, 4.0), ic_params(position_seed=8), 80)
    assert pool.wait(a) == 0 and pool.wait(b) == 0
    ra, rb = pool.result(a), pool.result(b)
    s = pool.stats()
    pool.close()
    assert ra["state"] == FAILED and "injected" in ra["err"]
    assert rb["state"] == DONE
    assert s["used_bytes"] == 0


def test_injected_worker_failure_fails_runs_and_refuses_new_ones():
    from coolbubble_b200 import _lib as L
    from coolbubble_b200.serving import Pool, ic_params, FAILED, INJECT_WORKER_EXCEPTION
    pool = Pool(8 << 30, 4)
    ids = [pool.submit(_params(3, 64, 16.0, 4.0), ic_params(position_seed=i), 100000, sums_every=1000) for i in range(3)]
    time.sleep(0.2)
    pool.inject(INJECT_WORKER_EXCEPTION)
    for rid in ids:
        assert pool.wait(rid, 60000) == 0
        r = pool.result(rid)
        assert r["state"] == FAILED and "worker stopped" in r["err"]
    with pytest.raises(L.CBError) as e:
        pool.submit(_params(2, 64, 16.0, 4.0), ic_params(), 10)
    assert "worker stopped" in str(e.value)
    pool.close()
