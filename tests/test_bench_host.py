"""Host logic of bench.py (no GPU): where the energy lines fall in a timed
window, and the shared workload description of both benchmark arms."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402


def lines_of(start, K):
    """Absolute steps of a window that carry an energy line."""
    out, at = [], start
    for k, measure in bench.event_chunks(start, K):
        at += k
        if measure:
            out.append(at)
    return out


def test_lines_fall_on_main_loop_steps():
    # main.cpp:280 writes a line when it % 40 == 0, counting from the run's first step
    assert lines_of(0, 100) == [40, 80]
    assert lines_of(5, 20) == []
    assert lines_of(20, 20) == [40]
    assert lines_of(39, 2) == [40]
    assert lines_of(40, 1000) == list(range(80, 1041, 40))
    for start in (0, 7, 33, 40, 79):
        for K in (1, 20, 39, 40, 41, 123):
            assert sum(k for k, _ in bench.event_chunks(start, K)) == K


def test_padded_warmup_puts_a_line_in_every_window():
    for W in (3, 5, 10, 40):
        for K in (1, 20, 39, 40, 200, 1000):
            Wp = bench.padded_warmup(W, K)
            assert Wp >= W and (Wp + K) % 40 == 0 and Wp - W < 40
            got = lines_of(Wp, K)
            assert len(got) == max(1, K // 40) and got[-1] == Wp + K


def test_both_arms_describe_the_workload_alike():
    for name, w in bench.WORKLOADS.items():
        cfg = bench.workload_config(name, w)
        assert cfg["workload"] == name and cfg["dt"] == 0.1 * w["L"] / w["n"]
        assert "precision" not in cfg            # the arms' arithmetic differs; the workload does not
    assert "thermal" in bench.workload_config("thermal-d3-n512", bench.WORKLOADS["thermal-d3-n512"])["ic"]
