"""The N > 1 path of bench.py on CPU: two gloo ranks (127.0.0.1) run the
rank plumbing the benchmark uses -- barrier, max-over-ranks timing, weak-
scaling aggregation of independent replicas -- with no GPU."""
import os
import socket
import subprocess
import sys
import textwrap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = textwrap.dedent("""
    import json, os, sys, time
    sys.path.insert(0, %r)
    import bench
    ws, rank, local = bench.dist_env()
    dist = bench.init_dist(ws)
    bench.barrier(dist)
    t = 0.1 * (rank + 1)                  # rank 1 is the slow one
    worst = bench.max_over_ranks(dist, t)
    sites, steps = 1000, 10
    value = ws * sites * steps / worst     # the weak-scaling aggregate bench.py reports
    bench.barrier(dist)
    print(json.dumps(dict(rank=rank, ws=ws, local=local, worst=worst, value=value)), flush=True)
    dist.destroy_process_group()
""") % ROOT


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_gloo_ranks_agree_on_max_time():
    import json
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, WORLD_SIZE="2", RANK=str(rank), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=180)
        assert p.returncode == 0, e
        outs.append(json.loads(o.strip().splitlines()[-1]))
    for o in outs:
        assert o["ws"] == 2
        assert abs(o["worst"] - 0.2) < 1e-12          # both ranks see the slower rank's time
        assert abs(o["value"] - 2 * 1000 * 10 / 0.2) < 1e-6


def test_reference_arm_on_other_ranks_exits_quietly():
    """Under torchrun the reference arm runs on rank 0 only; other ranks exit 0 without work."""
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
