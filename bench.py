"""Benchmark of the lattice-evolution path (one JSON line on rank 0).

Headline workload: the d = 3, N = 512, L = 64, c = 2 static lattice with the
reference's mode -3 thermal start (Trad = 0.05, thermal seed 12345;
dt = 0.1 dx), evolved in the FP32-compensated path; the plain FP64 path is
timed on the same lattice for the "vs plain FP64" figure. A "step" is one
leapfrog step over the whole lattice; box averages are measured on the steps
the reference's main loop writes them (every OutEnergyEvery = 40 steps,
def.h:65, counted from the start of the run, warm-up included; the warm-up is
lengthened so that the timed window ends on such a step and always holds its
share of them).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Timing: device time from CUDA events on the run's own stream, after the
warm-up, barrier and synchronisation on both sides; max over ranks. The
2 x 512^3 float fields (1 GiB) exceed the 126 MB L2, so no flush is needed
between steps. Multi-GPU: every rank evolves its own lattice (independent
runs, no collective on the data path: weak scaling).

On one GPU the same line also carries the other workloads under "configs":
the 512^2 FP64 run with 5 bubbles (all 1000 steps), the 256^3 expanding run
with 8 bubbles (FP32C and FP64), the ensemble of 256 lattices and two serving
streams (p50/p99 completion latency). The CPU baseline is the reference arm
run in a fresh process (`--impl reference`), the same code and settings as
the driver's reference run.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

# Runs of the serving loop and members of an ensemble each have their own
# stream; more hardware work queues than the default 8 keep unrelated streams
# from queueing behind one another. Read when the CUDA context is created.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # the headline: a 512^3 static lattice, c = 2, the reference's thermal start (HBM-resident stencil)
    "thermal-d3-n512": dict(d=3, n=512, L=64.0, c=2.0, expansion=0, mpl=200.0, precision="fp32c", nt=4000,
                            ic=dict(mode=-3, trad=0.05)),
    # the same stencil at 256^3 (2 x 64 MiB fields), for profiler captures
    "thermal-d3-n256": dict(d=3, n=256, L=32.0, c=2.0, expansion=0, mpl=200.0, precision="fp32c", nt=4000,
                            ic=dict(mode=-3, trad=0.05)),
    # a 256^3 lattice with 8 bubbles and the self-consistent expanding background (Mpl = 10)
    "bubbles-d3-n256-expanding": dict(d=3, n=256, L=32.0, c=4.0, expansion=1, mpl=10.0, precision="fp32c",
                                      nt=2000, ic=dict(mode=1, n_bubbles=8)),
    # the 512^2 run with 5 bubbles the reference can run on its host (FP64 throughout)
    "bubbles-d2-n512": dict(d=2, n=512, L=32.0, c=4.0, expansion=0, mpl=200.0, precision="fp64", nt=1000,
                            ic=dict(mode=1, n_bubbles=5)),
    # a large 2-D lattice (column-strip kernel), for profiler captures
    "plain-d2-n8192": dict(d=2, n=8192, L=1024.0, c=4.0, expansion=0, mpl=200.0, precision="fp32c", nt=1000,
                           ic=dict(mode="noise")),
}
OUT_ENERGY_EVERY = 40
BYTES_PER_SITE = {"fp32c": 16, "fp64": 32}   # read + write phi and pi once per step


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def committed_traffic(workload, precision):
    """DRAM bytes per launch of the step kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get(f"{workload}:{precision}")
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 100 ms."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None
        self.marks = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append((time.perf_counter(), line.strip()))

    def mark(self):
        self.marks.append(time.perf_counter())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        t0, t1 = (self.marks + [0, 1e30])[:2]
        rows = [s for (t, s) in self.samples if t0 - 0.05 <= t <= t1 + 0.15] or [s for (_, s) in self.samples]
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            parts = [p.strip() for p in r.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def event_chunks(start, K, every=OUT_ENERGY_EVERY):
    """Steps start+1 .. start+K of a run cut at its energy lines: (steps, measure)
    pairs, measure true for a chunk ending on a step main.cpp writes a line at
    (it % every == 0, main.cpp:280)."""
    out, done = [], 0
    while done < K:
        at = start + done
        k = min(every - at % every, K - done)
        out.append((k, (at + k) % every == 0))
        done += k
    return out


def padded_warmup(W, K, every=OUT_ENERGY_EVERY):
    """The smallest warm-up >= W after which a K-step window ends on an energy line."""
    return W + (-(W + K)) % every


def ic_text(w):
    ic = w["ic"]
    if ic["mode"] == -3:
        return "reference mode -3 thermal start: Trad %g, thermal seed 12345" % ic["trad"]
    if ic["mode"] == 1:
        return "reference mode 1: %d bubbles placed by srand(42)" % ic["n_bubbles"]
    return "seeded gaussian fluctuations, amplitude 0.05"


def workload_config(wname, w):
    """The workload as both arms run it (the same dict on both lines)."""
    cfg = {"workload": wname, "d": w["d"], "n": w["n"], "L": w["L"], "c": w["c"], "dt": 0.1 * w["L"] / w["n"],
           "expansion": w["expansion"], "ic": ic_text(w), "sums_every": OUT_ENERGY_EVERY}
    if w["expansion"]:
        cfg["mpl"] = w["mpl"]
    return cfg


def thermal_like_ic(n, d, seed):
    """Seeded Gaussian fluctuations around the false vacuum (phi = 0); the step's
    cost does not depend on the values."""
    rng = np.random.default_rng(seed)
    N = n ** d
    phi = rng.standard_normal(N, dtype=np.float32).astype(np.float64) * 0.05
    pi = rng.standard_normal(N, dtype=np.float32).astype(np.float64) * 0.05
    return phi, pi


def make_start(w, rank=0):
    """The workload's start at t = 0 (phi0, pi0), drawn by the library's host IC
    (cb_initial_condition: the reference's placement and thermal streams)."""
    ic = w["ic"]
    if ic["mode"] == "noise":
        return thermal_like_ic(w["n"], w["d"], seed=1 + rank)
    import coolbubble_b200 as cb
    from coolbubble_b200.ic import initial_condition
    p = cb.make_params(w["d"], w["n"], w["L"], w["c"], 0.1 * w["L"] / w["n"], expansion=w["expansion"],
                       mpl=w["mpl"], precision="fp64", memorysave=1)
    phi0, pi0, _ = initial_condition(p, mode=ic["mode"], n_bubbles=ic.get("n_bubbles", 5),
                                     trad=ic.get("trad", 0.2), thermal_seed=12345 + rank)
    return phi0, pi0


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def init_dist(ws):
    if ws <= 1:
        return None
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    return dist


def max_over_ranks(dist, x):
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


class quiet_stdout:
    """Send file descriptor 1 to /dev/null (the reference prints from C++)."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


def cpu_sample(w, max_steps, budget_s):
    with quiet_stdout():
        return _cpu_sample(w, max_steps, budget_s)


def _cpu_sample(w, max_steps, budget_s):
    """Time the reference's own CPU step (oracle/_ref, built from the reference
    sources) on this host's cores with the workload's own start, else the CPU
    restatement; bounded by max_steps and budget_s. Returns (site-updates/s,
    kind, cores, sample)."""
    from oracle import bridge as B
    cores = cpu_threads()
    os.environ["OMP_NUM_THREADS"] = str(cores)
    d, n, L, c = w["d"], w["n"], w["L"], w["c"]
    dt = 0.1 * L / n
    N = n ** d
    ic = w["ic"]
    t_setup = time.perf_counter()
    if os.path.exists(B.REF_SO) and ic["mode"] != "noise":
        kind = "reference"
        obj = B.Reference(d, n, L, c, ic["mode"], dt, nbubbles=ic.get("n_bubbles", 5), trad=ic.get("trad", 0.2),
                          expansion=w["expansion"], mpl=w["mpl"], memorysave=1)
        what = "reference Bubble::oneStep (src/bubble.cpp:849-876, FP64, OpenMP) from its own constructor's start"
    else:
        kind = "port"
        B.set_threads(cores)
        phi0, pi0 = thermal_like_ic(n, d, seed=1)
        obj = B.Oracle(d, n, L, c, dt, phi0, pi0, expansion=w["expansion"], mpl=w["mpl"], memorysave=1)
        what = "CPU restatement of Bubble::oneStep (FP64, OpenMP)"
    setup = time.perf_counter() - t_setup
    obj.step(1)   # warm-up (page faults, thread start)
    steps, t0 = 0, time.perf_counter()
    while steps < max_steps:
        obj.step(1)
        steps += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    del obj
    sample = (f"{steps} step(s) of the full {n}^{d} lattice: {what}; {cores} threads; "
              f"set-up {setup:.1f} s untimed")
    return N * steps / el, kind, cores, sample


def run_reference_arm(args, w, wname):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    value, kind, cores, sample = cpu_sample(w, max_steps=max(1, args.steps), budget_s=120.0)
    line = {
        "impl": "reference", "metric": "lattice site-updates/s", "value": value, "unit": "site-updates/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(wname, w),
        "cpu_baseline": {"value": value, "unit": "site-updates/s", "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": "site-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline_subprocess(wname, steps=20):
    """The reference arm in a fresh process (nothing else loaded, all host
    threads free); its line's cpu_baseline object, or None."""
    cmd = [sys.executable, os.path.abspath(__file__), "--impl", "reference", "--workload", wname,
           "--steps", str(steps), "--warmup", "1"]
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=900, env=env)
        for ln in reversed(r.stdout.strip().splitlines()):
            if ln.startswith("{"):
                out = json.loads(ln).get("cpu_baseline")
                if out:
                    out["process"] = "fresh process: bench.py --impl reference --steps %d" % steps
                return out
    except Exception:
        return None
    return None


def run_steps(s, start, K):
    """Steps start+1 .. start+K of the run, measuring the box averages on the
    steps main.cpp writes them; returns the kernel launches queued."""
    from coolbubble_b200 import _lib as L
    launches0, _ = s.counters()
    for k, measure in event_chunks(start, K):
        L.check(L.lib.cb_step(s._h, k, L.CB_STEP_SUMS if measure else 0, None), s._h)
    return s.counters()[0] - launches0


def timed_steps(s, start, K):
    """run_steps bracketed by CUDA events on the run's stream: (device ms, launches)."""
    from coolbubble_b200 import _lib as L
    s.sync()
    L.check(L.lib.cb_timer_start(s._h), s._h)
    launches = run_steps(s, start, K)
    ms = L.C.c_double()
    L.check(L.lib.cb_timer_stop(s._h, L.C.byref(ms)), s._h)
    return ms.value, launches


def step_kind_ms(s, reps=4):
    """Device ms of one step without and with the full box averages (single
    steps, each its own launch)."""
    from coolbubble_b200 import _lib as L
    out = {}
    for name, flags in (("plain", 0), ("sums", L.CB_STEP_SUMS)):
        s.sync()
        L.check(L.lib.cb_timer_start(s._h), s._h)
        for _ in range(reps):
            L.check(L.lib.cb_step(s._h, 1, flags, None), s._h)
        ms = L.C.c_double()
        L.check(L.lib.cb_timer_stop(s._h, L.C.byref(ms)), s._h)
        out[name] = ms.value / reps
    return out


def spectrum_ms(s, reps):
    """Device time of one power spectrum of the run's field (cb_power_spectrum:
    r2c FFT + shell binning, bubble.cpp:642-709), averaged over reps calls after
    one untimed call; each call also returns its bins to the host."""
    if reps <= 0:
        return None
    from coolbubble_b200 import _lib as L
    s.spectrum_sums()
    L.check(L.lib.cb_timer_start(s._h), s._h)
    for _ in range(reps):
        s.spectrum_sums()
    ms = L.C.c_double()
    L.check(L.lib.cb_timer_stop(s._h, L.C.byref(ms)), s._h)
    return ms.value / reps


def measure_lattice(w, prec, K, W, phi_h, pi_h, dist=None, clocks=None, spectra=0, kinds=True):
    """Device-resident throughput of one lattice in one precision: W' = padded
    warm-up steps, then K timed steps (energy lines on main.cpp's steps)."""
    import coolbubble_b200 as cb
    d, n = w["d"], w["n"]
    N = n ** d
    p = cb.make_params(d, n, w["L"], w["c"], 0.1 * w["L"] / n, expansion=w["expansion"], mpl=w["mpl"],
                       precision=prec, memorysave=1)
    s = cb.Bubble(p, phi_h, pi_h)
    Wp = padded_warmup(W, K)
    run_steps(s, 0, Wp)
    s.sync()
    if clocks is not None:
        clocks.start()
        time.sleep(0.3)
    barrier(dist)
    if clocks is not None:
        clocks.mark()
    ms, launches = timed_steps(s, Wp, K)
    if clocks is not None:
        clocks.mark()
    barrier(dist)
    ms = max_over_ranks(dist, ms)
    clk = clocks.stop() if clocks is not None else None
    final = s.sums()
    kind = step_kind_ms(s) if kinds else None
    spec = spectrum_ms(s, spectra)
    s.close()
    ws = 1 if dist is None else dist.get_world_size()
    peak, _ = measured_peak()
    per_launch = ms / launches
    # HBM passes over the lattice: a static launch is one pass (of one or two
    # steps); an expanding step is one pass, also inside a multi-step launch
    passes = K if w["expansion"] else launches
    alg = BYTES_PER_SITE[prec] * N * passes / launches
    achieved = alg / (per_launch / 1e3) / 1e9
    out = dict(value=N * K * ws / (ms / 1e3), ms=ms, ms_per_step=ms / K, launches=launches, passes=passes, warmup=Wp,
               per_launch_ms=per_launch, alg_bytes=alg, achieved_gbs=achieved, frac=achieved / peak,
               effective_gbs=N * K * BYTES_PER_SITE[prec] / (ms / 1e3) / 1e9, clocks=clk, final=final,
               spectrum_ms=spec)
    out["effective_frac"] = out["effective_gbs"] / peak
    if kind:
        out["plain_step_ms"], out["sums_step_ms"] = kind["plain"], kind["sums"]
    return out


def e2e_run(w, K, phi_h, pi_h, precision):
    """One run of K steps through the C ABI with host buffers: upload the start
    (pinned doubles), the energy line read back to the host every 40 steps,
    phi and pi downloaded (float) at the end."""
    import coolbubble_b200 as cb
    from coolbubble_b200 import _lib as L
    d, n = w["d"], w["n"]
    N = n ** d
    p = cb.make_params(d, n, w["L"], w["c"], 0.1 * w["L"] / n, expansion=w["expansion"], mpl=w["mpl"],
                       precision=precision, memorysave=1)
    out_phi, p1 = L.pinned_array(N, np.float32)
    out_pi, p2 = L.pinned_array(N, np.float32)
    try:
        t0 = time.perf_counter()
        s = cb.Bubble(p, phi_h, pi_h)
        reads = 0
        for k, measure in event_chunks(0, K):
            s.step(k, sums=True)      # every chunk ends on a line, or on the run's last step
            reads += 1
        L.check(L.lib.cb_get_fields_f32(s._h, L.fptr(out_phi), L.fptr(out_pi), None, None, None), s._h)
        el = time.perf_counter() - t0
        s.close()
    finally:
        L.lib.cb_pinned_free(p1)
        L.lib.cb_pinned_free(p2)
    h2d = 2 * N * 8
    d2h = reads * L.C.sizeof(L.cb_sums) + 2 * N * 4
    return N * K / el, h2d / K, d2h / K


def ensemble_members(count, seed):
    """The ensemble configuration: d = 2, n in {128, 256, 512} in equal thirds,
    c ~ U[1, 8], half mode 1 with 3-10 bubbles, half mode -3 with Trad ~ U[0.01, 0.1],
    dt = 0.1 dx; every member seeded."""
    rng = np.random.default_rng(seed)
    ns = ([128] * (count // 3) + [256] * (count // 3) + [512] * (count - 2 * (count // 3)))
    rng.shuffle(ns)
    specs = []
    for i, n in enumerate(ns):
        c = float(rng.uniform(1.0, 8.0))
        thermal = bool(rng.integers(0, 2))
        specs.append(dict(n=int(n), c=c, L=float(n) / 8.0, thermal=thermal,
                          nb=int(rng.integers(3, 11)), trad=float(rng.uniform(0.01, 0.1)),
                          pos_seed=int(rng.integers(1, 2 ** 31)), th_seed=int(rng.integers(1, 2 ** 62))))
    return specs


def ensemble_measure(steps, warmup, seed, dist=None):
    """The ensemble of 256 independent d = 2 lattices stepped together (FP32C) and
    the same ensemble in plain FP64: total site-updates/s over one
    cb_ensemble_step call of `steps` steps (host wall clock around it)."""
    import coolbubble_b200 as cb
    from coolbubble_b200.ensemble import Ensemble
    from coolbubble_b200.ic import initial_condition
    specs = ensemble_members(256, seed=seed)
    starts = []
    for sp in specs:
        p = cb.make_params(2, sp["n"], sp["L"], sp["c"], 0.1 * sp["L"] / sp["n"], precision="fp32c", memorysave=1)
        phi0, pi0, _ = initial_condition(p, mode=-3 if sp["thermal"] else 1, n_bubbles=sp["nb"], trad=sp["trad"],
                                         position_seed=sp["pos_seed"], thermal_seed=sp["th_seed"])
        starts.append((phi0, pi0))
    sites = sum(sp["n"] ** 2 for sp in specs)
    ws = 1 if dist is None else dist.get_world_size()
    out = {}
    for prec in ("fp32c", "fp64"):
        runs = [cb.Bubble(cb.make_params(2, sp["n"], sp["L"], sp["c"], 0.1 * sp["L"] / sp["n"], precision=prec,
                                         memorysave=1), a, b) for sp, (a, b) in zip(specs, starts)]
        ens = Ensemble(runs)
        plans = [ens.plan(i) for i in range(len(runs))]
        ens.step(warmup, 0)
        barrier(dist)
        t0 = time.perf_counter()
        ens.step(steps, OUT_ENERGY_EVERY)
        el = max_over_ranks(dist, time.perf_counter() - t0)
        out[prec] = dict(seconds=el, value=ws * sites * steps / el, plans=plans)
        del ens, runs
    resident = sum(1 for c, _ in out["fp32c"]["plans"] if c > 0)
    return {
        "value": out["fp32c"]["value"], "unit": "site-updates/s", "steps": steps,
        "ms_per_step": 1e3 * out["fp32c"]["seconds"] / steps, "members": len(specs), "sites_per_step": sites,
        "n_mix": {str(m): sum(1 for s in specs if s["n"] == m) for m in (128, 256, 512)},
        "thermal_members": sum(1 for s in specs if s["thermal"]), "resident_members_fp32c": resident,
        "fp64_value": out["fp64"]["value"], "speedup_vs_fp64": out["fp32c"]["value"] / out["fp64"]["value"],
        "hbm_equivalent_gbs": out["fp32c"]["value"] * 16 / 1e9,
        "timing": "host wall clock around one cb_ensemble_step call (launch, all steps, lines back)",
    }


def serving_requests(rate, duration, seed):
    """The serving stream: Poisson arrivals at `rate` per second for `duration`
    seconds; d in {2, 3}; n uniform in {64, 128, 192, 256, 384} (d = 3 at most
    256); c ~ U[1, 8]; nt ~ U[200, 5000]; mode 1 or -3 (seeded); expansion on
    for half of the d = 3 runs (Mpl = 10)."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t > duration:
            break
        d = int(rng.integers(2, 4))
        ns = [64, 128, 192, 256, 384] if d == 2 else [64, 128, 192, 256]
        n = int(ns[int(rng.integers(0, len(ns)))])
        out.append(dict(at=t, d=d, n=n, c=float(rng.uniform(1.0, 8.0)), nt=int(rng.integers(200, 5001)),
                        thermal=bool(rng.integers(0, 2)), expansion=int(d == 3 and rng.integers(0, 2)),
                        nb=int(rng.integers(3, 11)), trad=float(rng.uniform(0.01, 0.1)),
                        pos_seed=int(rng.integers(1, 2 ** 31)), th_seed=int(rng.integers(1, 2 ** 62))))
    return out


def serving_measure(rate, duration, slots, seed, dist=None):
    """One serving stream through the pool: aggregate site-updates/s over the
    makespan and the submit-to-finish latency percentiles."""
    import coolbubble_b200 as cb
    from coolbubble_b200.serving import Pool, ic_params, DONE
    reqs = serving_requests(rate, duration, seed=seed)
    pool = Pool(150 * 10 ** 9, slots)
    ids = []
    barrier(dist)
    t0 = time.perf_counter()
    for r in reqs:
        delay = r["at"] - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        L_box = r["n"] / 8.0
        p = cb.make_params(r["d"], r["n"], L_box, r["c"], 0.1 * L_box / r["n"], precision="fp32c", memorysave=1,
                           expansion=r["expansion"], mpl=10.0)
        ic = ic_params(mode=-3 if r["thermal"] else 1, n_bubbles=r["nb"], trad=r["trad"], position_seed=r["pos_seed"],
                       thermal_seed=r["th_seed"])
        ids.append(pool.submit(p, ic, r["nt"], sums_every=OUT_ENERGY_EVERY))
    lat, updates, states = [], 0.0, []
    for rid, r in zip(ids, reqs):
        pool.wait(rid, 3600 * 1000)
        res = pool.result(rid)
        states.append(res["state"])
        lat.append(res["latency"])
        if res["state"] == DONE:
            updates += float(r["n"] ** r["d"]) * r["nt"]
    el = time.perf_counter() - t0
    st = pool.stats()
    pool.close()
    el = max_over_ranks(dist, el)
    ws = 1 if dist is None else dist.get_world_size()
    lat = np.array(lat)
    return {
        "value": ws * updates / el, "unit": "site-updates/s", "rate_per_s": rate, "arrival_window_s": duration,
        "requests": len(reqs), "slots": slots, "budget_bytes": 150 * 10 ** 9, "precision": "fp32c",
        "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                      "max": float(lat.max()), "mean": float(lat.mean())},
        "completed": int(sum(1 for s_ in states if s_ == DONE)), "failed": int(st["failed"]),
        "makespan_s": el, "gpu_busy_s": st["busy_s"], "site_updates": updates,
    }


def lattice_summary(m, prec):
    return {"value": m["value"], "unit": "site-updates/s", "precision": prec, "ms_per_step": m["ms_per_step"],
            "steps": round(m["ms"] / m["ms_per_step"]), "warmup": m["warmup"],
            "roofline": {"bound": "hbm", "achieved": m["achieved_gbs"], "frac": m["frac"], "unit": "GB/s",
                         "alg_bytes_per_launch": m["alg_bytes"], "launch_ms": m["per_launch_ms"],
                         "passes_per_launch": m["passes"] / m["launches"]},
            "effective_frac": m["effective_frac"], "plain_step_ms": m.get("plain_step_ms"),
            "sums_step_ms": m.get("sums_step_ms"), "spectrum_ms": m.get("spectrum_ms")}


def other_workloads(args):
    """The other workloads on this GPU, one object each (one GPU only)."""
    out = {}
    # the 512^2 FP64 run with 5 bubbles: all 1000 of its steps, lines every 40
    w = WORKLOADS["bubbles-d2-n512"]
    phi0, pi0 = make_start(w)
    m64 = measure_lattice(w, "fp64", w["nt"], 3, phi0, pi0, spectra=3)
    m32 = measure_lattice(w, "fp32c", w["nt"], 3, phi0, pi0, kinds=False)
    o = lattice_summary(m64, "fp64")
    o["config"] = workload_config("bubbles-d2-n512", w)
    o["fp32c_value"] = m32["value"]
    o["l2"] = l2_note(w["n"], w["d"], "fp64")
    out["bubbles-d2-n512"] = o
    # the 256^3 expanding run with 8 bubbles: FP32C and FP64
    w = WORKLOADS["bubbles-d3-n256-expanding"]
    phi0, pi0 = make_start(w)
    K = max(args.steps, 200)
    m32 = measure_lattice(w, "fp32c", K, args.warmup, phi0, pi0, spectra=3)
    m64 = measure_lattice(w, "fp64", K, args.warmup, phi0, pi0)
    o = lattice_summary(m32, "fp32c")
    o["config"] = workload_config("bubbles-d3-n256-expanding", w)
    o["fp64"] = lattice_summary(m64, "fp64")
    o["speedup_vs_fp64"] = m32["value"] / m64["value"]
    o["l2"] = l2_note(w["n"], w["d"], "fp32c")
    out["bubbles-d3-n256-expanding"] = o
    # the ensemble of 256 d = 2 lattices, all 1500 steps
    out["ensemble-d2-256"] = ensemble_measure(1500, 3, seed=2026)
    # serving: a light stream (latency) and a saturating one (throughput)
    out["serving"] = {"light": serving_measure(10.0, 10.0, 64, seed=77),
                      "saturated": serving_measure(50.0, 6.0, 64, seed=78)}
    return out


def l2_note(n, d, prec):
    fields = 2 * n ** d * (4 if prec == "fp32c" else 8)
    if fields > 126 * 2 ** 20:
        return "inputs larger than L2 (2 x %d^%d %s = %.2f GiB)" % (n, d, "floats" if prec == "fp32c" else "doubles",
                                                                      fields / 2 ** 30)
    return "inputs smaller than L2 (%.0f MiB): L2-resident" % (fields / 2 ** 20)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="thermal-d3-n512",
                    choices=sorted(WORKLOADS) + ["ensemble-d2-256", "serving"])
    ap.add_argument("--rate", type=float, default=10.0, help="serving: arrivals per second")
    ap.add_argument("--duration", type=float, default=20.0, help="serving: arrival window in seconds")
    ap.add_argument("--slots", type=int, default=64, help="serving: runs on the GPU at once")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="only the headline workload")
    ap.add_argument("--quick", action="store_true", help="device-resident timing only (profiling runs)")
    ap.add_argument("--e2e-steps", type=int, default=0,
                    help="steps of the end-to-end run (default: the workload's full run length nt)")
    ap.add_argument("--spectra", type=int, default=5,
                    help="power spectra timed after the steps (per-snapshot cost; 0: none)")
    args = ap.parse_args()
    if args.workload in ("serving", "ensemble-d2-256"):
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the %s workload has no reference arm: the "
                              "reference runs one lattice per process" % args.workload}))
            return 0
        ws, rank, local = dist_env()
        dist = init_dist(ws)
        from coolbubble_b200 import _lib as L
        L.check(L.lib.cb_set_device(local))
        if args.workload == "serving":
            r = serving_measure(args.rate, args.duration, args.slots, seed=77 + rank, dist=dist)
        else:
            r = ensemble_measure(args.steps, args.warmup, seed=2026 + rank, dist=dist)
        line = {"metric": "lattice site-updates/s", "value": r.pop("value"), "unit": "site-updates/s",
                "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": args.workload}, **r}
        if rank == 0:
            print(json.dumps(line), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return 0
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        return run_reference_arm(args, w, args.workload)
    args.warmup = max(3, args.warmup)

    ws, rank, local = dist_env()
    dist = init_dist(ws)
    from coolbubble_b200 import _lib as L
    L.check(L.lib.cb_set_device(local))

    d, n = w["d"], w["n"]
    N = n ** d
    prec = w["precision"]
    phi0, pi0 = make_start(w, rank)
    phi_h, pi_h = L.pinned_array(N, np.float64), L.pinned_array(N, np.float64)
    phi_h[0][:] = phi0
    pi_h[0][:] = pi0
    del phi0, pi0

    # ---- device-resident throughput of the workload's path ------------------
    clocks = ClockSampler(local)
    m = measure_lattice(w, prec, args.steps, args.warmup, phi_h[0], pi_h[0], dist=dist, clocks=clocks,
                        spectra=args.spectra, kinds=not args.quick)
    value = m["value"]
    if args.quick:
        if rank == 0:
            print(json.dumps({"metric": "lattice site-updates/s", "value": value, "unit": "site-updates/s",
                              "ms_per_step": m["ms_per_step"], "config": {"workload": args.workload},
                              "spectrum_ms": m["spectrum_ms"], "quick": True}), flush=True)
        return 0

    # ---- plain FP64 path on the same lattice ----------------------------------
    m64 = None
    if prec != "fp64":
        m64 = measure_lattice(w, "fp64", min(args.steps, 200), 3, phi_h[0], pi_h[0], dist=dist)

    # ---- end to end through the C ABI with host buffers -----------------------
    K_e2e = args.e2e_steps or w["nt"]
    barrier(dist)
    e2e_val, h2d, d2h = e2e_run(w, K_e2e, phi_h[0], pi_h[0], prec)
    e2e_val = ws * N * K_e2e / max_over_ranks(dist, N * K_e2e / e2e_val)

    peak, peak_kind = measured_peak()
    line = {
        "metric": "lattice site-updates/s", "value": value, "unit": "site-updates/s", "n_gpus": ws,
        "steps": args.steps, "warmup": m["warmup"], "ms_per_step": m["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32" if prec == "fp32c" else "f64", "data": "synthetic",
        "config": workload_config(args.workload, w),
        "details": {"precision": prec, "parallelism": f"replicas{ws}", "l2": l2_note(n, d, prec),
                    "steps_per_launch": args.steps / m["launches"],
                    "temporal_block": os.environ.get("CB_TEMPORAL_BLOCK", "autotuned"),
                    "warmup_requested": args.warmup,
                    "energy_lines_in_window": sum(1 for _, e in event_chunks(m["warmup"], args.steps) if e)},
        "hbm_gbs": m["achieved_gbs"],
        # site-updates/s x the bytes a one-step pass moves per site-update: above the
        # DRAM rate when two-step passes move those bytes once per two steps
        "effective_gbs": m["effective_gbs"] / ws, "effective_frac": m["effective_frac"] / ws,
        "roofline": {"bound": "hbm", "achieved": m["achieved_gbs"], "peak": peak, "unit": "GB/s",
                     "frac": m["frac"], "traffic": committed_traffic(args.workload, prec), "peak_source": peak_kind,
                     "alg_bytes_per_launch": m["alg_bytes"], "launch_ms": m["per_launch_ms"]},
        "plain_step_ms": m.get("plain_step_ms"), "sums_step_ms": m.get("sums_step_ms"),
        "e2e": {"value": e2e_val, "unit": "site-updates/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": K_e2e,
                "run": "one run of the workload's %d steps through the C ABI: start uploaded from pinned host "
                       "doubles, set-up kernels, energy line read back every 40 steps, phi and pi downloaded "
                       "as float at the end" % K_e2e},
        "gpu_launches": m["launches"],
        "clocks": m["clocks"],
        "final_etot": m["final"]["etot"],
        # per snapshot, outside the timed steps: one power spectrum of the final field
        "spectrum_ms": m["spectrum_ms"],
    }
    if m64 is not None:
        line["fp64_value"] = m64["value"]
        line["fp64_ms_per_step"] = m64["ms_per_step"]
        line["speedup_vs_fp64"] = value / m64["value"]
        line["roofline"]["fp64_frac"] = m64["frac"]
    L.lib.cb_pinned_free(phi_h[1])
    L.lib.cb_pinned_free(pi_h[1])
    if ws == 1 and not args.no_extras:
        line["configs"] = other_workloads(args)
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cb_line = cpu_baseline_subprocess(args.workload)
        if cb_line:
            line["cpu_baseline"] = cb_line
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
