"""Benchmark of the lattice-evolution path (one JSON line on rank 0).

Workload (default): the d = 3, N = 512, L = 64, c = 2 static lattice with a
thermal-like start (dt = 0.1 dx), evolved in the FP32-compensated path; the
plain FP64 path is timed on the same lattice for the "vs plain FP64" figure.
A "step" is one leapfrog step over the whole lattice (one fused kernel
launch); box averages are measured every 40 steps as the reference's main
loop does (OutEnergyEvery, def.h:65).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Timing: device time from CUDA events on the run's own stream, after W
warm-up steps, barrier and synchronisation on both sides; max over ranks.
The 2 x 512^3 float fields (1 GiB) exceed the 126 MB L2, so no flush is
needed between steps. Multi-GPU: every rank evolves its own lattice
(independent runs, no collective on the data path: weak scaling).
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
    # the headline: a 512^3 static lattice, c = 2, thermal-like start (HBM-resident stencil)
    "thermal-d3-n512": dict(d=3, n=512, L=64.0, c=2.0, expansion=0, mpl=200.0, precision="fp32c"),
    # the same stencil at 256^3 (2 x 64 MiB fields), for profiler captures
    "thermal-d3-n256": dict(d=3, n=256, L=32.0, c=2.0, expansion=0, mpl=200.0, precision="fp32c"),
    # a 256^3 lattice with bubbles and the self-consistent expanding background
    "bubbles-d3-n256-expanding": dict(d=3, n=256, L=32.0, c=4.0, expansion=1, mpl=10.0, precision="fp32c"),
    # a large 2-D lattice (column-strip kernel), for profiler captures
    "plain-d2-n8192": dict(d=2, n=8192, L=1024.0, c=4.0, expansion=0, mpl=200.0, precision="fp32c"),
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


def thermal_like_ic(n, d, seed):
    """Seeded Gaussian fluctuations around the false vacuum (phi = 0).

    Stands in for the reference's mode -3 start (bubble.cpp:459-523); the
    step kernel's cost does not depend on the values."""
    rng = np.random.default_rng(seed)
    N = n ** d
    phi = rng.standard_normal(N, dtype=np.float32).astype(np.float64) * 0.05
    pi = rng.standard_normal(N, dtype=np.float32).astype(np.float64) * 0.05
    return phi, pi


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


def cpu_sample(w, phi0, pi0, max_steps, budget_s):
    with quiet_stdout():
        return _cpu_sample(w, phi0, pi0, max_steps, budget_s)


def _cpu_sample(w, phi0, pi0, max_steps, budget_s):
    """Time the reference's own CPU step (oracle/_ref, built from the reference
    sources) on this host's cores, else the CPU restatement; bounded by
    max_steps and budget_s. Returns (site-updates/s, kind, cores, sample)."""
    from oracle import bridge as B
    cores = cpu_threads()
    os.environ["OMP_NUM_THREADS"] = str(cores)
    d, n, L, c = w["d"], w["n"], w["L"], w["c"]
    dt = 0.1 * L / n
    N = n ** d
    t_setup = time.perf_counter()
    if os.path.exists(B.REF_SO):
        kind = "reference"
        # mode -2 (one centred bubble): the same per-step work without the FFT start-up
        obj = B.Reference(d, n, L, c, -2, dt, expansion=w["expansion"], mpl=w["mpl"])
        what = "reference Bubble::oneStep (src/bubble.cpp:849-876, FP64, OpenMP)"
    else:
        kind = "port"
        B.set_threads(cores)
        obj = B.Oracle(d, n, L, c, dt, phi0, pi0, expansion=w["expansion"], mpl=w["mpl"])
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
    sample = f"{steps} step(s) of the full {n}^{d} lattice: {what}; {cores} threads; set-up {setup:.1f} s untimed"
    return N * steps / el, kind, cores, sample


def run_reference_arm(args, w, wname):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    d, n = w["d"], w["n"]
    phi0 = pi0 = None
    from oracle import bridge as B
    if not os.path.exists(B.REF_SO):
        phi0, pi0 = thermal_like_ic(n, d, seed=1)
    value, kind, cores, sample = cpu_sample(w, phi0, pi0, max_steps=max(1, args.steps), budget_s=120.0)
    line = {
        "impl": "reference", "metric": "lattice site-updates/s", "value": value, "unit": "site-updates/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wname, "d": d, "n": n, "L": w["L"], "c": w["c"], "expansion": w["expansion"]},
        "cpu_baseline": {"value": value, "unit": "site-updates/s", "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": "site-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def timed_steps(s, K):
    """K steps with the box averages measured every OUT_ENERGY_EVERY steps;
    returns (device ms, kernel launches queued)."""
    from coolbubble_b200 import _lib as L
    s.sync()
    launches0, _ = s.counters()
    L.check(L.lib.cb_timer_start(s._h), s._h)
    done = 0
    while done < K:
        k = min(OUT_ENERGY_EVERY, K - done)
        flags = L.CB_STEP_SUMS if (done + k) % OUT_ENERGY_EVERY == 0 else 0
        L.check(L.lib.cb_step(s._h, k, flags, None), s._h)
        done += k
    ms = L.C.c_double()
    L.check(L.lib.cb_timer_stop(s._h, L.C.byref(ms)), s._h)
    return ms.value, s.counters()[0] - launches0


def e2e_run(w, K, phi_h, pi_h, precision):
    """One run through the C ABI with host buffers: upload the start (pinned),
    K steps with a sums read-back every 40 steps, download phi and pi (float)."""
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
        done, reads = 0, 0
        while done < K:
            k = min(OUT_ENERGY_EVERY, K - done)
            s.step(k, sums=True)
            reads += 1
            done += k
        L.check(L.lib.cb_get_fields_f32(s._h, L.fptr(out_phi), L.fptr(out_pi), None, None, None), s._h)
        el = time.perf_counter() - t0
        s.close()
    finally:
        L.lib.cb_pinned_free(p1)
        L.lib.cb_pinned_free(p2)
    h2d = 2 * N * 8
    d2h = reads * 144 + 2 * N * 4
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


def run_ensemble_bench(args):
    """The ensemble: 256 independent d = 2 lattices stepped together (FP32C), and the
    same ensemble in plain FP64; value = total site-updates/s of the ensemble."""
    import coolbubble_b200 as cb
    from coolbubble_b200 import _lib as L
    from coolbubble_b200.ensemble import Ensemble
    from coolbubble_b200.ic import initial_condition
    ws, rank, local = dist_env()
    dist = init_dist(ws)
    L.check(L.lib.cb_set_device(local))
    specs = ensemble_members(256, seed=2026 + rank)
    starts = []
    for sp in specs:
        p = cb.make_params(2, sp["n"], sp["L"], sp["c"], 0.1 * sp["L"] / sp["n"], precision="fp32c", memorysave=1)
        phi0, pi0, _ = initial_condition(p, mode=-3 if sp["thermal"] else 1, n_bubbles=sp["nb"], trad=sp["trad"],
                                         position_seed=sp["pos_seed"], thermal_seed=sp["th_seed"])
        starts.append((phi0, pi0))
    sites = sum(sp["n"] ** 2 for sp in specs)
    out = {}
    for prec in ("fp32c", "fp64"):
        runs = [cb.Bubble(cb.make_params(2, sp["n"], sp["L"], sp["c"], 0.1 * sp["L"] / sp["n"], precision=prec,
                                         memorysave=1), a, b) for sp, (a, b) in zip(specs, starts)]
        ens = Ensemble(runs)
        plans = [ens.plan(i) for i in range(len(runs))]
        ens.step(args.warmup, 0)
        barrier(dist)
        t0 = time.perf_counter()
        lines = ens.step(args.steps, OUT_ENERGY_EVERY)
        el = max_over_ranks(dist, time.perf_counter() - t0)
        out[prec] = dict(seconds=el, value=ws * sites * args.steps / el, plans=plans, lines=lines)
        del ens, runs
    resident = sum(1 for c, _ in out["fp32c"]["plans"] if c > 0)
    line = {
        "metric": "lattice site-updates/s", "value": out["fp32c"]["value"], "unit": "site-updates/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * out["fp32c"]["seconds"] / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "ensemble-d2-256", "members": len(specs), "sites_per_step": sites,
                   "n_mix": {"128": sum(1 for s in specs if s["n"] == 128), "256": sum(1 for s in specs if s["n"] == 256),
                             "512": sum(1 for s in specs if s["n"] == 512)},
                   "thermal_members": sum(1 for s in specs if s["thermal"]), "sums_every": OUT_ENERGY_EVERY,
                   "resident_members_fp32c": resident,
                   "timing": "host wall clock around one cb_ensemble_step call (launch, all steps, records back)"},
        "fp64_value": out["fp64"]["value"], "speedup_vs_fp64": out["fp32c"]["value"] / out["fp64"]["value"],
        "hbm_equivalent_gbs": out["fp32c"]["value"] * 16 / 1e9,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


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


def run_serving_bench(args):
    import coolbubble_b200 as cb
    from coolbubble_b200 import _lib as L
    from coolbubble_b200.serving import Pool, ic_params, DONE
    ws, rank, local = dist_env()
    dist = init_dist(ws)
    L.check(L.lib.cb_set_device(local))
    reqs = serving_requests(args.rate, args.duration, seed=77 + rank)
    pool = Pool(150 * 10 ** 9, args.slots)
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
    lat = np.array(lat)
    line = {
        "metric": "lattice site-updates/s", "value": ws * updates / el, "unit": "site-updates/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "serving", "rate_per_s": args.rate, "arrival_window_s": args.duration,
                   "requests": len(reqs), "slots": args.slots, "budget_bytes": 150 * 10 ** 9,
                   "precision": "fp32c", "sums_every": OUT_ENERGY_EVERY},
        "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                      "max": float(lat.max()), "mean": float(lat.mean())},
        "completed": int(sum(1 for s_ in states if s_ == DONE)), "failed": int(st["failed"]),
        "makespan_s": el, "gpu_busy_s": st["busy_s"],
        "site_updates": updates,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def l2_note(n, d, prec):
    fields = 2 * n ** d * (4 if prec == "fp32c" else 8)
    if fields > 126 * 2 ** 20:
        return "inputs larger than L2 (2 x %d^%d %s = %.2f GiB)" % (n, d, "floats" if prec == "fp32c" else "doubles",
                                                                      fields / 2 ** 30)
    return "inputs smaller than L2 (%.0f MiB): L2-resident" % (fields / 2 ** 20)


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
    ap.add_argument("--quick", action="store_true", help="device-resident timing only (profiling runs)")
    ap.add_argument("--spectra", type=int, default=5,
                    help="power spectra timed after the steps (per-snapshot cost; 0: none)")
    args = ap.parse_args()
    if args.workload == "serving":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the serving workload has no reference arm: "
                              "the reference runs one lattice per process"}))
            return 0
        return run_serving_bench(args)
    if args.workload == "ensemble-d2-256":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the ensemble workload has no reference arm: "
                              "the reference runs one lattice per process"}))
            return 0
        return run_ensemble_bench(args)
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        return run_reference_arm(args, w, args.workload)
    args.warmup = max(3, args.warmup)

    ws, rank, local = dist_env()
    dist = init_dist(ws)
    import coolbubble_b200 as cb
    from coolbubble_b200 import _lib as L
    L.check(L.lib.cb_set_device(local))

    d, n = w["d"], w["n"]
    N = n ** d
    dt = 0.1 * w["L"] / n
    prec = w["precision"]
    phi_h, pi_h = L.pinned_array(N, np.float64), L.pinned_array(N, np.float64)
    phi0, pi0 = thermal_like_ic(n, d, seed=1 + rank)
    phi_h[0][:] = phi0
    pi_h[0][:] = pi0

    # ---- device-resident throughput of the FP32C path --------------------------
    p = cb.make_params(d, n, w["L"], w["c"], dt, expansion=w["expansion"], mpl=w["mpl"], precision=prec,
                       memorysave=1)
    s = cb.Bubble(p, phi_h[0], pi_h[0])
    s.step(args.warmup, sums=True)
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    barrier(dist)
    clocks.mark()
    ms, launches = timed_steps(s, args.steps)
    clocks.mark()
    barrier(dist)
    ms = max_over_ranks(dist, ms)
    clk = clocks.stop()
    final = s.sums()
    spec_ms = spectrum_ms(s, args.spectra)
    s.close()
    value = N * args.steps * ws / (ms / 1e3)

    if args.quick:
        if rank == 0:
            print(json.dumps({"metric": "lattice site-updates/s", "value": value, "unit": "site-updates/s",
                              "ms_per_step": ms / args.steps, "config": {"workload": args.workload},
                              "spectrum_ms": spec_ms, "quick": True}), flush=True)
        return 0

    # ---- plain FP64 path on the same lattice ----------------------------------
    p64 = cb.make_params(d, n, w["L"], w["c"], dt, expansion=w["expansion"], mpl=w["mpl"], precision="fp64",
                         memorysave=1)
    s64 = cb.Bubble(p64, phi_h[0], pi_h[0])
    s64.step(3, sums=True)
    k64 = min(args.steps, 200)
    barrier(dist)
    ms64 = max_over_ranks(dist, timed_steps(s64, k64)[0])
    s64.close()
    value64 = N * k64 * ws / (ms64 / 1e3)

    # ---- end to end through the C ABI with host buffers -----------------------
    barrier(dist)
    e2e_val, h2d, d2h = e2e_run(w, args.steps, phi_h[0], pi_h[0], prec)
    e2e_val = ws * N * args.steps / max_over_ranks(dist, N * args.steps / e2e_val)

    peak, peak_kind = measured_peak()
    per_launch_ms = ms / launches
    # every launch (one step, or a two-step pass) reads phi and pi once and writes them once
    alg_bytes = BYTES_PER_SITE[prec] * N
    achieved = alg_bytes / (per_launch_ms / 1e3) / 1e9
    line = {
        "metric": "lattice site-updates/s", "value": value, "unit": "site-updates/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "d": d, "n": n, "L": w["L"], "c": w["c"], "dt": dt,
                   "expansion": w["expansion"], "precision": prec, "parallelism": f"replicas{ws}",
                   "l2": l2_note(n, d, prec),
                   "sums_every": OUT_ENERGY_EVERY, "ic": "seeded gaussian fluctuations, amplitude 0.05",
                   "steps_per_launch": args.steps / launches,
                   "temporal_block": os.environ.get("CB_TEMPORAL_BLOCK", "autotuned")},
        "fp64_value": value64, "fp64_ms_per_step": ms64 / k64, "speedup_vs_fp64": value / value64,
        "hbm_gbs": achieved,
        # site-updates/s x the 16 B a one-step pass moves per site-update: above the
        # DRAM rate when two-step passes move those bytes once per two steps
        "effective_gbs": value * BYTES_PER_SITE[prec] / 1e9 / ws,
        "effective_frac": value * BYTES_PER_SITE[prec] / 1e9 / ws / peak,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": committed_traffic(args.workload, prec), "peak_source": peak_kind,
                     "alg_bytes_per_launch": alg_bytes, "launch_ms": per_launch_ms,
                     "fp64_frac": (BYTES_PER_SITE["fp64"] * N / (ms64 / k64 / 1e3) / 1e9) / peak},
        "e2e": {"value": e2e_val, "unit": "site-updates/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "clocks": clk,
        "final_etot": final["etot"],
        # per snapshot, outside the timed steps: one power spectrum of the final field
        "spectrum_ms": spec_ms,
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        v, kind, cores, sample = cpu_sample(w, phi0, pi0, max_steps=20, budget_s=20.0)
        line["cpu_baseline"] = {"value": v, "unit": "site-updates/s", "cores": cores, "kind": kind,
                                "sample": sample}
    L.lib.cb_pinned_free(phi_h[1])
    L.lib.cb_pinned_free(pi_h[1])
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
