#!/usr/bin/env python3
"""Benchmark of the B200 Barnes-Hut hot path (one JSON line on rank 0).

Default workload (plummer-4m): one Plummer sphere, N = 4,194,304
(seed 2, G = M = a = 1), theta 0.5, eps 0.005, monopole + quadrupole,
max_leaf 16, target 16, group 256, advanced by the reference's leapfrog
schedule for 8 KDK steps of dt = 1/256 (main.cc:199-246: 9 force
evaluations).  One bench step = that whole 8-step sequence over the
GPU-resident particles; metric particle-steps/s = N * 8 * steps / time.

Other workloads (--workload):
  plummer-65k   N = 65,536, seed 1, eps 0.01, dt 1/128, 16 steps
  merger-16m    two Plummer spheres of 8,388,608 (a = 1 and 0.5,
                centres x = -5 / +5, approaching at 0.3), theta 0.6,
                eps 0.002, dt 1/256, 8 steps
  ensemble-512  512 independent Plummer systems, N log-uniform in
                [1,024, 262,144] (seed 3), eps 0.01, dt 1/128; one bench step
                = one lockstep KDK evaluation of every system, batched in one
                segmented key space, split precision, leaf/target sizes from
                the autotuner; also times the plain FP64 path looping over
                the systems one at a time (the batched-vs-plain comparison)
  serve-200rps  Poisson arrivals at 200 requests/s for 60 s, each
                a Plummer sphere or a merger (50/50), N log-uniform in
                [4,096, 2,097,152], 16-256 steps, theta from {0.4, 0.5, 0.7},
                eps 0.01, dt 1/128, generated on the device from a
                per-request seed and served by continuous batching under a
                150 GB HBM admission budget; reports p50/p99 per-step latency
                and aggregate particle-steps/s over a bounded wall window
                (120 s; --steps/--warmup do not apply)
  csv-4m        particle text ingest (read_csv on the GPU): the 4M Plummer
                sphere of plummer-4m as CSV (%.17g numbers, 639 MB); one step =
                one bhg_upload_csv_device of the text resident in HBM; metric
                particles/s (e2e: bhg_upload_csv from pinned host memory);
                CPU baseline: the reference's own read_csv (all host threads)
  plummer-1m    plummer-4m at N = 1,048,576, one KDK step, for profiler captures

--impl reference times the reference's own CPU implementation of the path
(oracle/_ref/ref_bench: the unmodified reference sources with a thread-pool
stand-in for TTG) on all host cores, on the same workload and metric.

Multi-GPU: one process per GPU, each an independent replica of the workload
(a system never spans GPUs; no collective on the data path); value =
particle-steps of all ranks / max over ranks of the device time.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "amt-bh-benchmark_b200"))

WORKLOADS = {
    "plummer-4m": dict(kind="single", n=4194304, seed=2, theta=0.5, eps=0.005, max_leaf=16, target=16, group=256,
                       dt=1.0 / 256, steps=8),
    "plummer-65k": dict(kind="single", n=65536, seed=1, theta=0.5, eps=0.01, max_leaf=16, target=16, group=256,
                        dt=1.0 / 128, steps=16),
    "plummer-1m": dict(kind="single", n=1048576, seed=2, theta=0.5, eps=0.005, max_leaf=16, target=16, group=256,
                       dt=1.0 / 256, steps=1),
    "merger-16m": dict(kind="merger", n=2 * 8388608, seed=4, theta=0.6, eps=0.002, max_leaf=16, target=16,
                       group=256, dt=1.0 / 256, steps=8),
    "ensemble-512": dict(kind="ensemble", nsys=512, seed=3, theta=0.5, eps=0.01, max_leaf=16, target=16, group=256,
                         dt=1.0 / 128, steps=32),
    "csv-4m": dict(kind="csv", n=4194304, seed=2),
    "serve-200rps": dict(kind="serve", rate=200.0, duration=60.0, seed=5, nmin=4096, nmax=2097152, smin=16,
                         smax=256, thetas=(0.4, 0.5, 0.7), eps=0.01, dt=1.0 / 128, max_leaf=16, target=16,
                         group=256, hbm_budget_gb=150.0, wall_limit_s=120.0),
}
METRIC = "particle-steps/s"
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
SORT_BYTES_PER_PASS = 24  # read + write of an 8-byte key and a 4-byte index
FLOPS_PP, FLOPS_PC = 20, 60


def TUNE_CANDIDATES():
    """The autotuner's search space: leaf (= target) size x walk-group cap."""
    from bhg import autotune

    return autotune.candidates(leaves=(16, 24, 32, 48), walk_groups=(32, 64))


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="bhg", choices=["bhg", "reference"])
    ap.add_argument("--workload", default="plummer-4m", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="split", choices=["split", "fp64"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="ensemble: skip the one-at-a-time FP64 path")
    ap.add_argument("--walk-group", type=int, default=0,
                    help="single systems: walk-group particle cap (0 = the library's default)")
    ap.add_argument("--no-gates", action="store_true",
                    help="plummer-4m: skip the ensemble and serving gates run after the main measurement")
    ap.add_argument("--serve-budget-gb", type=float, default=None, help="serve: HBM admission budget")
    ap.add_argument("--serve-wall", type=float, default=None, help="serve: wall-clock window in seconds")
    ap.add_argument("--serve-duration", type=float, default=None, help="serve: length of the arrival stream")
    ap.add_argument("--pipe-parts", type=int, default=8, help="ensemble e2e: contexts of the pipelined step")
    ap.add_argument("--serve-max-batch", type=int, default=None,
                    help="serve: also cap the particles one tick evaluates (latency-bounded batching)")
    return ap.parse_args()


def make_particles(w, rank=0):
    import bhg

    from bhg.replicas import replica_seed

    seed = replica_seed(w["seed"], rank)
    if w["kind"] == "single":
        return bhg.plummer(w["n"], seed)[0]
    if w["kind"] == "merger":
        return bhg.merger(w["n"] // 2, seed)
    return bhg.ensemble(w["nsys"], seed)


# ---------------------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = max(smax, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------- workload description

L2_NOTE = "inputs larger than L2 (particle state, Morton copy and tree exceed 126 MB)"


def workload_particles(w):
    """Total particles of a workload (numpy only: loads nothing of the GPU library)."""
    if w["kind"] in ("single", "csv", "merger"):
        return int(w["n"])
    if w["kind"] == "ensemble":
        import bhg

        return int(np.sum(bhg.ensemble_specs(w["nsys"], w["seed"])[0]))
    return None


def workload_config(name, w, world):
    """The `config` object of both arms' JSON lines (one function, so the two
    lines describe the workload identically)."""
    cfg = {"workload": name, **{k: (list(v) if isinstance(v, tuple) else v) for k, v in w.items() if k != "kind"}}
    cfg["n_particles"] = workload_particles(w)
    cfg["parallelism"] = f"replicas x{world}"
    cfg["l2"] = L2_NOTE
    return cfg


def workload_spheres(w, n=None):
    """The workload's initial conditions as generator spheres (same sampling as
    bhg.plummer / bhg.merger): a list of dicts n, a, mass, centre, bulk."""
    n = n or w["n"]
    if w["kind"] == "merger":
        return [dict(n=n // 2, a=1.0, mass=1.0, centre=(-5.0, 0.0, 0.0), bulk=(0.15, 0.0, 0.0)),
                dict(n=n // 2, a=0.5, mass=1.0, centre=(5.0, 0.0, 0.0), bulk=(-0.15, 0.0, 0.0))]
    return [dict(n=n, a=1.0, mass=1.0)]


# ---------------------------------------------------------------------------- CPU reference

def ref_binary():
    d = os.path.join(ROOT, "oracle", "_ref")
    flags = open("/proc/cpuinfo").read() if os.path.exists("/proc/cpuinfo") else ""
    native = os.path.join(d, "ref_bench")
    v3 = os.path.join(d, "ref_bench_v3")
    # ref_bench is the AVX-512 (x86-64-v4) build; hosts without AVX-512 get
    # the AVX2 (x86-64-v3) one
    if "avx512f" in flags and os.path.exists(native):
        return native
    return v3 if os.path.exists(v3) else None


def run_ref(spheres, seed, w, warmup_evals=0, timed_evals=None, leaf=None, theta=None):
    """The reference's schedule (oracle/_ref/ref_bench, its own process) on
    Plummer spheres it generates from `seed`: `warmup_evals` untimed
    evaluations, then `timed_evals` timed ones (default: one whole schedule),
    schedules back to back.  Returns (timed eval ms list, threads)."""
    exe = ref_binary()
    if exe is None:
        raise FileNotFoundError("oracle/_ref/ref_bench is not built")
    leaf = leaf or w["max_leaf"]
    cmd = [exe, "--seed", str(int(seed))]
    for sp in spheres:
        c, b = sp.get("centre", (0.0, 0.0, 0.0)), sp.get("bulk", (0.0, 0.0, 0.0))
        cmd += ["--sphere", ",".join(repr(float(x)) for x in (sp["n"], sp.get("a", 1.0), sp.get("mass", 1.0), *c, *b))]
    cmd += ["--steps", str(w["steps"]), "--dt", repr(w["dt"]), "--theta", repr(theta if theta is not None else w["theta"]),
            "--eps", repr(w["eps"]), "--max-leaf", str(leaf),
            "--target-size", str(w["target"] if leaf == w["max_leaf"] else leaf), "--group-size", str(w["group"]),
            "--warmup-evals", str(warmup_evals), "--timed-evals", str(timed_evals if timed_evals else w["steps"] + 1)]
    out = subprocess.run(cmd, check=True, capture_output=True, text=True).stdout
    rec = json.loads(out.strip().splitlines()[-1])
    return rec["eval_ms"], rec["threads"]


def ref_sample_n(w, evals, budget_s):
    """The largest system (the full one, else a power of two of the same kind
    and parameters) whose `evals` reference evaluations fit about budget_s,
    from a timed probe at 65,536 particles (the cost per particle grows
    slowly with N)."""
    n_probe = min(w["n"], 65536)
    ms, _ = run_ref(workload_spheres(w, n_probe), w["seed"], w, 1, 1)
    per = ms[-1] / n_probe / 1000.0  # s per particle per evaluation
    if per * w["n"] * 1.25 * evals <= budget_s:
        return w["n"]
    n = n_probe
    while n * 2 < w["n"] and per * 1.1 * (n * 2) * 1.25 * evals <= budget_s:
        n *= 2
        per *= 1.1
    return n


def cpu_rate(n, eval_ms, w):
    """particle-steps/s of the schedule (steps advances per steps+1 evaluations)."""
    t = float(np.mean(eval_ms)) / 1000.0
    return n * w["steps"] / ((w["steps"] + 1) * t)


def cpu_ensemble_sample(w, budget_particles=600000):
    """The reference on a seeded random subset of the ensemble's systems (one
    evaluation each after one untimed): rate = sum N / sum eval time."""
    import bhg

    ns, seeds = bhg.ensemble_specs(w["nsys"], w["seed"])
    order = np.random.default_rng(99).permutation(len(ns))
    n_tot, t_tot, used, threads = 0, 0.0, 0, None
    for s in order:
        ms, threads = run_ref([dict(n=int(ns[s]), a=1.0, mass=1.0)], int(seeds[s]), w, 1, 1)
        n_tot += int(ns[s])
        t_tot += ms[-1] / 1000.0
        used += 1
        if n_tot >= budget_particles:
            break
    sample = (f"{used} of {len(ns)} systems ({n_tot} particles), one timed (dt, dt) evaluation each after "
              f"one untimed, through bh::step_particles; rate = sum N / sum eval time")
    return n_tot / t_tot, threads, sample


def serve_stream(w):
    from bhg import serve

    return serve.poisson_stream(w["rate"], w["duration"], w["seed"], w["nmin"], w["nmax"], w["smin"], w["smax"],
                                w["thetas"])


def cpu_serve_sample(w, budget_particles=600000):
    """The reference on the stream's first requests, one at a time (it serves
    one simulation per process): one timed (dt, dt) evaluation per request
    after one untimed, at the request's own theta, its initial conditions
    drawn by the host generator from the request's seed (the distribution of
    the device generator).  Returns (rate, threads, sample)."""
    n_tot, t_tot, used, threads = 0, 0.0, 0, None
    for r in serve_stream(w):
        if n_tot + r.n > budget_particles:
            continue
        ms, threads = run_ref(r.spheres(), r.seed % (1 << 63), dict(w, steps=r.steps), 1, 1, theta=r.theta)
        n_tot += r.n
        t_tot += ms[-1] / 1000.0
        used += 1
        if n_tot >= budget_particles * 0.9:
            break
    sample = (f"the stream's first {used} requests that fit {budget_particles} particles ({n_tot} particles), "
              f"one at a time through bh::step_particles, one timed (dt, dt) evaluation each after one untimed; "
              f"rate = sum N / sum eval time")
    return n_tot / t_tot, threads, sample


def cpu_csv_sample(w):
    """The reference's read_csv (mmap + one thread per usable CPU) on the
    workload's CSV text, after one untimed read: (particles/s, threads, sample)."""
    import ctypes

    import bhg

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Reference

    parts, _ = bhg.plummer(w["n"], w["seed"])
    ref = Reference()
    with tempfile.NamedTemporaryFile(suffix=".csv", delete=False) as f:
        path = f.name
    try:
        bhg.write_csv(path, parts)
        buf = np.zeros(w["n"] + 1, bhg.PARTICLE)
        cnt = ctypes.c_size_t()
        err = ctypes.create_string_buffer(256)
        ref.lib.bhref_read_csv(path.encode(), buf.ctypes.data, len(buf), ctypes.byref(cnt), err, 256)
        t0 = time.perf_counter()
        ref.lib.bhref_read_csv(path.encode(), buf.ctypes.data, len(buf), ctypes.byref(cnt), err, 256)
        dt = time.perf_counter() - t0
        nb = os.path.getsize(path)
    finally:
        os.unlink(path)
    return w["n"] / dt, os.cpu_count(), f"the full text ({nb} bytes) through read_csv, after one untimed read"


def reference_arm(args, w):
    """The reference's own CPU implementation of the path (oracle/_ref/ref_bench:
    its unmodified sources, all host cores) on the same workload, metric and
    config.  Single systems: one bench step = one force evaluation of the
    workload's leapfrog schedule (schedules run back to back), --warmup
    untimed evaluations, then exactly --steps timed ones, on the full system
    when that fits a few minutes (else the largest power-of-two system of the
    same kind); value = N * steps / ((steps + 1) * mean evaluation time), the
    particle-steps/s of whole schedules.  The process loads nothing of the GPU
    library: ref_bench draws the initial conditions itself (same generator)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    unit = "particle-steps/s" if w["kind"] != "csv" else "particles/s"
    step_note = None
    steps_done, warm_done = args.steps, args.warmup
    if w["kind"] == "csv":
        value, threads, sample = cpu_csv_sample(w)
        ms_step = w["n"] / value * 1000.0
    elif w["kind"] == "serve":
        value, threads, sample = cpu_serve_sample(w)
        ms_step = None
    elif w["kind"] == "ensemble":
        value, threads, sample = cpu_ensemble_sample(w)
        ms_step = workload_particles(w) / value * 1000.0
    else:
        n = ref_sample_n(w, args.warmup + args.steps, budget_s=150.0)
        ms, threads = run_ref(workload_spheres(w, n), w["seed"], w, args.warmup, args.steps)
        value = cpu_rate(n, ms, w)
        ms_step = float(np.mean(ms))
        step_note = (f"one bench step = one force evaluation of the {w['steps']}-step schedule "
                     f"({w['steps'] + 1} evaluations per schedule, run back to back); "
                     f"ms per schedule = {ms_step * (w['steps'] + 1):.1f}")
        sample = (f"{'full system' if n == w['n'] else f'N={n}, same generator and parameters'}: "
                  f"{args.warmup} untimed then {len(ms)} timed force evaluations through bh::step_particles; "
                  f"rate = N*{w['steps']}/({w['steps'] + 1}*mean eval time)")
    line = {
        "impl": "reference", "metric": METRIC if w["kind"] != "csv" else "csv-ingest particles/s", "value": value,
        "unit": unit, "n_gpus": args.gpus, "steps": steps_done, "warmup": warm_done, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args.workload, w, world),
        "cpu_baseline": {"value": value, "unit": unit, "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if step_note:
        line["step"] = step_note
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------- GPU arm

class Rig:
    """Device, stream, replicas and the timing helpers of one rank."""

    def __init__(self):
        import torch

        from bhg.replicas import Replicas

        self.torch = torch
        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        self.rep = Replicas("nccl", f"cuda:{local}")
        self.world, self.rank, self.local = self.rep.world, self.rep.rank, self.rep.local
        self.stream = torch.cuda.Stream(device=self.local)

    def barrier(self):
        self.torch.cuda.synchronize(self.local)
        self.rep.barrier()

    def max_over_ranks(self, v):
        return self.rep.max(v)

    def sum_over_ranks(self, v):
        return self.rep.sum(v)

    def time_steps(self, fn, steps, warmup, after_warmup=None):
        """Device ms of `steps` calls of fn (CUDA events on the stream) and wall
        ms, both max over ranks, and the clock samples of the region."""
        for _ in range(warmup):
            fn()
        self.barrier()
        if after_warmup:
            after_warmup()
        clk = ClockSampler(self.local)
        with clk:
            e0 = self.torch.cuda.Event(enable_timing=True)
            e1 = self.torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            e0.record(self.stream)
            for _ in range(steps):
                fn()
            e1.record(self.stream)
            self.barrier()
            wall = (time.perf_counter() - t0) * 1000.0
        ms = max(e0.elapsed_time(e1), 0.0)
        return self.max_over_ranks(ms), self.max_over_ranks(wall), clk.summary()


def roofline(st, n_per_eval, fp32_peak, peaks):
    flops = FLOPS_PP * st["pp"] + FLOPS_PC * st["pc"]
    evals = max(1, st["evals"])
    walk_ms = st["walk_ms"]
    achieved = flops / (walk_ms / 1000.0) / 1e12 if walk_ms > 0 else 0.0
    traffic = None
    prof = os.path.join(ROOT, "profiles", "walk_ncu.json")
    if os.path.exists(prof):
        p = json.load(open(prof))
        # the capture's DRAM bytes scale with the particles a launch processes
        traffic = p["captured_dram_bytes"] * n_per_eval / p["captured_n"]
    sort_bytes = n_per_eval * (8 + SORT_BYTES_PER_PASS * st["sort_passes"]) * evals
    sort_gbs = sort_bytes / (st["sort_ms"] / 1000.0) / 1e9 if st["sort_ms"] > 0 else 0.0
    hbm = peaks.get("hbm_gbs")
    return {
        "roofline": {"bound": "fp32-fma", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                     "frac": achieved / fp32_peak if fp32_peak else None, "traffic": traffic,
                     "kernel": "k_walk (force walk + fused kick/drift)",
                     "peak_source": "measured: FFMA calibration loop on this GPU (bhg_measure_fp32_peak)",
                     "flops_per_launch": flops / evals, "ms_per_launch": walk_ms / evals,
                     "flop_model": "20 per particle-particle, 60 per particle-cell quadrupole interaction",
                     "traffic_source": "profiles/walk_ncu.json: dram read+write of one captured launch, scaled "
                                       "by particles per launch"},
        "roofline_sort": {"bound": "hbm", "achieved": sort_gbs, "peak": hbm, "unit": "GB/s",
                          "frac": sort_gbs / hbm if hbm else None,
                          "peak_source": "MEASURED_PEAKS.json hbm_gbs (copy)",
                          "bytes_model": "N*(8 + 24*passes) per sort", "ms_per_sort": st["sort_ms"] / evals},
        "phases_ms_per_eval": {k: st[k] / evals for k in ("pre_ms", "sort_ms", "tree_ms", "multipole_ms",
                                                          "targets_ms", "walk_ms")},
        "interactions_per_particle": {"pp": st["pp"] / (n_per_eval * evals), "pc": st["pc"] / (n_per_eval * evals)},
        "gpu_launches": st["kernels_per_eval"] * st["evals"],
    }


def force_error(ctx, parts, fp, leaf, group, target, eps2, nsample=4096):
    """rms / p99 relative force error of one walk vs FP64 direct sum on sampled particles."""
    ctx.upload(parts)
    ctx.build_tree(leaf, group)
    ctx.compute_multipoles()
    acc = ctx.walk_forces(fp, target)  # kick = drift = 0: positions unchanged (Morton order)
    n = len(parts)
    idx = np.sort(np.random.default_rng(12345).choice(n, size=min(nsample, n), replace=False)).astype(np.uint32)
    ref = ctx.direct_sum(idx, eps2)
    rel = np.linalg.norm(acc[idx] - ref, axis=1) / np.linalg.norm(ref, axis=1)
    return {"vs": f"FP64 direct sum (GPU, brute_force.h semantics) on {len(idx)} sampled particles",
            "rms": float(np.sqrt(np.mean(rel ** 2))), "p99": float(np.percentile(rel, 99)),
            "global": float(np.sqrt(np.sum((acc[idx] - ref) ** 2) / np.sum(ref ** 2)))}


def cpu_single(w):
    """The CPU-baseline leg of the GPU arm's line: the reference on the
    workload's system (bounded to ~20 s: the full system, else a smaller one
    of the same kind), one timed evaluation after one untimed."""
    try:
        n = ref_sample_n(w, 2, budget_s=20.0)
        ms, threads = run_ref(workload_spheres(w, n), w["seed"], w, 1, 1)
        return {"value": cpu_rate(n, ms, w), "unit": "particle-steps/s", "cores": threads, "kind": "reference",
                "sample": (f"{'full system' if n == w['n'] else f'N={n}, same generator and parameters'}: "
                           f"1 timed force evaluation (after 1 untimed) of the reference schedule through "
                           f"bh::step_particles; rate = N*{w['steps']}/({w['steps'] + 1}*eval time)")}
    except (OSError, subprocess.CalledProcessError) as e:
        return {"value": None, "unit": "particle-steps/s", "cores": None, "kind": "reference",
                "sample": f"unavailable: {e}"}


def bench_single(args, w, rig, bhg, fp32_peak, peaks):
    parts = make_particles(w, rig.rank)
    n = len(parts)
    prec = bhg.PRECISION_SPLIT if args.precision == "split" else bhg.PRECISION_FP64
    fp = bhg.Context.params(w["theta"], w["eps"] ** 2, 1.0, True, prec)
    walk_group, tuned = args.walk_group, None
    if not walk_group:
        # the walk-group cap from the autotuner (leaf and target sizes are the
        # workload's own; theta is never tuned)
        from bhg import autotune

        tuned = autotune.tune([parts], w["theta"], w["eps"] ** 2, w["group"], prec, device=rig.local,
                              cands=autotune.candidates(leaves=(w["max_leaf"],), walk_groups=(32, 64)))
        walk_group = tuned["walk_group"]
    ctx = bhg.Context(device=rig.local)
    ctx.set_stream(rig.stream.cuda_stream)
    ctx.set_walk_shape(walk_group)
    ctx.upload(parts)

    def one_step():
        ctx.run_schedule(fp, w["max_leaf"], w["group"], w["target"], w["dt"], w["steps"])

    one_step()
    ms, wall, clocks = rig.time_steps(one_step, args.steps, max(0, args.warmup - 1), lambda: ctx.stats(reset=True))
    st = ctx.stats(reset=True)
    ps = rig.sum_over_ranks(n * w["steps"] * args.steps)
    out = {"value": ps / (ms / 1000.0), "ms_per_step": ms / args.steps, "clocks": clocks,
           **roofline(st, n, fp32_peak, peaks)}

    if not args.no_e2e:
        # through the C ABI with host buffers: H2D of the state from pinned
        # memory, the schedule, D2H of the result, every step
        pin = rig.torch.empty(n * 64, dtype=rig.torch.uint8, pin_memory=True)
        host = np.frombuffer(pin.numpy(), dtype=bhg.PARTICLE)
        host[:] = ctx.download()
        ptr = pin.data_ptr()

        def e2e_step():
            ctx._ck(ctx.L.bhg_upload(ctx.h, ptr, n))
            one_step()
            ctx._ck(ctx.L.bhg_download(ctx.h, ptr))

        ems, ewall, _ = rig.time_steps(e2e_step, args.steps, 1)
        ems = max(ems, ewall)
        out["e2e"] = {"value": ps / (ems / 1000.0), "unit": "particle-steps/s", "h2d_bytes_per_step": n * 64,
                      "d2h_bytes_per_step": n * 64, "ms_per_step": ems / args.steps,
                      "path": "bhg_upload (pinned host) + bhg_run_schedule + bhg_download"}
    if rig.rank == 0:
        out["force_error"] = force_error(ctx, parts, fp, w["max_leaf"], w["group"], w["target"], w["eps"] ** 2)
    ctx.close()
    if rig.rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_single(w)
    out["config_extra"] = {"n": n, "walk_group": walk_group}
    if tuned is not None:
        out["autotune"] = {k: tuned[k] for k in ("walk_group", "rms_error", "err_budget", "table")}
    return out


def bench_ensemble(args, w, rig, bhg, fp32_peak, peaks, quick=False):
    """quick: the gate check inside the default run - fewer timed steps, no
    pipelined end-to-end leg, no CPU baseline."""
    from bhg import autotune

    if quick:
        args = argparse.Namespace(**vars(args))
        args.steps, args.warmup, args.no_e2e, args.no_cpu_baseline, args.no_plain = 3, 2, True, True, False

    systems = make_particles(w, rig.rank)
    ns = len(systems)
    n = sum(len(p) for p in systems)
    eps2 = w["eps"] ** 2
    tuned = autotune.tune(systems, w["theta"], eps2, w["group"], bhg.PRECISION_SPLIT, device=rig.local,
                          cands=TUNE_CANDIDATES())
    leaf = tuned["max_leaf"]
    fp = bhg.Context.params(w["theta"], eps2, 1.0, True, bhg.PRECISION_SPLIT)
    ctx = bhg.Context(device=rig.local)
    ctx.set_stream(rig.stream.cuda_stream)
    ctx.set_walk_shape(tuned["walk_group"])
    ctx.upload_systems(systems)
    ones = np.ones(ns)

    def one_step():  # one lockstep KDK evaluation of every system
        ctx.set_system_params(theta=ones * w["theta"], eps2=ones * eps2, kick_dt=ones * w["dt"],
                              drift_dt=ones * w["dt"])
        ctx.step_systems(fp, leaf, w["group"], leaf)

    one_step()
    ms, wall, clocks = rig.time_steps(one_step, args.steps, max(0, args.warmup - 1), lambda: ctx.stats(reset=True))
    st = ctx.stats(reset=True)
    ps = rig.sum_over_ranks(n * args.steps)
    out = {"value": ps / (ms / 1000.0), "ms_per_step": ms / args.steps, "clocks": clocks,
           **roofline(st, n, fp32_peak, peaks),
           "autotune": {k: tuned[k] for k in ("max_leaf", "target_size", "walk_group", "rms_error", "err_budget",
                                               "table")}}

    if not args.no_e2e:
        flat = np.concatenate(systems)
        pin = rig.torch.empty(n * 64, dtype=rig.torch.uint8, pin_memory=True)
        host = np.frombuffer(pin.numpy(), dtype=bhg.PARTICLE)
        host[:] = flat
        ptr = pin.data_ptr()
        counts = np.array([len(p) for p in systems], np.uint64)

        def e2e_step():
            ctx._ck(ctx.L.bhg_upload_systems(ctx.h, ptr, counts.ctypes.data, ns))
            one_step()
            ctx._ck(ctx.L.bhg_download(ctx.h, ptr))

        ems, ewall, _ = rig.time_steps(e2e_step, args.steps, 1)
        one_ctx_ms = max(ems, ewall)
        # the same through bhg.pipeline: the systems in --pipe-parts contexts,
        # each context's copies overlapping the others' evaluations (same bits)
        from bhg.pipeline import Pipeline

        host[:] = flat
        pipe = Pipeline(counts, parts=args.pipe_parts, device=rig.local, walk_group=tuned["walk_group"])

        def pipe_step():
            pipe.step(ptr, fp, leaf, w["group"], leaf, w["theta"], eps2, w["dt"], w["dt"])

        pms, pwall, _ = rig.time_steps(pipe_step, args.steps, 1)
        pipe.close()
        ems = max(pms, pwall)  # wall clock: the contexts' streams are not the timing stream
        out["e2e"] = {"value": ps / (ems / 1000.0), "unit": "particle-steps/s", "h2d_bytes_per_step": n * 64,
                      "d2h_bytes_per_step": n * 64, "ms_per_step": ems / args.steps,
                      "path": f"bhg.pipeline over {args.pipe_parts} contexts: bhg_upload_systems (pinned host) + "
                              "bhg_step_systems_async + bhg_download_async + bhg_sync",
                      "one_context": {"value": ps / (one_ctx_ms / 1000.0), "ms_per_step": one_ctx_ms / args.steps,
                                      "path": "bhg_upload_systems (pinned host) + bhg_step_systems + bhg_download"}}
    if rig.rank == 0:
        big = systems[int(np.argmax([len(p) for p in systems]))]
        out["force_error"] = force_error(ctx, big, fp, leaf, w["group"], leaf, eps2)
        out["force_error"]["system"] = f"largest system (N={len(big)}) at the tuned leaf {leaf}"
    ctx.close()

    if not args.no_plain:
        # the plain FP64 path, one system at a time: a resident context per
        # system, each evaluation stepping the 512 contexts in turn with the
        # reference's leaf/target/group sizes
        fp64 = bhg.Context.params(w["theta"], eps2, 1.0, True, bhg.PRECISION_FP64)
        ctxs = []
        for p in systems:
            c = bhg.Context(device=rig.local)
            # one system per context: below 131,072 particles the smaller
            # walk groups keep more warps busy (plummer-65k: 0.63 ms walk at
            # 32 against 0.85 ms at 64)
            c.set_walk_shape(32 if len(p) < 131072 else 64)
            c.upload(p)
            ctxs.append(c)

        def plain_step():
            for c in ctxs:
                c.step(fp64, w["max_leaf"], w["group"], w["target"], w["dt"], w["dt"])

        plain_step()
        rig.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            plain_step()
        rig.barrier()
        pms = rig.max_over_ranks((time.perf_counter() - t0) * 1000.0)
        for c in ctxs:
            c.close()
        pv = ps / (pms / 1000.0)
        out["plain_fp64_one_at_a_time"] = {
            "value": pv, "unit": "particle-steps/s", "ms_per_step": pms / args.steps,
            "path": "512 resident contexts stepped in turn, FP64 walk, leaf/target 16, group 256, walk groups of "
                    "32 particles below 131,072 particles and 64 above (wall clock)"}
        out["speedup_vs_plain"] = out["value"] / pv

    if rig.rank == 0 and not args.no_cpu_baseline:
        try:
            v, threads, sample = cpu_ensemble_sample(w)
            out["cpu_baseline"] = {"value": v, "unit": "particle-steps/s", "cores": threads, "kind": "reference",
                                   "sample": sample}
        except (OSError, subprocess.CalledProcessError) as e:
            out["cpu_baseline"] = {"value": None, "unit": "particle-steps/s", "cores": None, "kind": "reference",
                                   "sample": f"unavailable: {e}"}
    out["config_extra"] = {"systems": ns, "n_total": n, "max_leaf_tuned": leaf}
    return out


def bench_csv(args, w, rig, bhg, peaks):
    """read_csv on the GPU: the CSV text of the workload's particles, parsed
    into the context's state each step."""
    import ctypes

    torch = rig.torch
    parts, _ = bhg.plummer(w["n"], w["seed"])
    with tempfile.NamedTemporaryFile(suffix=".csv", delete=False) as f:
        path = f.name
    try:
        bhg.write_csv(path, parts)
        text = open(path, "rb").read()
    finally:
        os.unlink(path)
    nb = len(text)
    dev = torch.frombuffer(bytearray(text), dtype=torch.uint8).to(f"cuda:{rig.local}")
    ctx = bhg.Context(device=rig.local)
    ctx.set_stream(rig.stream.cuda_stream)

    def one_step():
        ctx.upload_csv_device(dev.data_ptr(), nb)

    ms, wall, clocks = rig.time_steps(one_step, args.steps, args.warmup)
    n = w["n"]
    assert ctx.n == n and ctx.download().tobytes() == parts.tobytes()  # the text round-trips exactly
    ps = rig.sum_over_ranks(n * args.steps)
    algo = nb + 64 * n  # text read once, particles written once
    hbm = peaks.get("hbm_gbs")
    gbs = algo / (ms / args.steps / 1000.0) / 1e9
    out = {"value": ps / (ms / 1000.0), "ms_per_step": ms / args.steps, "clocks": clocks,
           "roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s",
                        "frac": gbs / hbm if hbm else None, "traffic": None,
                        "kernel": "the whole ingest (newline count/scan/emit, k_csv_parse, compaction)",
                        "bytes_model": "text bytes + 64 B per particle"},
           "gpu_launches": 9 * args.steps}
    if not args.no_e2e:
        pin = torch.empty(nb, dtype=torch.uint8, pin_memory=True)
        pin.numpy()[:] = np.frombuffer(text, np.uint8)
        addr = ctypes.c_char_p(pin.data_ptr())

        def e2e_step():
            ctx._ck(ctx.L.bhg_upload_csv(ctx.h, addr, nb))

        ems, _, _ = rig.time_steps(e2e_step, args.steps, 1)
        out["e2e"] = {"value": ps / (ems / 1000.0), "unit": "particles/s", "h2d_bytes_per_step": nb,
                      "d2h_bytes_per_step": 0, "path": "bhg_upload_csv from pinned host memory"}
    # write_vtk on the device: formatted there, the text copied back into a
    # pinned host buffer (a Python bytes copy of it costs more than all of that:
    # reported beside it)
    snap = ctx.snapshot_vtk()
    spin = rig.torch.empty(ctx.snapshot_vtk_bound(), dtype=rig.torch.uint8, pin_memory=True).numpy()
    ctx.snapshot_vtk_into(spin)
    t0 = time.perf_counter()
    for _ in range(3):
        nsnap = ctx.snapshot_vtk_into(spin)
    snap_s = (time.perf_counter() - t0) / 3
    t0 = time.perf_counter()
    for _ in range(3):
        snap = ctx.snapshot_vtk()
    bytes_s = (time.perf_counter() - t0) / 3
    out["snapshot_vtk"] = {"particles_per_s": n / snap_s, "ms": snap_s * 1000.0, "bytes": nsnap,
                           "path": "bhg_snapshot_vtk into pinned host memory (wall clock)",
                           "as_python_bytes_ms": bytes_s * 1000.0}
    ctx.close()
    if rig.rank == 0 and not args.no_cpu_baseline:
        try:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            from oracle import Reference

            ref = Reference()
            t0 = time.perf_counter()
            ref_snap = ref.write_vtk(parts)
            out["snapshot_vtk"]["reference_particles_per_s"] = n / (time.perf_counter() - t0)
            out["snapshot_vtk"]["same_bytes_as_reference"] = ref_snap == snap
            with tempfile.NamedTemporaryFile(suffix=".csv", delete=False) as f:
                f.write(text)
                path = f.name
            try:
                cap = n + 1
                buf = np.zeros(cap, bhg.PARTICLE)
                cnt = ctypes.c_size_t()
                err = ctypes.create_string_buffer(256)
                ref.lib.bhref_read_csv(path.encode(), buf.ctypes.data, cap, ctypes.byref(cnt), err, 256)  # warm
                t0 = time.perf_counter()
                ref.lib.bhref_read_csv(path.encode(), buf.ctypes.data, cap, ctypes.byref(cnt), err, 256)
                dt = time.perf_counter() - t0
            finally:
                os.unlink(path)
            out["cpu_baseline"] = {"value": n / dt, "unit": "particles/s", "cores": os.cpu_count(),
                                   "kind": "reference",
                                   "sample": f"the full text ({nb} bytes) through the reference's read_csv (mmap + one "
                                             f"thread per usable CPU), after one untimed read"}
        except (OSError, AttributeError) as e:
            out["cpu_baseline"] = {"value": None, "unit": "particles/s", "cores": None, "kind": "reference",
                                   "sample": f"unavailable: {e}"}
    out["config_extra"] = {"text_bytes": nb, "number_format": "%.17g"}
    return out


def bench_serve(args, w, rig, bhg, fp32_peak, peaks, quick=False):
    """The request loop in real time over the Poisson stream, for a bounded
    wall window; value = particle-steps completed / wall time.  quick: the
    gate check inside the default run - a 30 s window, no CPU baseline."""
    from bhg import serve

    w = dict(w)
    if quick:
        args = argparse.Namespace(**vars(args))
        args.no_cpu_baseline = True
        args.serve_wall = args.serve_wall or 30.0

    if args.serve_budget_gb is not None:
        w["hbm_budget_gb"] = args.serve_budget_gb
    if args.serve_wall is not None:
        w["wall_limit_s"] = args.serve_wall
    if args.serve_duration is not None:
        w["duration"] = args.serve_duration
    if args.serve_max_batch is not None:
        w["max_batch_particles"] = args.serve_max_batch
    reqs = serve_stream(w)
    # leaf (= target) size from the autotuner, on a sample of the stream's
    # requests (their initial conditions from the same device generator) at
    # theta 0.5, the accuracy gate's theta; theta itself is never tuned
    from bhg import autotune

    sample, tot = [], 0
    for r in reqs[:64]:
        if tot + r.n <= 8_000_000 and len(sample) < 16:
            sample.append(r)
            tot += r.n
    with bhg.Context(device=rig.local) as c:
        for r in sample:
            c.add_generated(r.spheres(), r.seed, id0=0)
        allp = c.download()
    offs = np.cumsum([0] + [r.n for r in sample])
    tuned = autotune.tune([allp[offs[i]:offs[i + 1]] for i in range(len(sample))], 0.5, w["eps"] ** 2, w["group"],
                          bhg.PRECISION_SPLIT, device=rig.local, cands=TUNE_CANDIDATES())
    leaf = tuned["max_leaf"]
    # warm-up: a few small requests through the same loop (kernels loaded,
    # occupancy queried)
    warm = serve.Server(device=rig.local, hbm_budget=2e9, max_leaf=leaf, group_size=w["group"])
    warm.run([serve.Request(i, 0.0, "merger" if i % 2 else "plummer", 20000, 2, 0.5, 90 + i) for i in range(3)],
             realtime=False)
    warm.close()
    delivered = [0]

    def on_result(rid, parts):  # the finished state goes back to the host and is dropped
        delivered[0] += 1

    srv = serve.Server(device=rig.local, hbm_budget=w["hbm_budget_gb"] * 1e9, max_leaf=leaf,
                       group_size=w["group"], on_result=on_result, walk_group=tuned["walk_group"],
                       max_batch_particles=w.get("max_batch_particles"))
    srv.ctx.stats(reset=True)
    rig.barrier()
    clk = ClockSampler(rig.local)
    with clk:
        rep = srv.run(reqs, wall_limit=w["wall_limit_s"], realtime=True)
    rig.barrier()
    st = srv.ctx.stats(reset=True)
    ticks = max(1, rep["ticks"])
    n_eval = max(1, srv.particle_evals // ticks)
    srv.close()
    rep["offered_requests"] = len(reqs)
    rep["offered_particle_steps_per_s"] = sum(r.n * r.steps for r in reqs) / w["duration"]
    rep["delivered"] = delivered[0]
    wall = rig.max_over_ranks(rep["wall_s"])
    ps = rig.sum_over_ranks(rep["particle_steps"])
    out = {"value": ps / wall, "ms_per_step": float(np.mean(srv.tick_ms)) if srv.tick_ms else None,
           "clocks": clk.summary(), "serving": rep,
           "latency_ms": {"p50": rep["step_latency_ms_p50"], "p99": rep["step_latency_ms_p99"],
                          "per": "request step: wall time of the batched evaluation that advanced it"},
           **roofline(st, n_eval, fp32_peak, peaks)}
    out["e2e"] = {"value": ps / wall, "unit": "particle-steps/s",
                  "h2d_bytes_per_step": int(64 * srv.system_evals / ticks),  # one 64-byte parameter record per system
                  "d2h_bytes_per_step": int(srv.d2h_bytes / ticks),
                  "path": "the request loop itself: requests arrive as seeds (initial conditions generated on the "
                          "device), per-system parameters go up every tick, finished states come back to the "
                          "host; the wall clock runs around all of it"}
    if rig.rank == 0 and not args.no_cpu_baseline:
        try:
            v, threads, sample = cpu_serve_sample(w)
            out["cpu_baseline"] = {"value": v, "unit": "particle-steps/s", "cores": threads, "kind": "reference",
                                   "sample": sample}
        except (OSError, subprocess.CalledProcessError) as e:
            out["cpu_baseline"] = {"value": None, "unit": "particle-steps/s", "cores": None, "kind": "reference",
                                   "sample": f"unavailable: {e}"}
    if rig.rank == 0:
        # a served system's forces are those of the system alone, bit for bit
        # (tests/test_gpu_serve.py): the force error of the largest theta-0.5
        # request among the stream's first 64, its initial conditions made by
        # the same device generator
        pick = max((r for r in reqs[:64] if r.theta == 0.5), key=lambda r: r.n, default=None)
        if pick is not None:
            with bhg.Context(device=rig.local) as c:
                c.add_generated(pick.spheres(), pick.seed, id0=0)
                parts = c.download()
                fp = bhg.Context.params(0.5, pick.eps ** 2, 1.0, True, bhg.PRECISION_SPLIT)
                out["force_error"] = force_error(c, parts, fp, leaf, w["group"], leaf, pick.eps ** 2)
            out["force_error"]["system"] = f"request {pick.rid}: {pick.kind}, N={pick.n}, theta 0.5, leaf {leaf}"
    out["config_extra"] = {"mean_particles_per_tick": n_eval, "max_leaf_tuned": leaf}
    out["autotune"] = {k: tuned[k] for k in ("max_leaf", "target_size", "walk_group", "rms_error", "err_budget",
                                             "table")}
    out["autotune"]["sample"] = f"{len(sample)} of the stream's first 64 requests, {tot} particles, theta 0.5"
    return out


def gates_block(args, rig, bhg, fp32_peak, peaks):
    """The two throughput gates of the batched and served paths, measured in
    the default run (each with its own clock record):

    * ensemble-512: the 512-system ensemble in one segmented key space,
      split precision, tuned leaf, against the plain FP64 path stepping the
      systems one at a time (gate: >= 4x, rms force error <= 1e-3);
    * serve-200rps: the continuous-batching server on the Poisson request
      stream for a 30 s window (p50/p99 per-step latency, aggregate
      particle-steps/s)."""
    out = {}
    e = bench_ensemble(args, WORKLOADS["ensemble-512"], rig, bhg, fp32_peak, peaks, quick=True)
    if rig.rank == 0:
        out["ensemble_512"] = {
            "value": e["value"], "unit": "particle-steps/s", "ms_per_step": e["ms_per_step"], "steps": 3,
            "warmup": 2, "plain_fp64_one_at_a_time": e.get("plain_fp64_one_at_a_time"),
            "speedup_vs_plain": e.get("speedup_vs_plain"), "gate_speedup": 4.0,
            "force_error": e.get("force_error"), "clocks": e.get("clocks"),
            "walk_roofline_frac": e["roofline"]["frac"], "autotune": e.get("autotune"),
            "details": e.get("config_extra")}
    sv = bench_serve(args, WORKLOADS["serve-200rps"], rig, bhg, fp32_peak, peaks, quick=True)
    if rig.rank == 0:
        out["serve_200rps"] = {
            "value": sv["value"], "unit": "particle-steps/s", "latency_ms": sv.get("latency_ms"),
            "window_s": sv["serving"].get("wall_s"), "completed": sv["serving"].get("completed"),
            "admitted": sv["serving"].get("admitted"), "force_error": sv.get("force_error"),
            "clocks": sv.get("clocks"), "walk_roofline_frac": sv["roofline"]["frac"],
            "details": sv.get("config_extra")}
    return out


def main():
    args = parse()
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        return reference_arm(args, w)
    rig = Rig()
    import bhg

    peaks = json.load(open(MEASURED_PEAKS)) if os.path.exists(MEASURED_PEAKS) else {}
    fp32_peak = bhg.measure_fp32_peak(rig.local)
    if w["kind"] == "ensemble":
        res = bench_ensemble(args, w, rig, bhg, fp32_peak, peaks)
        dtype = "f32+f64"
    elif w["kind"] == "serve":
        res = bench_serve(args, w, rig, bhg, fp32_peak, peaks)
        dtype = "f32+f64"
    elif w["kind"] == "csv":
        res = bench_csv(args, w, rig, bhg, peaks)
        dtype = "u8->f64"
    else:
        res = bench_single(args, w, rig, bhg, fp32_peak, peaks)
        dtype = "f32+f64" if args.precision == "split" else "f64"
    # the gates are single-GPU ones: not repeated on every replica of a
    # multi-GPU run
    if w["kind"] == "single" and args.workload == "plummer-4m" and not args.no_gates and rig.world == 1:
        res["gates"] = gates_block(args, rig, bhg, fp32_peak, peaks)
    if rig.rank == 0:
        cfg = workload_config(args.workload, w, rig.world)
        metric, unit = (METRIC, "particle-steps/s") if w["kind"] != "csv" else ("csv-ingest particles/s", "particles/s")
        details = res.pop("config_extra")
        line = {"metric": metric, "value": res.pop("value"), "unit": unit, "n_gpus": rig.world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": res.pop("ms_per_step"),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
                "data": "synthetic", "config": cfg,
                "precision": args.precision if w["kind"] in ("single", "merger") else "split", "details": details,
                **res}
        print(json.dumps(line), flush=True)
    rig.rep.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
