#!/usr/bin/env python3
"""Benchmark of the B200 Barnes-Hut hot path (one JSON line on rank 0).

Workload (default): the single-system N = 4,194,304 Plummer sphere (seed 2,
G = M = a = 1, theta 0.5, eps 0.005, monopole + quadrupole, max_leaf 16,
target 16, group 256), advanced by the reference's leapfrog schedule for 8
KDK steps of dt = 1/256 (main.cc:199-246: 9 force evaluations).  One bench
step = that whole 8-step sequence over the GPU-resident particles; the
metric is particle-steps/s = N * 8 * steps / time.  Other workloads:
--workload plummer-65k (N = 65,536, seed 1, eps 0.01, dt 1/128, 16 steps).

--impl reference times the reference's own CPU implementation of the path
(oracle/_ref/ref_bench: the unmodified reference sources with a thread-pool
stand-in for TTG) on all host cores, on the same workload and metric.

Multi-GPU: one process per GPU, each an independent replica of the workload
(a Barnes-Hut system does not shard here; no collective on the data path);
value = particle-steps of all ranks / max over ranks of the device time.
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
    "plummer-4m": dict(n=4194304, seed=2, theta=0.5, eps=0.005, max_leaf=16, target=16, group=256,
                       dt=1.0 / 256, steps=8),
    "plummer-65k": dict(n=65536, seed=1, theta=0.5, eps=0.01, max_leaf=16, target=16, group=256,
                        dt=1.0 / 128, steps=16),
    # a smaller case of the 4M workload's parameters, for profiler captures
    "plummer-1m": dict(n=1048576, seed=2, theta=0.5, eps=0.005, max_leaf=16, target=16, group=256,
                       dt=1.0 / 256, steps=1),
}
METRIC = "particle-steps/s"
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
SORT_BYTES_PER_PASS = 24  # read + write of an 8-byte key and a 4-byte index
FLOPS_PP, FLOPS_PC = 20, 60


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
    return ap.parse_args()


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


def run_ref(parts, w, evals, threads=None):
    """Times `evals` evaluations of the reference schedule; returns eval ms list."""
    exe = ref_binary()
    if exe is None:
        raise FileNotFoundError("oracle/_ref/ref_bench is not built")
    with tempfile.NamedTemporaryFile(suffix=".bin", delete=False) as f:
        parts.tofile(f)
        path = f.name
    env = dict(os.environ)
    if threads:
        env["TTG_NUM_THREADS"] = str(threads)
    try:
        cmd = [exe, "--particles", path, "--steps", str(w["steps"]), "--evals", str(evals), "--dt", repr(w["dt"]),
               "--theta", repr(w["theta"]), "--eps", repr(w["eps"]), "--max-leaf", str(w["max_leaf"]),
               "--target-size", str(w["target"]), "--group-size", str(w["group"])]
        out = subprocess.run(cmd, check=True, capture_output=True, text=True, env=env).stdout
    finally:
        os.unlink(path)
    rec = json.loads(out.strip().splitlines()[-1])
    return rec["eval_ms"], rec["threads"]


def cpu_sample(w, budget_s=20.0):
    """A bounded sample of the workload on the reference: the full system if one
    evaluation fits the budget, else the largest power-of-two Plummer sphere of
    the same parameters that does.  Returns (n, per-eval ms list, threads)."""
    import bhg

    n_probe = min(w["n"], 65536)
    parts, _ = bhg.plummer(n_probe, w["seed"])
    ms, threads = run_ref(parts, w, 2)
    per = ms[-1] / n_probe  # ms per particle per evaluation
    n = n_probe
    while n * 2 <= w["n"] and per * (n * 2) * 1.15 * 2 / 1000.0 < budget_s:
        n *= 2
        per *= 1.1  # the walk cost per particle grows with log N
    if n != n_probe:
        parts, _ = bhg.plummer(n, w["seed"])
        ms, threads = run_ref(parts, w, 2)
    return n, ms, threads


def cpu_rate(n, eval_ms, w):
    """particle-steps/s of the schedule (steps advances per steps+1 evaluations)."""
    t = float(np.mean(eval_ms[1:] if len(eval_ms) > 1 else eval_ms)) / 1000.0
    return n * w["steps"] / ((w["steps"] + 1) * t)


def reference_arm(args, w):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import bhg

    n, _, _ = cpu_sample(w)
    parts, _ = bhg.plummer(n, w["seed"])
    ms, threads = run_ref(parts, w, args.warmup + args.steps)
    timed = ms[args.warmup:]
    value = cpu_rate(n, [0.0] + timed, w)
    sample = (f"{'full system' if n == w['n'] else f'N={n} Plummer sphere (same generator and parameters)'}: "
              f"{len(timed)} force evaluations of the reference schedule through bh::step_particles, "
              f"rate = N*{w['steps']}/({w['steps'] + 1}*mean eval time)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(timed)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "n": w["n"], "sample_n": n, "theta": w["theta"], "eps": w["eps"],
                   "max_leaf": w["max_leaf"], "target_size": w["target"], "group_size": w["group"],
                   "dt": w["dt"], "kdk_steps": w["steps"], "threads": threads},
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------- GPU arm

def main():
    args = parse()
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        return reference_arm(args, w)

    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import bhg

    peaks = json.load(open(MEASURED_PEAKS)) if os.path.exists(MEASURED_PEAKS) else {}
    fp32_peak = bhg.measure_fp32_peak(local)

    parts, _ = bhg.plummer(w["n"], w["seed"] + rank)
    prec = bhg.PRECISION_SPLIT if args.precision == "split" else bhg.PRECISION_FP64
    fp = bhg.Context.params(w["theta"], w["eps"] ** 2, 1.0, True, prec)
    stream = torch.cuda.Stream(device=local)
    ctx = bhg.Context(device=local)
    ctx.set_stream(stream.cuda_stream)
    ctx.upload(parts)

    def one_step():
        ctx.run_schedule(fp, w["max_leaf"], w["group"], w["target"], w["dt"], w["steps"])

    def barrier():
        torch.cuda.synchronize(local)
        if world > 1:
            torch.distributed.barrier()

    for _ in range(args.warmup):
        one_step()
    ctx.stats(reset=True)
    barrier()
    with ClockSampler(local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            one_step()
        e1.record(stream)
        barrier()
    ms = e0.elapsed_time(e1)
    st = ctx.stats(reset=True)
    if world > 1:
        t = torch.tensor([ms], device=f"cuda:{local}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    ps = w["n"] * w["steps"] * args.steps * world
    value = ps / (ms / 1000.0)

    # the walk kernel against the FP32 FMA roofline
    flops = FLOPS_PP * st["pp"] + FLOPS_PC * st["pc"]
    walk_ms = st["walk_ms"]
    evals = max(1, st["evals"])
    achieved = flops / (walk_ms / 1000.0) / 1e12 if walk_ms > 0 else 0.0
    traffic = None
    prof = os.path.join(ROOT, "profiles", "walk_ncu.json")
    if os.path.exists(prof):
        traffic = json.load(open(prof)).get("dram_bytes_per_launch")
    sort_bytes = w["n"] * (8 + SORT_BYTES_PER_PASS * st["sort_passes"]) * evals
    sort_gbs = sort_bytes / (st["sort_ms"] / 1000.0) / 1e9 if st["sort_ms"] > 0 else 0.0
    hbm = peaks.get("hbm_gbs")

    # end to end through the C ABI with host buffers: H2D of the state from
    # pinned memory, the schedule, D2H of the result, every step
    e2e = None
    if not args.no_e2e:
        pin = torch.empty(w["n"] * 64, dtype=torch.uint8, pin_memory=True)
        host = np.frombuffer(pin.numpy(), dtype=bhg.PARTICLE)
        host[:] = ctx.download()
        ptr = pin.data_ptr()

        def e2e_step():
            ctx._ck(ctx.L.bhg_upload(ctx.h, ptr, w["n"]))
            one_step()
            ctx._ck(ctx.L.bhg_download(ctx.h, ptr))

        e2e_step()
        barrier()
        t0 = time.perf_counter()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.steps):
            e2e_step()
        f1.record(stream)
        barrier()
        ems = max(f0.elapsed_time(f1), (time.perf_counter() - t0) * 1000.0)
        if world > 1:
            t = torch.tensor([ems], device=f"cuda:{local}")
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            ems = float(t.item())
        e2e = {"value": ps / (ems / 1000.0), "unit": "particle-steps/s", "h2d_bytes_per_step": w["n"] * 64,
               "d2h_bytes_per_step": w["n"] * 64, "ms_per_step": ems / args.steps,
               "path": "bhg_upload (pinned host) + bhg_run_schedule + bhg_download"}

    # accuracy: rms and 99th-percentile relative force error of this walk
    # against an FP64 direct sum on 4,096 sampled particles
    acc_err = None
    if rank == 0:
        ctx.build_tree(w["max_leaf"], w["group"])
        ctx.compute_multipoles()
        acc = ctx.walk_forces(fp, w["target"])  # kick = drift = 0: positions unchanged
        idx = np.sort(np.random.default_rng(12345).choice(w["n"], size=min(4096, w["n"]), replace=False))
        ref = ctx.direct_sum(idx.astype(np.uint32), w["eps"] ** 2)
        rel = np.linalg.norm(acc[idx] - ref, axis=1) / np.linalg.norm(ref, axis=1)
        acc_err = {"vs": "FP64 direct sum (GPU, brute_force.h semantics) on 4096 sampled particles",
                   "rms": float(np.sqrt(np.mean(rel ** 2))), "p99": float(np.percentile(rel, 99)),
                   "global": float(np.sqrt(np.sum((acc[idx] - ref) ** 2) / np.sum(ref ** 2)))}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            n, ems_cpu, threads = cpu_sample(w)
            cpu = {"value": cpu_rate(n, ems_cpu, w), "unit": "particle-steps/s", "cores": threads,
                   "kind": "reference",
                   "sample": (f"{'full system' if n == w['n'] else f'N={n} Plummer sphere, same parameters'}: "
                              f"1 timed force evaluation (after 1 untimed) of the reference schedule through "
                              f"bh::step_particles; rate = N*{w['steps']}/({w['steps'] + 1}*eval time)")}
        except (OSError, subprocess.CalledProcessError) as e:
            cpu = {"value": None, "unit": "particle-steps/s", "cores": None, "kind": "reference",
                   "sample": f"unavailable: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64" if prec == bhg.PRECISION_SPLIT else "f64", "data": "synthetic",
            "config": {"workload": args.workload, "n": w["n"], "seed": w["seed"], "theta": w["theta"],
                       "eps": w["eps"], "max_leaf": w["max_leaf"], "target_size": w["target"],
                       "group_size": w["group"], "dt": w["dt"], "kdk_steps_per_bench_step": w["steps"],
                       "precision": args.precision, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (particles 256 MB + tree ~150 MB per evaluation)"},
            "gpu_launches": st["kernels_per_eval"] * st["evals"],
            "roofline": {"bound": "fp32-fma", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": achieved / fp32_peak if fp32_peak else None, "traffic": traffic,
                         "kernel": "k_walk (force walk + fused kick/drift)",
                         "peak_source": "measured: FFMA calibration loop on this GPU (bhg_measure_fp32_peak)",
                         "flops_per_launch": flops / evals, "ms_per_launch": walk_ms / evals,
                         "flop_model": "20 per particle-particle, 60 per particle-cell quadrupole interaction"},
            "roofline_sort": {"bound": "hbm", "achieved": sort_gbs, "peak": hbm, "unit": "GB/s",
                              "frac": sort_gbs / hbm if hbm else None,
                              "peak_source": "MEASURED_PEAKS.json hbm_gbs (copy)",
                              "bytes_model": "N*(8 + 24*passes) per sort", "ms_per_sort": st["sort_ms"] / evals},
            "phases_ms_per_eval": {k: st[k] / evals for k in ("pre_ms", "sort_ms", "tree_ms", "multipole_ms",
                                                              "targets_ms", "walk_ms")},
            "interactions_per_particle": {"pp": st["pp"] / (w["n"] * evals), "pc": st["pc"] / (w["n"] * evals)},
            "clocks": clk.summary(),
            "force_error": acc_err,
            "e2e": e2e,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
