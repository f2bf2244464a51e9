"""Autotuner of the walk's shape for a set of systems.

theta is never tuned.  The tuned knobs are the reference's own (main.cc:27-33
exposes max_leaf, target_size and group_size as independent options) plus the
GPU walk's shape:

* ``max_leaf`` (= ``target_size``): the leaf and walk-target size;
* ``walk_group``: the particle cap of one warp's walk group (the targets of
  a group share one traversal; 0 = the library's default);
* ``walk_warps``: warps per block of the walk kernels (0 = the default).

For every candidate configuration it measures the force error of the largest
system against an FP64 direct sum on sampled particles, then times a few
batched evaluations of all systems (device time of the phases, CUDA events).
The fastest candidate whose rms relative error stays within the budget wins;
if none does, the one with the smallest error.  Results are cached in a JSON
file under a key that covers everything the choice depends on: the particle
count and system-count buckets, theta, eps2, precision, group size, error
budget, the candidate set, the device name and the library's walk version.
"""
from __future__ import annotations

import itertools
import json
import math
import os
import time

import numpy as np

from . import PRECISION_SPLIT, Context

DEFAULT_LEAVES = (16, 24, 32, 48, 64)
CACHE = os.path.join(os.path.expanduser("~"), ".cache", "bhg_autotune.json")
#: bumped whenever the walk kernels change in a way that can change timings
WALK_VERSION = "joint-walk-1"


def candidates(leaves=DEFAULT_LEAVES, walk_groups=(0,), walk_warps=(0,)):
    """The cross product of the knobs' values, as a list of dicts."""
    return [{"max_leaf": l, "target_size": l, "walk_group": g, "walk_warps": w}
            for l, g, w in itertools.product(leaves, walk_groups, walk_warps)]


def cache_key(total_n, nsys, theta, eps2, precision, group_size, err_budget, cands, device_name):
    cand = ",".join(f"{c['max_leaf']}/{c.get('walk_group', 0)}/{c.get('walk_warps', 0)}" for c in cands)
    return (f"{WALK_VERSION}|{device_name}|n2^{round(math.log2(max(total_n, 1)))}|sys2^{round(math.log2(max(nsys, 1)))}"
            f"|theta{theta:g}|eps2{eps2:g}|p{precision}|g{group_size}|err{err_budget:g}|{cand}")


def _apply_shape(ctx, cand):
    if (cand.get("walk_group") or cand.get("walk_warps")) and hasattr(ctx, "set_walk_shape"):
        ctx.set_walk_shape(cand.get("walk_group", 0), cand.get("walk_warps", 0))


def _error(ctx, systems, theta, eps2, cand, group_size, precision, nsample=512, seed=7):
    """rms relative force error of the largest system vs FP64 direct sum."""
    s = int(np.argmax([len(p) for p in systems]))
    ctx.upload(systems[s])
    _apply_shape(ctx, cand)
    fp = Context.params(theta, eps2, 1.0, True, precision)
    ctx.build_tree(cand["max_leaf"], group_size)
    ctx.compute_multipoles()
    acc = ctx.walk_forces(fp, cand["target_size"])
    n = len(systems[s])
    idx = np.sort(np.random.default_rng(seed).choice(n, size=min(nsample, n), replace=False)).astype(np.uint32)
    ref = ctx.direct_sum(idx, eps2)
    rel = np.linalg.norm(acc[idx] - ref, axis=1) / np.linalg.norm(ref, axis=1)
    return float(np.sqrt(np.mean(rel ** 2)))


def choose(table, err_budget):
    """The fastest row within the error budget, else the most accurate row."""
    ok = [r for r in table if r["rms_error"] <= err_budget]
    if ok:
        return min(ok, key=lambda r: r["ms_per_eval"])
    return min(table, key=lambda r: r["rms_error"])


def device_name(device):
    try:
        import torch

        return torch.cuda.get_device_name(device)
    except Exception:  # noqa: BLE001 - no torch or no device: the key just says so
        return "unknown-device"


def tune(systems, theta, eps2, group_size=256, precision=PRECISION_SPLIT, cands=None, err_budget=1e-3, evals=3,
         device=0, use_cache=True, log=None, context_factory=None, cache_path=None, dev_name=None):
    """Returns {"max_leaf", "target_size", "walk_group", "walk_warps", "ms_per_eval", "rms_error", "table", ...}.

    ``context_factory(device)`` makes the context (default: bhg.Context);
    tests pass a fake one."""
    cands = cands or candidates()
    make = context_factory or (lambda d: Context(device=d))
    path = cache_path or CACHE
    total = sum(len(p) for p in systems)
    key = cache_key(total, len(systems), theta, eps2, precision, group_size, err_budget, cands,
                    dev_name or device_name(device))
    cache = {}
    if use_cache and os.path.exists(path):
        try:
            cache = json.load(open(path))
        except (OSError, ValueError):
            cache = {}
        if key in cache:
            return dict(cache[key], cached=True)
    table = []
    ns = len(systems)
    ctx = make(device)
    try:
        for cand in cands:
            err = _error(ctx, systems, theta, eps2, cand, group_size, precision)
            ctx.upload_systems(systems)
            _apply_shape(ctx, cand)
            ctx.set_system_params(theta=np.full(ns, theta), eps2=np.full(ns, eps2), kick_dt=np.zeros(ns),
                                  drift_dt=np.zeros(ns))
            fp = Context.params(theta, eps2, 1.0, True, precision)
            ctx.step_systems(fp, cand["max_leaf"], group_size, cand["target_size"])  # warm-up, graph capture
            ctx.stats(reset=True)
            t0 = time.perf_counter()
            for _ in range(evals):
                ctx.step_systems(fp, cand["max_leaf"], group_size, cand["target_size"])
            wall = (time.perf_counter() - t0) * 1000.0 / evals
            st = ctx.stats(reset=True)
            dev = sum(st[k] for k in ("pre_ms", "sort_ms", "tree_ms", "multipole_ms", "targets_ms", "walk_ms"))
            row = dict(cand, ms_per_eval=dev / max(1, st["evals"]), wall_ms_per_eval=wall, rms_error=err)
            table.append(row)
            if log:
                log(row)
    finally:
        ctx.close()
    best = choose(table, err_budget)
    res = {"max_leaf": best["max_leaf"], "target_size": best["target_size"], "walk_group": best["walk_group"],
           "walk_warps": best["walk_warps"], "group_size": group_size, "ms_per_eval": best["ms_per_eval"],
           "rms_error": best["rms_error"], "table": table, "err_budget": err_budget, "theta": theta, "key": key}
    if use_cache:
        cache[key] = res
        try:
            os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
            json.dump(cache, open(path, "w"), indent=1)
        except OSError:
            pass
    return dict(res, cached=False)
