"""Autotuner of the walk's leaf and target sizes for a set of systems.

theta is never tuned.  For each candidate max_leaf (target_size = max_leaf,
group_size unchanged) it times a few force evaluations of the systems and
measures the force error against an FP64 direct sum on sampled particles of
the largest system; the fastest candidate whose rms relative error stays
within the budget wins.  Results are cached per (particle-count bucket,
theta, eps, precision) in a JSON file.
"""
from __future__ import annotations

import json
import math
import os
import time

import numpy as np

from . import PRECISION_SPLIT, Context

DEFAULT_CANDIDATES = (16, 24, 32, 48, 64)
CACHE = os.path.join(os.path.expanduser("~"), ".cache", "bhg_autotune.json")


def _key(total_n, theta, eps2, precision):
    return f"n2^{round(math.log2(max(total_n, 1)))}/theta{theta:g}/eps2{eps2:g}/p{precision}"


def _error(ctx, systems, theta, eps2, leaf, group_size, precision, nsample=512, seed=7):
    """rms relative force error of the largest system vs FP64 direct sum."""
    s = int(np.argmax([len(p) for p in systems]))
    ctx.upload(systems[s])
    fp = Context.params(theta, eps2, 1.0, True, precision)
    ctx.build_tree(leaf, group_size)
    ctx.compute_multipoles()
    acc = ctx.walk_forces(fp, leaf)
    n = len(systems[s])
    idx = np.sort(np.random.default_rng(seed).choice(n, size=min(nsample, n), replace=False)).astype(np.uint32)
    ref = ctx.direct_sum(idx, eps2)
    rel = np.linalg.norm(acc[idx] - ref, axis=1) / np.linalg.norm(ref, axis=1)
    return float(np.sqrt(np.mean(rel ** 2)))


def tune(systems, theta, eps2, group_size=256, precision=PRECISION_SPLIT, candidates=DEFAULT_CANDIDATES,
         err_budget=1e-3, evals=3, device=0, use_cache=True, log=None):
    """Returns {"max_leaf", "target_size", "ms_per_eval", "rms_error", "table"}."""
    total = sum(len(p) for p in systems)
    key = _key(total, theta, eps2, precision)
    cache = {}
    if use_cache and os.path.exists(CACHE):
        try:
            cache = json.load(open(CACHE))
        except (OSError, ValueError):
            cache = {}
        if key in cache:
            return cache[key]
    table = []
    with Context(device=device) as ctx:
        for leaf in candidates:
            err = _error(ctx, systems, theta, eps2, leaf, group_size, precision)
            ctx.upload_systems(systems)
            ctx.set_system_params(theta=np.full(len(systems), theta), eps2=np.full(len(systems), eps2),
                                  kick_dt=np.zeros(len(systems)), drift_dt=np.zeros(len(systems)))
            fp = Context.params(theta, eps2, 1.0, True, precision)
            ctx.step_systems(fp, leaf, group_size, leaf)  # warm-up, graph capture
            ctx.stats(reset=True)
            t0 = time.perf_counter()
            for _ in range(evals):
                ctx.step_systems(fp, leaf, group_size, leaf)
            wall = (time.perf_counter() - t0) * 1000.0 / evals
            st = ctx.stats(reset=True)
            dev = sum(st[k] for k in ("pre_ms", "sort_ms", "tree_ms", "multipole_ms", "targets_ms", "walk_ms"))
            row = {"max_leaf": leaf, "ms_per_eval": dev / max(1, st["evals"]), "wall_ms_per_eval": wall,
                   "rms_error": err}
            table.append(row)
            if log:
                log(row)
    ok = [r for r in table if r["rms_error"] <= err_budget] or table[:1]
    best = min(ok, key=lambda r: r["ms_per_eval"])
    res = {"max_leaf": best["max_leaf"], "target_size": best["max_leaf"], "group_size": group_size,
           "ms_per_eval": best["ms_per_eval"], "rms_error": best["rms_error"], "table": table,
           "err_budget": err_budget, "theta": theta}
    if use_cache:
        cache[key] = res
        try:
            os.makedirs(os.path.dirname(CACHE), exist_ok=True)
            json.dump(cache, open(CACHE, "w"), indent=1)
        except OSError:
            pass
    return res
