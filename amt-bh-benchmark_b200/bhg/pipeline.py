"""Many systems stepped end to end from pinned host memory through several
contexts, so that one context's host<->device copies overlap the others'
evaluations.

Each context (its own CUDA stream) holds a contiguous part of the systems.
A step uploads every part, enqueues its evaluation (bhg_step_systems_async)
and its download (bhg_download_async), then waits for all (bhg_sync).  A
system's result does not depend on the systems evaluated beside it, so the
split changes no bits: the particles come back as one context stepping all
systems would return them.
"""
import ctypes as C

import numpy as np

from . import PARTICLE, Context


def split_systems(counts, parts):
    """Contiguous runs of systems with about equal particle totals."""
    counts = np.asarray(counts, np.int64)
    parts = max(1, min(int(parts), len(counts)))
    ends = np.cumsum(counts)
    cuts = [0]
    for k in range(1, parts):
        i = int(np.searchsorted(ends, ends[-1] * k / parts))
        cuts.append(min(max(i + 1, cuts[-1] + 1), len(counts) - (parts - k)))
    cuts.append(len(counts))
    return [(cuts[k], cuts[k + 1]) for k in range(parts)]


class Pipeline:
    """`counts`: particles per system, back to back in the host buffer the
    steps read and write (pinned, PARTICLE records)."""

    def __init__(self, counts, parts=4, device=0, hbm_budget=0, walk_group=0):
        self.counts = np.asarray(counts, np.uint64)
        self.runs = split_systems(self.counts, parts)
        offs = np.concatenate([[0], np.cumsum(self.counts.astype(np.int64))])
        self.ctxs = [Context(device=device, hbm_budget=hbm_budget) for _ in self.runs]
        for c in self.ctxs:
            if walk_group:
                c.set_walk_shape(walk_group)
        self.spans = [(int(offs[a]), int(offs[b]), np.ascontiguousarray(self.counts[a:b])) for a, b in self.runs]

    def step(self, host_ptr, fp, max_leaf, group_size, target_size, theta, eps2, kick_dt, drift_dt):
        """One evaluation of every system, particles read from and written back
        to the pinned host buffer at host_ptr; per-system parameters as arrays
        over all systems (or scalars)."""
        rec = PARTICLE.itemsize
        ns = len(self.counts)
        full = [np.broadcast_to(np.asarray(v, np.float64), (ns,)) for v in (theta, eps2, kick_dt, drift_dt)]
        for ctx, (a, b), (p0, _, cnt) in zip(self.ctxs, self.runs, self.spans):
            ctx._ck(ctx.L.bhg_upload_systems(ctx.h, C.c_void_p(host_ptr + p0 * rec), cnt.ctypes.data, len(cnt)))
            ctx.n = int(cnt.sum())
            ctx.set_system_params(*(np.ascontiguousarray(v[a:b]) for v in full))
            ctx.step_systems_async(fp, max_leaf, group_size, target_size)
        for ctx, (p0, _, _) in zip(self.ctxs, self.spans):
            ctx.download_async(host_ptr + p0 * rec)
        err = None
        for ctx in self.ctxs:  # wait for every context, then report the first failure
            try:
                ctx.sync()
            except Exception as e:  # noqa: BLE001 - re-raised below
                err = err or e
        if err is not None:
            raise err

    def close(self):
        for c in self.ctxs:
            c.close()
        self.ctxs = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
