"""Continuous-batching request loop over the B200 Barnes-Hut path.

Each request is one independent simulation - a Plummer sphere or a
two-sphere merger of N particles, advanced `steps` leapfrog steps (the
reference's schedule, main.cc:199-246: a (dt/2, dt) evaluation, steps-1
(dt, dt) evaluations, a closing (dt/2, 0) one) at its own theta.  Requests
join one batched context as they arrive and memory allows (their initial
conditions are generated on the device from the request seed), every tick
advances every admitted request by one evaluation in one segmented build +
walk, and finished requests leave at the end of the tick.  So requests that
arrive while others are on the GPU start at the next tick: their work
overlaps with the others' on the device.

A system's result does not depend on what it was batched with (each
system's tree, walk and sums only ever touch its own particles), which the
GPU tests check bit for bit against running the request alone.
"""
from __future__ import annotations

import dataclasses
import time

import numpy as np

from . import ENOMEM, PRECISION_SPLIT, BhgError, Context

#: device bytes per particle of a resident system: state and staging copy
#: (128), sources (32), sort keys and values (24), marks (4), ~0.45 node
#: slots of 264 bytes (~119), rounded up
BYTES_PER_PARTICLE = 320
RESERVED_SYSTEMS = 4096  # per-system tables sized up front by Server


@dataclasses.dataclass
class Request:
    rid: int
    arrival: float  # seconds after the start
    kind: str  # "plummer" or "merger"
    n: int
    steps: int
    theta: float
    seed: int
    eps: float = 0.01
    dt: float = 1.0 / 128
    text: bytes | None = None  # initial conditions as CSV (read_csv's format) instead of a generator
    snapshot: bool = False  # return the final state as write_vtk's text

    def spheres(self):
        """The request's initial conditions as device-generated spheres: one
        Plummer sphere (M = a = 1), or two (M = 1 each, a = 1 and 0.5) 10
        apart approaching at 0.3."""
        if self.kind == "plummer":
            return [dict(n=self.n, a=1.0, mass=1.0)]
        half = self.n // 2
        return [dict(n=half, a=1.0, mass=1.0, centre=(-5.0, 0, 0), bulk=(0.15, 0, 0)),
                dict(n=self.n - half, a=0.5, mass=1.0, centre=(5.0, 0, 0), bulk=(-0.15, 0, 0))]


def poisson_stream(rate=200.0, duration=60.0, seed=5, nmin=4096, nmax=2097152, smin=16, smax=256,
                   thetas=(0.4, 0.5, 0.7)):
    """Requests with Poisson arrivals: kind 50/50, N log-uniform in [nmin, nmax],
    steps uniform in [smin, smax], theta from `thetas`, per-request seed from
    (stream seed, request id)."""
    rng = np.random.default_rng(seed)
    out, t, rid = [], 0.0, 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            return out
        kind = "plummer" if rng.random() < 0.5 else "merger"
        n = int(np.rint(np.exp(rng.uniform(np.log(nmin), np.log(nmax)))))
        steps = int(rng.integers(smin, smax + 1))
        theta = float(thetas[int(rng.integers(len(thetas)))])
        rseed = int(np.random.SeedSequence([seed, rid]).generate_state(1, np.uint64)[0])
        out.append(Request(rid, t, kind, n, steps, theta, rseed))
        rid += 1


@dataclasses.dataclass
class _Active:
    req: Request
    handle: int
    evals_done: int = 0
    admitted_at: float = 0.0
    counted: int = 0  # particle-steps credited so far


@dataclasses.dataclass
class Checkpoint:
    """A request's state between two evaluations: its particles (storage
    order) and how far along its schedule it is."""
    particles: np.ndarray
    evals_done: int
    counted: int


class Server:
    """The request loop.  hbm_budget caps the admitted particles (about
    BYTES_PER_PARTICLE each); max_leaf/group_size are the walk's sizes."""

    def __init__(self, device=0, hbm_budget=150e9, max_leaf=16, group_size=256, precision=PRECISION_SPLIT,
                 keep_results=False, on_result=None, max_batch_particles=None, walk_group=0):
        """keep_results: store each finished request's particles in
        self.results[rid]; on_result(rid, particles): hand them to a caller
        instead.  With neither, finished requests leave the GPU uncopied.
        max_batch_particles: a second admission cap, on the particles one
        tick evaluates (bounds the per-step latency; None = memory only).
        walk_group: the walk-group particle cap (0 = the library's default)."""
        # the context's own hard limit leaves room for its fixed tables, the
        # buffers' growth slack and the state's second copy while it grows
        self.ctx = Context(device=device, hbm_budget=int(hbm_budget * 1.15) + (512 << 20))
        if walk_group:
            self.ctx.set_walk_shape(walk_group)
        self.budget = hbm_budget
        # the buffers for a full batch up front: admissions then neither
        # allocate nor copy the resident state (without the memory for it
        # they grow as systems join)
        try:
            self.ctx.reserve(int(hbm_budget // BYTES_PER_PARTICLE), RESERVED_SYSTEMS)
        except BhgError as e:
            if e.code != ENOMEM:
                raise
        self.max_batch = max_batch_particles
        self.max_leaf, self.group_size, self.precision = max_leaf, group_size, precision
        self.keep_results = keep_results
        self.on_result = on_result
        self.d2h_bytes = 0
        self.particle_evals = 0  # resident particles summed over ticks
        self.system_evals = 0  # resident systems summed over ticks
        self.results = {}
        self.snapshots = {}  # request id -> write_vtk text of its final state
        self.active: list[_Active] = []
        self.requeue: list[Request] = []
        self.tick_ms: list[float] = []
        self._lat: list[tuple[int, float]] = []  # (request id, ms) per request step
        self.particle_steps = 0
        self.completed = 0
        self.admitted = 0
        self.preempted = 0
        self.hold = False  # after a preemption: admit nothing until a request completes
        self.saved: dict[int, Checkpoint] = {}  # suspended requests, resumed at their next admission
        self.cancelled: set[int] = set()
        self.admit_s = 0.0  # wall seconds spent adding systems (admissions, resumptions)
        self.retire_s = 0.0  # wall seconds spent taking finished systems off (with their copies)
        self.n_cancelled = 0

    def close(self):
        self.ctx.close()

    def _resident(self):
        return sum(a.req.n for a in self.active)

    def admit(self, req: Request, now: float) -> bool:
        """Adds the request to the batch if the budget allows (a request alone
        is always tried)."""
        if self.active:
            after = self._resident() + req.n
            if self.hold or after * BYTES_PER_PARTICLE > self.budget or (self.max_batch and after > self.max_batch):
                return False
        ck = self.saved.get(req.rid)
        t0 = time.perf_counter()
        try:
            if ck is not None:  # resumed where it was suspended
                h = self.ctx.add_system(ck.particles)
            elif req.text is not None:  # parsed on the device
                h = self.ctx.add_csv(req.text)
            else:
                h = self.ctx.add_generated(req.spheres(), req.seed, id0=0)
        except BhgError as e:
            if e.code == ENOMEM and self.active:  # no room until some request leaves
                return False
            raise
        finally:
            self.admit_s += time.perf_counter() - t0
        if ck is not None:
            del self.saved[req.rid]
            self.active.append(_Active(req, h, ck.evals_done, now, ck.counted))
        else:
            self.active.append(_Active(req, h, 0, now))
            self.admitted += 1
        return True

    def suspend(self, rid) -> Checkpoint:
        """Takes an admitted request off the GPU with its state; it resumes
        from that state (not from its seed) when it is admitted again, which
        run() does as soon as memory allows."""
        a = next(x for x in self.active if x.req.rid == rid)
        parts = self.ctx.remove_systems([a.handle], want=True, sizes=[a.req.n])[0]
        self.active = [x for x in self.active if x is not a]
        ck = Checkpoint(parts, a.evals_done, a.counted)
        self.saved[rid] = ck
        self.requeue.append(a.req)
        return ck

    def cancel(self, rid):
        """Drops a request: off the GPU if admitted, never admitted if queued."""
        self.cancelled.add(rid)
        for a in self.active:
            if a.req.rid == rid:
                self.ctx.remove_systems([a.handle])
                self.active = [x for x in self.active if x is not a]
                self.n_cancelled += 1
                break
        self.saved.pop(rid, None)

    def _preempt(self):
        """Suspends the most recently admitted request (its state is kept and
        it resumes from there) and holds admission until a request completes."""
        self.suspend(self.active[-1].req.rid)
        self.preempted += 1
        self.hold = True

    def tick(self):
        """One evaluation of every admitted request; retires the finished ones.
        Returns the tick's wall milliseconds (None if the batch did not fit and
        a request was sent back to the queue)."""
        if not self.active:
            return 0.0
        k = len(self.active)
        theta = np.array([a.req.theta for a in self.active])
        eps2 = np.array([a.req.eps ** 2 for a in self.active])
        kick = np.empty(k)
        drift = np.empty(k)
        for i, a in enumerate(self.active):
            dt = a.req.dt
            if a.evals_done == 0:
                kick[i], drift[i] = dt / 2, dt
            elif a.evals_done == a.req.steps:
                kick[i], drift[i] = dt / 2, 0.0
            else:
                kick[i], drift[i] = dt, dt
        self.ctx.set_system_params(theta=theta, eps2=eps2, kick_dt=kick, drift_dt=drift)
        # fp gives G, the quadrupole switch and the precision; eps2 > 0 in
        # every system selects the walk without the r^2 = 0 mask
        fp = Context.params(0.5, float(eps2.min()), 1.0, True, self.precision)
        t0 = time.perf_counter()
        try:
            self.ctx.step_systems(fp, self.max_leaf, self.group_size, self.max_leaf)
        except BhgError as e:
            if e.code != ENOMEM or len(self.active) < 2:
                raise
            self._preempt()  # the batch's trees did not fit: the newest request waits
            return None
        ms = (time.perf_counter() - t0) * 1000.0  # step_systems returns once the step is done
        self.tick_ms.append(ms)
        self.particle_evals += self._resident()
        self.system_evals += k
        done = []
        for i, a in enumerate(self.active):
            if drift[i] != 0.0:  # the closing half-kick completes the last step
                self.particle_steps += a.req.n
                a.counted += a.req.n
                self._lat.append((a.req.rid, ms))
            a.evals_done += 1
            if a.evals_done == a.req.steps + 1:
                done.append(a)
        if done:
            t1 = time.perf_counter()
            for a in done:  # snapshots are formatted on the device before the systems leave
                if a.req.snapshot:
                    self.snapshots[a.req.rid] = self.ctx.snapshot_vtk(a.handle)
            want = self.keep_results or self.on_result is not None
            parts = self.ctx.remove_systems([a.handle for a in done], want=want, sizes=[a.req.n for a in done])
            for j, a in enumerate(done):
                if parts is None:
                    continue
                self.d2h_bytes += parts[j].nbytes
                if self.keep_results:
                    self.results[a.req.rid] = parts[j]
                if self.on_result is not None:
                    self.on_result(a.req.rid, parts[j])
            self.completed += len(done)
            self.retire_s += time.perf_counter() - t1
            self.hold = False
            gone = {id(a) for a in done}
            self.active = [a for a in self.active if id(a) not in gone]
        return ms

    def run(self, requests, wall_limit=None, realtime=True, log=None):
        """Serves `requests` (sorted by arrival).  realtime: arrivals follow the
        wall clock; otherwise every pending request is offered at each tick.
        Stops when all are done or after wall_limit seconds."""
        pending = list(reversed(requests))  # next arrival last
        start = time.perf_counter()
        while pending or self.active or self.requeue:
            now = time.perf_counter() - start
            if wall_limit is not None and now > wall_limit:
                break
            while self.requeue:
                pending.append(self.requeue.pop())
            while pending and (not realtime or pending[-1].arrival <= now):
                if pending[-1].rid in self.cancelled:
                    pending.pop()
                    self.n_cancelled += 1
                    continue
                if not self.admit(pending[-1], now):
                    break
                pending.pop()
            if not self.active:
                if pending and realtime:
                    time.sleep(max(0.0, min(0.05, pending[-1].arrival - now)))
                continue
            self.tick()
            if log and len(self.tick_ms) % 20 == 0:
                log(self.report(time.perf_counter() - start, len(pending)))
        return self.report(time.perf_counter() - start, len(pending))

    @property
    def step_latency_ms(self):
        """Per-step latency samples: one per request step, the wall time of the
        tick that advanced it."""
        return [ms for _, ms in self._lat]

    def report(self, wall_s, queued=0):
        lat = np.array(self.step_latency_ms) if self._lat else np.zeros(1)
        return {"wall_s": wall_s, "admitted": self.admitted, "completed": self.completed,
                "in_flight": len(self.active), "queued": queued, "preempted": self.preempted,
                "cancelled": self.n_cancelled,
                "ticks": len(self.tick_ms), "tick_s": sum(self.tick_ms) / 1000.0, "admit_s": self.admit_s,
                "retire_s": self.retire_s, "particle_steps": self.particle_steps,
                "particle_steps_per_s": self.particle_steps / wall_s if wall_s > 0 else 0.0,
                "step_latency_ms_p50": float(np.percentile(lat, 50)),
                "step_latency_ms_p99": float(np.percentile(lat, 99)),
                "resident_particles": self._resident()}
