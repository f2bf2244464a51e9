"""The serving loop's host logic (no GPU): the request stream, admission
under the memory budget, and preemption when a batch does not fit."""
import numpy as np

from bhg import serve


def test_poisson_stream_matches_its_spec():
    reqs = serve.poisson_stream(rate=200, duration=60, seed=5)
    assert 11000 < len(reqs) < 13000
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) > 0) and arr[-1] < 60
    n = np.array([r.n for r in reqs])
    assert n.min() >= 4096 and n.max() <= 2097152
    assert abs(np.mean(np.log(n)) - 0.5 * (np.log(4096) + np.log(2097152))) < 0.1
    steps = np.array([r.steps for r in reqs])
    assert steps.min() >= 16 and steps.max() <= 256
    assert {r.theta for r in reqs} == {0.4, 0.5, 0.7}
    kinds = [r.kind for r in reqs]
    assert 0.45 < kinds.count("merger") / len(kinds) < 0.55
    assert len({r.seed for r in reqs}) == len(reqs)
    again = serve.poisson_stream(rate=200, duration=60, seed=5)
    assert [r.seed for r in again] == [r.seed for r in reqs]


def test_request_spheres():
    assert serve.Request(0, 0, "plummer", 1001, 4, 0.5, 1).spheres() == [dict(n=1001, a=1.0, mass=1.0)]
    m = serve.Request(0, 0, "merger", 1001, 4, 0.5, 1).spheres()
    assert [s["n"] for s in m] == [500, 501] and m[0]["centre"][0] == -m[1]["centre"][0]


class _FakeContext:
    """Stands in for the device context: systems are only sizes, and a step
    of more than `limit` resident particles fails like a full device."""

    limit = 0

    def __init__(self, device=0, hbm_budget=0):
        self.sizes = {}
        self.next = 1
        self.reserved = None

    def reserve(self, particles, systems):
        self.reserved = (particles, systems)

    @staticmethod
    def params(*a):
        return a

    def add_generated(self, spheres, seed, id0=0):
        h = self.next
        self.next += 1
        self.sizes[h] = sum(s["n"] for s in spheres)
        return h

    def set_system_params(self, **kw):
        assert all(len(v) == len(self.sizes) for v in kw.values())

    def step_systems(self, fp, max_leaf, group_size, target_size):
        if sum(self.sizes.values()) > self.limit:
            raise serve.BhgError(serve.ENOMEM, "device out of memory")

    def add_system(self, parts):
        h = self.next
        self.next += 1
        self.sizes[h] = len(parts)
        return h

    def remove_systems(self, handles, want=False, sizes=None):
        out = [np.zeros(self.sizes[h]) for h in handles] if want else None
        for h in handles:
            del self.sizes[h]
        return out

    def close(self):
        pass


def test_server_preempts_when_the_batch_does_not_fit(monkeypatch):
    monkeypatch.setattr(serve, "Context", _FakeContext)
    monkeypatch.setattr(_FakeContext, "limit", 250_000)
    reqs = [serve.Request(i, 0.0, "plummer" if i % 2 else "merger", 100_000, 3 + i % 4, 0.5, i) for i in range(6)]
    srv = serve.Server(hbm_budget=1e12)  # the admission estimate alone lets everything in
    rep = srv.run(reqs, realtime=False)
    assert rep["completed"] == 6 and rep["in_flight"] == 0 and rep["queued"] == 0
    assert rep["preempted"] > 0
    # work thrown away by a preemption is not credited
    assert rep["particle_steps"] == sum(r.n * r.steps for r in reqs)
    assert len(srv.step_latency_ms) == sum(r.steps for r in reqs)


def test_server_admission_budget(monkeypatch):
    monkeypatch.setattr(serve, "Context", _FakeContext)
    monkeypatch.setattr(_FakeContext, "limit", 1 << 40)
    reqs = [serve.Request(i, 0.0, "plummer", 50_000, 4, 0.7, i) for i in range(5)]
    budget = 2.5 * 50_000 * serve.BYTES_PER_PARTICLE
    srv = serve.Server(hbm_budget=budget)
    assert srv.admit(reqs[0], 0.0) and srv.admit(reqs[1], 0.0) and not srv.admit(reqs[2], 0.0)
    srv = serve.Server(hbm_budget=budget)
    rep = srv.run(reqs, realtime=False)
    assert rep["completed"] == 5 and rep["particle_steps"] == 5 * 50_000 * 4
    assert rep["preempted"] == 0


def test_server_schedule_kicks(monkeypatch):
    """Each request sees the reference's schedule: (dt/2, dt), (dt, dt) x
    (steps - 1), (dt/2, 0)."""
    monkeypatch.setattr(serve, "Context", _FakeContext)
    monkeypatch.setattr(_FakeContext, "limit", 1 << 40)
    seen = []
    orig = _FakeContext.set_system_params

    def record(self, **kw):
        orig(self, **kw)
        seen.append((kw["kick_dt"][0], kw["drift_dt"][0]))

    monkeypatch.setattr(_FakeContext, "set_system_params", record)
    dt = 1.0 / 128
    serve.Server(hbm_budget=1e12).run([serve.Request(0, 0.0, "plummer", 1000, 3, 0.5, 7, dt=dt)], realtime=False)
    assert seen == [(dt / 2, dt), (dt, dt), (dt, dt), (dt / 2, 0.0)]


def test_server_batch_cap(monkeypatch):
    monkeypatch.setattr(serve, "Context", _FakeContext)
    monkeypatch.setattr(_FakeContext, "limit", 1 << 40)
    reqs = [serve.Request(i, 0.0, "plummer", 40_000, 2, 0.5, i) for i in range(4)]
    srv = serve.Server(hbm_budget=1e12, max_batch_particles=100_000)
    assert srv.admit(reqs[0], 0.0) and srv.admit(reqs[1], 0.0) and not srv.admit(reqs[2], 0.0)
    rep = serve.Server(hbm_budget=1e12, max_batch_particles=100_000).run(reqs, realtime=False)
    assert rep["completed"] == 4


def test_suspended_request_resumes_where_it_stopped(monkeypatch):
    monkeypatch.setattr(serve, "Context", _FakeContext)
    monkeypatch.setattr(_FakeContext, "limit", 1 << 40)
    reqs = [serve.Request(i, 0.0, "plummer", 1000 * (i + 1), 5, 0.5, i) for i in range(3)]
    srv = serve.Server(hbm_budget=1e12)
    for r in reqs:
        srv.admit(r, 0.0)
    srv.tick(), srv.tick()
    ck = srv.suspend(1)
    assert ck.evals_done == 2 and len(ck.particles) == 2000 and len(srv.active) == 2
    rep = srv.run([], realtime=False)  # the suspended request is resumed, not restarted
    assert rep["completed"] == 3
    assert rep["particle_steps"] == sum(r.n * r.steps for r in reqs)
    assert len(srv.step_latency_ms) == sum(r.steps for r in reqs)


def test_cancel_active_and_queued(monkeypatch):
    monkeypatch.setattr(serve, "Context", _FakeContext)
    monkeypatch.setattr(_FakeContext, "limit", 1 << 40)
    reqs = [serve.Request(i, 0.0, "plummer", 1000, 4, 0.5, i) for i in range(4)]
    budget = 2.5 * 1000 * serve.BYTES_PER_PARTICLE  # two at a time
    srv = serve.Server(hbm_budget=budget)
    srv.admit(reqs[0], 0.0), srv.admit(reqs[1], 0.0)
    srv.tick()
    srv.cancel(0)  # admitted
    srv.cancel(3)  # still queued
    rep = srv.run(reqs[2:], realtime=False)
    assert rep["cancelled"] == 2 and rep["completed"] == 2
    assert srv.ctx.sizes == {}


def test_pipeline_split_is_contiguous_and_balanced():
    from bhg.pipeline import split_systems

    assert split_systems([10, 10, 10, 10], 2) == [(0, 2), (2, 4)]
    assert split_systems([10, 10, 10, 10], 3) == [(0, 2), (2, 3), (3, 4)]
    assert split_systems([100, 1, 1, 1], 2) == [(0, 1), (1, 4)]
    assert split_systems([5, 5], 8) == [(0, 1), (1, 2)]
    runs = split_systems(list(range(1, 101)), 4)
    assert runs[0][0] == 0 and runs[-1][1] == 100
    assert all(a < b for a, b in runs) and all(runs[i][1] == runs[i + 1][0] for i in range(3))
