"""Continuous batching on the GPU: systems joining and leaving a resident
set, device-generated initial conditions, and the request loop.  A request
served in a changing batch must end bit for bit where it ends alone."""
import numpy as np
import pytest

import bhg
from bhg import serve

pytestmark = pytest.mark.gpu

G_MAX_LEAF, G_GROUP = 16, 256


def run_alone(req, precision):
    """The request by itself: its own context, the same schedule."""
    with bhg.Context(device=0) as ctx:
        ctx.add_generated(req.spheres(), req.seed, id0=0)
        fp = bhg.Context.params(0.5, req.eps ** 2, 1.0, True, precision)
        for e in range(req.steps + 1):
            kick = req.dt / 2 if e in (0, req.steps) else req.dt
            drift = 0.0 if e == req.steps else req.dt
            ctx.set_system_params(theta=[req.theta], eps2=[req.eps ** 2], kick_dt=[kick], drift_dt=[drift])
            ctx.step_systems(fp, G_MAX_LEAF, G_GROUP, G_MAX_LEAF)
        return ctx.download()


@pytest.mark.parametrize("precision", [bhg.PRECISION_SPLIT, bhg.PRECISION_FP64])
def test_served_request_equals_request_alone(precision):
    reqs = [serve.Request(i, 0.0, "plummer" if i % 2 else "merger", n, steps, theta, 1000 + i)
            for i, (n, steps, theta) in enumerate([(9000, 4, 0.5), (5000, 2, 0.7), (12000, 3, 0.4),
                                                   (7000, 5, 0.5), (3000, 2, 0.7)])]
    # room for about two requests at a time: later ones join as earlier leave
    srv = serve.Server(hbm_budget=22000 * serve.BYTES_PER_PARTICLE, keep_results=True, precision=precision)
    rep = srv.run(reqs, realtime=False)
    srv.close()
    assert rep["completed"] == len(reqs) and rep["in_flight"] == 0
    assert rep["particle_steps"] == sum(r.n * r.steps for r in reqs)
    for r in reqs:
        got, want = srv.results[r.rid], run_alone(r, precision)
        assert got.tobytes() == want.tobytes(), f"request {r.rid} differs from its run alone"


def test_device_generator_distribution():
    n = 200_000
    with bhg.Context(device=0) as ctx:
        ctx.add_generated([dict(n=n, a=1.0, mass=1.0)], seed=12345, id0=7)
        p = ctx.download()
        ctx.add_generated([dict(n=n, a=1.0, mass=1.0)], seed=12345, id0=7)
        ctx.add_generated([dict(n=n, a=1.0, mass=1.0)], seed=12346, id0=7)
        q = ctx.download()
    assert np.array_equal(p["id"], np.arange(7, 7 + n))
    assert q[n:2 * n].tobytes() == p.tobytes()  # the seed is the initial conditions
    assert not np.array_equal(q[2 * n:]["pos"], p["pos"])
    r = np.linalg.norm(p["pos"], axis=1)
    assert r.max() < 10.0
    assert abs(p["mass"].sum() - 1.0) < 1e-12
    # half-mass radius of a Plummer sphere: a / sqrt(2^(2/3) - 1)
    assert abs(np.median(r) - 1.0 / np.sqrt(2 ** (2 / 3) - 1)) < 0.02
    # kinetic energy 3 pi / 64 (G = M = a = 1; the 10a truncation moves it < 1%)
    ke = 0.5 * np.sum(p["mass"] * np.sum(p["vel"] ** 2, axis=1))
    assert abs(ke / (3 * np.pi / 64) - 1.0) < 0.02
    # the host generator draws the same distribution
    h = bhg.plummer(n, 99)[0]
    rh = np.linalg.norm(h["pos"], axis=1)
    assert abs(np.median(rh) - np.median(r)) < 0.02


def test_generated_merger():
    n = 60_000
    req = serve.Request(0, 0.0, "merger", n, 1, 0.5, 77)
    with bhg.Context(device=0) as ctx:
        ctx.add_generated(req.spheres(), req.seed, id0=0)
        p = ctx.download()
    assert np.array_equal(p["id"], np.arange(n))
    a, b = p[: n // 2], p[n // 2:]
    assert abs(np.median(a["pos"][:, 0]) + 5.0) < 0.05 and abs(np.median(b["pos"][:, 0]) - 5.0) < 0.05
    assert abs(a["vel"][:, 0].mean() - 0.15) < 0.02 and abs(b["vel"][:, 0].mean() + 0.15) < 0.02
    assert abs(a["mass"].sum() - 1.0) < 1e-12 and abs(b["mass"].sum() - 1.0) < 1e-12
    # the smaller sphere (a = 0.5) is twice as compact
    ra = np.median(np.linalg.norm(a["pos"] - (-5.0, 0, 0), axis=1))
    rb = np.median(np.linalg.norm(b["pos"] - (5.0, 0, 0), axis=1))
    assert abs(ra / rb - 2.0) < 0.1


def test_add_and_remove_keep_the_others():
    rng = np.random.default_rng(4)
    systems = [bhg.plummer(int(n), int(s))[0] for n, s in zip(rng.integers(2000, 9000, 4), rng.integers(1, 1 << 40, 4))]
    fp = bhg.Context.params(0.5, 1e-4, 1.0, True, bhg.PRECISION_SPLIT)
    with bhg.Context(device=0) as ctx:
        hs = [ctx.add_system(s) for s in systems]
        assert list(ctx.system_ids()) == hs and len(set(hs)) == 4
        assert ctx.n == sum(len(s) for s in systems)
        # remove the second and the last: the removed come back as they were
        gone = ctx.remove_systems([hs[3], hs[1]], want=True, sizes=[len(systems[3]), len(systems[1])])
        assert gone[0].tobytes() == systems[3].tobytes() and gone[1].tobytes() == systems[1].tobytes()
        assert list(ctx.system_ids()) == [hs[0], hs[2]]
        assert ctx.download().tobytes() == np.concatenate([systems[0], systems[2]]).tobytes()
        # a step of what is left equals a step of those systems uploaded fresh
        ctx.set_system_params(theta=[0.5, 0.5], eps2=[1e-4, 1e-4], kick_dt=[0.01, 0.01], drift_dt=[0.01, 0.01])
        ctx.step_systems(fp, 16, 256, 16)
        got = ctx.download()
        h5 = ctx.add_system(systems[1])
        assert list(ctx.system_ids()) == [hs[0], hs[2], h5]
    with bhg.Context(device=0) as ref:
        ref.upload_systems([systems[0], systems[2]])
        ref.set_system_params(theta=[0.5, 0.5], eps2=[1e-4, 1e-4], kick_dt=[0.01, 0.01], drift_dt=[0.01, 0.01])
        ref.step_systems(fp, 16, 256, 16)
        assert ref.download().tobytes() == got.tobytes()


def test_add_beyond_budget_leaves_the_resident_systems():
    sysA = bhg.plummer(20000, 5)[0]
    with bhg.Context(device=0, hbm_budget=40000 * serve.BYTES_PER_PARTICLE) as ctx:
        h = ctx.add_system(sysA)
        with pytest.raises(bhg.BhgError) as e:
            ctx.add_generated([dict(n=400000, a=1.0, mass=1.0)], seed=3)
        assert e.value.code == bhg.ENOMEM
        assert list(ctx.system_ids()) == [h]
        assert ctx.download().tobytes() == sysA.tobytes()
        fp = bhg.Context.params(0.5, 1e-4, 1.0, True, bhg.PRECISION_SPLIT)
        ctx.set_system_params(theta=[0.5], eps2=[1e-4], kick_dt=[0.01], drift_dt=[0.01])
        ctx.step_systems(fp, 16, 256, 16)  # still usable
        got = ctx.download()
    with bhg.Context(device=0) as ref:
        ref.upload(sysA)
        ref.step(fp, 16, 256, 16, 0.01, 0.01)
        assert ref.download().tobytes() == got.tobytes()


def test_text_request_served_with_snapshot(oracle):
    """A request whose initial state arrives as CSV text (parsed on the device)
    and whose final state leaves as a VTK snapshot (formatted on the device)
    ends where the same text stepped alone ends."""
    from text_cases import csv_text

    parts, _ = bhg.plummer(6000, 21)
    text = csv_text(parts, 3, styles=(0, 1))
    treq = serve.Request(100, 0.0, "plummer", len(parts), 3, 0.6, 0, text=text, snapshot=True)
    others = [serve.Request(i, 0.0, "merger", 5000, 2 + i, 0.5, 40 + i) for i in range(3)]
    srv = serve.Server(hbm_budget=1e10, keep_results=True)
    rep = srv.run([others[0], treq, *others[1:]], realtime=False)
    srv.close()
    assert rep["completed"] == 4
    with bhg.Context(device=0) as ctx:
        ctx.upload_csv(text)
        fp = bhg.Context.params(0.5, treq.eps ** 2, 1.0, True, bhg.PRECISION_SPLIT)
        for e in range(treq.steps + 1):
            kick = treq.dt / 2 if e in (0, treq.steps) else treq.dt
            drift = 0.0 if e == treq.steps else treq.dt
            ctx.set_system_params(theta=[treq.theta], eps2=[treq.eps ** 2], kick_dt=[kick], drift_dt=[drift])
            ctx.step_systems(fp, G_MAX_LEAF, G_GROUP, G_MAX_LEAF)
        alone = ctx.download()
    assert srv.results[100].tobytes() == alone.tobytes()
    assert srv.snapshots[100] == oracle.write_vtk(alone)


@pytest.mark.parametrize("precision", [bhg.PRECISION_SPLIT, bhg.PRECISION_FP64])
def test_suspended_request_resumes_bit_for_bit(precision):
    """Suspend (state to the host) and resume (state back as a new system)
    in the middle of the schedule: the request ends where it ends without
    the interruption."""
    reqs = [serve.Request(i, 0.0, "merger" if i % 2 else "plummer", 6000 + 1000 * i, 4, 0.5, 500 + i)
            for i in range(3)]
    srv = serve.Server(hbm_budget=1e10, keep_results=True, precision=precision)
    for r in reqs:
        srv.admit(r, 0.0)
    srv.tick(), srv.tick()
    srv.suspend(1)
    srv.tick()  # the others move on without it
    rep = srv.run([], realtime=False)
    srv.close()
    assert rep["completed"] == 3
    for r in reqs:
        assert srv.results[r.rid].tobytes() == run_alone(r, precision).tobytes()


def test_pipeline_equals_one_context():
    """Systems stepped through three contexts with asynchronous steps and
    downloads from pinned memory come back as one context returns them."""
    import torch

    from bhg.pipeline import Pipeline

    systems = [bhg.plummer(n, 300 + i)[0] for i, n in enumerate((3000, 9000, 1500, 20000, 6000, 700, 12000))]
    counts = [len(s) for s in systems]
    th = np.array([0.5, 0.6, 0.4, 0.5, 0.7, 0.5, 0.5])
    e2 = np.array([1e-4, 1e-4, 4e-4, 1e-4, 1e-4, 2.5e-5, 1e-4])
    kick, drift = np.full(7, 0.01), np.full(7, 0.02)
    fp = bhg.Context.params(0.5, 1e-4, 1.0, True, bhg.PRECISION_SPLIT)
    with bhg.Context(device=0) as one:
        one.upload_systems(systems)
        for _ in range(2):
            one.set_system_params(theta=th, eps2=e2, kick_dt=kick, drift_dt=drift)
            one.step_systems(fp, 16, 256, 16)
        want = one.download()
    n = sum(counts)
    buf = torch.empty(n * bhg.PARTICLE.itemsize, dtype=torch.uint8, pin_memory=True)
    host = np.frombuffer(buf.numpy(), dtype=bhg.PARTICLE)
    host[:] = np.concatenate(systems)
    with Pipeline(counts, parts=3) as pl:
        assert len(pl.ctxs) == 3
        for _ in range(2):
            pl.step(buf.data_ptr(), fp, 16, 256, 16, th, e2, kick, drift)
    assert host.tobytes() == want.tobytes()


def test_async_step_reports_node_overflow():
    """An asynchronous evaluation whose octree outgrows the node slots is
    reported by bhg_sync as EAGAIN with the slots grown; run again it gives
    what the blocking step gives."""
    from helpers import cube

    parts = cube(4000, 12, spread=10.0)
    parts["pos"] = np.repeat(parts["pos"][::8], 8, axis=0) + np.random.default_rng(3).uniform(-1e-7, 1e-7, (4000, 3))
    fp = bhg.Context.params(0.5, 1e-8, 1.0, True, bhg.PRECISION_FP64)
    with bhg.Context(device=0) as ctx:
        ctx.upload(parts)
        ctx.set_system_params(theta=[0.5], eps2=[1e-8], kick_dt=[0.01], drift_dt=[0.01])
        ctx.step_systems_async(fp, 1, 64, 0)
        with pytest.raises(bhg.BhgError) as e:
            ctx.sync()
        assert e.value.code == bhg.EAGAIN
        assert ctx.download().tobytes() == parts.tobytes()  # nothing moved
        for _ in range(8):  # each overflow grows the slots past the level it reached
            ctx.step_systems_async(fp, 1, 64, 0)
            try:
                ctx.sync()
                break
            except bhg.BhgError as again:
                assert again.code == bhg.EAGAIN
        got = ctx.download()
    with bhg.Context(device=0) as ref:
        ref.upload(parts)
        ref.step(fp, 1, 64, 0, 0.01, 0.01)
        assert ref.download().tobytes() == got.tobytes()


def test_reserve_then_add_equals_growth():
    """bhg_reserve sizes the buffers up front: systems added afterwards step
    to the same bits as in a context that grew for them; past the HBM budget
    the reservation is a clean ENOMEM."""
    systems = [bhg.plummer(n, 400 + i)[0] for i, n in enumerate((5000, 12000, 3000))]
    fp = bhg.Context.params(0.5, 1e-4, 1.0, True, bhg.PRECISION_SPLIT)
    out = []
    for reserve in (True, False):
        with bhg.Context(device=0) as ctx:
            if reserve:
                ctx.reserve(40000, 8)
            for s in systems:
                ctx.add_system(s)
            ctx.set_system_params(theta=np.full(3, 0.5), eps2=np.full(3, 1e-4), kick_dt=np.full(3, 0.01),
                                  drift_dt=np.full(3, 0.01))
            ctx.step_systems(fp, 16, 256, 16)
            out.append(ctx.download())
    assert out[0].tobytes() == out[1].tobytes()
    with bhg.Context(device=0, hbm_budget=64 << 20) as small:
        with pytest.raises(bhg.BhgError) as e:
            small.reserve(10_000_000, 8)
        assert e.value.code == bhg.ENOMEM
        small.add_system(systems[0])  # still usable
        assert small.download().tobytes() == systems[0].tobytes()
