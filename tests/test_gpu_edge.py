"""Edge cases of the GPU path against the oracle: one particle, coincident
particles (leaves at the maximum depth holding more than max_leaf, and r = 0
pairs without softening), collinear particles, a system far from the origin,
a very small one, and a very large max_leaf.  Build bit for bit, walk within
the usual tolerances, interaction counts equal."""
import numpy as np
import pytest

import bhg
from helpers import cube, rel_error
from oracle import PARTICLE, Params, soa
from test_gpu_parity import _oracle_build

pytestmark = pytest.mark.gpu


def one():
    p = np.zeros(1, PARTICLE)
    p["mass"], p["pos"] = 2.0, [[0.3, -0.2, 0.1]]
    return p


def coincident():
    p = cube(1000, 31)
    p["pos"][:200] = [1.25, -3.5, 2.0]  # 200 at one point: a depth-21 leaf
    p["pos"][200:203] = [-7.0, 7.0, 7.0]
    return p


def collinear():
    p = cube(3000, 32)
    p["pos"][:, 1:] = 0.0
    return p


def far():
    return cube(4000, 33, spread=1.0, centre=(1e6, -1e6, 5e5))


def tiny():
    return cube(3000, 34, spread=1e-9, centre=(1.0, 1.0, 1.0))


def tracers():
    """Massless particles among massive ones, and a clump made only of them:
    its nodes have zero mass, so the reference's centre of mass is 0/0 (NaN)
    there, and such nodes are opened, never accepted."""
    p = cube(3000, 36)
    p["mass"][::3] = 0.0
    p["pos"][:300] = np.random.default_rng(7).normal(0, 0.01, (300, 3)) + [6.0, 6.0, -6.0]
    p["mass"][:300] = 0.0
    return p


CASES = [
    # name, particles, max_leaf, group_size, target_size, theta, eps2
    ("one", one, 16, 256, 16, 0.5, 1e-4),
    ("coincident", coincident, 8, 256, 16, 0.5, 1e-4),
    ("coincident_nosoft", coincident, 8, 256, 16, 0.5, 0.0),
    ("collinear", collinear, 16, 256, 16, 0.5, 1e-6),
    ("far", far, 16, 256, 16, 0.6, 1e-6),
    ("tiny", tiny, 16, 256, 16, 0.5, 1e-22),
    ("big_leaf", lambda: cube(5000, 35), 200, 256, 0, 0.5, 1e-4),
    ("tracers", tracers, 8, 256, 16, 0.5, 1e-4),
]


@pytest.mark.parametrize("name,make,max_leaf,gs,ts,theta,eps2", CASES, ids=[c[0] for c in CASES])
def test_edge_case_matches_oracle(gpu, oracle, name, make, max_leaf, gs, ts, theta, eps2):
    parts = make()
    dom, sk, perm, mp, t = _oracle_build(oracle, parts, max_leaf)
    gpu.upload(parts)
    gpu.build_tree(max_leaf, gs)
    gpu.compute_multipoles()
    assert np.array_equal(gpu.export(bhg.EXPORT_KEYS), sk)
    assert np.array_equal(gpu.export(bhg.EXPORT_PERM), perm)
    g = gpu.tree()
    n = t["n"]
    assert g["n"] == n
    for k in ("begin", "count", "first_child", "nchild", "leaf", "depth"):
        assert np.array_equal(g[k], t[k][:n]), k
    for k in ("center", "hw", "mass", "com", "iab"):
        assert np.array_equal(g[k], np.asarray(t[k][:n]), equal_nan=True), k
    tg = oracle.targets(t, ts, gs)
    racc, counts = oracle.walk(t, tg, soa(mp), [Params(theta, eps2, 1.0, 1)] * len(tg))
    for precision, tol in ((bhg.PRECISION_FP64, 1e-12), (bhg.PRECISION_SPLIT, 1e-5)):
        gpu.upload(parts)
        gpu.stats(reset=True)
        gpu.build_tree(max_leaf, gs)
        gpu.compute_multipoles()
        acc = gpu.walk_forces(bhg.Context.params(theta, eps2, 1.0, True, precision), ts)
        st = gpu.stats()
        assert (st["pp"], st["pc"]) == (int(counts[0]), int(counts[1]))
        assert np.all(np.isfinite(acc))
        if np.any(racc != 0):
            assert rel_error(acc, racc) <= tol
        else:
            assert np.all(acc == 0)


def test_bounded_wait_gives_up_and_context_survives(oracle):
    """The sorts' and scans' look-back wait on a predecessor tile that never
    publishes (a flag nothing sets) gives up after its poll limit: the kernel
    finishes, the status bit comes back as BHG_EDEVICE naming the wait, and
    the context then steps particles normally.  With the predecessor
    published the same wait returns the full prefix."""
    with bhg.Context(device=0) as ctx:
        r, pre = ctx.selftest_wait(True, 1000)
        assert r == bhg.OK and pre == 8
        r, _ = ctx.selftest_wait(False, 1000)
        assert r == bhg.EDEVICE
        assert "bounded wait" in ctx.last_error()
        assert ctx.device_status() == 0  # cleared: the next step starts clean
        parts = cube(2000, 4)
        out, _, _ = oracle.step(parts, theta=0.5, eps2=1e-6, max_leaf=8, group_size=64, target_size=0)
        ctx.upload(parts)
        ctx.step(bhg.Context.params(0.5, 1e-6, 1.0, True, bhg.PRECISION_FP64), 8, 64, 0, 0.0, 0.0)
        assert np.array_equal(ctx.download()["id"], out["id"])
        for bad in (0, (1 << 20) + 1):
            r, _ = ctx.selftest_wait(False, bad)
            assert r == bhg.EINVAL
