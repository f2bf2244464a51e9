"""GPU parity of every phase against the oracle (oracle/bh_oracle.c), through
the C ABI.  Integer results (keys, order, topology) and the FP64 build
(domain, cell geometry, multipoles) must be bit-identical; forces within
the stated tolerances:

  FP64 walk   vs oracle walk: global relative error <= 1e-12
  split walk  vs oracle walk: global relative error <= 1e-5 (the split-precision gate)
  theta = 0   vs direct sum:  <= 1e-8 (FP64) / 1e-5 (split), as
              test_bh_vs_bruteforce.cc:55-76 requires of the reference
"""
import numpy as np
import pytest

import bhg
from helpers import cube, rel_error
from oracle import Params, soa

pytestmark = pytest.mark.gpu

CASES = [
    # name, particles, max_leaf, group_size, target_size, theta, eps2
    ("cube2000_leaf8", lambda: cube(2000, 4), 8, 64, 0, 0.5, 1e-6),
    ("cube20000_leaf16", lambda: cube(20000, 5), 16, 64, 0, 0.5, 1e-6),
    ("plummer32k_leaf16", lambda: bhg.plummer(32768, 1)[0], 16, 256, 16, 0.5, 1e-4),
    ("cube2000_leaf1_ts32", lambda: cube(2000, 6), 1, 64, 32, 0.5, 1e-6),
    ("cube3000_leaf4_gs1M", lambda: cube(3000, 7), 4, 1 << 20, 0, 0.6, 1e-6),
]


def _oracle_build(oracle, parts, max_leaf):
    dom, bad = oracle.domain(parts)
    assert bad == 0
    keys = oracle.keys(parts, dom)
    perm, sk = oracle.sort(keys)
    mp = parts[perm]
    t = oracle.build(sk, [0], [len(parts)], dom[None], max_leaf, soa(mp))
    return dom, sk, perm, mp, t


@pytest.mark.parametrize("name,make,max_leaf,gs,ts,theta,eps2", CASES, ids=[c[0] for c in CASES])
def test_build_bit_exact(gpu, oracle, name, make, max_leaf, gs, ts, theta, eps2):
    parts = make()
    dom, sk, perm, mp, t = _oracle_build(oracle, parts, max_leaf)
    gpu.upload(parts)
    gpu.build_tree(max_leaf, gs)
    gpu.compute_multipoles()
    assert np.array_equal(gpu.export(bhg.EXPORT_DOMAINS)[0], dom), "domain differs"
    assert np.array_equal(gpu.export(bhg.EXPORT_KEYS), sk), "sorted keys differ"
    assert np.array_equal(gpu.export(bhg.EXPORT_PERM), perm), "sort permutation differs"
    g = gpu.tree()
    n = t["n"]
    assert g["n"] == n, f"node count {g['n']} != {n}"
    for k in ("begin", "count", "first_child", "nchild", "leaf", "depth"):
        assert np.array_equal(g[k], t[k][:n]), f"node {k} differs"
    for k in ("center", "hw", "mass", "com", "iab"):
        assert np.array_equal(g[k], np.asarray(t[k][:n])), f"node {k} not bit-identical"


def test_build_bit_exact_per_level_multipoles(gpu, oracle):
    """Above 393,216 particles the multipoles run one launch per level instead
    of the one-launch upward pass the small cases take: the same bits."""
    parts = bhg.plummer(450000, 12)[0]
    dom, sk, perm, mp, t = _oracle_build(oracle, parts, 16)
    gpu.upload(parts)
    gpu.build_tree(16, 256)
    gpu.compute_multipoles()
    g = gpu.tree()
    n = t["n"]
    assert g["n"] == n
    for k in ("begin", "count", "first_child", "nchild", "leaf", "depth", "center", "hw", "mass", "com", "iab"):
        assert np.array_equal(g[k], np.asarray(t[k][:n])), f"node {k} differs"


@pytest.mark.parametrize("precision,tol", [(bhg.PRECISION_FP64, 1e-12), (bhg.PRECISION_SPLIT, 1e-5)])
@pytest.mark.parametrize("name,make,max_leaf,gs,ts,theta,eps2", CASES, ids=[c[0] for c in CASES])
def test_walk_matches_oracle(gpu, oracle, name, make, max_leaf, gs, ts, theta, eps2, precision, tol):
    parts = make()
    for quad in (True, False):
        dom, sk, perm, mp, t = _oracle_build(oracle, parts, max_leaf)
        tg = oracle.targets(t, ts, gs)
        racc, counts = oracle.walk(t, tg, soa(mp), [Params(theta, eps2, 1.0, int(quad))] * len(tg))
        gpu.upload(parts)
        gpu.stats(reset=True)
        gpu.build_tree(max_leaf, gs)
        gpu.compute_multipoles()
        acc = gpu.walk_forces(bhg.Context.params(theta, eps2, 1.0, quad, precision), ts)
        assert np.array_equal(gpu.export(bhg.EXPORT_TARGETS), tg), "targets differ"
        st = gpu.stats()
        assert (st["pp"], st["pc"]) == (int(counts[0]), int(counts[1])), "interaction counts differ"
        err = rel_error(acc, racc)
        assert err <= tol, f"quad={quad} relative error {err:.3e} > {tol}"
        out = gpu.download()
        assert np.array_equal(out["id"], mp["id"]), "output not in Morton order"


@pytest.mark.parametrize("precision,tol", [(bhg.PRECISION_FP64, 1e-8), (bhg.PRECISION_SPLIT, 1e-5)])
def test_theta0_is_direct_sum(gpu, oracle, precision, tol):
    # test_bh_vs_bruteforce.cc:55-76: theta = 0 degenerates into brute force
    parts = cube(200, 1)
    gpu.upload(parts)
    gpu.build_tree(4, 16)
    gpu.compute_multipoles()
    acc = gpu.walk_forces(bhg.Context.params(0.0, 1e-6, 1.0, True, precision), 0)
    out = gpu.download()
    ref = oracle.direct(soa(out), np.arange(len(out)), 1e-6)
    assert rel_error(acc, ref) <= tol


@pytest.mark.parametrize("precision,tol", [(bhg.PRECISION_FP64, 1e-12), (bhg.PRECISION_SPLIT, 1e-6)])
@pytest.mark.parametrize("max_leaf,theta", [(4, 0.5), (1, 0.7)], ids=["pair", "cell"])
def test_two_body_analytic(gpu, precision, tol, max_leaf, theta):
    """test_force_kernel.cc:17-43 through the whole GPU path: a source of mass
    3 at distance 4 pulls with G m / 16 (G = 2), whether it arrives as a direct
    particle (one leaf) or as an accepted one-particle cell whose second moment
    is zero; softening weakens it."""
    parts = np.zeros(2, dtype=bhg.PARTICLE)
    parts["id"] = [0, 1]
    parts["mass"] = [1.0, 3.0]
    parts["pos"][1] = (4.0, 0.0, 0.0)
    for eps2, mag in ((0.0, 2.0 / 16.0), (4.0, 2.0 * 4.0 / 20.0 ** 1.5)):
        gpu.upload(parts)
        gpu.build_tree(max_leaf, 16)
        gpu.compute_multipoles()
        acc = gpu.walk_forces(bhg.Context.params(theta, eps2, 2.0, True, precision), 0)
        out = gpu.download()
        a0 = acc[out["id"] == 0][0]
        a1 = acc[out["id"] == 1][0]
        assert abs(a0[0] - 3.0 * mag) <= tol * 3.0 * mag and abs(a0[1]) + abs(a0[2]) <= tol * mag
        assert abs(a1[0] + mag) <= tol * mag and abs(a1[1]) + abs(a1[2]) <= tol * mag


@pytest.mark.parametrize("precision", [bhg.PRECISION_FP64, bhg.PRECISION_SPLIT])
def test_quadrupole_beats_monopole(gpu, oracle, precision):
    """test_bh_vs_bruteforce.cc:78-113: two tight clusters 100 apart, theta
    0.6, leaf 4: the quadrupole term lowers the error against the direct sum."""
    parts = np.concatenate([cube(100, 2, spread=1.0, centre=(-50.0, 0.0, 0.0)),
                            cube(100, 3, spread=1.0, centre=(50.0, 0.0, 0.0))])
    parts["id"] = np.arange(200)
    err = {}
    for quad in (False, True):
        gpu.upload(parts)
        gpu.build_tree(4, 64)
        gpu.compute_multipoles()
        acc = gpu.walk_forces(bhg.Context.params(0.6, 1e-6, 1.0, quad, precision), 0)
        out = gpu.download()
        err[quad] = rel_error(acc, oracle.direct(soa(out), np.arange(len(out)), 1e-6))
    assert err[True] < err[False], err


@pytest.mark.parametrize("precision,tol", [(bhg.PRECISION_FP64, 1e-12), (bhg.PRECISION_SPLIT, 1e-5)])
def test_list_overflow_falls_back(oracle, precision, tol):
    """theta 0.15 on a uniform cube with one particle per leaf: for about one
    group in five the sources only some of its targets take outgrow the
    warp's list (8,192 entries), and those groups' targets walk on their own
    from the root.  Lists and forces still match the oracle's, for every
    walk-group size."""
    parts = cube(20000, 5)
    theta, eps2 = 0.15, 1e-6
    dom, sk, perm, mp, t = _oracle_build(oracle, parts, 1)
    tg = oracle.targets(t, 1, 64)
    racc, counts = oracle.walk(t, tg, soa(mp), [Params(theta, eps2, 1.0, 1)] * len(tg))
    for group in (64, 8):
        with bhg.Context(device=0) as ctx:
            ctx.set_walk_shape(group)
            ctx.upload(parts)
            ctx.build_tree(1, 64)
            ctx.compute_multipoles()
            acc = ctx.walk_forces(bhg.Context.params(theta, eps2, 1.0, True, precision), 1)
            st = ctx.stats()
            assert (st["pp"], st["pc"]) == (int(counts[0]), int(counts[1])), "interaction counts differ"
            assert rel_error(acc, racc) <= tol


@pytest.mark.parametrize("precision,tol", [(bhg.PRECISION_FP64, 1e-12), (bhg.PRECISION_SPLIT, 1e-5)])
@pytest.mark.parametrize("group", [1, 5, 16, 33, 64])
def test_walk_group_sizes_match_oracle(gpu, oracle, precision, tol, group):
    """Any walk-group cap gives every target exactly its own list (the
    interaction counts equal the oracle's) and the oracle's forces."""
    parts = bhg.plummer(30000, 31)[0]
    dom, sk, perm, mp, t = _oracle_build(oracle, parts, 16)
    tg = oracle.targets(t, 16, 256)
    racc, counts = oracle.walk(t, tg, soa(mp), [Params(0.5, 1e-4, 1.0, 1)] * len(tg))
    gpu.set_walk_shape(group)
    try:
        gpu.upload(parts)
        gpu.stats(reset=True)
        gpu.build_tree(16, 256)
        gpu.compute_multipoles()
        acc = gpu.walk_forces(bhg.Context.params(0.5, 1e-4, 1.0, True, precision), 16)
        st = gpu.stats()
    finally:
        gpu.set_walk_shape(0)
    assert (st["pp"], st["pc"]) == (int(counts[0]), int(counts[1])), "interaction counts differ"
    assert rel_error(acc, racc) <= tol


@pytest.mark.parametrize("precision", [bhg.PRECISION_SPLIT, bhg.PRECISION_FP64])
def test_two_pass_walk_equals_one_pass(precision):
    """About 550 walk groups: with the full set of list slots (two per warp)
    the walk runs its two-pass schedule (shared walks, then every target's
    pass as a job of its own); under a 20 MB budget there is room for ~260
    slots only, so it runs one warp per group on fewer blocks.  Same bits."""
    parts = bhg.plummer(30000, 31)[0]
    fp = bhg.Context.params(0.5, 1e-4, 1.0, True, precision)
    out, stats = {}, {}
    for budget in (0, 20 << 20):
        with bhg.Context(device=0, hbm_budget=budget) as ctx:
            ctx.upload(parts)
            for _ in range(2):
                ctx.step(fp, 16, 256, 16, 0.01, 0.01)
            out[budget] = ctx.download()
            stats[budget] = ctx.stats()
    assert (stats[0]["pp"], stats[0]["pc"]) == (stats[20 << 20]["pp"], stats[20 << 20]["pc"])
    assert out[0].tobytes() == out[20 << 20].tobytes()


def test_no_softening_masks_self(gpu, oracle):
    # eps = 0: r^2 == 0 entries masked (accumulate_list Mask, grouped_ttg.h:117-123)
    parts = cube(3000, 9)
    parts["pos"][7] = parts["pos"][8]  # a duplicate position
    gpu.upload(parts)
    gpu.build_tree(8, 64)
    gpu.compute_multipoles()
    acc = gpu.walk_forces(bhg.Context.params(0.5, 0.0, 1.0, True, bhg.PRECISION_FP64), 0)
    assert np.all(np.isfinite(acc))
    out, racc, _ = oracle.step(parts, theta=0.5, eps2=0.0, max_leaf=8, group_size=64, target_size=0, want_acc=True)
    assert rel_error(acc, racc) <= 1e-12


def test_step_integrates_like_oracle(gpu, oracle):
    parts = bhg.plummer(20000, 3)[0]
    kw = dict(theta=0.5, eps2=1e-4, max_leaf=16, group_size=256, target_size=16)
    ref, racc, _ = oracle.step(parts, kick_dt=1 / 256, drift_dt=1 / 128, want_acc=True, **kw)
    gpu.upload(parts)
    fp = bhg.Context.params(0.5, 1e-4, 1.0, True, bhg.PRECISION_FP64)
    gpu.step(fp, 16, 256, 16, 1 / 256, 1 / 128)
    out = gpu.download()
    assert np.array_equal(out["id"], ref["id"])
    # positions/velocities move by dt * (a few e-16 relative force differences)
    assert np.max(np.abs(out["vel"] - ref["vel"])) < 1e-12
    assert np.max(np.abs(out["pos"] - ref["pos"])) < 1e-12


def test_schedule_matches_oracle(gpu, oracle):
    parts = bhg.plummer(8192, 4)[0]
    dt, steps = 1 / 128, 3
    kw = dict(theta=0.5, eps2=1e-4, max_leaf=16, group_size=256, target_size=16)
    ref = parts
    sched = [(dt / 2, dt)] + [(dt, dt)] * (steps - 1) + [(dt / 2, 0.0)]
    for k, d in sched:
        ref, _, _ = oracle.step(ref, kick_dt=k, drift_dt=d, **kw)
    gpu.upload(parts)
    gpu.run_schedule(bhg.Context.params(0.5, 1e-4, 1.0, True, bhg.PRECISION_FP64), 16, 256, 16, dt, steps)
    out = gpu.download()
    assert np.array_equal(out["id"], ref["id"])
    assert np.max(np.abs(out["pos"] - ref["pos"])) < 1e-10


def test_systems_match_one_at_a_time(gpu, oracle):
    systems = [bhg.plummer(n, 100 + i, id0=0)[0] for i, n in enumerate((1500, 5000, 1024, 9000))]
    gpu.upload_systems(systems)
    th = np.array([0.5, 0.4, 0.7, 0.5])
    e2 = np.array([1e-4, 1e-4, 2.5e-5, 1e-4])
    gpu.set_system_params(theta=th, eps2=e2, kick_dt=np.full(4, 0.01), drift_dt=np.full(4, 0.02))
    gpu.step_systems(bhg.Context.params(0.5, 1e-4, 1.0, True, bhg.PRECISION_FP64), 16, 256, 16)
    out = gpu.download()
    at = 0
    for i, s in enumerate(systems):
        ref, _, _ = oracle.step(s, theta=th[i], eps2=e2[i], kick_dt=0.01, drift_dt=0.02, max_leaf=16,
                                group_size=256, target_size=16)
        got = out[at:at + len(s)]
        at += len(s)
        assert np.array_equal(got["id"], ref["id"])
        assert np.max(np.abs(got["pos"] - ref["pos"])) < 1e-12


def test_direct_sum_matches_cpu(gpu, oracle):
    parts = bhg.plummer(5000, 8)[0]
    gpu.upload(parts)
    idx = np.arange(0, 5000, 7, dtype=np.uint32)
    got = gpu.direct_sum(idx, 1e-4)
    ref = oracle.direct(soa(parts), idx, 1e-4)
    assert rel_error(got, ref) < 1e-13


def test_energy_matches_cpu(gpu, oracle):
    parts = bhg.plummer(3000, 9)[0]
    gpu.upload(parts)
    k, p = gpu.energy()
    assert abs(k - oracle.kinetic(parts)) <= 1e-12 * abs(k)
    assert abs(p - oracle.potential(parts)) <= 1e-12 * abs(p)


def test_nonfinite_input_is_rejected(gpu):
    parts = cube(1000, 2)
    parts["pos"][10, 1] = np.nan
    gpu.upload(parts)
    with pytest.raises(bhg.BhgError) as e:
        gpu.build_tree(8, 64)
    assert e.value.code == bhg.ENONFINITE
    # the context stays usable
    gpu.upload(cube(1000, 3))
    gpu.build_tree(8, 64)


def test_node_overflow_regrows(gpu, oracle):
    # max_leaf 1 on tight clusters of 8: chains of single-child cells down to
    # depth ~21 give far more nodes than the first estimate
    parts = cube(4000, 12, spread=10.0)
    parts["pos"] = np.repeat(parts["pos"][::8], 8, axis=0) + np.random.default_rng(3).uniform(-1e-7, 1e-7, (4000, 3))
    gpu.upload(parts)
    fp = bhg.Context.params(0.5, 1e-8, 1.0, True, bhg.PRECISION_FP64)
    gpu.step(fp, 1, 64, 0, 0.0, 0.0)
    out = gpu.download()
    ref, _, _ = oracle.step(parts, theta=0.5, eps2=1e-8, max_leaf=1, group_size=64, target_size=0)
    assert np.array_equal(out["id"], ref["id"])


def test_hbm_budget_is_enforced():
    # a budget too small for the particle arrays: a clean BHG_ENOMEM, no fault
    ctx = bhg.Context(device=0, hbm_budget=1 << 20)
    with pytest.raises(bhg.BhgError) as e:
        ctx.upload(cube(100000, 1))
    assert e.value.code == bhg.ENOMEM
    ctx.close()


@pytest.mark.parametrize("precision", [bhg.PRECISION_SPLIT, bhg.PRECISION_FP64])
def test_system_alone_equals_in_the_mix(precision):
    # a system's step does not depend on the systems batched beside it: bit
    # for bit the same particles alone and inside a 5-system batch
    systems = [bhg.plummer(n, 200 + i)[0] for i, n in enumerate((3000, 12000, 1100, 40000, 7000))]
    fp = bhg.Context.params(0.5, 1e-4, 1.0, True, precision)
    with bhg.Context(device=0) as mix:
        mix.upload_systems(systems)
        mix.set_system_params(theta=np.full(5, 0.5), eps2=np.full(5, 1e-4), kick_dt=np.full(5, 0.01),
                              drift_dt=np.full(5, 0.01))
        mix.step_systems(fp, 16, 256, 16)
        out = mix.download()
    at = 0
    with bhg.Context(device=0) as alone:
        for s in systems:
            alone.upload(s)
            alone.step(fp, 16, 256, 16, 0.01, 0.01)
            got = alone.download()
            assert got.tobytes() == out[at:at + len(s)].tobytes()
            at += len(s)


@pytest.mark.parametrize("precision", [bhg.PRECISION_FP64, bhg.PRECISION_SPLIT])
def test_energy_conservation_cold_cube(precision):
    """The scenario of the reference's test_energy_conservation.cc:13-71: a
    cold cube of 1,000 particles (positions U(-5, 5), masses U(0.5, 1.5)),
    theta 0.5, eps2 1e-4, max_leaf 8, 30 KDK steps of dt 1e-3; the total
    energy (kinetic + unsoftened potential, integrate.h:27-43) may drift by
    at most 5%.  Each KDK is two evaluations here: (dt/2, dt), then (dt/2, 0)
    at the new positions, so the velocities are synchronised when measured."""
    parts = cube(1000, 42, spread=5.0)
    fp = bhg.Context.params(0.5, 1e-4, 1.0, True, precision)
    dt = 1e-3
    with bhg.Context(device=0) as ctx:
        ctx.upload(parts)
        ke, pe = ctx.energy()
        e0 = ke + pe
        drift = 0.0
        for _ in range(30):
            ctx.step(fp, 8, 256, 8, dt / 2, dt)
            ctx.step(fp, 8, 256, 8, dt / 2, 0.0)
            ke, pe = ctx.energy()
            drift = max(drift, abs((ke + pe - e0) / e0))
    assert drift <= 0.05, drift


@pytest.mark.parametrize("precision", [bhg.PRECISION_SPLIT, bhg.PRECISION_FP64])
def test_unsoftened_system_among_softened_ones(precision):
    """Per-system parameters: one system with eps2 0 batched beside softened
    ones, the step's force params carrying eps2 > 0.  The unsoftened system
    still gets the reference's r^2 = 0 self-term mask (accumulate_list,
    grouped_ttg.h:117-123): finite forces, bit for bit those of the system
    stepped alone with eps2 0."""
    systems = [bhg.plummer(n, 300 + i)[0] for i, n in enumerate((4000, 2500, 6000))]
    e2 = np.array([1e-4, 0.0, 1e-4])
    fp = bhg.Context.params(0.5, 1e-4, 1.0, True, precision)
    with bhg.Context(device=0) as mix:
        mix.upload_systems(systems)
        mix.set_system_params(theta=np.full(3, 0.5), eps2=e2, kick_dt=np.full(3, 0.01), drift_dt=np.full(3, 0.01))
        mix.step_systems(fp, 16, 256, 16)
        out = mix.download()
    assert np.all(np.isfinite(out["pos"])) and np.all(np.isfinite(out["vel"]))
    at = sum(len(s) for s in systems[:1])
    with bhg.Context(device=0) as alone:
        alone.upload(systems[1])
        alone.step(bhg.Context.params(0.5, 0.0, 1.0, True, precision), 16, 256, 16, 0.01, 0.01)
        got = alone.download()
    assert got.tobytes() == out[at:at + len(systems[1])].tobytes()


def _cut(g, lim):
    """Topmost nodes holding at most lim particles, or leaves, depth first in
    child order from each root (the target rule of bho_targets)."""
    out = []
    for r in np.flatnonzero(g["depth"] == 0):
        st = [int(r)]
        while st:
            i = st.pop()
            if g["leaf"][i] or g["count"][i] <= lim:
                out.append(i)
                continue
            st.extend(int(g["first_child"][i]) + c for c in range(int(g["nchild"][i]) - 1, -1, -1))
    return np.array(out, np.uint32)


def _pack(g, targets, chunks, pack, max_targets=24):
    """Walk groups: inside each packing chunk, consecutive targets packed
    greedily while the group holds at most `pack` particles and max_targets
    targets (a larger target is a group of its own); the index of each
    group's first target."""
    begin, count = g["begin"], g["count"]
    tb = begin[targets]
    starts = []
    for c in chunks:
        cb, ce = int(begin[c]), int(begin[c]) + int(count[c])
        j = int(np.searchsorted(tb, cb, side="left"))
        first, cnt, k = True, 0, 0
        while j < len(targets) and tb[j] < ce:
            n = int(count[targets[j]])
            if first or cnt + n > pack or k >= max_targets:
                starts.append(j)
                first, cnt, k = False, 0, 0
            cnt += n
            k += 1
            j += 1
    return np.array(starts, np.uint32)


@pytest.mark.parametrize("group", [1, 5, 32, 64])
def test_walk_groups_follow_the_packing_rule(group):
    """The walk groups of a three-system batch are the greedy packing of each
    system's targets inside its packing chunks (nodes of at most 2,048
    particles), whatever the walk-group cap."""
    systems = [bhg.plummer(65536, 1)[0], bhg.plummer(3000, 7)[0], bhg.plummer(40000, 8)[0]]
    fp = bhg.Context.params(0.5, 1e-4, 1.0, True, bhg.PRECISION_SPLIT)
    with bhg.Context(device=0) as ctx:
        ctx.set_walk_shape(group)
        ctx.upload_systems(systems)
        ctx.set_system_params(theta=np.full(3, 0.5), eps2=np.full(3, 1e-4), kick_dt=np.full(3, 0.01),
                              drift_dt=np.full(3, 0.01))
        ctx.step_systems(fp, 16, 256, 16)
        g = ctx.tree()
        targets = ctx.export(bhg.EXPORT_TARGETS)
        groups = ctx.export(bhg.EXPORT_GROUPS)
    assert np.array_equal(targets, _cut(g, 16))
    want = _pack(g, targets, _cut(g, 2048), group)
    assert len(groups) == len(want) and np.array_equal(groups, want)
