"""The autotuner's choice and cache rules, with a fake context (no GPU).

The knobs follow the reference's own options (main.cc:27-33: max_leaf,
target_size and group_size are independent) plus the walk's shape; theta is
never tuned."""
import numpy as np
import pytest

import bhg
from bhg import autotune


class FakeCtx:
    """Plays a context: times and errors come from tables keyed by leaf."""

    def __init__(self, ms, err, seen):
        self.ms, self.err, self.seen = ms, err, seen
        self.leaf = None
        self.n = 0
        self.shape = (0, 0)

    def upload(self, p):
        self.n = len(p)

    def upload_systems(self, systems):
        self.n = sum(len(p) for p in systems)

    def set_walk_shape(self, group, warps):
        self.shape = (group, warps)

    def set_system_params(self, **kw):
        self.seen["theta"].update(np.unique(kw["theta"]).tolist())

    def build_tree(self, leaf, group):
        self.leaf = leaf

    def compute_multipoles(self):
        pass

    def walk_forces(self, fp, target):
        self.seen["theta"].add(round(fp.theta, 12))
        acc = np.ones((self.n, 3))
        acc[:, 0] += self.err[(self.leaf, self.shape[0])]  # relative error err in x of a (1, 1, 1) field
        return acc

    def direct_sum(self, idx, eps2):
        return np.ones((len(idx), 3))

    def step_systems(self, fp, leaf, group, target):
        self.leaf = leaf
        self.seen["theta"].add(round(fp.theta, 12))

    def stats(self, reset=False):
        ms = self.ms[(self.leaf, self.shape[0])]
        return {"pre_ms": 0.0, "sort_ms": 0.0, "tree_ms": 0.0, "multipole_ms": 0.0, "targets_ms": 0.0,
                "walk_ms": ms * 3, "evals": 3}

    def close(self):
        pass


def _systems():
    return [np.zeros(1000, bhg.PARTICLE), np.zeros(5000, bhg.PARTICLE)]


def _tune(tmp_path, ms, err, cands, **kw):
    seen = {"theta": set()}
    res = autotune.tune(_systems(), 0.5, 1e-4, 256, cands=cands, context_factory=lambda d: FakeCtx(ms, err, seen),
                        cache_path=str(tmp_path / "c.json"), dev_name="fake", **kw)
    return res, seen


def test_fastest_within_budget_wins_and_theta_is_untouched(tmp_path):
    cands = autotune.candidates(leaves=(16, 32, 64))
    ms = {(16, 0): 5.0, (32, 0): 3.0, (64, 0): 2.0}
    # relative error sqrt(e^2 / 3) per particle: leaf 64 breaks a 1e-3 budget
    err = {(16, 0): 1e-4, (32, 0): 5e-4, (64, 0): 5e-3}
    res, seen = _tune(tmp_path, ms, err, cands)
    assert res["max_leaf"] == 32 and res["target_size"] == 32
    assert seen["theta"] == {0.5}
    assert [r["max_leaf"] for r in res["table"]] == [16, 32, 64]


def test_no_candidate_within_budget_takes_the_most_accurate(tmp_path):
    cands = autotune.candidates(leaves=(16, 32))
    res, _ = _tune(tmp_path, {(16, 0): 5.0, (32, 0): 1.0}, {(16, 0): 0.02, (32, 0): 0.05}, cands)
    assert res["max_leaf"] == 16


def test_walk_group_is_a_tuned_dimension(tmp_path):
    cands = autotune.candidates(leaves=(16,), walk_groups=(32, 64))
    res, _ = _tune(tmp_path, {(16, 32): 2.0, (16, 64): 1.5}, {(16, 32): 1e-4, (16, 64): 1e-4}, cands)
    assert res["walk_group"] == 64
    assert {(r["max_leaf"], r["walk_group"]) for r in res["table"]} == {(16, 32), (16, 64)}


def test_cache_hit_and_key_changes(tmp_path):
    cands = autotune.candidates(leaves=(16, 32))
    ms, err = {(16, 0): 5.0, (32, 0): 3.0}, {(16, 0): 1e-4, (32, 0): 1e-4}
    first, _ = _tune(tmp_path, ms, err, cands)
    assert first["cached"] is False
    again, _ = _tune(tmp_path, ms, err, cands)
    assert again["cached"] is True and again["max_leaf"] == first["max_leaf"]
    base = dict(total_n=6000, nsys=2, theta=0.5, eps2=1e-4, precision=0, group_size=256, err_budget=1e-3,
                cands=cands, device_name="fake")
    k0 = autotune.cache_key(**base)
    for change in (dict(group_size=64), dict(err_budget=1e-4), dict(cands=autotune.candidates(leaves=(16,))),
                   dict(device_name="other"), dict(nsys=512), dict(theta=0.4), dict(precision=1),
                   dict(total_n=60000)):
        assert autotune.cache_key(**dict(base, **change)) != k0, change


@pytest.mark.parametrize("budget,expect", [(1e-3, 32), (2e-4, 16)])
def test_budget_moves_the_choice(tmp_path, budget, expect):
    cands = autotune.candidates(leaves=(16, 32))
    res, _ = _tune(tmp_path, {(16, 0): 5.0, (32, 0): 3.0}, {(16, 0): 1e-4, (32, 0): 5e-4}, cands, err_budget=budget)
    assert res["max_leaf"] == expect
