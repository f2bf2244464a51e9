"""Pins the CPU oracle (oracle/bh_oracle.c) to the reference.

1. Against the committed golden fixtures (tests/golden/, made by
   make_golden.py from the reference's own code): keys, order, node set, cell
   geometry, mass and centre of mass bit for bit; second moments to the last
   bits (the reference binary contracts a*b+c into FMAs); forces and a full
   step to rounding.
2. Against the reference compiled here (oracle/_ref) on fresh inputs, when it
   is present: the same, and bit for bit against its no-contraction build.
3. The reference's own test programs, built against the stand-in TTG runtime.
"""
import glob
import os
import subprocess

import numpy as np
import pytest

from helpers import cube, plummer_np, rel_error
from oracle import PARTICLE, Params, Reference, node_order, node_tuples, soa

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# the tree/force fixtures; text_*.npz are the CSV/VTK fixtures of the text tests
GOLDEN = sorted(p for p in glob.glob(os.path.join(ROOT, "tests", "golden", "*.npz"))
                if not os.path.basename(p).startswith("text_"))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def load(path):
    z = np.load(path)
    parts = z["input"].reshape(-1).view(PARTICLE)
    ml, gs, ts, th, e2 = z["params"]
    return z, parts, dict(max_leaf=int(ml), group_size=int(gs), target_size=int(ts), theta=float(th), eps2=float(e2))


def oracle_tree(oracle, parts, max_leaf):
    dom, bad = oracle.domain(parts)
    keys = oracle.keys(parts, dom)
    perm, sk = oracle.sort(keys)
    mp = parts[perm]
    t = oracle.build(sk, [0], [len(parts)], dom[None], max_leaf, soa(mp))
    return dom, sk, mp, t


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_golden(oracle, path):
    z, parts, kw = load(path)
    dom, sk, mp, t = oracle_tree(oracle, parts, kw["max_leaf"])
    assert np.array_equal(dom, z["domain"])
    assert np.array_equal(sk, z["keys"])
    assert np.array_equal(mp["id"], z["order"])
    n = t["n"]
    ref_tuples = sorted(map(tuple, z["node_u32"].T.tolist()))
    assert node_tuples(t) == ref_tuples
    a = node_order(t)
    rb = np.lexsort((z["node_u32"][1].astype(np.int64), z["node_u32"][0].astype(np.int64)))
    for k in ("center", "hw", "mass", "com"):
        assert np.array_equal(np.asarray(t[k][:n])[a], z["node_" + k][rb]), k
    iab_o, iab_r = np.asarray(t["iab"][:n])[a], z["node_iab"][rb]
    scale = np.abs(iab_r).max(axis=1, keepdims=True) + 1e-300
    assert np.max(np.abs(iab_o - iab_r) / scale) < 1e-13
    tg = oracle.targets(t, kw["target_size"], kw["group_size"])
    for quad, key in ((True, "acc_quad"), (False, "acc_mono")):
        acc, _ = oracle.walk(t, tg, soa(mp), [Params(kw["theta"], kw["eps2"], 1.0, int(quad))] * len(tg))
        assert rel_error(acc, z[key]) < 1e-13, key
    step, _, _ = oracle.step(parts, theta=kw["theta"], eps2=kw["eps2"], max_leaf=kw["max_leaf"],
                             group_size=kw["group_size"], target_size=kw["target_size"], kick_dt=1e-3,
                             drift_dt=2e-3)
    ref = z["step"].reshape(-1).view(PARTICLE)
    assert np.array_equal(step["id"], ref["id"])
    assert np.max(np.abs(step["vel"] - ref["vel"])) <= 1e-13 * max(1.0, np.abs(ref["vel"]).max())
    assert np.max(np.abs(step["pos"] - ref["pos"])) <= 1e-13 * max(1.0, np.abs(ref["pos"]).max())
    if len(z["brute"]):
        d = oracle.direct(soa(mp), np.arange(len(mp)), max(kw["eps2"], 1e-12))
        assert rel_error(d, z["brute"]) < 1e-13


needs_ref = pytest.mark.skipif(not Reference.available(), reason="reference-built checkers not present")


@needs_ref
@pytest.mark.parametrize("make,max_leaf,gs,ts", [
    (lambda: cube(3000, 21), 8, 64, 0),
    (lambda: plummer_np(20000, 22), 16, 256, 16),
    (lambda: cube(2500, 23, spread=1e-3), 1, 64, 32),
])
def test_oracle_matches_live_reference(oracle, make, max_leaf, gs, ts):
    parts = make()
    R = Reference()
    rt = R.build(parts, max_leaf, gs)
    dom, sk, mp, t = oracle_tree(oracle, parts, max_leaf)
    assert np.array_equal(dom, rt["domain"]) and np.array_equal(sk, rt["keys"])
    assert mp.tobytes() == rt["particles"].tobytes()
    assert node_tuples(t) == node_tuples(rt)
    tg = oracle.targets(t, ts, gs)
    acc, _ = oracle.walk(t, tg, soa(mp), [Params(0.5, 1e-6, 1.0, 1)] * len(tg))
    racc, missing = R.walk(rt, 0.5, 1e-6, 1.0, True, ts)
    assert missing == 0
    assert rel_error(acc, racc) < 1e-13
    R.free(rt)


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_DIR, "libbhref_nocontract.so")),
                    reason="no-contraction reference build not present")
def test_multipoles_bit_exact_without_contraction(oracle):
    R = Reference(os.path.join(REF_DIR, "libbhref_nocontract.so"))
    parts = plummer_np(30000, 31)
    rt = R.build(parts, 16, 256)
    dom, sk, mp, t = oracle_tree(oracle, parts, 16)
    a, b = node_order(t), node_order(rt)
    for k in ("center", "hw", "mass", "com", "iab"):
        assert np.array_equal(np.asarray(t[k][:t["n"]])[a], np.asarray(rt[k])[b]), k
    R.free(rt)


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_DIR, "test_force_kernel")), reason="not built")
@pytest.mark.parametrize("prog", ["test_force_kernel", "test_morton", "test_bh_vs_bruteforce",
                                  "test_energy_conservation"])
def test_reference_own_tests_pass(prog):
    env = dict(os.environ, TTG_NUM_THREADS=str(min(8, os.cpu_count() or 1)))
    r = subprocess.run([os.path.join(REF_DIR, prog)], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "FAIL" not in r.stdout + r.stderr
