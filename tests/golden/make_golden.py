"""Generates the golden fixtures of tests/golden/ from the reference itself.

Runs the reference's own code - build_flat_tree, run_grouped_pass,
step_particles and brute_force_accel compiled from the unmodified sources
into oracle/_ref/libbhref.so (oracle/Makefile) - on small inputs and stores
inputs and outputs as .npz files.  Needs the reference tree (only present
where oracle/_ref was built); the fixtures it writes are committed, so the
tests that read them run anywhere.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

from helpers import cube, plummer_np  # noqa: E402
from oracle import PARTICLE, Reference  # noqa: E402

REF_DATA = "/root/reference/ttg-parsec/data"


def read_ref_csv(name):
    rows = [ln.split(",") for ln in open(os.path.join(REF_DATA, name)).read().split() if ln.strip()]
    p = np.zeros(len(rows), PARTICLE)
    for i, r in enumerate(rows):
        p[i]["id"] = int(r[0])
        p[i]["mass"] = float(r[1])
        p[i]["pos"] = [float(x) for x in r[2:5]]
        p[i]["vel"] = [float(x) for x in r[5:8]]
    return p


def cases():
    yield "shared_ic_20", read_ref_csv("shared_ic_20.csv"), dict(max_leaf=8, group_size=256, target_size=32,
                                                                  theta=0.5, eps2=1e-4)
    yield "two_body", read_ref_csv("two_body.csv"), dict(max_leaf=8, group_size=256, target_size=32, theta=0.5,
                                                          eps2=0.0)
    yield "cube2000", cube(2000, 4), dict(max_leaf=8, group_size=64, target_size=0, theta=0.5, eps2=1e-6)
    yield "cube2000_leaf1_ts32", cube(2000, 6), dict(max_leaf=1, group_size=64, target_size=32, theta=0.5,
                                                     eps2=1e-6)
    yield "plummer4096", plummer_np(4096, 7), dict(max_leaf=16, group_size=256, target_size=16, theta=0.5,
                                                   eps2=1e-4)


def main():
    R = Reference()
    for name, parts, kw in cases():
        t = R.build(parts, kw["max_leaf"], kw["group_size"])
        acc_q, miss = R.walk(t, kw["theta"], kw["eps2"], 1.0, True, kw["target_size"])
        acc_m, _ = R.walk(t, kw["theta"], kw["eps2"], 1.0, False, kw["target_size"])
        n = t["n"]
        step, _ = R.step(parts, theta=kw["theta"], eps2=kw["eps2"], max_leaf=kw["max_leaf"],
                         group_size=kw["group_size"], target_size=kw["target_size"], kick_dt=1e-3, drift_dt=2e-3)
        brute = R.brute(t["particles"], max(kw["eps2"], 1e-12)) if len(parts) <= 4096 else None
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"),
            input=parts.view(np.uint8).reshape(len(parts), 64),
            params=np.array([kw["max_leaf"], kw["group_size"], kw["target_size"], kw["theta"], kw["eps2"]]),
            domain=t["domain"], keys=t["keys"], order=t["particles"]["id"],
            node_u32=np.stack([t[k][:n] for k in ("depth", "begin", "count", "leaf", "nchild")]),
            node_center=t["center"][:n], node_hw=t["hw"][:n], node_mass=t["mass"][:n], node_com=t["com"][:n],
            node_iab=t["iab"][:n], acc_quad=acc_q, acc_mono=acc_m, missing=np.array([miss]),
            step=step.view(np.uint8).reshape(len(step), 64), step_kick_drift=np.array([1e-3, 2e-3]),
            brute=brute if brute is not None else np.zeros((0, 3)),
        )
        R.free(t)
        print(name, len(parts), "nodes", n)


if __name__ == "__main__":
    main()
