"""The multi-GPU path is independent replicas (no collective on the data
path): ranks only line up and combine their numbers.  These run that
plumbing as two gloo ranks on the CPU, as torchrun would start them."""
import json
import os
import socket
import subprocess
import sys
import time

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _launch(ranks, world, timeout_s=60):
    port = _free_port()
    procs = []
    for rank in ranks:
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), REPLICA_TIMEOUT=str(timeout_s))
        procs.append(subprocess.Popen([sys.executable, os.path.join(HERE, "replica_worker.py")], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    return procs


def test_two_replicas_combine_their_numbers():
    procs = _launch([0, 1], 2)
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=120)
        assert p.returncode == 0, e
        outs.append(json.loads(o.strip().splitlines()[-1]))
    for o in outs:
        assert o["world"] == 2
        assert o["max"] == 3.0 and o["sum"] == 21.0
        # (1000 + 2000) particle-steps in the slowest rank's 3 ms
        assert abs(o["value"] - 3000 / 0.003) < 1e-6
    assert {o["seed"] for o in outs} == {7, 8}  # every rank simulates its own particles


def test_single_rank_needs_no_process_group():
    env = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    o = subprocess.run([sys.executable, os.path.join(HERE, "replica_worker.py")], env=env, capture_output=True,
                       text=True, timeout=120)
    assert o.returncode == 0, o.stderr
    d = json.loads(o.stdout.strip().splitlines()[-1])
    assert d["world"] == 1 and d["max"] == 1.5 and d["value"] == 1000 / 0.002


def test_missing_rank_ends_with_an_error():
    """A rank that never joins: the other gives up after the process group's
    timeout instead of waiting for ever."""
    t0 = time.time()
    (p,) = _launch([0], 2, timeout_s=5)
    try:
        _, e = p.communicate(timeout=120)
    except subprocess.TimeoutExpired:
        p.kill()
        pytest.fail("rank 0 kept waiting for the missing rank")
    assert p.returncode != 0
    assert time.time() - t0 < 120
