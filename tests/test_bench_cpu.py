"""The benchmark's reference arm, on the CPU: its JSON line times exactly the
requested warm-up and timed evaluations, describes the workload with the same
`config` object as the GPU arm (one function builds both), and the process
never loads the GPU library (the reference's timing binary generates its own
initial conditions)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402


_RUN_REFERENCE_ARM = """
import json, sys
sys.path.insert(0, {root!r})
sys.argv = ["bench.py", "--impl", "reference", "--workload", "plummer-65k", "--steps", "2", "--warmup", "1"]
import bench
rc = bench.main()
maps = open("/proc/self/maps").read()
print(json.dumps({{"rc": rc, "libbhg_mapped": "libbhg.so" in maps}}))
"""


def test_reference_arm_line_is_consistent():
    if bench.ref_binary() is None:
        pytest.skip("oracle/_ref/ref_bench is not built")
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, "-c", _RUN_REFERENCE_ARM.format(root=ROOT)], capture_output=True, text=True,
                       env=env, timeout=600)
    assert r.returncode == 0, r.stderr
    out = [json.loads(x) for x in r.stdout.strip().splitlines() if x.startswith("{")]
    line, proc = out[-2], out[-1]
    assert proc == {"rc": 0, "libbhg_mapped": False}, "the reference arm's process loaded the GPU library"
    w = bench.WORKLOADS["plummer-65k"]
    assert line["impl"] == "reference"
    assert (line["steps"], line["warmup"]) == (2, 1)
    assert line["config"] == json.loads(json.dumps(bench.workload_config("plummer-65k", w, 1)))
    assert line["metric"] == bench.METRIC and line["unit"] == "particle-steps/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"]["value"] == line["value"]
    # one step = one evaluation of the 16-step schedule; the rate counts 16
    # particle-steps per 17 evaluations
    assert abs(line["value"] - 65536 * 16 / (17 * line["ms_per_step"] / 1000.0)) <= 1e-6 * line["value"]


def test_workload_config_is_deterministic():
    for name, w in bench.WORKLOADS.items():
        a = bench.workload_config(name, w, 2)
        b = bench.workload_config(name, w, 2)
        assert a == b and a["workload"] == name and a["parallelism"] == "replicas x2"
