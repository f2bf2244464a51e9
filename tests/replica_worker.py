"""One rank of the multi-process replica test (launched by
test_replicas_cpu.py with torchrun's environment variables set)."""
import json
import os
import sys

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "amt-bh-benchmark_b200"))
from bhg.replicas import Replicas, replica_seed  # noqa: E402

r = Replicas("gloo", "cpu", timeout_s=int(os.environ.get("REPLICA_TIMEOUT", "60")))
out = {"rank": r.rank, "world": r.world}
out["max"] = r.max(1.5 * (r.rank + 1))
out["sum"] = r.sum(r.rank + 10)
r.barrier()
# the benchmark's combination: every rank its own work, the slowest rank's time
units, ms = 1000 * (r.rank + 1), 2.0 + r.rank
out["value"] = r.sum(units) / (r.max(ms) / 1000.0)
out["seed"] = replica_seed(7, r.rank)
r.close()
print(json.dumps(out), flush=True)
