"""The C++ drop-in for bh::step_particles (amt-bh-benchmark_b200/include/
bhg_step_particles.hpp): it compiles against the reference's own types (CPU,
where the reference tree exists) and, on the GPU, runs the reference's
leapfrog schedule to the oracle's result."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "amt-bh-benchmark_b200")
SRC = os.path.join(ROOT, "tests", "cpp", "adapter_main.cc")


def _reference_src():
    """The reference's src directory: BHG_REFERENCE_DIR, else the directory the
    oracle build recorded (oracle/_ref/reference_dir.txt); None if neither."""
    d = os.environ.get("BHG_REFERENCE_DIR")
    rec = os.path.join(ROOT, "oracle", "_ref", "reference_dir.txt")
    if not d and os.path.exists(rec):
        d = open(rec).read().strip()
    return os.path.join(d, "src") if d and os.path.isdir(os.path.join(d, "src")) else None


REF_SRC = _reference_src()
INC = ["-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(PKG, "include")]
LINK = ["-L" + PKG, "-lbhg", "-Wl,-rpath," + PKG]


def compile_adapter(out, reference_types=False):
    cmd = ["g++", "-std=c++20", "-O2", *INC, SRC, "-o", out, *LINK, "-pthread"]
    if reference_types:
        cmd[3:3] = ["-DBHG_WITH_REFERENCE_TYPES", "-I" + os.path.join(ROOT, "oracle", "ttg_shim"), "-I" + REF_SRC]
        cmd.insert(-4, os.path.join(REF_SRC, "tree.cc"))
    subprocess.run(cmd, check=True, capture_output=True, text=True)


@pytest.mark.skipif(REF_SRC is None, reason="reference sources not present (BHG_REFERENCE_DIR unset, nothing recorded by the build)")
def test_adapter_compiles_against_reference_types(tmp_path):
    compile_adapter(str(tmp_path / "adapter_ref"), reference_types=True)


def test_adapter_compiles_against_layout_twins(tmp_path):
    compile_adapter(str(tmp_path / "adapter_local"))


# split: FP32 interactions with FP64 sums (the drop-in's default); the
# forces differ from the FP64 oracle's by ~1e-7 relative, positions after 3
# steps of dt 1/128 by far less than 1e-9
@pytest.mark.gpu
@pytest.mark.parametrize("precision,pos_tol", [("0", 1e-9), ("1", 1e-10)], ids=["split", "fp64"])
def test_adapter_schedule_matches_oracle(tmp_path, oracle, precision, pos_tol):
    import bhg

    parts, _ = bhg.plummer(8192, 41)
    exe = str(tmp_path / "adapter")
    compile_adapter(exe)
    src, dst = tmp_path / "in.bin", tmp_path / "out.bin"
    parts.tofile(src)
    dt, steps = 1 / 128, 3
    r = subprocess.run([exe, str(src), str(dst), "0.5", "0.01", repr(dt), str(steps), precision],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = np.fromfile(dst, dtype=bhg.PARTICLE)
    ref = parts
    for k, d in [(dt / 2, dt)] + [(dt, dt)] * (steps - 1) + [(dt / 2, 0.0)]:
        ref, _, _ = oracle.step(ref, theta=0.5, eps2=1e-4, max_leaf=16, group_size=256, target_size=16,
                                kick_dt=k, drift_dt=d)
    # by particle id: a split-precision position may round into the
    # neighbouring Morton cell and change the output order
    o, r = out[np.argsort(out["id"])], ref[np.argsort(ref["id"])]
    assert np.array_equal(o["id"], r["id"])
    assert np.max(np.abs(o["pos"] - r["pos"])) < pos_tol


@pytest.mark.gpu
def test_adapter_empty_input_comes_back_empty(tmp_path):
    """An empty particle vector: the reference builds an empty tree and walks
    nothing (flat_build_ttg.h:215); the drop-in returns the empty vector."""
    exe = str(tmp_path / "adapter")
    compile_adapter(exe)
    src, dst = tmp_path / "in.bin", tmp_path / "out.bin"
    src.write_bytes(b"")
    r = subprocess.run([exe, str(src), str(dst), "0.5", "0.01", repr(1 / 128), "2", "0"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert dst.read_bytes() == b""
