"""read_csv / write_vtk (io.cc): the oracle's restatement against the
reference's own io.cc (compiled here into oracle/_ref), and the exact number
conversions the GPU uses (bhg_decimal.cuh, compiled for the host) against the
C++ library."""
import os
import subprocess

import numpy as np
import pytest

from oracle import Reference
from text_cases import MALFORMED, csv_text, random_particles

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
needs_ref = pytest.mark.skipif(not Reference.available(), reason="oracle/_ref not built")


def same(a, b):
    """bitwise, with every NaN equal to every NaN of the same sign"""
    if len(a) != len(b):
        return False
    for f in ("mass", "pos", "vel"):
        x, y = np.asarray(a[f], np.float64), np.asarray(b[f], np.float64)
        nan = np.isnan(x) & np.isnan(y) & (np.signbit(x) == np.signbit(y))
        if not np.all((x.view(np.uint64) == y.view(np.uint64)) | nan):
            return False
    return np.array_equal(a["id"], b["id"])


CASES = [
    dict(seed=1),
    dict(seed=2, header=True),
    dict(seed=3, crlf=True, blanks=True),
    dict(seed=4, blank_lines=True, final_newline=False),
    dict(seed=5, header=True, crlf=True, blanks=True, blank_lines=True),
]


@needs_ref
@pytest.mark.parametrize("case", CASES, ids=[str(i) for i in range(len(CASES))])
def test_oracle_read_csv_matches_reference(oracle, case):
    parts = random_particles(3000, case["seed"], special=True)
    text = csv_text(parts, **case)
    got, bad = oracle.read_csv(text)
    want, err = Reference().read_csv(text)
    assert bad is None and err is None
    assert same(got, want)
    # the %.17g and shortest forms round-trip: the parsed particles are the
    # originals wherever those forms were written (checked on a pure case)
    pure = csv_text(parts, case["seed"], styles=(0, 1))
    back, _ = oracle.read_csv(pure)
    assert same(back, parts)


@needs_ref
@pytest.mark.parametrize("bad", MALFORMED)
def test_oracle_rejects_what_the_reference_rejects(oracle, bad):
    good = csv_text(random_particles(5, 9), 9, styles=(0,))
    text = good + bad + good
    got, line = oracle.read_csv(text)
    want, err = Reference().read_csv(text)
    assert got is None and want is None
    assert line == 5
    assert bad.strip().decode() in err


@needs_ref
def test_oracle_write_vtk_matches_reference(oracle):
    parts = random_particles(5000, 11, special=True)
    parts["mass"][:3] = [np.nan, -np.nan, 5e-324]
    assert oracle.write_vtk(parts) == Reference().write_vtk(parts)


def test_decimal_conversions_match_the_cxx_library(tmp_path):
    exe = tmp_path / "decimal_check"
    subprocess.run(["g++", "-std=c++20", "-O2", "-I", os.path.join(ROOT, "amt-bh-benchmark_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "decimal_check.cc"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe), "100000"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("ok")


@pytest.mark.parametrize("name", ["text_mixed", "text_crlf"])
def test_oracle_matches_text_golden(oracle, name):
    """The reference's own read_csv/write_vtk outputs, committed (made by
    tests/golden/make_text_golden.py), against the oracle, anywhere."""
    g = np.load(os.path.join(ROOT, "tests", "golden", name + ".npz"))
    got, bad = oracle.read_csv(g["text"].tobytes())
    assert bad is None and same(got, g["particles"])
    assert oracle.write_vtk(g["particles"]) == g["vtk"].tobytes()
