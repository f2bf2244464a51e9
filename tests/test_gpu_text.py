"""Particle text on the GPU (bhg_upload_csv / bhg_add_csv /
bhg_snapshot_vtk) against the oracle's read_csv / write_vtk, which the CPU
tests pin to the reference's io.cc: parsed particles bit for bit, snapshots
byte for byte, malformed lines reported at the same line."""
import numpy as np
import pytest

import bhg
from oracle import PARTICLE
from test_text_cpu import CASES, same
from text_cases import MALFORMED, csv_text, random_particles

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", CASES, ids=[str(i) for i in range(len(CASES))])
def test_csv_ingest_matches_oracle(gpu, oracle, case):
    parts = random_particles(20000, case["seed"], special=True)
    text = csv_text(parts, **case)
    want, bad = oracle.read_csv(text)
    assert bad is None
    gpu.upload_csv(text)
    assert same(gpu.download(), want)


def test_csv_ingest_long_and_odd_numbers(gpu, oracle):
    rng = np.random.default_rng(7)
    lines = []
    for i in range(3000):
        x = float(rng.normal()) * 10.0 ** int(rng.integers(-300, 300))
        forms = [("%.60e" % x), ("-0." + "0" * int(rng.integers(0, 300)) + "1234567890123456789012345"),
                 "00000" + repr(abs(x)), "1" + "0" * int(rng.integers(0, 300)) + ".5e-" + str(int(rng.integers(0, 320))),
                 "inf", "-INFINITY", "4.9406564584124654e-324", "2.4703282292062328e-324", "-0", ".5", "7."]
        f = [str(i)] + [forms[int(rng.integers(len(forms)))] for _ in range(7)]
        lines.append(",".join(f))
    text = ("\n".join(lines) + "\n").encode()
    want, bad = oracle.read_csv(text)
    assert bad is None
    gpu.upload_csv(text)
    assert same(gpu.download(), want)


@pytest.mark.parametrize("bad", MALFORMED)
def test_csv_malformed_line_is_reported(gpu, oracle, bad):
    good = csv_text(random_particles(5, 9), 9, styles=(0,))
    text = good + bad + good
    _, line = oracle.read_csv(text)
    with pytest.raises(bhg.BhgError) as e:
        gpu.upload_csv(text)
    assert e.value.code == bhg.EINVAL
    assert f"malformed line {line + 1}:" in str(e.value)
    assert bad.strip().decode() in str(e.value)


def test_csv_round_trip_and_systems(oracle):
    a, _ = bhg.plummer(100000, 3)
    b, _ = bhg.plummer(777, 4)
    with bhg.Context(device=0) as ctx:
        ha = ctx.add_csv(csv_text(a, 1, styles=(0, 1)))  # shortest and %.17g forms round-trip
        hb = ctx.add_csv(csv_text(b, 2, header=True, crlf=True, styles=(1,)))
        assert list(ctx.system_ids()) == [ha, hb]
        got = ctx.download()
    assert same(got[: len(a)], a) and same(got[len(a):], b)


def test_vtk_snapshot_matches_oracle(oracle):
    parts = random_particles(30000, 11, special=True)
    parts["mass"][:3] = [np.nan, -np.nan, 5e-324]
    with bhg.Context(device=0) as ctx:
        h = ctx.add_system(parts)
        assert ctx.snapshot_vtk(h) == oracle.write_vtk(parts)


def test_vtk_snapshot_after_a_step(oracle):
    parts, _ = bhg.plummer(50000, 5)
    with bhg.Context(device=0) as ctx:
        ctx.upload(parts)
        ctx.step(bhg.Context.params(0.5, 1e-4, 1.0, True, bhg.PRECISION_SPLIT), 16, 256, 16, 0.01, 0.01)
        out = ctx.download()  # Morton order, as step_particles returns it
        assert ctx.snapshot_vtk() == oracle.write_vtk(out)


def test_empty_and_header_only_texts(gpu):
    for text in (b"", b"id,mass,x,y,z,vx,vy,vz\n", b"\n\n  \n"):
        with pytest.raises(bhg.BhgError) as e:
            gpu.upload_csv(text)
        assert "no particles" in str(e.value)


@pytest.mark.parametrize("name", ["text_mixed", "text_crlf"])
def test_gpu_matches_text_golden(gpu, name):
    """The reference's own read_csv/write_vtk outputs, committed, against the GPU."""
    import os

    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", name + ".npz"))
    gpu.upload_csv(g["text"].tobytes())
    got = gpu.download()
    assert same(got, g["particles"])
    assert gpu.snapshot_vtk() == g["vtk"].tobytes()
