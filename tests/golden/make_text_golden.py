"""Generates the text fixtures of tests/golden/ from the reference itself:
CSV texts in every number form and layout read_csv accepts, with the
particles the reference's read_csv (io.cc, compiled from the unmodified
sources into oracle/_ref/libbhref.so) parses from them, and the bytes its
write_vtk writes for those particles.  Needs oracle/_ref; the fixtures it
writes are committed, so the tests that read them run anywhere.

    python tests/golden/make_text_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

from oracle import Reference  # noqa: E402
from text_cases import csv_text, random_particles  # noqa: E402

CASES = {
    "text_mixed": dict(n=2000, seed=41, kw=dict(header=True, blanks=True, blank_lines=True)),
    "text_crlf": dict(n=1000, seed=42, kw=dict(crlf=True, final_newline=False)),
}


def main():
    ref = Reference()
    for name, c in CASES.items():
        parts = random_particles(c["n"], c["seed"], special=True)
        text = csv_text(parts, c["seed"], **c["kw"])
        got, err = ref.read_csv(text)
        assert err is None, err
        vtk = ref.write_vtk(got)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), text=np.frombuffer(text, np.uint8), particles=got,
                            vtk=np.frombuffer(vtk, np.uint8))
        print(name, len(text), len(got), len(vtk))


if __name__ == "__main__":
    main()
