"""CPU checks of the C ABI library: it loads without a GPU and exports every
entry point include/bhg.h declares."""
import os
import re

import bhg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "bhg.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(bhg_[a-z0-9_]+)\s*\(", src)))


def test_header_and_binding_agree():
    assert declared() == sorted(bhg.EXPORTED)


def test_library_exports_every_declared_symbol():
    L = bhg.lib()
    for name in declared():
        assert hasattr(L, name), name


def test_plummer_generator_is_deterministic():
    a, n1 = bhg.plummer(1000, 5)
    b, n2 = bhg.plummer(1000, 5)
    assert a.tobytes() == b.tobytes() and n1 == n2
    r = (a["pos"] ** 2).sum(1) ** 0.5
    assert r.max() < 10.0 and abs(a["mass"].sum() - 1.0) < 1e-12
