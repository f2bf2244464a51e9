"""TEST INFRASTRUCTURE ONLY - ctypes access to the oracle libraries.

``Oracle`` wraps ``oracle/libbhoracle.so`` (the plain-C restatement of the
reference's grouped Barnes-Hut pipeline, ``bh_oracle.c``).  ``Reference``
wraps ``oracle/_ref/libbhref.so`` (the reference's own code compiled from its
unmodified sources, present only where it was built).  Only the tests, the
smoke check and the benchmark's CPU-baseline leg import this module; the
product library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

#: bh::Particle (particle.h:7-24): 64 bytes, 4 bytes of padding after id.
PARTICLE = np.dtype(
    [("id", "<u4"), ("pad", "<u4"), ("mass", "<f8"), ("pos", "<f8", (3,)), ("vel", "<f8", (3,))]
)
assert PARTICLE.itemsize == 64


class Params(C.Structure):
    """ForceParams (traversal_ttg.h:136-141)."""

    _fields_ = [("theta", C.c_double), ("eps2", C.c_double), ("G", C.c_double), ("use_quadrupole", C.c_int)]


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def build_oracle() -> str:
    """Compile the restatement (no reference sources needed)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    return os.path.join(HERE, "libbhoracle.so")


class Oracle:
    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "libbhoracle.so")
        if not os.path.exists(path):
            path = build_oracle()
        L = self.lib = C.CDLL(path)
        vp, sz, u32, f64 = C.c_void_p, C.c_size_t, C.c_uint32, C.c_double
        L.bho_domain.argtypes = [vp, sz, vp]
        L.bho_domain.restype = C.c_int
        L.bho_keys.argtypes = [vp, sz, vp, vp]
        L.bho_sort.argtypes = [vp, sz, vp, vp]
        L.bho_count_nodes.argtypes = [vp, vp, vp, sz, C.c_uint]
        L.bho_count_nodes.restype = sz
        L.bho_build.argtypes = [vp, vp, vp, sz, vp, C.c_uint, vp]
        L.bho_build.restype = sz
        L.bho_multipoles.argtypes = [vp, sz, vp, vp, vp, vp]
        L.bho_targets.argtypes = [vp, sz, u32, u32, vp]
        L.bho_targets.restype = sz
        L.bho_walk.argtypes = [vp, sz, vp, sz, vp, vp, vp, vp, vp, vp, vp, vp]
        L.bho_direct.argtypes = [vp, vp, vp, vp, sz, vp, sz, f64, f64, vp]
        L.bho_integrate.argtypes = [vp, sz, vp, f64, f64]
        L.bho_kinetic.argtypes = [vp, sz]
        L.bho_kinetic.restype = f64
        L.bho_potential.argtypes = [vp, sz, f64]
        L.bho_potential.restype = f64
        L.bho_step.argtypes = [vp, vp, vp, sz, vp, vp, vp, C.c_uint, u32, u32, vp, vp]
        L.bho_step.restype = C.c_int
        L.bho_read_csv.argtypes = [C.c_char_p, sz, vp, sz, C.POINTER(sz), C.POINTER(sz)]
        L.bho_read_csv.restype = C.c_int
        L.bho_write_vtk.argtypes = [vp, sz, C.c_char_p, sz]
        L.bho_write_vtk.restype = sz

    # -- pieces ---------------------------------------------------------
    def domain(self, parts: np.ndarray) -> tuple[np.ndarray, int]:
        parts = np.ascontiguousarray(parts, dtype=PARTICLE)
        out = np.zeros(4)
        bad = self.lib.bho_domain(_p(parts), len(parts), _p(out))
        return out, bad

    def keys(self, parts: np.ndarray, dom: np.ndarray) -> np.ndarray:
        parts = np.ascontiguousarray(parts, dtype=PARTICLE)
        k = np.zeros(len(parts), np.uint64)
        self.lib.bho_keys(_p(parts), len(parts), _p(np.ascontiguousarray(dom, np.float64)), _p(k))
        return k

    def sort(self, keys: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        keys = np.ascontiguousarray(keys, np.uint64)
        perm = np.zeros(len(keys), np.uint32)
        sk = np.zeros(len(keys), np.uint64)
        self.lib.bho_sort(_p(keys), len(keys), _p(perm), _p(sk))
        return perm, sk

    def build(self, sorted_keys, seg_begin, seg_n, doms, max_leaf, soa=None) -> dict:
        """Level-order octree (+ multipoles when ``soa`` = (x, y, z, m))."""
        sk = np.ascontiguousarray(sorted_keys, np.uint64)
        sb = np.ascontiguousarray(seg_begin, np.uint32)
        sn = np.ascontiguousarray(seg_n, np.uint32)
        dm = np.ascontiguousarray(doms, np.float64).reshape(-1)
        cap = self.lib.bho_count_nodes(_p(sk), _p(sb), _p(sn), len(sb), max_leaf)
        c = max(cap, 1)
        t = {
            "begin": np.zeros(c, np.uint32), "count": np.zeros(c, np.uint32),
            "first_child": np.zeros(c, np.uint32), "nchild": np.zeros(c, np.uint32),
            "leaf": np.zeros(c, np.uint32), "depth": np.zeros(c, np.uint32),
            "center": np.zeros((c, 3)), "hw": np.zeros(c), "mass": np.zeros(c),
            "com": np.zeros((c, 3)), "iab": np.zeros((c, 6)),
        }
        tree = self._tree_struct(t)
        nn = self.lib.bho_build(_p(sk), _p(sb), _p(sn), len(sb), _p(dm), max_leaf, C.byref(tree))
        assert nn == cap
        if soa is not None:
            x, y, z, m = (np.ascontiguousarray(a, np.float64) for a in soa)
            self.lib.bho_multipoles(C.byref(tree), nn, _p(x), _p(y), _p(z), _p(m))
        t["_struct"] = tree
        t["n"] = nn
        return t

    @staticmethod
    def _tree_struct(t):
        class Tree(C.Structure):
            _fields_ = [(k, C.c_void_p) for k in
                        ("begin", "count", "first_child", "nchild", "leaf", "depth",
                         "center", "hw", "mass", "com", "iab")]
        return Tree(*[t[k].ctypes.data for k in
                      ("begin", "count", "first_child", "nchild", "leaf", "depth",
                       "center", "hw", "mass", "com", "iab")])

    def targets(self, tree: dict, target_size: int, group_size: int) -> np.ndarray:
        out = np.zeros(max(tree["n"], 1), np.uint32)
        k = self.lib.bho_targets(C.byref(tree["_struct"]), tree["n"], target_size, group_size, _p(out))
        return out[:k].copy()

    def walk(self, tree, targets, soa, params_per_target, roots=None):
        x, y, z, m = (np.ascontiguousarray(a, np.float64) for a in soa)
        n = len(x)
        acc = np.zeros((n, 3))
        counts = np.zeros(2, np.uint64)
        tg = np.ascontiguousarray(targets, np.uint32)
        pr = (Params * len(tg))(*params_per_target) if not isinstance(params_per_target, C.Array) \
            else params_per_target
        rt = None if roots is None else np.ascontiguousarray(roots, np.uint32)
        self.lib.bho_walk(C.byref(tree["_struct"]), tree["n"], _p(tg), len(tg),
                          None if rt is None else _p(rt), _p(x), _p(y), _p(z), _p(m),
                          C.cast(pr, C.c_void_p), _p(acc), _p(counts))
        return acc, counts

    def direct(self, soa, idx, eps2, G=1.0) -> np.ndarray:
        x, y, z, m = (np.ascontiguousarray(a, np.float64) for a in soa)
        idx = np.ascontiguousarray(idx, np.uint32)
        out = np.zeros((len(idx), 3))
        self.lib.bho_direct(_p(x), _p(y), _p(z), _p(m), len(x), _p(idx), len(idx), eps2, G, _p(out))
        return out

    def read_csv(self, text: bytes):
        """read_csv (io.cc:122-178) of a text in memory: (particles, None), or
        (None, 0-based number of the first malformed line)."""
        n, bad = C.c_size_t(), C.c_size_t()
        cap = text.count(b"\n") + 1
        out = np.zeros(cap, PARTICLE)
        r = self.lib.bho_read_csv(text, len(text), _p(out), cap, C.byref(n), C.byref(bad))
        if r:
            return None, bad.value
        return out[: n.value].copy(), None

    def write_vtk(self, parts) -> bytes:
        """write_vtk (io.cc:180-195) as bytes."""
        parts = np.ascontiguousarray(parts, dtype=PARTICLE)
        need = self.lib.bho_write_vtk(_p(parts), len(parts), None, 0)
        buf = C.create_string_buffer(need)
        self.lib.bho_write_vtk(_p(parts), len(parts), buf, need)
        return buf.raw[:need]

    def kinetic(self, parts) -> float:
        parts = np.ascontiguousarray(parts, dtype=PARTICLE)
        return self.lib.bho_kinetic(_p(parts), len(parts))

    def potential(self, parts, G=1.0) -> float:
        parts = np.ascontiguousarray(parts, dtype=PARTICLE)
        return self.lib.bho_potential(_p(parts), len(parts), G)

    # -- whole step ----------------------------------------------------------
    def step(self, parts, *, theta, eps2, G=1.0, quad=True, max_leaf=16, group_size=256,
             target_size=16, kick_dt=0.0, drift_dt=0.0, segments=None, want_acc=False):
        """One step_particles call per segment; returns (particles, acc, counts).

        ``segments``: list of (begin, n) or None for one system.  theta,
        eps2, kick_dt, drift_dt may be scalars or per-segment sequences."""
        parts = np.array(parts, dtype=PARTICLE, copy=True)
        if segments is None:
            segments = [(0, len(parts))]
        ns = len(segments)
        sb = np.array([s[0] for s in segments], np.uint32)
        sn = np.array([s[1] for s in segments], np.uint32)

        def per(v):
            return np.broadcast_to(np.asarray(v, np.float64), (ns,)).copy()

        th, e2, kd, dd = per(theta), per(eps2), per(kick_dt), per(drift_dt)
        fp = (Params * ns)(*[Params(th[i], e2[i], G, int(quad)) for i in range(ns)])
        acc = np.zeros((len(parts), 3)) if want_acc else None
        counts = np.zeros(2, np.uint64)
        rc = self.lib.bho_step(_p(parts), _p(sb), _p(sn), ns, C.cast(fp, C.c_void_p), _p(kd), _p(dd),
                               max_leaf, group_size, target_size,
                               None if acc is None else _p(acc), _p(counts))
        if rc != 0:
            raise ValueError("non-finite particle coordinates")
        return parts, acc, counts


class Reference:
    """The reference's own build / walk / step (oracle/_ref/libbhref.so)."""

    PATH = os.environ.get("BHREF_LIB", os.path.join(HERE, "_ref", "libbhref.so"))

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(cls.PATH)

    def __init__(self, path=None):
        L = self.lib = C.CDLL(path or self.PATH)
        vp, sz, u32, f64 = C.c_void_p, C.c_size_t, C.c_uint32, C.c_double
        L.bhref_build.argtypes = [vp, sz, C.c_uint, u32]
        L.bhref_build.restype = vp
        L.bhref_free.argtypes = [vp]
        L.bhref_num_nodes.argtypes = [vp]
        L.bhref_num_nodes.restype = sz
        L.bhref_num_groups.argtypes = [vp]
        L.bhref_num_groups.restype = sz
        L.bhref_export.argtypes = [vp, vp, vp, vp, vp, vp, vp]
        L.bhref_walk.argtypes = [vp, f64, f64, f64, C.c_int, u32, vp]
        L.bhref_walk.restype = C.c_uint64
        L.bhref_step.argtypes = [vp, sz, f64, f64, f64, C.c_int, C.c_uint, u32, u32, f64, f64, vp]
        L.bhref_step.restype = C.c_int
        L.bhref_brute.argtypes = [vp, sz, f64, f64, vp]
        L.bhref_accel_from_source.argtypes = [vp, f64, vp, vp, f64, C.c_int, f64, vp]
        L.bhref_kinetic.argtypes = [vp, sz]
        L.bhref_kinetic.restype = f64
        L.bhref_potential.argtypes = [vp, sz, f64]
        L.bhref_potential.restype = f64
        L.bhref_read_csv.argtypes = [C.c_char_p, vp, sz, C.POINTER(sz), C.c_char_p, sz]
        L.bhref_read_csv.restype = C.c_int
        L.bhref_write_vtk.argtypes = [C.c_char_p, vp, sz]
        L.bhref_write_vtk.restype = C.c_int

    def read_csv(self, text: bytes):
        """The reference's read_csv on a temporary file holding `text`:
        (particles, None) or (None, the exception's message)."""
        import tempfile

        with tempfile.NamedTemporaryFile(suffix=".csv", delete=False) as f:
            f.write(text)
            path = f.name
        try:
            cap = text.count(b"\n") + 1
            out = np.zeros(cap, PARTICLE)
            n = C.c_size_t()
            err = C.create_string_buffer(4096)
            r = self.lib.bhref_read_csv(path.encode(), _p(out), cap, C.byref(n), err, 4096)
        finally:
            os.unlink(path)
        if r:
            return None, err.value.decode(errors="replace")
        return out[: n.value].copy(), None

    def write_vtk(self, parts) -> bytes:
        """The reference's write_vtk, read back as bytes."""
        import tempfile

        parts = np.ascontiguousarray(parts, dtype=PARTICLE)
        with tempfile.NamedTemporaryFile(suffix=".vtk", delete=False) as f:
            path = f.name
        try:
            if self.lib.bhref_write_vtk(path.encode(), _p(parts), len(parts)):
                raise RuntimeError("write_vtk threw")
            with open(path, "rb") as f:
                return f.read()
        finally:
            os.unlink(path)

    def build(self, parts, max_leaf, group_size) -> dict:
        parts = np.ascontiguousarray(parts, dtype=PARTICLE)
        h = self.lib.bhref_build(_p(parts), len(parts), max_leaf, group_size)
        M = self.lib.bhref_num_nodes(h)
        G = self.lib.bhref_num_groups(h)
        out_p = np.zeros(len(parts), PARTICLE)
        keys = np.zeros(len(parts), np.uint64)
        u = np.zeros((6, max(M, 1)), np.uint32)
        f = np.zeros(14 * max(M, 1))
        dom = np.zeros(4)
        groups = np.zeros(max(G, 1), np.uint32)
        self.lib.bhref_export(h, _p(out_p), _p(keys), _p(u), _p(f), _p(dom), _p(groups))
        Mx = max(M, 1)
        t = {
            "handle": h, "n": M, "particles": out_p, "keys": keys, "domain": dom,
            "groups": groups[:G],
            "begin": u[0, :M], "count": u[1, :M], "first_child": u[2, :M], "nchild": u[3, :M],
            "leaf": u[4, :M], "depth": u[5, :M],
            "center": f[:3 * Mx].reshape(Mx, 3)[:M], "hw": f[3 * Mx:4 * Mx][:M],
            "mass": f[4 * Mx:5 * Mx][:M], "com": f[5 * Mx:8 * Mx].reshape(Mx, 3)[:M],
            "iab": f[8 * Mx:14 * Mx].reshape(Mx, 6)[:M],
        }
        return t

    def walk(self, tree, theta, eps2, G=1.0, quad=True, target_size=0):
        acc = np.zeros((len(tree["particles"]), 3))
        missing = self.lib.bhref_walk(tree["handle"], theta, eps2, G, int(quad), target_size, _p(acc))
        return acc, missing

    def free(self, tree):
        if tree.get("handle"):
            self.lib.bhref_free(tree["handle"])
            tree["handle"] = None

    def step(self, parts, *, theta, eps2, G=1.0, quad=True, max_leaf=16, group_size=256,
             target_size=16, kick_dt=0.0, drift_dt=0.0):
        parts = np.array(parts, dtype=PARTICLE, copy=True)
        tm = np.zeros(3)
        rc = self.lib.bhref_step(_p(parts), len(parts), theta, eps2, G, int(quad), max_leaf,
                                 group_size, target_size, kick_dt, drift_dt, _p(tm))
        if rc != 0:
            raise RuntimeError("reference step_particles threw")
        return parts, tm

    def brute(self, parts, eps2, G=1.0):
        parts = np.ascontiguousarray(parts, dtype=PARTICLE)
        acc = np.zeros((len(parts), 3))
        self.lib.bhref_brute(_p(parts), len(parts), eps2, G, _p(acc))
        return acc

    def accel_from_source(self, target, mass, com, iab, eps2, quad, G):
        out = np.zeros(3)
        t = np.ascontiguousarray(target, np.float64)
        c = np.ascontiguousarray(com, np.float64)
        i = np.ascontiguousarray(iab, np.float64)
        self.lib.bhref_accel_from_source(_p(t), mass, _p(c), _p(i), eps2, int(quad), G, _p(out))
        return out

    def kinetic(self, parts):
        parts = np.ascontiguousarray(parts, dtype=PARTICLE)
        return self.lib.bhref_kinetic(_p(parts), len(parts))

    def potential(self, parts, G=1.0):
        parts = np.ascontiguousarray(parts, dtype=PARTICLE)
        return self.lib.bhref_potential(_p(parts), len(parts), G)


def soa(parts: np.ndarray):
    """(x, y, z, m) float64 arrays of a particle array."""
    return (np.ascontiguousarray(parts["pos"][:, 0]), np.ascontiguousarray(parts["pos"][:, 1]),
            np.ascontiguousarray(parts["pos"][:, 2]), np.ascontiguousarray(parts["mass"]))


def node_tuples(t: dict) -> list:
    """The node set, independent of numbering: (depth, begin, count, leaf, nchild)."""
    n = t["n"]
    return sorted(zip(t["depth"][:n].tolist(), t["begin"][:n].tolist(), t["count"][:n].tolist(),
                      t["leaf"][:n].tolist(), t["nchild"][:n].tolist()))


def node_order(t: dict) -> np.ndarray:
    """Permutation that sorts nodes by (depth, begin) - a numbering-free order."""
    n = t["n"]
    return np.lexsort((np.asarray(t["begin"][:n], np.int64), np.asarray(t["depth"][:n], np.int64)))
