"""Python binding of the B200 Barnes-Hut hot path (``libbhg.so``, include/bhg.h).

This is the host-side mirror the tests and the benchmark drive: a thin
ctypes layer over the C ABI plus :func:`step_particles`, which has the
meaning of the reference's ``bh::step_particles`` grouped branch
(integrate_ttg.h:66-148): build the tree, walk, kick/drift, and return the
particles in Morton order.  There is no CPU fallback: if ``libbhg.so`` is
missing or no GPU is present, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "libbhg.so")

#: bh::Particle (particle.h:7-24): 64 bytes, 4 bytes of padding after id.
PARTICLE = np.dtype(
    [("id", "<u4"), ("pad", "<u4"), ("mass", "<f8"), ("pos", "<f8", (3,)), ("vel", "<f8", (3,))]
)

OK, EINVAL, ECUDA, ENOMEM, ENONFINITE, ESTATE, EDEVICE, ECANCELLED, EAGAIN = range(9)
PRECISION_SPLIT, PRECISION_FP64 = 0, 1
EXPORT_KEYS, EXPORT_PERM, EXPORT_NODES_U32, EXPORT_NODES_F64, EXPORT_DOMAINS, EXPORT_TARGETS, EXPORT_ACCEL, EXPORT_GROUPS = range(1, 9)

#: Every entry point include/bhg.h declares.
EXPORTED = (
    "bhg_create", "bhg_destroy", "bhg_last_error", "bhg_set_stream", "bhg_upload", "bhg_upload_device",
    "bhg_upload_systems", "bhg_download", "bhg_download_device", "bhg_num_particles", "bhg_reserve", "bhg_add_system",
    "bhg_add_generated", "bhg_remove_systems", "bhg_num_systems", "bhg_system_ids", "bhg_upload_csv",
    "bhg_upload_csv_device", "bhg_add_csv", "bhg_snapshot_vtk", "bhg_build_tree",
    "bhg_compute_multipoles", "bhg_walk_forces", "bhg_integrate", "bhg_step", "bhg_step_systems",
    "bhg_step_systems_async", "bhg_download_async", "bhg_sync",
    "bhg_run_schedule", "bhg_set_system_params", "bhg_get_stats", "bhg_device_status", "bhg_debug_export",
    "bhg_direct_sum", "bhg_energy", "bhg_energy_noalloc", "bhg_ic_plummer", "bhg_write_csv",
    "bhg_measure_fp32_peak", "bhg_selftest_wait", "bhg_set_walk_group",
)


class BhgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"bhg error {code}: {msg}")
        self.code = code


class Sphere(C.Structure):
    _fields_ = [("n", C.c_uint64), ("a", C.c_double), ("mass", C.c_double), ("centre", C.c_double * 3),
                ("bulk", C.c_double * 3)]


class Config(C.Structure):
    _fields_ = [("device", C.c_int), ("hbm_budget", C.c_uint64), ("flags", C.c_uint32)]


class ForceParams(C.Structure):
    _fields_ = [("theta", C.c_double), ("eps2", C.c_double), ("G", C.c_double),
                ("use_quadrupole", C.c_int), ("precision", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("pre_ms", C.c_double), ("sort_ms", C.c_double), ("tree_ms", C.c_double),
                ("multipole_ms", C.c_double), ("targets_ms", C.c_double), ("walk_ms", C.c_double),
                ("last_walk_ms", C.c_double), ("pp", C.c_uint64), ("pc", C.c_uint64), ("evals", C.c_uint32),
                ("nodes", C.c_uint32), ("targets", C.c_uint32), ("depth", C.c_uint32),
                ("sort_passes", C.c_uint32), ("kernels_per_eval", C.c_uint32)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["build_ms"] = d["pre_ms"] + d["sort_ms"] + d["tree_ms"]
        return d


_lib = None


def lib() -> C.CDLL:
    """Load libbhg.so (raises if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run __graft_entry__.build() or make -C {PKG}")
    L = C.CDLL(LIB_PATH)
    vp, sz, u32, u64, f64, i32 = C.c_void_p, C.c_size_t, C.c_uint32, C.c_uint64, C.c_double, C.c_int
    sigs = {
        "bhg_create": ([C.POINTER(vp), C.POINTER(Config)], i32),
        "bhg_destroy": ([vp], i32),
        "bhg_last_error": ([vp], C.c_char_p),
        "bhg_set_stream": ([vp, vp], i32),
        "bhg_upload": ([vp, vp, sz], i32),
        "bhg_upload_device": ([vp, vp, sz], i32),
        "bhg_upload_systems": ([vp, vp, vp, sz], i32),
        "bhg_download": ([vp, vp], i32),
        "bhg_download_device": ([vp, vp], i32),
        "bhg_num_particles": ([vp], sz),
        "bhg_reserve": ([vp, sz, sz], i32),
        "bhg_add_system": ([vp, vp, sz, C.POINTER(u64)], i32),
        "bhg_add_generated": ([vp, vp, i32, u64, u32, C.POINTER(u64)], i32),
        "bhg_remove_systems": ([vp, vp, sz, vp], i32),
        "bhg_num_systems": ([vp], sz),
        "bhg_system_ids": ([vp, vp], i32),
        "bhg_upload_csv": ([vp, C.c_char_p, sz], i32),
        "bhg_upload_csv_device": ([vp, vp, sz], i32),
        "bhg_add_csv": ([vp, C.c_char_p, sz, C.POINTER(u64)], i32),
        "bhg_snapshot_vtk": ([vp, u64, C.c_char_p, sz, C.POINTER(sz)], i32),
        "bhg_build_tree": ([vp, C.c_uint, u32], i32),
        "bhg_compute_multipoles": ([vp], i32),
        "bhg_walk_forces": ([vp, C.POINTER(ForceParams), u32, f64, f64, vp, vp], i32),
        "bhg_integrate": ([vp, f64, f64], i32),
        "bhg_step": ([vp, C.POINTER(ForceParams), C.c_uint, u32, u32, f64, f64], i32),
        "bhg_step_systems": ([vp, C.POINTER(ForceParams), C.c_uint, u32, u32], i32),
        "bhg_step_systems_async": ([vp, C.POINTER(ForceParams), C.c_uint, u32, u32], i32),
        "bhg_download_async": ([vp, vp], i32),
        "bhg_sync": ([vp], i32),
        "bhg_run_schedule": ([vp, C.POINTER(ForceParams), C.c_uint, u32, u32, f64, i32], i32),
        "bhg_set_system_params": ([vp, vp, vp, vp, vp], i32),
        "bhg_get_stats": ([vp, C.POINTER(Stats), i32], i32),
        "bhg_device_status": ([vp, C.POINTER(u32)], i32),
        "bhg_debug_export": ([vp, i32, vp, sz, C.POINTER(sz)], i32),
        "bhg_direct_sum": ([vp, i32, vp, sz, f64, f64, vp], i32),
        "bhg_energy": ([vp, i32, f64, C.POINTER(f64), C.POINTER(f64)], i32),
        "bhg_energy_noalloc": ([vp, sz, f64, vp, vp], i32),
        "bhg_ic_plummer": ([vp, sz, f64, f64, vp, vp, u32, u64], u64),
        "bhg_write_csv": ([C.c_char_p, vp, sz], i32),
        "bhg_measure_fp32_peak": ([i32, C.POINTER(f64)], i32),
        "bhg_selftest_wait": ([vp, i32, u32, C.POINTER(u32)], i32),
        "bhg_set_walk_group": ([vp, u32], i32),
    }
    for name, (args, res) in sigs.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def plummer(n, seed, a=1.0, mass=1.0, centre=(0.0, 0.0, 0.0), bulk=(0.0, 0.0, 0.0), id0=0):
    """Plummer sphere (Aarseth-Henon-Wielen); returns (particles, next_seed)."""
    out = np.zeros(n, PARTICLE)
    c = np.asarray(centre, np.float64)
    b = np.asarray(bulk, np.float64)
    nxt = lib().bhg_ic_plummer(_p(out), n, a, mass, _p(c), _p(b), id0, seed)
    return out, nxt


def merger(n_each, seed, a1=1.0, a2=0.5, sep=10.0, v_rel=0.3):
    """Two Plummer spheres (M = 1 each) at x = -sep/2 and +sep/2 moving toward
    each other with relative speed v_rel; the second continues the first's
    random stream."""
    p1, nxt = plummer(n_each, seed, a=a1, mass=1.0, centre=(-sep / 2, 0, 0), bulk=(v_rel / 2, 0, 0))
    p2, _ = plummer(n_each, nxt, a=a2, mass=1.0, centre=(sep / 2, 0, 0), bulk=(-v_rel / 2, 0, 0), id0=n_each)
    return np.concatenate([p1, p2])


def write_csv(path, parts):
    parts = np.ascontiguousarray(parts, PARTICLE)
    r = lib().bhg_write_csv(path.encode(), _p(parts), len(parts))
    if r:
        raise OSError(f"cannot write {path}")


def measure_fp32_peak(device=0) -> float:
    v = C.c_double()
    r = lib().bhg_measure_fp32_peak(device, C.byref(v))
    if r:
        raise BhgError(r, "FP32 peak calibration failed")
    return v.value


class Context:
    """One device context: particles resident on the GPU between calls."""

    def __init__(self, device=0, hbm_budget=0):
        self.L = lib()
        h = C.c_void_p()
        cfg = Config(device, hbm_budget, 0)
        r = self.L.bhg_create(C.byref(h), C.byref(cfg))
        if r:
            raise BhgError(r, "bhg_create failed (no GPU?)")
        self.h = h
        self.n = 0
        self._snapbuf = None  # host buffer reused by snapshot_vtk

    def close(self):
        if self.h:
            self.L.bhg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _ck(self, r):
        if r:
            raise BhgError(r, self.L.bhg_last_error(self.h).decode())

    # -- particles --------------------------------------------------------------
    def upload(self, parts):
        parts = np.ascontiguousarray(parts, PARTICLE)
        self._ck(self.L.bhg_upload(self.h, _p(parts), len(parts)))
        self.n = len(parts)

    def upload_device(self, ptr, n):
        self._ck(self.L.bhg_upload_device(self.h, C.c_void_p(ptr), n))
        self.n = n

    def upload_systems(self, systems):
        parts = np.ascontiguousarray(np.concatenate(systems), PARTICLE)
        counts = np.array([len(s) for s in systems], np.uint64)
        self._ck(self.L.bhg_upload_systems(self.h, _p(parts), _p(counts), len(counts)))
        self.n = len(parts)

    def reserve(self, particles, systems):
        """Grows the buffers now for up to `particles` particles in up to
        `systems` systems (no allocation or state copy when systems join later)."""
        self._ck(self.L.bhg_reserve(self.h, int(particles), int(systems)))

    def add_system(self, parts) -> int:
        """Appends one system (host particles); returns its handle."""
        parts = np.ascontiguousarray(parts, PARTICLE)
        h = C.c_uint64()
        self._ck(self.L.bhg_add_system(self.h, _p(parts), len(parts), C.byref(h)))
        self.n = self.L.bhg_num_particles(self.h)
        return h.value

    def add_generated(self, spheres, seed, id0=0) -> int:
        """Appends one system generated on the device from `seed`: one or two
        spheres, each a dict with n, a, mass and optional centre, bulk."""
        arr = (Sphere * len(spheres))()
        for k, sp in enumerate(spheres):
            arr[k] = Sphere(int(sp["n"]), float(sp.get("a", 1.0)), float(sp.get("mass", 1.0)),
                            (C.c_double * 3)(*sp.get("centre", (0.0, 0.0, 0.0))),
                            (C.c_double * 3)(*sp.get("bulk", (0.0, 0.0, 0.0))))
        h = C.c_uint64()
        self._ck(self.L.bhg_add_generated(self.h, arr, len(spheres), int(seed) % (1 << 64), id0, C.byref(h)))
        self.n = self.L.bhg_num_particles(self.h)
        return h.value

    def remove_systems(self, handles, want=False, sizes=None):
        """Removes systems by handle.  want: also return their particles, a
        list of arrays (sizes: their particle counts, in the same order)."""
        hs = np.ascontiguousarray(handles, np.uint64)
        out = None
        if want:
            out = np.zeros(int(sum(sizes)), PARTICLE)
        self._ck(self.L.bhg_remove_systems(self.h, _p(hs), len(hs), None if out is None else _p(out)))
        self.n = self.L.bhg_num_particles(self.h)
        if out is None:
            return None
        return np.split(out, np.cumsum(sizes)[:-1])

    def upload_csv(self, text: bytes):
        """The particles of a CSV text (read_csv's format), parsed on the GPU,
        as the only system."""
        self._ck(self.L.bhg_upload_csv(self.h, text, len(text)))
        self.n = self.L.bhg_num_particles(self.h)

    def upload_csv_device(self, ptr: int, nbytes: int):
        """upload_csv for text at a device address of this context's GPU."""
        self._ck(self.L.bhg_upload_csv_device(self.h, C.c_void_p(ptr), nbytes))
        self.n = self.L.bhg_num_particles(self.h)

    def add_csv(self, text: bytes) -> int:
        """The same, appended as one more system; returns its handle."""
        h = C.c_uint64()
        self._ck(self.L.bhg_add_csv(self.h, text, len(text), C.byref(h)))
        self.n = self.L.bhg_num_particles(self.h)
        return h.value

    def snapshot_vtk(self, handle=None) -> bytes:
        """write_vtk's text of a system (the first when handle is None),
        formatted on the GPU."""
        if handle is None:
            handle = int(self.system_ids()[0])
        # one call, into a buffer of the largest possible size, kept for the
        # next snapshot (its pages are then already mapped); the bytes object
        # is a copy
        cap = self.snapshot_vtk_bound()
        if self._snapbuf is None or len(self._snapbuf) < cap:
            self._snapbuf = np.zeros(cap, np.uint8)
        n = self.snapshot_vtk_into(self._snapbuf, handle)
        return self._snapbuf[:n].tobytes()

    def snapshot_vtk_bound(self) -> int:
        """Bytes that always hold a snapshot of this context's largest system:
        three lines of at most 98 bytes per particle, plus the headers."""
        return 98 * int(self.n) + 512

    def snapshot_vtk_into(self, out: np.ndarray, handle=None) -> int:
        """write_vtk's text of a system written into the caller's uint8 array
        (pinned memory takes the fastest copy); returns the bytes written."""
        if handle is None:
            handle = int(self.system_ids()[0])
        n = C.c_size_t()
        self._ck(self.L.bhg_snapshot_vtk(self.h, handle, out.ctypes.data_as(C.c_char_p), out.nbytes, C.byref(n)))
        return n.value

    def system_ids(self) -> np.ndarray:
        out = np.zeros(self.L.bhg_num_systems(self.h), np.uint64)
        if len(out):
            self._ck(self.L.bhg_system_ids(self.h, _p(out)))
        return out

    def download(self) -> np.ndarray:
        out = np.zeros(self.n, PARTICLE)
        self._ck(self.L.bhg_download(self.h, _p(out)))
        return out

    def download_into(self, out: np.ndarray):
        self._ck(self.L.bhg_download(self.h, _p(out)))

    def set_stream(self, handle: int):
        self._ck(self.L.bhg_set_stream(self.h, C.c_void_p(handle)))

    # -- phases -------------------------------------------------------------------
    @staticmethod
    def params(theta, eps2, G=1.0, quad=True, precision=PRECISION_SPLIT):
        return ForceParams(theta, eps2, G, int(bool(quad)), precision)

    def build_tree(self, max_leaf, group_size):
        self._ck(self.L.bhg_build_tree(self.h, max_leaf, group_size))

    def compute_multipoles(self):
        self._ck(self.L.bhg_compute_multipoles(self.h))

    def walk_forces(self, fp, target_size, kick_dt=0.0, drift_dt=0.0, want_accel=True):
        acc = np.zeros((self.n, 3)) if want_accel else None
        missing = C.c_uint64()
        self._ck(self.L.bhg_walk_forces(self.h, C.byref(fp), target_size, kick_dt, drift_dt,
                                        None if acc is None else _p(acc), C.byref(missing)))
        return acc

    def integrate(self, kick_dt, drift_dt):
        self._ck(self.L.bhg_integrate(self.h, kick_dt, drift_dt))

    def step(self, fp, max_leaf, group_size, target_size, kick_dt, drift_dt):
        self._ck(self.L.bhg_step(self.h, C.byref(fp), max_leaf, group_size, target_size, kick_dt, drift_dt))

    def step_systems(self, fp, max_leaf, group_size, target_size):
        self._ck(self.L.bhg_step_systems(self.h, C.byref(fp), max_leaf, group_size, target_size))

    def step_systems_async(self, fp, max_leaf, group_size, target_size):
        """Enqueues one evaluation of every system and returns; sync() reports it."""
        self._ck(self.L.bhg_step_systems_async(self.h, C.byref(fp), max_leaf, group_size, target_size))

    def download_async(self, out_ptr: int):
        """Enqueues the copy of the particles to host address out_ptr (pinned
        memory: the call does not block); valid after sync()."""
        self._ck(self.L.bhg_download_async(self.h, C.c_void_p(out_ptr)))

    def sync(self):
        """Waits for the context's stream; raises for the enqueued evaluations
        that did not run (EAGAIN: node slots regrown, run them again)."""
        self._ck(self.L.bhg_sync(self.h))

    def run_schedule(self, fp, max_leaf, group_size, target_size, dt, steps):
        self._ck(self.L.bhg_run_schedule(self.h, C.byref(fp), max_leaf, group_size, target_size, dt, steps))

    def set_system_params(self, theta=None, eps2=None, kick_dt=None, drift_dt=None):
        arrs = [None if v is None else np.ascontiguousarray(v, np.float64) for v in (theta, eps2, kick_dt, drift_dt)]
        self._ck(self.L.bhg_set_system_params(self.h, *[None if a is None else _p(a) for a in arrs]))

    def stats(self, reset=True) -> dict:
        """Phase times and interaction counts summed since the last reset."""
        s = Stats()
        self._ck(self.L.bhg_get_stats(self.h, C.byref(s), int(reset)))
        return s.as_dict()

    def device_status(self) -> int:
        v = C.c_uint32()
        self._ck(self.L.bhg_device_status(self.h, C.byref(v)))
        return v.value

    def export(self, what):
        size = C.c_size_t()
        self._ck(self.L.bhg_debug_export(self.h, what, None, 0, C.byref(size)))
        buf = np.zeros(size.value, np.uint8)
        self._ck(self.L.bhg_debug_export(self.h, what, _p(buf), size.value, C.byref(size)))
        if what == EXPORT_KEYS:
            return buf.view(np.uint64)
        if what in (EXPORT_PERM, EXPORT_TARGETS, EXPORT_GROUPS):
            return buf.view(np.uint32)
        if what == EXPORT_NODES_U32:
            u = buf.view(np.uint32).reshape(6, -1)
            return {"begin": u[0], "count": u[1], "first_child": u[2], "nchild": u[3], "leaf": u[4], "depth": u[5],
                    "n": u.shape[1]}
        if what == EXPORT_NODES_F64:
            d = buf.view(np.float64).reshape(-1, 14)
            return {"center": d[:, 0:3], "hw": d[:, 3], "mass": d[:, 4], "com": d[:, 5:8], "iab": d[:, 8:14]}
        if what == EXPORT_DOMAINS:
            return buf.view(np.float64).reshape(-1, 4)
        if what == EXPORT_ACCEL:
            return buf.view(np.float64).reshape(-1, 3)
        return buf

    def tree(self) -> dict:
        """Nodes of the last build (level order) with their multipoles."""
        t = self.export(EXPORT_NODES_U32)
        t.update(self.export(EXPORT_NODES_F64))
        return t

    def direct_sum(self, idx, eps2, G=1.0, system=0):
        idx = np.ascontiguousarray(idx, np.uint32)
        out = np.zeros((len(idx), 3))
        self._ck(self.L.bhg_direct_sum(self.h, system, _p(idx), len(idx), eps2, G, _p(out)))
        return out

    #: warps per block of the walk kernels (a compile-time shape)
    WALK_WARPS = 4

    def set_walk_shape(self, group_particles=0, warps=0):
        """The walk's shape: the particle cap of a walk group (0 = default 64);
        warps per block is fixed at WALK_WARPS (0 or that value)."""
        if warps not in (0, self.WALK_WARPS):
            raise ValueError(f"the walk kernels run {self.WALK_WARPS} warps per block")
        self._ck(self.L.bhg_set_walk_group(self.h, group_particles))

    def selftest_wait(self, publish_first: bool, spin_limit: int):
        """bhg_selftest_wait: (status code, prefix) of the bounded look-back
        wait run on a prepared array whose first tile publishes or never does."""
        pre = C.c_uint32()
        r = self.L.bhg_selftest_wait(self.h, 1 if publish_first else 0, spin_limit, C.byref(pre))
        return r, pre.value

    def last_error(self) -> str:
        return (self.L.bhg_last_error(self.h) or b"").decode(errors="replace")

    def energy(self, G=1.0, system=0):
        k, p = C.c_double(), C.c_double()
        self._ck(self.L.bhg_energy(self.h, system, G, C.byref(k), C.byref(p)))
        return k.value, p.value


def step_particles(particles, theta, eps2, G=1.0, use_quadrupole=True, max_leaf=8, group_size=256,
                   target_size=32, kick_dt=0.0, drift_dt=0.0, precision=PRECISION_SPLIT, workspace=None):
    """bh::step_particles, grouped branch (integrate_ttg.h:66-148), on the GPU.

    Takes and returns a particle array; the result is in Morton order, as
    the reference returns it.  ``workspace`` (a :class:`Context`) keeps the
    device storage between calls like ``GroupedWorkspace``."""
    ctx = workspace if workspace is not None else Context()
    ctx.upload(particles)
    fp = Context.params(theta, eps2, G, use_quadrupole, precision)
    ctx.step(fp, max_leaf, group_size, target_size, kick_dt, drift_dt)
    return ctx.download()


def ensemble(nsys=512, seed=3, nmin=1024, nmax=262144):
    """Independent Plummer systems (M = a = 1 each) with N log-uniform in
    [nmin, nmax]: N_s = round(exp(U(ln nmin, ln nmax))) and per-system seeds,
    both from numpy's PCG64 stream `seed`.  Returns a list of particle arrays."""
    ns, seeds = ensemble_specs(nsys, seed, nmin, nmax)
    return [plummer(int(n), int(sd))[0] for n, sd in zip(ns, seeds)]


def ensemble_specs(nsys=512, seed=3, nmin=1024, nmax=262144):
    """The sizes and generator seeds of :func:`ensemble`'s systems (numpy only:
    loads nothing of the GPU library)."""
    rng = np.random.default_rng(seed)
    ns = np.rint(np.exp(rng.uniform(np.log(nmin), np.log(nmax), nsys))).astype(np.int64)
    seeds = rng.integers(1, 2**63 - 1, nsys)
    return ns, seeds
