"""bhg_energy_noalloc, the energy diagnostic for callers that cannot allocate
GPU memory (their memory pool already owns the device, or they cannot afford
the device-wide synchronisation of cudaFree): called through the C ABI with
caller-owned device buffers, it must give what bhg_energy gives and what the
oracle's kinetic/potential energies give, on two calls in a row (the calls
share one fixed scratch array in the library), up to the largest size the
array allows, on a caller's stream and on the default stream, without
changing the device's free memory.

Kept in its own file, collected last."""
import ctypes as C

import numpy as np
import pytest

import bhg

pytestmark = pytest.mark.gpu

MAX_N = 262144  # 1,024 blocks of 256: the whole fixed array


def _dev_buffers(parts):
    import torch

    dev = torch.device("cuda", 0)
    src = torch.from_numpy(np.ascontiguousarray(parts).view(np.uint8).copy()).to(dev)
    res = torch.zeros(2, dtype=torch.float64, device=dev)
    return src, res


def _call(src, res, n, stream, G=1.0):
    rc = bhg.lib().bhg_energy_noalloc(C.c_void_p(src.data_ptr()), n, G, C.c_void_p(res.data_ptr()),
                                      None if stream is None else C.c_void_p(stream.cuda_stream))
    assert rc == bhg.OK


def _noalloc(parts, G=1.0, default_stream=False):
    import torch

    src, res = _dev_buffers(parts)
    stream = None if default_stream else torch.cuda.current_stream(0)
    torch.cuda.synchronize(0)
    _call(src, res, len(parts), stream, G)
    torch.cuda.synchronize(0)
    return res.cpu().numpy()


def test_energy_noalloc_matches_energy_twice():
    import torch

    torch.cuda.init()
    ctx = bhg.Context(device=0)
    for seed, n in ((5, 3000), (6, 20000)):
        parts, _ = bhg.plummer(n, seed)
        ctx.upload(parts)
        k, p = ctx.energy(G=1.0)
        got = _noalloc(parts)
        assert abs(got[0] - k) <= 1e-12 * abs(k)
        assert abs(got[1] - p) <= 1e-12 * abs(p)
    ctx.close()


def test_energy_noalloc_matches_oracle(oracle):
    parts, _ = bhg.plummer(3000, 9)
    for default_stream in (False, True):
        got = _noalloc(parts, G=1.0, default_stream=default_stream)
        assert abs(got[0] - oracle.kinetic(parts)) <= 1e-12 * abs(got[0])
        assert abs(got[1] - oracle.potential(parts)) <= 1e-12 * abs(got[1])


def test_energy_noalloc_at_the_array_limit():
    """n = 262,144 fills all 1,024 partial-sum slots; compared with bhg_energy,
    twice in a row, once on a caller's stream and once on the default stream."""
    parts, _ = bhg.plummer(MAX_N, 17)
    with bhg.Context(device=0) as ctx:
        ctx.upload(parts)
        k, p = ctx.energy(G=1.0)
    for default_stream in (False, True):
        got = _noalloc(parts, default_stream=default_stream)
        assert abs(got[0] - k) <= 1e-12 * abs(k)
        assert abs(got[1] - p) <= 1e-12 * abs(p)


def test_energy_noalloc_leaves_free_memory_unchanged():
    """After a first call (which may load the library's kernels), further
    calls change the device's free memory by nothing."""
    import torch

    parts, _ = bhg.plummer(50000, 3)
    src, res = _dev_buffers(parts)
    stream = torch.cuda.current_stream(0)
    _call(src, res, len(parts), stream)
    torch.cuda.synchronize(0)
    free0, _ = torch.cuda.mem_get_info(0)
    outs = []
    for _ in range(3):
        _call(src, res, len(parts), stream)
        torch.cuda.synchronize(0)
        outs.append(res.cpu().numpy().copy())
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0
    assert outs[0].tobytes() == outs[1].tobytes() == outs[2].tobytes()


def test_energy_noalloc_rejects_too_many_particles():
    parts = np.zeros(MAX_N + 1, bhg.PARTICLE)
    rc = bhg.lib().bhg_energy_noalloc(C.c_void_p(parts.ctypes.data), len(parts), 1.0, C.c_void_p(16), None)
    assert rc == bhg.EINVAL
