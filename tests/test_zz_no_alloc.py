"""bhg_energy_noalloc, the energy diagnostic for callers that cannot allocate
GPU memory (their memory pool already owns the device, or they cannot afford
the device-wide synchronisation of cudaFree): called through the C ABI with
caller-owned device buffers, it must give what bhg_energy gives, on two calls
in a row (the calls share one fixed scratch array in the library).

Kept in its own file, collected last."""
import ctypes as C

import numpy as np
import pytest

import bhg

pytestmark = pytest.mark.gpu


def _noalloc(parts, G=1.0):
    import torch

    dev = torch.device("cuda", 0)
    src = torch.from_numpy(np.ascontiguousarray(parts).view(np.uint8).copy()).to(dev)
    res = torch.zeros(2, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    rc = bhg.lib().bhg_energy_noalloc(C.c_void_p(src.data_ptr()), len(parts), G, C.c_void_p(res.data_ptr()),
                                      C.c_void_p(stream.cuda_stream))
    assert rc == bhg.OK
    stream.synchronize()
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


def test_energy_noalloc_rejects_too_many_particles():
    parts = np.zeros(262145, bhg.PARTICLE)
    rc = bhg.lib().bhg_energy_noalloc(C.c_void_p(parts.ctypes.data), len(parts), 1.0, C.c_void_p(16), None)
    assert rc == bhg.EINVAL
