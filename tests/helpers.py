"""Inputs and error metrics shared by the tests."""
import numpy as np

from oracle import PARTICLE, soa  # noqa: F401


def cube(n, seed, spread=10.0, centre=(0.0, 0.0, 0.0)):
    """Uniform cube with masses U(0.5, 1.5), as the reference's tests draw them
    (test_bh_vs_bruteforce.cc:15-27), from numpy's generator."""
    rng = np.random.default_rng(seed)
    p = np.zeros(n, PARTICLE)
    p["id"] = np.arange(n)
    p["mass"] = rng.uniform(0.5, 1.5, n)
    p["pos"] = rng.uniform(-spread, spread, (n, 3)) + np.asarray(centre)
    return p


def plummer_np(n, seed, a=1.0):
    """A numpy Plummer sampler for CPU-only tests (not the product generator)."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(1e-12, 1.0, n)
    r = a / np.sqrt(x ** (-2.0 / 3.0) - 1.0)
    r = np.where(r < 10 * a, r, 9.5 * a)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    p = np.zeros(n, PARTICLE)
    p["id"] = np.arange(n)
    p["mass"] = 1.0 / n
    p["pos"] = d * r[:, None]
    p["vel"] = rng.normal(size=(n, 3)) * 0.2
    return p


def rel_error(test, ref):
    """relative_error of test_bh_vs_bruteforce.cc:30-40: sqrt(sum|a-b|^2 / sum|b|^2)."""
    test = np.asarray(test)
    ref = np.asarray(ref)
    return float(np.sqrt(np.sum((test - ref) ** 2) / np.sum(ref ** 2)))


def per_particle_rel(test, ref):
    """|a - b| / |b| per particle."""
    return np.linalg.norm(np.asarray(test) - np.asarray(ref), axis=1) / np.linalg.norm(np.asarray(ref), axis=1)
