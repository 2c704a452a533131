"""Shared helpers of the parity tests (media, random states, norms)."""
import numpy as np

from mrm_b200 import media


def random_m(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def rel_l2(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def small_medium(nx=16, ny=None, boundary=1, seed=3, temperature=0.0, hex_oe=500.0, ms=700.0):
    m = media.mh_medium(nx, ny=ny, boundary=boundary, seed=seed, temperature=temperature,
                        hex_oe=hex_oe, ms=ms)
    return m


def two_layer(nx=16, ny=8, seed=5, temperature=0.0, boundary=1):
    return media.two_layer_medium(nx, ny, seed=seed, temperature=temperature, boundary=boundary)
