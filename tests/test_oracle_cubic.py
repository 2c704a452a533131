"""Cubic anisotropy of the oracle (get_cubic_hk, src/field.f90:377-395)
against its energy: h = -(hk_scale / 2) grad_m w(m) with
w = K1 (a1^2 a2^2 + a1^2 a3^2 + a2^2 a3^2) + K2 a1^2 a2^2 a3^2 and a_i = m . e_i
(the crystal axes e_i), zero along every crystal axis."""
import numpy as np

from mrm_b200 import media
from oracle import pyoracle


def _cubic_only(seed=3, side=8):
    med = media.cubic_medium(side, seed=seed, hex_oe=0.0, k1_oe=4000.0, k2_oe=1500.0)
    lay = med.layers[0]
    lay.hdir = (0.0, 0.0, 0.0)  # no applied field, no exchange, no demag: h is the cubic term alone
    lay.hk_scale = np.linspace(0.5, 1.5, lay.N)
    return med, lay


def _w(m, A, k1, k2):
    a = A @ m
    a2 = a * a
    return k1 * (a2[0] * a2[1] + a2[0] * a2[2] + a2[1] * a2[2]) + k2 * a2[0] * a2[1] * a2[2]


def test_cubic_field_is_energy_gradient():
    med, lay = _cubic_only()
    rng = np.random.default_rng(7)
    m = rng.standard_normal((lay.N, 3))
    m /= np.linalg.norm(m, axis=1, keepdims=True)
    sim = pyoracle.OracleSim(med, demag=False)
    sim.set_state(0, m)
    sim.eval_field(0.0)
    h = sim.get_field(0)
    sim.close()
    eps = 1e-6
    for n in range(0, lay.N, 7):
        A, hs = lay.cubic_axis[n], lay.hk_scale[n]
        k1, k2 = lay.hk[n]
        g = np.zeros(3)
        for k in range(3):
            d = np.zeros(3)
            d[k] = eps
            g[k] = (_w(m[n] + d, A, k1, k2) - _w(m[n] - d, A, k1, k2)) / (2 * eps)
        np.testing.assert_allclose(h[n], -0.5 * hs * g, rtol=1e-7, atol=1e-6)


def test_cubic_field_zero_along_axes_and_off_for_nonpositive_scale():
    med, lay = _cubic_only(seed=5)
    lay.hk_scale[::2] = -1.0  # get_cubic_hk returns 0 for hk_scale <= 0
    m = np.array([lay.cubic_axis[n, n % 3] for n in range(lay.N)])
    sim = pyoracle.OracleSim(med, demag=False)
    sim.set_state(0, m)
    sim.eval_field(0.0)
    assert np.max(np.abs(sim.get_field(0))) < 1e-9
    m2 = np.tile(np.array([1.0, 1.0, 1.0]) / np.sqrt(3.0), (lay.N, 1))
    sim.set_state(0, m2)
    sim.eval_field(0.0)
    h = sim.get_field(0)
    sim.close()
    assert np.all(np.abs(h[::2]) == 0.0)
    assert np.all(np.linalg.norm(h[1::2], axis=1) > 0.0)
