"""The oracle's FFT demag (demag.f90:33-135) against a direct FP64 summation
with the same real-space tensor."""
import numpy as np
import pytest

from tests.helpers import random_m, rel_l2, small_medium, two_layer


def _grid(sim, medium, l):
    px, py = sim.px, sim.py
    m = sim.get_state(l)
    g = np.zeros((3, py, px))
    for n in range(medium.layers[l].N):
        i, j = medium.layers[l].g2c[n] - 1
        g[:, j, i] = medium.layers[l].ms[n] * m[n]
    return g


@pytest.mark.parametrize("boundary", [0, 1])
def test_fft_demag_vs_direct(oracle, boundary):
    med = small_medium(16, boundary=boundary)
    sim = oracle.OracleSim(med)
    sim.set_state(0, random_m(256, 2))
    sim.eval_field(0.0)
    hd = sim.get_demag(0)
    mg = _grid(sim, med, 0)[None]
    obs = np.array([[i, j] for j in range(16) for i in range(16)], np.int32)
    hdir = oracle.demag_direct(sim.n2d, mg, obs, 0)
    assert rel_l2(hd, hdir) < 1e-12


def test_fft_demag_two_layers(oracle):
    med = two_layer(8, 8)
    sim = oracle.OracleSim(med)
    for l in range(2):
        sim.set_state(l, random_m(64, 10 + l))
    sim.eval_field(0.0)
    mg = np.stack([_grid(sim, med, l) for l in range(2)])
    obs = np.array([[i, j] for j in range(8) for i in range(8)], np.int32)
    for ko in range(2):
        assert rel_l2(sim.get_demag(ko), oracle.demag_direct(sim.n2d, mg, obs, ko)) < 1e-12


def test_uniform_film_perpendicular(oracle):
    # uniform Mz with periodic images: H_z = Mz * sum(N_zz) ~ -4 pi Mz, H_x = H_y = 0
    med = small_medium(32, boundary=0, ms=700.0)
    sim = oracle.OracleSim(med)
    m = np.zeros((1024, 3))
    m[:, 2] = 1.0
    sim.set_state(0, m)
    sim.eval_field(0.0)
    hd = sim.get_demag(0)
    assert np.allclose(hd[:, 2], hd[0, 2], rtol=1e-10)
    assert abs(hd[0, 2] / (-4 * np.pi * 700.0) - 1) < 0.01
    assert np.abs(hd[:, :2]).max() < 1e-6 * abs(hd[0, 2])
