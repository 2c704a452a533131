"""Closed-form checks of the restated tensor (tensor_element.f90, tensor.f90)."""
import math

import numpy as np
import pytest


def test_cube_self_term(oracle):
    n = oracle.volume_averaged_n(0, 0, 0, 1, 1, 1, 1, 1, 1)
    assert np.allclose(np.diag(n), -4 * math.pi / 3, rtol=1e-12)
    assert np.allclose(n - np.diag(np.diag(n)), 0, atol=1e-12)


@pytest.mark.parametrize("dims", [(8e-7, 8e-7, 10e-7), (7e-7, 7e-7, 4e-7), (1.0, 1.0, 3.0)])
def test_self_term_trace(oracle, dims):
    dx, dy, dz = dims
    n = oracle.volume_averaged_n(0, 0, 0, dx, dy, dz, dx, dy, dz) / (dx * dy * dz)
    assert abs(np.trace(n) / (-4 * math.pi) - 1) < 1e-10


def test_far_field_is_dipolar(oracle):
    d = 1.0
    for r in [(10.0, 3.0, 0.0), (0.0, 12.0, 2.0), (7.0, -9.0, 1.0)]:
        n = oracle.volume_averaged_n(*r, d, d, d, d, d, d)  # source - observation
        rv = np.array(r)
        rr = np.linalg.norm(rv)
        dip = (3 * np.outer(rv, rv) - rr**2 * np.eye(3)) / rr**5  # V_s * V_o / V_o
        assert np.allclose(n, dip, rtol=0, atol=2e-2 * np.abs(dip).max())


def test_tensor_symmetry_and_parity(oracle):
    nx = ny = 16
    T = oracle.calculate_tensor(nx, ny, 8e-7, 8e-7, [10e-7], [0.0], 0)[0, 0]
    # c = 3*field + source: N_ab == N_ba (t(2,1)=t(1,2) etc., tensor_element.f90:52-62)
    for a in range(3):
        for b in range(3):
            assert np.array_equal(T[3 * a + b], T[3 * b + a])
    # parity under offset reflection: xx, yy, zz even; xy odd in x and y; xz, yz vanish at rz=0
    idx = (-np.arange(nx)) % nx
    scale = np.abs(T[0]).max()
    assert np.allclose(T[0][:, idx], T[0], atol=1e-9 * scale)
    assert np.allclose(T[1][:, idx], -T[1], atol=1e-9 * scale)
    assert np.allclose(T[1][idx, :], -T[1], atol=1e-9 * scale)
    assert np.abs(T[2]).max() < 1e-9 * scale


def test_periodic_film_sum_rule(oracle):
    # sum of N_zz over the plane (2 image pairs) ~ -4 pi for a thin film
    nx = ny = 32
    dx, dz = 8e-7, 10e-7
    T = oracle.calculate_tensor(nx, ny, dx, dx, [dz], [0.0], 2)[0, 0]
    s = T.reshape(9, -1).sum(axis=1) * nx * ny  # normalisation 1/(dx dy dz nx ny) undone per cell volume
    assert abs(s[8] / (-4 * math.pi) - 1) < 0.01
    assert abs(s[0]) < 0.05 and abs(s[4]) < 0.05


def test_normalisation(oracle):
    nx, ny = 8, 8
    dx, dz = 8e-7, 10e-7
    T = oracle.calculate_tensor(nx, ny, dx, dx, [dz], [0.0], 0)[0, 0]
    # slot (0,0) is the self term / (dx dy dz nx ny)
    n = oracle.volume_averaged_n(0, 0, 0, dx, dx, dz, dx, dx, dz)
    assert np.allclose(T[:, 0, 0].reshape(3, 3).T, n / (dx * dx * dz * nx * ny), rtol=1e-12)
