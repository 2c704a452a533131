"""The analytic-rotation push (llg_type 1 and -1, src/llg.f90:1093-1107) in the
oracle: for a grain in a constant field (no anisotropy, exchange or demag) it
is the exact solution of the LLG equation whatever the time step --
precession at gamma H / (1 + alpha^2) and tan(theta/2) decaying as
exp(-alpha gamma H t / (1 + alpha^2))."""
import math

import numpy as np
import pytest

from mrm_b200 import media


def _free_spins(h_oe=10000.0, theta0=math.radians(60.0)):
    med = media.mh_medium(4, hk=0.0, k_sigma=0.0, hex_oe=0.0, seed=2)
    lay = med.layers[0]
    lay.hdir = (0.0, 0.0, 1.0)
    lay.t_start, lay.t_end, lay.s_start, lay.s_end, lay.scale = 0.0, 1.0, h_oe, h_oe, 1.0
    m0 = np.tile([math.sin(theta0), 0.0, math.cos(theta0)], (lay.N, 1))
    med.m0 = [m0]
    return med, lay


@pytest.mark.parametrize("llg_type", [1, -1])
@pytest.mark.parametrize("dt", [1e-13, 2e-12])
def test_rotation_is_exact_in_a_constant_field(oracle, llg_type, dt):
    h, theta0 = 10000.0, math.radians(60.0)
    med, lay = _free_spins(h, theta0)
    orc = oracle.OracleSim(med, demag=False)
    nsteps = 150
    orc.step(nsteps, dt, llg_type=llg_type)
    m = orc.get_state(0)
    t = nsteps * dt
    a, g = lay.alpha, lay.gamma
    theta = 2.0 * math.atan(math.tan(0.5 * theta0) * math.exp(-a * g * h * t / (1 + a * a)))
    phi = g * h * t / (1 + a * a)
    exact = np.array([math.sin(theta) * math.cos(phi), math.sin(theta) * math.sin(phi), math.cos(theta)])
    assert np.abs(m - exact).max() < 1e-10
    assert theta < theta0  # the damping turned the spins towards the field
    orc.close()


def test_heun_is_not_exact_at_large_steps(oracle):
    """The same spins under Heun at the large step differ from the exact
    solution: the rotation push's exactness is its own."""
    h, theta0 = 10000.0, math.radians(60.0)
    med, lay = _free_spins(h, theta0)
    orc = oracle.OracleSim(med, demag=False)
    orc.step(150, 2e-12, llg_type=-3)
    t = 150 * 2e-12
    a, g = lay.alpha, lay.gamma
    theta = 2.0 * math.atan(math.tan(0.5 * theta0) * math.exp(-a * g * h * t / (1 + a * a)))
    assert abs(math.acos(orc.get_state(0)[0, 2]) - theta) > 1e-6
    orc.close()
