"""The analytic-rotation push (llg_type 1 and -1, src/llg.f90:1093-1107) on the
GPU: exact for free spins in a constant field, and against the oracle on a
medium with demag, anisotropy and exchange through switching and at
T = 300 K on the same Philox stream."""
import math

import numpy as np
import pytest

from mrm_b200 import FP32, FP64, GpuSim
from tests.helpers import small_medium, two_layer
from tests.test_oracle_rotation import _free_spins

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("llg_type", [1, -1])
def test_free_spins_exact(gpulib, llg_type):
    h, theta0 = 10000.0, math.radians(60.0)
    med, lay = _free_spins(h, theta0)
    gpu = GpuSim(med, precision=FP64, demag=False)
    gpu.step(150, 2e-12, llg_type=llg_type)
    t = 150 * 2e-12
    a, g = lay.alpha, lay.gamma
    theta = 2.0 * math.atan(math.tan(0.5 * theta0) * math.exp(-a * g * h * t / (1 + a * a)))
    phi = g * h * t / (1 + a * a)
    exact = np.array([math.sin(theta) * math.cos(phi), math.sin(theta) * math.sin(phi), math.cos(theta)])
    assert np.abs(gpu.get_state(0) - exact).max() < 1e-10
    gpu.close()


# FP32: the push is FP64 arithmetic on the FP32 state and field; grains near
# their switching field amplify the FP32 rounding of the field over the 2,000
# steps (measured 3.2e-3 at the end of the ramp), so the per-component
# tolerance is 5e-3, and the mean magnetisation's 1e-3
@pytest.mark.parametrize("llg_type", [1, -1])
@pytest.mark.parametrize("precision,tol", [(FP64, 1e-9), (FP32, 5e-3)])
def test_rotation_t0_trajectory(oracle, gpulib, llg_type, precision, tol):
    med = small_medium(16, boundary=1)
    med.layers[0].t_end = 2e-10
    orc = oracle.OracleSim(med)
    gpu = GpuSim(med, precision=precision, tensor=orc.n2d)
    for chunk in range(4):
        so = orc.step(500, 1e-13, llg_type=llg_type)
        sg = gpu.step(500, 1e-13, llg_type=llg_type)
        assert np.abs(gpu.get_state(0) - orc.get_state(0)).max() < tol, chunk
        assert np.abs(sg["mave"] - so["mave"]).max() < max(tol / 5, 1e-10), chunk
    assert so["mave"][2] < 0.5  # the ramp reversed a large part of the grains
    for key in ("errmx", "errmx1", "mmag"):
        assert sg[key] == pytest.approx(so[key], rel=max(tol, 1e-9) * 50, abs=1e-30), key
    gpu.close()
    orc.close()


@pytest.mark.parametrize("llg_type", [1, -1])
def test_rotation_thermal_two_layers_fp64(oracle, gpulib, llg_type):
    med = two_layer(16, 8, temperature=300.0)
    orc = oracle.OracleSim(med, rng_mode=1, seed=4)
    gpu = GpuSim(med, precision=FP64, thermal_seed=4, tensor=orc.n2d)
    orc.step(150, 1e-13, llg_type=llg_type)
    gpu.step(150, 1e-13, llg_type=llg_type)
    for l in range(2):
        assert np.abs(gpu.get_state(l) - orc.get_state(l)).max() < 1e-8
    gpu.close()
    orc.close()
