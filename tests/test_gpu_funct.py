"""The GPU path's applied-field time functions (SIN, COS, EXP, STE, NEW, ROT;
src/applied.f90:328-396) against the oracle: total field at several times
and FP64 trajectories on the same Philox stream."""
import numpy as np
import pytest

from mrm_b200 import FP64, GpuSim
from tests.test_oracle_funct import CODES, with_function

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("func", list(CODES))
def test_time_function_field_and_trajectory(oracle, gpulib, func):
    med = with_function(func, seed=5)
    med.layers[0].temperature = 300.0
    med.layers[0].thermal = True
    orc = oracle.OracleSim(med, rng_mode=1, seed=7)
    gpu = GpuSim(med, precision=FP64, thermal_seed=7, tensor=orc.n2d)
    for t in (0.0, 4.1e-11, 1.234e-10):
        orc.eval_field(t)
        gpu.eval_field(t, 0)
        assert np.abs(gpu.get_field(0) - orc.get_field(0)).max() < 1e-8, (func, t)
    so = orc.step(300, 1e-13)
    sg = gpu.step(300, 1e-13)
    assert np.abs(gpu.get_state(0) - orc.get_state(0)).max() < 1e-8, func
    assert np.allclose(sg["have"], so["have"], rtol=1e-8, atol=1e-6), func
    gpu.close()
    orc.close()


def test_rot_following_the_magnetisation_is_refused(gpulib):
    from mrm_b200 import FP32, MrmError
    med = with_function("ROT")
    gpu = GpuSim(med, precision=FP32)
    with pytest.raises(MrmError):
        gpu.set_field_function(0, (1.0, 0.0, 0.0), 7, 1.0, 1.0)
    gpu.close()
