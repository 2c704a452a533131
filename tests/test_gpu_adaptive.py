"""Adaptive time step on the GPU path (mrm_gpu_step_adaptive) against the
oracle's restatement of llg()'s adaptive loop: FP64 at T = 300 K on the same
Philox stream (dt sequence, time, state), including retries; FP32 at T = 0."""
import numpy as np
import pytest

from mrm_b200 import FP32, FP64, GpuSim, media

pytestmark = pytest.mark.gpu


def _medium(temperature):
    med = media.mh_medium(16, boundary=1, temperature=temperature, seed=2)
    med.layers[0].t_end = 2e-10
    return med


def _pair(oracle, med, precision, seed=4):
    orc = oracle.OracleSim(med, rng_mode=1, seed=seed)
    gpu = GpuSim(med, precision=precision, demag=False, thermal_seed=seed)
    gpu.upload_tensor(orc.n2d)
    gpu.set_demag(True)
    return orc, gpu


def test_adaptive_fp64_thermal(oracle, gpulib):
    orc, gpu = _pair(oracle, _medium(300.0), FP64)
    a = b = (1e-14, 1.0)
    retries = 0
    for k in range(8):
        so, *a2 = orc.step_adaptive(10, *a, max_dm=[0.03])
        sg, *b2 = gpu.step_adaptive(10, *b, max_dm=[0.03])
        # the same decisions from FP64 values that agree to rounding (2e-16 measured)
        assert b2[0] == pytest.approx(a2[0], rel=1e-11), k
        assert b2[1] == pytest.approx(a2[1], rel=1e-11), k
        assert sg["t"] == pytest.approx(so["t"], rel=1e-12)
        assert sg["step"] == so["step"] == 10 * (k + 1)
        assert np.abs(gpu.get_state(0) - orc.get_state(0)).max() < 1e-10
        retries += a2[1] < a[1]
        a, b = tuple(a2), tuple(b2)
    assert retries > 0  # the rotation bound was active


def test_adaptive_fp32_t0(oracle, gpulib):
    orc, gpu = _pair(oracle, _medium(0.0), FP32)
    a = b = (1e-14, 1.0)
    for k in range(5):
        so, *a = orc.step_adaptive(40, *a, max_dm=[0.1])
        sg, *b = gpu.step_adaptive(40, *b, max_dm=[0.1])
    assert sg["t"] == pytest.approx(so["t"], rel=1e-3)
    assert np.abs(gpu.get_state(0) - orc.get_state(0)).max() < 1e-3
