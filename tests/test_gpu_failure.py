"""The device failure path: a kernel whose bounded wait for its bulk copies
runs out raises the engine's error flag and returns (no trap, no hang); the
host reports MRM_ERR_DEVICE at its next synchronisation, clears the flag, and
the handle keeps working.  mrm_gpu_selftest_timeout makes the wait run out on
purpose (a barrier that expects bytes no copy sends); nothing faults."""
import numpy as np
import pytest

from tests.helpers import small_medium

pytestmark = pytest.mark.gpu

MRM_ERR_DEVICE = 6


@pytest.mark.parametrize("prec_name", ["fp32", "fp64"])
def test_wait_runs_out_and_handle_recovers(gpulib, prec_name):
    from mrm_b200 import FP32, FP64, GpuSim

    precision = FP32 if prec_name == "fp32" else FP64
    med = small_medium(32, boundary=1, temperature=300.0)
    sim = GpuSim(med, precision=precision, thermal_seed=4)
    sim.step(20, 1e-13)
    m_before, h_before = sim.get_state(0), sim.get_field(0)

    rc = gpulib.mrm_gpu_selftest_timeout(sim.h)
    assert rc == MRM_ERR_DEVICE
    assert b"a bulk-copy wait ran out" in gpulib.mrm_gpu_last_error(sim.h)
    # the failed launch wrote nothing: state and stored field as they were
    assert np.array_equal(sim.get_state(0), m_before)
    assert np.array_equal(sim.get_field(0), h_before)
    # the flag was cleared on that report; the handle steps on as a fresh one does
    assert gpulib.mrm_gpu_check_device(sim.h) == 0
    sim.step(30, 1e-13)
    assert gpulib.mrm_gpu_check_device(sim.h) == 0
    ref = GpuSim(med, precision=precision, thermal_seed=4)
    ref.step(50, 1e-13)
    assert np.array_equal(sim.get_state(0), ref.get_state(0))
    sim.close()
    ref.close()
