"""Cubic anisotropy (get_cubic_hk, src/field.f90:377-395) on the GPU path
against the oracle: the assembled field on random states, and T=0 Heun
trajectories through switching, with the full field (demag, exchange,
applied ramp) around it."""
import numpy as np
import pytest

from mrm_b200 import FP32, FP64, GpuSim, media
from tests.helpers import random_m, rel_l2

pytestmark = pytest.mark.gpu


def _cubic(side=16, seed=3):
    med = media.cubic_medium(side, seed=seed, k1_oe=4000.0, k2_oe=1500.0)
    lay = med.layers[0]
    lay.hk_scale = np.where(np.arange(lay.N) % 9 == 0, -1.0, np.linspace(0.6, 1.4, lay.N))  # some grains off
    lay.t_end = 2e-10  # faster ramp: switching inside 2000 steps
    return med


def _pair(oracle, med, precision):
    orc = oracle.OracleSim(med, demag=True)
    gpu = GpuSim(med, precision=precision, demag=False)
    gpu.upload_tensor(orc.n2d)
    gpu.set_demag(True)
    return orc, gpu


@pytest.mark.parametrize("precision,tol", [(FP64, 1e-12), (FP32, 1e-5)])
def test_cubic_field(oracle, gpulib, precision, tol):
    med = _cubic()
    orc, gpu = _pair(oracle, med, precision)
    for k in range(2):
        m = random_m(med.layers[0].N, 40 + k)
        orc.set_state(0, m)
        gpu.set_state(0, m)
        orc.eval_field(3e-11)
        gpu.eval_field(3e-11, 0)
        assert rel_l2(gpu.get_field(0), orc.get_field(0)) < tol
    # back to uniaxial: the same medium without the cubic axes
    gpu.set_cubic_axes(0, None)
    med_u = _cubic()
    med_u.layers[0].cubic_axis = None
    orc_u = oracle.OracleSim(med_u, demag=True)
    orc_u.set_state(0, m)
    orc_u.eval_field(3e-11)
    gpu.eval_field(3e-11, 0)
    assert rel_l2(gpu.get_field(0), orc_u.get_field(0)) < tol
    assert rel_l2(orc_u.get_field(0), orc.get_field(0)) > 1e-3  # the two anisotropies differ


@pytest.mark.parametrize("precision,tol", [(FP64, 1e-9), (FP32, 2e-4)])
def test_cubic_t0_trajectory(oracle, gpulib, precision, tol):
    med = _cubic()
    orc, gpu = _pair(oracle, med, precision)
    for chunk in range(4):
        so = orc.step(500, 1e-13)
        sg = gpu.step(500, 1e-13)
        assert np.abs(gpu.get_state(0) - orc.get_state(0)).max() < tol, chunk
        assert np.allclose(sg["mave"], so["mave"], rtol=0, atol=tol)
    assert so["mave"][2] < 0.5  # the ramp reversed a large part of the grains
    # the energy includes the cubic term with the reference's factors
    assert sg["energy"] == pytest.approx(so["energy"], rel=max(tol, 1e-9) * 50)
