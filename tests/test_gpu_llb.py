"""LLB integrator on the GPU (mrm_gpu_set_llb) against the oracle's
restatement of push_llb: heat-assisted trajectories with thermal noise (FP64,
FP32), grains of several cells, the mean-field equilibrium, the |m| = 0
branch, the magnitude round trip and the combinations the path refuses."""
import numpy as np
import pytest

from mrm_b200 import FP32, FP64, GpuSim, MrmError, media
from tests.helpers import rel_l2
from tests.test_oracle_llb import GMUB_KB, _find_meq, _quiet

pytestmark = pytest.mark.gpu


def _pair(oracle, med, precision, seed=5, demag=True):
    orc = oracle.OracleSim(med, rng_mode=1, seed=seed, demag=demag)
    gpu = GpuSim(med, precision=precision, demag=False, thermal_seed=seed)
    if demag:
        gpu.upload_tensor(orc.n2d)
        gpu.set_demag(True)
    return orc, gpu


def test_llb_trajectory_fp64(oracle, gpulib):
    med = media.llb_medium(16, seed=3)
    orc, gpu = _pair(oracle, med, FP64)
    for chunk in range(4):
        so = orc.step(250, 1e-14)
        sg = gpu.step(250, 1e-14)
        assert np.abs(gpu.get_state(0) - orc.get_state(0)).max() < 1e-9, chunk
        assert np.abs(gpu.get_mag(0) - orc.get_mag(0)).max() < 1e-9, chunk
    for k in ("mmag", "errmx", "errmx1", "energy"):
        assert sg[k] == pytest.approx(so[k], rel=1e-7), k
    np.testing.assert_allclose(sg["mave"], so["mave"], rtol=1e-9, atol=1e-10)
    gpu.close()
    orc.close()


@pytest.mark.parametrize("llg_type", [2, -2])
def test_llb_semi_implicit_fp64(oracle, gpulib, llg_type):
    med = media.llb_medium(16, seed=5)
    orc, gpu = _pair(oracle, med, FP64)
    orc.step(600, 1e-14, llg_type=llg_type)
    gpu.step(600, 1e-14, llg_type=llg_type)
    assert np.abs(gpu.get_state(0) - orc.get_state(0)).max() < 1e-9
    assert np.abs(gpu.get_mag(0) - orc.get_mag(0)).max() < 1e-9
    gpu.close()
    orc.close()


@pytest.mark.parametrize("meq_bs,garanin_tau", [(False, False), (True, True)])
@pytest.mark.parametrize("llg_type", [-3, 2, -2])
def test_mt_fp64(oracle, gpulib, meq_bs, garanin_tau, llg_type):
    med = media.mt_medium(16, seed=7, meq_bs=meq_bs, garanin_tau=garanin_tau)
    orc, gpu = _pair(oracle, med, FP64)
    orc.step(500, 1e-14, llg_type=llg_type)
    gpu.step(500, 1e-14, llg_type=llg_type)
    assert np.abs(gpu.get_state(0) - orc.get_state(0)).max() < 1e-9
    assert np.abs(gpu.get_mag(0) - orc.get_mag(0)).max() < 1e-9
    gpu.close()
    orc.close()


@pytest.mark.parametrize("meq_bs,garanin_tau", [(False, False), (True, True)])
@pytest.mark.parametrize("llg_type", [-3, 2, -2])
def test_zhang_fp64(oracle, gpulib, meq_bs, garanin_tau, llg_type):
    med = media.zhang_medium(16, seed=8, meq_bs=meq_bs, garanin_tau=garanin_tau)
    orc, gpu = _pair(oracle, med, FP64)
    orc.step(500, 1e-14, llg_type=llg_type)
    gpu.step(500, 1e-14, llg_type=llg_type)
    assert np.abs(gpu.get_state(0) - orc.get_state(0)).max() < 1e-9
    assert np.abs(gpu.get_mag(0) - orc.get_mag(0)).max() < 1e-9
    gpu.close()
    orc.close()


def test_llb_trajectory_fp32(oracle, gpulib):
    # the LLB push runs in FP64 arithmetic on FP32 state; FP32 runs draw their
    # noise from the 32-bit Philox stream, so the comparison runs without noise
    # (T = 600 K still sets the longitudinal physics)
    med = media.llb_medium(16, seed=4)
    med.layers[0].thermal = False
    orc, gpu = _pair(oracle, med, FP32)
    orc.step(500, 1e-14)
    gpu.step(500, 1e-14)
    assert np.abs(gpu.get_state(0) - orc.get_state(0)).max() < 1e-3
    assert np.abs(gpu.get_mag(0) - orc.get_mag(0)).max() < 1e-3
    gpu.close()
    orc.close()


def test_llb_grain_map(oracle, gpulib):
    med = media.grain_map_medium(16, 16, seed=6, temperature=600.0)
    lay = med.layers[0]
    tc = np.full(lay.N, 700.0)
    lay.llb = dict(spin=0.5, tc=tc, lambda_ms=3.0 * tc / (GMUB_KB * 1.5))
    lay.thermal, lay.temperature = True, 600.0
    orc, gpu = _pair(oracle, med, FP64)
    orc.step(500, 1e-14)
    gpu.step(500, 1e-14)
    assert np.abs(gpu.get_state(0) - orc.get_state(0)).max() < 1e-9
    assert np.abs(gpu.get_mag(0) - orc.get_mag(0)).max() < 1e-9
    gpu.close()
    orc.close()


def test_llb_equilibrium_and_zero_branch(gpulib):
    med = _quiet(media.llb_medium(8, tc=700.0, tc_sigma=0.0, temperature=560.0), 560.0)
    g = GpuSim(med, precision=FP64, demag=False)
    g.step(3000, 1e-14)
    lam = med.layers[0].llb["lambda_ms"][0] * 3.0
    np.testing.assert_allclose(g.get_mag(0), _find_meq(0.0, GMUB_KB * 0.5 * lam / 560.0), rtol=2e-5)
    g.set_mag(0, np.zeros(med.layers[0].N))
    np.testing.assert_array_equal(g.get_mag(0), 0.0)
    g.step(1, 1e-14)
    assert np.all(g.get_mag(0) >= 0.0)
    g.close()


def test_llb_refusals(gpulib):
    med = media.llb_medium(16, seed=1)
    g = GpuSim(med, precision=FP64)
    g.set_thermal(0, False, 0.0, 1)
    with pytest.raises(MrmError):
        g.step(2, 1e-14)
    g.close()
    med = media.llb_medium(16, seed=1)
    med.window = dict(nx=8, ny=16)
    g = GpuSim(med, precision=FP64)
    with pytest.raises(MrmError):
        g.step(2, 1e-14)
    g.close()
