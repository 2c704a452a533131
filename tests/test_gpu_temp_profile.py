"""Moving super-Gaussian temperature profile on the GPU
(mrm_gpu_set_temp_profile) against the oracle: a heat-assisted LLB write under
the moving spot with thermal noise, and an LLG layer whose thermal variance
follows the spot."""
import numpy as np
import pytest

from mrm_b200 import FP64, GpuSim, media

pytestmark = pytest.mark.gpu


def _pair(oracle, med, seed=3):
    orc = oracle.OracleSim(med, rng_mode=1, seed=seed)
    gpu = GpuSim(med, precision=FP64, demag=False, thermal_seed=seed)
    gpu.upload_tensor(orc.n2d)
    gpu.set_demag(True)
    return orc, gpu


@pytest.mark.parametrize("llg_type", [-3, -2])
def test_hamr_llb_write(oracle, gpulib, llg_type):
    med = media.hamr_medium(32, seed=2, velocity_cm_s=4e5, sigma_nm=40.0)
    med.layers[0].temp_profile["time"] = dict(func=0, t_start=0.0, t_end=2e-11, s_start=0.2, s_end=1.0, scale=1.0)
    orc, gpu = _pair(oracle, med)
    for chunk in range(3):
        orc.step(250, 1e-14, llg_type=llg_type)
        gpu.step(250, 1e-14, llg_type=llg_type)
        assert np.abs(gpu.get_state(0) - orc.get_state(0)).max() < 1e-9, chunk
        assert np.abs(gpu.get_mag(0) - orc.get_mag(0)).max() < 1e-9, chunk
    gpu.close()
    orc.close()


def test_llg_thermal_follows_spot(oracle, gpulib):
    med = media.mh_medium(32, seed=5, boundary=1, temperature=300.0)
    med.layers[0].temp_profile = dict(background=300.0, dtemp=300.0, sigma=(6e-6, 6e-6), expn=1, vel=(2e5, 0.0),
                                      offset=(0.0, None))
    orc, gpu = _pair(oracle, med)
    orc.step(600, 1e-13)
    gpu.step(600, 1e-13)
    assert np.abs(gpu.get_state(0) - orc.get_state(0)).max() < 1e-9
    gpu.close()
    orc.close()
