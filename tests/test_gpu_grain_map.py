"""Grains of several cells (get_mag data.f90:322-390 scatters each grain's
Ms m over its cells; get_magnetostatic field.f90:438-517 averages the cells'
demag per grain) on the GPU path against the oracle, with empty cells and
exchange between grains sharing an edge."""
import numpy as np
import pytest

from mrm_b200 import FP32, FP64, GpuSim, media
from tests.helpers import random_m, rel_l2

pytestmark = pytest.mark.gpu


def _pair(oracle, med, precision, seed=3):
    orc = oracle.OracleSim(med, rng_mode=1, seed=seed)
    gpu = GpuSim(med, precision=precision, demag=False, thermal_seed=seed)
    if orc.n2d.shape[-2:] == tuple(reversed(gpu.fft_grid())):
        gpu.upload_tensor(orc.n2d)
    else:  # the oracle pads an open grid to 2n, this path to a power of two: each its own tensor
        gpu.build_tensor()
    gpu.set_demag(True)
    return orc, gpu


@pytest.mark.parametrize("precision,tol", [(FP64, 1e-9), (FP32, 1e-5)])
def test_grain_map_demag_and_field(oracle, gpulib, precision, tol):
    med = media.grain_map_medium(16, 16, seed=3)
    orc, gpu = _pair(oracle, med, precision)
    n = med.layers[0].N
    for k in range(2):
        m = random_m(n, 60 + k)
        orc.set_state(0, m)
        gpu.set_state(0, m)
        assert np.abs(gpu.get_state(0) - m).max() < (1e-15 if precision == FP64 else 1e-7)
        orc.eval_field(5e-11)
        assert rel_l2(gpu.eval_field(5e-11, 0), orc.get_demag(0)) < tol
        assert rel_l2(gpu.get_field(0), orc.get_field(0)) < tol


@pytest.mark.parametrize("precision,tol", [(FP64, 1e-9), (FP32, 2e-4)])
def test_grain_map_t0_trajectory(oracle, gpulib, precision, tol):
    med = media.grain_map_medium(16, 16, seed=5)
    orc, gpu = _pair(oracle, med, precision)
    for chunk in range(4):
        so = orc.step(500, 1e-13)
        sg = gpu.step(500, 1e-13)
        assert np.abs(gpu.get_state(0) - orc.get_state(0)).max() < tol, chunk
        assert np.allclose(sg["mave"], so["mave"], rtol=0, atol=tol)
    assert so["mave"][2] < 0.5  # the ramp reversed a large part of the grains
    assert sg["nup_l"][0] == so["nup_l"][0]
    assert sg["vol_l"][0] == pytest.approx(so["vol_l"][0], rel=1e-12)
    assert sg["energy"] == pytest.approx(so["energy"], rel=max(tol, 1e-9) * 50)


def test_grain_map_thermal_fp64_same_stream(oracle, gpulib):
    med = media.grain_map_medium(16, 16, seed=7, temperature=300.0)
    orc, gpu = _pair(oracle, med, FP64, seed=9)
    so = orc.step(200, 1e-13)
    sg = gpu.step(200, 1e-13)
    assert np.abs(gpu.get_state(0) - orc.get_state(0)).max() < 1e-8
    assert np.allclose(sg["mave"], so["mave"], atol=1e-9)


def test_grain_map_rejects_bad_maps(gpulib):
    from mrm_b200 import MrmError
    med = media.grain_map_medium(8, 8, seed=2)
    lay = med.layers[0]
    lay.g2c = lay.g2c.copy()
    lay.g2c[1] = lay.g2c[0]  # a cell in two grains (or twice in one)
    with pytest.raises(MrmError, match="two grains"):
        GpuSim(med, precision=FP64)


def test_grain_map_two_layers_interlayer(oracle, gpulib):
    import copy
    med = media.grain_map_medium(16, 8, seed=11)
    top = med.layers[0]
    bot = copy.deepcopy(top)
    bot.ms = np.full(bot.N, 900.0)
    bot.hk = bot.hk * 0.4
    n = top.N
    top.lhx = media.columnar_coupling(n, 1500.0)
    bot.uhx = media.columnar_coupling(n, 1500.0)
    med.layers = [top, bot]
    med.dz = [med.dz[0], 0.5 * med.dz[0]]
    med.il_space = [0.0, 0.0]
    med.m0 = [med.m0[0], med.m0[0].copy()]
    orc, gpu = _pair(oracle, med, FP64)
    so = orc.step(400, 1e-13)
    sg = gpu.step(400, 1e-13)
    for l in range(2):
        assert np.abs(gpu.get_state(l) - orc.get_state(l)).max() < 1e-9
    assert np.allclose(sg["mave_l"][:2], so["mave_l"][:2], atol=1e-10)


def test_medium_from_grain_file(oracle, gpulib, tmp_path):
    # a reference-format grain file (maps, cubic layer, interlayer coupling) on the GPU path
    from mrm_b200 import formats
    from tests.test_formats import _two_layer_map_medium
    med = _two_layer_map_medium()
    p = str(tmp_path / "grain.bin")
    formats.write_grain_file(p, formats.grain_file_layers(med), med.nx, med.ny, med.dx, med.dy)
    back = formats.medium_from_grain_file(p, med.dz, boundary=1)
    for lay, orig in zip(back.layers, med.layers):
        lay.hdir, lay.t_start, lay.t_end, lay.s_start, lay.s_end = (orig.hdir, orig.t_start, orig.t_end,
                                                                     orig.s_start, orig.s_end)
    orc, gpu = _pair(oracle, back, FP64)
    so = orc.step(300, 1e-13)
    sg = gpu.step(300, 1e-13)
    for l in range(2):
        assert np.abs(gpu.get_state(l) - orc.get_state(l)).max() < 1e-9
    assert sg["energy"] == pytest.approx(so["energy"], rel=1e-8)


@pytest.mark.parametrize("shape", [(12, 10), (16, 10), (12, 16)])
def test_non_power_of_two_grids(oracle, gpulib, shape):
    # one grain per cell on grids that are not powers of two (open boundary:
    # the oracle pads to 2n, this path to the next power of two)
    nx, ny = shape
    med = media.mh_medium(nx, ny=ny, seed=4, boundary=1)
    med.layers[0].t_end = 2e-10
    orc, gpu = _pair(oracle, med, FP64)
    m = random_m(med.layers[0].N, 3)
    orc.set_state(0, m)
    gpu.set_state(0, m)
    orc.eval_field(1e-11)
    assert rel_l2(gpu.eval_field(1e-11, 0), orc.get_demag(0)) < 1e-9
    orc.set_state(0, med.m0[0])
    gpu.set_state(0, med.m0[0])
    orc.set_time(0.0, 0)
    gpu.set_time(0.0, 0)
    orc.step(500, 1e-13)
    gpu.step(500, 1e-13)
    assert np.abs(gpu.get_state(0) - orc.get_state(0)).max() < 1e-8
