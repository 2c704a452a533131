"""Tabulated (moving) applied-field profile on the GPU (mrm_gpu_set_field_table)
against the oracle's restatement of set / interpolate / get_applied: the
field at several times, trajectories of a moving tabulated write head (one
grain per cell and grains of several cells), FP32, and a profile read from a
field file."""
import numpy as np
import pytest

from mrm_b200 import FP32, FP64, GpuSim, formats, media
from tests.helpers import random_m, rel_l2

pytestmark = pytest.mark.gpu


def _moving_table(med, seed=3):
    rng = np.random.default_rng(seed)
    half_x, half_y = 0.4 * med.nx * med.dx, 0.4 * med.ny * med.dy
    xp = np.sort(rng.uniform(-half_x, half_x, 11))
    yp = np.sort(rng.uniform(-half_y, half_y, 7))
    v = rng.normal(scale=3000.0, size=(7, 11, 3))
    for lay in med.layers:
        lay.field_table = dict(xpos=xp, ypos=yp, vfld=v, vel=(4000.0, -1500.0), offset=(None, 1e-6),
                               ref=(5e-7, 0.0), t_origin=2e-11)
        lay.func, lay.amp, lay.fgamma, lay.param, lay.dc, lay.scale = 4, 1.2, 3e-10, 4e-11, 0.05, 1.0
    return med


def _pair(oracle, med, precision, seed=3, demag=True):
    orc = oracle.OracleSim(med, rng_mode=1, seed=seed, demag=demag)
    gpu = GpuSim(med, precision=precision, demag=False, thermal_seed=seed)
    if demag:
        gpu.upload_tensor(orc.n2d)
        gpu.set_demag(True)
    return orc, gpu


@pytest.mark.parametrize("mapped", [False, True])
def test_table_field_at_times(oracle, gpulib, mapped):
    med = media.grain_map_medium(16, 16, seed=4) if mapped else media.mh_medium(16, seed=4, boundary=1)
    _moving_table(med)
    orc, gpu = _pair(oracle, med, FP64, demag=False)
    m = random_m(med.layers[0].N, 5)
    orc.set_state(0, m)
    gpu.set_state(0, m)
    for t in (0.0, 1.3e-10, 4.4e-10):
        orc.eval_field(t)
        gpu.eval_field(t, 0)
        assert rel_l2(gpu.get_field(0), orc.get_field(0)) < 1e-12
    gpu.close()
    orc.close()


@pytest.mark.parametrize("mapped", [False, True])
def test_table_trajectory_fp64(oracle, gpulib, mapped):
    med = media.grain_map_medium(16, 16, seed=6, temperature=300.0) if mapped else \
        media.mh_medium(16, seed=6, boundary=1, temperature=300.0)
    _moving_table(med)
    orc, gpu = _pair(oracle, med, FP64)
    for sim in (orc, gpu):
        sim.set_state(0, med.m0[0])
        sim.set_time(0.0, 0)
    so = orc.step(1500, 1e-13)
    sg = gpu.step(1500, 1e-13)
    assert np.abs(gpu.get_state(0) - orc.get_state(0)).max() < 1e-8
    assert abs(sg["energy"] - so["energy"]) <= 1e-8 * abs(so["energy"])
    gpu.close()
    orc.close()


# As for the analytic head: grains switching under the moving head amplify
# rounding near their switching field (FP32 per-component tolerance 1e-3 after
# 1,000 steps; the written pattern must agree within 1 % of the grains).
@pytest.mark.parametrize("precision,tol", [(FP64, 1e-9), (FP32, 1e-3)])
def test_table_write_two_layers(oracle, gpulib, precision, tol):
    """The tabulated write head of table_write_medium sweeping the 64-column
    grid (4 km/s, alternating 280 nm bits from the STE time function), T = 0."""
    med = media.table_write_medium(64, 16, seed=2, temperature=0.0, velocity_cm_s=4e5, bit_nm=280.0)
    orc, gpu = _pair(oracle, med, precision)
    for chunk in range(4):
        so = orc.step(250, 1e-13)
        sg = gpu.step(250, 1e-13)
        for l in range(2):
            assert np.abs(gpu.get_state(l) - orc.get_state(l)).max() < tol, (chunk, l)
    assert np.allclose(sg["have_l"][:2], so["have_l"][:2], rtol=max(tol, 1e-9) * 50, atol=1e-6)
    assert (orc.get_state(0)[:, 2] < 0).mean() > 0.05
    for l in range(2):
        assert np.mean((gpu.get_state(l)[:, 2] < 0) != (orc.get_state(l)[:, 2] < 0)) <= 0.01
    gpu.close()
    orc.close()


def test_table_from_field_file(oracle, gpulib, tmp_path):
    med = media.mh_medium(32, seed=8, boundary=1)
    xp, yp, v = media.tabulated_head_profile(25e-7, 12e-7, 15000.0, 16 * med.dy)
    p = str(tmp_path / "head.dat")
    formats.write_field_file(p, xp, yp, v)
    xf, yf, vf = formats.read_field_file(p)
    lay = med.layers[0]
    lay.s_start = lay.s_end = lay.scale = 1.0
    lay.field_table = dict(xpos=xf, ypos=yf, vfld=vf, vel=(2000.0, 0.0), offset=(0.0, None), ref=(0.0, 0.0),
                           t_origin=0.0)
    orc, gpu = _pair(oracle, med, FP64)
    orc.step(1000, 1e-13)
    gpu.step(1000, 1e-13)
    assert np.abs(gpu.get_state(0) - orc.get_state(0)).max() < 1e-8
    gpu.set_field_table(0, None, None, None)  # removed: back to the uniform field
    gpu.close()
    orc.close()
