"""Moving demag window on the GPU (mrm_gpu_set_window) against the oracle's
restatement of window_m / update_do_grain and the do_grain masks: a
stationary window (open and periodic boundary, thermal noise), the window
following a tabulated write head down a longer track, the llg_type 2 push,
the window's origin, and the combinations the path refuses."""
import numpy as np
import pytest

from mrm_b200 import FP32, FP64, GpuSim, MrmError, media
from mrm_b200.batch import Batch

pytestmark = pytest.mark.gpu


def _pair(oracle, med, precision, seed=3):
    orc = oracle.OracleSim(med, rng_mode=1, seed=seed)
    gpu = GpuSim(med, precision=precision, demag=False, thermal_seed=seed)
    gpu.upload_tensor(orc.n2d)
    gpu.set_demag(True)
    return orc, gpu


def _close(*sims):
    for s in sims:
        s.close()


@pytest.mark.parametrize("boundary", [1, 0])
def test_stationary_window(oracle, gpulib, boundary):
    med = media.mh_medium(32, ny=16, seed=3, boundary=boundary, temperature=300.0)
    med.window = dict(nx=16, ny=8, v=(0.0, 0.0), offset=(1.1e-6, -0.7e-6))
    orc, gpu = _pair(oracle, med, FP64)
    so = orc.step(600, 1e-13)
    sg = gpu.step(600, 1e-13)
    assert gpu.get_window() == orc.get_window()
    assert np.abs(gpu.get_state(0) - orc.get_state(0)).max() < 1e-9
    for k in ("mave", "have"):
        np.testing.assert_allclose(sg[k], so[k], rtol=1e-9, atol=1e-9)
    for k in ("mmag", "energy", "errmx", "errmx1"):
        assert sg[k] == pytest.approx(so[k], rel=1e-8), k
    assert sg["vol_l"][0] == pytest.approx(so["vol_l"][0], rel=1e-14)
    assert sg["nup_l"][0] == so["nup_l"][0]
    _close(orc, gpu)


@pytest.mark.parametrize("precision,tol", [(FP64, 1e-9), (FP32, 1e-3)])
def test_window_follows_write_head(oracle, gpulib, precision, tol):
    """A 128-column two-layer track written by the tabulated head at 4 km/s with a
    32-column window that follows it (window offset -nx dx/2: centred on the
    head); the window moves every few steps, the grains it leaves freeze."""
    med = media.table_write_medium(128, 16, seed=2, temperature=0.0, velocity_cm_s=4e5, bit_nm=280.0)
    med.window = dict(nx=32, ny=16, v=(4e5, 0.0), offset=(-0.5 * 128 * med.dx, 0.0))
    orc, gpu = _pair(oracle, med, precision)
    origins = set()
    for chunk in range(6):
        so = orc.step(250, 1e-13)
        sg = gpu.step(250, 1e-13)
        assert gpu.get_window() == orc.get_window(), chunk
        origins.add(orc.get_window()[2])
        for l in range(2):
            assert np.abs(gpu.get_state(l) - orc.get_state(l)).max() < tol, (chunk, l)
    assert len(origins) >= 4  # the window travelled
    if precision == FP64:
        np.testing.assert_allclose(sg["have_l"][:2], so["have_l"][:2], rtol=1e-7, atol=1e-6)
        assert sg["mmag"] == pytest.approx(so["mmag"], rel=1e-9)
    for l in range(2):
        assert np.mean((gpu.get_state(l)[:, 2] < 0) != (orc.get_state(l)[:, 2] < 0)) <= 0.01
    _close(orc, gpu)


@pytest.mark.parametrize("llg_type", [-3, 2, -2])
def test_window_moving_all_pushes(oracle, gpulib, llg_type):
    # 40 steps per cell: the window's edge lands on an exact half cell every 40
    # steps, where only the accumulated time (t = t + dt, as llg() keeps it)
    # decides the move
    med = media.mh_medium(32, ny=16, seed=7, boundary=1, temperature=300.0)
    med.window = dict(nx=16, ny=16, v=(2e5, 0.0), offset=(-1.0e-5, 0.0))
    orc, gpu = _pair(oracle, med, FP64)
    for chunk in range(4):
        orc.step(100, 1e-13, llg_type=llg_type)
        gpu.step(100, 1e-13, llg_type=llg_type)
        assert gpu.get_window() == orc.get_window(), chunk
        assert np.abs(gpu.get_state(0) - orc.get_state(0)).max() < 1e-9, chunk
    assert orc.get_window()[2] >= 4
    _close(orc, gpu)


def test_window_refusals(gpulib):
    med = media.grain_map_medium(16, 16, seed=1)
    g = GpuSim(med, precision=FP64, demag=False)
    with pytest.raises(MrmError):
        g.set_window(8, 8)
    g.close()
    med = media.mh_medium(16, seed=1)
    med.window = dict(nx=8, ny=8)
    g = GpuSim(med, precision=FP64)
    with pytest.raises(MrmError):
        g.step_adaptive(2, 1e-13)
    g.close()
    b = Batch(FP64, 0)
    r = b.add(media.mh_medium(16, seed=2), dt=1e-13, steps=10)
    with pytest.raises(MrmError):
        r.set_window(8, 8)
    b.close()


def test_window_long_track(oracle, gpulib):
    # a 4096-column track, whose own FFT (8192 wide) exceeds the path's limits,
    # computes through a 64-column window that follows the tabulated head
    # (the head starts 100 cells in, the window centred on it: origin 67 at
    # t = 0, about 29 cells further after the 500 steps)
    med = media.table_write_medium(4096, 8, seed=4, temperature=0.0, velocity_cm_s=4e5, bit_nm=280.0)
    for lay in med.layers:
        lay.field_table["offset"] = (100 * med.dx, None)
    med.window = dict(nx=64, ny=8, v=(4e5, 0.0), offset=(-1948 * med.dx, 0.0))
    orc, gpu = _pair(oracle, med, FP64)
    assert gpu.get_window()[2] == 67
    for chunk in range(2):
        orc.step(250, 1e-13)
        gpu.step(250, 1e-13)
        assert gpu.get_window() == orc.get_window(), chunk
        for l in range(2):
            assert np.abs(gpu.get_state(l) - orc.get_state(l)).max() < 1e-9, (chunk, l)
    assert orc.get_window()[2] >= 90
    _close(orc, gpu)
    med.window = None
    with pytest.raises(MrmError):  # no window: no demag on this grid
        GpuSim(med, precision=FP64)
