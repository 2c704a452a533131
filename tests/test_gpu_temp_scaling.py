"""Temperature scaling on the GPU (mrm_gpu_set_temp_scaling) against the
oracle's find_temp_scaling (temp_scaling.f90:365-430): HAMR trajectories of
an LLG layer (power laws and tables; Heun, the semi-implicit push and its
midpoint form) and of an LLB layer (Ms from |m|) on the same Philox stream,
the FP32 path, the batched form, the host library's table reduction and the
combination the path refuses."""
import numpy as np
import pytest

from mrm_b200 import FP32, FP64, GpuSim, MrmError, media
from mrm_b200.batch import Batch
from tests.test_oracle_temp_scaling import TABLES, _hamr_llg, reduce_literal

pytestmark = pytest.mark.gpu

FAST = 1.0e5  # spot speed (cm/s): 40 nm over the 400-step window, so T(t) moves between stages


def _pair(oracle, med, precision, seed=5):
    orc = oracle.OracleSim(med, rng_mode=1, seed=seed)
    gpu = GpuSim(med, precision=precision, demag=False, thermal_seed=seed)
    gpu.upload_tensor(orc.n2d)
    gpu.set_demag(True)
    return orc, gpu


@pytest.mark.parametrize("llg_type", [-3, -2, 2])
def test_llg_hamr_fp64(oracle, gpulib, llg_type):
    tables = {2: TABLES["unsorted with a triple"], 3: TABLES["kelvin"]}
    med = _hamr_llg(16, vel=FAST, msexp=0.35, tables=tables)
    orc, gpu = _pair(oracle, med, FP64)
    for chunk in range(4):
        so = orc.step(100, 1e-13, llg_type)
        sg = gpu.step(100, 1e-13, llg_type)
        assert np.abs(gpu.get_state(0) - orc.get_state(0)).max() < 1e-8, chunk
    assert (orc.get_scales(0)[0] == 0.0).any()  # grains above Tc were on the path
    np.testing.assert_allclose(sg["mave"], so["mave"], rtol=1e-8, atol=1e-10)
    for k in ("mmag", "energy"):
        assert sg[k] == pytest.approx(so[k], rel=1e-7), k
    gpu.close()
    orc.close()


def test_hk_power_law_ms_table_fp64(oracle, gpulib):
    med = _hamr_llg(16, vel=FAST, hkexp=1.7, tables={1: TABLES["equal ends trimmed"]})
    orc, gpu = _pair(oracle, med, FP64)
    for chunk in range(3):
        orc.step(100, 1e-13)
        gpu.step(100, 1e-13)
        assert np.abs(gpu.get_state(0) - orc.get_state(0)).max() < 1e-8, chunk
    gpu.close()
    orc.close()


def test_llb_hamr_ms_from_magnitude_fp64(oracle, gpulib):
    med = media.hamr_medium(16, seed=4, velocity_cm_s=FAST)
    lay = med.layers[0]
    lay.temp_scaling = dict(tc=lay.llb["tc"], use_mag=True, hkexp=2.0, tables={2: TABLES["kelvin"]})
    orc, gpu = _pair(oracle, med, FP64, seed=3)
    for chunk in range(4):
        so = orc.step(250, 1e-14)
        sg = gpu.step(250, 1e-14)
        assert np.abs(gpu.get_state(0) - orc.get_state(0)).max() < 1e-8, chunk
        assert np.abs(gpu.get_mag(0) - orc.get_mag(0)).max() < 1e-8, chunk
    assert sg["mmag"] == pytest.approx(so["mmag"], rel=1e-7)
    gpu.close()
    orc.close()


def test_llg_hamr_fp32_deterministic(oracle, gpulib):
    tables = {2: TABLES["unsorted with a triple"], 3: TABLES["kelvin"]}
    med = _hamr_llg(16, vel=FAST, msexp=0.35, tables=tables)
    for lay in med.layers:
        lay.thermal = False
    orc, gpu = _pair(oracle, med, FP32)
    for chunk in range(4):
        orc.step(100, 1e-13)
        gpu.step(100, 1e-13)
        assert np.abs(gpu.get_state(0) - orc.get_state(0)).max() < 2e-3, chunk
    gpu.close()
    orc.close()


def test_batched_equals_alone(gpulib):
    med = _hamr_llg(16, vel=FAST, msexp=0.35, tables={3: TABLES["kelvin"]})
    plain = media.mh_medium(16, seed=9, temperature=300.0)
    b = Batch(FP64)
    r1 = b.add(med, dt=1e-13, steps=150, thermal_seed=7)
    r2 = b.add(plain, dt=1e-13, steps=150, thermal_seed=8)
    b.step(150)
    for r, m, sd in ((r1, med, 7), (r2, plain, 8)):
        g = GpuSim(m, precision=FP64, thermal_seed=sd)
        g.step(150, 1e-13)
        assert np.array_equal(r.get_state(0), g.get_state(0))
        g.close()
    b.close()


@pytest.mark.parametrize("name", sorted(TABLES))
def test_host_table_reduction(gpulib, name):
    temps, scales = TABLES[name]
    med = _hamr_llg(8, tables={3: (temps, scales)})
    gpu = GpuSim(med, precision=FP64)
    tt, vv = gpu.get_temp_scaling_table(0, 3)
    lt, lv = reduce_literal(temps, scales)
    np.testing.assert_array_equal(tt, lt)
    np.testing.assert_array_equal(vv, lv)
    gpu.close()


def test_refusals(gpulib):
    med = _hamr_llg(8, msexp=0.5)
    med.layers[0].ms_scale = med.layers[0].ms_scale.copy()
    med.layers[0].ms_scale[3] = 0.9  # the reference's scales start at 1 and only this scaling moves them
    with pytest.raises(MrmError, match="upload them as 1"):
        GpuSim(med, precision=FP64)


def _csr_exchange(lay):
    """A CSR exchange that the 4-neighbour lattice form cannot hold: every
    grain also couples to its diagonal neighbour (i+1, j+1)."""
    nx, ny = lay.nx, lay.ny
    idx, gr, cf = lay.hx_index, lay.hx_grain, lay.hx
    new_idx, new_gr, new_cf = [0], [], []
    for g in range(lay.N):
        i, j = g % nx, g // nx
        new_gr.extend(gr[idx[g]:idx[g + 1]])
        new_cf.extend(cf[idx[g]:idx[g + 1]])
        new_gr.append(((j + 1) % ny) * nx + (i + 1) % nx + 1)
        new_cf.append(120.0)
        new_idx.append(len(new_gr))
    lay.hx_index = np.array(new_idx, np.int32)
    lay.hx_grain = np.array(new_gr, np.int32)
    lay.hx = np.array(new_cf, float)


def test_csr_exchange_fp64(oracle, gpulib):
    """The neighbours' scales on the CSR form of the exchange."""
    med = _hamr_llg(16, vel=FAST, msexp=0.35, tables={3: TABLES["kelvin"]})
    _csr_exchange(med.layers[0])
    orc, gpu = _pair(oracle, med, FP64)
    for chunk in range(3):
        orc.step(100, 1e-13)
        gpu.step(100, 1e-13)
        assert np.abs(gpu.get_state(0) - orc.get_state(0)).max() < 1e-8, chunk
    assert (orc.get_scales(0)[0] == 0.0).any()
    gpu.close()
    orc.close()
