"""The batched form with this path's wider features: LLB runs, a tabulated
write field and an LLG run beside an LLB run, each stepped in one batch
against the same runs stepped alone."""
import numpy as np
import pytest

from mrm_b200 import FP64, GpuSim, media
from mrm_b200.batch import Batch

pytestmark = pytest.mark.gpu


def _alone(med, n, dt, seed):
    g = GpuSim(med, precision=FP64, thermal_seed=seed)
    g.step(n, dt)
    out = [g.get_state(l) for l in range(med.n_lay)]
    mag = g.get_mag(0)
    g.close()
    return out, mag


def test_llb_runs_batched(gpulib):
    meds = [media.llb_medium(16, seed=1), media.llb_medium(32, seed=2)]
    n, dt = 300, 1e-14
    alone = [_alone(m, n, dt, 11 + i) for i, m in enumerate(meds)]
    b = Batch(FP64)
    runs = [b.add(m, dt=dt, steps=n, thermal_seed=11 + i) for i, m in enumerate(meds)]
    b.step(n)
    for r, (ms, mag) in zip(runs, alone):
        assert np.array_equal(r.get_state(0), ms[0])
        assert np.array_equal(r.get_mag(0), mag)
    b.close()


def test_table_and_llg_beside_llb(gpulib):
    tab = media.table_write_medium(32, 16, seed=3, temperature=300.0, velocity_cm_s=4e5, bit_nm=280.0)
    llg = media.mh_medium(16, seed=4, temperature=300.0)
    llb = media.llb_medium(16, seed=5)
    n, dt = 200, 1e-14
    alone = [_alone(m, n, dt, 21 + i) for i, m in enumerate((tab, llg, llb))]
    b = Batch(FP64)
    runs = [b.add(m, dt=dt, steps=n, thermal_seed=21 + i) for i, m in enumerate((tab, llg, llb))]
    b.step(n)
    # the batch runs every run with the kernels its LLB run needs: the other
    # runs take the same arithmetic in another instantiation
    for r, m, (ms, _) in zip(runs, (tab, llg, llb), alone):
        for l in range(m.n_lay):
            np.testing.assert_allclose(r.get_state(l), ms[l], rtol=0, atol=1e-12)
    b.close()
