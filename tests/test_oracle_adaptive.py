"""The oracle's adaptive time step (llg.f90:240-269, get_fields :363-388,
push_m :1195-1271): the first dt from the field magnitude, the rotation bound
of every accepted step, t as the sum of the steps taken."""
import math

import numpy as np

from mrm_b200 import media
from oracle import pyoracle


def _medium(temperature=0.0):
    med = media.mh_medium(16, boundary=1, temperature=temperature, seed=2)
    med.layers[0].t_end = 2e-10
    return med


def test_first_dt_from_field_magnitude():
    med = _medium()
    lay = med.layers[0]
    sim = pyoracle.OracleSim(med)
    sim.eval_field(0.0)
    hmax = np.linalg.norm(sim.get_field(0), axis=1).max()
    dt_frac, dt_max = 0.2, 1e-8
    fact1 = (1 + lay.alpha ** 2) / ((1 + lay.alpha) * lay.gamma) * dt_frac
    st, dt, md = sim.step_adaptive(1, 1e-14, 1.0, dt_frac=dt_frac, dt_max=dt_max, max_dm=[math.pi])
    sim.close()
    assert dt == fact1 / max(1.0, hmax)  # no retry at max_dm = pi: the step taken is dt * 1
    assert st["t"] == dt and st["step"] == 1
    r = math.acos(1 - 0.5 * st["errmx1_l"][0]) / math.pi
    assert md == (min(2.0, 1.0 / (r + 1e-200)) if r < 2 / 3 else 1.0)


def test_rotation_bound_and_time():
    sim = pyoracle.OracleSim(_medium(temperature=300.0), rng_mode=1, seed=4)
    dt, md, t = 1e-14, 1.0, 0.0
    max_dm = 0.03
    retries = 0
    for k in range(30):
        st, dt2, md2 = sim.step_adaptive(1, dt, md, max_dm=[max_dm])
        assert math.acos(1 - 0.5 * st["errmx1_l"][0]) <= max_dm * (1 + 1e-12)
        t += dt2
        assert st["t"] == t
        retries += md2 < md
        dt, md = dt2, md2
    sim.close()
    assert retries > 0  # the bound was active
