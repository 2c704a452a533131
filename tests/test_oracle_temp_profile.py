"""Moving super-Gaussian temperature profile on the oracle (suprgaus_temp,
set_sg / get_sg, applied.f90:446-483,1778-1809; get_applied's grain average,
field.f90:546-560) against a literal port of those loops, and a heat-assisted
write with the LLB integrator under the moving spot."""
import math

import numpy as np

from mrm_b200 import media


def _set_sg(expn, sig, dl, n, dd):
    """applied.f90:1778-1790 as written (i 1-based)."""
    return [math.exp(-((dd * (i - 0.5) + dl) * sig) ** expn) for i in range(1, n + 1)]


def test_profile_matches_literal_loops(oracle):
    med = media.grain_map_medium(12, 10, seed=3, temperature=300.0)
    lay = med.layers[0]
    lay.temp_profile = dict(background=310.0, dtemp=420.0, sigma=(3e-6, 5e-6), expn=2, vel=(3000.0, -800.0),
                            offset=(None, 2e-6), ref=(1e-6, 0.0), t_origin=1e-10,
                            time=dict(func=4, amp=1.0, gamma=5e-10, param=5e-11, scale=1.0))
    orc = oracle.OracleSim(med, demag=False)
    for t in (0.0, 2.3e-10, 7e-10):
        orc.eval_field(t)
        ox, oy = med.dx * med.nx * 0.5, 2e-6
        fx = _set_sg(4, 1 / 3e-6, 1e-6 - 3000.0 * (t - 1e-10) - ox, med.nx, med.dx)
        fy = _set_sg(4, 1 / 5e-6, 0.0 + 800.0 * (t - 1e-10) - oy, med.ny, med.dy)
        g, p = 5e-10, 5e-11
        x = math.fmod(t, g)
        ste = (2 * x / p if x < 0.5 * p else 1.0 if x < 0.5 * (g - p) else (g - 2 * x) / p if x < 0.5 * (g + p)
               else -1.0 if x < g - 0.5 * p else 2 * (x - g) / p)
        s = 420.0 * ste
        want = np.zeros(lay.N)
        for n in range(lay.N):
            v = 0.0
            for q in range(lay.g2c_index[n], lay.g2c_index[n + 1]):
                i, j = lay.g2c[q]
                v += s * fy[j - 1] * fx[i - 1]
            want[n] = v / (lay.g2c_index[n + 1] - lay.g2c_index[n]) + 310.0
        np.testing.assert_allclose(orc.get_temp(0), want, rtol=1e-13)
    orc.close()


def test_hamr_write_heats_and_reverses(oracle):
    # the spot heats the grains under it above Tc: their |m| collapses while the
    # cold grains keep theirs, and the heated track reverses in the field
    med = media.hamr_medium(32, seed=2, velocity_cm_s=0.0, sigma_nm=40.0)
    med.layers[0].temp_profile["offset"] = (None, None)  # the spot at the grid centre
    orc = oracle.OracleSim(med, rng_mode=1, seed=3)
    orc.step(3000, 1e-14)
    T = orc.get_temp(0)
    mag = orc.get_mag(0)
    hot, cold = T > 700.0, T < 320.0
    assert hot.any() and cold.any()
    assert mag[hot].mean() < 0.5 * mag[cold].mean()
    orc.close()
