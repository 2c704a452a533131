"""LLB integrator on the oracle (push_llb, llg.f90:916-1064): the longitudinal
relaxation to the mean-field equilibrium |m| that find_meq (llg.f90:712-725)
solves, the paramagnetic decay above Tc, the |m| = 0 branch, and the thermal
variance over |m| (get_thermal, field.f90:416-417)."""
import math

import numpy as np
import pytest

from mrm_b200 import media

GMUB_KB = 1.343427768e-4


def _lv(x):
    return 1.0 / math.tanh(x) - 1.0 / x if abs(x) > 1e-2 else x / 3.0


def _find_meq(heff, hx):
    """find_meq (llg.f90:712-725): b = lv(heff + hx b) by bisection."""
    b0, b1 = 0.0, 1.0
    while b1 - b0 > 1e-13:
        b = 0.5 * (b0 + b1)
        if b > _lv(heff + hx * b):
            b1 = b
        else:
            b0 = b
    return 0.5 * (b0 + b1)


def _quiet(med, temperature):
    # no applied field, no anisotropy, no exchange, no noise: only the
    # longitudinal (mean-field) term acts
    for lay in med.layers:
        lay.scale = 0.0
        lay.hk[:] = 0.0
        lay.hx = np.zeros_like(lay.hx)
        lay.thermal = False
        lay.temperature = temperature
    return med


@pytest.mark.parametrize("ratio", [0.5, 0.8, 0.95])
def test_relaxes_to_mean_field_equilibrium(oracle, ratio):
    med = _quiet(media.llb_medium(8, tc=700.0, tc_sigma=0.0, temperature=700.0 * ratio), 700.0 * ratio)
    orc = oracle.OracleSim(med, demag=False)
    orc.step(3000, 1e-14)
    lam = med.layers[0].llb["lambda_ms"][0] * 1.5 / 0.5
    T = 700.0 * ratio
    want = _find_meq(0.0, GMUB_KB * 0.5 * lam / T)
    np.testing.assert_allclose(orc.get_mag(0), want, rtol=2e-5)
    orc.close()


def test_paramagnetic_above_tc(oracle):
    med = _quiet(media.llb_medium(8, tc=700.0, tc_sigma=0.0, temperature=650.0), 800.0)
    orc = oracle.OracleSim(med, demag=False)
    orc.step(4000, 1e-14)
    assert orc.get_mag(0).max() < 1e-3
    orc.close()


def test_zero_magnitude_branch(oracle):
    # |m| = 0 (llg.f90:1048-1060): the direction follows h and |m| takes
    # (y/s2 + lv(meq)) (1 - exp(-2 gamma dt s2 2 T alpha/(3 Tc)))
    med = _quiet(media.llb_medium(4, tc=700.0, tc_sigma=0.0, temperature=600.0), 600.0)
    lay = med.layers[0]
    lay.scale = 1.0
    lay.s_start = lay.s_end = 5000.0
    orc = oracle.OracleSim(med, demag=False)
    orc.set_mag(0, np.zeros(lay.N))
    orc.step(1, 1e-14)
    hdir = np.asarray(lay.hdir, float)
    np.testing.assert_allclose(orc.get_state(0), np.tile(hdir / np.linalg.norm(hdir), (lay.N, 1)), rtol=1e-12)
    y = 5000.0 * np.linalg.norm(hdir)
    lam = lay.llb["lambda_ms"][0] * 3.0
    meq = GMUB_KB * 0.5 * y / 600.0
    dlv = 1.0 / 3.0 if abs(meq) <= 4e-3 else 1.0 / meq ** 2 - 1.0 / math.sinh(meq) ** 2
    s2 = lam * 600.0 / (3.0 * dlv * 700.0)
    want = (y / s2 + _lv(meq)) * (1.0 - math.exp(2.0 * (-0.5 * lay.gamma * 1e-14) * s2 * 2.0 * 600.0 * lay.alpha /
                                                 (3.0 * 700.0)))
    np.testing.assert_allclose(orc.get_mag(0), want, rtol=1e-12)
    orc.close()


def test_thermal_llb_runs_and_reverses(oracle):
    # the heat-assisted medium at T/Tc ~ 0.86 with noise and a reversing field:
    # |m| stays near its equilibrium and the layer starts to reverse
    med = media.llb_medium(16, seed=3)
    orc = oracle.OracleSim(med, rng_mode=1, seed=5)
    st = orc.step(2000, 1e-14)
    mag = orc.get_mag(0)
    assert np.isfinite(orc.get_state(0)).all() and 0.2 < mag.mean() < 0.7
    assert st["mave"][2] < 0.95
    assert st["mmag"] == pytest.approx(mag @ med.layers[0].vol / med.layers[0].vol.sum(), rel=1e-12)
    orc.close()


@pytest.mark.parametrize("llg_type", [2, -2])
def test_semi_implicit_relaxes_to_equilibrium(oracle, llg_type):
    # push_llb's |type| = 2 branch (llg.f90:935-999) reaches the same
    # mean-field magnitude as the Heun branch
    med = _quiet(media.llb_medium(8, tc=700.0, tc_sigma=0.0, temperature=560.0), 560.0)
    orc = oracle.OracleSim(med, demag=False)
    orc.step(3000, 1e-14, llg_type=llg_type)
    lam = med.layers[0].llb["lambda_ms"][0] * 3.0
    np.testing.assert_allclose(orc.get_mag(0), _find_meq(0.0, GMUB_KB * 0.5 * lam / 560.0), rtol=2e-5)
    orc.close()


def _bs(x, s):
    b = x / (2.0 * s)
    if b != 0.0:
        b = ((2.0 * s + 1.0) / math.tanh((2.0 * s + 1.0) * b) - 1.0 / math.tanh(b)) / (2.0 * s)
    return b


@pytest.mark.parametrize("kind", ["mt", "zhang"])
@pytest.mark.parametrize("meq_bs", [False, True])
@pytest.mark.parametrize("llg_type", [-3, 2, -2])
def test_mt_relaxes_to_mean_field(oracle, kind, meq_bs, llg_type):
    # push_mt (llg.f90:735-915) and push_zhang (:410-703) without field or
    # noise: |m| decays to the equilibrium m = L(y lambda_m m) (Langevin) or
    # B_S(y lambdaMs m) (Brillouin)
    make = media.mt_medium if kind == "mt" else media.zhang_medium
    med = make(8, tc=700.0, tc_sigma=0.0, temperature=560.0, meq_bs=meq_bs)
    for lay in med.layers:
        lay.scale = 0.0
        lay.hk[:] = 0.0
        lay.hx = np.zeros_like(lay.hx)
        lay.thermal = False
    orc = oracle.OracleSim(med, demag=False)
    orc.step(4000, 1e-14, llg_type=llg_type)
    lms = (med.layers[0].mt or med.layers[0].zhang)["lambda_ms"][0]
    y = GMUB_KB * 0.5 / 560.0
    if meq_bs:
        b0, b1 = 0.0, 1.0
        while b1 - b0 > 1e-13:
            b = 0.5 * (b0 + b1)
            b0, b1 = (b0, b) if b > _bs(y * lms * b, 0.5) else (b, b1)
        want = 0.5 * (b0 + b1)
    else:
        want = _find_meq(0.0, y * lms * 3.0)
    np.testing.assert_allclose(orc.get_mag(0), want, rtol=1e-4)
    orc.close()
