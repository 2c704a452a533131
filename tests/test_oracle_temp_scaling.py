"""Temperature scaling in the oracle: find_temp_scaling and file_temp_scaling's
table reduction (temp_scaling.f90:152-203,365-430) against literal
pure-Python ports of the reference's loops (1-based, as written), and the
scaled fields it feeds."""
import numpy as np
import pytest

from mrm_b200 import media


def reduce_literal(temps, scales):
    """file_temp_scaling's sort / merge / trim / normalise (temp_scaling.f90:152-203)."""
    n = len(temps)
    t2 = [0.0] + list(map(float, temps))  # dat(k,1,2), dat(k,2,2)
    v2 = [0.0] + list(map(float, scales))
    t1 = [0.0] * (n + 2)  # dat(k,1,1), dat(k,2,1)
    v1 = [0.0] * (n + 2)
    t1[1], v1[1] = t2[1], v2[1]
    k = 1
    for i in range(2, n + 1):
        j = 1
        while j <= k:
            if t2[i] < t1[j]:
                break
            j += 1
        for k1 in range(k, j - 1, -1):
            t1[k1 + 1], v1[k1 + 1] = t1[k1], v1[k1]
        t1[j], v1[j] = t2[i], v2[i]
        k += 1
    k = 0
    for i in range(n, 1, -1):
        if t1[i - 1] == t1[i]:
            k += 1
            v1[i - 1] = 0.5 * (v1[i - 1] + v1[i])
            for j in range(i + 1, n + 1):
                t1[j - 1], v1[j - 1] = t1[j], v1[j]
    n = max(1, n - k)
    if v1[1] == v1[2]:
        for i in range(2, n + 1):
            t1[i - 1], v1[i - 1] = t1[i], v1[i]
        n -= 1
    if n > 1 and v1[n - 1] == v1[n]:
        n -= 1
    if t1[n] > 5.0:
        top = t1[n]
        for i in range(1, n + 1):
            t1[i] = t1[i] / top
    return np.array(t1[1:n + 1]), np.array(v1[1:n + 1])


def table_literal(tt, vv, x):
    """find_temp_scaling's bisection and interpolation (temp_scaling.f90:397-414), 1-based."""
    t = [0.0] + list(tt)
    v = [0.0] + list(vv)
    k1, k2 = 1, len(tt)
    if x <= t[1]:
        y = 0.0
    elif x >= t[k2]:
        y = 0.0
        k1 = k2
    else:
        while k2 - k1 > 1:
            k = (k2 + k1) // 2
            if x < t[k]:
                k2 = k
            else:
                k1 = k
        y = max(0.0, min(1.0, (x - t[k1]) / (t[k2] - t[k1])))
    return v[k1] + y * (v[k2] - v[k1])


def scales_literal(temp, tc, mag, msexp, hkexp, use_mag, tables):
    """find_temp_scaling for every grain of a layer (do_grain all set), starting
    from the reference's unit scales; returns ms_scale, alpha_scale, hk_scale."""
    out = [np.ones(len(temp)) for _ in range(3)]
    for i in range(3):  # Ms, alpha, Hk (Hx's values are used nowhere)
        for n in range(len(temp)):
            x = temp[n] / tc[n]
            if i == 0 and use_mag:
                out[i][n] = min(1.0, max(0.0, abs(mag[n])))
            elif i == 0 and msexp >= 0.0:
                out[i][n] = min(1.0, max(0.0, 1.0 - temp[n] / tc[n])) ** msexp
            elif i == 2 and hkexp >= 0.0:
                out[i][n] = min(1.0, max(0.0, 1.0 - temp[n] / tc[n])) ** hkexp
            elif (i + 1) in tables:
                tt, vv = reduce_literal(*tables[i + 1])
                if len(tt) > 1:
                    out[i][n] = table_literal(tt, vv, x)
    return out


TABLES = {
    "unsorted with a triple": ([0.2, 0.0, 0.9, 0.5, 0.5, 0.5, 1.0, 0.7],
                               [0.8, 1.0, 0.1, 0.55, 0.6, 0.5, 0.0, 0.3]),
    "equal ends trimmed": ([0.0, 0.1, 0.4, 0.8, 0.9], [1.0, 1.0, 0.6, 0.2, 0.2]),
    "kelvin": ([300.0, 0.0, 650.0, 500.0, 700.0], [0.7, 1.0, 0.05, 0.4, 0.0]),
    "one pair of equal temperatures": ([0.3, 0.3, 0.6], [0.9, 0.7, 0.1]),
}


def _hamr_llg(side=16, seed=2, peak=450.0, tc=700.0, vel=2000.0, **scaling):
    """mh_medium's LLG layer under a laser spot moving at `vel` cm/s from the
    grid's left edge, its Ms / alpha / Hk scaled with T/Tc (Tc ~ N(tc, 5 %))."""
    med = media.mh_medium(side, seed=seed, temperature=300.0)
    rng = np.random.default_rng(seed + 77)
    for lay in med.layers:
        lay.temp_profile = dict(background=300.0, dtemp=peak, sigma=(40e-7, 40e-7), expn=1,
                                vel=(vel, 0.0), offset=(0.0, None), ref=(0.0, 0.0), t_origin=0.0)
        lay.temp_scaling = dict(tc=np.clip(rng.normal(tc, 0.05 * tc, lay.N), 350.0, None), **scaling)
    return med


@pytest.mark.parametrize("name", sorted(TABLES))
def test_table_reduction_matches_literal_port(oracle, name):
    temps, scales = TABLES[name]
    med = _hamr_llg(8, tables={1: (temps, scales)}, msexp=-1.0)
    orc = oracle.OracleSim(med, rng_mode=1, seed=1)
    tt, vv = orc.get_temp_scaling_table(0, 1)
    lt, lv = reduce_literal(temps, scales)
    np.testing.assert_array_equal(tt, lt)
    np.testing.assert_array_equal(vv, lv)
    orc.close()


def test_scales_match_literal_port(oracle):
    """Power law for Ms, tables for alpha and Hk, at a time when the spot has
    pushed part of the grid above Tc."""
    tables = {2: TABLES["unsorted with a triple"], 3: TABLES["kelvin"], 4: TABLES["equal ends trimmed"]}
    med = _hamr_llg(16, msexp=0.35, hkexp=-1.0, tables=tables)
    orc = oracle.OracleSim(med, rng_mode=1, seed=1)
    orc.eval_field(2.0e-10)
    temp = orc.get_temp(0)
    assert temp.max() > med.layers[0].temp_scaling["tc"].min()  # some grains above their Tc
    got = orc.get_scales(0)
    want = scales_literal(temp, med.layers[0].temp_scaling["tc"], None, 0.35, -1.0, False, tables)
    for g, w, name in zip(got, want, ("ms", "alpha", "hk")):
        np.testing.assert_allclose(g, w, rtol=0, atol=1e-15, err_msg=name)
    assert (got[0] == 0).any() and (got[0] > 0).any()
    orc.close()


def test_hk_power_law_and_ms_table(oracle):
    tables = {1: TABLES["equal ends trimmed"]}
    med = _hamr_llg(16, msexp=-1.0, hkexp=1.7, tables=tables)
    orc = oracle.OracleSim(med, rng_mode=1, seed=1)
    orc.eval_field(3.0e-10)
    got = orc.get_scales(0)
    want = scales_literal(orc.get_temp(0), med.layers[0].temp_scaling["tc"], None, -1.0, 1.7, False, tables)
    for g, w in zip(got, want):
        np.testing.assert_allclose(g, w, rtol=0, atol=1e-15)
    orc.close()


def test_ms_from_llb_magnitude(oracle):
    med = media.hamr_medium(16, seed=4)
    lay = med.layers[0]
    lay.temp_scaling = dict(tc=lay.llb["tc"], use_mag=True, hkexp=2.0)
    orc = oracle.OracleSim(med, rng_mode=1, seed=3)
    orc.step(200, 1e-14)
    mag = orc.get_mag(0)
    orc.eval_field(200 * 1e-14)
    ms_s, al_s, hk_s = orc.get_scales(0)
    np.testing.assert_array_equal(ms_s, np.clip(np.abs(mag), 0.0, 1.0))
    assert (mag < 1.0).all() and np.all(al_s == 1.0)
    want_hk = np.clip(1.0 - orc.get_temp(0) / lay.llb["tc"], 0.0, 1.0) ** 2.0
    np.testing.assert_allclose(hk_s, want_hk, rtol=0, atol=1e-15)
    orc.close()


def test_grain_above_tc_follows_the_field(oracle):
    """ms_scale = 0 above Tc: push_llg puts m along the (non-thermal) field
    (llg.f90:1140-1148) and the grain drops out of the demag source."""
    med = _hamr_llg(8, peak=2000.0, tc=400.0, msexp=0.5)
    for lay in med.layers:
        lay.thermal = False
    orc = oracle.OracleSim(med, rng_mode=1, seed=1)
    orc.step(1, 1e-13)
    ms_s = orc.get_scales(0)[0]
    hot = np.where(ms_s == 0.0)[0]
    assert hot.size > 0
    h = orc.get_field(0)[hot]
    m = orc.get_state(0)[hot]
    np.testing.assert_allclose(m, h / np.linalg.norm(h, axis=1, keepdims=True), atol=1e-12)
    orc.close()
