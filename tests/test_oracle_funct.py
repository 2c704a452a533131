"""The oracle's applied-field time functions against a literal port of funct
(src/applied.f90:328-396) and get_appl's scaling (:866-869): SIN, COS, EXP,
STE, NEW and ROT (its branch with the rotation angles present and
|gamma| != 1: unit magnitude along the in-plane direction that rot_fld sets,
(cos((2 gamma t + phase) pi), sin((2 gamma t + phase) pi), 0))."""
import math

import numpy as np
import pytest

from tests.helpers import small_medium

CODES = {"SIN": 1, "COS": 2, "EXP": 3, "STE": 4, "NEW": 5, "ROT": 7}


def funct_port(func, t, gamm, phase, param, duty, moddepth):
    """applied.f90:328-377, statement by statement (Fortran mod = fmod)."""
    if func == "SIN":
        return math.sin(t * gamm + phase)
    if func == "EXP":
        return math.exp(t * gamm + phase)
    if func == "COS":
        return math.cos(t * gamm + phase)
    if func == "NEW":
        x = gamm / param
        y = math.exp(duty * x)
        w = math.exp(x)
        x = t + phase
        if x < 0.0:
            x = x + gamm * (1 + int(abs(x / gamm)))
        x = math.fmod(x, gamm)
        if x > duty * gamm:
            x = math.exp((gamm - x) / param)
            return 1.0 - moddepth + x * (y - 1.0) * moddepth / (w - 1.0)
        x = math.exp(-x / param)
        return 1.0 + x * (y - w) * moddepth / (w - 1.0)
    if func == "STE":
        x = t + phase
        if x < 0.0:
            x = x + gamm * (1 + int(abs(x / gamm)))
        x = math.fmod(x, gamm)
        if x < 0.5 * param:
            return 2.0 * x / param
        if x < 0.5 * (gamm - param):
            return 1.0
        if x < 0.5 * (gamm + param):
            return (gamm - 2.0 * x) / param
        if x < gamm - 0.5 * param:
            return -1.0
        return 2.0 * (x - gamm) / param
    if func == "ROT":
        return 1.0
    return 0.0


def applied_port(lay, func, t):
    """get_appl's uniform field: (amp f(t) + dc) scale along the field direction."""
    s = (lay.amp * funct_port(func, t, lay.fgamma, lay.phase, lay.param, lay.duty, lay.moddepth) + lay.dc) * lay.scale
    d = np.array(lay.hdir, float)
    if func == "ROT":
        th = (2.0 * lay.fgamma * t + lay.phase) * math.acos(-1.0)
        d = np.array([math.cos(th), math.sin(th), 0.0])
    return s * d


def with_function(func, amp=1500.0, gamma=3.0e10, phase=0.3, param=2.0e-11, duty=0.35, moddepth=0.6,
                  dc=200.0, scale=2.0, seed=3):
    med = small_medium(8, boundary=1, seed=seed)
    lay = med.layers[0]
    lay.hdir = (math.sin(0.4), 0.0, math.cos(0.4))
    lay.func, lay.amp, lay.fgamma, lay.phase = CODES[func], amp, gamma, phase
    lay.param, lay.duty, lay.moddepth, lay.dc, lay.scale = param, duty, moddepth, dc, scale
    if func in ("STE", "NEW"):
        lay.fgamma = 1.5e-10  # a period (s)
    if func == "ROT":
        lay.fgamma = 2.5e9  # turns per second
    return med


@pytest.mark.parametrize("func", list(CODES))
def test_applied_field_against_literal_port(oracle, func):
    med = with_function(func)
    orc = oracle.OracleSim(med, demag=False)
    lay = med.layers[0]
    for t in (0.0, 7.3e-12, 4.1e-11, 1.234e-10, 2.9e-10):
        orc.eval_field(t)
        h = orc.get_applied(0)
        ref = applied_port(lay, func, t)
        assert np.abs(h - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()), (func, t)
    orc.close()


def test_ste_and_new_shapes(oracle):
    """The port's own known answers: STE rises over param, holds at +1,
    falls to -1; NEW has unit high level at the start of its period."""
    g, p = 1.0, 0.1
    assert funct_port("STE", 0.025, g, 0.0, p, 0, 0) == pytest.approx(0.5)
    assert funct_port("STE", 0.25, g, 0.0, p, 0, 0) == 1.0
    assert funct_port("STE", 0.5, g, 0.0, p, 0, 0) == pytest.approx(0.0)
    assert funct_port("STE", 0.75, g, 0.0, p, 0, 0) == -1.0
    assert funct_port("NEW", 0.0, g, 0.0, p, 0.5, 0.0) == pytest.approx(1.0)
