"""Moving demag window on the oracle (window_m / update_do_grain,
data.f90:1-65,120-157; get_mag and get_magnetostatic with a window,
data.f90:357-385, field.f90:472-495; do_grain in get_field / push_llg):
the origin against a literal restatement of update_do_grain, a window
covering the grid against no window, frozen grains, and the windowed demag
against the open-boundary convolution restricted to the window."""
import math

import numpy as np
import pytest

from mrm_b200 import media
from tests.helpers import random_m


def _nint(x):
    """Fortran NINT: nearest integer, halves away from zero."""
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))


def _origin(nx, ny, nxw, nyw, dx, dy, v, off, t):
    """update_do_grain (data.f90:128-131) with get_window(t=t) (:59): 0-based i0, j0."""
    ox, oy = v[0] * t + off[0], v[1] * t + off[1]
    i = max(1, min(nx - nxw + 1, _nint((nx - nxw) * 0.5 + ox / dx))) - 1
    j = max(1, min(ny - nyw + 1, _nint((ny - nyw) * 0.5 + oy / dy))) - 1
    return i, j


def test_window_origin_follows_update_do_grain(oracle):
    med = media.mh_medium(32, ny=16, seed=1, boundary=1)
    v, off = (3.0e4, -1.2e4), (-9e-6, 2e-6)
    med.window = dict(nx=8, ny=4, v=v, offset=off)
    orc = oracle.OracleSim(med, demag=True)
    for t in (0.0, 1e-11, 5.5e-11, 1.3e-10, 4e-10, 9e-10):
        orc.eval_field(t)
        want = _origin(32, 16, 8, 4, med.dx, med.dy, v, off, t)
        assert orc.get_window() == (8, 4) + want, t
    orc.close()


def test_full_window_is_no_window(oracle):
    med = media.mh_medium(16, seed=2, boundary=1, temperature=300.0)
    a = oracle.OracleSim(med, rng_mode=1, seed=3)
    med.window = dict(nx=16, ny=16, v=(1e4, 0.0), offset=(0.0, 0.0))
    b = oracle.OracleSim(med, rng_mode=1, seed=3)
    sa, sb = a.step(300, 1e-13), b.step(300, 1e-13)
    assert np.array_equal(a.get_state(0), b.get_state(0))
    # (the oracle's OpenMP energy sum has no fixed order)
    assert sa["energy"] == pytest.approx(sb["energy"], rel=1e-14) and sa["mmag"] == pytest.approx(sb["mmag"], rel=1e-14)
    a.close()
    b.close()


def test_frozen_grains_keep_state(oracle):
    # a stationary window: grains outside it never change, the stats still
    # count them (volume of every grain)
    med = media.mh_medium(32, ny=16, seed=3, boundary=1, temperature=300.0)
    med.window = dict(nx=16, ny=8, v=(0.0, 0.0), offset=(1.0e-6, 0.0))
    orc = oracle.OracleSim(med, rng_mode=1, seed=4)
    m0 = orc.get_state(0).copy()
    st = orc.step(400, 1e-13)
    nxw, nyw, i0, j0 = orc.get_window()
    m1 = orc.get_state(0)
    inside = np.zeros((16, 32), bool)
    inside[j0:j0 + nyw, i0:i0 + nxw] = True
    inside = inside.ravel()
    assert np.array_equal(m1[~inside], m0[~inside])
    assert np.abs(m1[inside] - m0[inside]).max() > 1e-3
    assert st["vol_l"][0] == pytest.approx(med.layers[0].vol.sum(), rel=1e-14)
    orc.close()


def test_window_demag_is_restricted_convolution(oracle):
    # open boundary: the window's (zero-padded) FFT is the linear convolution of
    # the window's magnetisation, i.e. the full grid's with no moment outside it
    med = media.mh_medium(32, ny=16, seed=5, boundary=1)
    m = random_m(med.layers[0].N, 6)
    med.window = dict(nx=16, ny=8, v=(0.0, 0.0), offset=(2.0e-6, -1.0e-6))
    w = oracle.OracleSim(med)
    w.set_state(0, m)
    w.eval_field(0.0)
    nxw, nyw, i0, j0 = w.get_window()
    inside = np.zeros((16, 32), bool)
    inside[j0:j0 + nyw, i0:i0 + nxw] = True
    inside = inside.ravel()
    med.window = None
    lay = med.layers[0]
    lay.ms_scale = np.where(inside, lay.ms_scale, 0.0)
    f = oracle.OracleSim(med)
    f.set_state(0, m)
    f.eval_field(0.0)
    np.testing.assert_allclose(w.get_demag(0)[inside], f.get_demag(0)[inside], rtol=1e-11, atol=1e-9)
    w.close()
    f.close()
