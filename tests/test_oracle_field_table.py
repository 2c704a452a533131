"""Tabulated (moving) applied-field profile on the oracle: its restatement of
set / interpolate / get_applied (applied.f90:1471-1520,1757-1776,
field.f90:546-560) against a literal pure-Python port of those loops
(1-based indices, the sweep as written), the bilinear property on a linear
profile, and the field-file reader (file_applied, applied.f90:711-813)."""
import numpy as np
import pytest

from mrm_b200 import formats, media
from tests.helpers import random_m


def _set_literal(offset, n, dd, pos):
    """applied.f90:1757-1776 as written (1-based ind)."""
    npos = len(pos)
    ind, f = [0] * (n + 1), [0.0] * (n + 1)
    i0 = 2
    for i in range(1, n + 1):
        x = (i - .5) * dd - offset
        while pos[i0 - 1] <= x and i0 < npos:
            i0 += 1
        ind[i] = min(npos - 1, i0 - 1)
        f[i] = max(0.0, min(1.0, (pos[i0 - 1] - x) / (pos[i0 - 1] - pos[i0 - 2])))
    return ind, f


def _applied_literal(med, layer, t, s):
    """get_appl's moving branch + interpolate + get_applied's cell average."""
    lay = med.layers[layer]
    tb = lay.field_table
    xp, yp, v = tb["xpos"], tb["ypos"], tb["vfld"]
    ox = tb["offset"][0] if tb["offset"][0] is not None else med.dx * med.nx * 0.5
    oy = tb["offset"][1] if tb["offset"][1] is not None else med.dy * med.ny * 0.5
    ix, fx = _set_literal(ox + tb["vel"][0] * (t - tb["t_origin"]) - tb["ref"][0], med.nx, med.dx, xp)
    iy, fy = _set_literal(oy + tb["vel"][1] * (t - tb["t_origin"]) - tb["ref"][1], med.ny, med.dy, yp)

    def vfi(c, i, j):  # vfi(c, i, j), 1-based node indices
        return v[j - 1, i - 1, c]

    app = np.zeros((med.nx + 1, med.ny + 1, 3))
    for j in range(1, med.ny + 1):
        yf, yfc = s * fy[j], s * (1.0 - fy[j])
        for i in range(1, med.nx + 1):
            for c in range(3):
                app[i, j, c] = (fx[i] * yf * vfi(c, ix[i], iy[j]) + (1.0 - fx[i]) * yf * vfi(c, ix[i] + 1, iy[j]) +
                                fx[i] * yfc * vfi(c, ix[i], iy[j] + 1) +
                                (1.0 - fx[i]) * yfc * vfi(c, ix[i] + 1, iy[j] + 1))
    out = np.zeros((lay.N, 3))
    for n in range(lay.N):
        y = np.zeros(3)
        for q in range(lay.g2c_index[n], lay.g2c_index[n + 1]):
            i, j = lay.g2c[q]
            y += app[i, j]
        out[n] = y / (lay.g2c_index[n + 1] - lay.g2c_index[n])
    return out


def _table(seed, nxt=9, nyt=6, half_x=6e-6, half_y=5e-6):
    rng = np.random.default_rng(seed)
    xp = np.sort(rng.uniform(-half_x, half_x, nxt))
    yp = np.sort(rng.uniform(-half_y, half_y, nyt))
    v = rng.normal(scale=2000.0, size=(nyt, nxt, 3))
    return xp, yp, v


@pytest.mark.parametrize("mapped", [False, True])
def test_table_matches_literal_loops(oracle, mapped):
    if mapped:
        med = media.grain_map_medium(12, 10, seed=5)
    else:
        med = media.mh_medium(12, ny=10, seed=5, boundary=1)
    xp, yp, v = _table(3)
    lay = med.layers[0]
    # moving in x and y, ragged nodes narrower than the grid: cells beyond the
    # table's ends clamp to its edge intervals
    lay.field_table = dict(xpos=xp, ypos=yp, vfld=v, vel=(3000.0, -1000.0), offset=(None, 2e-6),
                           ref=(1e-6, 5e-7), t_origin=1e-10)
    lay.func, lay.amp, lay.fgamma, lay.param, lay.dc, lay.scale = 4, 1.3, 4e-10, 5e-11, 0.1, 0.9
    orc = oracle.OracleSim(med, demag=False)
    orc.set_state(0, random_m(lay.N, 2))
    for t in (0.0, 3.7e-10, 1.05e-9):
        orc.eval_field(t)
        s = (1.3 * _ste(t, 4e-10, 5e-11) + 0.1) * 0.9
        np.testing.assert_allclose(orc.get_applied(0), _applied_literal(med, 0, t, s), rtol=1e-13, atol=1e-9)
    orc.close()


def _ste(t, g, param):
    x = np.fmod(t, g)
    if x < 0.5 * param:
        return 2.0 * x / param
    if x < 0.5 * (g - param):
        return 1.0
    if x < 0.5 * (g + param):
        return (g - 2.0 * x) / param
    if x < g - 0.5 * param:
        return -1.0
    return 2.0 * (x - g) / param


def test_linear_profile_is_reproduced(oracle):
    # bilinear interpolation reproduces a linear profile at every cell inside the table
    med = media.mh_medium(16, ny=8, seed=2, boundary=1)
    lay = med.layers[0]
    xp = np.array([-1e-5, -4e-6, -1e-6, 0.0, 3e-6, 1e-5])
    yp = np.array([-1e-5, -2e-6, 1e-6, 1e-5])
    X, Y = np.meshgrid(xp, yp)
    v = np.stack([100.0 + 2e8 * X, -50.0 + 1e8 * Y, 3e7 * X - 4e7 * Y], axis=-1)
    lay.field_table = dict(xpos=xp, ypos=yp, vfld=v, vel=(0.0, 0.0), offset=(None, None), ref=(0.0, 0.0),
                           t_origin=0.0)
    lay.s_start = lay.s_end = lay.scale = 1.0  # time scale 1
    orc = oracle.OracleSim(med, demag=False)
    orc.eval_field(0.0)
    i, j = np.meshgrid(np.arange(med.nx), np.arange(med.ny))
    x = ((i + 0.5) * med.dx - med.nx * med.dx / 2).ravel()
    y = ((j + 0.5) * med.dy - med.ny * med.dy / 2).ravel()
    want = np.stack([100.0 + 2e8 * x, -50.0 + 1e8 * y, 3e7 * x - 4e7 * y], axis=-1)
    np.testing.assert_allclose(orc.get_applied(0), want, rtol=1e-12, atol=1e-9)
    orc.close()


def test_field_file_reader(tmp_path):
    # file_applied's FEM orientation on a hand-written 2 x 2 zone: x reversed and
    # negated, the file's z is the model's y, H = (-Hx, Hz, Hy)
    p = tmp_path / "head.dat"
    p.write_text('TITLE = "head"\nVARIABLES = "x" "y" "z" "Bx" "By" "Bz"\nZONE T="a", I=2, J=2, F=POINT\n'
                 "-1.0d-6 0 -2.0E-6 1 2 3\n"
                 "2.0e-6 0 -2.0e-6 4 5 6\n"
                 "-1.0e-6 0.0 3.0e-6 7 8\n9\n"
                 "2.0e-6, 0.0, 3.0e-6, 10, 11, 12 99\n")
    xp, yp, v = formats.read_field_file(str(p), scale=2.0)
    np.testing.assert_array_equal(xp, [-2e-6, 1e-6])
    np.testing.assert_array_equal(yp, [-2e-6, 3e-6])
    np.testing.assert_array_equal(v[0, 0], [-8, 12, 10])   # file node 2 of row 1: (4, 5, 6)
    np.testing.assert_array_equal(v[0, 1], [-2, 6, 4])     # file node 1: (1, 2, 3)
    np.testing.assert_array_equal(v[1, 1], [-14, 18, 16])  # (7, 8, 9) across two lines
    np.testing.assert_array_equal(v[1, 0], [-20, 24, 22])  # trailing value skipped
    q = tmp_path / "back.dat"
    formats.write_field_file(str(q), xp, yp, v)
    xp2, yp2, v2 = formats.read_field_file(str(q))
    np.testing.assert_array_equal(xp2, xp)
    np.testing.assert_array_equal(yp2, yp)
    np.testing.assert_array_equal(v2, v)


def test_table_write_medium_runs(oracle):
    # a short write with the tabulated head on the oracle: the head's field reaches
    # the grains under it and the state stays normalised
    med = media.table_write_medium(32, 16, seed=1, temperature=0.0)
    orc = oracle.OracleSim(med, rng_mode=1, seed=1)
    orc.step(200, 1e-13)
    for l in range(2):
        m = orc.get_state(l)
        np.testing.assert_allclose(np.linalg.norm(m, axis=1), 1.0, rtol=1e-12)
    orc.eval_field(2e-11)
    ha = orc.get_applied(0)
    assert np.abs(ha).max() > 1000.0
    orc.close()


def test_scalar_field_file(tmp_path):
    # file_applied with nval = 1 (a temperature table): records `x y value`,
    # x fastest, no axis mapping, scaled
    p = tmp_path / "temp.dat"
    p.write_text('TITLE = "T"\nZONE I=3, J=2\n'
                 "-1e-6 0 10\n0 0 20\n1e-6 0 30\n"
                 "-1e-6 2e-6 40\n0 2e-6 50\n1e-6 2e-6 60\n")
    xp, yp, v = formats.read_field_file(str(p), nval=1, scale=0.5)
    np.testing.assert_array_equal(xp, [-1e-6, 0.0, 1e-6])
    np.testing.assert_array_equal(yp, [0.0, 2e-6])
    np.testing.assert_array_equal(v, [[5, 10, 15], [20, 25, 30]])
