"""Moving write head (the two-layer write workload's Karlqvist head and PRBS
pattern): the oracle's applied field against a direct evaluation of the
formula, the deep-gap normalisation and the bit pattern."""
import math

import numpy as np

from mrm_b200 import media


def _karlqvist(u, g, z, hg):
    a, b = u + 0.5 * g, u - 0.5 * g
    return (hg / math.pi * (np.arctan(a / z) - np.arctan(b / z)),
            hg / (2 * math.pi) * np.log((b * b + z * z) / (a * a + z * z)))


def test_deep_gap_normalisation():
    g, z = 25e-7, 6e-7
    hg = media.karlqvist_deep_gap(12000.0, g, z)
    hx, hz = _karlqvist(np.array([0.0]), g, z, hg)
    assert abs(hx[0] - 12000.0) < 1e-9 and abs(hz[0]) < 1e-9
    # h_x peaks under the gap centre; h_z is odd in u
    u = np.linspace(-200e-7, 200e-7, 4001)
    hx, hz = _karlqvist(u, g, z, hg)
    assert np.argmax(hx) == 2000
    assert np.allclose(hz, -hz[::-1], atol=1e-9)


def test_prbs_pattern():
    p1, p2 = media.prbs_pattern(64, 1), media.prbs_pattern(64, 2)
    assert p1 != p2 and p1 == media.prbs_pattern(64, 1)
    ones = bin(p1).count("1")
    assert 20 <= ones <= 44  # a balanced-ish maximal-length sequence segment
    assert 0 < p1 < 2 ** 64


def test_oracle_head_field(oracle):
    """With demag, anisotropy and exchange off, the oracle's field is the head's."""
    med = media.head_write_medium(32, 8, temperature=0.0)
    rng = np.random.default_rng(0)
    for lay in med.layers:
        lay.hk[:] = 0.0
        lay.hx = None
        lay.hx_index = lay.hx_grain = None
        lay.uhx = lay.lhx = None
        lay.head["velocity"] = 4e5   # crosses the 32-column grid in ~0.56 ns
        lay.head["bit_time"] = 7e-11
    orc = oracle.OracleSim(med, demag=False, rng_mode=1, seed=1)
    for l in range(2):
        orc.set_state(l, media.easy_axes(rng, med.layers[l].N, 90.0))
    for t in (0.0, 1.3e-10, 3.9e-10):
        orc.eval_field(t)
        for l, lay in enumerate(med.layers):
            hd = lay.head
            k = int(math.floor((t - hd["t0"]) / hd["bit_time"])) % hd["nbits"]
            pol = 1.0 if (hd["pattern"] >> k) & 1 else -1.0
            i = np.arange(lay.N) % med.nx
            u = (i + 0.5) * med.dx - (hd["x0"] + hd["velocity"] * (t - hd["t0"]))
            hx, hz = _karlqvist(u, hd["gap"], hd["z"], pol * hd["hg"])
            h = orc.get_field(l)
            assert np.allclose(h[:, 0], hx, rtol=1e-12, atol=1e-9)
            assert np.allclose(h[:, 1], 0.0, atol=1e-9)
            assert np.allclose(h[:, 2], hz, rtol=1e-12, atol=1e-9)
