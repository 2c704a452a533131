"""Pins the oracle's random streams against independent implementations.

MT19937 (src/random.f90:166-249): the reference seeds with a 69069 LCG
(random.f90:173-181) and twists/tempers with the standard MT19937
constants (random.f90:10).  numpy's RandomState runs the same twist and
tempering from any 624-word state, so the oracle's outputs must agree
bit for bit once its seeded state is handed to numpy.
Philox4x64-10 (the GPU thermal stream) is pinned against numpy.random.Philox.
"""
import numpy as np
import pytest


@pytest.mark.parametrize("seed", [34, 10034, 20034, -7, 0])
def test_mt19937_matches_numpy(oracle, seed):
    st = oracle.mt_state(seed)
    # random.f90:173-179: mt(0) = 4357+|seed|, mt(i) = 69069*mt(i-1) mod 2^32
    exp = np.zeros(624, np.uint64)
    exp[0] = 4357 + abs(seed)
    for i in range(1, 624):
        exp[i] = (69069 * int(exp[i - 1])) & 0xFFFFFFFF
    assert np.array_equal(st.astype(np.uint64), exp)
    rs = np.random.RandomState()
    rs.set_state(("MT19937", st, 624))
    ref = rs.randint(0, 2**32, size=3000, dtype=np.uint64).astype(np.uint32)
    assert np.array_equal(oracle.mt_u32(seed, 3000), ref)


def test_polar_box_muller_sequence(oracle):
    # random.f90:215-229 restated from the uniform stream: cached second deviate
    u = oracle.mt_u32(34, 4000).astype(np.float64) / 2.0**32
    out, k, cached = [], 0, None
    while len(out) < 500:
        if cached is not None:
            out.append(cached)
            cached = None
            continue
        while True:
            v1, v2 = 2 * u[k] - 1, 2 * u[k + 1] - 1
            k += 2
            rsq = v1 * v1 + v2 * v2
            if 0.0 < rsq < 1.0:
                break
        f = np.sqrt(-2.0 * np.log(rsq) / rsq)
        cached = v1 * f
        out.append(v2 * f)
    assert np.allclose(oracle.mt_normals(34, 500), out, rtol=0, atol=1e-15)


@pytest.mark.parametrize("ctr,key", [([5, 7, 9, 11], [123, 456]),
                                     ([2**63 + 17, 1, 2, 3], [2**64 - 1, 0]),
                                     ([1, 0, 0, 0], [0x1234567890, 0x6d726d])])
def test_philox4x64_matches_numpy(oracle, ctr, key):
    c = np.array(ctr, np.uint64)
    bg = np.random.Philox(counter=c - np.array([1, 0, 0, 0], np.uint64), key=np.array(key, np.uint64))
    ref = np.array(bg.random_raw(4), np.uint64)
    assert np.array_equal(oracle.philox4x64(ctr, key), ref)


def test_philox_normals_statistics(oracle):
    z = np.array([oracle.philox_normal3(7, 0, s, g) for s in range(40) for g in range(500)]).ravel()
    assert abs(z.mean()) < 0.02
    assert abs(z.var() - 1.0) < 0.03
    # distinct streams for distinct layers / steps
    a = oracle.philox_normal3(7, 0, 3, 11)
    b = oracle.philox_normal3(7, 1, 3, 11)
    c = oracle.philox_normal3(7, 0, 4, 11)
    assert not np.allclose(a, b) and not np.allclose(a, c)
