"""The reference's on-disk formats (mrm_b200/formats.py): record framing,
round trips, and media read back from a grain file running identically on the
oracle."""
import struct

import numpy as np

from mrm_b200 import formats, media
from oracle import pyoracle


def test_record_framing(tmp_path):
    p = tmp_path / "r.bin"
    with open(p, "wb") as f:
        formats.write_record(f, 3, 2.5, True, np.array([[1, 2], [3, 4]], dtype=np.int32))
    b = p.read_bytes()
    body = struct.pack("<idi", 3, 2.5, 1) + struct.pack("<4i", 1, 3, 2, 4)  # Fortran (column) order
    assert b == struct.pack("<i", len(body)) + body + struct.pack("<i", len(body))
    with open(p, "rb") as f:
        assert formats.read_record(f) == body


def test_subrecords_are_joined(tmp_path):
    p = tmp_path / "s.bin"
    a, c = b"x" * 10, b"y" * 6
    with open(p, "wb") as f:  # a record continued in a second subrecord (negative leading marker)
        f.write(struct.pack("<i", -10) + a + struct.pack("<i", 10))
        f.write(struct.pack("<i", 6) + c + struct.pack("<i", -6))
    with open(p, "rb") as f:
        assert formats.read_record(f) == a + c


def _two_layer_map_medium():
    import copy
    med = media.grain_map_medium(12, 10, seed=4)
    top = med.layers[0]
    bot = copy.deepcopy(top)
    bot.ms = np.full(bot.N, 900.0)
    bot.vol = 0.5 * top.vol  # half as thick
    bot.cubic_axis = media.cubic_frames(np.random.default_rng(3), bot.N)
    n = top.N
    top.lhx = media.columnar_coupling(n, 1200.0)
    bot.uhx = media.columnar_coupling(n, 1200.0)
    med.layers = [top, bot]
    med.dz = [med.dz[0], 0.5 * med.dz[0]]
    med.il_space = [0.0, 0.0]
    med.m0 = [med.m0[0], med.m0[0].copy()]
    return med


def test_grain_file_round_trip_and_dynamics(tmp_path):
    med = _two_layer_map_medium()
    p = str(tmp_path / "grain.bin")
    formats.write_grain_file(p, formats.grain_file_layers(med), med.nx, med.ny, med.dx, med.dy)
    head, ls = formats.read_grain_file(p)
    assert head == dict(nx=med.nx, ny=med.ny, dx=med.dx, dy=med.dy)
    for L, lay in zip(ls, med.layers):
        assert np.array_equal(L["grain2gridindex"], lay.g2c_index)
        assert np.array_equal(L["grain2grid"], lay.g2c)
        assert np.array_equal(L["hk"], lay.hk)
        if lay.cubic_axis is not None:
            assert L["uni_axis"] is None and np.array_equal(L["cubic_axis"], lay.cubic_axis)
        else:
            assert L["cubic_axis"] is None and np.array_equal(L["uni_axis"], lay.axis)
        assert np.array_equal(L["hx"][1], lay.hx_grain) and np.array_equal(L["hx"][2], lay.hx)
    back = formats.medium_from_grain_file(p, med.dz, boundary=med.boundary)
    for lay, orig in zip(back.layers, med.layers):
        assert np.allclose(lay.vol, orig.vol, rtol=1e-15)
        lay.hdir, lay.t_start, lay.t_end = orig.hdir, orig.t_start, orig.t_end
        lay.s_start, lay.s_end = orig.s_start, orig.s_end
        lay.axis = orig.axis if lay.cubic_axis is None else lay.axis
    runs = []
    for m in (med, back):
        sim = pyoracle.OracleSim(m)
        st = sim.step(200, 1e-13)
        runs.append((st, [sim.get_state(l) for l in range(2)]))
        sim.close()
    (s0, m0), (s1, m1) = runs
    for a, b in zip(m0, m1):
        assert np.array_equal(a, b)
    # the energy weighs by the volumes, which the file's dz round trip returns to 1e-15
    assert abs(s0["energy"] - s1["energy"]) <= 1e-14 * abs(s0["energy"])


def test_tensor_cache_round_trip(tmp_path):
    nx, ny, nl = 16, 8, 2
    n2d = pyoracle.calculate_tensor(nx, ny, 8e-7, 8e-7, [8e-7, 4e-7], [0.0, 0.0], 1)
    p = str(tmp_path / "mrm_1.dat")
    formats.write_tensor_cache(p, n2d, nx=nx, ny=ny, imx=1, imy=1, dx=8e-7, dy=8e-7, dz=[8e-7, 4e-7],
                               il_space=[0.0, 0.0])
    h, back = formats.read_tensor_cache(p)
    assert (h["nx"], h["ny"], h["n_lay"], h["imx"]) == (nx, ny, nl, 1)
    assert np.array_equal(back, n2d)
    # the record is the reference's n2d(nx, ny, 9, n_lay, n_lay) in column order
    raw = open(p, "rb").read()
    first = struct.unpack("<i", raw[:4])[0]
    off = 8 + first + 4
    vals = np.frombuffer(raw[off:off + 8 * n2d.size], "<f8")
    assert vals[1] == n2d[0, 0, 0, 0, 1]  # next in memory: i + 1


def test_magnetisation_files(tmp_path):
    med = media.grain_map_medium(8, 6, seed=8)
    lay = med.layers[0]
    rng = np.random.default_rng(2)
    m = rng.standard_normal((lay.N, 3))
    m /= np.linalg.norm(m, axis=1, keepdims=True)
    p = str(tmp_path / "m.bin")
    formats.write_mag(p, [m], [lay.ms], med.nx, med.ny, [700.0])
    r = formats.read_mag(p, 1)[0]
    assert (r["nx"], r["ny"], r["ms_nom"]) == (med.nx, med.ny, 700.0)
    assert np.allclose(r["m"], m, atol=1e-15) and np.allclose(r["ms_file"], lay.ms)
    grid = formats.grain_file_layers(med)[0]["grid2grain"]
    pa = str(tmp_path / "m.dat")
    formats.write_mag_ascii(pa, [m], [lay.ms], [lay.ms_scale], [grid], med.nx, med.ny)
    first = open(pa).readline()
    assert first.startswith('ZONE T="     0.00", I=    8, J=    6, K=  1 F=POINT')
    back = formats.read_mag_ascii(pa, [grid], [lay.N])[0]
    assert np.allclose(back, m, atol=1e-5)  # 6 significant digits in the file
