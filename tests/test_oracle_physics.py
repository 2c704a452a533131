"""Known-answer physics for the restated integrator (llg.f90 push_llg Heun)."""
import math

import numpy as np

from mrm_b200 import media


def _bare_medium(side, hk, alpha, hdir, s_start, s_end, t_end, temperature=0.0, ms=700.0):
    m = media.mh_medium(side, hk=hk, k_sigma=0.0, k_ang_deg=0.0, hex_oe=0.0, alpha=alpha,
                        temperature=temperature, ms=ms)
    lay = m.layers[0]
    lay.hdir = tuple(hdir)
    lay.t_start, lay.t_end, lay.s_start, lay.s_end, lay.scale = 0.0, t_end, s_start, s_end, 1.0
    return m


def test_stoner_wohlfarth_switching(oracle):
    # h_sw = Hk / (cos^(2/3) psi + sin^(2/3) psi)^(3/2); psi = 10 deg -> 0.6738 Hk.
    # Quasi-static bracket: a reversed field 3% below h_sw leaves m in its well,
    # 3% above it switches m (alpha = 1, 2 ns at constant field).
    hk, psi = 15000.0, math.radians(10.0)
    hsw = hk / (math.cos(psi) ** (2 / 3) + math.sin(psi) ** (2 / 3)) ** 1.5
    hdir = (math.sin(psi), 0.0, math.cos(psi))
    for f, switched in ((0.97, False), (1.03, True)):
        med = _bare_medium(2, hk, 1.0, hdir, -f * hsw, -f * hsw, 1.0)
        sim = oracle.OracleSim(med, demag=False)
        st = sim.step(20000, 1e-13)
        assert (st["mave"][2] < 0) == switched, (f, st["mave"])


def test_larmor_precession(oracle):
    # alpha -> 0, H along z: m precesses at omega = gamma H / (1 + alpha^2)
    H, alpha, gamma = 1000.0, 1e-6, 1.76e7
    med = _bare_medium(2, 0.0, alpha, (0, 0, 1), H, H, 1.0)
    m0 = np.tile([1.0, 0.0, 0.0], (4, 1))
    med.m0 = [m0]
    sim = oracle.OracleSim(med, demag=False)
    dt, nsteps = 1e-14, 20000
    sim.step(nsteps, dt)
    m = sim.get_state(0)[0]
    phi = math.atan2(m[1], m[0])
    w = gamma * H / (1 + alpha**2)
    expect = w * nsteps * dt  # dm/dt = -gamma m x H: counter-clockwise about +z
    d = (phi - expect + math.pi) % (2 * math.pi) - math.pi
    assert abs(d) < 1e-6


def test_boltzmann_equilibrium(oracle):
    # uniaxial grains, no field: <m_z^2> = int c^2 e^{s c^2} dc / int e^{s c^2} dc, s = K V / kT
    hk, ms, T = 1000.0, 700.0, 300.0
    med = _bare_medium(32, hk, 1.0, (0, 0, 1), 0.0, 0.0, 1.0, temperature=T, ms=ms)
    lay = med.layers[0]
    sigma = 0.5 * hk * ms * lay.vol[0] / (1.380662e-16 * T)
    c = np.linspace(-1, 1, 200001)
    w = np.exp(sigma * (c**2 - 1))
    expect = np.trapezoid(c**2 * w, c) / np.trapezoid(w, c)
    sim = oracle.OracleSim(med, demag=False, rng_mode=0, seed=34)
    dt = 1e-12
    sim.step(500, dt)
    acc = []
    for _ in range(150):
        sim.step(20, dt)
        acc.append(np.mean(sim.get_state(0)[:, 2] ** 2))
    assert abs(np.mean(acc) / expect - 1) < 0.03, (np.mean(acc), expect)
