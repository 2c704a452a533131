"""Generates tests/golden/c1_mh.npz with the CPU oracle (test infrastructure).

The 4,096-grain M(H) workload (64 x 64 grains as lattice nodes, 8 nm pitch,
10 nm thick, Ms 700 emu/cm3, Hk 15 kOe with 5 % Gaussian spread, easy axes
within 3 degrees, 500 Oe nearest-neighbour exchange, alpha 0.1, open boundary
on a 128 x 128 padded FFT grid), driven by the linear ramp from +20 kOe to
-20 kOe along (sin 10 deg, 0, cos 10 deg) over 2 ns (src/applied.f90:871-883)
with Heun steps of 0.1 ps (src/llg.f90:1122-1139), 20,000 steps:

* T = 0, FP64: the M(H) branch sampled every 100 steps (applied field and the
  Ms-weighted mean of m along the field direction) and the final state;
* T = 300 K, FP64, Philox thermal stream seeds 1..8 (the stream the GPU's FP64
  runs draw): the coercivity and remanence of each seed's branch.

The reference itself cannot be built here (no Fortran compiler, no FFTW), so
these vectors pin the GPU path to the oracle's restatement of it at the full
4,096-grain size; tests/test_oracle_golden.py checks that the oracle still
reproduces them.  Run from the repository root:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from mrm_b200 import media  # noqa: E402
from oracle import pyoracle  # noqa: E402

SIDE, STEPS, CHUNK, DT = 64, 20000, 100, 1e-13
SEEDS = tuple(range(1, 9))


def applied(t):
    """Ramp magnitude (Oe) at time t."""
    return 20000.0 - 40000.0 * min(1.0, max(0.0, t / (STEPS * DT)))


def coercivity(h, mh):
    """Hc, Mr of a descending branch by linear interpolation at the sign changes."""
    hc = mr = None
    for k in range(1, len(h)):
        if mh[k - 1] > 0 >= mh[k] and hc is None:
            hc = -(h[k - 1] + (h[k] - h[k - 1]) * mh[k - 1] / (mh[k - 1] - mh[k]))
        if h[k - 1] > 0 >= h[k] and mr is None:
            mr = mh[k - 1] + (mh[k] - mh[k - 1]) * h[k - 1] / (h[k - 1] - h[k])
    return hc, mr


def branch(sim, hdir):
    hs, mhs = [], []
    for _ in range(STEPS // CHUNK):
        st = sim.step(CHUNK, DT)
        hs.append(applied(float(st["t"])))
        mhs.append(float(st["mms_l"][0] @ hdir))
    return np.array(hs), np.array(mhs)


def main():
    pyoracle.build()
    pyoracle.set_threads(os.cpu_count() or 1)
    out = {}
    med = media.mh_medium(SIDE, boundary=1, temperature=0.0, seed=1)
    hdir = np.array(med.layers[0].hdir)
    sim = pyoracle.OracleSim(med)
    h, mh = branch(sim, hdir)
    out.update(t0_h=h, t0_mh=mh, t0_m=sim.get_state(0))
    sim.close()
    hcs, mrs = [], []
    for s in SEEDS:
        med = media.mh_medium(SIDE, boundary=1, temperature=300.0, seed=1)
        sim = pyoracle.OracleSim(med, rng_mode=1, seed=s)
        h, mh = branch(sim, hdir)
        sim.close()
        hc, mr = coercivity(h, mh)
        hcs.append(hc)
        mrs.append(mr)
        print(f"seed {s}: Hc {hc:.2f} Oe, Mr {mr:.5f}", flush=True)
    out.update(t300_seeds=np.array(SEEDS), t300_hc=np.array(hcs), t300_mr=np.array(mrs))
    hc0, mr0 = coercivity(out["t0_h"], out["t0_mh"])
    print(f"T=0: Hc {hc0:.2f} Oe, Mr {mr0:.5f}")
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "c1_mh.npz"), **out)


if __name__ == "__main__":
    main()
