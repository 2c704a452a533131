"""Generates tests/golden/c2_mh.npz with the CPU oracle (test infrastructure).

The 65,536-grain M(H) workload: the 4,096-grain medium of make_golden.py
scaled to 256 x 256 grains as lattice nodes (8 nm pitch, 10 nm thick, Ms 700
emu/cm3, Hk 15 kOe with 5 % Gaussian spread, easy axes within 3 degrees,
500 Oe nearest-neighbour exchange, alpha 0.1), open boundary on a 512 x 512
padded FFT grid, T = 300 K, the linear ramp from +20 kOe to -20 kOe along
(sin 10 deg, 0, cos 10 deg) over 2 ns (src/applied.f90:871-883), Heun steps
of 0.1 ps (src/llg.f90:1122-1139), 20,000 steps.

Stored, per seed of the FP64 Philox thermal stream (seeds 1..4): the M(H)
branch sampled every 100 steps (applied field and the Ms-weighted mean of m
along the field direction), its coercivity and remanence.  The ensemble means
are the Hc/Mr gate of the FP32 batched GPU path; the seed-to-seed spread at
this size is about 0.1 % of Hc.

The reference itself cannot be built here (no Fortran compiler, no FFTW), so
these vectors pin the GPU path to the oracle's restatement of it at the full
65,536-grain size.  About 45 minutes on 8 host cores.  Run from the
repository root:  python tests/golden/make_golden_c2.py
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from mrm_b200 import media  # noqa: E402
from oracle import pyoracle  # noqa: E402
from tests.golden.make_golden import CHUNK, DT, STEPS, applied, coercivity  # noqa: E402

SIDE = 256
SEEDS = (1, 2, 3, 4)


def main():
    pyoracle.build()
    pyoracle.set_threads(os.cpu_count() or 1)
    hs_all, mh_all, hcs, mrs = [], [], [], []
    for s in SEEDS:
        t0 = time.time()
        med = media.mh_medium(SIDE, boundary=1, temperature=300.0, seed=1)
        hdir = np.array(med.layers[0].hdir)
        sim = pyoracle.OracleSim(med, rng_mode=1, seed=s)
        hs, mhs = [], []
        for _ in range(STEPS // CHUNK):
            st = sim.step(CHUNK, DT)
            hs.append(applied(float(st["t"])))
            mhs.append(float(st["mms_l"][0] @ hdir))
        sim.close()
        hc, mr = coercivity(hs, mhs)
        hs_all.append(hs)
        mh_all.append(mhs)
        hcs.append(hc)
        mrs.append(mr)
        print(f"seed {s}: Hc {hc:.2f} Oe, Mr {mr:.5f} ({time.time() - t0:.0f} s)", flush=True)
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "c2_mh.npz"),
                        seeds=np.array(SEEDS), h=np.array(hs_all[0]), mh=np.array(mh_all),
                        hc=np.array(hcs), mr=np.array(mrs))


if __name__ == "__main__":
    main()
