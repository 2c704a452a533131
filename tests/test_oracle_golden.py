"""The oracle still reproduces the golden vectors of tests/golden/c1_mh.npz
(the first 1,000 steps of the T = 0 branch), and the vectors are consistent:
the T = 0 branch switches, and the T = 300 K coercivities sit below it."""
import os

import numpy as np

from mrm_b200 import media
from oracle import pyoracle

HERE = os.path.dirname(os.path.abspath(__file__))


def test_oracle_reproduces_c1_branch_start():
    g = np.load(os.path.join(HERE, "golden", "c1_mh.npz"))
    med = media.mh_medium(64, boundary=1, temperature=0.0, seed=1)
    hdir = np.array(med.layers[0].hdir)
    sim = pyoracle.OracleSim(med)
    mh = []
    for _ in range(10):
        st = sim.step(100, 1e-13)
        mh.append(float(st["mms_l"][0] @ hdir))
    sim.close()
    # threads only reorder FP64 reductions
    assert np.max(np.abs(np.array(mh) - g["t0_mh"][:10])) < 1e-12


def test_golden_vectors_consistent():
    g = np.load(os.path.join(HERE, "golden", "c1_mh.npz"))
    assert g["t0_mh"][0] > 0.9 and g["t0_mh"][-1] < -0.9
    assert g["t0_m"].shape == (4096, 3)
    assert np.allclose(np.linalg.norm(g["t0_m"], axis=1), 1.0, atol=1e-12)
    assert len(g["t300_hc"]) == 8 and np.all(g["t300_hc"] > 0)
    t0 = g["t0_mh"]
    k = int(np.argmax(t0 <= 0))
    h0 = g["t0_h"]
    hc0 = -(h0[k - 1] + (h0[k] - h0[k - 1]) * t0[k - 1] / (t0[k - 1] - t0[k]))
    assert np.all(g["t300_hc"] < hc0)  # thermal activation lowers the coercivity
