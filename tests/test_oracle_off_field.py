"""The oracle's off-plane field (off_field.f90): a slab coinciding with the
only layer gives that layer's demag field; the field decays with height;
linearity in m."""
import numpy as np

from mrm_b200 import media
from oracle import pyoracle
from tests.helpers import random_m


def test_slab_on_the_layer_is_its_demag():
    med = media.mh_medium(16, boundary=0, seed=3)  # periodic, one grain per cell
    sim = pyoracle.OracleSim(med)
    m = random_m(med.layers[0].N, 5)
    sim.set_state(0, m)
    sim.eval_field(0.0)
    hd = sim.get_demag(0)  # per grain = per cell, grain n at (n % nx, n // nx)
    dz = med.dz[0]
    h = sim.off_field(-dz, dz, num_images=med.images, space_to_sul=med.space_to_sul)
    grid = np.stack([h[c].reshape(-1) for c in range(3)], axis=1)
    assert np.abs(grid - hd).max() < 1e-9 * np.abs(hd).max()
    sim.close()


def test_decay_and_linearity():
    med = media.mh_medium(16, boundary=0, seed=4)
    sim = pyoracle.OracleSim(med)
    m = random_m(med.layers[0].N, 6)
    sim.set_state(0, m)
    near = sim.off_field(2e-7, 1e-7)
    far = sim.off_field(20e-7, 1e-7)
    assert np.abs(far).max() < 0.5 * np.abs(near).max()
    sim.set_state(0, -m)
    assert np.allclose(sim.off_field(2e-7, 1e-7), -near, rtol=0, atol=1e-12 * np.abs(near).max())
    sim.close()
