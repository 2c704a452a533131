"""Off-plane (readback) field on the GPU (mrm_gpu_off_field) against the
oracle's restatement of off_field.f90: one and two layers, soft-underlayer
and head images, a grain map."""
import numpy as np
import pytest

from mrm_b200 import FP32, FP64, GpuSim, media
from tests.helpers import random_m, rel_l2

pytestmark = pytest.mark.gpu


def _both(oracle, med, precision, states, **kw):
    orc = oracle.OracleSim(med, demag=False)
    gpu = GpuSim(med, precision=precision, demag=False)
    for l, m in enumerate(states):
        orc.set_state(l, m)
        gpu.set_state(l, m)
    out = gpu.off_field(**kw), orc.off_field(**kw)
    gpu.close()
    orc.close()
    return out


# The device tensor's closed forms (CUDA atan/log) differ from the host's by
# ulps inside the cancellation-prone 64-corner sums, and the periodic image
# sums add them up: 3e-7 relative measured on the field (the device-built
# demag tensor of periodic grids shows the same, 1e-7); FP32 states are rounded.
@pytest.mark.parametrize("precision,tol", [(FP64, 1e-6), (FP32, 2e-6)])
def test_off_field_one_layer(oracle, gpulib, precision, tol):
    med = media.mh_medium(32, boundary=0, seed=3)
    m = random_m(med.layers[0].N, 8)
    g, o = _both(oracle, med, precision, [m], zoff=3e-7, dzobs=2e-7)
    assert rel_l2(g, o) < tol


def test_off_field_two_layers_images(oracle, gpulib):
    med = media.two_layer_medium(32, 16, seed=2, temperature=0.0, boundary=0)
    st = [random_m(lay.N, 20 + k) for k, lay in enumerate(med.layers)]
    g, o = _both(oracle, med, FP64, st, zoff=4e-7, dzobs=1e-7, head_mu=50.0, fly_height=6e-7, sul_mu=100.0,
                 space_to_sul=20e-7, num_images=1)
    assert rel_l2(g, o) < 1e-6  # 7.7e-8 measured


def test_off_field_grain_map(oracle, gpulib):
    med = media.grain_map_medium(16, 16, seed=6, boundary=0)
    m = random_m(med.layers[0].N, 9)
    g, o = _both(oracle, med, FP64, [m], zoff=2e-7, dzobs=2e-7)
    assert rel_l2(g, o) < 1e-6
