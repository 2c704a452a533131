"""Allocation-free demag evaluation (mrm_gpu_demag_noalloc) against the
allocating entry point (mrm_gpu_eval_field) of the same handle.

Collected last on purpose: it must pass alone and after every other test (the
static scratch and the per-device set-up outlive the handles of the tests
before it)."""
import ctypes as C

import numpy as np
import pytest

from helpers import random_m, rel_l2, small_medium, two_layer

# the same four kernels on the same inputs: equal up to FP32 rounding of m
TOL = 1e-6


def _demag_both(gpulib, sim, states, stream=None):
    """Demag of each state through eval_field and through two noalloc calls in a row."""
    import torch

    nl, n = sim.medium.n_lay, sim.medium.layers[0].N
    ref = []
    for st in states:
        for l in range(nl):
            sim.set_state(l, st[l])
        ref.append(np.stack([sim.eval_field(0.0, l) for l in range(nl)]))
    outs = []
    for st in states:
        m_dev = torch.tensor(np.asarray(st, np.float32).reshape(nl, n, 3), device="cuda")
        h_dev = torch.full((nl, n, 3), float("nan"), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        rc = gpulib.mrm_gpu_demag_noalloc(sim.h, C.c_void_p(m_dev.data_ptr()), C.c_void_p(h_dev.data_ptr()),
                                          C.c_void_p(stream))
        assert rc == 0, gpulib.mrm_gpu_last_error(sim.h)
        outs.append((m_dev, h_dev))
    torch.cuda.synchronize()
    return ref, [h.cpu().numpy().astype(float) for _, h in outs]


@pytest.mark.gpu
@pytest.mark.parametrize("boundary", [0, 1])
def test_noalloc_matches_eval_field(gpulib, boundary):
    from mrm_b200 import FP32, GpuSim

    med = small_medium(64, boundary=boundary, seed=21)
    sim = GpuSim(med, precision=FP32)
    states = [[random_m(med.layers[0].N, 100 + k)] for k in range(2)]
    ref, got = _demag_both(gpulib, sim, states)
    for r, g in zip(ref, got):
        assert np.isfinite(g).all()
        assert rel_l2(g, r) < TOL
    assert rel_l2(got[0], got[1]) > 1e-2  # the two calls saw different states


@pytest.mark.gpu
def test_noalloc_two_layers_on_torch_stream(gpulib):
    import torch

    from mrm_b200 import FP32, GpuSim

    med = two_layer(32, 16, seed=9)
    sim = GpuSim(med, precision=FP32)
    states = [[random_m(med.layers[0].N, 200 + 2 * k + l) for l in range(2)] for k in range(2)]
    ref, got = _demag_both(gpulib, sim, states, stream=torch.cuda.current_stream().cuda_stream)
    for r, g in zip(ref, got):
        assert rel_l2(g, r) < TOL


@pytest.mark.gpu
def test_noalloc_rejects_oversize_and_fp64(gpulib):
    from mrm_b200 import FP32, FP64, GpuSim, _lib
    from mrm_b200.media import mh_medium

    # 1024 x 1024 grains, open boundary: two 2048 x 1025 half spectra alone exceed the scratch
    big = GpuSim(mh_medium(1024, boundary=1, seed=1), precision=FP32, demag=False)
    rc = gpulib.mrm_gpu_demag_noalloc(big.h, C.c_void_p(16), C.c_void_p(16), None)
    assert rc == 3 and b"scratch" in gpulib.mrm_gpu_last_error(big.h)
    big.close()
    d = GpuSim(small_medium(16, boundary=1), precision=FP64)
    rc = gpulib.mrm_gpu_demag_noalloc(d.h, C.c_void_p(16), C.c_void_p(16), None)
    assert rc == 3 and b"FP32" in gpulib.mrm_gpu_last_error(d.h)
    d.close()
    assert _lib.ERROR_NAMES[3] == "MRM_ERR_UNSUPPORTED"
