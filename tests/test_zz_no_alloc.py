"""Allocation-free demag evaluation (mrm_gpu_demag_noalloc) against the
allocating entry point (mrm_gpu_eval_field) of the same handle.

Collected last on purpose: it must pass alone and after every other test (the
static scratch and the per-device set-up outlive the handles of the tests
before it)."""
import contextlib
import ctypes as C

import numpy as np
import pytest

from helpers import random_m, rel_l2, small_medium, two_layer

# the same four kernels on the same inputs: equal up to FP32 rounding of m
TOL = 1e-6


def _demag_both(gpulib, sim, states, stream=None):
    """Demag of each state through eval_field and through two noalloc calls in
    a row.  stream: a torch stream the tensors are made on and the calls are
    enqueued on (None: the handle's own stream)."""
    import torch

    nl, n = sim.medium.n_lay, sim.medium.layers[0].N
    ref = []
    for st in states:
        for l in range(nl):
            sim.set_state(l, st[l])
        ref.append(np.stack([sim.eval_field(0.0, l) for l in range(nl)]))
    outs = []
    ctx = torch.cuda.stream(stream) if stream is not None else contextlib.nullcontext()
    with ctx:
        for st in states:
            m_dev = torch.tensor(np.asarray(st, np.float32).reshape(nl, n, 3), device="cuda")
            h_dev = torch.full((nl, n, 3), float("nan"), dtype=torch.float32, device="cuda")
            if stream is None:
                torch.cuda.synchronize()
            handle = C.c_void_p(stream.cuda_stream) if stream is not None else None
            rc = gpulib.mrm_gpu_demag_noalloc(sim.h, C.c_void_p(m_dev.data_ptr()), C.c_void_p(h_dev.data_ptr()),
                                              handle)
            assert rc == 0, gpulib.mrm_gpu_last_error(sim.h)
            outs.append((m_dev, h_dev))
    if stream is not None:
        stream.synchronize()  # only the caller's stream: the work was enqueued there
    else:
        torch.cuda.synchronize()
    got = [h.cpu().numpy().astype(float) for _, h in outs]
    # a kernel failure of the calls is recorded in the handle's device error word
    assert gpulib.mrm_gpu_check_device(sim.h) == 0, gpulib.mrm_gpu_last_error(sim.h)
    return ref, got


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
    # a stream of the caller's own, not the default stream (whose handle is 0,
    # which the entry point reads as "the handle's stream")
    ref, got = _demag_both(gpulib, sim, states, stream=torch.cuda.Stream())
    for r, g in zip(ref, got):
        assert rel_l2(g, r) < TOL


@pytest.mark.gpu
def test_noalloc_allocates_nothing(gpulib):
    """After the first call on the device (its set-up), further calls leave the
    device's free memory and torch's allocator untouched."""
    import torch

    from mrm_b200 import FP32, GpuSim

    med = small_medium(64, boundary=1, seed=23)
    sim = GpuSim(med, precision=FP32)
    n = med.layers[0].N
    m_dev = torch.tensor(np.asarray(random_m(n, 5), np.float32), device="cuda")
    h_dev = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    call = lambda: gpulib.mrm_gpu_demag_noalloc(sim.h, C.c_void_p(m_dev.data_ptr()),  # noqa: E731
                                                C.c_void_p(h_dev.data_ptr()), None)
    assert call() == 0
    torch.cuda.synchronize()

    def snapshot():
        f, t = C.c_int64(), C.c_int64()
        assert gpulib.mrm_device_memory(0, C.byref(f), C.byref(t)) == 0
        st = torch.cuda.memory_stats()
        return f.value, torch.cuda.memory_allocated(), st.get("allocation.all.allocated", 0)

    before = snapshot()
    for _ in range(5):
        assert call() == 0
    torch.cuda.synchronize()
    assert snapshot() == before
    assert np.isfinite(h_dev.cpu().numpy()).all()


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
