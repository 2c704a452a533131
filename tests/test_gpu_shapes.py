"""Kernel shapes (rows per block, threads, columns per task) and the autotuner
change how the work is split, never the arithmetic: trajectories must be
bit-identical across every compiled shape."""
import numpy as np
import pytest

from helpers import small_medium, two_layer

DT = 1e-13


def _run(med, precision, shape=None, autotune=True, steps=40):
    from mrm_b200 import GpuSim
    sim = GpuSim(med, precision=precision, thermal_seed=5)
    if shape is not None:
        sim.set_shape(*shape)
    else:
        sim.set_autotune(autotune)
    st = sim.step(steps, DT)
    out = [sim.get_state(l) for l in range(med.n_lay)], sim.get_shape(), st
    sim.close()
    return out


def _shapes(precision):
    from mrm_b200 import FP32
    nrow, ncol = (5, 3) if precision == FP32 else (3, 2)
    return [(rv, cv, cpt) for rv in range(nrow) for cv, cpt in ((0, 0), (ncol - 1, 1), (1, 4))]


@pytest.mark.gpu
@pytest.mark.parametrize("prec_name", ["fp32", "fp64"])
def test_shapes_bit_identical(gpulib, prec_name):
    from mrm_b200 import FP32, FP64
    precision = FP32 if prec_name == "fp32" else FP64
    med = small_medium(64, boundary=1, seed=4, temperature=300.0)  # 128 x 128 padded grid
    ref, _, st_ref = _run(med, precision, shape=(0, 0, 0))
    for shape in _shapes(precision):
        m, used, st = _run(med, precision, shape=shape)
        assert used == shape
        for a, b in zip(m, ref):
            assert np.array_equal(a, b), f"shape {shape} differs"
        assert st["mave"].tolist() == st_ref["mave"].tolist()


@pytest.mark.gpu
def test_shapes_two_layers_bit_identical(gpulib):
    from mrm_b200 import FP32
    med = two_layer(64, 32, seed=6, temperature=300.0)
    ref, _, _ = _run(med, FP32, shape=(0, 0, 0))
    for shape in [(1, 1, 1), (2, 2, 2), (3, 0, 4), (4, 1, 8)]:
        m, _, _ = _run(med, FP32, shape=shape)
        for a, b in zip(m, ref):
            assert np.array_equal(a, b), f"shape {shape} differs"


@pytest.mark.gpu
def test_autotune_restores_state(gpulib):
    """The tuner runs the kernels on the runs themselves; the trajectory after
    tuning is the one of a fixed shape."""
    from mrm_b200 import FP32
    med = small_medium(128, boundary=1, seed=8, temperature=300.0)
    ref, _, _ = _run(med, FP32, shape=(0, 0, 0), steps=64)
    m, used, _ = _run(med, FP32, autotune=True, steps=64)
    assert 0 <= used[0] < 5 and 0 <= used[1] < 3
    assert np.array_equal(m[0], ref[0])


@pytest.mark.gpu
@pytest.mark.parametrize("llg_type", [2, -2])
def test_semi_implicit_shapes_and_batch(gpulib, llg_type):
    """The semi-implicit integrators are shape-independent and batch == alone."""
    from mrm_b200 import FP32, GpuSim
    from mrm_b200.batch import Batch
    med = small_medium(64, boundary=1, seed=12, temperature=300.0)
    outs = []
    for shape in [(0, 0, 0), (1, 1, 2), (3, 2, 4)]:
        sim = GpuSim(med, precision=FP32, thermal_seed=2)
        sim.set_shape(*shape)
        st = sim.step(48, DT, llg_type=llg_type)
        outs.append((sim.get_state(0), st["mave"].copy()))
        sim.close()
    for m, mv in outs[1:]:
        assert np.array_equal(m, outs[0][0]) and np.array_equal(mv, outs[0][1])
    b = Batch(FP32)
    r = b.add(med, dt=DT, steps=48, thermal_seed=2)
    b.add(small_medium(32, boundary=1, seed=13, temperature=300.0), dt=DT, steps=48, thermal_seed=3)
    b.step(48, llg_type=llg_type)
    assert np.array_equal(r.get_state(0), outs[0][0])
    assert np.array_equal(b.stats([r])[0]["mave"], outs[0][1])
    b.close()
