"""The FP32 thermal stream's Philox4x32-10 against cuRAND's implementation of
the same published generator, bit for bit on random counters and keys."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.gpu
def test_philox4x32_matches_curand(tmp_path):
    so = str(tmp_path / "philox_pin.so")
    subprocess.run(["/usr/local/cuda/bin/nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O2",
                    "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-o", so,
                    os.path.join(HERE, "gpu_helpers", "philox_pin.cu")], check=True)
    lib = C.CDLL(so)
    n = 4096
    rng = np.random.default_rng(5)
    inp = rng.integers(0, 2 ** 32, size=(n, 6), dtype=np.uint64).astype(np.uint32)
    inp[:4] = [[0] * 6, [0xFFFFFFFF] * 6, [0, 1, 2, 3, 4, 5], [7, 0, 0, 1, 0xC0FFEE, 0x6D726D]]
    mine = np.zeros((n, 4), np.uint32)
    ref = np.zeros((n, 4), np.uint32)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    assert lib.philox_pin(p(inp), n, p(mine), p(ref)) == 0
    assert np.array_equal(mine, ref)
    assert len(np.unique(mine)) > 4 * n - 10  # not degenerate
