"""Pins the oracle FFT to FFTW's unnormalised r2c/c2r semantics (fftw.f90:37-93)
using numpy's pocketfft."""
import numpy as np
import pytest


@pytest.mark.parametrize("shape", [(8, 8), (16, 32), (5, 12), (64, 128), (3, 7)])
def test_r2c_c2r(oracle, shape):
    x = np.random.default_rng(1).standard_normal(shape)
    c = oracle.fft_r2c(x)
    assert np.allclose(c, np.fft.rfft2(x), rtol=0, atol=1e-11 * x.size)
    r = oracle.fft_c2r(c, shape[1])
    assert np.allclose(r, x * x.size, rtol=0, atol=1e-10 * x.size)
