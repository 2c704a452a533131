"""Precision of the magnetostatic tensor elements.

The reference's closed forms (src/tensor_element.f90:78-100) sum 64 signed
corner terms that grow like r^3 log r into a result of order 1/r^3.  Evaluated
in FP64 (as the reference and the oracle do) the far-field elements lose about
(r / cell)^6 of the 2^-53 precision; the oracle's quadruple-precision
evaluation of the same formula measures that.  The device evaluates the
formula in double-double arithmetic (mrm_b200/csrc/dd.cuh), whose operations
are checked here against quadruple precision on the host; the device tensor
itself is checked against quadruple precision in tests/test_gpu_parity_full.py.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from mrm_b200 import media

HERE = os.path.dirname(os.path.abspath(__file__))


def _slot(oracle, med, o, fi, fj):
    q = oracle.tensor_slot_q(o.px, o.py, med.dx, med.dy, med.dz[0], med.dz[0], 0.0, fi, fj)
    return q.reshape(3, 3).T.reshape(9), o.n2d[0, 0, :, fj, fi]  # n2d component 3b + a holds t(a, b)


def test_fp64_tensor_far_field_is_rounding_noise(oracle):
    med = media.mh_medium(256, boundary=1, seed=1)  # 512 x 512 open grid
    o = oracle.OracleSim(med)
    scale = np.abs(o.n2d).max()
    for fi, fj in [(0, 0), (1, 0), (0, 1), (2, 3)]:  # near field: FP64 to ~1e-11
        q, n = _slot(oracle, med, o, fi, fj)
        assert np.abs(n - q).max() < 1e-10 * np.abs(q).max(), (fi, fj)
    far = []
    for fi, fj in [(128, 100), (250, 3), (256, 256), (300, 400)]:
        q, n = _slot(oracle, med, o, fi, fj)
        assert np.abs(q).max() < 1e-7 * scale  # far field: ~1e-8 of the self term
        far.append(np.abs(n - q).max() / np.abs(q).max())
    # the FP64 values of the far elements are wrong by several percent and more
    assert min(far) > 1e-3, far
    o.close()


def test_double_double_against_quad(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    exe = str(tmp_path / "dd_check")
    subprocess.run([gxx, "-O2", "-std=gnu++17", os.path.join(HERE, "cpu_helpers", "dd_check.cpp"), "-o", exe,
                    "-lquadmath"], check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()
    err_log, err_atan, err_sqrt, err_div = (float(x) for x in out)
    # about 106 significant bits: 2^-106 ~ 1.2e-32
    assert err_log < 1e-29 and err_atan < 1e-29 and err_sqrt < 1e-30 and err_div < 1e-30, out
