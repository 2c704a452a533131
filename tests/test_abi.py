"""The C-ABI library loads and exports every symbol include/mrm_gpu.h declares
(no compute call: this runs without a GPU)."""
import os
import re

from mrm_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "mrm_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mrm_[a-z0-9_]+)\s*\(", text)))


def test_header_matches_binding_list():
    assert declared_functions() == sorted(_lib.EXPORTS)


def test_library_exports_every_symbol(gpulib):
    for name in declared_functions():
        assert hasattr(gpulib, name), name


def test_stats_layout():
    # t, step, mave/mvar/have, errmx/errmx1/mmag/energy, 4 x [8][3] per layer,
    # vol_l, msvol_l, nup_l, errmx1_l
    assert _lib.STATS_DTYPE.itemsize == 8 * (2 + 9 + 4 + 4 * 24 + 4 * 8)
