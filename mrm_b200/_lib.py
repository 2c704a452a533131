"""ctypes bindings of include/mrm_gpu.h (the C ABI in mrm_b200/libmrm_gpu.so).

There is no CPU fallback: if the library is missing or cannot be loaded,
loading raises.  The Fortran host binds the same symbols through the
ISO_C_BINDING interface in mrm_b200/shim/mrm_gpu_m.f90.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmrm_gpu.so")

MAX_LAYERS = 8
OK, ERR_ARG, ERR_CUDA, ERR_UNSUPPORTED, ERR_STATE, ERR_NOMEM, ERR_DEVICE = range(7)
PERIODIC, OPEN = 0, 1
FP32, FP64 = 0, 1

ERROR_NAMES = {0: "MRM_OK", 1: "MRM_ERR_ARG", 2: "MRM_ERR_CUDA", 3: "MRM_ERR_UNSUPPORTED",
               4: "MRM_ERR_STATE", 5: "MRM_ERR_NOMEM", 6: "MRM_ERR_DEVICE"}

# every symbol include/mrm_gpu.h declares
EXPORTS = [
    "mrm_gpu_create", "mrm_gpu_destroy", "mrm_gpu_last_error", "mrm_gpu_upload_layer",
    "mrm_gpu_upload_interlayer", "mrm_gpu_build_tensor", "mrm_gpu_upload_tensor",
    "mrm_gpu_download_tensor", "mrm_gpu_fft_grid", "mrm_gpu_tensor_residual", "mrm_gpu_set_demag",
    "mrm_gpu_set_uniform_field", "mrm_gpu_set_thermal", "mrm_gpu_set_state", "mrm_gpu_get_state",
    "mrm_gpu_get_field", "mrm_gpu_set_time", "mrm_gpu_get_time", "mrm_gpu_eval_field",
    "mrm_gpu_step", "mrm_gpu_enqueue_steps", "mrm_gpu_read_stats", "mrm_gpu_stream", "mrm_gpu_profile",
    "mrm_batch_enqueue", "mrm_batch_stream", "mrm_batch_create", "mrm_batch_destroy", "mrm_batch_last_error",
    "mrm_batch_add", "mrm_batch_remove", "mrm_batch_adopt", "mrm_batch_set_run", "mrm_batch_delay_run",
    "mrm_batch_step", "mrm_batch_stats",
    "mrm_run_footprint", "mrm_device_memory", "mrm_gpu_copy_tensor", "mrm_batch_occupancy",
    "mrm_gpu_set_field_function", "mrm_gpu_demag_noalloc", "mrm_batch_profile", "mrm_gpu_set_head_field",
    "mrm_gpu_set_shape", "mrm_gpu_set_autotune", "mrm_gpu_get_shape", "mrm_gpu_check_device",
    "mrm_gpu_selftest_timeout",
    "mrm_gpu_set_cubic_axes", "mrm_gpu_step_adaptive", "mrm_gpu_off_field", "mrm_gpu_set_field_table",
    "mrm_gpu_set_window", "mrm_gpu_get_window", "mrm_gpu_set_llb", "mrm_gpu_set_mag", "mrm_gpu_get_mag",
    "mrm_gpu_set_mt", "mrm_gpu_set_temp_profile", "mrm_gpu_set_temp_function",
    "mrm_gpu_set_zhang", "mrm_gpu_set_temp_scaling", "mrm_gpu_set_temp_scaling_table",
    "mrm_gpu_get_temp_scaling_table",
]


class Geom(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("n_lay", C.c_int32),
        ("boundary", C.c_int32), ("num_images", C.c_int32), ("precision", C.c_int32),
        ("dx", C.c_double), ("dy", C.c_double),
        ("dz", C.c_double * MAX_LAYERS), ("il_space", C.c_double * MAX_LAYERS),
        ("space_to_sul", C.c_double), ("sul_mu", C.c_double), ("head_mu", C.c_double),
        ("fly_height", C.c_double),
    ]


STATS_DTYPE = np.dtype([
    ("t", "f8"), ("step", "i8"),
    ("mave", "f8", 3), ("mvar", "f8", 3), ("have", "f8", 3),
    ("errmx", "f8"), ("errmx1", "f8"), ("mmag", "f8"), ("energy", "f8"),
    ("mave_l", "f8", (MAX_LAYERS, 3)), ("mvar_l", "f8", (MAX_LAYERS, 3)),
    ("have_l", "f8", (MAX_LAYERS, 3)), ("mms_l", "f8", (MAX_LAYERS, 3)),
    ("vol_l", "f8", MAX_LAYERS), ("msvol_l", "f8", MAX_LAYERS), ("nup_l", "i8", MAX_LAYERS),
    ("errmx1_l", "f8", MAX_LAYERS),
])

_L = None


class MrmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


def load(path: str = LIB_PATH):
    """Loads the CUDA library; raises if it is missing (no fallback)."""
    global _L
    if _L is not None:
        return _L
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m mrm_b200.build` "
                          "(there is no CPU fallback)")
    L = C.CDLL(path)
    P = C.POINTER
    d, i, i32, vp, u64, i64 = C.c_double, C.c_int, C.c_int32, C.c_void_p, C.c_uint64, C.c_int64
    pd, pi32 = P(d), P(i32)
    sig = {
        "mrm_gpu_create": ([P(Geom), i, P(vp)], i),
        "mrm_gpu_destroy": ([vp], i),
        "mrm_gpu_last_error": ([vp], C.c_char_p),
        "mrm_gpu_upload_layer": ([vp, i, i, pd, pd, pd, pd, pd, pd, pd, d, d, d, pi32, pi32, pi32,
                                  pi32, pd], i),
        "mrm_gpu_upload_interlayer": ([vp, i, i, pi32, pi32, pd], i),
        "mrm_gpu_build_tensor": ([vp], i),
        "mrm_gpu_upload_tensor": ([vp, pd, i, i], i),
        "mrm_gpu_download_tensor": ([vp, pd], i),
        "mrm_gpu_fft_grid": ([vp, P(i), P(i)], i),
        "mrm_gpu_tensor_residual": ([vp, pd, pd], i),
        "mrm_gpu_set_demag": ([vp, i], i),
        "mrm_gpu_set_uniform_field": ([vp, i, pd, d, d, d, d, d], i),
        "mrm_gpu_set_thermal": ([vp, i, i, d, u64], i),
        "mrm_gpu_set_state": ([vp, i, pd], i),
        "mrm_gpu_get_state": ([vp, i, pd], i),
        "mrm_gpu_get_field": ([vp, i, pd], i),
        "mrm_gpu_set_time": ([vp, d, i64], i),
        "mrm_gpu_get_time": ([vp, pd, P(i64)], i),
        "mrm_gpu_eval_field": ([vp, d, i, pd], i),
        "mrm_gpu_step": ([vp, i, d, i, vp], i),
        "mrm_gpu_enqueue_steps": ([vp, i, d, i], i),
        "mrm_gpu_read_stats": ([vp, vp], i),
        "mrm_gpu_stream": ([vp, P(vp)], i),
        "mrm_gpu_profile": ([vp, i, d, pd], i),
        "mrm_batch_enqueue": ([vp, i, i], i),
        "mrm_batch_stream": ([vp, P(vp)], i),
        "mrm_batch_create": ([i, i, P(vp)], i),
        "mrm_batch_destroy": ([vp], i),
        "mrm_batch_last_error": ([vp], C.c_char_p),
        "mrm_batch_add": ([vp, P(Geom), P(vp)], i),
        "mrm_batch_remove": ([vp, vp], i),
        "mrm_batch_adopt": ([vp, vp, vp], i),
        "mrm_batch_set_run": ([vp, d, i64, i], i),
        "mrm_batch_delay_run": ([vp, i64], i),
        "mrm_batch_step": ([vp, i, i], i),
        "mrm_batch_stats": ([vp, i, P(vp), vp], i),
        "mrm_run_footprint": ([P(Geom)], i64),
        "mrm_gpu_copy_tensor": ([vp, vp], i),
        "mrm_gpu_set_field_function": ([vp, i, pd, i, d, d, d, d, d, d, d, d], i),
        "mrm_batch_occupancy": ([vp, P(i)], i),
        "mrm_device_memory": ([i, P(i64), P(i64)], i),
        "mrm_gpu_demag_noalloc": ([vp, vp, vp, vp], i),
        "mrm_batch_profile": ([vp, i, pd], i),
        "mrm_gpu_set_head_field": ([vp, i, d, d, d, d, d, d, d, u64, i], i),
        "mrm_gpu_set_cubic_axes": ([vp, i, pd], i),
        "mrm_gpu_step_adaptive": ([vp, i, i, d, d, pd, pd, pd, vp], i),
        "mrm_gpu_off_field": ([vp, d, d, d, d, d, d, i, pd], i),
        "mrm_gpu_set_field_table": ([vp, i, i, i, pd, pd, pd, d, d, d, d, d, d, d], i),
        "mrm_gpu_set_window": ([vp, i, i, d, d, d, d], i),
        "mrm_gpu_get_window": ([vp, P(i)], i),
        "mrm_gpu_set_llb": ([vp, i, d, pd, pd], i),
        "mrm_gpu_set_mt": ([vp, i, d, pd, i, i], i),
        "mrm_gpu_set_zhang": ([vp, i, d, pd, i, i], i),
        "mrm_gpu_set_temp_profile": ([vp, i, d, d, d, d, i, d, d, d, d, d, d, d], i),
        "mrm_gpu_set_temp_function": ([vp, i, i] + [d] * 12, i),
        "mrm_gpu_set_temp_scaling": ([vp, i, pd, d, d, i], i),
        "mrm_gpu_set_temp_scaling_table": ([vp, i, i, i, pd, pd], i),
        "mrm_gpu_get_temp_scaling_table": ([vp, i, i, C.POINTER(C.c_int), pd, pd], i),
        "mrm_gpu_set_mag": ([vp, i, pd], i),
        "mrm_gpu_get_mag": ([vp, i, pd], i),
        "mrm_gpu_set_shape": ([vp, i, i, i], i),
        "mrm_gpu_set_autotune": ([vp, i], i),
        "mrm_gpu_get_shape": ([vp, P(i)], i),
        "mrm_gpu_check_device": ([vp], i),
        "mrm_gpu_selftest_timeout": ([vp], i),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _L = L
    return L


def fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def iptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32)) if a is not None else None


def f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def i32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int32)
