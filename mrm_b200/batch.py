"""Batched form: many media realisations advanced by one launch sequence.

A `Batch` wraps the C ABI's mrm_batch: every active run (a medium with its
own size, schedule, temperature, seed, dt and step budget) is covered by one
task table, so each Heun stage is a single kernel launch over all runs'
rows and spectral columns, replayed from captured CUDA graphs.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import MrmError
from .llg import _RunMixin, geom_of


class BatchRun(_RunMixin):
    """One run inside a Batch (the mrm_gpu handle it owns)."""

    def __init__(self, batch: "Batch", h: C.c_void_p, medium):
        self.batch = batch
        self.h = h
        self.medium = medium
        self.dt = None
        self.step_end = None

    def set_run(self, dt: float, step_end: int, active: bool = True):
        self._check(_lib.load().mrm_batch_set_run(self.h, float(dt), int(step_end), 1 if active else 0))
        self.dt = dt
        self.step_end = step_end

    def delay(self, idle_steps: int):
        """Aligned start: the run idles through the first `idle_steps` steps of
        the batch's next call, then executes its budget unchanged."""
        self._check(_lib.load().mrm_batch_delay_run(self.h, int(idle_steps)))


class Batch:
    def __init__(self, precision: int = _lib.FP32, device: int = 0):
        L = _lib.load()
        b = C.c_void_p()
        rc = L.mrm_batch_create(precision, device, C.byref(b))
        if rc != 0:
            raise MrmError(rc, (L.mrm_batch_last_error(None) or b"").decode())
        self.b = b
        self.precision = precision
        self.device = device
        self.runs: List[BatchRun] = []

    def _check(self, rc: int):
        if rc != 0:
            raise MrmError(rc, (_lib.load().mrm_batch_last_error(self.b) or b"").decode())

    def add(self, medium, dt: float = 1e-13, steps: Optional[int] = None, thermal_seed: int = 1,
            demag: bool = True, tensor_from: Optional[_RunMixin] = None,
            tensor: Optional[np.ndarray] = None) -> BatchRun:
        """Adds a run; `steps` is its step budget from its current step (None: unbounded)."""
        g = geom_of(medium, self.precision)
        h = C.c_void_p()
        self._check(_lib.load().mrm_batch_add(self.b, C.byref(g), C.byref(h)))
        run = BatchRun(self, h, medium)
        run.upload_medium(medium, thermal_seed)
        if demag:
            if tensor_from is not None:
                run._check(_lib.load().mrm_gpu_copy_tensor(run.h, tensor_from.h))
            elif tensor is not None:
                run.upload_tensor(tensor)
            else:
                run.build_tensor()
        else:
            run.set_demag(False)
        run.set_run(dt, int(steps) if steps is not None else 2**62)
        self.runs.append(run)
        return run

    def remove(self, run: BatchRun):
        """Takes the run out; its device memory is released at the next
        stats, step or close."""
        self._check(_lib.load().mrm_batch_remove(self.b, run.h))
        self.runs.remove(run)
        run.h = None

    def adopt(self, run: BatchRun):
        """Moves a run of another batch (same precision and device) into this
        one, without a device copy."""
        src = run.batch
        self._check(_lib.load().mrm_batch_adopt(self.b, src.b, run.h))
        src.runs.remove(run)
        run.batch = self
        self.runs.append(run)

    def step(self, nsteps: int, llg_type: int = -3):
        self._check(_lib.load().mrm_batch_step(self.b, int(nsteps), int(llg_type)))

    def enqueue(self, nsteps: int, llg_type: int = -3):
        self._check(_lib.load().mrm_batch_enqueue(self.b, int(nsteps), int(llg_type)))

    def stats(self, runs: Optional[Sequence[BatchRun]] = None) -> np.ndarray:
        runs = list(self.runs if runs is None else runs)
        out = np.zeros(len(runs), _lib.STATS_DTYPE)
        arr = (C.c_void_p * max(1, len(runs)))(*[r.h for r in runs])
        self._check(_lib.load().mrm_batch_stats(self.b, len(runs), arr, out.ctypes.data))
        return out

    def stream(self) -> int:
        s = C.c_void_p()
        self._check(_lib.load().mrm_batch_stream(self.b, C.byref(s)))
        return s.value or 0

    def profile(self, reps: int) -> np.ndarray:
        """Per-kernel ms of one Heun step (predictor row, column, corrector row, column)."""
        out = np.zeros(4)
        self._check(_lib.load().mrm_batch_profile(self.b, int(reps), out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def occupancy(self):
        o = (C.c_int * 2)()
        self._check(_lib.load().mrm_batch_occupancy(self.b, o))
        return int(o[0]), int(o[1])

    def close(self):
        if getattr(self, "b", None):
            _lib.load().mrm_batch_destroy(self.b)
            self.b = None
            for r in self.runs:
                r.h = None
            self.runs = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def footprint(medium, precision: int = _lib.FP32) -> int:
    """Device bytes a run of this medium holds (plus its tensor)."""
    g = geom_of(medium, precision)
    return int(_lib.load().mrm_run_footprint(C.byref(g)))


def device_memory(device: int = 0):
    f, t = C.c_int64(), C.c_int64()
    rc = _lib.load().mrm_device_memory(device, C.byref(f), C.byref(t))
    if rc != 0:
        raise MrmError(rc, "mrm_device_memory failed")
    return f.value, t.value
