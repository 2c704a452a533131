"""Host-side mirror of the reference's LLG/field interface on the GPU path.

`GpuSim` plays the role the Fortran modules play in the reference:
`construct_field`/`file_grain` hand over the per-layer arrays
(upload_layer), `init_demag` builds the tensor (build_tensor),
`set_fld`/`uniform_fld` set the applied-field schedule, `start_field` the
thermal seeds, and `llg()` advances fixed-dt steps (step).  Every call goes
through the C ABI of include/mrm_gpu.h; the class only marshals arrays.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib
from ._lib import MrmError, f64, fptr, i32, iptr


def geom_of(medium, precision: int) -> _lib.Geom:
    g = _lib.Geom()
    g.nx, g.ny, g.n_lay = medium.nx, medium.ny, medium.n_lay
    g.boundary = medium.boundary
    g.num_images = medium.images
    g.precision = precision
    g.dx, g.dy = medium.dx, medium.dy
    for l in range(medium.n_lay):
        g.dz[l] = medium.dz[l]
        g.il_space[l] = medium.il_space[l]
    g.space_to_sul = medium.space_to_sul
    g.sul_mu = medium.sul_mu
    g.head_mu = medium.head_mu
    g.fly_height = medium.fly_height
    return g


class _RunMixin:
    """C-ABI calls shared by the plain handle and batched runs."""

    h: C.c_void_p

    def _check(self, rc: int):
        if rc != 0:
            msg = _lib.load().mrm_gpu_last_error(self.h)
            raise MrmError(rc, (msg or b"").decode())

    def upload_medium(self, medium, thermal_seed: int = 1):
        L = _lib.load()
        self.medium = medium
        for l, lay in enumerate(medium.layers):
            arrs = [f64(lay.ms), f64(lay.vol), f64(lay.axis), f64(lay.hk), f64(lay.hk_scale),
                    f64(lay.ms_scale), f64(lay.alpha_scale)]
            g2ci, g2c = i32(lay.g2c_index), i32(lay.g2c)
            hxi, hxg, hx = i32(lay.hx_index), i32(lay.hx_grain), f64(lay.hx)
            self._check(L.mrm_gpu_upload_layer(self.h, l, lay.N, *[fptr(a) for a in arrs], lay.alpha,
                                               lay.gamma, lay.floor_ms, iptr(g2ci), iptr(g2c),
                                               iptr(hxi), iptr(hxg), fptr(hx)))
        for l, lay in enumerate(medium.layers):
            for side, cpl in ((0, lay.uhx), (1, lay.lhx)):
                if cpl is not None:
                    idx, gr, cf = i32(cpl[0]), i32(cpl[1]), f64(cpl[2])
                    self._check(L.mrm_gpu_upload_interlayer(self.h, l, side, iptr(idx), iptr(gr), fptr(cf)))
            if getattr(lay, "func", 0):
                self.set_field_function(l, lay.hdir, lay.func, lay.amp, lay.fgamma, lay.phase,
                                        lay.param, lay.duty, lay.moddepth, lay.dc, lay.scale)
            else:
                self.set_uniform_field(l, lay.hdir, lay.t_start, lay.t_end, lay.s_start, lay.s_end,
                                       lay.scale)
            if getattr(lay, "head", None):
                self.set_head_field(l, **lay.head)
            if getattr(lay, "field_table", None):
                self.set_field_table(l, **lay.field_table)
            if getattr(lay, "llb", None):
                self.set_llb(l, **lay.llb)
            if getattr(lay, "mt", None):
                self.set_mt(l, **lay.mt)
            if getattr(lay, "zhang", None):
                self.set_zhang(l, **lay.zhang)
            if getattr(lay, "temp_profile", None):
                self.set_temp_profile(l, **lay.temp_profile)
            if getattr(lay, "temp_scaling", None):
                self.set_temp_scaling(l, **lay.temp_scaling)
            if getattr(lay, "cubic_axis", None) is not None:
                self.set_cubic_axes(l, lay.cubic_axis)
            self.set_thermal(l, lay.thermal, lay.temperature, thermal_seed)
        if medium.m0 is not None:
            for l, m in enumerate(medium.m0):
                self.set_state(l, m)

    def build_tensor(self):
        self._check(_lib.load().mrm_gpu_build_tensor(self.h))

    def upload_tensor(self, n2d: np.ndarray):
        """Real-space FP64 tensor (n_lay, n_lay, 9, py, px) on this handle's FFT grid."""
        n2d = f64(n2d)
        px, py = self.fft_grid()
        nl = self.medium.n_lay
        if n2d.shape != (nl, nl, 9, py, px):
            raise ValueError(f"tensor of shape {n2d.shape}; this handle's grid needs {(nl, nl, 9, py, px)}")
        self._check(_lib.load().mrm_gpu_upload_tensor(self.h, fptr(n2d), px, py))

    def download_tensor(self) -> np.ndarray:
        px, py = self.fft_grid()
        nl = self.medium.n_lay
        out = np.zeros((nl, nl, 9, py, px))
        self._check(_lib.load().mrm_gpu_download_tensor(self.h, fptr(out)))
        return out

    def fft_grid(self):
        a, b = C.c_int(), C.c_int()
        self._check(_lib.load().mrm_gpu_fft_grid(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def tensor_residual(self):
        a, b = C.c_double(), C.c_double()
        self._check(_lib.load().mrm_gpu_tensor_residual(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def set_demag(self, on: bool):
        self._check(_lib.load().mrm_gpu_set_demag(self.h, 1 if on else 0))

    def set_uniform_field(self, layer, hdir, t_start, t_end, s_start, s_end, scale=1.0):
        d = f64(hdir)
        self._check(_lib.load().mrm_gpu_set_uniform_field(self.h, layer, fptr(d), t_start, t_end,
                                                          s_start, s_end, scale))

    def set_field_function(self, layer, hdir, func, amp, gamma, phase=0.0, param=0.0, duty=0.0,
                           moddepth=0.0, dc=0.0, scale=1.0):
        d = f64(hdir)
        self._check(_lib.load().mrm_gpu_set_field_function(self.h, layer, fptr(d), int(func), amp,
                                                           gamma, phase, param, duty, moddepth,
                                                           dc, scale))

    def set_head_field(self, layer, gap, z, hg, velocity, x0, t0, bit_time, pattern, nbits):
        self._check(_lib.load().mrm_gpu_set_head_field(self.h, layer, gap, z, hg, velocity, x0, t0,
                                                       bit_time, int(pattern), int(nbits)))

    def set_field_table(self, layer, xpos, ypos, vfld, vel=(0.0, 0.0), offset=(None, None), ref=(0.0, 0.0),
                        t_origin=0.0):
        """Tabulated (moving) field profile on `layer` (include/mrm_gpu.h
        mrm_gpu_set_field_table): vfld (ny_tab, nx_tab, 3) in Oe at ascending
        node positions xpos (nx_tab), ypos (ny_tab) in cm; offset None: the
        grid centre; vfld None removes the profile."""
        L = _lib.load()
        if vfld is None:
            self._check(L.mrm_gpu_set_field_table(self.h, layer, 0, 0, None, None, None, 0.0, 0.0, 0.0, 0.0,
                                                  0.0, 0.0, 0.0))
            return
        xp, yp, v = f64(xpos), f64(ypos), f64(vfld)
        if v.shape != (yp.size, xp.size, 3):
            raise ValueError(f"vfld of shape {v.shape}; the nodes need {(yp.size, xp.size, 3)}")
        off = [-1e300 if o is None else float(o) for o in offset]
        self._check(L.mrm_gpu_set_field_table(self.h, layer, xp.size, yp.size, fptr(xp), fptr(yp), fptr(v),
                                              float(vel[0]), float(vel[1]), off[0], off[1], float(ref[0]),
                                              float(ref[1]), float(t_origin)))

    def set_llb(self, layer, spin, tc, lambda_ms):
        """LLB integrator on `layer` (include/mrm_gpu.h mrm_gpu_set_llb): spin,
        per-grain Curie temperature (K) and lambdaMs (Oe); tc None turns it off."""
        L = _lib.load()
        if tc is None:
            self._check(L.mrm_gpu_set_llb(self.h, layer, 0.0, None, None))
            return
        t, lm = f64(tc), f64(lambda_ms)
        self._check(L.mrm_gpu_set_llb(self.h, layer, float(spin), fptr(t), fptr(lm)))

    def set_mt(self, layer, spin, lambda_ms, meq_bs=False, garanin_tau=False):
        """MT integrator on `layer` (include/mrm_gpu.h mrm_gpu_set_mt); lambda_ms
        None turns it off."""
        L = _lib.load()
        if lambda_ms is None:
            self._check(L.mrm_gpu_set_mt(self.h, layer, 0.0, None, 0, 0))
            return
        lm = f64(lambda_ms)
        self._check(L.mrm_gpu_set_mt(self.h, layer, float(spin), fptr(lm), int(bool(meq_bs)),
                                     int(bool(garanin_tau))))

    def set_temp_profile(self, layer, background, dtemp, sigma=(0.0, 0.0), expn=1, vel=(0.0, 0.0),
                         offset=(None, None), ref=(0.0, 0.0), t_origin=0.0, time=None):
        """Moving super-Gaussian temperature profile (include/mrm_gpu.h
        mrm_gpu_set_temp_profile); `time`: dict of mrm_gpu_set_temp_function's
        arguments (func, t_start, t_end, s_start, s_end, amp, gamma, phase, param,
        duty, moddepth, dc, scale); None: constant 1."""
        L = _lib.load()
        off = [-1e300 if o is None else float(o) for o in offset]
        self._check(L.mrm_gpu_set_temp_profile(self.h, layer, float(background), float(dtemp), float(sigma[0]),
                                               float(sigma[1]), int(expn), float(vel[0]), float(vel[1]), off[0],
                                               off[1], float(ref[0]), float(ref[1]), float(t_origin)))
        if time:
            tf = time
            self._check(L.mrm_gpu_set_temp_function(
                self.h, layer, int(tf.get("func", 0)), float(tf.get("t_start", -1e22)), float(tf.get("t_end", 1e22)),
                float(tf.get("s_start", 1.0)), float(tf.get("s_end", 1.0)), float(tf.get("amp", 0.0)),
                float(tf.get("gamma", 0.0)), float(tf.get("phase", 0.0)), float(tf.get("param", 0.0)),
                float(tf.get("duty", 0.0)), float(tf.get("moddepth", 0.0)), float(tf.get("dc", 0.0)),
                float(tf.get("scale", 1.0))))

    def set_temp_scaling(self, layer, tc, msexp=-1.0, hkexp=-1.0, use_mag=False, tables=None):
        """Temperature scaling of Ms, alpha and Hk on `layer` (include/mrm_gpu.h
        mrm_gpu_set_temp_scaling): per-grain Curie temperature `tc` (K), power-law
        exponents (negative: none), Ms from |m| (`use_mag`), and `tables`
        {which: (temperatures, scales)} with which 1 Ms, 2 alpha, 3 Hk, 4 Hx (as
        read; reduced by the library).  tc None turns it off."""
        L = _lib.load()
        if tc is None:
            self._check(L.mrm_gpu_set_temp_scaling(self.h, layer, None, 0.0, 0.0, 0))
            return
        t = f64(tc)
        for which, (temps, scales) in (tables or {}).items():
            tt, vv = f64(temps), f64(scales)
            self._check(L.mrm_gpu_set_temp_scaling_table(self.h, layer, int(which), len(tt), fptr(tt), fptr(vv)))
        self._check(L.mrm_gpu_set_temp_scaling(self.h, layer, fptr(t), float(msexp), float(hkexp),
                                               1 if use_mag else 0))

    def get_temp_scaling_table(self, layer, which):
        """The reduced scaling table `which`: (T/Tc, scale)."""
        L = _lib.load()
        n = C.c_int(0)
        L.mrm_gpu_get_temp_scaling_table(self.h, layer, int(which), C.byref(n), None, None)
        tt, vv = np.zeros(max(n.value, 1)), np.zeros(max(n.value, 1))
        self._check(L.mrm_gpu_get_temp_scaling_table(self.h, layer, int(which), C.byref(n), fptr(tt), fptr(vv)))
        return tt[:n.value].copy(), vv[:n.value].copy()

    def set_zhang(self, layer, spin, lambda_ms, meq_bs=False, garanin_tau=False):
        """Zhang integrator on `layer` (include/mrm_gpu.h mrm_gpu_set_zhang)."""
        L = _lib.load()
        if lambda_ms is None:
            self._check(L.mrm_gpu_set_zhang(self.h, layer, 0.0, None, 0, 0))
            return
        lm = f64(lambda_ms)
        self._check(L.mrm_gpu_set_zhang(self.h, layer, float(spin), fptr(lm), int(bool(meq_bs)),
                                        int(bool(garanin_tau))))

    def set_mag(self, layer: int, mag):
        """The LLB magnitude |m| per grain."""
        a = f64(mag)
        self._check(_lib.load().mrm_gpu_set_mag(self.h, layer, fptr(a)))

    def get_mag(self, layer: int) -> np.ndarray:
        out = np.zeros(self.medium.layers[layer].N)
        self._check(_lib.load().mrm_gpu_get_mag(self.h, layer, fptr(out)))
        return out

    def set_window(self, nx_win: int, ny_win: int, v=(0.0, 0.0), offset=(0.0, 0.0)):
        """Moving demag window (include/mrm_gpu.h mrm_gpu_set_window); the tensor
        must be built or uploaded again afterwards."""
        self._check(_lib.load().mrm_gpu_set_window(self.h, int(nx_win), int(ny_win), float(v[0]), float(v[1]),
                                                   float(offset[0]), float(offset[1])))

    def get_window(self):
        """(nx_win, ny_win, i0, j0): the window's size and current origin."""
        out = (C.c_int * 4)()
        self._check(_lib.load().mrm_gpu_get_window(self.h, out))
        return tuple(out)

    def set_cubic_axes(self, layer, cubic_axis):
        """Cubic anisotropy on `layer`: cubic_axis (N,3,3), row i = crystal axis i in
        lab coordinates (None: back to uniaxial)."""
        if cubic_axis is None:
            self._check(_lib.load().mrm_gpu_set_cubic_axes(self.h, layer, None))
            return
        a = f64(cubic_axis)
        if a.shape != (self.medium.layers[layer].N, 3, 3):
            raise ValueError("cubic_axis must be (N, 3, 3)")
        self._check(_lib.load().mrm_gpu_set_cubic_axes(self.h, layer, fptr(a)))

    def set_thermal(self, layer, on, temperature, seed):
        self._check(_lib.load().mrm_gpu_set_thermal(self.h, layer, 1 if on else 0,
                                                    float(temperature), int(seed)))

    def set_state(self, layer: int, m: np.ndarray):
        mm = f64(m)
        self._check(_lib.load().mrm_gpu_set_state(self.h, layer, fptr(mm)))

    def get_state(self, layer: int, out: Optional[np.ndarray] = None) -> np.ndarray:
        """m of `layer` as (N, 3) float64; `out`: a C-contiguous (N, 3) float64
        array to fill instead of a new one (pinned host memory copies fastest)."""
        n = self.medium.layers[layer].N
        if out is None:
            out = np.zeros((n, 3))
        elif out.shape != (n, 3) or out.dtype != np.float64 or not out.flags["C_CONTIGUOUS"]:
            raise ValueError(f"out must be a C-contiguous ({n}, 3) float64 array")
        self._check(_lib.load().mrm_gpu_get_state(self.h, layer, fptr(out)))
        return out

    def get_field(self, layer: int) -> np.ndarray:
        out = np.zeros((self.medium.layers[layer].N, 3))
        self._check(_lib.load().mrm_gpu_get_field(self.h, layer, fptr(out)))
        return out

    def set_time(self, t: float, step: int = 0):
        self._check(_lib.load().mrm_gpu_set_time(self.h, t, step))

    def get_time(self):
        t, s = C.c_double(), C.c_int64()
        self._check(_lib.load().mrm_gpu_get_time(self.h, C.byref(t), C.byref(s)))
        return t.value, s.value

    def set_shape(self, row_shape: int, col_shape: int, cols_per_task: int = 0):
        """Forces compiled kernel shapes (negative: automatic)."""
        self._check(_lib.load().mrm_gpu_set_shape(self.h, int(row_shape), int(col_shape), int(cols_per_task)))

    def set_autotune(self, on: bool):
        self._check(_lib.load().mrm_gpu_set_autotune(self.h, 1 if on else 0))

    def get_shape(self):
        out = (C.c_int * 3)()
        self._check(_lib.load().mrm_gpu_get_shape(self.h, out))
        return int(out[0]), int(out[1]), int(out[2])

    def eval_field(self, t: float, layer: int = 0) -> np.ndarray:
        """get_field(t) on the current state; returns H_demag of `layer`."""
        out = np.zeros((self.medium.layers[layer].N, 3))
        self._check(_lib.load().mrm_gpu_eval_field(self.h, t, layer, fptr(out)))
        return out


class GpuSim(_RunMixin):
    """Plain single-run handle (the drop-in for llg()'s loop body)."""

    def __init__(self, medium, precision: int = _lib.FP32, device: int = 0, demag: bool = True,
                 thermal_seed: int = 1, tensor: Optional[np.ndarray] = None):
        L = _lib.load()
        self.medium = medium
        self.precision = precision
        g = geom_of(medium, precision)
        h = C.c_void_p()
        rc = L.mrm_gpu_create(C.byref(g), device, C.byref(h))
        if rc != 0:
            raise MrmError(rc, (L.mrm_gpu_last_error(None) or b"").decode())
        self.h = h
        win = getattr(medium, "window", None)
        if win:
            self.set_window(win["nx"], win["ny"], win.get("v", (0.0, 0.0)), win.get("offset", (0.0, 0.0)))
        self.upload_medium(medium, thermal_seed)
        if demag:
            if tensor is None:
                self.build_tensor()
            else:
                self.upload_tensor(tensor)
        else:
            self.set_demag(False)

    def close(self):
        if getattr(self, "h", None):
            _lib.load().mrm_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def enqueue(self, nsteps: int, dt: float, llg_type: int = -3):
        self._check(_lib.load().mrm_gpu_enqueue_steps(self.h, int(nsteps), float(dt), int(llg_type)))

    def stats(self):
        st = np.zeros(1, _lib.STATS_DTYPE)
        self._check(_lib.load().mrm_gpu_read_stats(self.h, st.ctypes.data))
        return st[0]

    def stream(self) -> int:
        s = C.c_void_p()
        self._check(_lib.load().mrm_gpu_stream(self.h, C.byref(s)))
        return s.value or 0

    def profile(self, reps: int, dt: float) -> np.ndarray:
        out = np.zeros(4)
        self._check(_lib.load().mrm_gpu_profile(self.h, int(reps), float(dt), fptr(out)))
        return out

    def off_field(self, zoff: float, dzobs: float, head_mu: float = 1.0, fly_height: float = 8e-7,
                  sul_mu: float = 1.0, space_to_sul: float = 40e-7, num_images: int = 2) -> np.ndarray:
        """Stray field (3, ny, nx) in Oe averaged over a slab dzobs thick whose bottom is
        zoff above the media (include/mrm_gpu.h mrm_gpu_off_field); lengths in cm."""
        out = np.zeros((3, self.medium.ny, self.medium.nx))
        self._check(_lib.load().mrm_gpu_off_field(self.h, float(zoff), float(dzobs), float(head_mu),
                                                  float(fly_height), float(sul_mu), float(space_to_sul),
                                                  int(num_images), fptr(out)))
        return out

    def step_adaptive(self, nsteps: int, dt: float, max_dmdt: float = 1.0, llg_type: int = -3,
                      dt_frac: float = 0.2, dt_max: float = 1e-8, max_dm=None):
        """nsteps steps with the reference's adaptive dt (include/mrm_gpu.h
        mrm_gpu_step_adaptive); returns (stats, dt, max_dmdt) for the next call."""
        st = np.zeros(1, _lib.STATS_DTYPE)
        md = f64(max_dm if max_dm is not None else [3.1415925] * self.medium.n_lay)
        a, b = C.c_double(dt), C.c_double(max_dmdt)
        self._check(_lib.load().mrm_gpu_step_adaptive(self.h, int(nsteps), int(llg_type), float(dt_frac),
                                                      float(dt_max), fptr(md), C.byref(a), C.byref(b),
                                                      st.ctypes.data))
        return st[0], a.value, b.value

    def step(self, nsteps: int, dt: float, llg_type: int = -3, stats: bool = True):
        st = np.zeros(1, _lib.STATS_DTYPE) if stats else None
        self._check(_lib.load().mrm_gpu_step(self.h, int(nsteps), float(dt), int(llg_type),
                                             st.ctypes.data if stats else None))
        return st[0] if stats else None
