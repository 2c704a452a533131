"""ctypes wrapper of the CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this
module.  It loads oracle/liboracle.so (built by oracle/Makefile) and mirrors
the GPU host API closely enough that a parity test can drive both with the
same media and schedule.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

MAX_LAYERS = 8
STATS_DTYPE = np.dtype([
    ("t", "f8"), ("step", "i8"),
    ("mave", "f8", 3), ("mvar", "f8", 3), ("have", "f8", 3),
    ("errmx", "f8"), ("errmx1", "f8"), ("mmag", "f8"), ("energy", "f8"),
    ("mave_l", "f8", (MAX_LAYERS, 3)), ("mvar_l", "f8", (MAX_LAYERS, 3)),
    ("have_l", "f8", (MAX_LAYERS, 3)), ("mms_l", "f8", (MAX_LAYERS, 3)),
    ("vol_l", "f8", MAX_LAYERS), ("msvol_l", "f8", MAX_LAYERS), ("nup_l", "i8", MAX_LAYERS),
    ("errmx1_l", "f8", MAX_LAYERS),
])


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "liboracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        d, i, u64, vp = C.c_double, C.c_int, C.c_uint64, C.c_void_p
        P = C.POINTER
        L.orc_create.restype = vp
        L.orc_create.argtypes = [i, i, i, i, i, d, d, P(d), P(d), d, d, d, d, i]
        L.orc_destroy.argtypes = [vp]
        L.orc_build_tensor.argtypes = [vp, P(d)]
        L.orc_set_tensor.argtypes = [vp, P(d)]
        L.orc_upload_layer.argtypes = [vp, i, i, P(d), P(d), P(d), P(d), P(d), P(d), P(d), d, d, d,
                                       P(i), P(i), P(i), P(i), P(d)]
        L.orc_upload_interlayer.argtypes = [vp, i, i, P(i), P(i), P(d)]
        L.orc_set_uniform_field.argtypes = [vp, i, P(d), d, d, d, d, d]
        L.orc_set_thermal.argtypes = [vp, i, i, d, i, C.c_longlong]
        L.orc_set_field_function.argtypes = [vp, i, P(d), i, d, d, d, d, d, d, d, d]
        L.orc_set_head_field.argtypes = [vp, i, d, d, d, d, d, d, d, u64, i]
        L.orc_set_cubic_axes.argtypes = [vp, i, P(d)]
        L.orc_set_field_table.argtypes = [vp, i, i, i, P(d), P(d), P(d), d, d, d, d, d, d, d]
        L.orc_set_window.argtypes = [vp, i, i, d, d, d, d]
        L.orc_set_llb.argtypes = [vp, i, d, P(d), P(d)]
        L.orc_set_mt.argtypes = [vp, i, d, P(d), i, i, i]
        L.orc_set_temp_profile.argtypes = [vp, i, d, d, d, d, i, d, d, d, d, d, d, d]
        L.orc_set_temp_function.argtypes = [vp, i, i] + [d] * 12
        L.orc_set_temp_scaling.argtypes = [vp, i, P(d), d, d, i]
        L.orc_set_temp_scaling_table.argtypes = [vp, i, i, i, P(d), P(d)]
        L.orc_get_temp_scaling_table.argtypes = [vp, i, i, P(i), P(d), P(d)]
        L.orc_get_scales.argtypes = [vp, i, P(d), P(d), P(d)]
        L.orc_get_temp.argtypes = [vp, i, P(d)]
        L.orc_set_mag.argtypes = [vp, i, P(d)]
        L.orc_get_mag.argtypes = [vp, i, P(d)]
        L.orc_get_window.argtypes = [vp, P(i)]
        L.orc_set_state.argtypes = [vp, i, P(d)]
        L.orc_get_state.argtypes = [vp, i, P(d)]
        L.orc_get_field.argtypes = [vp, i, P(d)]
        L.orc_get_demag.argtypes = [vp, i, P(d)]
        L.orc_get_applied.argtypes = [vp, i, P(d)]
        L.orc_set_time.argtypes = [vp, d, C.c_longlong]
        L.orc_eval_field.argtypes = [vp, d]
        L.orc_step.argtypes = [vp, i, d, i, vp, vp]
        L.orc_step_adaptive.argtypes = [vp, i, i, d, d, P(d), P(d), P(d), vp]
        L.orc_off_field.argtypes = [vp, d, d, d, d, d, d, i, P(d)]
        L.orc_mt_u32.argtypes = [i, i, P(C.c_uint32)]
        L.orc_mt_state.argtypes = [i, P(C.c_uint32)]
        L.orc_mt_normals.argtypes = [i, i, P(d)]
        L.orc_philox4x64.argtypes = [P(u64), P(u64), P(u64)]
        L.orc_philox_normal3.argtypes = [u64, u64, u64, u64, P(d)]
        L.orc_volume_averaged_n.argtypes = [d] * 9 + [P(d)]
        L.orc_volume_averaged_n_q.argtypes = [i, P(i), P(i)] + [d] * 9 + [P(d)]
        L.orc_calculate_tensor.argtypes = [i, i, i, d, d, P(d), P(d), i, i, d, d, d, d, P(d)]
        L.orc_fft_r2c.argtypes = [i, i, P(d), P(d)]
        L.orc_fft_c2r.argtypes = [i, i, P(d), P(d)]
        L.orc_demag_direct.argtypes = [i, i, i, P(d), P(d), i, P(i), i, P(d)]
        L.orc_set_threads.argtypes = [i]
        L.orc_set_fft_precision.argtypes = [vp, i]
        L.orc_get_threads.restype = i
        L.orc_stats_size.restype = i
        assert L.orc_stats_size() == STATS_DTYPE.itemsize, "Stats layout mismatch"
        _LIB = L
    return _LIB


def _p(a, ct=C.c_double):
    return a.ctypes.data_as(C.POINTER(ct))


def _temp_function_args(tf):
    """(func, t_start, t_end, s_start, s_end, amp, gamma, phase, param, duty, moddepth, dc, scale)"""
    return (int(tf.get("func", 0)), float(tf.get("t_start", -1e22)), float(tf.get("t_end", 1e22)),
            float(tf.get("s_start", 1.0)), float(tf.get("s_end", 1.0)), float(tf.get("amp", 0.0)),
            float(tf.get("gamma", 0.0)), float(tf.get("phase", 0.0)), float(tf.get("param", 0.0)),
            float(tf.get("duty", 0.0)), float(tf.get("moddepth", 0.0)), float(tf.get("dc", 0.0)),
            float(tf.get("scale", 1.0)))


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


# ---------------- probes ----------------
def mt_u32(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n, np.uint32)
    lib().orc_mt_u32(seed, n, _p(out, C.c_uint32))
    return out


def mt_state(seed: int) -> np.ndarray:
    out = np.zeros(624, np.uint32)
    lib().orc_mt_state(seed, _p(out, C.c_uint32))
    return out


def mt_normals(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n)
    lib().orc_mt_normals(seed, n, _p(out))
    return out


def philox4x64(ctr, key) -> np.ndarray:
    c = np.ascontiguousarray(ctr, np.uint64)
    k = np.ascontiguousarray(key, np.uint64)
    out = np.zeros(4, np.uint64)
    lib().orc_philox4x64(_p(c, C.c_uint64), _p(k, C.c_uint64), _p(out, C.c_uint64))
    return out


def philox_normal3(seed, stream, step, grain) -> np.ndarray:
    out = np.zeros(3)
    lib().orc_philox_normal3(seed, stream, step, grain, _p(out))
    return out


def volume_averaged_n(rx, ry, rz, xs, ys, zs, xo, yo, zo) -> np.ndarray:
    n = np.zeros(9)
    lib().orc_volume_averaged_n(rx, ry, rz, xs, ys, zs, xo, yo, zo, _p(n))
    return n.reshape(3, 3)


def tensor_slot_q(px, py, dx, dy, dz_s, dz_o, rz, fi, fj) -> np.ndarray:
    """One slot (fi, fj) of an open-boundary FFT grid's tensor (no images) in
    quadruple precision: the offsets that wrap onto the slot (two on the
    n/2 lines, src/tensor_element.f90:233-257), normalised by
    1/(dx dy dz_o px py) (src/tensor.f90:183); returns t(a, b) as [a*3+b]."""
    def offs(f, n):
        if n % 2 == 0 and f == n // 2:
            return [-n // 2, n // 2]
        return [0 if f == 0 else (-f if f <= n // 2 else n - f)]
    pts = [(i, j) for j in offs(fj, py) for i in offs(fi, px)]
    ix = np.array([p[0] for p in pts], np.int32)
    iy = np.array([p[1] for p in pts], np.int32)
    out = np.zeros(9)
    lib().orc_volume_averaged_n_q(len(pts), _p(ix, C.c_int), _p(iy, C.c_int), dx, dy, rz, dx, dy, dz_s, dx, dz_o,
                                  1.0 / (dx * dy * dz_o * px * py), _p(out))
    return out


def calculate_tensor(nx, ny, dx, dy, dz, il_space, images, space_to_sul=0.0, sul_mu=1.0,
                     head_mu=1.0, fly_height=0.0) -> np.ndarray:
    """Real-space tensor, reference layout [ks][ko][9][ny][nx]."""
    nl = len(dz)
    out = np.zeros((nl, nl, 9, ny, nx))
    dzv, ilv = f64(dz), f64(il_space)
    lib().orc_calculate_tensor(nx, ny, nl, dx, dy, _p(dzv), _p(ilv), images, images, space_to_sul,
                               sul_mu, head_mu, fly_height, _p(out))
    return out


def fft_r2c(r: np.ndarray) -> np.ndarray:
    ny, nx = r.shape
    r = f64(r)
    c = np.zeros((ny, nx // 2 + 1), np.complex128)
    lib().orc_fft_r2c(nx, ny, _p(r), c.ctypes.data_as(C.POINTER(C.c_double)))
    return c


def fft_c2r(c: np.ndarray, nx: int) -> np.ndarray:
    ny = c.shape[0]
    c = np.ascontiguousarray(c, np.complex128)
    r = np.zeros((ny, nx))
    lib().orc_fft_c2r(nx, ny, c.ctypes.data_as(C.POINTER(C.c_double)), _p(r))
    return r


def demag_direct(n2d: np.ndarray, mgrid: np.ndarray, obs_ij: np.ndarray, ko: int) -> np.ndarray:
    """Direct FP64 convolution at observation cells; n2d [nl][nl][9][py][px], mgrid [nl][3][py][px]."""
    nl, _, _, py, px = n2d.shape
    n2d = f64(n2d)
    mg = f64(mgrid)
    obs = i32(obs_ij)
    out = np.zeros((obs.shape[0], 3))
    lib().orc_demag_direct(px, py, nl, _p(n2d), _p(mg), obs.shape[0], _p(obs, C.c_int), ko, _p(out))
    return out


def set_threads(n: int):
    lib().orc_set_threads(int(n))


def get_threads() -> int:
    return int(lib().orc_get_threads())


class OracleSim:
    """CPU restatement driven like the GPU handle (mrm_b200.GpuSim)."""

    def __init__(self, medium, demag: bool = True, rng_mode: int = 1, seed: int = 1,
                 tensor: np.ndarray | None = None, fft_bits: int = 64):
        L = lib()
        self.medium = medium
        dz = f64(medium.dz)
        il = f64(medium.il_space)
        self.h = L.orc_create(medium.nx, medium.ny, medium.n_lay, medium.boundary, medium.images,
                              medium.dx, medium.dy, _p(dz), _p(il), medium.space_to_sul,
                              medium.sul_mu, medium.head_mu, medium.fly_height, 1 if demag else 0)
        self._keep = []
        assert L.orc_set_fft_precision(self.h, int(fft_bits)) == 0
        for l, lay in enumerate(medium.layers):
            arrs = [f64(lay.ms), f64(lay.vol), f64(lay.axis), f64(lay.hk), f64(lay.hk_scale),
                    f64(lay.ms_scale), f64(lay.alpha_scale)]
            g2ci, g2c = i32(lay.g2c_index), i32(lay.g2c)
            if lay.hx_index is not None:
                hxi, hxg, hx = i32(lay.hx_index), i32(lay.hx_grain), f64(lay.hx)
                hxa = (_p(hxi, C.c_int), _p(hxg, C.c_int), _p(hx))
            else:
                hxa = (None, None, None)
            rc = L.orc_upload_layer(self.h, l, lay.N, *[_p(a) for a in arrs], lay.alpha, lay.gamma,
                                    lay.floor_ms, _p(g2ci, C.c_int), _p(g2c, C.c_int), *hxa)
            assert rc == 0
            d = f64(lay.hdir)
            if getattr(lay, "func", 0):
                L.orc_set_field_function(self.h, l, _p(d), lay.func, lay.amp, lay.fgamma, lay.phase,
                                         lay.param, lay.duty, lay.moddepth, lay.dc, lay.scale)
            else:
                L.orc_set_uniform_field(self.h, l, _p(d), lay.t_start, lay.t_end, lay.s_start,
                                        lay.s_end, lay.scale)
            hd = getattr(lay, "head", None)
            if hd:
                rc = L.orc_set_head_field(self.h, l, hd["gap"], hd["z"], hd["hg"], hd["velocity"], hd["x0"],
                                          hd["t0"], hd["bit_time"], int(hd["pattern"]), int(hd["nbits"]))
                assert rc == 0
            tb = getattr(lay, "field_table", None)
            if tb:
                self.set_field_table(l, **tb)
            lb = getattr(lay, "llb", None)
            if lb:
                self.set_llb(l, **lb)
            mt = getattr(lay, "mt", None)
            if mt:
                self.set_mt(l, **mt)
            zh = getattr(lay, "zhang", None)
            if zh:
                self.set_mt(l, **zh, mode=2)
            tp = getattr(lay, "temp_profile", None)
            if tp:
                self.set_temp_profile(l, **tp)
            ts = getattr(lay, "temp_scaling", None)
            if ts:
                self.set_temp_scaling(l, **ts)
            L.orc_set_thermal(self.h, l, 1 if lay.thermal else 0, lay.temperature, rng_mode, seed)
            cub = getattr(lay, "cubic_axis", None)
            if cub is not None:
                ca = f64(cub)
                assert ca.shape == (lay.N, 3, 3)
                assert L.orc_set_cubic_axes(self.h, l, _p(ca)) == 0
        for l, lay in enumerate(medium.layers):
            for side, cpl in ((0, lay.uhx), (1, lay.lhx)):
                if cpl is not None:
                    idx, gr, cf = i32(cpl[0]), i32(cpl[1]), f64(cpl[2])
                    L.orc_upload_interlayer(self.h, l, side, _p(idx, C.c_int), _p(gr, C.c_int), _p(cf))
        fx, fy = medium.nx, medium.ny
        win = getattr(medium, "window", None)
        if win:
            assert L.orc_set_window(self.h, win["nx"], win["ny"], *win.get("v", (0.0, 0.0)),
                                    *win.get("offset", (0.0, 0.0))) == 0
            fx, fy = win["nx"], win["ny"]
        px = fx * (2 if medium.boundary == 1 else 1)
        py = fy * (2 if medium.boundary == 1 else 1)
        self.px, self.py = px, py
        if demag:
            if tensor is None:
                self.n2d = np.zeros((medium.n_lay, medium.n_lay, 9, py, px))
                L.orc_build_tensor(self.h, _p(self.n2d))
            else:
                self.n2d = f64(tensor)
                L.orc_set_tensor(self.h, _p(self.n2d))
        if medium.m0 is not None:
            for l, m in enumerate(medium.m0):
                self.set_state(l, m)

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, layer: int, m: np.ndarray):
        mm = f64(m)
        lib().orc_set_state(self.h, layer, _p(mm))

    def get_state(self, layer: int) -> np.ndarray:
        n = self.medium.layers[layer].N
        out = np.zeros((n, 3))
        lib().orc_get_state(self.h, layer, _p(out))
        return out

    def get_field(self, layer: int) -> np.ndarray:
        n = self.medium.layers[layer].N
        out = np.zeros((n, 3))
        lib().orc_get_field(self.h, layer, _p(out))
        return out

    def get_demag(self, layer: int) -> np.ndarray:
        n = self.medium.layers[layer].N
        out = np.zeros((n, 3))
        lib().orc_get_demag(self.h, layer, _p(out))
        return out

    def set_llb(self, layer, spin, tc, lambda_ms):
        """LLB integrator on `layer` (GpuSim.set_llb's arguments; tc None: off)."""
        if tc is None:
            assert lib().orc_set_llb(self.h, layer, 0.0, None, None) == 0
            return
        t, lm = f64(tc), f64(lambda_ms)
        self._keep += [t, lm]
        assert lib().orc_set_llb(self.h, layer, float(spin), _p(t), _p(lm)) == 0

    def set_mt(self, layer, spin, lambda_ms, meq_bs=False, garanin_tau=False, mode=1):
        """MT (mode 1) or Zhang (mode 2) integrator on `layer` (GpuSim.set_mt's arguments)."""
        if lambda_ms is None:
            assert lib().orc_set_mt(self.h, layer, 0.0, None, 0, 0, mode) == 0
            return
        lm = f64(lambda_ms)
        assert lib().orc_set_mt(self.h, layer, float(spin), _p(lm), int(bool(meq_bs)), int(bool(garanin_tau)),
                                mode) == 0

    def set_temp_profile(self, layer, background, dtemp, sigma=(0.0, 0.0), expn=1, vel=(0.0, 0.0),
                         offset=(None, None), ref=(0.0, 0.0), t_origin=0.0, time=None):
        """Temperature profile (GpuSim.set_temp_profile's arguments)."""
        off = [-1e300 if o is None else float(o) for o in offset]
        assert lib().orc_set_temp_profile(self.h, layer, float(background), float(dtemp), float(sigma[0]),
                                          float(sigma[1]), int(expn), float(vel[0]), float(vel[1]), off[0], off[1],
                                          float(ref[0]), float(ref[1]), float(t_origin)) == 0
        if time:
            a = _temp_function_args(time)
            assert lib().orc_set_temp_function(self.h, layer, *a) == 0

    def set_temp_scaling(self, layer, tc, msexp=-1.0, hkexp=-1.0, use_mag=False, tables=None):
        """Temperature scaling (GpuSim.set_temp_scaling's arguments; tc None: off)."""
        if tc is None:
            assert lib().orc_set_temp_scaling(self.h, layer, None, 0.0, 0.0, 0) == 0
            return
        t = f64(tc)
        self._keep.append(t)
        assert lib().orc_set_temp_scaling(self.h, layer, _p(t), float(msexp), float(hkexp), int(bool(use_mag))) == 0
        for which, (temps, scales) in (tables or {}).items():
            tt, vv = f64(temps), f64(scales)
            assert lib().orc_set_temp_scaling_table(self.h, layer, int(which), len(tt), _p(tt), _p(vv)) == 0

    def get_temp_scaling_table(self, layer, which):
        """The reduced scaling table `which` (1 Ms, 2 alpha, 3 Hk, 4 Hx): (T/Tc, scale)."""
        n = C.c_int(4096)
        tt, vv = np.zeros(4096), np.zeros(4096)
        assert lib().orc_get_temp_scaling_table(self.h, layer, int(which), C.byref(n), _p(tt), _p(vv)) == 0
        return tt[:n.value].copy(), vv[:n.value].copy()

    def get_scales(self, layer):
        """ms_scale, alpha_scale, hk_scale per grain after the last field evaluation."""
        N = self.medium.layers[layer].N
        a, b, c = np.zeros(N), np.zeros(N), np.zeros(N)
        assert lib().orc_get_scales(self.h, layer, _p(a), _p(b), _p(c)) == 0
        return a, b, c

    def get_temp(self, layer):
        """Grain temperatures of the last field evaluation."""
        out = np.zeros(self.medium.layers[layer].N)
        assert lib().orc_get_temp(self.h, layer, _p(out)) == 0
        return out

    def set_mag(self, layer, mag):
        a = f64(mag)
        assert lib().orc_set_mag(self.h, layer, _p(a)) == 0

    def get_mag(self, layer):
        out = np.zeros(self.medium.layers[layer].N)
        lib().orc_get_mag(self.h, layer, _p(out))
        return out

    def get_window(self):
        """(nx_win, ny_win, i0, j0) of the moving demag window."""
        out = (C.c_int * 4)()
        lib().orc_get_window(self.h, out)
        return tuple(out)

    def get_applied(self, layer: int) -> np.ndarray:
        """Applied field per grain of the last field evaluation."""
        n = self.medium.layers[layer].N
        out = np.zeros((n, 3))
        lib().orc_get_applied(self.h, layer, _p(out))
        return out

    def set_time(self, t: float, step: int = 0):
        lib().orc_set_time(self.h, t, step)

    def eval_field(self, t: float):
        lib().orc_eval_field(self.h, t)

    def set_field_table(self, layer, xpos, ypos, vfld, vel=(0.0, 0.0), offset=(None, None), ref=(0.0, 0.0),
                        t_origin=0.0):
        """Tabulated field profile (GpuSim.set_field_table's arguments; vfld None removes it)."""
        if vfld is None:
            assert lib().orc_set_field_table(self.h, layer, 0, 0, None, None, None, 0, 0, 0, 0, 0, 0, 0) == 0
            return
        xp, yp, v = f64(xpos), f64(ypos), f64(vfld)
        assert v.shape == (yp.size, xp.size, 3)
        off = [-1e300 if o is None else float(o) for o in offset]
        assert lib().orc_set_field_table(self.h, layer, xp.size, yp.size, _p(xp), _p(yp), _p(v), float(vel[0]),
                                         float(vel[1]), off[0], off[1], float(ref[0]), float(ref[1]),
                                         float(t_origin)) == 0

    def off_field(self, zoff: float, dzobs: float, head_mu: float = 1.0, fly_height: float = 8e-7,
                  sul_mu: float = 1.0, space_to_sul: float = 40e-7, num_images: int = 2) -> np.ndarray:
        """Stray field (3, ny, nx) at the observation slab (off_field.f90)."""
        out = np.zeros((3, self.medium.ny, self.medium.nx))
        assert lib().orc_off_field(self.h, zoff, dzobs, head_mu, fly_height, sul_mu, space_to_sul, num_images,
                                   _p(out)) == 0
        return out

    def step_adaptive(self, nsteps: int, dt: float, max_dmdt: float = 1.0, llg_type: int = -3,
                      dt_frac: float = 0.2, dt_max: float = 1e-8, max_dm=None):
        """nsteps adaptive steps; returns (stats, dt, max_dmdt) to pass to the next call."""
        st = np.zeros(1, STATS_DTYPE)
        md = f64(max_dm if max_dm is not None else [3.1415925] * self.medium.n_lay)
        a, b = C.c_double(dt), C.c_double(max_dmdt)
        rc = lib().orc_step_adaptive(self.h, nsteps, llg_type, dt_frac, dt_max, _p(md), C.byref(a), C.byref(b),
                                     st.ctypes.data)
        if rc != 0:
            raise RuntimeError(f"orc_step_adaptive failed rc={rc}")
        return st[0], a.value, b.value

    def step(self, nsteps: int, dt: float, llg_type: int = -3, traj: bool = False):
        st = np.zeros(1, STATS_DTYPE)
        tr = np.zeros((nsteps, self.medium.n_lay, 3)) if traj else None
        rc = lib().orc_step(self.h, nsteps, dt, llg_type, st.ctypes.data,
                            tr.ctypes.data if traj else None)
        if rc != 0:
            raise RuntimeError(f"orc_step failed rc={rc}")
        return (st[0], tr) if traj else st[0]
